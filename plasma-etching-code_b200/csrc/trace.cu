// Flux kernels: Monte-Carlo ions and Russian-roulette neutrals on the device BVH, plus the
// nearest-face queries (velocity extension and coverage warm start).
//
// Work distribution: persistent lanes with per-lane refill.  A lane whose ray has ended takes the
// next ray id from a global counter (one atomic per warp per refill), so warps stay full through
// the long bounce tails of the Russian-roulette and reflected-ion paths instead of idling behind
// their longest ray.  Sources are generated in-kernel from the ray's Philox stream; there are no
// origin/direction arrays.
#include <cub/cub.cuh>
#include <map>
#include <mutex>
#include <utility>
#include "common.cuh"
#include "mesh.cuh"
#include "trace.cuh"

namespace petch {
namespace {

constexpr int kTB = 128;
#ifndef PETCH_TRACE_MIN_BLOCKS
#define PETCH_TRACE_MIN_BLOCKS 8
#endif
#ifndef PETCH_TRACE_MIN_BLOCKS_RR
#define PETCH_TRACE_MIN_BLOCKS_RR 8
#endif
#ifndef PETCH_TRACE_MIN_BLOCKS_RR_BATCH
#define PETCH_TRACE_MIN_BLOCKS_RR_BATCH 9
#endif
#ifndef PETCH_TRACE_MIN_BLOCKS_RR_TAN
#define PETCH_TRACE_MIN_BLOCKS_RR_TAN 8
#endif
// Resident blocks of the persistent tracers per SM (the binary-traversal launches use no shared
// memory, so registers alone set them): 8 x 4 warps (<= 64 registers per thread) for the ion
// shaders; 8 x 4 (<= 64 registers, no spills) for the single-instance Russian-roulette neutral
// shaders (trench workload, 100-step run: 1.1 % faster than 9 blocks at 56 registers, which
// spill ~90 B per thread, and than 10 blocks at 48; 12 blocks at 40 registers spill ~300 B and
// ran 4.8 % slower); 9 x 4 (<= 56 registers) for the batched neutral kinds (64 ragged holes: 12
// blocks 9 % slower, 10 blocks 1.3 % slower, 8 blocks 2 % slower); 8 x 4 (<= 64 registers) for
// the neutral tangent shaders, which carry three weight tangents per ray (the batched inverse
// design's device time 8 % below 10 blocks at 48 registers).
constexpr int kTraceMinBlocks = PETCH_TRACE_MIN_BLOCKS;
constexpr int kTraceMinBlocksRR = PETCH_TRACE_MIN_BLOCKS_RR;
constexpr int kTraceMinBlocksRRBatch = PETCH_TRACE_MIN_BLOCKS_RR_BATCH;
constexpr int kTraceMinBlocksRRTan = PETCH_TRACE_MIN_BLOCKS_RR_TAN;
constexpr long long kMaxRounds = 1LL << 24;   // per-warp bound on tracer rounds (error bit 4)
constexpr unsigned kFull = 0xffffffffu;

// Tracer configuration (process-wide host state, set by petch_tracer_config): BVH width,
// traversal steps per warp round, and how many lanes may still be traversing when a warp stops
// stepping to shade and refill (only while the ray pool has rays).  The defaults were the fastest
// of a sweep over the 8x4x40 trench's 100-step run at 2^22 rays with leaf grouping 2 (within
// ~2 % of 64 steps / keep 12; grouping off is 25 % slower).
int g_bvh_width = 2;
int g_steps = 32;
int g_keep = 16;
bool g_tally_agg = false;   // warp-aggregated deposits (petch_tally_aggregation)
int g_group = 2;            // leaf grouping of the binary traversal (petch_tracer_grouping)

// Deterministic tallies (petch_set_deterministic): caller-registered scratch for 64-bit
// fixed-point accumulators; NULL = float atomics.
void* g_det_scratch = nullptr;
long long g_det_bytes = 0;

constexpr float kTallyScale = 4294967296.0f;      // 2^32: one unit = 2^-32

}  // namespace

bool wide_bvh_enabled() { return g_bvh_width == 8; }

namespace {
// The tally mode word of a trace launch: kTallyDet with deterministic tallies, kTallyAgg with
// warp aggregation configured.
int tally_mode(bool det) { return (det ? 1 : 0) | (g_tally_agg ? 2 : 0); }
}  // namespace

namespace {

struct Domain {
    float lx, ly, lz, z_src;
    int periodic;
};

// _gen_source (threed.py:441-458): origin uniform on [0,Lx]x[0,Ly] at z_src; ion direction from
// a Gaussian tilt (sigma) in x and y, neutral direction cosine-distributed about -z.
__device__ __forceinline__ void source(Rng& g, bool ion, float sigma, const Domain& D, float3& o,
                                       float3& d) {
    float ox = g.uniform() * D.lx;
    float oy = g.uniform() * D.ly;
    o = make_float3(ox, oy, D.z_src);
    if (ion) {
        float ax = g.normal() * sigma, ay = g.normal() * sigma;
        d = make_float3(sinf(ax), sinf(ay), -cosf(ax) * cosf(ay));
    } else {
        float r1 = g.uniform(), r2 = g.uniform();
        float ct = sqrtf(r1), s = sqrtf(1.0f - r1), ph = 6.2831853f * r2;
        d = make_float3(s * cosf(ph), s * sinf(ph), -ct);
    }
    d = normalize3(d);
}

// Cosine-weighted re-emission about n with the reference's tangent frame (threed.py:584-595).
__device__ __forceinline__ float3 cosine_emit(Rng& g, float3 n) {
    float3 a = fabsf(n.x) > 0.9f ? make_float3(0.0f, 1.0f, 0.0f) : make_float3(1.0f, 0.0f, 0.0f);
    float3 t = normalize3(cross3(a, n));
    float3 b = cross3(n, t);
    float r1 = g.uniform(), r2 = g.uniform();
    float ct = sqrtf(r1), st = sqrtf(1.0f - r1), ph = 6.2831853f * r2;
    return (st * cosf(ph)) * t + (st * sinf(ph)) * b + ct * n;
}

// Warp-cooperative refill: lanes with ray == -1 take consecutive ids from *counter.  The counter
// is advanced in unsigned arithmetic: lanes that find the pool empty still advance it (each lane
// at most once, since a lane with ray == -2 never asks again), so it ends at most one id per
// resident lane above n, far below 2^32 for any n < 2^31, and no id wraps back below n.
__device__ __forceinline__ bool refill(int& ray, int n, int* counter) {
    const int lane = threadIdx.x & 31;
    bool need = (ray == -1);
    unsigned mask = __ballot_sync(kFull, need);
    if (mask) {
        int leader = __ffs(mask) - 1;
        unsigned base = 0;
        if (lane == leader) base = atomicAdd(reinterpret_cast<unsigned*>(counter), (unsigned)__popc(mask));
        base = __shfl_sync(kFull, base, leader);
        if (need) {
            const unsigned idx = base + (unsigned)__popc(mask & ((1u << lane) - 1u));
            ray = idx < (unsigned)n ? (int)idx : -2;
            return ray >= 0;
        }
    }
    return false;
}

// _apply_bc's wrap (threed.py:311-346): a ray that missed leaves through x or y before the open
// top -> re-enter at the opposite face with the same direction; false if it escapes the top.
__device__ __forceinline__ bool periodic_wrap(const Domain& D, float3& o, float3 d) {
    float tx = 1.0e30f, ty = 1.0e30f, tz = 1.0e30f;
    if (d.x > 1.0e-9f) tx = (D.lx - o.x) / d.x;
    if (d.x < -1.0e-9f) tx = (0.0f - o.x) / d.x;
    if (d.y > 1.0e-9f) ty = (D.ly - o.y) / d.y;
    if (d.y < -1.0e-9f) ty = (0.0f - o.y) / d.y;
    if (d.z > 1.0e-9f) tz = (D.lz - o.z) / d.z;
    if (tx < tz && tx < ty && tx > 1.0e-7f) {
        float hy = o.y + tx * d.y, hz = o.z + tx * d.z;
        o = make_float3(d.x < 0.0f ? D.lx - 1.0e-4f : 1.0e-4f, hy, hz);
        return true;
    }
    if (ty < tz && ty < 1.0e29f && ty > 1.0e-7f) {
        float hx = o.x + ty * d.x, hz = o.z + ty * d.z;
        o = make_float3(hx, d.y < 0.0f ? D.ly - 1.0e-4f : 1.0e-4f, hz);
        return true;
    }
    return false;
}

// Lateral position after the wraps of a ray that moves by `dist` along one axis from `p` in
// [0, L]: each exit through a face re-enters 1e-4 inside the opposite one (periodic_wrap), so
// after the first exit every full crossing covers L - 1e-4.  Adds the number of exits to `k`.
__device__ __forceinline__ float wrap_axis(float p, float dist, float L, float& k) {
    const float span = L - 1.0e-4f;
    if (dist > 0.0f) {
        const float e = p + dist - L;            // past the far face
        if (e <= 0.0f) return p + dist;
        const float n = floorf(e / span);
        k += 1.0f + n;
        return fminf(fmaxf(1.0e-4f + (e - n * span), 0.0f), L);
    }
    const float e = -(p + dist);                 // past the near face
    if (e <= 0.0f) return p + dist;
    const float n = floorf(e / span);
    k += 1.0f + n;
    return fminf(fmaxf(span - (e - n * span), 0.0f), L);
}

// A ray above every face (o.z > ztop, the top of the BVH root box) hits nothing until it comes
// down to ztop.  Wrapped one miss at a time (_apply_bc), such a ray costs a query per lateral
// crossing -- two thirds of the neutral queries in a deep trench.  This takes it there in one
// step, through the same wraps (counted into `wraps`; the axes wrap independently, as each
// periodic_wrap moves one coordinate), leaving o on the z = ztop plane.  Returns false when the
// ray never comes down (d.z >= 0) or needs more wraps than the 256 a bounce may take: the
// step-by-step wraps end such a ray too, with nothing deposited.
__device__ __forceinline__ bool descend_wrapped(const Domain& D, float ztop, float3& o, float3 d,
                                                int& wraps) {
    if (!(o.z > ztop)) return true;
    if (!(d.z < 0.0f)) return false;
    const float t = (o.z - ztop) / -d.z;
    float k = 0.0f;
    float x = o.x, y = o.y;
    if (fabsf(d.x) > 1.0e-9f) x = wrap_axis(o.x, t * d.x, D.lx, k);
    else x = o.x + t * d.x;
    if (fabsf(d.y) > 1.0e-9f) y = wrap_axis(o.y, t * d.y, D.ly, k);
    else y = o.y + t * d.y;
    if (!(k <= (float)(256 - wraps))) return false;   // also catches an infinite t
    wraps += (int)k;
    o = make_float3(x, y, ztop);
    return true;
}

// Top of the mesh's BVH root box (+inf for a mesh without leaves).
__device__ __forceinline__ float root_top(const MeshView& m, int L) {
    return L > 0 ? __int_as_float(__ldg(m.hdr + HDR_ROOTBOX + 5)) : 3.0e38f;
}

}  // namespace
}  // namespace petch

namespace petch {
namespace {

struct IonP {
    float meanE, sigmaE, A_sp, Eth_sp, B_sp, A_ie, Eth_ie, A_p, Eth_p;
    float inflect, minang, n_l, A_en, minE, thrmin, thrmax, sigma;
};

__global__ void k_zero_faces(const int* hdr, int MT, float* a, int na, float* b, int nb) {
    const int F = min(hdr[HDR_F], MT);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F * na; i += gridDim.x * blockDim.x) a[i] = 0.0f;
    if (b)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F * nb; i += gridDim.x * blockDim.x) b[i] = 0.0f;
}


// One deposit into a tally.  mode bit 0 (kTallyDet) clear: float atomic add into out[i].  Set:
// out is an int64 accumulator array (same indexing) and v is added in units of 2^-32 -- integer
// sums do not depend on the order of the additions, so the result is the same on every run.
//
// Mode bit 1 (kTallyAgg, petch_tally_aggregation): warp aggregation.  The lanes of a warp that
// deposit into the same address in the same call (matched on the address, since lanes of one
// warp may write different arrays: the two species of a paired launch, the instances of a
// batched one) are found with one match instruction; the lowest of them adds the group's sum
// (gathered by shuffles in lane order) and the others issue nothing.  With deterministic tallies
// each lane converts its own deposit to fixed point before the integer sum, so the accumulator
// receives exactly the sum of the per-deposit units either way.  The match costs every deposit a
// few instructions, so it pays only where lanes of a warp often deposit on the same face.
constexpr int kTallyDet = 1, kTallyAgg = 2;

template <class T>
__device__ __forceinline__ T group_sum(unsigned peers, T v) {
    T s = T(0);
    for (unsigned r = peers; r; r &= r - 1) s += __shfl_sync(peers, v, __ffs(r) - 1);
    return s;
}

__device__ __forceinline__ void tally(float* out, long long i, float v, int mode) {
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(out) + i;
    float* dst = out + i;
    if (mode & kTallyAgg) {
        const unsigned peers = __match_any_sync(
            __activemask(), (mode & kTallyDet) ? reinterpret_cast<unsigned long long>(acc)
                                               : reinterpret_cast<unsigned long long>(dst));
        const bool lead = (threadIdx.x & 31) == __ffs(peers) - 1;
        if (mode & kTallyDet) {
            long long u = __float2ll_rn(v * kTallyScale);
            if (peers & (peers - 1)) u = group_sum(peers, u);
            if (lead) atomicAdd(acc, (unsigned long long)u);
        } else {
            if (peers & (peers - 1)) v = group_sum(peers, v);
            if (lead) atomicAdd(dst, v);
        }
    } else if (mode & kTallyDet) {
        atomicAdd(acc, (unsigned long long)__float2ll_rn(v * kTallyScale));
    } else {
        atomicAdd(dst, v);
    }
}

// The float-atomic ion deposit (four yields-and-weight entries of one face plus cos * w),
// aggregated as one group per face when `agg`.
__device__ __forceinline__ void tally_ion(float4* tal4, float* ang, int f, float4 dep, float a,
                                          bool agg) {
    if (agg) {
        const unsigned peers =
            __match_any_sync(__activemask(), reinterpret_cast<unsigned long long>(tal4 + f));
        if (peers & (peers - 1)) {
            dep.x = group_sum(peers, dep.x);
            dep.y = group_sum(peers, dep.y);
            dep.z = group_sum(peers, dep.z);
            dep.w = group_sum(peers, dep.w);
            a = group_sum(peers, a);
        }
        if ((threadIdx.x & 31) != __ffs(peers) - 1) return;
    }
    atomicAdd(tal4 + f, dep);
    atomicAdd(ang + f, a);
}

// The face's unit winding normal as stored by the mesh build (float32, bit-identical to
// normalize(cross(b - a, c - a)) on the float32 vertices, the normal Warp's query returns).
__device__ __forceinline__ float3 stored_normal(const MeshView& m, int f) {
    return make_float3(__ldg(m.normal + 3 * f), __ldg(m.normal + 3 * f + 1), __ldg(m.normal + 3 * f + 2));
}

// Per-ray state carried between queries.
struct RayState {
    float w, E;
    int bounce, wraps, id;
    float dE;        // tangent of E w.r.t. the mean ion energy (tangent shaders only)
    float dw[3];     // tangents of the neutral weight (tangent shaders only)
};

// _trace3d_cov_rr (threed.py:549-596): deposit the weight on every hit, W *= 1 - bare * beta,
// stop at W <= 1e-6, Russian roulette below 0.1 (survive with probability W / 0.3 at weight
// 0.3), cosine re-emission; at most 1024 bounces.
__device__ __forceinline__ bool neutral_hit(const float* bare, float beta, float* flux, Rng& g,
                                            const Tracer& T, int f, float t, float3& o, float3& d,
                                            RayState& s, int det) {
    float3 nrm = stored_normal(T.m, f);
    if (dot3(nrm, d) > 0.0f) nrm = -nrm;
    tally(flux, f, s.w, det);
    float S = (bare ? __ldg(bare + f) : 1.0f) * beta;
    s.w = s.w - s.w * S;
    if (s.w <= 1.0e-6f) return false;
    if (s.w < 0.1f) {
        if (g.uniform() < (1.0f - s.w / 0.3f)) return false;
        s.w = 0.3f;
    }
    float3 h = o + t * d;
    d = cosine_emit(g, nrm);
    o = h + 1.0e-4f * nrm;
    return true;
}

// neutral_hit with weight tangents: d(deposit) = dw, dw' = dw (1 - S) - w dS with
// dS = dbare * beta (dbare[0..2][MT]); the roulette decisions are those of the primal path.
__device__ __forceinline__ bool neutral_hit_tan(const float* bare, const float* dbare, float beta,
                                                float* flux, float* dflux, Rng& g, const Tracer& T,
                                                int f, float t, float3& o, float3& d, RayState& s,
                                                int det) {
    float3 nrm = stored_normal(T.m, f);
    if (dot3(nrm, d) > 0.0f) nrm = -nrm;
    const long long MT = T.m.MT;
    tally(flux, f, s.w, det);
#pragma unroll
    for (int k = 0; k < 3; ++k) tally(dflux, k * MT + f, s.dw[k], det);
    float S = (bare ? __ldg(bare + f) : 1.0f) * beta;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float dS = dbare ? __ldg(dbare + k * MT + f) * beta : 0.0f;
        s.dw[k] = s.dw[k] - (s.dw[k] * S + s.w * dS);
    }
    s.w = s.w - s.w * S;
    if (s.w <= 1.0e-6f) return false;
    if (s.w < 0.1f) {
        if (g.uniform() < (1.0f - s.w / 0.3f)) return false;
        // the survivor stands for weight w with probability w / 0.3: with that probability held
        // fixed, its weight 0.3 = w / p has tangent dw / p = dw * 0.3 / w (an unbiased estimate of
        // the derivative of the expected deposits)
        const float r = 0.3f / s.w;
#pragma unroll
        for (int k = 0; k < 3; ++k) s.dw[k] *= r;
        s.w = 0.3f;
    }
    float3 h = o + t * d;
    d = cosine_emit(g, nrm);
    o = h + 1.0e-4f * nrm;
    return true;
}

struct NeutralShader {
    const float* bare;
    float beta;
    float* flux;
    int det;
    static constexpr int kMaxBounce = 1024;
    static constexpr int kMinBlocks = kTraceMinBlocksRR;
    __device__ __forceinline__ int count(const MeshView&, int n) const { return n; }
    __device__ __forceinline__ void init(Rng& g, const Tracer&, const Domain& D, int, float3& o,
                                         float3& d, RayState& s) const {
        source(g, false, 0.0f, D, o, d);
        s.w = 1.0f;
    }
    __device__ __forceinline__ bool hit(Rng& g, const Tracer& T, int f, float t, float3& o,
                                        float3& d, RayState& s) const {
        return neutral_hit(bare, beta, flux, g, T, f, t, o, d, s, det);
    }
};

// Both neutral species of one coverage round in one launch (threed.py:898-902: the F trace with
// betaE and seed s_a, then the O trace with betaO and seed s_b, on the same coverage): rays
// [0, n) are species a, rays [n, 2n) species b.  Ray r of a species draws the Philox stream of ray
// r in the single-species launch with that species' seed, so each tally equals its own launch's
// up to the order of float atomic additions (and exactly with deterministic tallies); one launch
// has one tail instead of two.
struct NeutralPairShader {
    const float* bare;
    float beta_a, beta_b;
    float* flux_a;
    float* flux_b;
    uint32_t seed_delta, domain;   // species b's seed minus species a's (the launch's seed)
    int n;
    int det;
    static constexpr int kMaxBounce = 1024;
    static constexpr int kMinBlocks = kTraceMinBlocksRR;
    __device__ __forceinline__ int count(const MeshView&, int n2) const { return n2; }
    __device__ __forceinline__ void init(Rng& g, const Tracer&, const Domain& D, int ray, float3& o,
                                         float3& d, RayState& s) const {
        if (ray >= n) g.init(g.key.x + seed_delta, domain, (uint32_t)(ray - n));
        source(g, false, 0.0f, D, o, d);
        s.w = 1.0f;
    }
    __device__ __forceinline__ bool hit(Rng& g, const Tracer& T, int f, float t, float3& o,
                                        float3& d, RayState& s) const {
        const bool b = s.id >= n;
        return neutral_hit(bare, b ? beta_b : beta_a, b ? flux_b : flux_a, g, T, f, t, o, d, s,
                           det);
    }
};

// The electron trace of the electron-shadowing charging model (threed.py:847-857):
// _trace3d_cov_rr with bare = 1 and beta = 1 on rays from the ion-type (Gaussian angle, sigma =
// e_ang_sigma) source, so every electron sticks where it first lands and deposits weight 1; the
// lateral wrap follows the domain.
struct ElectronShader {
    float sigma;
    float* flux;
    int det;
    static constexpr int kMaxBounce = 1;
    static constexpr int kMinBlocks = kTraceMinBlocksRR;
    __device__ __forceinline__ int count(const MeshView&, int n) const { return n; }
    __device__ __forceinline__ void init(Rng& g, const Tracer&, const Domain& D, int, float3& o,
                                         float3& d, RayState& s) const {
        source(g, true, sigma, D, o, d);
        s.w = 1.0f;
    }
    __device__ __forceinline__ bool hit(Rng&, const Tracer&, int f, float, float3&, float3&,
                                        RayState& s) const {
        tally(flux, f, s.w, det);
        return false;
    }
};

// _trace3d_ion_yield (threed.py:599-712): E ~ N(meanE, sigmaE) clipped at 0; on every hit
// deposit the yield-weighted sputter / ion-enhanced / passivation rates, the weight and
// cos * weight; then angle-dependent sticking, energy loss (<= 4 truncated-normal tries), weight
// reduction and coned-cosine reflection about the specular axis (<= 64 accept-reject draws);
// at most 1024 bounces.  tal4[f] = (sp, ie, ip, arr), ang[f] = sum cos * w.
// TAN: also accumulate d(sputter, ion-enhanced, passivation tallies) / d(mean ion energy) into
// dtal[0..2][MT] along the same path (hits, sticking and energy-acceptance decisions fixed) and
// carry dE / dE_mean through the energy losses.
template <bool TAN = false>
__device__ __forceinline__ bool ion_hit(const IonP& P, float4* tal4, float* ang, Rng& g,
                                        const Tracer& T, int f, float t, float3& o, float3& d,
                                        RayState& s, int det, float* dtal = nullptr) {
    const float PI_2 = 1.5707963f;
    float3 nrm = stored_normal(T.m, f);
    if (dot3(nrm, d) > 0.0f) nrm = -nrm;
    float cosT = fminf(fmaxf(-dot3(d, nrm), 0.0f), 1.0f);
    float incAng = acosf(cosT);
    float sqrtE = sqrtf(s.E);
    float f_sp = fmaxf((1.0f + P.B_sp * (1.0f - cosT * cosT)) * cosT, 0.0f);
    float f_ie = 1.0f;
    if (cosT < 0.5f) f_ie = fmaxf(3.0f - 6.0f * incAng / 3.14159265f, 0.0f);
    float w = s.w;
    const float4 dep = make_float4(P.A_sp * fmaxf(sqrtE - sqrtf(P.Eth_sp), 0.0f) * f_sp * w,
                                   P.A_ie * fmaxf(sqrtE - sqrtf(P.Eth_ie), 0.0f) * f_ie * w,
                                   P.A_p * fmaxf(sqrtE - sqrtf(P.Eth_p), 0.0f) * f_ie * w, w);
    if (det & kTallyDet) {
        float* t4 = reinterpret_cast<float*>(tal4);
        tally(t4, 4LL * f, dep.x, det);
        tally(t4, 4LL * f + 1, dep.y, det);
        tally(t4, 4LL * f + 2, dep.z, det);
        tally(t4, 4LL * f + 3, dep.w, det);
        tally(ang, f, cosT * w, det);
    } else {
        tally_ion(tal4, ang, f, dep, cosT * w, det & kTallyAgg);
    }
    if (TAN) {
        const long long MT = T.m.MT;
        const float dsq = s.E > 0.0f ? 0.5f * s.dE / sqrtE : 0.0f;
        if (sqrtE > sqrtf(P.Eth_sp)) tally(dtal, f, P.A_sp * dsq * f_sp * w, det);
        if (sqrtE > sqrtf(P.Eth_ie)) tally(dtal, MT + f, P.A_ie * dsq * f_ie * w, det);
        if (sqrtE > sqrtf(P.Eth_p)) tally(dtal, 2 * MT + f, P.A_p * dsq * f_ie * w, det);
    }
    float stick = 1.0f;
    if (incAng > P.thrmin) stick = 1.0f - fminf(fmaxf((incAng - P.thrmin) / (P.thrmax - P.thrmin), 0.0f), 1.0f);
    if (stick >= 1.0f) return false;
    float Eref = incAng >= P.inflect
                     ? 1.0f - (1.0f - P.A_en) * (PI_2 - incAng) / (PI_2 - P.inflect)
                     : P.A_en * powf(incAng / P.inflect, P.n_l);
    const float E = s.E;
    float newE = Eref * E;
    float slope = Eref;                      // d newE / d E on the taken branch
    for (int e = 0; e < 4; ++e) {
        const float z = g.normal();
        float cand = Eref * E + 0.1f * E * z;
        if (cand >= 0.0f && cand <= E) {
            newE = cand;
            slope = Eref + 0.1f * z;
            break;
        }
    }
    if (newE < 0.0f) slope = 0.0f;
    if (newE > E) slope = 1.0f;
    newE = fminf(fmaxf(newE, 0.0f), E);
    if (newE <= P.minE) return false;
    if (TAN) s.dE = slope * s.dE;
    s.E = newE;
    s.w = w - w * stick;
    if (s.w <= 1.0e-4f) return false;
    float3 h = o + t * d;
    float3 axis = normalize3(d - (2.0f * dot3(d, nrm)) * nrm);
    float3 tt, bb;
    if (axis.z < -0.9999999f) {
        tt = make_float3(0.0f, -1.0f, 0.0f);
        bb = make_float3(-1.0f, 0.0f, 0.0f);
    } else {
        float aa = 1.0f / (1.0f + axis.z);
        float cc = -axis.x * axis.y * aa;
        tt = make_float3(1.0f - axis.x * axis.x * aa, cc, -axis.x);
        bb = make_float3(cc, 1.0f - axis.y * axis.y * aa, -axis.y);
    }
    float maxcone = PI_2 - fminf(incAng, P.minang);
    float theta = 0.0f;
    for (int q = 0; q < 64; ++q) {
        float uu = sqrtf(g.uniform());
        float ss = sqrtf(fmaxf(1.0f - uu, 0.0f));
        theta = maxcone * ss;
        if (g.uniform() * theta * uu <= cosf(PI_2 * ss) * sinf(theta)) break;
    }
    float ph = 6.2831853f * g.uniform();
    float st = sinf(theta);
    float3 nd = normalize3((st * cosf(ph)) * tt + (st * sinf(ph)) * bb + cosf(theta) * axis);
    float dn = dot3(nd, nrm);
    if (dn <= 0.0f) nd = nd - (2.0f * dn) * nrm;
    d = nd;
    o = h + 1.0e-4f * nrm;
    return true;
}

struct IonShader {
    IonP P;
    float4* tal4;
    float* ang;
    int det;
    static constexpr int kMaxBounce = 1024;
    static constexpr int kMinBlocks = kTraceMinBlocks;
    __device__ __forceinline__ int count(const MeshView&, int n) const { return n; }
    __device__ __forceinline__ void init(Rng& g, const Tracer&, const Domain& D, int, float3& o,
                                         float3& d, RayState& s) const {
        source(g, true, P.sigma, D, o, d);
        s.E = fmaxf(P.meanE + P.sigmaE * g.normal(), 0.0f);
        s.w = 1.0f;
    }
    __device__ __forceinline__ bool hit(Rng& g, const Tracer& T, int f, float t, float3& o,
                                        float3& d, RayState& s) const {
        return ion_hit(P, tal4, ang, g, T, f, t, o, d, s, det);
    }
};

// _trace3d (threed.py:352-406), the legacy species: specular == 1 deposits (1 - R) and reflects
// specularly below cos_thr with energy retention eta; otherwise the particle sticks with
// probability `sticking` or at re-emission n_reemit, depositing w and w * cos.
struct LegacyShader {
    int ion, n_reemit, specular;
    float sigma, sticking, cos_thr, eta;
    float* flux;
    float* angacc;
    int det;
    static constexpr int kMaxBounce = 1 << 30;
    static constexpr int kMinBlocks = kTraceMinBlocks;
    __device__ __forceinline__ int count(const MeshView&, int n) const { return n; }
    __device__ __forceinline__ void init(Rng& g, const Tracer&, const Domain& D, int, float3& o,
                                         float3& d, RayState& s) const {
        source(g, ion != 0, sigma, D, o, d);
        s.w = 1.0f;
    }
    __device__ __forceinline__ bool hit(Rng& g, const Tracer& T, int f, float t, float3& o,
                                        float3& d, RayState& s) const {
        float3 nrm = stored_normal(T.m, f);
        if (dot3(nrm, d) > 0.0f) nrm = -nrm;
        float cosang = fmaxf(-dot3(d, nrm), 0.0f);
        float3 h = o + t * d;
        if (specular == 1) {
            if (cosang >= cos_thr || s.bounce == n_reemit) {
                tally(flux, f, s.w, det);
                tally(angacc, f, s.w * cosang, det);
                return false;
            }
            float R = (cos_thr - cosang) / cos_thr;
            float dep = s.w * (1.0f - R);
            tally(flux, f, dep, det);
            tally(angacc, f, dep * cosang, det);
            s.w = s.w * R * eta;
            d = d - (2.0f * dot3(d, nrm)) * nrm;
        } else {
            if (g.uniform() < sticking || s.bounce == n_reemit) {
                tally(flux, f, s.w, det);
                tally(angacc, f, s.w * cosang, det);
                return false;
            }
            d = cosine_emit(g, nrm);
        }
        o = h + 1.0e-4f * nrm;
        return true;
    }
};

// Tangent versions of the ion and neutral shaders (the primal tallies plus their tangents).
struct IonTanShader {
    IonP P;
    float4* tal4;
    float* ang;
    float* dtal;            // [3][MT]: d(sp, ie, ip) / d(mean ion energy)
    int det;
    static constexpr int kMaxBounce = 1024;
    static constexpr int kMinBlocks = kTraceMinBlocks;
    __device__ __forceinline__ int count(const MeshView&, int n) const { return n; }
    __device__ __forceinline__ void init(Rng& g, const Tracer&, const Domain& D, int, float3& o,
                                         float3& d, RayState& s) const {
        source(g, true, P.sigma, D, o, d);
        s.E = fmaxf(P.meanE + P.sigmaE * g.normal(), 0.0f);
        s.dE = s.E > 0.0f ? 1.0f : 0.0f;
        s.w = 1.0f;
    }
    __device__ __forceinline__ bool hit(Rng& g, const Tracer& T, int f, float t, float3& o,
                                        float3& d, RayState& s) const {
        return ion_hit<true>(P, tal4, ang, g, T, f, t, o, d, s, det, dtal);
    }
};

struct NeutralTanShader {
    const float* bare;
    const float* dbare;     // [3][MT]
    float beta;
    float* flux;
    float* dflux;           // [3][MT]
    int det;
    static constexpr int kMaxBounce = 1024;
    static constexpr int kMinBlocks = kTraceMinBlocksRRTan;
    __device__ __forceinline__ int count(const MeshView&, int n) const { return n; }
    __device__ __forceinline__ void init(Rng& g, const Tracer&, const Domain& D, int, float3& o,
                                         float3& d, RayState& s) const {
        source(g, false, 0.0f, D, o, d);
        s.w = 1.0f;
        s.dw[0] = s.dw[1] = s.dw[2] = 0.0f;
    }
    __device__ __forceinline__ bool hit(Rng& g, const Tracer& T, int f, float t, float3& o,
                                        float3& d, RayState& s) const {
        return neutral_hit_tan(bare, dbare, beta, flux, dflux, g, T, f, t, o, d, s, det);
    }
};

// NeutralPairShader with weight tangents: both species of a coverage round in one launch, each
// carrying d(weight) / d(theta) along its path (the species' own beta scales dbare).
struct NeutralTanPairShader {
    const float* bare;
    const float* dbare;     // [3][MT]
    float beta_a, beta_b;
    float* flux_a;
    float* dflux_a;         // [3][MT]
    float* flux_b;
    float* dflux_b;         // [3][MT]
    uint32_t seed_delta, domain;   // species b's seed minus species a's (the launch's seed)
    int n;
    int det;
    static constexpr int kMaxBounce = 1024;
    static constexpr int kMinBlocks = kTraceMinBlocksRRTan;
    __device__ __forceinline__ int count(const MeshView&, int n2) const { return n2; }
    __device__ __forceinline__ void init(Rng& g, const Tracer&, const Domain& D, int ray, float3& o,
                                         float3& d, RayState& s) const {
        if (ray >= n) g.init(g.key.x + seed_delta, domain, (uint32_t)(ray - n));
        source(g, false, 0.0f, D, o, d);
        s.w = 1.0f;
        s.dw[0] = s.dw[1] = s.dw[2] = 0.0f;
    }
    __device__ __forceinline__ bool hit(Rng& g, const Tracer& T, int f, float t, float3& o,
                                        float3& d, RayState& s) const {
        const bool b = s.id >= n;
        return neutral_hit_tan(bare, dbare, b ? beta_b : beta_a, b ? flux_b : flux_a,
                               b ? dflux_b : dflux_a, g, T, f, t, o, d, s, det);
    }
};

// _trace_ff + the emission of mc_flux_3d_radiosity (threed.py:908-920, 947-956): ray p leaves
// face j = p / n_ff from centroid + 1e-3 * n_gas in a cosine direction about the into-gas normal
// (the tangent frame of _cosine_dirs, threed.py:1571-1579); its first hit face is recorded (the
// entries stay -1 for rays that escape to the open top).  Only F * n_ff rays exist.
struct FormFactorShader {
    const float* fn;     // into-gas unit normals, float[3 * MT]
    int n_ff;
    int* hitface;
    static constexpr int kMaxBounce = 1;
    static constexpr int kMinBlocks = kTraceMinBlocks;
    __device__ __forceinline__ int count(const MeshView& m, int n) const {
        const long long F = min(m.hdr[HDR_F], m.MT);
        return (int)min((long long)n, F * n_ff);
    }
    __device__ __forceinline__ void init(Rng& g, const Tracer& T, const Domain&, int ray,
                                         float3& o, float3& d, RayState& s) const {
        const int j = ray / n_ff;
        const float3 n = make_float3(__ldg(fn + 3 * j), __ldg(fn + 3 * j + 1), __ldg(fn + 3 * j + 2));
        const float3 c = make_float3(__ldg(T.m.centroid + 3 * j), __ldg(T.m.centroid + 3 * j + 1),
                                     __ldg(T.m.centroid + 3 * j + 2));
        o = c + 1.0e-3f * n;
        d = cosine_emit(g, n);
        s.w = 1.0f;
    }
    __device__ __forceinline__ bool hit(Rng&, const Tracer&, int f, float, float3&, float3&,
                                        RayState& s) const {
        hitface[s.id] = f;
        return false;
    }
};

// mc_redep_3d (threed.py:1582-1605): etch product leaves face j with probability
// w_j / sum(w), w = max(V * area, 0) (cdf: inclusive float64 prefix of w), from centroid + 1e-3 n_gas
// in a cosine direction about the into-gas normal, then moves like a Russian-roulette neutral
// that sticks with probability s_redep everywhere (bare = 1, beta = s_redep).
struct RedepShader {
    NeutralShader rr;
    const double* cdf;
    const float* fn;
    static constexpr int kMaxBounce = NeutralShader::kMaxBounce;
    static constexpr int kMinBlocks = kTraceMinBlocksRR;
    __device__ __forceinline__ int count(const MeshView& m, int n) const {
        const int F = min(m.hdr[HDR_F], m.MT);
        return (F > 0 && cdf[F - 1] > 0.0) ? n : 0;
    }
    __device__ __forceinline__ void init(Rng& g, const Tracer& T, const Domain&, int, float3& o,
                                         float3& d, RayState& s) const {
        const int F = min(T.m.hdr[HDR_F], T.m.MT);
        const uint32_t a = g.next_u32() >> 5, b = g.next_u32() >> 6;   // 27 + 26 bits
        const double u = ((double)a * 67108864.0 + (double)b) * (1.0 / 9007199254740992.0);
        const double target = u * cdf[F - 1];
        int lo = 0, hi = F - 1;                  // first j with cdf[j] > target
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (cdf[mid] > target) hi = mid;
            else lo = mid + 1;
        }
        const int j = lo;
        const float3 n = make_float3(__ldg(fn + 3 * j), __ldg(fn + 3 * j + 1), __ldg(fn + 3 * j + 2));
        const float3 c = make_float3(__ldg(T.m.centroid + 3 * j), __ldg(T.m.centroid + 3 * j + 1),
                                     __ldg(T.m.centroid + 3 * j + 2));
        o = c + 1.0e-3f * n;
        d = cosine_emit(g, n);
        s.w = 1.0f;
    }
    __device__ __forceinline__ bool hit(Rng& g, const Tracer& T, int f, float t, float3& o,
                                        float3& d, RayState& s) const {
        return rr.hit(g, T, f, t, o, d, s);
    }
};

// w_j = max(V_j * area_j, 0) in float64 (the CDF's input); scanned in place afterwards.
__global__ void k_redep_weights(MeshView m, const float* __restrict__ V, double* __restrict__ w) {
    const int F = min(m.hdr[HDR_F], m.MT);
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.MT; f += gridDim.x * blockDim.x)
        w[f] = f < F ? fmax((double)V[f] * (double)m.area[f], 0.0) : 0.0;
}

// Rf = flux * (sum(w) / n) / area; V = max(V - k_redep * Rf, 0); stats[1] = bits of max V.
__global__ void k_redep_apply(MeshView m, const float* __restrict__ flux,
                              const double* __restrict__ cdf, int n, float k_redep,
                              float* __restrict__ V, float* __restrict__ Rf, int* stats) {
    const int F = min(m.hdr[HDR_F], m.MT);
    const double tot = F > 0 ? cdf[F - 1] : 0.0;
    float vmax = 0.0f;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x) {
        float r = 0.0f;
        if (tot > 0.0 && n > 0) r = (float)((double)flux[f] * (tot / n) / (double)m.area[f]);
        if (Rf) Rf[f] = r;
        const float v = fmaxf(V[f] - k_redep * r, 0.0f);
        V[f] = v;
        vmax = fmaxf(vmax, v);
    }
    for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(kFull, vmax, o));
    if ((threadIdx.x & 31) == 0 && stats) atomicMax(stats + 1, __float_as_int(vmax));
}

// Launch controls of the persistent tracers: traversal steps per warp round, lanes kept
// traversing, leaf grouping (0 = off), and, when `step` is set, the seed taken on the device:
// seed + (*step + seed_off) * seed_mul (the step counter of a captured etch step).
struct TraceCtl {
    int steps, keep, group;
    const int* step;
    uint32_t seed_mul, seed_off;
};

// The visit bound of grouped steps, checked once per round rather than on every step (2-3 %
// faster on the trench run): a query past kMaxVisits visits is closed with error bit 1; the
// bound is exceeded by at most one round's steps.
__device__ __forceinline__ void visit_bound_round(Query& q, int& phase, int* err) {
    if (phase == 1 && q.visits > kMaxVisits) {
        *err |= 1;
        q.cur = kDone;
        phase = 2;
    }
}

// Traversal steps of a warp (binary or 8-wide tree) with the node and leaf halves grouped: each
// iteration runs leaf steps for the lanes at a leaf when they are at least 1/group of the open
// lanes, otherwise node steps for the lanes at an internal node, so the triangle and the box
// paths do not take turns inside one iteration with few lanes each (each iteration advances at
// least one lane).
template <bool WIDE, class St>
__device__ __forceinline__ void grouped_steps(const Tracer& T, Query& q, St& stk, int& phase,
                                              int steps, int keep_now, int group, int* err) {
    for (int s = 0; s < steps; ++s) {
        const bool open = phase == 1;
        const int no = __popc(__ballot_sync(kFull, open));
        if (no <= keep_now) break;
        const bool at_leaf = open && q.cur < 0;
        const int nl = __popc(__ballot_sync(kFull, at_leaf));
        const bool leaves = nl * group >= no;
        if (open && at_leaf == leaves) {
            ++q.visits;                   // bounded once per round by visit_bound_round
            bool fin;
            if (leaves) fin = step_leaf(T, q, stk);
            else if (WIDE) fin = step_wide_node(T, q, stk, err);
            else fin = step_binary_node(T, q, stk, err);
            if (fin) phase = 2;
        }
    }
}

// Persistent tracer.  Each warp loops: refill lanes whose ray ended (one atomic per warp), run
// traversal steps on every lane with an open query (up to `steps`, and only while more than
// `keep` lanes still have one), then resolve the lanes whose query finished -- a miss wraps laterally (periodic domains, <= 256 wraps per bounce, then one
// final query) or ends the ray; a hit goes to the shader, which deposits and either re-emits
// (new query) or ends the ray.
template <class S, bool WIDE>
__global__ void __launch_bounds__(kTB, S::kMinBlocks) k_trace(MeshView m, Domain D, S sh, uint32_t seed,
                                               uint32_t domain, int n, TraceCtl c, int* work) {
    extern __shared__ float4 s_wn[];
    const Tracer T = make_tracer(m, s_wn, WIDE);
    const int steps = c.steps, keep = c.keep;
    if (c.step) seed += ((uint32_t)*c.step + c.seed_off) * c.seed_mul;
    n = sh.count(m, n);
    LocalStack stk;
    int err = 0;
    if (WIDE && T.L > 0 && m.hdr[HDR_WLEVELS] < 0) {   // mesh built without the 8-wide tree
        err = 8;
        n = 0;
    }
    unsigned long long n_query = 0, n_visit = 0;
    int ray = -1, phase = 0;   // phase 1: query open, 2: query finished
    Query q;
    RayState rs;
    Rng g;
    bool pool_empty = false;   // warp-uniform: once set, no lane can be refilled any more
    for (long long round = 0;; ++round) {
        if (round >= kMaxRounds) {   // last-resort bound (never reached by a valid mesh)
            err |= 4;
            break;
        }
        if (refill(ray, n, work)) {
            g.init(seed, domain, (uint32_t)ray);
            float3 o, d;
            rs.id = ray;
            sh.init(g, T, D, ray, o, d, rs);
            rs.bounce = 0;
            rs.wraps = 0;
            if (D.periodic && !descend_wrapped(D, root_top(T.m, T.L), o, d, rs.wraps)) {
                ray = -1;                     // never reaches the surface
                phase = 0;
            } else {
                query_begin(q, T, o, d, 1.0e6f, WIDE);
                ++n_query;
                phase = q.cur == kDone ? 2 : 1;   // an empty mesh: the query is over at once
            }
        }
        if (__all_sync(kFull, ray == -2)) break;
        // Traverse while more than `keep` lanes still have an open query (at most `steps` steps),
        // so lanes that finished early idle only while most of the warp is still busy.  Once the
        // ray pool is empty no lane can be refilled, so the warp then steps until every query is
        // done (keep 0): each round makes progress.
        pool_empty = pool_empty || __any_sync(kFull, ray == -2);
        const int keep_now = pool_empty ? 0 : keep;
        if (c.group > 0) {
            visit_bound_round(q, phase, &err);
            grouped_steps<WIDE>(T, q, stk, phase, steps, keep_now, c.group, &err);
        }
        else
        for (int s = 0; s < steps; ++s) {
            if (__popc(__ballot_sync(kFull, phase == 1)) <= keep_now) break;
            if (phase == 1) {
                bool fin = WIDE ? step_wide(T, q, stk, &err) : step_binary(T, q, stk, &err);
                if (fin) phase = 2;
            }
        }
        if (phase == 2) {
            float3 o = q.r.o, d = q.r.d;
            bool cont;
            if (q.f < 0) {
                cont = D.periodic && rs.wraps < 256 && periodic_wrap(D, o, d);
                if (cont) {
                    ++rs.wraps;
                    cont = descend_wrapped(D, root_top(T.m, T.L), o, d, rs.wraps);
                }
            } else {
                cont = sh.hit(g, T, q.f, q.t, o, d, rs);
                rs.wraps = 0;
                if (cont && ++rs.bounce >= S::kMaxBounce) cont = false;
            }
            n_visit += q.visits;
            if (cont) {
                query_begin(q, T, o, d, 1.0e6f, WIDE);
                ++n_query;
                phase = q.cur == kDone ? 2 : 1;
            } else {
                ray = -1;
                phase = 0;
            }
        }
    }
    if (err) atomicOr(work + 1, err);
    // work[2..3]: queries started, work[4..5]: node + leaf visits (64-bit, warp-reduced)
    for (int o = 16; o > 0; o >>= 1) {
        n_query += __shfl_xor_sync(kFull, n_query, o);
        n_visit += __shfl_xor_sync(kFull, n_visit, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(work + 2), n_query);
        atomicAdd(reinterpret_cast<unsigned long long*>(work + 4), n_visit);
    }
}

// ---------------------------------------------------------------------------------------------
// Batched tracing: one persistent launch over the rays of up to kMaxBatch independent instances
// (feature / recipe pairs), each with its own mesh buffer (all laid out for the same capacities),
// domain, ion parameters and output tallies.  Rays are drawn from ONE global queue; ray r of
// instance b has the Philox key ((step + seed_b) * seed_mul + seed_add, domain) and counter r,
// exactly the stream the single-instance launch gives it, so a batched step reproduces the
// per-instance steps' paths.  The instance table is a kernel parameter, read from the parameter
// space; each lane resolves its ray's instance when it takes the ray.
// ---------------------------------------------------------------------------------------------
constexpr int kMaxBatch = 64;

struct BatchItem {
    const char* mesh;
    Domain D;
    IonP P;
    const float* bare;
    float* out;
    float* ang;
    int ray_start;
    uint32_t seed;
};

// Tangent outputs of a batched tangent trace: dout = d(ion tallies) [3][MT] or d(neutral flux)
// [3][MT]; dbare = the coverage tangents [3][MT] (neutrals; NULL = 0).
struct BatchTan {
    float* dout;
    const float* dbare;
};

struct BatchTable {
    BatchItem it[kMaxBatch];
    BatchTan tn[kMaxBatch];
    float* dout2[kMaxBatch];   // kind 5: the second species' weight tangents [3][MT]
    int B;
    int total;
};

struct MeshOffsets {
    long long off[SEG_COUNT];
};

__device__ __forceinline__ MeshView view_at(const char* base, const MeshOffsets& L, int MT, int MV) {
    MeshView v;
    char* b = const_cast<char*>(base);
    v.hdr = (int*)(b + L.off[SEG_HDR]);
    v.vnode = (float*)(b + L.off[SEG_VNODE]);
    v.verts = (float*)(b + L.off[SEG_VERTS]);
    v.faces = (int*)(b + L.off[SEG_FACES]);
    v.tri = (float4*)(b + L.off[SEG_TRI]);
    v.area = (float*)(b + L.off[SEG_AREA]);
    v.normal = (float*)(b + L.off[SEG_NORMAL]);
    v.centroid = (float*)(b + L.off[SEG_CENTROID]);
    v.fmask = (uint8_t*)(b + L.off[SEG_FMASK]);
    v.nbr = (int*)(b + L.off[SEG_NBR]);
    v.nbrw = (float*)(b + L.off[SEG_NBRW]);
    v.leaf_code = (uint32_t*)(b + L.off[SEG_LEAF_CODE]);
    v.leaf_start = (int*)(b + L.off[SEG_LEAF_START]);
    v.nodes = (float4*)(b + L.off[SEG_NODES]);
    v.parent = (int*)(b + L.off[SEG_PARENT]);
    v.flags = (int*)(b + L.off[SEG_FLAGS]);
    v.wnodes = (WNode*)(b + L.off[SEG_WNODES]);
    v.wfront = (int2*)(b + L.off[SEG_WFRONT]);
    v.MT = MT;
    v.MV = MV;
    return v;
}

// Zero each instance's tallies on its live faces (blockIdx.y = instance), and with tan the three
// tangent directions of dout.
__global__ void k_zero_batch(BatchTable tab, MeshOffsets L, int MT, int MV, int per_face, int tan) {
    const int b = blockIdx.y;
    if (b >= tab.B) return;
    const BatchItem& it = tab.it[b];
    const int F = min(((const int*)(it.mesh + L.off[SEG_HDR]))[HDR_F], MT);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F * per_face; i += gridDim.x * blockDim.x)
        it.out[i] = 0.0f;
    if (it.ang)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
            it.ang[i] = 0.0f;
    if (tan)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
            for (int k = 0; k < 3; ++k) tab.tn[b].dout[i + (long long)k * MT] = 0.0f;
    if (tab.dout2[b])
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
            for (int k = 0; k < 3; ++k) tab.dout2[b][i + (long long)k * MT] = 0.0f;
}

// KIND: 0 ions, 1 neutrals, 2 ions with energy tangents, 3 neutrals with weight tangents (the
// single-instance tangent shaders' hit functions, outputs per instance from tab.tn), 4 both
// neutral species of a coverage round: an item's rays [0, n) follow kind 1 with (beta, seed_add)
// into out, rays [n, 2n) with (beta2, seed_add2) into ang, each species' ray r on the Philox
// stream of ray r of its own kind-1 launch; 5 the same with the weight tangents of kind 3 (the
// second species' into dout2).
template <int KIND>
__global__ void __launch_bounds__(kTB, (KIND == 1 || KIND == 4) ? kTraceMinBlocksRRBatch
                                    : ((KIND == 3 || KIND == 5) ? kTraceMinBlocksRRTan
                                                                : kTraceMinBlocks))
k_trace_batch(BatchTable tab, MeshOffsets L, int MT, int MV, float beta, float beta2,
              const int* step, uint32_t seed_mul, uint32_t seed_add, uint32_t seed_add2,
              uint32_t domain, int steps, int keep, int group, int det, int* work) {
    constexpr bool ION = KIND == 0 || KIND == 2;
    constexpr bool TAN = KIND == 2 || KIND == 3 || KIND == 5;
    constexpr bool PAIR = KIND == 4 || KIND == 5;
    // The instance table is read where it lies, in the kernel's parameter space: a warp's lanes
    // mostly hold rays of one instance (the queue hands out consecutive ray ids), so the reads are
    // near-uniform, and no shared memory is taken from the L1.
    const BatchItem* s_it = tab.it;
    const BatchTan* s_tn = tab.tn;
    auto s_start = [&](int i) { return i < tab.B ? tab.it[i].ray_start : tab.total; };
    const int n = tab.total;
    const uint32_t stepv = step ? (uint32_t)*step : 0u;
    LocalStack stk;
    int err = 0;
    unsigned long long n_query = 0, n_visit = 0;
    int ray = -1, phase = 0, inst = 0;
    Query q;
    RayState rs;
    Rng g;
    Tracer T;
    T.WN = 0;
    T.nsm = 0;
    T.snodes = nullptr;
    T.L = 0;
    T.m = view_at(s_it[0].mesh, L, MT, MV);
    bool pool_empty = false;
    for (long long round = 0;; ++round) {
        if (round >= kMaxRounds) {
            err |= 4;
            break;
        }
        if (refill(ray, n, work)) {
            int lo = 0, hi = tab.B - 1;           // last instance whose range starts at or before ray
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (s_start(mid) <= ray) lo = mid;
                else hi = mid - 1;
            }
            inst = lo;
            const BatchItem& it = s_it[inst];
            T.m = view_at(it.mesh, L, MT, MV);
            T.L = min(T.m.hdr[HDR_L], MT);
            uint32_t local = (uint32_t)(ray - it.ray_start);
            uint32_t sadd = seed_add;
            if (PAIR) {
                const uint32_t nb = (uint32_t)(s_start(inst + 1) - it.ray_start) >> 1;
                if (local >= nb) {
                    local -= nb;
                    sadd = seed_add2;
                }
            }
            g.init((stepv + it.seed) * seed_mul + sadd, domain, local);
            float3 o, d;
            if (ION) {
                source(g, true, it.P.sigma, it.D, o, d);
                rs.E = fmaxf(it.P.meanE + it.P.sigmaE * g.normal(), 0.0f);
                if (TAN) rs.dE = rs.E > 0.0f ? 1.0f : 0.0f;
            } else {
                source(g, false, 0.0f, it.D, o, d);
                if (TAN) rs.dw[0] = rs.dw[1] = rs.dw[2] = 0.0f;
            }
            rs.w = 1.0f;
            rs.bounce = 0;
            rs.wraps = 0;
            rs.id = ray;
            if (it.D.periodic && !descend_wrapped(it.D, root_top(T.m, T.L), o, d, rs.wraps)) {
                ray = -1;                     // never reaches the surface
                phase = 0;
            } else {
                query_begin(q, T, o, d, 1.0e6f, false);
                ++n_query;
                phase = q.cur == kDone ? 2 : 1;
            }
        }
        if (__all_sync(kFull, ray == -2)) break;
        pool_empty = pool_empty || __any_sync(kFull, ray == -2);
        const int keep_now = pool_empty ? 0 : keep;
        if (group > 0) {
            visit_bound_round(q, phase, &err);
            grouped_steps<false>(T, q, stk, phase, steps, keep_now, group, &err);
        }
        else
            for (int s = 0; s < steps; ++s) {
                if (__popc(__ballot_sync(kFull, phase == 1)) <= keep_now) break;
                if (phase == 1) {
                    if (step_binary(T, q, stk, &err)) phase = 2;
                }
            }
        if (phase == 2) {
            const BatchItem& it = s_it[inst];
            float3 o = q.r.o, d = q.r.d;
            bool cont;
            if (q.f < 0) {
                cont = it.D.periodic && rs.wraps < 256 && periodic_wrap(it.D, o, d);
                if (cont) {
                    ++rs.wraps;
                    cont = descend_wrapped(it.D, root_top(T.m, T.L), o, d, rs.wraps);
                }
            } else {
                if (KIND == 0)
                    cont = ion_hit(it.P, reinterpret_cast<float4*>(it.out), it.ang, g, T, q.f, q.t,
                                   o, d, rs, det);
                else if (KIND == 1)
                    cont = neutral_hit(it.bare, beta, it.out, g, T, q.f, q.t, o, d, rs, det);
                else if (KIND == 2)
                    cont = ion_hit<true>(it.P, reinterpret_cast<float4*>(it.out), it.ang, g, T,
                                         q.f, q.t, o, d, rs, det, s_tn[inst].dout);
                else if (KIND == 4) {
                    const int nb = (s_start(inst + 1) - it.ray_start) >> 1;
                    const bool second = rs.id - it.ray_start >= nb;
                    cont = neutral_hit(it.bare, second ? beta2 : beta, second ? it.ang : it.out,
                                       g, T, q.f, q.t, o, d, rs, det);
                } else if (KIND == 5) {
                    const int nb = (s_start(inst + 1) - it.ray_start) >> 1;
                    const bool second = rs.id - it.ray_start >= nb;
                    cont = neutral_hit_tan(it.bare, s_tn[inst].dbare, second ? beta2 : beta,
                                           second ? it.ang : it.out,
                                           second ? tab.dout2[inst] : s_tn[inst].dout, g, T, q.f,
                                           q.t, o, d, rs, det);
                } else
                    cont = neutral_hit_tan(it.bare, s_tn[inst].dbare, beta, it.out,
                                           s_tn[inst].dout, g, T, q.f, q.t, o, d, rs, det);
                rs.wraps = 0;
                if (cont && ++rs.bounce >= 1024) cont = false;
            }
            n_visit += q.visits;
            if (cont) {
                query_begin(q, T, o, d, 1.0e6f, false);
                ++n_query;
                phase = q.cur == kDone ? 2 : 1;
            } else {
                ray = -1;
                phase = 0;
            }
        }
    }
    if (err) atomicOr(work + 1, err);
    for (int o = 16; o > 0; o >>= 1) {
        n_query += __shfl_xor_sync(kFull, n_query, o);
        n_visit += __shfl_xor_sync(kFull, n_visit, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(work + 2), n_query);
        atomicAdd(reinterpret_cast<unsigned long long*>(work + 4), n_visit);
    }
}

// Deterministic tallies back to float: out[i] = acc[i] * 2^-32.
__global__ void k_acc_to_float(const long long* __restrict__ acc, float* __restrict__ out,
                               long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (float)((double)acc[i] * (1.0 / 4294967296.0));
}

struct GridArgs {
    int nx, ny, nz;
    long long plane, n;
    double dx, band;
};

// extend_velocity_gpu / _extend_kernel (threed.py:1324-1346): cells with |phi| < band take the
// velocity of the nearest face, all other cells get 0.  With fold != 0, mask cells are written as
// -1 (the advection's pinned-cell marker) and band cells with F > 0 are listed in `active` for
// the sparse advection.  With dV (tangents [3][MT]) the same nearest face also gives
// dF[c + k n] = dV[f + k MT] on the band (0 elsewhere), as petch_extend_tangent.
//
// Each warp walks 32 consecutive cells at a time (a z-run of a column, of which only the few
// cells near the front are in the band) and queues its band cells in shared memory; whenever 32
// are queued, the warp runs 32 nearest-face queries with every lane busy.  A query first searches
// within |phi| + 1.5 dx (phi is a distance to the front, which the mesh follows to within a
// cell), then within band + 2 dx, then without a limit: each stage returns the nearest face
// within its radius (exact ties to the lower face index), so the result is the global nearest
// face whichever stage finds one.  Pinned cells skip the query unless tangents are wanted.
constexpr int kExtQ = 64;   // queue slots per warp: < 32 carried over + 32 added

template <bool CENTROID>
__device__ __forceinline__ void extend_cell(const MeshView& m, int L, const GridArgs& G,
                                            long long c, float v, bool pinned,
                                            const float* __restrict__ V, float* __restrict__ Fs,
                                            int fold, int* active, int* n_active, int max_active,
                                            const float* __restrict__ dV, float* __restrict__ dF,
                                            int* err) {
    float out = 0.0f;
    float dout[3] = {0.0f, 0.0f, 0.0f};
    if (!pinned || dV) {
        const long long r = c / G.nz;
        const int k = (int)(c - r * G.nz);
        const int i = (int)(r / G.ny);
        const int j = (int)(r - (long long)i * G.ny);
        const float3 p = make_float3((float)(i * G.dx), (float)(j * G.dx), (float)(k * G.dx));
        const float r_near = (float)(G.band + 2.0 * G.dx);
        const float r_small = fabsf(v) + (float)(1.5 * G.dx);
        int f = -1;
        if (r_small < r_near) f = nearest_prim<CENTROID>(m, L, p, r_small * r_small, err);
        if (f < 0) f = nearest_prim<CENTROID>(m, L, p, r_near * r_near, err);
        if (f < 0) f = nearest_prim<CENTROID>(m, L, p, 1.0e12f, err);
        if (f >= 0) {
            out = V[f];
            if (dV)
                for (int q = 0; q < 3; ++q) dout[q] = dV[f + (long long)q * m.MT];
        }
    }
    if (pinned) out = -1.0f;
    Fs[c] = out;
    if (dF)
        for (int q = 0; q < 3; ++q) dF[c + q * G.n] = dout[q];
    if (fold && active && out > 0.0f) {
        const int s = atomicAdd(n_active, 1);
        if (s < max_active) active[s] = (int)c;
        else *err |= 2;
    }
}

template <bool CENTROID>
__global__ void __launch_bounds__(kTB) k_extend(MeshView m, GridArgs G, const float* __restrict__ phi,
                                                const uint8_t* __restrict__ mask,
                                                const float* __restrict__ V, float* __restrict__ Fs,
                                                int fold, int* active, int* n_active, int max_active,
                                                int* work, const float* __restrict__ dV = nullptr,
                                                float* __restrict__ dF = nullptr) {
    __shared__ long long s_cell[kTB / 32][kExtQ];
    __shared__ float s_phi[kTB / 32][kExtQ];
    const int L = min(m.hdr[HDR_L], m.MT);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    long long* qc = s_cell[wid];
    float* qv = s_phi[wid];
    int err = 0;
    int nq = 0;                                      // warp-uniform queue length
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long base = ((long long)blockIdx.x * (blockDim.x >> 5) + wid) * 32; base < G.n;
         base += warps * 32) {
        const long long c = base + lane;
        const bool in = c < G.n;
        const float v = in ? phi[c] : 0.0f;
        const bool band = in && (double)fabsf(v) < G.band;
        if (in && !band) {
            Fs[c] = (fold && mask && mask[c]) ? -1.0f : 0.0f;
            if (dF)
                for (int q = 0; q < 3; ++q) dF[c + q * G.n] = 0.0f;
        }
        const unsigned bal = __ballot_sync(kFull, band);
        if (band) {
            const int slot = nq + __popc(bal & ((1u << lane) - 1u));
            qc[slot] = c;
            qv[slot] = v;
        }
        nq += __popc(bal);
        __syncwarp();
        if (nq >= 32) {
            const long long cc = qc[lane];
            const float vv = qv[lane];
            const int rest = nq - 32;
            long long tc = 0;
            float tv = 0.0f;
            if (lane < rest) {
                tc = qc[32 + lane];
                tv = qv[32 + lane];
            }
            __syncwarp();
            if (lane < rest) {
                qc[lane] = tc;
                qv[lane] = tv;
            }
            nq = rest;
            __syncwarp();
            extend_cell<CENTROID>(m, L, G, cc, vv, fold && mask && mask[cc], V, Fs, fold, active,
                                  n_active, max_active, dV, dF, &err);
        }
    }
    if (lane < nq) {
        const long long cc = qc[lane];
        extend_cell<CENTROID>(m, L, G, cc, qv[lane], fold && mask && mask[cc], V, Fs, fold, active,
                              n_active, max_active, dV, dF, &err);
    }
    if (err) atomicOr(work + 1, err);
}

// _nearest_face_cov + gpu_warmstart_bare (threed.py:1619-1639): each new face centroid takes
// the coverage of the nearest face of the previous mesh (1.0 if none), clipped to [0, 1] as
// mc_flux_3d_coupled does with bare_init.
// With prev_dbare (tangents [3][prev MT]) also dbare = the nearest face's tangents where its
// coverage is strictly inside (0, 1) (the clip's derivative), 0 elsewhere, as petch_warmstart_tangent.
__global__ void __launch_bounds__(kTB) k_warmstart(MeshView prev, const float* __restrict__ prev_bare,
                                                   MeshView cur, float* __restrict__ bare, int* work,
                                                   const float* __restrict__ prev_dbare = nullptr,
                                                   float* __restrict__ dbare = nullptr) {
    const int Lp = min(prev.hdr[HDR_L], prev.MT);
    const int F = min(cur.hdr[HDR_F], cur.MT);
    int err = 0;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x) {
        float3 p = make_float3(cur.centroid[3 * f], cur.centroid[3 * f + 1], cur.centroid[3 * f + 2]);
        int q = nearest_face(prev, Lp, p, 1.0e12f, &err);
        float b = q >= 0 ? prev_bare[q] : 1.0f;
        bare[f] = fminf(fmaxf(b, 0.0f), 1.0f);
        if (dbare) {
            const bool pass = q >= 0 && prev_bare[q] > 0.0f && prev_bare[q] < 1.0f;
            for (int k = 0; k < 3; ++k)
                dbare[f + (long long)k * cur.MT] = pass ? prev_dbare[q + (long long)k * prev.MT] : 0.0f;
        }
    }
    if (err) atomicOr(work + 1, err);
}

__global__ void __launch_bounds__(kTB) k_raycast(MeshView m, const float* __restrict__ o,
                                                 const float* __restrict__ d, int n, float tmax,
                                                 int* __restrict__ face, float* __restrict__ t,
                                                 int* work, int wide) {
    extern __shared__ float4 s_wn[];
    const Tracer T = make_tracer(m, s_wn, wide);
    LocalStack stk;
    int err = 0;
    const bool missing = wide && T.L > 0 && m.hdr[HDR_WLEVELS] < 0;   // no 8-wide tree built
    if (missing) err = 8;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Query q;
        query_begin(q, T, make_float3(o[3 * i], o[3 * i + 1], o[3 * i + 2]),
                    make_float3(d[3 * i], d[3 * i + 1], d[3 * i + 2]), tmax, wide);
        if (missing) q.cur = kDone;
        if (q.cur != kDone)
            while (!(wide ? step_wide(T, q, stk, &err) : step_binary(T, q, stk, &err))) {
            }
        face[i] = q.f;
        t[i] = q.f >= 0 ? q.t : 0.0f;
    }
    if (err) atomicOr(work + 1, err);
}

__global__ void __launch_bounds__(kTB) k_nearest(MeshView m, const float* __restrict__ p, int n,
                                                 float r2max, int* __restrict__ face, int* work) {
    const int L = min(m.hdr[HDR_L], m.MT);
    int err = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        face[i] = nearest_face(m, L, make_float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]), r2max, &err);
    if (err) atomicOr(work + 1, err);
}

constexpr int kSmemBytes = kSmemNodes * 96;


// Resident blocks per SM x SMs for a persistent launch, cached per (kernel, device) so that calls
// made during stream capture issue no driver queries.
int persistent_blocks(const void* kernel, int block, size_t dyn_smem = kSmemBytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_pair(kernel, dev);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, dyn_smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const int blocks = per_sm * sm_count();
    cache[key] = blocks;
    return blocks;
}

}  // namespace
}  // namespace petch

using namespace petch;

static Domain to_domain(const petch_domain* d) {
    Domain D;
    D.lx = d->lx;
    D.ly = d->ly;
    D.lz = d->lz;
    D.z_src = d->z_src;
    D.periodic = d->periodic;
    return D;
}

// Accumulators of one deterministic trace call, carved from the registered scratch.
struct DetArena {
    char* base = static_cast<char*>(g_det_scratch);
    long long cap = g_det_bytes, used = 0;
    bool on() const { return base != nullptr; }
    long long* take(long long count) {
        const long long bytes = ((8 * count) + 255) & ~255LL;
        if (used + bytes > cap) return nullptr;
        long long* p = reinterpret_cast<long long*>(base + used);
        used += bytes;
        return p;
    }
};

static int acc_zero(long long* acc, long long n, cudaStream_t st) {
    PETCH_CUDA(cudaMemsetAsync(acc, 0, sizeof(long long) * (size_t)n, st), "zero tally accumulators");
    return PETCH_OK;
}

static int acc_convert(const long long* acc, float* out, long long n, cudaStream_t st) {
    k_acc_to_float<<<grid_for(n, 256), 256, 0, st>>>(acc, out, n);
    PETCH_LAUNCH_CHECK("k_acc_to_float");
    return PETCH_OK;
}

#define PETCH_DET_TAKE(var, count)                                                           \
    long long* var = arena.take(count);                                                      \
    PETCH_REQUIRE(var, "deterministic tallies: the registered scratch (%lld bytes) is too small", \
                  g_det_bytes);                                                              \
    do {                                                                                     \
        int _rc = acc_zero(var, count, st);                                                  \
        if (_rc) return _rc;                                                                 \
    } while (0)

#define PETCH_DET_CONVERT(var, out, count)                                                   \
    do {                                                                                     \
        int _rc = acc_convert(var, out, count, st);                                          \
        if (_rc) return _rc;                                                                 \
    } while (0)

extern "C" int petch_set_deterministic(void* scratch, long long scratch_bytes) {
    PETCH_REQUIRE(scratch == nullptr || scratch_bytes >= 256,
                  "petch_set_deterministic: scratch too small");
    g_det_scratch = scratch;
    g_det_bytes = scratch ? scratch_bytes : 0;
    return PETCH_OK;
}

template <class S>
static int launch_trace(const MeshView& m, const Domain& D, const S& sh, uint32_t seed,
                        uint32_t domain, int n, int* work, cudaStream_t st, const char* what,
                        const int* step = nullptr, uint32_t seed_mul = 0, uint32_t seed_off = 0) {
    const TraceCtl c{g_steps, g_keep, g_group, step, seed_mul, seed_off};
    if (g_bvh_width == 2) {
        // binary traversal reads no tree from shared memory: launching without the 12 KB of the
        // wide tree's top leaves the L1 / shared split and the resident blocks to the registers
        k_trace<S, false><<<persistent_blocks((const void*)k_trace<S, false>, kTB, 0), kTB, 0, st>>>(
            m, D, sh, seed, domain, n, c, work);
    } else {
        k_trace<S, true><<<persistent_blocks((const void*)k_trace<S, true>, kTB), kTB, kSmemBytes, st>>>(
            m, D, sh, seed, domain, n, c, work);
    }
    PETCH_LAUNCH_CHECK(what);
    return PETCH_OK;
}

extern "C" int petch_tracer_config(int bvh_width, int steps_per_round, int keep_lanes) {
    PETCH_REQUIRE(bvh_width == 2 || bvh_width == 8, "petch_tracer_config: bvh_width must be 2 or 8");
    PETCH_REQUIRE(steps_per_round >= 1 && steps_per_round <= 4096,
                  "petch_tracer_config: steps_per_round must be in [1, 4096]");
    PETCH_REQUIRE(keep_lanes >= 0 && keep_lanes <= 31,
                  "petch_tracer_config: keep_lanes must be in [0, 31]");
    g_bvh_width = bvh_width;
    g_steps = steps_per_round;
    g_keep = keep_lanes;
    return PETCH_OK;
}

extern "C" int petch_tracer_settings(int* out) {
    PETCH_REQUIRE(out, "petch_tracer_settings: null pointer");
    out[0] = g_bvh_width;
    out[1] = g_steps;
    out[2] = g_keep;
    out[3] = g_tally_agg ? 1 : 0;
    out[4] = g_group;
    return PETCH_OK;
}

extern "C" int petch_tracer_grouping(int group) {
    PETCH_REQUIRE(group == 0 || (group >= 2 && group <= 8),
                  "petch_tracer_grouping: group must be 0 (off) or 2..8");
    g_group = group;
    return PETCH_OK;
}

extern "C" int petch_tally_aggregation(int on) {
    PETCH_REQUIRE(on == 0 || on == 1, "petch_tally_aggregation: on must be 0 or 1");
    g_tally_agg = on != 0;
    return PETCH_OK;
}

namespace petch {

// petch_trace_ions with the seed seed_add + (*step + seed_off) * seed_mul read on the device
// (step NULL: seed_add itself).
int trace_ions_stepped(const void* mesh, int max_tris, int max_verts, const petch_domain* dom,
                       const petch_ion_params* p, const int* step, uint32_t seed_mul,
                       uint32_t seed_off, uint32_t seed_add, int n_ion, float* tally4, float* ang,
                       int* work, void* stream) {
    PETCH_REQUIRE(mesh && dom && p && tally4 && ang && work, "petch_trace_ions: null pointer");
    PETCH_REQUIRE(n_ion >= 0 && max_tris > 0 && max_verts > 0, "petch_trace_ions: bad size");
    PETCH_REQUIRE(((uintptr_t)tally4 & 15) == 0, "petch_trace_ions: tally4 must be 16-byte aligned");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    IonShader sh;
    sh.P = IonP{p->meanE, p->sigmaE, p->A_sp, p->Eth_sp, p->B_sp, p->A_ie, p->Eth_ie, p->A_p,
                p->Eth_p, p->inflect, p->minang, p->n_l, p->A_en, p->minE, p->thrmin, p->thrmax,
                p->sigma};
    sh.tal4 = (float4*)tally4;
    sh.ang = ang;
    sh.det = tally_mode(false);
    k_zero_faces<<<grid_for(4LL * max_tris, 256), 256, 0, st>>>(m.hdr, max_tris, tally4, 4, ang, 1);
    PETCH_LAUNCH_CHECK("k_zero_faces");
    PETCH_CUDA(cudaMemsetAsync(work, 0, sizeof(int), st), "reset ray counter");
    if (n_ion == 0) return PETCH_OK;
    DetArena arena;
    if (!arena.on())
        return launch_trace(m, to_domain(dom), sh, seed_add, 0x696f6e73u, n_ion, work, st,
                            "k_trace<ions>", step, seed_mul, seed_off);
    PETCH_DET_TAKE(a_t, 4LL * max_tris);
    PETCH_DET_TAKE(a_a, (long long)max_tris);
    sh.tal4 = reinterpret_cast<float4*>(a_t);
    sh.ang = reinterpret_cast<float*>(a_a);
    sh.det = tally_mode(true);
    int rc = launch_trace(m, to_domain(dom), sh, seed_add, 0x696f6e73u, n_ion, work, st,
                          "k_trace<ions>", step, seed_mul, seed_off);
    if (rc) return rc;
    PETCH_DET_CONVERT(a_t, tally4, 4LL * max_tris);
    PETCH_DET_CONVERT(a_a, ang, (long long)max_tris);
    return PETCH_OK;
}

}  // namespace petch

extern "C" int petch_trace_ions(const void* mesh, int max_tris, int max_verts,
                                const petch_domain* dom, const petch_ion_params* p, uint32_t seed,
                                int n_ion, float* tally4, float* ang, int* work, void* stream) {
    return petch::trace_ions_stepped(mesh, max_tris, max_verts, dom, p, nullptr, 0, 0, seed, n_ion,
                                     tally4, ang, work, stream);
}

extern "C" int petch_trace_neutrals(const void* mesh, int max_tris, int max_verts,
                                    const petch_domain* dom, const float* bare, float beta,
                                    uint32_t seed, uint32_t stream_id, int n_neu, float* flux,
                                    int* work, void* stream) {
    PETCH_REQUIRE(mesh && dom && flux && work, "petch_trace_neutrals: null pointer");
    PETCH_REQUIRE(n_neu >= 0 && max_tris > 0 && max_verts > 0, "petch_trace_neutrals: bad size");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    NeutralShader sh{bare, beta, flux, tally_mode(false)};
    k_zero_faces<<<grid_for(max_tris, 256), 256, 0, st>>>(m.hdr, max_tris, flux, 1, nullptr, 0);
    PETCH_LAUNCH_CHECK("k_zero_faces");
    PETCH_CUDA(cudaMemsetAsync(work, 0, sizeof(int), st), "reset ray counter");
    if (n_neu == 0) return PETCH_OK;
    DetArena arena;
    if (!arena.on())
        return launch_trace(m, to_domain(dom), sh, seed, 0x6e657500u ^ stream_id, n_neu, work, st,
                            "k_trace<neutrals>");
    PETCH_DET_TAKE(a_f, (long long)max_tris);
    sh.flux = reinterpret_cast<float*>(a_f);
    sh.det = tally_mode(true);
    int rc = launch_trace(m, to_domain(dom), sh, seed, 0x6e657500u ^ stream_id, n_neu, work, st,
                          "k_trace<neutrals>");
    if (rc) return rc;
    PETCH_DET_CONVERT(a_f, flux, (long long)max_tris);
    return PETCH_OK;
}

namespace petch {

// petch_trace_neutral_pair with the seeds seed_add_{a,b} + (*step + seed_off) * seed_mul read on
// the device (step NULL: seed_add_a and seed_add_b themselves).
int trace_neutral_pair_stepped(const void* mesh, int max_tris, int max_verts,
                               const petch_domain* dom, const float* bare, float beta_a,
                               float beta_b, const int* step, uint32_t seed_mul, uint32_t seed_off,
                               uint32_t seed_add_a, uint32_t seed_add_b, uint32_t stream_id,
                               int n_neu, float* flux_a, float* flux_b, int* work, void* stream) {
    PETCH_REQUIRE(mesh && dom && flux_a && flux_b && work, "petch_trace_neutral_pair: null pointer");
    PETCH_REQUIRE(flux_a != flux_b, "petch_trace_neutral_pair: flux_a and flux_b must differ");
    PETCH_REQUIRE(n_neu >= 0 && n_neu < (1 << 30) && max_tris > 0 && max_verts > 0,
                  "petch_trace_neutral_pair: bad size");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    const uint32_t domain = 0x6e657500u ^ stream_id;
    NeutralPairShader sh{bare, beta_a, beta_b, flux_a, flux_b, seed_add_b - seed_add_a, domain,
                         n_neu, tally_mode(false)};
    k_zero_faces<<<grid_for(max_tris, 256), 256, 0, st>>>(m.hdr, max_tris, flux_a, 1, flux_b, 1);
    PETCH_LAUNCH_CHECK("k_zero_faces");
    PETCH_CUDA(cudaMemsetAsync(work, 0, sizeof(int), st), "reset ray counter");
    if (n_neu == 0) return PETCH_OK;
    DetArena arena;
    if (!arena.on())
        return launch_trace(m, to_domain(dom), sh, seed_add_a, domain, 2 * n_neu, work, st,
                            "k_trace<neutral pair>", step, seed_mul, seed_off);
    PETCH_DET_TAKE(a_a, (long long)max_tris);
    PETCH_DET_TAKE(a_b, (long long)max_tris);
    sh.flux_a = reinterpret_cast<float*>(a_a);
    sh.flux_b = reinterpret_cast<float*>(a_b);
    sh.det = tally_mode(true);
    int rc = launch_trace(m, to_domain(dom), sh, seed_add_a, domain, 2 * n_neu, work, st,
                          "k_trace<neutral pair>", step, seed_mul, seed_off);
    if (rc) return rc;
    PETCH_DET_CONVERT(a_a, flux_a, (long long)max_tris);
    PETCH_DET_CONVERT(a_b, flux_b, (long long)max_tris);
    return PETCH_OK;
}

}  // namespace petch

extern "C" int petch_trace_neutral_pair(const void* mesh, int max_tris, int max_verts,
                                        const petch_domain* dom, const float* bare, float beta_a,
                                        float beta_b, uint32_t seed_a, uint32_t seed_b,
                                        uint32_t stream_id, int n_neu, float* flux_a,
                                        float* flux_b, int* work, void* stream) {
    return petch::trace_neutral_pair_stepped(mesh, max_tris, max_verts, dom, bare, beta_a, beta_b,
                                             nullptr, 0, 0, seed_a, seed_b, stream_id, n_neu,
                                             flux_a, flux_b, work, stream);
}

extern "C" int petch_trace_electrons(const void* mesh, int max_tris, int max_verts,
                                     const petch_domain* dom, float sigma, uint32_t seed, int n,
                                     float* flux, int* work, void* stream) {
    PETCH_REQUIRE(mesh && dom && flux && work, "petch_trace_electrons: null pointer");
    PETCH_REQUIRE(n >= 0 && max_tris > 0 && max_verts > 0, "petch_trace_electrons: bad size");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    ElectronShader sh{sigma, flux, tally_mode(false)};
    k_zero_faces<<<grid_for(max_tris, 256), 256, 0, st>>>(m.hdr, max_tris, flux, 1, nullptr, 0);
    PETCH_LAUNCH_CHECK("k_zero_faces");
    PETCH_CUDA(cudaMemsetAsync(work, 0, sizeof(int), st), "reset ray counter");
    if (n == 0) return PETCH_OK;
    DetArena arena;
    if (!arena.on())
        return launch_trace(m, to_domain(dom), sh, seed, 0x656c6563u, n, work, st,
                            "k_trace<electrons>");
    PETCH_DET_TAKE(a_f, (long long)max_tris);
    sh.flux = reinterpret_cast<float*>(a_f);
    sh.det = tally_mode(true);
    int rc = launch_trace(m, to_domain(dom), sh, seed, 0x656c6563u, n, work, st,
                          "k_trace<electrons>");
    if (rc) return rc;
    PETCH_DET_CONVERT(a_f, flux, (long long)max_tris);
    return PETCH_OK;
}

extern "C" int petch_trace_ff(const void* mesh, int max_tris, int max_verts,
                              const petch_domain* dom, const float* fn, uint32_t seed, int n_ff,
                              int* hitface, int* work, void* stream) {
    PETCH_REQUIRE(mesh && dom && fn && hitface && work, "petch_trace_ff: null pointer");
    PETCH_REQUIRE(max_tris > 0 && max_verts > 0 && n_ff >= 1 &&
                      (long long)max_tris * n_ff < (1LL << 31),
                  "petch_trace_ff: max_tris * n_ff must be in [1, 2^31)");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    FormFactorShader sh{fn, n_ff, hitface};
    PETCH_CUDA(cudaMemsetAsync(hitface, 0xff, sizeof(int) * (size_t)max_tris * n_ff, st),
               "hitface = -1");
    PETCH_CUDA(cudaMemsetAsync(work, 0, sizeof(int), st), "reset ray counter");
    return launch_trace(m, to_domain(dom), sh, seed, 0x66666600u, max_tris * n_ff, work, st,
                        "k_trace<form factors>");
}

extern "C" int petch_prepare_device(void) {
    sm_count();
    persistent_blocks((const void*)k_trace_batch<0>, kTB, 0);
    persistent_blocks((const void*)k_trace_batch<1>, kTB, 0);
    persistent_blocks((const void*)k_trace_batch<2>, kTB, 0);
    persistent_blocks((const void*)k_trace_batch<3>, kTB, 0);
    persistent_blocks((const void*)k_trace_batch<4>, kTB, 0);
    persistent_blocks((const void*)k_trace_batch<5>, kTB, 0);
    persistent_blocks((const void*)k_trace<IonShader, false>, kTB, 0);
    persistent_blocks((const void*)k_trace<NeutralShader, false>, kTB, 0);
    persistent_blocks((const void*)k_trace<NeutralPairShader, false>, kTB, 0);
    persistent_blocks((const void*)k_trace<ElectronShader, false>, kTB, 0);
    persistent_blocks((const void*)k_trace<LegacyShader, false>, kTB, 0);
    persistent_blocks((const void*)k_trace<FormFactorShader, false>, kTB, 0);
    persistent_blocks((const void*)k_trace<RedepShader, false>, kTB, 0);
    PETCH_CUDA(cudaGetLastError(), "petch_prepare_device");
    return PETCH_OK;
}

namespace {

template <int KIND>
void launch_batch(const BatchTable& tab, const MeshOffsets& L, int max_tris, int max_verts,
                  float beta, float beta2, const int* step, uint32_t seed_mul, uint32_t seed_add,
                  uint32_t seed_add2, uint32_t domain, int det, int* work, cudaStream_t st) {
    k_trace_batch<KIND><<<persistent_blocks((const void*)k_trace_batch<KIND>, kTB, 0), kTB, 0, st>>>(
        tab, L, max_tris, max_verts, beta, beta2, step, seed_mul, seed_add, seed_add2, domain,
        g_steps, g_keep, g_group, det, work);
}

// kind: 0 ions, 1 neutrals, 2 ions with energy tangents, 3 neutrals with weight tangents,
// 4 both neutral species of a round (the second species' flux in the item's ang), 5 kind 4 with
// weight tangents (the second species' in tans2[b].dout).
int trace_batch(int kind, const petch_batch_item* items, const petch_batch_tangent* tans, int B,
                int max_tris, int max_verts, float beta, float beta2, const int* step,
                uint32_t seed_mul, uint32_t seed_add, uint32_t seed_add2, int* work, void* stream,
                const char* who, const petch_batch_tangent* tans2 = nullptr) {
    PETCH_REQUIRE(items && work, "%s: null pointer", who);
    PETCH_REQUIRE(B >= 1 && B <= kMaxBatch, "%s: 1 <= B <= %d", who, kMaxBatch);
    PETCH_REQUIRE(max_tris > 0 && max_verts > 0, "%s: bad capacities", who);
    const bool ion = kind == 0 || kind == 2, tan = kind == 2 || kind == 3 || kind == 5;
    const bool pair = kind == 4 || kind == 5;
    PETCH_REQUIRE(kind != 5 || tans2, "%s: null second tangent table", who);
    PETCH_REQUIRE(!tan || tans, "%s: null tangent table", who);
    BatchTable tab;
    long long total = 0;
    for (int b = 0; b < B; ++b) {
        const petch_batch_item& x = items[b];
        PETCH_REQUIRE(x.mesh && x.out && x.n_rays >= 0, "%s: item %d incomplete", who, b);
        PETCH_REQUIRE(!ion || (x.ang && ((uintptr_t)x.out & 15) == 0),
                      "%s: ion item %d needs ang and a 16-byte aligned tally", who, b);
        PETCH_REQUIRE(!pair || (x.ang && x.ang != x.out && x.n_rays <= (1 << 29)),
                      "%s: pair item %d needs a second flux (ang) and n_rays <= 2^29", who, b);
        BatchItem& it = tab.it[b];
        it.mesh = (const char*)x.mesh;
        it.D = to_domain(&x.dom);
        const petch_ion_params& p = x.ion;
        it.P = IonP{p.meanE, p.sigmaE, p.A_sp, p.Eth_sp, p.B_sp, p.A_ie, p.Eth_ie, p.A_p, p.Eth_p,
                    p.inflect, p.minang, p.n_l, p.A_en, p.minE, p.thrmin, p.thrmax, p.sigma};
        it.bare = x.bare;
        it.out = x.out;
        it.ang = (ion || pair) ? x.ang : nullptr;
        it.ray_start = (int)total;
        it.seed = x.seed;
        tab.tn[b].dout = nullptr;
        tab.tn[b].dbare = nullptr;
        tab.dout2[b] = nullptr;
        if (tan) {
            PETCH_REQUIRE(tans[b].dout, "%s: tangent item %d has no output", who, b);
            tab.tn[b].dout = tans[b].dout;
            tab.tn[b].dbare = ion ? nullptr : tans[b].dbare;
        }
        if (kind == 5) {
            PETCH_REQUIRE(tans2[b].dout && tans2[b].dout != tans[b].dout,
                          "%s: item %d needs a distinct second tangent output", who, b);
            tab.dout2[b] = tans2[b].dout;
        }
        total += pair ? 2LL * x.n_rays : (long long)x.n_rays;
    }
    PETCH_REQUIRE(total < (1LL << 31), "%s: more than 2^31 - 1 rays", who);
    tab.B = B;
    tab.total = (int)total;
    MeshOffsets L;
    const MeshLayout ml = mesh_layout(max_tris, max_verts);
    for (int i = 0; i < SEG_COUNT; ++i) L.off[i] = ml.off[i];
    cudaStream_t st = as_stream(stream);
    dim3 zg(grid_for(4LL * max_tris, 256, 2), B);
    k_zero_batch<<<zg, 256, 0, st>>>(tab, L, max_tris, max_verts, ion ? 4 : 1, tan ? 1 : 0);
    PETCH_LAUNCH_CHECK("k_zero_batch");
    PETCH_CUDA(cudaMemsetAsync(work, 0, sizeof(int), st), "reset ray counter");
    if (total == 0) return PETCH_OK;
    const uint32_t domain = ion ? 0x696f6e73u : 0x6e657500u;
    DetArena arena;
    const int det = tally_mode(arena.on());
    const bool det_on = det & kTallyDet;
    const long long per_out = (ion ? 4LL : 1LL) * max_tris;
    long long* acc_out[kMaxBatch] = {};
    long long* acc_ang[kMaxBatch] = {};
    long long* acc_d[kMaxBatch] = {};
    long long* acc_d2[kMaxBatch] = {};
    if (det_on) {
        for (int b = 0; b < B; ++b) {
            PETCH_DET_TAKE(ao, per_out);
            acc_out[b] = ao;
            tab.it[b].out = reinterpret_cast<float*>(ao);
            if (ion || pair) {
                PETCH_DET_TAKE(aa, (long long)max_tris);
                acc_ang[b] = aa;
                tab.it[b].ang = reinterpret_cast<float*>(aa);
            }
            if (tan) {
                PETCH_DET_TAKE(ad, 3LL * max_tris);
                acc_d[b] = ad;
                tab.tn[b].dout = reinterpret_cast<float*>(ad);
            }
            if (kind == 5) {
                PETCH_DET_TAKE(ad2, 3LL * max_tris);
                acc_d2[b] = ad2;
                tab.dout2[b] = reinterpret_cast<float*>(ad2);
            }
        }
    }
#define PETCH_LB(K)                                                                            \
    launch_batch<K>(tab, L, max_tris, max_verts, beta, beta2, step, seed_mul, seed_add, seed_add2, \
                    domain, det, work, st)
    switch (kind) {
        case 0: PETCH_LB(0); break;
        case 1: PETCH_LB(1); break;
        case 2: PETCH_LB(2); break;
        case 3: PETCH_LB(3); break;
        case 4: PETCH_LB(4); break;
        default: PETCH_LB(5); break;
    }
#undef PETCH_LB
    PETCH_LAUNCH_CHECK("k_trace_batch");
    if (det_on) {
        for (int b = 0; b < B; ++b) {
            PETCH_DET_CONVERT(acc_out[b], items[b].out, per_out);
            if (ion || pair) PETCH_DET_CONVERT(acc_ang[b], items[b].ang, (long long)max_tris);
            if (tan) PETCH_DET_CONVERT(acc_d[b], tans[b].dout, 3LL * max_tris);
            if (kind == 5) PETCH_DET_CONVERT(acc_d2[b], tans2[b].dout, 3LL * max_tris);
        }
    }
    return PETCH_OK;
}

}  // namespace

extern "C" int petch_trace_batch(int kind, const petch_batch_item* items, int B, int max_tris,
                                 int max_verts, float beta, const int* step, uint32_t seed_mul,
                                 uint32_t seed_add, int* work, void* stream) {
    PETCH_REQUIRE(kind == 0 || kind == 1, "petch_trace_batch: kind must be 0 (ions) or 1 (neutrals)");
    return trace_batch(kind, items, nullptr, B, max_tris, max_verts, beta, beta, step, seed_mul,
                       seed_add, seed_add, work, stream, "petch_trace_batch");
}

extern "C" int petch_trace_batch_pair(const petch_batch_item* items, int B, int max_tris,
                                      int max_verts, float beta_a, float beta_b, const int* step,
                                      uint32_t seed_mul, uint32_t seed_add_a, uint32_t seed_add_b,
                                      int* work, void* stream) {
    return trace_batch(4, items, nullptr, B, max_tris, max_verts, beta_a, beta_b, step, seed_mul,
                       seed_add_a, seed_add_b, work, stream, "petch_trace_batch_pair");
}

extern "C" int petch_trace_batch_tangent(int kind, const petch_batch_item* items,
                                         const petch_batch_tangent* tans, int B, int max_tris,
                                         int max_verts, float beta, const int* step,
                                         uint32_t seed_mul, uint32_t seed_add, int* work,
                                         void* stream) {
    PETCH_REQUIRE(kind == 0 || kind == 1,
                  "petch_trace_batch_tangent: kind must be 0 (ions) or 1 (neutrals)");
    return trace_batch(kind + 2, items, tans, B, max_tris, max_verts, beta, beta, step, seed_mul,
                       seed_add, seed_add, work, stream, "petch_trace_batch_tangent");
}

extern "C" int petch_trace_batch_pair_tangent(const petch_batch_item* items,
                                              const petch_batch_tangent* tans_a,
                                              const petch_batch_tangent* tans_b, int B,
                                              int max_tris, int max_verts, float beta_a,
                                              float beta_b, const int* step, uint32_t seed_mul,
                                              uint32_t seed_add_a, uint32_t seed_add_b, int* work,
                                              void* stream) {
    return trace_batch(5, items, tans_a, B, max_tris, max_verts, beta_a, beta_b, step, seed_mul,
                       seed_add_a, seed_add_b, work, stream, "petch_trace_batch_pair_tangent",
                       tans_b);
}

extern "C" int petch_redep_scratch_bytes(int max_tris, long long* bytes) {
    PETCH_REQUIRE(bytes && max_tris > 0, "petch_redep_scratch_bytes: bad argument");
    size_t b = 0;
    PETCH_CUDA(cub::DeviceScan::InclusiveSum(nullptr, b, (double*)nullptr, (double*)nullptr,
                                             max_tris),
               "petch_redep_scratch_bytes: scan size query");
    *bytes = (long long)b;
    return PETCH_OK;
}

extern "C" int petch_trace_redep(const void* mesh, int max_tris, int max_verts,
                                 const petch_domain* dom, const float* fn, const float* V,
                                 float s_redep, uint32_t seed, int n, float* flux, double* cdf,
                                 void* scratch, long long scratch_bytes, int* work, void* stream) {
    PETCH_REQUIRE(mesh && dom && fn && V && flux && cdf && scratch && work,
                  "petch_trace_redep: null pointer");
    PETCH_REQUIRE(n >= 0 && max_tris > 0 && max_verts > 0, "petch_trace_redep: bad size");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    k_redep_weights<<<grid_for(max_tris, 256), 256, 0, st>>>(m, V, cdf);
    PETCH_LAUNCH_CHECK("k_redep_weights");
    size_t b = (size_t)scratch_bytes;
    PETCH_CUDA(cub::DeviceScan::InclusiveSum(scratch, b, cdf, cdf, max_tris, st), "redep cdf scan");
    k_zero_faces<<<grid_for(max_tris, 256), 256, 0, st>>>(m.hdr, max_tris, flux, 1, nullptr, 0);
    PETCH_LAUNCH_CHECK("k_zero_faces");
    PETCH_CUDA(cudaMemsetAsync(work, 0, sizeof(int), st), "reset ray counter");
    if (n == 0) return PETCH_OK;
    RedepShader sh;
    sh.rr = NeutralShader{nullptr, s_redep, flux, tally_mode(false)};
    sh.cdf = cdf;
    sh.fn = fn;
    Domain D = to_domain(dom);
    D.periodic = 0;                      // mc_redep_3d traces without the lateral wrap
    DetArena arena;
    if (!arena.on())
        return launch_trace(m, D, sh, seed, 0x72656470u, n, work, st, "k_trace<redeposition>");
    PETCH_DET_TAKE(a_f, (long long)max_tris);
    sh.rr.flux = reinterpret_cast<float*>(a_f);
    sh.rr.det = tally_mode(true);
    int rc = launch_trace(m, D, sh, seed, 0x72656470u, n, work, st, "k_trace<redeposition>");
    if (rc) return rc;
    PETCH_DET_CONVERT(a_f, flux, (long long)max_tris);
    return PETCH_OK;
}

extern "C" int petch_redep_apply(const void* mesh, int max_tris, int max_verts, const float* flux,
                                 const double* cdf, int n, float k_redep, float* V, float* Rf,
                                 int* stats, void* stream) {
    PETCH_REQUIRE(mesh && flux && cdf && V, "petch_redep_apply: null pointer");
    PETCH_REQUIRE(n >= 0 && max_tris > 0, "petch_redep_apply: bad size");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    if (stats) PETCH_CUDA(cudaMemsetAsync(stats + 1, 0, sizeof(int), st), "reset max V");
    k_redep_apply<<<grid_for(max_tris, 256), 256, 0, st>>>(m, flux, cdf, n, k_redep, V, Rf, stats);
    PETCH_LAUNCH_CHECK("k_redep_apply");
    return PETCH_OK;
}

extern "C" int petch_trace_ions_tangent(const void* mesh, int max_tris, int max_verts,
                                        const petch_domain* dom, const petch_ion_params* p,
                                        uint32_t seed, int n_ion, float* tally4, float* ang,
                                        float* dtal, int* work, void* stream) {
    PETCH_REQUIRE(mesh && dom && p && tally4 && ang && dtal && work,
                  "petch_trace_ions_tangent: null pointer");
    PETCH_REQUIRE(n_ion >= 0 && max_tris > 0 && max_verts > 0, "petch_trace_ions_tangent: bad size");
    PETCH_REQUIRE(((uintptr_t)tally4 & 15) == 0, "petch_trace_ions_tangent: tally4 alignment");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    IonTanShader sh;
    sh.P = IonP{p->meanE, p->sigmaE, p->A_sp, p->Eth_sp, p->B_sp, p->A_ie, p->Eth_ie, p->A_p,
                p->Eth_p, p->inflect, p->minang, p->n_l, p->A_en, p->minE, p->thrmin, p->thrmax,
                p->sigma};
    sh.tal4 = (float4*)tally4;
    sh.ang = ang;
    sh.dtal = dtal;
    sh.det = tally_mode(false);
    k_zero_faces<<<grid_for(4LL * max_tris, 256), 256, 0, st>>>(m.hdr, max_tris, tally4, 4, ang, 1);
    PETCH_LAUNCH_CHECK("k_zero_faces");
    PETCH_CUDA(cudaMemsetAsync(dtal, 0, sizeof(float) * 3 * (size_t)max_tris, st), "zero dtal");
    PETCH_CUDA(cudaMemsetAsync(work, 0, sizeof(int), st), "reset ray counter");
    if (n_ion == 0) return PETCH_OK;
    DetArena arena;
    if (!arena.on())
        return launch_trace(m, to_domain(dom), sh, seed, 0x696f6e73u, n_ion, work, st,
                            "k_trace<ions, tangent>");
    PETCH_DET_TAKE(a_t, 4LL * max_tris);
    PETCH_DET_TAKE(a_a, (long long)max_tris);
    PETCH_DET_TAKE(a_d, 3LL * max_tris);
    sh.tal4 = reinterpret_cast<float4*>(a_t);
    sh.ang = reinterpret_cast<float*>(a_a);
    sh.dtal = reinterpret_cast<float*>(a_d);
    sh.det = tally_mode(true);
    int rc = launch_trace(m, to_domain(dom), sh, seed, 0x696f6e73u, n_ion, work, st,
                          "k_trace<ions, tangent>");
    if (rc) return rc;
    PETCH_DET_CONVERT(a_t, tally4, 4LL * max_tris);
    PETCH_DET_CONVERT(a_a, ang, (long long)max_tris);
    PETCH_DET_CONVERT(a_d, dtal, 3LL * max_tris);
    return PETCH_OK;
}

extern "C" int petch_trace_neutral_pair_tangent(const void* mesh, int max_tris, int max_verts,
                                                const petch_domain* dom, const float* bare,
                                                const float* dbare, float beta_a, float beta_b,
                                                uint32_t seed_a, uint32_t seed_b,
                                                uint32_t stream_id, int n_neu, float* flux_a,
                                                float* dflux_a, float* flux_b, float* dflux_b,
                                                int* work, void* stream) {
    PETCH_REQUIRE(mesh && dom && flux_a && dflux_a && flux_b && dflux_b && work,
                  "petch_trace_neutral_pair_tangent: null pointer");
    PETCH_REQUIRE(flux_a != flux_b && dflux_a != dflux_b,
                  "petch_trace_neutral_pair_tangent: the two species' outputs must differ");
    PETCH_REQUIRE(n_neu >= 0 && n_neu < (1 << 30) && max_tris > 0 && max_verts > 0,
                  "petch_trace_neutral_pair_tangent: bad size");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    const uint32_t domain = 0x6e657500u ^ stream_id;
    NeutralTanPairShader sh{bare, dbare, beta_a, beta_b, flux_a, dflux_a, flux_b, dflux_b,
                            seed_b - seed_a, domain, n_neu, tally_mode(false)};
    k_zero_faces<<<grid_for(max_tris, 256), 256, 0, st>>>(m.hdr, max_tris, flux_a, 1, flux_b, 1);
    PETCH_LAUNCH_CHECK("k_zero_faces");
    PETCH_CUDA(cudaMemsetAsync(dflux_a, 0, sizeof(float) * 3 * (size_t)max_tris, st), "zero dflux");
    PETCH_CUDA(cudaMemsetAsync(dflux_b, 0, sizeof(float) * 3 * (size_t)max_tris, st), "zero dflux");
    PETCH_CUDA(cudaMemsetAsync(work, 0, sizeof(int), st), "reset ray counter");
    if (n_neu == 0) return PETCH_OK;
    DetArena arena;
    if (!arena.on())
        return launch_trace(m, to_domain(dom), sh, seed_a, domain, 2 * n_neu, work, st,
                            "k_trace<neutral pair, tangent>");
    PETCH_DET_TAKE(a_fa, (long long)max_tris);
    PETCH_DET_TAKE(a_da, 3LL * max_tris);
    PETCH_DET_TAKE(a_fb, (long long)max_tris);
    PETCH_DET_TAKE(a_db, 3LL * max_tris);
    sh.flux_a = reinterpret_cast<float*>(a_fa);
    sh.dflux_a = reinterpret_cast<float*>(a_da);
    sh.flux_b = reinterpret_cast<float*>(a_fb);
    sh.dflux_b = reinterpret_cast<float*>(a_db);
    sh.det = tally_mode(true);
    int rc = launch_trace(m, to_domain(dom), sh, seed_a, domain, 2 * n_neu, work, st,
                          "k_trace<neutral pair, tangent>");
    if (rc) return rc;
    PETCH_DET_CONVERT(a_fa, flux_a, (long long)max_tris);
    PETCH_DET_CONVERT(a_da, dflux_a, 3LL * max_tris);
    PETCH_DET_CONVERT(a_fb, flux_b, (long long)max_tris);
    PETCH_DET_CONVERT(a_db, dflux_b, 3LL * max_tris);
    return PETCH_OK;
}

extern "C" int petch_trace_neutrals_tangent(const void* mesh, int max_tris, int max_verts,
                                            const petch_domain* dom, const float* bare,
                                            const float* dbare, float beta, uint32_t seed,
                                            uint32_t stream_id, int n_neu, float* flux,
                                            float* dflux, int* work, void* stream) {
    PETCH_REQUIRE(mesh && dom && flux && dflux && work, "petch_trace_neutrals_tangent: null pointer");
    PETCH_REQUIRE(n_neu >= 0 && max_tris > 0 && max_verts > 0,
                  "petch_trace_neutrals_tangent: bad size");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    NeutralTanShader sh{bare, dbare, beta, flux, dflux, tally_mode(false)};
    k_zero_faces<<<grid_for(max_tris, 256), 256, 0, st>>>(m.hdr, max_tris, flux, 1, nullptr, 0);
    PETCH_LAUNCH_CHECK("k_zero_faces");
    PETCH_CUDA(cudaMemsetAsync(dflux, 0, sizeof(float) * 3 * (size_t)max_tris, st), "zero dflux");
    PETCH_CUDA(cudaMemsetAsync(work, 0, sizeof(int), st), "reset ray counter");
    if (n_neu == 0) return PETCH_OK;
    DetArena arena;
    if (!arena.on())
        return launch_trace(m, to_domain(dom), sh, seed, 0x6e657500u ^ stream_id, n_neu, work, st,
                            "k_trace<neutrals, tangent>");
    PETCH_DET_TAKE(a_f, (long long)max_tris);
    PETCH_DET_TAKE(a_d, 3LL * max_tris);
    sh.flux = reinterpret_cast<float*>(a_f);
    sh.dflux = reinterpret_cast<float*>(a_d);
    sh.det = tally_mode(true);
    int rc = launch_trace(m, to_domain(dom), sh, seed, 0x6e657500u ^ stream_id, n_neu, work, st,
                          "k_trace<neutrals, tangent>");
    if (rc) return rc;
    PETCH_DET_CONVERT(a_f, flux, (long long)max_tris);
    PETCH_DET_CONVERT(a_d, dflux, 3LL * max_tris);
    return PETCH_OK;
}

extern "C" int petch_trace_legacy(const void* mesh, int max_tris, int max_verts,
                                  const petch_domain* dom, int ion, float sigma, float sticking,
                                  int n_reemit, int specular, float cos_thr, float eta,
                                  uint32_t seed, int n, float* flux, float* angacc, int* work,
                                  void* stream) {
    PETCH_REQUIRE(mesh && dom && flux && angacc && work, "petch_trace_legacy: null pointer");
    PETCH_REQUIRE(n >= 0 && n_reemit >= 0 && max_tris > 0 && max_verts > 0,
                  "petch_trace_legacy: bad size");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    LegacyShader sh{ion, n_reemit, specular, sigma, sticking, cos_thr, eta, flux, angacc,
                    tally_mode(false)};
    k_zero_faces<<<grid_for(max_tris, 256), 256, 0, st>>>(m.hdr, max_tris, flux, 1, angacc, 1);
    PETCH_LAUNCH_CHECK("k_zero_faces");
    PETCH_CUDA(cudaMemsetAsync(work, 0, sizeof(int), st), "reset ray counter");
    if (n == 0) return PETCH_OK;
    Domain D = to_domain(dom);
    D.periodic = 0;
    DetArena arena;
    if (!arena.on())
        return launch_trace(m, D, sh, seed, ion ? 0x6c696f6eu : 0x6c6e6575u, n, work, st,
                            "k_trace<legacy>");
    PETCH_DET_TAKE(a_f, (long long)max_tris);
    PETCH_DET_TAKE(a_a, (long long)max_tris);
    sh.flux = reinterpret_cast<float*>(a_f);
    sh.angacc = reinterpret_cast<float*>(a_a);
    sh.det = tally_mode(true);
    int rc = launch_trace(m, D, sh, seed, ion ? 0x6c696f6eu : 0x6c6e6575u, n, work, st,
                          "k_trace<legacy>");
    if (rc) return rc;
    PETCH_DET_CONVERT(a_f, flux, (long long)max_tris);
    PETCH_DET_CONVERT(a_a, angacc, (long long)max_tris);
    return PETCH_OK;
}

static int extend_velocity(const void* mesh, int max_tris, int max_verts, const float* phi,
                           const uint8_t* mask, int nx, int ny, int nz, double dx, double band,
                           const float* V, float* Fs, int fold_mask, int* active, int* n_active,
                           int max_active, int* work, void* stream, bool centroid,
                           const float* dV = nullptr, float* dF = nullptr) {
    PETCH_REQUIRE(mesh && phi && V && Fs && work, "petch_extend_velocity: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && dx > 0, "petch_extend_velocity: bad grid");
    PETCH_REQUIRE(!fold_mask || !active || n_active, "petch_extend_velocity: n_active is null");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    GridArgs G{nx, ny, nz, (long long)ny * nz, (long long)nx * ny * nz, dx, band};
    if (fold_mask && active) PETCH_CUDA(cudaMemsetAsync(n_active, 0, sizeof(int), st), "memset n_active");
    if (centroid) {
        k_extend<true><<<grid_for(G.n, kTB, 16), kTB, 0, st>>>(m, G, phi, mask, V, Fs, fold_mask,
                                                               active, n_active, max_active, work);
    } else {
        k_extend<false><<<grid_for(G.n, kTB, 16), kTB, 0, st>>>(m, G, phi, mask, V, Fs, fold_mask,
                                                                active, n_active, max_active, work,
                                                                dV, dF);
    }
    PETCH_LAUNCH_CHECK("k_extend");
    return PETCH_OK;
}

extern "C" int petch_extend_velocity(const void* mesh, int max_tris, int max_verts,
                                     const float* phi, const uint8_t* mask, int nx, int ny, int nz,
                                     double dx, double band, const float* V, float* Fs, int fold_mask,
                                     int* active, int* n_active, int max_active, int* work,
                                     void* stream) {
    return extend_velocity(mesh, max_tris, max_verts, phi, mask, nx, ny, nz, dx, band, V, Fs,
                           fold_mask, active, n_active, max_active, work, stream, false);
}

extern "C" int petch_extend_velocity_dual(const void* mesh, int max_tris, int max_verts,
                                          const float* phi, const uint8_t* mask, int nx, int ny,
                                          int nz, double dx, double band, const float* V,
                                          const float* dV, float* Fs, float* dF, int fold_mask,
                                          int* active, int* n_active, int max_active, int* work,
                                          void* stream) {
    PETCH_REQUIRE(dV && dF, "petch_extend_velocity_dual: null pointer");
    return extend_velocity(mesh, max_tris, max_verts, phi, mask, nx, ny, nz, dx, band, V, Fs,
                           fold_mask, active, n_active, max_active, work, stream, false, dV, dF);
}

extern "C" int petch_extend_velocity_centroid(const void* mesh, int max_tris, int max_verts,
                                              const float* phi, const uint8_t* mask, int nx,
                                              int ny, int nz, double dx, double band,
                                              const float* V, float* Fs, int fold_mask,
                                              int* active, int* n_active, int max_active,
                                              int* work, void* stream) {
    return extend_velocity(mesh, max_tris, max_verts, phi, mask, nx, ny, nz, dx, band, V, Fs,
                           fold_mask, active, n_active, max_active, work, stream, true);
}

extern "C" int petch_warmstart(const void* prev_mesh, int prev_max_tris, int prev_max_verts,
                               const float* prev_bare, const void* mesh, int max_tris,
                               int max_verts, float* bare, int* work, void* stream) {
    PETCH_REQUIRE(prev_mesh && prev_bare && mesh && bare && work, "petch_warmstart: null pointer");
    cudaStream_t st = as_stream(stream);
    MeshView pm = mesh_view(const_cast<void*>(prev_mesh), prev_max_tris, prev_max_verts);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    k_warmstart<<<grid_for(max_tris, kTB), kTB, 0, st>>>(pm, prev_bare, m, bare, work);
    PETCH_LAUNCH_CHECK("k_warmstart");
    return PETCH_OK;
}

extern "C" int petch_warmstart_dual(const void* prev_mesh, int prev_max_tris, int prev_max_verts,
                                    const float* prev_bare, const float* prev_dbare,
                                    const void* mesh, int max_tris, int max_verts, float* bare,
                                    float* dbare, int* work, void* stream) {
    PETCH_REQUIRE(prev_mesh && prev_bare && prev_dbare && mesh && bare && dbare && work,
                  "petch_warmstart_dual: null pointer");
    cudaStream_t st = as_stream(stream);
    MeshView pm = mesh_view(const_cast<void*>(prev_mesh), prev_max_tris, prev_max_verts);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    k_warmstart<<<grid_for(max_tris, kTB), kTB, 0, st>>>(pm, prev_bare, m, bare, work, prev_dbare,
                                                        dbare);
    PETCH_LAUNCH_CHECK("k_warmstart");
    return PETCH_OK;
}

extern "C" int petch_raycast(const void* mesh, int max_tris, int max_verts, const float* o,
                             const float* d, int n, float tmax, int* face, float* t, int* work,
                             void* stream) {
    PETCH_REQUIRE(mesh && (n == 0 || (o && d && face && t)) && work, "petch_raycast: null pointer");
    PETCH_REQUIRE(n >= 0, "petch_raycast: n must be >= 0");
    if (n == 0) return PETCH_OK;
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    k_raycast<<<grid_for(n, kTB, 16), kTB, kSmemBytes, as_stream(stream)>>>(m, o, d, n, tmax, face, t, work,
                                                                          g_bvh_width != 2);
    PETCH_LAUNCH_CHECK("k_raycast");
    return PETCH_OK;
}

extern "C" int petch_nearest_face(const void* mesh, int max_tris, int max_verts, const float* p,
                                  int n, float max_dist, int* face, int* work, void* stream) {
    PETCH_REQUIRE(mesh && (n == 0 || (p && face)) && work, "petch_nearest_face: null pointer");
    PETCH_REQUIRE(n >= 0, "petch_nearest_face: n must be >= 0");
    if (n == 0) return PETCH_OK;
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    k_nearest<<<grid_for(n, kTB, 16), kTB, 0, as_stream(stream)>>>(m, p, n, max_dist * max_dist,
                                                                    face, work);
    PETCH_LAUNCH_CHECK("k_nearest");
    return PETCH_OK;
}
