// Device-side ray machinery shared by the flux kernels: Philox4x32-10 streams, the watertight
// ray/triangle test, closest-hit and nearest-face BVH queries over a MeshView.
#pragma once
#include <cstdint>
#include "mesh.cuh"

namespace petch {

// ---------------------------------------------------------------------------------------------
// Counter-based RNG: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  A ray's stream is keyed
// by (seed, domain) and counted by (ray id, call index), so any path can be replayed exactly.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k.x += 0x9E3779B9u;
            k.y += 0xBB67AE85u;
        }
        uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    return c;
}

struct Rng {
    uint4 buf;
    uint2 key;
    uint32_t ray, n;
    int left;
    float spare;
    bool has_spare;

    __device__ __forceinline__ void init(uint32_t seed, uint32_t domain, uint32_t ray_id) {
        key = make_uint2(seed, domain);
        ray = ray_id;
        n = 0;
        left = 0;
        has_spare = false;
    }
    __device__ __forceinline__ uint32_t next_u32() {
        if (left == 0) {
            buf = philox4x32_10(make_uint4(ray, n++, 0x70657463u, 0u), key);
            left = 4;
        }
        uint32_t x = buf.x;
        buf.x = buf.y;
        buf.y = buf.z;
        buf.z = buf.w;
        --left;
        return x;
    }
    // uniform in [0, 1)
    __device__ __forceinline__ float uniform() { return (float)(next_u32() >> 8) * (1.0f / 16777216.0f); }
    // standard normal (Box-Muller, both outputs used)
    __device__ __forceinline__ float normal() {
        if (has_spare) {
            has_spare = false;
            return spare;
        }
        float u1 = 1.0f - uniform();   // (0, 1]
        float u2 = uniform();
        float r = sqrtf(-2.0f * logf(u1));
        float s, c;
        sincosf(6.28318530718f * u2, &s, &c);
        spare = r * s;
        has_spare = true;
        return r * c;
    }
};

// ---------------------------------------------------------------------------------------------
// small vector helpers
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalize3(float3 a) {
    float l = sqrtf(dot3(a, a));
    return l > 0.0f ? (1.0f / l) * a : make_float3(0.0f, 0.0f, 0.0f);
}
__device__ __forceinline__ float comp(float3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

// ---------------------------------------------------------------------------------------------
// Ray setup for the watertight test (Woop, Benthin, Wald, JCGT 2013) and the slab test.
// ---------------------------------------------------------------------------------------------
struct Ray {
    float3 o, d, inv;
    int kx, ky, kz;
    float Sx, Sy, Sz;
};

__device__ __forceinline__ float safe_inv(float x) {
    const float eps = 1.0e-20f;
    return 1.0f / (fabsf(x) > eps ? x : copysignf(eps, x));
}

__device__ __forceinline__ Ray make_ray(float3 o, float3 d) {
    Ray r;
    r.o = o;
    r.d = d;
    r.inv = make_float3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    if (comp(d, kz) < 0.0f) {
        int t = kx;
        kx = ky;
        ky = t;
    }
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    float dz = comp(d, kz);
    r.Sx = comp(d, kx) / dz;
    r.Sy = comp(d, ky) / dz;
    r.Sz = 1.0f / dz;
    return r;
}

// Watertight ray/triangle intersection; on a hit with 0 <= t < tbest, sets tbest and returns
// true.  Edge functions that round to zero are recomputed in double (as the paper prescribes).
__device__ __forceinline__ bool hit_triangle(const Ray& r, float3 a, float3 b, float3 c,
                                             float& tbest) {
    float3 A = a - r.o, B = b - r.o, C = c - r.o;
    float Az = comp(A, r.kz), Bz = comp(B, r.kz), Cz = comp(C, r.kz);
    float Ax = comp(A, r.kx) - r.Sx * Az, Ay = comp(A, r.ky) - r.Sy * Az;
    float Bx = comp(B, r.kx) - r.Sx * Bz, By = comp(B, r.ky) - r.Sy * Bz;
    float Cx = comp(C, r.kx) - r.Sx * Cz, Cy = comp(C, r.ky) - r.Sy * Cz;
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = U + V + W;
    if (det == 0.0f) return false;
    Az *= r.Sz;
    Bz *= r.Sz;
    Cz *= r.Sz;
    float T = U * Az + V * Bz + W * Cz;
    if (det < 0.0f) {
        T = -T;
        det = -det;
    }
    if (T < 0.0f || T >= tbest * det) return false;
    tbest = T / det;
    return true;
}

__device__ __forceinline__ bool slab(const Ray& r, float lx, float hx, float ly, float hy, float lz,
                                     float hz, float tmax, float& tnear) {
    float tx0 = (lx - r.o.x) * r.inv.x, tx1 = (hx - r.o.x) * r.inv.x;
    float ty0 = (ly - r.o.y) * r.inv.y, ty1 = (hy - r.o.y) * r.inv.y;
    float tz0 = (lz - r.o.z) * r.inv.z, tz1 = (hz - r.o.z) * r.inv.z;
    float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
    float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    tnear = tn;
    return tn <= tf;
}

constexpr int kStack = 64;
constexpr int kMaxVisits = 1 << 16;   // node + leaf visits per query (bounded loop)

struct HitRec {
    float t;
    int f;
};

__device__ __forceinline__ float3 tri_v(const float4* tri, int f, int v) {
    float4 p = __ldg(tri + 3 * f + v);
    return make_float3(p.x, p.y, p.z);
}

// Closest hit with 0 <= t < tmax.  Returns f = -1 on a miss.  *err gets bit 1 if the visit
// bound or the stack depth was exceeded (the query then reports what it found so far).
__device__ __forceinline__ HitRec closest_hit(const MeshView& m, int L, const Ray& r, float tmax,
                                              int* err) {
    HitRec h{tmax, -1};
    if (L <= 0) return h;
    int stack[kStack];
    int sp = 0;
    int node = (L == 1) ? ~0 : 0;
    for (int visits = 0; visits < kMaxVisits; ++visits) {
        if (node >= 0) {
            const float4* n = m.nodes + 4 * node;
            float4 n0 = __ldg(n), n1 = __ldg(n + 1), n2 = __ldg(n + 2), n3 = __ldg(n + 3);
            float t0, t1;
            bool h0 = slab(r, n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, h.t, t0);
            bool h1 = slab(r, n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, h.t, t1);
            int c0 = __float_as_int(n3.x), c1 = __float_as_int(n3.y);
            if (h0 && h1) {
                int nearc = c0, farc = c1;
                if (t1 < t0) {
                    nearc = c1;
                    farc = c0;
                }
                if (sp < kStack) stack[sp++] = farc;
                else *err |= 1;
                node = nearc;
                continue;
            }
            if (h0) { node = c0; continue; }
            if (h1) { node = c1; continue; }
        } else {
            int l = ~node;
            int f0 = __ldg(m.leaf_start + l), f1 = min(__ldg(m.leaf_start + l + 1), m.MT);
            for (int f = f0; f < f1; ++f)
                if (hit_triangle(r, tri_v(m.tri, f, 0), tri_v(m.tri, f, 1), tri_v(m.tri, f, 2), h.t))
                    h.f = f;
        }
        if (sp == 0) return h;
        node = stack[--sp];
    }
    *err |= 1;
    return h;
}

// ---------------------------------------------------------------------------------------------
// Resumable closest-hit queries.  A Query advances one BVH node or one leaf per step, so a warp
// can run a bounded number of steps for all its lanes, shade the lanes whose query finished and
// start new queries, instead of waiting for its slowest lane's whole traversal.
//
// Two acceleration structures share the interface:
//  * 8-wide quantised BVH (WIDE): children tested together, sorted by entry distance with a fixed
//    19-comparator network in registers; the nearest is visited next, the others pushed
//    far-to-near with their entry distance (entries beyond the current hit are popped without a
//    fetch); the first `nsm` nodes (the top levels, BFS order) come from shared memory.
//  * binary LBVH: both child boxes per node (64 B), near child first.
// Box planes are decoded in space (p + q * s) before the ray offset is taken, so the slab test
// keeps the sign of (plane - origin) for rays nearly parallel to a plane.
// ---------------------------------------------------------------------------------------------
constexpr int kWStack = 48;
constexpr int kSmemNodes = 128;   // 12 KB of the tree top per block
constexpr int kDone = -2147483647 - 1;

struct Tracer {
    MeshView m;
    int WN;                    // wide nodes
    int L;                     // binary leaves
    const float4* snodes;      // shared-memory copy of wide nodes [0, nsm)
    int nsm;
};

struct Query {
    Ray r;
    float t;    // closest hit so far
    int f;      // its face, -1 if none
    int cur;    // current node ref (kDone when finished)
    int sp;     // stack depth
    int visits;
};

__device__ __forceinline__ void query_begin(Query& q, const Tracer& T, float3 o, float3 d,
                                            float tmax, bool wide) {
    q.r = make_ray(o, d);
    q.t = tmax;
    q.f = -1;
    q.sp = 0;
    q.visits = 0;
    if (wide) q.cur = T.WN > 0 ? 0 : kDone;
    else q.cur = T.L <= 0 ? kDone : (T.L == 1 ? leaf_ref(T.m, 0) : 0);
}

__device__ __forceinline__ void cas(float& ka, int& va, float& kb, int& vb) {
    bool sw = kb < ka;
    float tk = sw ? kb : ka;
    int tv = sw ? vb : va;
    kb = sw ? ka : kb;
    vb = sw ? va : vb;
    ka = tk;
    va = tv;
}

__device__ __forceinline__ float qbyte(uint32_t lo4, uint32_t hi4, int k) {
    uint32_t w = (k < 4) ? lo4 : hi4;
    return (float)((w >> (8 * (k & 3))) & 255u);
}

// Traversal stack: (node ref, entry distance) pairs in the lane's local memory, at most kWStack
// deep (deeper pushes set error bit 1).  pop() takes the nearest stacked entry that can still
// beat the current hit (entries beyond it are dropped without a fetch); false if none is left.
// (Variants measured on the trench workload: the top 4 or 8 entries in shared memory, 2-4 %
// slower, since its shared memory comes out of the L1 that caches the tree; node references
// only, each popped entry culled by its own box tests instead of its stored distance, 4.5 %
// slower.)
#ifndef PETCH_STACK_PACKED
#define PETCH_STACK_PACKED 1
#endif
struct LocalStack {
#if PETCH_STACK_PACKED
    int2 e[kWStack];          // (ref, entry distance bits): one 8-byte access per push / pop
    __device__ __forceinline__ void push(Query& q, int r, float tt, int* err) {
        if (q.sp < kWStack) {
            e[q.sp] = make_int2(r, __float_as_int(tt));
            ++q.sp;
        } else {
            *err |= 1;
        }
    }
    __device__ __forceinline__ bool pop(Query& q) {
        while (q.sp > 0) {
            --q.sp;
            const int2 x = e[q.sp];
            if (__int_as_float(x.y) <= q.t) {
                q.cur = x.x;
                return true;
            }
        }
        q.cur = kDone;
        return false;
    }
#else
    int ref[kWStack];
    float t[kWStack];
    __device__ __forceinline__ void push(Query& q, int r, float tt, int* err) {
        if (q.sp < kWStack) {
            ref[q.sp] = r;
            t[q.sp] = tt;
            ++q.sp;
        } else {
            *err |= 1;
        }
    }
    __device__ __forceinline__ bool pop(Query& q) {
        while (q.sp > 0) {
            --q.sp;
            if (t[q.sp] <= q.t) {
                q.cur = ref[q.sp];
                return true;
            }
        }
        q.cur = kDone;
        return false;
    }
#endif
};


// Faces f0 .. f1 - 1 of one leaf; a face index is never taken past the buffer's capacity.
__device__ __forceinline__ void query_leaf(const Tracer& T, Query& q, int f0, int f1) {
    f1 = min(f1, T.m.MT);
    for (int f = f0; f < f1; ++f)
        if (hit_triangle(q.r, tri_v(T.m.tri, f, 0), tri_v(T.m.tri, f, 1), tri_v(T.m.tri, f, 2), q.t))
            q.f = f;
}

// Leaf step of either tree: q.cur = -(start * 8 + count) - 1 (leaf_ref); all the leaf's faces in
// ascending order.  (Capping a step at 1, 2 or 3 triangles, the rest left in q.cur for the next
// step so a warp's leaf lanes test similar counts, measured 8 %, 3.5 % and 2 % slower on the
// trench workload: the extra steps cost more than the divergence they remove.)
template <class St>
__device__ __forceinline__ bool step_leaf(const Tracer& T, Query& q, St& st) {
    const int code = -q.cur - 1;
    const int f0 = code >> 3;
    query_leaf(T, q, f0, f0 + (code & 7));
    return !st.pop(q);
}

// One step of the 8-wide traversal; returns true once the query has finished.  The internal-node
// and leaf halves are also callable on their own, as the binary traversal's (leaf grouping).
template <class St>
__device__ __forceinline__ bool step_wide_node(const Tracer& T, Query& q, St& st, int* err) {
    const int cur = q.cur;
    {
        float4 v0, v1, v2, v3, v4, v5;
        if (cur < T.nsm) {
            const float4* p = T.snodes + 6 * cur;
            v0 = p[0]; v1 = p[1]; v2 = p[2]; v3 = p[3]; v4 = p[4]; v5 = p[5];
        } else {
            const float4* p = reinterpret_cast<const float4*>(T.m.wnodes) + 6 * (long long)cur;
            v0 = __ldg(p); v1 = __ldg(p + 1); v2 = __ldg(p + 2);
            v3 = __ldg(p + 3); v4 = __ldg(p + 4); v5 = __ldg(p + 5);
        }
        const Ray& r = q.r;
        uint32_t meta = __float_as_uint(v0.w);
        float sx = __int_as_float((int)((meta & 255u) << 23));
        float sy = __int_as_float((int)(((meta >> 8) & 255u) << 23));
        float sz = __int_as_float((int)(((meta >> 16) & 255u) << 23));
        int nc = (int)(meta >> 24);
        int ch[8] = {__float_as_int(v4.x), __float_as_int(v4.y), __float_as_int(v4.z),
                     __float_as_int(v4.w), __float_as_int(v5.x), __float_as_int(v5.y),
                     __float_as_int(v5.z), __float_as_int(v5.w)};
        float key[8];
        int nh = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float lx = fmaf(qbyte(__float_as_uint(v1.x), __float_as_uint(v1.y), k), sx, v0.x);
            float hx = fmaf(qbyte(__float_as_uint(v1.z), __float_as_uint(v1.w), k), sx, v0.x);
            float ly = fmaf(qbyte(__float_as_uint(v2.x), __float_as_uint(v2.y), k), sy, v0.y);
            float hy = fmaf(qbyte(__float_as_uint(v2.z), __float_as_uint(v2.w), k), sy, v0.y);
            float lz = fmaf(qbyte(__float_as_uint(v3.x), __float_as_uint(v3.y), k), sz, v0.z);
            float hz = fmaf(qbyte(__float_as_uint(v3.z), __float_as_uint(v3.w), k), sz, v0.z);
            float tn;
            bool hit = (k < nc) && slab(r, lx, hx, ly, hy, lz, hz, q.t, tn);
            key[k] = hit ? tn : 3.0e38f;
            nh += hit;
        }
        if (nh > 0) {
            // children hit are visited front to back (sorted by entry distance); visiting them
            // unsorted measured 25 % slower on the trench workload (more visits)
            if (nh > 1) {
                cas(key[0], ch[0], key[1], ch[1]); cas(key[2], ch[2], key[3], ch[3]);
                cas(key[4], ch[4], key[5], ch[5]); cas(key[6], ch[6], key[7], ch[7]);
                cas(key[0], ch[0], key[2], ch[2]); cas(key[1], ch[1], key[3], ch[3]);
                cas(key[4], ch[4], key[6], ch[6]); cas(key[5], ch[5], key[7], ch[7]);
                cas(key[1], ch[1], key[2], ch[2]); cas(key[5], ch[5], key[6], ch[6]);
                cas(key[0], ch[0], key[4], ch[4]); cas(key[1], ch[1], key[5], ch[5]);
                cas(key[2], ch[2], key[6], ch[6]); cas(key[3], ch[3], key[7], ch[7]);
                cas(key[2], ch[2], key[4], ch[4]); cas(key[3], ch[3], key[5], ch[5]);
                cas(key[1], ch[1], key[2], ch[2]); cas(key[3], ch[3], key[4], ch[4]);
                cas(key[5], ch[5], key[6], ch[6]);
#pragma unroll
                for (int k = 7; k >= 1; --k)
                    if (k < nh) st.push(q, ch[k], key[k], err);
                q.cur = ch[0];
            } else {
                int c = ch[0];
#pragma unroll
                for (int k = 1; k < 8; ++k) c = key[k] < 1.0e38f ? ch[k] : c;
                q.cur = c;
            }
            return false;
        }
    }
    return !st.pop(q);
}

template <class St>
__device__ __forceinline__ bool step_wide(const Tracer& T, Query& q, St& st, int* err) {
    if (q.cur == kDone) return true;
    if (++q.visits > kMaxVisits) {
        *err |= 1;
        q.cur = kDone;
        return true;
    }
    return q.cur >= 0 ? step_wide_node(T, q, st, err) : step_leaf(T, q, st);
}

// One step of the binary traversal; returns true once the query has finished.  The internal-node
// and leaf halves are also callable on their own (a warp can run one kind of step at a time for
// the lanes at that kind of node, see k_trace).  Children are followed by their traversal refs
// (the node's last two words), so a leaf child's faces need no lookup.
template <class St>
__device__ __forceinline__ bool step_binary_node(const Tracer& T, Query& q, St& st, int* err) {
    const float4* n = T.m.nodes + 4 * q.cur;
    float4 n0 = __ldg(n), n1 = __ldg(n + 1), n2 = __ldg(n + 2), n3 = __ldg(n + 3);
    float t0, t1;
    bool h0 = slab(q.r, n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, q.t, t0);
    bool h1 = slab(q.r, n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, q.t, t1);
    int c0 = __float_as_int(n3.z), c1 = __float_as_int(n3.w);
    if (h0 && h1) {
        bool swap = t1 < t0;
        st.push(q, swap ? c0 : c1, swap ? t0 : t1, err);
        q.cur = swap ? c1 : c0;
        return false;
    }
    if (h0 || h1) {
        q.cur = h0 ? c0 : c1;
        return false;
    }
    return !st.pop(q);
}

__device__ __forceinline__ bool visit_bound(Query& q, int* err) {
    if (++q.visits > kMaxVisits) {
        *err |= 1;
        q.cur = kDone;
        return true;
    }
    return false;
}

template <class St>
__device__ __forceinline__ bool step_binary(const Tracer& T, Query& q, St& st, int* err) {
    if (q.cur == kDone) return true;
    if (visit_bound(q, err)) return true;
    return q.cur >= 0 ? step_binary_node(T, q, st, err) : step_leaf(T, q, st);
}

// Stage the top of the wide tree in shared memory (call from every thread of the block).
__device__ __forceinline__ Tracer make_tracer(const MeshView& m, float4* smem, bool wide) {
    Tracer T;
    T.m = m;
    T.WN = m.hdr[HDR_WN];
    T.L = min(m.hdr[HDR_L], m.MT);
    T.nsm = wide ? min(T.WN, kSmemNodes) : 0;
    const float4* g = reinterpret_cast<const float4*>(m.wnodes);
    for (int i = threadIdx.x; i < 6 * T.nsm; i += blockDim.x) smem[i] = __ldg(g + i);
    __syncthreads();
    T.snodes = smem;
    return T;
}

// Unit winding normal of face f (normalize(cross(b - a, c - a)), as Warp's query normal).
__device__ __forceinline__ float3 face_normal(const MeshView& m, int f) {
    float3 a = tri_v(m.tri, f, 0), b = tri_v(m.tri, f, 1), c = tri_v(m.tri, f, 2);
    return normalize3(cross3(b - a, c - a));
}

// Closest point on triangle (a, b, c) to p: squared distance (Ericson, Real-Time Collision
// Detection, 5.1.5, Voronoi-region walk).
__device__ __forceinline__ float point_tri_d2(float3 p, float3 a, float3 b, float3 c) {
    float3 ab = b - a, ac = c - a, ap = p - a;
    float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    float3 q;
    if (d1 <= 0.0f && d2 <= 0.0f) { q = a; }
    else {
        float3 bp = p - b;
        float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
        if (d3 >= 0.0f && d4 <= d3) { q = b; }
        else {
            float vc = d1 * d4 - d3 * d2;
            if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) { q = a + (d1 / (d1 - d3)) * ab; }
            else {
                float3 cp = p - c;
                float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
                if (d6 >= 0.0f && d5 <= d6) { q = c; }
                else {
                    float vb = d5 * d2 - d1 * d6;
                    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) { q = a + (d2 / (d2 - d6)) * ac; }
                    else {
                        float va = d3 * d6 - d5 * d4;
                        if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
                            q = b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
                        } else {
                            float den = 1.0f / (va + vb + vc);
                            q = a + (vb * den) * ab + (vc * den) * ac;
                        }
                    }
                }
            }
        }
    }
    float3 dd = p - q;
    return dot3(dd, dd);
}

__device__ __forceinline__ float box_d2(float3 p, float lx, float hx, float ly, float hy, float lz,
                                        float hz) {
    float dx = fmaxf(fmaxf(lx - p.x, 0.0f), p.x - hx);
    float dy = fmaxf(fmaxf(ly - p.y, 0.0f), p.y - hy);
    float dz = fmaxf(fmaxf(lz - p.z, 0.0f), p.z - hz);
    return dx * dx + dy * dy + dz * dz;
}

// Nearest face to p within sqrt(r2max); ties go to the lower face index.  Returns -1 if none.
// Nearest face to p within sqrt(r2max): by distance to the triangle (CENTROID false, the
// mesh_query_point contract) or to the face centroid (CENTROID true, a KD-tree over centroids);
// exact ties go to the lower face index.  Node boxes bound the triangles, hence their centroids.
template <bool CENTROID>
__device__ __forceinline__ int nearest_prim(const MeshView& m, int L, float3 p, float r2max,
                                            int* err) {
    int best = -1;
    float bd = r2max;
    if (L <= 0) return -1;
    int stack[kStack];
    int sp = 0;
    int node = (L == 1) ? ~0 : 0;
    for (int visits = 0; visits < kMaxVisits; ++visits) {
        if (node >= 0) {
            const float4* n = m.nodes + 4 * node;
            float4 n0 = __ldg(n), n1 = __ldg(n + 1), n2 = __ldg(n + 2), n3 = __ldg(n + 3);
            float e0 = box_d2(p, n0.x, n0.y, n0.z, n0.w, n2.x, n2.y);
            float e1 = box_d2(p, n1.x, n1.y, n1.z, n1.w, n2.z, n2.w);
            int c0 = __float_as_int(n3.x), c1 = __float_as_int(n3.y);
            bool h0 = e0 <= bd, h1 = e1 <= bd;
            if (h0 && h1) {
                int nearc = c0, farc = c1;
                if (e1 < e0) {
                    nearc = c1;
                    farc = c0;
                }
                if (sp < kStack) stack[sp++] = farc;
                else *err |= 1;
                node = nearc;
                continue;
            }
            if (h0) { node = c0; continue; }
            if (h1) { node = c1; continue; }
        } else {
            int l = ~node;
            int f0 = __ldg(m.leaf_start + l), f1 = min(__ldg(m.leaf_start + l + 1), m.MT);
            for (int f = f0; f < f1; ++f) {
                float d2;
                if (CENTROID) {
                    float3 c = make_float3(__ldg(m.centroid + 3 * f), __ldg(m.centroid + 3 * f + 1),
                                           __ldg(m.centroid + 3 * f + 2));
                    d2 = dot3(p - c, p - c);
                } else {
                    d2 = point_tri_d2(p, tri_v(m.tri, f, 0), tri_v(m.tri, f, 1), tri_v(m.tri, f, 2));
                }
                if (d2 < bd || (d2 == bd && (best < 0 || f < best))) {
                    bd = d2;
                    best = f;
                }
            }
        }
        if (sp == 0) return best;
        node = stack[--sp];
    }
    *err |= 1;
    return best;
}

__device__ __forceinline__ int nearest_face(const MeshView& m, int L, float3 p, float r2max,
                                            int* err) {
    return nearest_prim<false>(m, L, p, r2max, err);
}

}  // namespace petch
