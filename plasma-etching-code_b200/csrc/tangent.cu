// Tangent (forward-mode) kernels of the etch step for the recipe gradient: each runs the primal
// update and carries N = 3 directional derivatives of every value, taking exactly the primal's
// branches (upwind choices, min / max selections, clamps, nearest faces).  Tangent arrays are
// direction-major: the k-th direction of a field of n entries is at d + k * n.
//   * dense advection substep (advect_3d_gpu / _advect_iter, threed.py:1262-1292);
//   * Eikonal reinit: init, Jacobi sweeps, finalisation (reinit_fsm, threed.py:1421-1537);
//   * velocity extension (extend_velocity_gpu, threed.py:1324-1346): dF = dV[nearest face];
//   * coverage warm start (gpu_warmstart_bare, threed.py:1619-1639).
#include <cmath>
#include "common.cuh"
#include "dual.cuh"
#include "levelset.cuh"
#include "mesh.cuh"
#include "trace.cuh"

namespace petch {
namespace {

constexpr int kTanB = 256;
constexpr int ND = 3;
using D3 = Dual<float, ND>;

__device__ __forceinline__ D3 dload(const float* __restrict__ v, const float* __restrict__ d,
                                    long long c, long long n) {
    D3 r;
    r.v = v[c];
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = d[c + k * n];
    return r;
}

__device__ __forceinline__ void dstore(float* __restrict__ v, float* __restrict__ d, long long c,
                                       long long n, const D3& x) {
    v[c] = x.v;
#pragma unroll
    for (int k = 0; k < ND; ++k) d[c + k * n] = x.d[k];
}

// One cell of a mask-array advection substep with tangents (the value equals petch_advect's).
__device__ __forceinline__ void advect_tan_cell(const float* __restrict__ phi,
                                                const float* __restrict__ dphi,
                                                float* __restrict__ out, float* __restrict__ dout,
                                                const float* __restrict__ F,
                                                const float* __restrict__ dF,
                                                const uint8_t* __restrict__ mask,
                                                const float* __restrict__ mask_phi, const LGrid& g,
                                                float inv_dx, float dt, long long c) {
    const long long n = g.n;
    {
        if (mask[c]) {
            out[c] = mask_phi[c];
#pragma unroll
            for (int k = 0; k < ND; ++k) dout[c + k * n] = 0.0f;
            return;
        }
        const D3 v = dload(phi, dphi, c, n);
        const D3 f = dload(F, dF, c, n);
        int i, j, kk;
        lsplit(g, c, i, j, kk);
        D3 gg = dconst<float, ND>(0.0f);
        const D3 zero = dconst<float, ND>(0.0f);
        const long long st[3] = {g.plane, (long long)g.nz, 1};
        const int pos[3] = {i, j, kk};
        const int ext[3] = {g.nx, g.ny, g.nz};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const D3 dm = pos[a] >= 1 ? (v - dload(phi, dphi, c - st[a], n)) * inv_dx : zero;
            const D3 dp = pos[a] <= ext[a] - 2 ? (dload(phi, dphi, c + st[a], n) - v) * inv_dx : zero;
            const D3 t = vmax(dm, 0.0f);
            const D3 s = vmin(dp, 0.0f);
            gg = gg + (t * t + s * s);
        }
        D3 o = v - (dt * f) * vsqrt(gg);
        // the value exactly as the primal kernels compute it (same expression, same rounding)
        o.v = f.v == 0.0f ? v.v : advect_cell(phi, c, g, inv_dx, f.v, dt);
        dstore(out, dout, c, n, o);
    }
}

__global__ void __launch_bounds__(kTanB) k_advect_tan(const float* __restrict__ phi,
                                                      const float* __restrict__ dphi,
                                                      float* __restrict__ out,
                                                      float* __restrict__ dout,
                                                      const float* __restrict__ F,
                                                      const float* __restrict__ dF,
                                                      const uint8_t* __restrict__ mask,
                                                      const float* __restrict__ mask_phi, LGrid g,
                                                      float inv_dx, float dt) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.n;
         c += (long long)gridDim.x * blockDim.x)
        advect_tan_cell(phi, dphi, out, dout, F, dF, mask, mask_phi, g, inv_dx, dt, c);
}

// eik_solve with tangents (same sort and branch structure as the primal).
__device__ __forceinline__ D3 eik_solve_tan(D3 a1, D3 a2, D3 a3, float dx) {
    D3 t;
    if (a1.v > a2.v) { t = a1; a1 = a2; a2 = t; }
    if (a2.v > a3.v) { t = a2; a2 = a3; a3 = t; }
    if (a1.v > a2.v) { t = a1; a1 = a2; a2 = t; }
    D3 x = a1 + dx;
    if (x.v <= a2.v) return x;
    D3 d2 = 2.0f * dx * dx - (a1 - a2) * (a1 - a2);
    d2 = vmax(d2, 0.0f);
    x = 0.5f * (a1 + a2 + vsqrt(d2));
    if (x.v <= a3.v) return x;
    D3 s1 = a1 + a2 + a3;
    D3 s2 = a1 * a1 + a2 * a2 + a3 * a3;
    D3 d3 = s1 * s1 - 3.0f * (s2 - dx * dx);
    d3 = vmax(d3, 0.0f);
    return (s1 + vsqrt(d3)) / 3.0f;
}

__device__ __forceinline__ void eik_init_tan_cell(const float* __restrict__ phi0,
                                                  const float* __restrict__ dphi0,
                                                  float* __restrict__ U, float* __restrict__ dU,
                                                  const LGrid& g, float inv_dx, float big,
                                                  long long c) {
    const long long n = g.n;
    {
        int i, j, k;
        lsplit(g, c, i, j, k);
        const D3 v = dload(phi0, dphi0, c, n);
        const D3 oxm = dload(phi0, dphi0, i >= 1 ? c - g.plane : c, n);
        const D3 oxp = dload(phi0, dphi0, i <= g.nx - 2 ? c + g.plane : c, n);
        const D3 oym = dload(phi0, dphi0, j >= 1 ? c - g.nz : c, n);
        const D3 oyp = dload(phi0, dphi0, j <= g.ny - 2 ? c + g.nz : c, n);
        const D3 ozm = dload(phi0, dphi0, k >= 1 ? c - 1 : c, n);
        const D3 ozp = dload(phi0, dphi0, k <= g.nz - 2 ? c + 1 : c, n);
        const bool iface = (v.v * oxm.v < 0.0f) || (v.v * oxp.v < 0.0f) || (v.v * oym.v < 0.0f) ||
                           (v.v * oyp.v < 0.0f) || (v.v * ozm.v < 0.0f) || (v.v * ozp.v < 0.0f);
        D3 u;
        if (iface) {
            const D3 gx = ((oxp - oxm) * 0.5f) * inv_dx;
            const D3 gy = ((oyp - oym) * 0.5f) * inv_dx;
            const D3 gz = ((ozp - ozm) * 0.5f) * inv_dx;
            const D3 grad0 = vmax(vsqrt(gx * gx + gy * gy + gz * gz), 0.5f);
            const float dxl = 1.0f / inv_dx;
            const D3 Dd = vmin(vabs(v) / grad0, 1.8f * dxl);
            u = -Dd;                              // frozen: the distance with the sign bit set
            u.v = copysignf(Dd.v, -1.0f);
        } else {
            u = dconst<float, ND>(big);
        }
        dstore(U, dU, c, n, u);
    }
}

__global__ void __launch_bounds__(kTanB) k_eik_init_tan(const float* __restrict__ phi0,
                                                        const float* __restrict__ dphi0,
                                                        float* __restrict__ U,
                                                        float* __restrict__ dU, LGrid g,
                                                        float inv_dx, float big) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.n;
         c += (long long)gridDim.x * blockDim.x)
        eik_init_tan_cell(phi0, dphi0, U, dU, g, inv_dx, big, c);
}

template <bool FINAL>
__device__ __forceinline__ void eik_sweep_tan_cell(const float* __restrict__ Uin,
                                                   const float* __restrict__ dUin,
                                                   float* __restrict__ Uout,
                                                   float* __restrict__ dUout,
                                                   const float* __restrict__ phi_in,
                                                   float* __restrict__ phi_out,
                                                   float* __restrict__ dphi_out, const LGrid& g,
                                                   float dx, float big, float cap, long long c) {
    const long long n = g.n;
    {
        const D3 u = dload(Uin, dUin, c, n);
        D3 un;
        if (frozen(u.v)) {
            un = FINAL ? vabs(u) : u;
        } else {
            int i, j, k;
            lsplit(g, c, i, j, k);
            const D3 bigd = dconst<float, ND>(big);
            D3 um = (i >= 1) ? vabs(dload(Uin, dUin, c - g.plane, n)) : bigd;
            D3 up = (i <= g.nx - 2) ? vabs(dload(Uin, dUin, c + g.plane, n)) : bigd;
            const D3 ax = vmin(um, up);
            um = (j >= 1) ? vabs(dload(Uin, dUin, c - g.nz, n)) : bigd;
            up = (j <= g.ny - 2) ? vabs(dload(Uin, dUin, c + g.nz, n)) : bigd;
            const D3 ay = vmin(um, up);
            um = (k >= 1) ? vabs(dload(Uin, dUin, c - 1, n)) : bigd;
            up = (k <= g.nz - 2) ? vabs(dload(Uin, dUin, c + 1, n)) : bigd;
            const D3 az = vmin(um, up);
            un = vmin(u, eik_solve_tan(ax, ay, az, dx));
        }
        if (FINAL) {
            const float s = phi_in[c];
            const float sg = s < 0.0f ? -1.0f : 1.0f;
            const D3 o = sg * vmin(un, dconst<float, ND>(cap));
            phi_out[c] = o.v + 0.0f;
#pragma unroll
            for (int k = 0; k < ND; ++k) dphi_out[c + k * n] = o.d[k];
        } else {
            dstore(Uout, dUout, c, n, un);
        }
    }
}

template <bool FINAL>
__global__ void __launch_bounds__(kTanB) k_eik_sweep_tan(const float* __restrict__ Uin,
                                                         const float* __restrict__ dUin,
                                                         float* __restrict__ Uout,
                                                         float* __restrict__ dUout,
                                                         const float* __restrict__ phi_in,
                                                         float* __restrict__ phi_out,
                                                         float* __restrict__ dphi_out, LGrid g,
                                                         float dx, float big, float cap) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.n;
         c += (long long)gridDim.x * blockDim.x)
        eik_sweep_tan_cell<FINAL>(Uin, dUin, Uout, dUout, phi_in, phi_out, dphi_out, g, dx, big,
                                  cap, c);
}

struct TGrid {
    int nx, ny, nz;
    long long plane, n;
    double dx, band;
};

// dF = dV[nearest face] on |phi| < band (the primal's nearest-face choice), 0 elsewhere.
__global__ void __launch_bounds__(kTanB) k_extend_tan(MeshView m, TGrid G,
                                                      const float* __restrict__ phi,
                                                      const float* __restrict__ dV,
                                                      float* __restrict__ dF, int* work) {
    const int L = min(m.hdr[HDR_L], m.MT);
    const long long MT = m.MT;
    int err = 0;
    const float r_near = (float)(G.band + 2.0 * G.dx);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < G.n;
         c += (long long)gridDim.x * blockDim.x) {
        float o[ND] = {0.0f, 0.0f, 0.0f};
        if ((double)fabsf(phi[c]) < G.band) {
            long long r = c / G.nz;
            int k = (int)(c - r * G.nz);
            int i = (int)(r / G.ny);
            int j = (int)(r - (long long)i * G.ny);
            float3 p = make_float3((float)(i * G.dx), (float)(j * G.dx), (float)(k * G.dx));
            int f = nearest_face(m, L, p, r_near * r_near, &err);
            if (f < 0) f = nearest_face(m, L, p, 1.0e12f, &err);
            if (f >= 0)
                for (int q = 0; q < ND; ++q) o[q] = dV[f + q * MT];
        }
        for (int q = 0; q < ND; ++q) dF[c + q * G.n] = o[q];
    }
    if (err) atomicOr(work + 1, err);
}

__global__ void __launch_bounds__(kTanB) k_warmstart_tan(MeshView prev,
                                                         const float* __restrict__ prev_bare,
                                                         const float* __restrict__ prev_dbare,
                                                         MeshView cur, float* __restrict__ dbare,
                                                         int* work) {
    const int Lp = min(prev.hdr[HDR_L], prev.MT);
    const int F = min(cur.hdr[HDR_F], cur.MT);
    const long long PMT = prev.MT, MT = cur.MT;
    int err = 0;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x) {
        float3 p = make_float3(cur.centroid[3 * f], cur.centroid[3 * f + 1], cur.centroid[3 * f + 2]);
        int q = nearest_face(prev, Lp, p, 1.0e12f, &err);
        const bool pass = q >= 0 && prev_bare[q] > 0.0f && prev_bare[q] < 1.0f;
        for (int k = 0; k < ND; ++k) dbare[f + k * MT] = pass ? prev_dbare[q + k * PMT] : 0.0f;
    }
    if (err) atomicOr(work + 1, err);
}

// ---- batched tangent level-set stages: blockIdx.y selects the instance ----
constexpr int kTMaxInst = 64;

struct TBItem {
    float* phi;
    float* tmp;
    float* ua;
    float* ub;
    const float* F;
    const float* mask_phi;
    float* dphi;
    float* dtmp;
    float* dua;
    float* dub;
    const float* dF;
    const uint8_t* mask;
    LGrid g;
    double dx, dt;
    const int* stats;
    const int* hdr;
    int* sub;
};

struct TBTable {
    TBItem it[kTMaxInst];
    int B;
};

__global__ void k_bt_nsub(TBTable t) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= t.B) return;
    const TBItem& x = t.it[b];
    cfl_substeps(x.hdr[HDR_F], x.stats, x.dt, x.dx, x.sub);
}

// Substep s of every instance with s < nsub (dense, mask array; buffers of parity s into the
// other).
__global__ void __launch_bounds__(kTanB) k_bt_adv(TBTable t, int s) {
    const int b = blockIdx.y;
    if (b >= t.B) return;
    const TBItem& x = t.it[b];
    if (s >= x.sub[0]) return;
    const float* a = (s & 1) ? x.tmp : x.phi;
    const float* da = (s & 1) ? x.dtmp : x.dphi;
    float* o = (s & 1) ? x.phi : x.tmp;
    float* dout = (s & 1) ? x.dphi : x.dtmp;
    const float inv_dx = (float)(1.0 / x.dx);
    const float dt = __int_as_float(x.sub[1]);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < x.g.n;
         c += (long long)gridDim.x * blockDim.x)
        advect_tan_cell(a, da, o, dout, x.F, x.dF, x.mask, x.mask_phi, x.g, inv_dx, dt, c);
}

// After an odd number of substeps the state lives in tmp / dtmp: copy it back.
__global__ void k_bt_adv_finish(TBTable t) {
    const int b = blockIdx.y;
    if (b >= t.B) return;
    const TBItem& x = t.it[b];
    if ((x.sub[0] & 1) == 0) return;
    const long long n = x.g.n;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        x.phi[c] = x.tmp[c];
#pragma unroll
        for (int k = 0; k < ND; ++k) x.dphi[c + k * n] = x.dtmp[c + k * n];
    }
}

__global__ void __launch_bounds__(kTanB) k_bt_eik_init(TBTable t, double band_r) {
    const int b = blockIdx.y;
    if (b >= t.B) return;
    const TBItem& x = t.it[b];
    const float inv_dx = (float)(1.0 / x.dx);
    const float big = (float)(band_r + 4.0 * x.dx);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < x.g.n;
         c += (long long)gridDim.x * blockDim.x)
        eik_init_tan_cell(x.phi, x.dphi, x.ua, x.dua, x.g, inv_dx, big, c);
}

template <bool FINAL>
__global__ void __launch_bounds__(kTanB) k_bt_eik_sweep(TBTable t, double band_r, int parity) {
    const int b = blockIdx.y;
    if (b >= t.B) return;
    const TBItem& x = t.it[b];
    const float* in = parity ? x.ub : x.ua;
    const float* din = parity ? x.dub : x.dua;
    float* out = parity ? x.ua : x.ub;
    float* dout = parity ? x.dua : x.dub;
    const float dxf = (float)x.dx;
    const float big = (float)(band_r + 4.0 * x.dx), cap = (float)(band_r + x.dx);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < x.g.n;
         c += (long long)gridDim.x * blockDim.x) {
        if (FINAL)
            eik_sweep_tan_cell<true>(in, din, nullptr, nullptr, x.phi, x.phi, x.dphi, x.g, dxf, big,
                                     cap, c);
        else
            eik_sweep_tan_cell<false>(in, din, out, dout, nullptr, nullptr, nullptr, x.g, dxf, big,
                                      cap, c);
    }
}

int make_ttable(const petch_batch_grid* grids, const petch_batch_tangent_grid* tans, int B,
                TBTable* t, long long* max_cells, const char* who) {
    PETCH_REQUIRE(grids && tans, "%s: null table", who);
    PETCH_REQUIRE(B >= 1 && B <= kTMaxInst, "%s: 1 <= B <= %d", who, kTMaxInst);
    t->B = B;
    long long mc = 0;
    for (int b = 0; b < B; ++b) {
        const petch_batch_grid& s = grids[b];
        const petch_batch_tangent_grid& d = tans[b];
        PETCH_REQUIRE(s.phi && s.tmp && s.ua && s.ub && s.F && s.mask_phi && s.stats && s.hdr &&
                          s.sub && d.dphi && d.dtmp && d.dF && d.mask && d.du_a && d.du_b,
                      "%s: instance %d incomplete", who, b);
        PETCH_REQUIRE(s.nx > 0 && s.ny > 0 && s.nz > 0 && s.dx > 0.0 && s.dt >= 0.0,
                      "%s: instance %d has a bad size", who, b);
        TBItem& x = t->it[b];
        x.phi = s.phi;
        x.tmp = s.tmp;
        x.ua = s.ua;
        x.ub = s.ub;
        x.F = s.F;
        x.mask_phi = s.mask_phi;
        x.dphi = d.dphi;
        x.dtmp = d.dtmp;
        x.dua = d.du_a;
        x.dub = d.du_b;
        x.dF = d.dF;
        x.mask = d.mask;
        x.g = make_lgrid(s.nx, s.ny, s.nz);
        x.dx = s.dx;
        x.dt = s.dt;
        x.stats = s.stats;
        x.hdr = s.hdr;
        x.sub = s.sub;
        if (x.g.n > mc) mc = x.g.n;
    }
    *max_cells = mc;
    return PETCH_OK;
}

}  // namespace
}  // namespace petch

using namespace petch;

extern "C" int petch_advect_tangent(float* phi, float* tmp, float* dphi, float* dtmp,
                                    const float* F, const float* dF, const uint8_t* mask,
                                    const float* mask_phi, int nx, int ny, int nz, float inv_dx,
                                    float dt_sub, int nsub, void* stream) {
    PETCH_REQUIRE(phi && tmp && dphi && dtmp && F && dF && mask && mask_phi,
                  "petch_advect_tangent: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && nsub >= 0, "petch_advect_tangent: bad size");
    const LGrid g = make_lgrid(nx, ny, nz);
    cudaStream_t st = as_stream(stream);
    const int blocks = grid_for(g.n, kTanB);
    float *a = phi, *b = tmp, *da = dphi, *db = dtmp;
    for (int s = 0; s < nsub; ++s) {
        k_advect_tan<<<blocks, kTanB, 0, st>>>(a, da, b, db, F, dF, mask, mask_phi, g, inv_dx,
                                               dt_sub);
        PETCH_LAUNCH_CHECK("k_advect_tan");
        float* t = a; a = b; b = t;
        t = da; da = db; db = t;
    }
    if (a != phi) {
        PETCH_CUDA(cudaMemcpyAsync(phi, a, sizeof(float) * g.n, cudaMemcpyDeviceToDevice, st),
                   "copy-back phi");
        PETCH_CUDA(cudaMemcpyAsync(dphi, da, sizeof(float) * ND * g.n, cudaMemcpyDeviceToDevice, st),
                   "copy-back dphi");
    }
    return PETCH_OK;
}

extern "C" int petch_reinit_tangent(float* phi, float* dphi, float* u_a, float* u_b, float* du_a,
                                    float* du_b, int nx, int ny, int nz, double dx, float big,
                                    float cap, int n_iter, void* stream) {
    PETCH_REQUIRE(phi && dphi && u_a && u_b && du_a && du_b, "petch_reinit_tangent: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && dx > 0.0 && n_iter >= 1,
                  "petch_reinit_tangent: bad size");
    const LGrid g = make_lgrid(nx, ny, nz);
    cudaStream_t st = as_stream(stream);
    const int blocks = grid_for(g.n, kTanB);
    const float dxf = (float)dx, inv_dx = (float)(1.0 / dx);
    k_eik_init_tan<<<blocks, kTanB, 0, st>>>(phi, dphi, u_a, du_a, g, inv_dx, big);
    PETCH_LAUNCH_CHECK("k_eik_init_tan");
    float *a = u_a, *b = u_b, *da = du_a, *db = du_b;
    for (int it = 0; it < n_iter - 1; ++it) {
        k_eik_sweep_tan<false><<<blocks, kTanB, 0, st>>>(a, da, b, db, nullptr, nullptr, nullptr, g,
                                                         dxf, big, cap);
        PETCH_LAUNCH_CHECK("k_eik_sweep_tan");
        float* t = a; a = b; b = t;
        t = da; da = db; db = t;
    }
    k_eik_sweep_tan<true><<<blocks, kTanB, 0, st>>>(a, da, nullptr, nullptr, phi, phi, dphi, g, dxf,
                                                    big, cap);
    PETCH_LAUNCH_CHECK("k_eik_sweep_tan<final>");
    return PETCH_OK;
}

extern "C" int petch_extend_tangent(const void* mesh, int max_tris, int max_verts, const float* phi,
                                    int nx, int ny, int nz, double dx, double band, const float* dV,
                                    float* dF, int* work, void* stream) {
    PETCH_REQUIRE(mesh && phi && dV && dF && work, "petch_extend_tangent: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && dx > 0, "petch_extend_tangent: bad grid");
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    TGrid G{nx, ny, nz, (long long)ny * nz, (long long)nx * ny * nz, dx, band};
    k_extend_tan<<<grid_for(G.n, kTanB, 16), kTanB, 0, as_stream(stream)>>>(m, G, phi, dV, dF, work);
    PETCH_LAUNCH_CHECK("k_extend_tan");
    return PETCH_OK;
}

extern "C" int petch_warmstart_tangent(const void* prev_mesh, int prev_max_tris,
                                       int prev_max_verts, const float* prev_bare,
                                       const float* prev_dbare, const void* mesh, int max_tris,
                                       int max_verts, float* dbare, int* work, void* stream) {
    PETCH_REQUIRE(prev_mesh && prev_bare && prev_dbare && mesh && dbare && work,
                  "petch_warmstart_tangent: null pointer");
    MeshView pm = mesh_view(const_cast<void*>(prev_mesh), prev_max_tris, prev_max_verts);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    k_warmstart_tan<<<grid_for(max_tris, kTanB), kTanB, 0, as_stream(stream)>>>(pm, prev_bare,
                                                                              prev_dbare, m, dbare,
                                                                              work);
    PETCH_LAUNCH_CHECK("k_warmstart_tan");
    return PETCH_OK;
}

extern "C" int petch_batch_advect_tangent(const petch_batch_grid* grids,
                                          const petch_batch_tangent_grid* tans, int B,
                                          void* stream) {
    TBTable t;
    long long mc = 0;
    int rc = make_ttable(grids, tans, B, &t, &mc, "petch_batch_advect_tangent");
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    k_bt_nsub<<<1, kTMaxInst, 0, st>>>(t);
    PETCH_LAUNCH_CHECK("k_bt_nsub");
    dim3 gc(grid_for(mc, kTanB, 2), B);
    for (int s = 0; s < 160; ++s) {
        k_bt_adv<<<gc, kTanB, 0, st>>>(t, s);
        PETCH_LAUNCH_CHECK("k_bt_adv");
    }
    k_bt_adv_finish<<<gc, kTanB, 0, st>>>(t);
    PETCH_LAUNCH_CHECK("k_bt_adv_finish");
    return PETCH_OK;
}

extern "C" int petch_batch_reinit_tangent(const petch_batch_grid* grids,
                                          const petch_batch_tangent_grid* tans, int B,
                                          double band_r, void* stream) {
    TBTable t;
    long long mc = 0;
    int rc = make_ttable(grids, tans, B, &t, &mc, "petch_batch_reinit_tangent");
    if (rc) return rc;
    const double dx = grids[0].dx;
    for (int b = 1; b < B; ++b)
        PETCH_REQUIRE(grids[b].dx == dx, "petch_batch_reinit_tangent: all grids need the same dx");
    const int n_iter = (int)std::ceil(band_r / dx) + 4;
    cudaStream_t st = as_stream(stream);
    dim3 gc(grid_for(mc, kTanB, 2), B);
    k_bt_eik_init<<<gc, kTanB, 0, st>>>(t, band_r);
    PETCH_LAUNCH_CHECK("k_bt_eik_init");
    int parity = 0;
    for (int it = 0; it < n_iter - 1; ++it) {
        k_bt_eik_sweep<false><<<gc, kTanB, 0, st>>>(t, band_r, parity);
        PETCH_LAUNCH_CHECK("k_bt_eik_sweep");
        parity ^= 1;
    }
    k_bt_eik_sweep<true><<<gc, kTanB, 0, st>>>(t, band_r, parity);
    PETCH_LAUNCH_CHECK("k_bt_eik_sweep<final>");
    return PETCH_OK;
}
