// Per-cell level-set updates shared by the single-grid kernels (levelset.cu, surface.cu) and
// the batched kernels (batch.cu), so that every path computes bit-identical values.
#pragma once
#include <cstdint>

namespace petch {

struct LGrid {
    int nx, ny, nz;
    long long plane;  // ny * nz
    long long n;      // nx * ny * nz
};

__host__ __device__ inline LGrid make_lgrid(int nx, int ny, int nz) {
    LGrid g;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.plane = (long long)ny * nz;
    g.n = g.plane * nx;
    return g;
}

// (i, j, k) of cell c; 32-bit divisions when the grid has fewer than 2^31 cells (the 64-bit ones
// cost several times more and dominate a stencil cell's instruction count).
__device__ __forceinline__ void lsplit(const LGrid& g, long long c, int& i, int& j, int& k) {
    if (g.n < (1LL << 31)) {
        const unsigned cc = (unsigned)c, nz = (unsigned)g.nz, ny = (unsigned)g.ny;
        const unsigned r = cc / nz;
        k = (int)(cc - r * nz);
        i = (int)(r / ny);
        j = (int)(r - (unsigned)i * ny);
        return;
    }
    long long r = c / g.nz;
    k = (int)(c - r * g.nz);
    i = (int)(r / g.ny);
    j = (int)(r - (long long)i * g.ny);
}

// One first-order Godunov upwind substep of cell c with speed f (threed.py:1262-1292): a zero
// one-sided difference at the domain faces.  Every operation is rounded on its own (no fused
// multiply-add), so every kernel that advects -- dense, band list, batched, tangent -- produces
// the same bits.
__device__ __forceinline__ float advect_cell_at(const float* __restrict__ phi, long long c, int i,
                                                int j, int k, const LGrid& g, float inv_dx,
                                                float f, float dt) {
    const float v = phi[c];
    const long long st[3] = {g.plane, (long long)g.nz, 1};
    const int pos[3] = {i, j, k};
    const int ext[3] = {g.nx, g.ny, g.nz};
    float gg = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float dm = pos[a] >= 1 ? __fmul_rn(__fsub_rn(v, phi[c - st[a]]), inv_dx) : 0.0f;
        const float dp = pos[a] <= ext[a] - 2 ? __fmul_rn(__fsub_rn(phi[c + st[a]], v), inv_dx) : 0.0f;
        const float t = fmaxf(dm, 0.0f);
        const float s = fminf(dp, 0.0f);
        gg = __fadd_rn(gg, __fadd_rn(__fmul_rn(t, t), __fmul_rn(s, s)));
    }
    return __fsub_rn(v, __fmul_rn(__fmul_rn(dt, f), __fsqrt_rn(gg)));
}

__device__ __forceinline__ float advect_cell(const float* __restrict__ phi, long long c,
                                             const LGrid& g, float inv_dx, float f, float dt) {
    int i, j, k;
    lsplit(g, c, i, j, k);
    return advect_cell_at(phi, c, i, j, k, g, inv_dx, f, dt);
}

// Godunov solution of |grad U| = 1 from the three upwind neighbour minima (threed.py:1421-1452):
// sort ascending, then take the 1-, 2- or 3-term root while it stays below the next neighbour.
// Each operation rounded on its own, in the order the tangent kernels' dual version uses.
__device__ __forceinline__ float eik_solve(float a1, float a2, float a3, float dx) {
    float t;
    if (a1 > a2) { t = a1; a1 = a2; a2 = t; }
    if (a2 > a3) { t = a2; a2 = a3; a3 = t; }
    if (a1 > a2) { t = a1; a1 = a2; a2 = t; }
    float x = __fadd_rn(a1, dx);
    if (x <= a2) return x;
    const float t12 = __fsub_rn(a1, a2);
    float d2 = __fsub_rn(__fmul_rn(__fmul_rn(2.0f, dx), dx), __fmul_rn(t12, t12));
    d2 = fmaxf(d2, 0.0f);
    x = __fmul_rn(__fadd_rn(__fadd_rn(a1, a2), __fsqrt_rn(d2)), 0.5f);
    if (x <= a3) return x;
    const float s1 = __fadd_rn(__fadd_rn(a1, a2), a3);
    const float s2 = __fadd_rn(__fadd_rn(__fmul_rn(a1, a1), __fmul_rn(a2, a2)), __fmul_rn(a3, a3));
    float d3 = __fsub_rn(__fmul_rn(s1, s1), __fmul_rn(3.0f, __fsub_rn(s2, __fmul_rn(dx, dx))));
    d3 = fmaxf(d3, 0.0f);
    return __fdiv_rn(__fadd_rn(s1, __fsqrt_rn(d3)), 3.0f);
}

// Frozen cells carry their distance with the sign bit set (U >= 0 everywhere else).
__device__ __forceinline__ bool frozen(float u) { return signbit(u); }

// _eik_init (threed.py:1455-1479) for cell c: interface cells (a face neighbour, index-clamped,
// of opposite sign) get the sub-cell distance min(|phi0| / max(|grad phi0|, 0.5), 1.8 dx),
// frozen; others `big`.  SEED: nodes where phi0 is exactly 0 are frozen at distance 0.
template <bool SEED>
__device__ __forceinline__ float eik_init_cell_at(const float* __restrict__ phi0, long long c,
                                                  int i, int j, int k, const LGrid& g,
                                                  float inv_dx, float big) {
    float v = phi0[c];
    float oxm = phi0[i >= 1 ? c - g.plane : c];
    float oxp = phi0[i <= g.nx - 2 ? c + g.plane : c];
    float oym = phi0[j >= 1 ? c - g.nz : c];
    float oyp = phi0[j <= g.ny - 2 ? c + g.nz : c];
    float ozm = phi0[k >= 1 ? c - 1 : c];
    float ozp = phi0[k <= g.nz - 2 ? c + 1 : c];
    bool iface = (v * oxm < 0.0f) || (v * oxp < 0.0f) || (v * oym < 0.0f) ||
                 (v * oyp < 0.0f) || (v * ozm < 0.0f) || (v * ozp < 0.0f);
    if (SEED && v == 0.0f) return -0.0f;
    if (iface) {
        const float gx = __fmul_rn(__fmul_rn(__fsub_rn(oxp, oxm), 0.5f), inv_dx);
        const float gy = __fmul_rn(__fmul_rn(__fsub_rn(oyp, oym), 0.5f), inv_dx);
        const float gz = __fmul_rn(__fmul_rn(__fsub_rn(ozp, ozm), 0.5f), inv_dx);
        const float gg = __fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), __fmul_rn(gz, gz));
        const float grad0 = fmaxf(__fsqrt_rn(gg), 0.5f);
        const float dxl = __fdiv_rn(1.0f, inv_dx);
        const float D = fminf(__fdiv_rn(fabsf(v), grad0), __fmul_rn(1.8f, dxl));
        return copysignf(D, -1.0f);
    }
    return big;
}

template <bool SEED>
__device__ __forceinline__ float eik_init_cell(const float* __restrict__ phi0, long long c,
                                               const LGrid& g, float inv_dx, float big) {
    int i, j, k;
    lsplit(g, c, i, j, k);
    return eik_init_cell_at<SEED>(phi0, c, i, j, k, g, inv_dx, big);
}

// One Jacobi sweep of _eik_jacobi (threed.py:1482-1512) for cell c; FINAL returns
// sign(phi_in) * min(U, cap) (reinit_fsm's finalisation, threed.py:1535-1537) instead of U.
template <bool FINAL, bool SEED>
__device__ __forceinline__ float eik_sweep_cell_at(const float* __restrict__ Uin, long long c,
                                                   int i, int j, int k, const LGrid& g, float dx,
                                                   float big, float cap,
                                                   const float* __restrict__ phi_in) {
    float u = Uin[c];
    float un;
    if (frozen(u)) {
        un = FINAL ? fabsf(u) : u;
    } else {
        float um = (i >= 1) ? fabsf(Uin[c - g.plane]) : big;
        float up = (i <= g.nx - 2) ? fabsf(Uin[c + g.plane]) : big;
        float ax = fminf(um, up);
        um = (j >= 1) ? fabsf(Uin[c - g.nz]) : big;
        up = (j <= g.ny - 2) ? fabsf(Uin[c + g.nz]) : big;
        float ay = fminf(um, up);
        um = (k >= 1) ? fabsf(Uin[c - 1]) : big;
        up = (k <= g.nz - 2) ? fabsf(Uin[c + 1]) : big;
        float az = fminf(um, up);
        un = fminf(u, eik_solve(ax, ay, az, dx));
    }
    if (FINAL) {
        float s = phi_in[c];
        float sg = s < 0.0f ? -1.0f : (SEED && s == 0.0f ? 0.0f : 1.0f);
        return __fadd_rn(__fmul_rn(sg, fminf(un, cap)), 0.0f);
    }
    return un;
}

template <bool FINAL, bool SEED>
__device__ __forceinline__ float eik_sweep_cell(const float* __restrict__ Uin, long long c,
                                                const LGrid& g, float dx, float big, float cap,
                                                const float* __restrict__ phi_in) {
    int i = 0, j = 0, k = 0;
    if (!frozen(Uin[c])) lsplit(g, c, i, j, k);
    return eik_sweep_cell_at<FINAL, SEED>(Uin, c, i, j, k, g, dx, big, cap, phi_in);
}

// Row-mapped stencil launches: a block of (bz, br) threads covers br rows (i, j) of the grid,
// threadIdx.x running along z (coalesced), with one division per row instead of per cell; blocks
// stride over the nx * ny rows.  The block shape is a tuning knob (petch_stencil_config).
struct RowShape {
    int bz, br;
};
RowShape stencil_shape();
int stencil_blocks(long long rows, const RowShape& s);

// run_etch_3d's CFL substep count (threed.py:1750-1756) from the device-side rate statistics:
// nsub = clamp(ceil(Vmax dt / (0.4 dx)), 1, 160), Vmax = max(max V if finite (0 without faces),
// 1e-6); sub[0] = nsub, sub[1] = float bits of float(dt / nsub).
__device__ __forceinline__ void cfl_substeps(int n_faces, const int* stats, double dt, double dx,
                                             int* sub) {
    const float vmx = n_faces > 0 ? __int_as_float(stats[1]) : 0.0f;
    double V = isfinite(vmx) ? (double)vmx : 0.0;
    V = fmax(V, 1e-6);
    const double q = ceil(V * dt / (0.4 * dx));
    const int nsub = (int)fmin(fmax(q, 1.0), 160.0);
    sub[0] = nsub;
    sub[1] = __float_as_int((float)(dt / nsub));
}

}  // namespace petch
