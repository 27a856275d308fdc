// Batched level-set stages of the etch step for many independent instances (grids of different
// sizes) in a fixed number of launches, with every step-dependent quantity kept on the device so
// a whole step can be captured in a CUDA graph and replayed:
//   * the CFL substep count of run_etch_3d (petch/threed.py:1750-1756) per instance, from the
//     max surface velocity that petch_surface_rate / petch_redep_apply leave in stats[1];
//   * the narrow-band advection of petch_advect_sparse (advect_3d_gpu, threed.py:1262-1307) as a
//     fixed sequence of kMaxSub substep launches over all instances, each instance stepping while
//     s < nsub[b];
//   * the Jacobi Godunov-Eikonal reinit of petch_reinit_eik mode 0 (reinit_fsm, threed.py:
//     1421-1537): init, n_iter - 1 sweeps and the finalising sweep, each one launch for the batch.
// The instance table travels as a kernel parameter; blockIdx.y selects the instance.
#include <algorithm>
#include <cmath>
#include "common.cuh"
#include "levelset.cuh"
#include "mesh.cuh"

namespace petch {
namespace {

constexpr int kBB = 256;
constexpr int kMaxInst = 64;
constexpr int kMaxSub = 160;     // run_etch_3d's substep cap

struct BGrid {
    float* phi;
    float* tmp;
    float* ua;
    float* ub;
    const float* F;          // extended speed, -1 on mask cells (petch_extend_velocity fold_mask)
    const float* mask_phi;
    const int* mask_idx;
    int n_mask;
    const int* active;
    const int* n_active;
    int max_active;
    LGrid g;
    double dx, dt;
    const int* stats;        // [1]: float bits of max V
    const int* hdr;          // mesh header ([0] = faces)
    int* sub;                // [0] nsub, [1] float bits of dt / nsub
    const int* hold;         // non-NULL and nonzero: leave this level set as it is this step
};

__device__ __forceinline__ bool held(const BGrid& x) { return x.hold && *x.hold; }

struct BTable {
    BGrid it[kMaxInst];
    int B;
};

// nsub = clamp(ceil(Vmax dt / (0.4 dx)), 1, 160), Vmax = max(max V if finite (0 without faces),
// 1e-6); dt_sub = float(dt / nsub).
__global__ void k_b_nsub(BTable t) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= t.B) return;
    const BGrid& x = t.it[b];
    cfl_substeps(x.hdr[HDR_F], x.stats, x.dt, x.dx, x.sub);
    if (held(x)) x.sub[0] = 0;
}

// tmp = phi with the mask cells pinned (the first substep's write target).
__global__ void k_b_adv_prep(BTable t) {
    const int b = blockIdx.y;
    if (b >= t.B) return;
    const BGrid& x = t.it[b];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < x.g.n;
         c += (long long)gridDim.x * blockDim.x)
        x.tmp[c] = x.F[c] < 0.0f ? x.mask_phi[c] : x.phi[c];
}

// Substep s of every instance with s < nsub: band cells from the buffer of parity s into the
// other.  The launch of s = 1 also pins phi's mask cells (phi was the first substep's input).
__global__ void k_b_adv_step(BTable t, int s) {
    const int b = blockIdx.y;
    if (b >= t.B) return;
    const BGrid& x = t.it[b];
    if (s == 1)
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < x.n_mask; q += gridDim.x * blockDim.x) {
            const int c = x.mask_idx[q];
            x.phi[c] = x.mask_phi[c];
        }
    if (s >= x.sub[0]) return;
    const float* a = (s & 1) ? x.tmp : x.phi;
    float* o = (s & 1) ? x.phi : x.tmp;
    const float inv_dx = (float)(1.0 / x.dx);
    const float dt = __int_as_float(x.sub[1]);
    const int na = min(*x.n_active, x.max_active);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < na; q += gridDim.x * blockDim.x) {
        const long long c = x.active[q];
        o[c] = advect_cell(a, c, x.g, inv_dx, x.F[c], dt);
    }
}

// After an odd number of substeps the band lives in tmp: copy it back.
__global__ void k_b_adv_finish(BTable t) {
    const int b = blockIdx.y;
    if (b >= t.B) return;
    const BGrid& x = t.it[b];
    if ((x.sub[0] & 1) == 0) return;
    const int na = min(*x.n_active, x.max_active);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < na; q += gridDim.x * blockDim.x) {
        const int c = x.active[q];
        x.phi[c] = x.tmp[c];
    }
}

// The Eikonal passes row-mapped (petch::RowShape: threadIdx.x along z, threadIdx.y a row of the
// block's, blockIdx.x striding over the instance's nx * ny rows), each row restricted to the z
// range the sweeps can have reached.  A cell keeps `big` until a face neighbour holds a finite
// value, so after sweep s a row's finite cells lie within its own range of sweep s - 1 widened by
// one cell and its four lateral neighbours' ranges; the row ranges (int2 per row: nz - kmin,
// kmax + 1, 0 = empty, so a union is a max) ping-pong in the advection's scratch grid tmp, which
// is free during the reinit.  Cells outside a row's range are not touched: the init writes the
// starting field into both sweep buffers, so they hold `big`, as the dense sweep would leave them.
__device__ __forceinline__ int2* row_ranges(const BGrid& x, int which) {
    return reinterpret_cast<int2*>(x.tmp) + (long long)which * x.g.nx * x.g.ny;
}

__global__ void k_b_rows_clear(BTable t) {
    const int b = blockIdx.y;
    if (b >= t.B) return;
    const BGrid& x = t.it[b];
    if (held(x)) return;
    int2* r = row_ranges(x, 0);
    const int rows = x.g.nx * x.g.ny;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rows; q += gridDim.x * blockDim.x)
        r[q] = make_int2(0, 0);
}

__global__ void k_b_eik_init(BTable t, double band_r) {
    const int b = blockIdx.y;
    if (b >= t.B) return;
    const BGrid& x = t.it[b];
    if (held(x)) return;
    const float inv_dx = (float)(1.0 / x.dx);
    const float big = (float)(band_r + 4.0 * x.dx);
    const int rows = x.g.nx * x.g.ny, nz = x.g.nz;
    int2* r0 = row_ranges(x, 0);
    for (int row = blockIdx.x * blockDim.y + threadIdx.y; row < rows; row += gridDim.x * blockDim.y) {
        const int i = row / x.g.ny, j = row - i * x.g.ny;
        const long long base = (long long)row * nz;
        for (int k = threadIdx.x; k < nz; k += blockDim.x) {
            const float v = eik_init_cell_at<false>(x.phi, base + k, i, j, k, x.g, inv_dx, big);
            x.ua[base + k] = v;
            x.ub[base + k] = v;
            if (v != big) {
                atomicMax(&r0[row].x, nz - k);
                atomicMax(&r0[row].y, k + 1);
            }
        }
    }
}

template <bool FINAL>
__global__ void k_b_eik_sweep(BTable t, double band_r, int parity) {
    const int b = blockIdx.y;
    if (b >= t.B) return;
    const BGrid& x = t.it[b];
    if (held(x)) return;
    const float* in = parity ? x.ub : x.ua;
    float* out = parity ? x.ua : x.ub;
    const int2* rin = row_ranges(x, parity);
    int2* rout = row_ranges(x, parity ^ 1);
    const float dxf = (float)x.dx;
    const float big = (float)(band_r + 4.0 * x.dx), cap = (float)(band_r + x.dx);
    const int nx = x.g.nx, ny = x.g.ny, nz = x.g.nz, rows = nx * ny;
    for (int row = blockIdx.x * blockDim.y + threadIdx.y; row < rows; row += gridDim.x * blockDim.y) {
        const int i = row / ny, j = row - i * ny;
        const long long base = (long long)row * nz;
        int2 e = rin[row];
        if (i >= 1) { const int2 f = rin[row - ny]; e = make_int2(max(e.x, f.x), max(e.y, f.y)); }
        if (i + 1 < nx) { const int2 f = rin[row + ny]; e = make_int2(max(e.x, f.x), max(e.y, f.y)); }
        if (j >= 1) { const int2 f = rin[row - 1]; e = make_int2(max(e.x, f.x), max(e.y, f.y)); }
        if (j + 1 < ny) { const int2 f = rin[row + 1]; e = make_int2(max(e.x, f.x), max(e.y, f.y)); }
        int k0 = nz, k1 = -1;                 // this sweep's range [k0, k1], widened by one cell
        if (e.y > 0) {
            k0 = max(nz - e.x - 1, 0);
            k1 = min(e.y, nz - 1);
        }
        if (!FINAL && threadIdx.x == 0)
            rout[row] = e.y > 0 ? make_int2(nz - k0, k1 + 1) : make_int2(0, 0);
        if (FINAL) {
            // every cell gets its final value; outside the range U is `big`, so the value is
            // sign(phi) * cap without the solve
            for (int k = threadIdx.x; k < nz; k += blockDim.x) {
                float v;
                if (k >= k0 && k <= k1) {
                    v = eik_sweep_cell_at<true, false>(in, base + k, i, j, k, x.g, dxf, big, cap,
                                                       x.phi);
                } else {
                    const float sg = x.phi[base + k] < 0.0f ? -1.0f : 1.0f;
                    v = __fadd_rn(__fmul_rn(sg, fminf(big, cap)), 0.0f);
                }
                x.phi[base + k] = v;
            }
        } else {
            for (int k = k0 + threadIdx.x; k <= k1; k += blockDim.x)
                out[base + k] = eik_sweep_cell_at<false, false>(in, base + k, i, j, k, x.g, dxf,
                                                                big, cap, x.phi);
        }
    }
}

__global__ void k_b_step(int* step) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *step += 1;
}

int make_table(const petch_batch_grid* grids, int B, BTable* t, long long* max_cells) {
    PETCH_REQUIRE(grids, "petch batch: null grid table");
    PETCH_REQUIRE(B >= 1 && B <= kMaxInst, "petch batch: 1 <= B <= %d", kMaxInst);
    t->B = B;
    long long mc = 0;
    for (int b = 0; b < B; ++b) {
        const petch_batch_grid& s = grids[b];
        PETCH_REQUIRE(s.phi && s.tmp && s.ua && s.ub && s.F && s.mask_phi && s.active &&
                          s.n_active && s.stats && s.hdr && s.sub && (s.n_mask == 0 || s.mask_idx),
                      "petch batch: grid %d incomplete", b);
        PETCH_REQUIRE(s.nx > 0 && s.ny > 0 && s.nz > 0 && s.dx > 0.0 && s.dt >= 0.0,
                      "petch batch: grid %d has a bad size", b);
        BGrid& x = t->it[b];
        x.phi = s.phi;
        x.tmp = s.tmp;
        x.ua = s.ua;
        x.ub = s.ub;
        x.F = s.F;
        x.mask_phi = s.mask_phi;
        x.mask_idx = s.mask_idx;
        x.n_mask = s.n_mask;
        x.active = s.active;
        x.n_active = s.n_active;
        x.max_active = s.max_active;
        x.g = make_lgrid(s.nx, s.ny, s.nz);
        x.dx = s.dx;
        x.dt = s.dt;
        x.stats = s.stats;
        x.hdr = s.hdr;
        x.sub = s.sub;
        x.hold = s.hold;
        if (x.g.n > mc) mc = x.g.n;
    }
    *max_cells = mc;
    return PETCH_OK;
}

}  // namespace
}  // namespace petch

using namespace petch;

extern "C" int petch_batch_advect(const petch_batch_grid* grids, int B, void* stream) {
    BTable t;
    long long mc = 0;
    int rc = make_table(grids, B, &t, &mc);
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    k_b_nsub<<<1, kMaxInst, 0, st>>>(t);
    PETCH_LAUNCH_CHECK("k_b_nsub");
    dim3 gc(grid_for(mc, kBB, 2), B);
    k_b_adv_prep<<<gc, kBB, 0, st>>>(t);
    PETCH_LAUNCH_CHECK("k_b_adv_prep");
    dim3 ga(grid_for(mc / 8 + 1, kBB, 2), B);
    for (int s = 0; s < kMaxSub; ++s) {
        k_b_adv_step<<<ga, kBB, 0, st>>>(t, s);
        PETCH_LAUNCH_CHECK("k_b_adv_step");
    }
    k_b_adv_finish<<<ga, kBB, 0, st>>>(t);
    PETCH_LAUNCH_CHECK("k_b_adv_finish");
    return PETCH_OK;
}

extern "C" int petch_batch_reinit(const petch_batch_grid* grids, int B, double band_r,
                                  void* stream) {
    BTable t;
    long long mc = 0;
    int rc = make_table(grids, B, &t, &mc);
    if (rc) return rc;
    const double dx = grids[0].dx;
    for (int b = 1; b < B; ++b)
        PETCH_REQUIRE(grids[b].dx == dx, "petch_batch_reinit: all grids need the same dx");
    for (int b = 0; b < B; ++b)   // two row-range arrays (16 bytes per row) fit in tmp
        PETCH_REQUIRE(grids[b].nz >= 4 && ((uintptr_t)grids[b].tmp & 7) == 0,
                      "petch_batch_reinit: grid %d needs nz >= 4 and an 8-byte aligned tmp", b);
    const int n_iter = (int)std::ceil(band_r / dx) + 4;
    cudaStream_t st = as_stream(stream);
    long long max_rows = 0;
    for (int b = 0; b < B; ++b) max_rows = std::max(max_rows, (long long)grids[b].nx * grids[b].ny);
    const RowShape rs = stencil_shape();
    const dim3 blk(rs.bz, rs.br);
    const dim3 gc(std::max(1, stencil_blocks(max_rows, rs) / std::max(1, B / 4)), B);
    k_b_rows_clear<<<dim3(grid_for(max_rows, kBB, 2), B), kBB, 0, st>>>(t);
    PETCH_LAUNCH_CHECK("k_b_rows_clear");
    k_b_eik_init<<<gc, blk, 0, st>>>(t, band_r);
    PETCH_LAUNCH_CHECK("k_b_eik_init");
    int parity = 0;
    for (int it = 0; it < n_iter - 1; ++it) {
        k_b_eik_sweep<false><<<gc, blk, 0, st>>>(t, band_r, parity);
        PETCH_LAUNCH_CHECK("k_b_eik_sweep");
        parity ^= 1;
    }
    k_b_eik_sweep<true><<<gc, blk, 0, st>>>(t, band_r, parity);
    PETCH_LAUNCH_CHECK("k_b_eik_sweep<final>");
    return PETCH_OK;
}

extern "C" int petch_batch_step_advance(int* step, void* stream) {
    PETCH_REQUIRE(step, "petch_batch_step_advance: null pointer");
    k_b_step<<<1, 32, 0, as_stream(stream)>>>(step);
    PETCH_LAUNCH_CHECK("k_b_step");
    return PETCH_OK;
}
