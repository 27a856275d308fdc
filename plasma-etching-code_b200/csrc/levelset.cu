// Level-set stencils: analytic seed field, first-order Godunov upwind advection, and the Jacobi
// Godunov-Eikonal reinitialisation.  All grids are (nx, ny, nz) C-order with z fastest.
//
// Each kernel is a grid-stride loop over cells; consecutive threads take consecutive z cells, so
// the centre and +-z loads are coalesced and the +-y / +-x neighbours hit lines that adjacent
// warps of the same block (y) or L2 (x) already hold.  The working set of the advection and
// reinit loops (three or four grids) stays resident in the 126 MB L2 for grids up to ~8M cells,
// so the repeated sweeps inside one etch step mostly run at L2 rather than HBM bandwidth.
#include "common.cuh"
#include "levelset.cuh"

namespace {

constexpr int kBlock = 256;

struct Grid {
    int nx, ny, nz;
    long long plane;  // ny * nz
    long long n;      // nx * ny * nz
};

__host__ __device__ inline Grid make_grid(int nx, int ny, int nz) {
    Grid g;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.plane = (long long)ny * nz;
    g.n = g.plane * nx;
    return g;
}

__device__ __forceinline__ void split(const Grid& g, long long c, int& i, int& j, int& k) {
    long long r = c / g.nz;
    k = (int)(c - r * g.nz);
    i = (int)(r / g.ny);
    j = (int)(r - (long long)i * g.ny);
}

// make_trench_3d's analytic CSG field (threed.py:51-55) and mask (threed.py:37-43), in double.
__global__ void k_seed(float* __restrict__ phi, uint8_t* __restrict__ mask, Grid g, double dx,
                       double Lx, double Ly, double sub_top, double mask_th, double width,
                       int hole) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.n;
         c += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        split(g, c, i, j, k);
        double X = i * dx, Y = j * dx, Z = k * dx;
        double ddx = X - Lx / 2.0, ddy = Y - Ly / 2.0;
        bool opening, band;
        double r;
        if (hole) {
            double r2 = ddx * ddx + ddy * ddy;
            opening = r2 < (width / 2.0) * (width / 2.0);
            r = sqrt(r2);
        } else {
            opening = fabs(ddx) < width / 2.0;
            r = fabs(ddx);
        }
        band = (Z >= sub_top) && (Z < sub_top + mask_th);
        double d_sub = sub_top - Z;
        double d_slab = fmin(Z - sub_top, sub_top + mask_th - Z);
        double d_mask = fmin(d_slab, r - width / 2.0);
        phi[c] = (float)fmax(d_sub, d_mask);
        mask[c] = (band && !opening) ? 1 : 0;
    }
}

// One advection substep (threed.py:1262-1292).  F == 0 cells keep phi exactly (the reference's
// phi - dt*0*sqrt(g) == phi), so they skip the neighbour loads.
template <bool MASK_ARRAY>
__global__ void __launch_bounds__(kBlock) k_advect(const float* __restrict__ phi,
                                                   float* __restrict__ out,
                                                   const float* __restrict__ F,
                                                   const uint8_t* __restrict__ mask,
                                                   const float* __restrict__ mask_phi, Grid g,
                                                   float inv_dx, float dt) {
    const petch::LGrid lg = petch::make_lgrid(g.nx, g.ny, g.nz);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.n;
         c += (long long)gridDim.x * blockDim.x) {
        float f = F[c];
        bool pinned = MASK_ARRAY ? (mask[c] != 0) : (f < 0.0f);
        if (pinned) {
            out[c] = mask_phi[c];
            continue;
        }
        float v = phi[c];
        if (f == 0.0f) {
            out[c] = v;
            continue;
        }
        out[c] = petch::advect_cell(phi, c, lg, inv_dx, f, dt);
    }
}

// The Eikonal passes, row-mapped (see petch::RowShape): threadIdx.x runs along z, threadIdx.y
// picks one of the block's rows, blocks stride over the nx * ny rows.
template <bool SEED>
__global__ void __launch_bounds__(kBlock) k_eik_init(const float* __restrict__ phi0,
                                                     float* __restrict__ U, Grid g, float inv_dx,
                                                     float big) {
    const petch::LGrid lg = petch::make_lgrid(g.nx, g.ny, g.nz);
    const int rows = g.nx * g.ny;
    for (int row = blockIdx.x * blockDim.y + threadIdx.y; row < rows; row += gridDim.x * blockDim.y) {
        const int i = row / g.ny, j = row - i * g.ny;
        const long long base = (long long)row * g.nz;
        for (int k = threadIdx.x; k < g.nz; k += blockDim.x)
            U[base + k] = petch::eik_init_cell_at<SEED>(phi0, base + k, i, j, k, lg, inv_dx, big);
    }
}

template <bool FINAL, bool SEED>
__global__ void __launch_bounds__(kBlock) k_eik_sweep(const float* __restrict__ Uin,
                                                      float* __restrict__ Uout,
                                                      const float* __restrict__ phi_in,
                                                      float* __restrict__ phi_out, Grid g,
                                                      float dx, float big, float cap) {
    const petch::LGrid lg = petch::make_lgrid(g.nx, g.ny, g.nz);
    const int rows = g.nx * g.ny;
    for (int row = blockIdx.x * blockDim.y + threadIdx.y; row < rows; row += gridDim.x * blockDim.y) {
        const int i = row / g.ny, j = row - i * g.ny;
        const long long base = (long long)row * g.nz;
        for (int k = threadIdx.x; k < g.nz; k += blockDim.x) {
            const float v = petch::eik_sweep_cell_at<FINAL, SEED>(Uin, base + k, i, j, k, lg, dx,
                                                                  big, cap, phi_in);
            if (FINAL) phi_out[base + k] = v;
            else Uout[base + k] = v;
        }
    }
}

// Block shape of the row-mapped stencils (petch_stencil_config): bz threads along z x br rows.
int g_row_bz = 128, g_row_br = 2;

}  // namespace

namespace petch {
RowShape stencil_shape() { return RowShape{g_row_bz, g_row_br}; }
int stencil_blocks(long long rows, const RowShape& s) {
    return grid_for(rows, s.br, 2048 / (s.bz * s.br));
}
}  // namespace petch

extern "C" int petch_stencil_config(int bz, int br) {
    PETCH_REQUIRE(bz >= 32 && bz % 32 == 0 && br >= 1 && bz * br <= kBlock,
                  "petch_stencil_config: bz a multiple of 32, bz * br <= %d (got %d x %d)", kBlock,
                  bz, br);
    g_row_bz = bz;
    g_row_br = br;
    return PETCH_OK;
}

extern "C" int petch_seed_level_set(float* phi, uint8_t* mask, int nx, int ny, int nz, double dx,
                                    double Lx, double Ly, double sub_top, double mask_th,
                                    double width, int hole, void* stream) {
    PETCH_REQUIRE(phi && mask, "petch_seed_level_set: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && dx > 0, "petch_seed_level_set: bad grid");
    Grid g = make_grid(nx, ny, nz);
    k_seed<<<petch::grid_for(g.n, kBlock), kBlock, 0, petch::as_stream(stream)>>>(
        phi, mask, g, dx, Lx, Ly, sub_top, mask_th, width, hole);
    PETCH_LAUNCH_CHECK("k_seed");
    return PETCH_OK;
}

extern "C" int petch_advect(float* phi, float* tmp, const float* F, const uint8_t* mask,
                            const float* mask_phi, int nx, int ny, int nz, float inv_dx,
                            float dt_sub, int nsub, void* stream) {
    PETCH_REQUIRE(phi && tmp && F && mask_phi, "petch_advect: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0, "petch_advect: bad grid %d %d %d", nx, ny, nz);
    PETCH_REQUIRE(nsub >= 0, "petch_advect: nsub must be >= 0");
    PETCH_REQUIRE(phi != tmp, "petch_advect: phi and tmp must differ");
    Grid g = make_grid(nx, ny, nz);
    cudaStream_t st = petch::as_stream(stream);
    int blocks = petch::grid_for(g.n, kBlock);
    float* a = phi;
    float* b = tmp;
    for (int s = 0; s < nsub; ++s) {
        if (mask)
            k_advect<true><<<blocks, kBlock, 0, st>>>(a, b, F, mask, mask_phi, g, inv_dx, dt_sub);
        else
            k_advect<false><<<blocks, kBlock, 0, st>>>(a, b, F, mask, mask_phi, g, inv_dx, dt_sub);
        PETCH_LAUNCH_CHECK("k_advect");
        float* t = a;
        a = b;
        b = t;
    }
    if (a != phi)
        PETCH_CUDA(cudaMemcpyAsync(phi, a, sizeof(float) * g.n, cudaMemcpyDeviceToDevice, st),
                   "petch_advect copy-back");
    return PETCH_OK;
}

extern "C" int petch_reinit_eik(const float* phi_in, float* phi_out, float* u_a, float* u_b,
                                int nx, int ny, int nz, double dx, float big, float cap, int n_iter,
                                int mode, void* stream) {
    PETCH_REQUIRE(phi_in && phi_out && u_a && u_b, "petch_reinit_eik: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && dx > 0, "petch_reinit_eik: bad grid");
    PETCH_REQUIRE(n_iter >= 1, "petch_reinit_eik: n_iter must be >= 1");
    PETCH_REQUIRE(u_a != u_b && (float*)phi_in != u_a && (float*)phi_in != u_b &&
                      phi_out != u_a && phi_out != u_b,
                  "petch_reinit_eik: scratch buffers must be distinct from phi");
    Grid g = make_grid(nx, ny, nz);
    cudaStream_t st = petch::as_stream(stream);
    const petch::RowShape rs = petch::stencil_shape();
    const dim3 blk(rs.bz, rs.br);
    const int blocks = petch::stencil_blocks((long long)nx * ny, rs);
    const float dxf = (float)dx, inv_dx = (float)(1.0 / dx);
    PETCH_REQUIRE(mode == 0 || mode == 1, "petch_reinit_eik: mode must be 0 or 1");
    if (mode == 1) k_eik_init<true><<<blocks, blk, 0, st>>>(phi_in, u_a, g, inv_dx, big);
    else k_eik_init<false><<<blocks, blk, 0, st>>>(phi_in, u_a, g, inv_dx, big);
    PETCH_LAUNCH_CHECK("k_eik_init");
    float* a = u_a;
    float* b = u_b;
    for (int it = 0; it < n_iter - 1; ++it) {
        k_eik_sweep<false, false><<<blocks, blk, 0, st>>>(a, b, nullptr, nullptr, g, dxf, big, cap);
        PETCH_LAUNCH_CHECK("k_eik_sweep");
        float* t = a;
        a = b;
        b = t;
    }
    if (mode == 1)
        k_eik_sweep<true, true><<<blocks, blk, 0, st>>>(a, nullptr, phi_in, phi_out, g, dxf, big, cap);
    else
        k_eik_sweep<true, false><<<blocks, blk, 0, st>>>(a, nullptr, phi_in, phi_out, g, dxf, big, cap);
    PETCH_LAUNCH_CHECK("k_eik_sweep<final>");
    return PETCH_OK;
}

// ---------------------------------------------------------------------------------------------
// Allocation-free reinit.  Some callers cannot allocate device memory at all: a host application
// or plugin framework that owns the whole device heap and forbids driver allocations, or a
// fixed-budget real-time loop where an allocation's latency and implicit device synchronisation
// are not acceptable.  They still own their input and output grids, but cannot provide the two
// Eikonal scratch grids petch_reinit_eik needs.  This variant keeps that scratch in a fixed
// file-scope device array instead.
//
// The array is part of the library's device image: every GPU that loads the library holds it
// (16 MiB) until the process exits.  Its host-side name is only a stand-in for the symbol, so
// the device address is looked up with cudaGetSymbolAddress once per device, on the first call
// made with that device current; make that first call before any stream capture.  All calls
// share the one array, so calls whose kernels overlap on the GPU (different streams, threads or
// processes sharing a context) race on it.  Nothing carries over between calls: the init kernel
// writes every scratch cell before any sweep reads it.
// ---------------------------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr long long kNoAllocMaxCells = 1LL << 21;   // 2,097,152 cells (e.g. 128^3): 8 MiB a grid

__device__ __align__(256) float g_reinit_scratch[2 * kNoAllocMaxCells];

float* g_scratch_addr[64] = {nullptr};
std::mutex g_scratch_mu;

int reinit_scratch_address(float** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return petch::cuda_fail(e, "petch_reinit_eik_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= 64) {
        petch::set_error("petch_reinit_eik_noalloc: device ordinal %d out of range", dev);
        return PETCH_E_INVALID;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (g_scratch_addr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_reinit_scratch);
        if (e != cudaSuccess)
            return petch::cuda_fail(e, "petch_reinit_eik_noalloc: cudaGetSymbolAddress");
        g_scratch_addr[dev] = static_cast<float*>(p);
    }
    *out = g_scratch_addr[dev];
    return PETCH_OK;
}

}  // namespace

extern "C" int petch_reinit_eik_noalloc(const float* phi_in, float* phi_out, int nx, int ny, int nz,
                                        double dx, float big, float cap, int n_iter, int mode,
                                        void* stream) {
    PETCH_REQUIRE(phi_in && phi_out, "petch_reinit_eik_noalloc: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && dx > 0, "petch_reinit_eik_noalloc: bad grid");
    PETCH_REQUIRE(n_iter >= 1, "petch_reinit_eik_noalloc: n_iter must be >= 1");
    PETCH_REQUIRE(mode == 0 || mode == 1, "petch_reinit_eik_noalloc: mode must be 0 or 1");
    const long long cells = (long long)nx * ny * nz;
    PETCH_REQUIRE(cells <= kNoAllocMaxCells,
                  "petch_reinit_eik_noalloc: grid of %lld cells exceeds the fixed scratch of %lld "
                  "cells (use petch_reinit_eik with caller scratch)",
                  cells, kNoAllocMaxCells);
    float* base = nullptr;
    int rc = reinit_scratch_address(&base);
    if (rc) return rc;
    float* a = base;
    float* b = base + kNoAllocMaxCells;
    Grid g = make_grid(nx, ny, nz);
    cudaStream_t st = petch::as_stream(stream);
    const petch::RowShape rs = petch::stencil_shape();
    const dim3 blk(rs.bz, rs.br);
    const int blocks = petch::stencil_blocks((long long)nx * ny, rs);
    const float dxf = (float)dx, inv_dx = (float)(1.0 / dx);
    if (mode == 1) k_eik_init<true><<<blocks, blk, 0, st>>>(phi_in, a, g, inv_dx, big);
    else k_eik_init<false><<<blocks, blk, 0, st>>>(phi_in, a, g, inv_dx, big);
    PETCH_LAUNCH_CHECK("k_eik_init");
    for (int it = 0; it < n_iter - 1; ++it) {
        k_eik_sweep<false, false><<<blocks, blk, 0, st>>>(a, b, nullptr, nullptr, g, dxf, big, cap);
        PETCH_LAUNCH_CHECK("k_eik_sweep");
        float* t = a;
        a = b;
        b = t;
    }
    if (mode == 1)
        k_eik_sweep<true, true><<<blocks, blk, 0, st>>>(a, nullptr, phi_in, phi_out, g, dxf, big, cap);
    else
        k_eik_sweep<true, false><<<blocks, blk, 0, st>>>(a, nullptr, phi_in, phi_out, g, dxf, big, cap);
    PETCH_LAUNCH_CHECK("k_eik_sweep<final>");
    return PETCH_OK;
}
