// The level-set options of run_etch_3d beside the default path:
//   * reinit_method="gpu": the PDE reinitialisation phi_tau + sgn(phi0)(|grad phi| - 1) = 0 with
//     the Russo-Smereka sub-cell fix at interface cells (reinit_gpu / _reinit_iter,
//     petch/threed.py:1349-1418), n_iter forward-Euler sweeps of step 0.3 dx;
//   * surf_smooth > 0: scipy.ndimage.gaussian_filter(phi, surf_smooth) and the mask re-pin
//     (petch/threed.py:1779-1782): three separable passes (axis 0, 1, 2) of the normalised
//     Gaussian truncated at int(truncate * sigma + 0.5) cells, 'reflect' boundaries
//     (d c b a | a b c d | d c b a), accumulated in double.
// Both are memory-bound stencils: one read of each input cell (neighbours come from L1 / L2) and
// one write per pass.
#include <cmath>
#include "common.cuh"

namespace {

constexpr int kLB = 256;
constexpr int kMaxRadius = 64;

struct G3 {
    int nx, ny, nz;
    long long plane, n;
};

G3 make_g3(int nx, int ny, int nz) {
    G3 g{nx, ny, nz, (long long)ny * nz, 0};
    g.n = g.plane * nx;
    return g;
}

__device__ __forceinline__ void split3(const G3& g, long long c, int& i, int& j, int& k) {
    long long r = c / g.nz;
    k = (int)(c - r * g.nz);
    i = (int)(r / g.ny);
    j = (int)(r - (long long)i * g.ny);
}

// One sweep of _reinit_iter (float32 arithmetic, clamped neighbour indices).
__global__ void __launch_bounds__(kLB) k_reinit_pde(const float* __restrict__ phi,
                                                    const float* __restrict__ phi0,
                                                    float* __restrict__ out, G3 g, float inv_dx,
                                                    float dtau) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.n;
         c += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        split3(g, c, i, j, k);
        const long long xm = c - (i > 0 ? g.plane : 0), xp = c + (i < g.nx - 1 ? g.plane : 0);
        const long long ym = c - (j > 0 ? g.nz : 0), yp = c + (j < g.ny - 1 ? g.nz : 0);
        const long long zm = c - (k > 0 ? 1 : 0), zp = c + (k < g.nz - 1 ? 1 : 0);
        const float v = phi[c];
        const float s0 = phi0[c];
        const float o_xm = phi0[xm], o_xp = phi0[xp], o_ym = phi0[ym], o_yp = phi0[yp];
        const float o_zm = phi0[zm], o_zp = phi0[zp];
        const bool interface = (s0 * o_xm < 0.0f) || (s0 * o_xp < 0.0f) || (s0 * o_ym < 0.0f) ||
                               (s0 * o_yp < 0.0f) || (s0 * o_zm < 0.0f) || (s0 * o_zp < 0.0f);
        if (interface) {
            const float gx0 = (o_xp - o_xm) * 0.5f * inv_dx;
            const float gy0 = (o_yp - o_ym) * 0.5f * inv_dx;
            const float gz0 = (o_zp - o_zm) * 0.5f * inv_dx;
            const float grad0 = fmaxf(sqrtf(gx0 * gx0 + gy0 * gy0 + gz0 * gz0), 0.5f);
            const float dxl = 1.0f / inv_dx;
            const float D = fminf(fmaxf(s0 / grad0, -1.8f * dxl), 1.8f * dxl);
            const float sgn0 = s0 < 0.0f ? -1.0f : 1.0f;
            out[c] = v - dtau * inv_dx * (sgn0 * fabsf(v) - D);
            continue;
        }
        const float Dxm = (v - phi[xm]) * inv_dx, Dxp = (phi[xp] - v) * inv_dx;
        const float Dym = (v - phi[ym]) * inv_dx, Dyp = (phi[yp] - v) * inv_dx;
        const float Dzm = (v - phi[zm]) * inv_dx, Dzp = (phi[zp] - v) * inv_dx;
        const float sgn = s0 / sqrtf(s0 * s0 + 0.25f / (inv_dx * inv_dx));
        float gx, gy, gz;
        if (sgn > 0.0f) {
            gx = fmaxf(fmaxf(Dxm, 0.0f), -fminf(Dxp, 0.0f));
            gy = fmaxf(fmaxf(Dym, 0.0f), -fminf(Dyp, 0.0f));
            gz = fmaxf(fmaxf(Dzm, 0.0f), -fminf(Dzp, 0.0f));
        } else {
            gx = fmaxf(-fminf(Dxm, 0.0f), fmaxf(Dxp, 0.0f));
            gy = fmaxf(-fminf(Dym, 0.0f), fmaxf(Dyp, 0.0f));
            gz = fmaxf(-fminf(Dzm, 0.0f), fmaxf(Dzp, 0.0f));
        }
        const float Gm = sqrtf(gx * gx + gy * gy + gz * gz);
        out[c] = v - dtau * sgn * (Gm - 1.0f);
    }
}

struct Taps {
    double w[2 * kMaxRadius + 1];
    int radius;
};

// scipy's 'reflect' extension: half-sample symmetric with period 2n.
__device__ __forceinline__ int reflect_index(int i, int n) {
    if (n == 1) return 0;
    const int p = 2 * n;
    int m = i % p;
    if (m < 0) m += p;
    return m < n ? m : p - 1 - m;
}

// One 1-D Gaussian pass along `axis`; the last pass re-pins mask cells to mask_phi.
__global__ void __launch_bounds__(kLB) k_gauss_pass(const float* __restrict__ in,
                                                    float* __restrict__ out, G3 g, int axis,
                                                    Taps taps, const uint8_t* __restrict__ mask,
                                                    const float* __restrict__ mask_phi) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.n;
         c += (long long)gridDim.x * blockDim.x) {
        if (mask && mask[c]) {
            out[c] = mask_phi[c];
            continue;
        }
        int i, j, k;
        split3(g, c, i, j, k);
        const int pos = axis == 0 ? i : (axis == 1 ? j : k);
        const int n = axis == 0 ? g.nx : (axis == 1 ? g.ny : g.nz);
        const long long stride = axis == 0 ? g.plane : (axis == 1 ? (long long)g.nz : 1LL);
        const long long base = c - (long long)pos * stride;
        double acc = 0.0;
        for (int t = -taps.radius; t <= taps.radius; ++t) {
            const int q = reflect_index(pos + t, n);
            acc += taps.w[t + taps.radius] * (double)in[base + (long long)q * stride];
        }
        out[c] = (float)acc;
    }
}

// The floor of a column for the depth metrics (threed.py:1822-1830): column (i, j) of phi is the
// contiguous run phi[(i ny + j) nz + k], k = 0..nz-1.  A column whose top cell is not gas
// (phi < 0) has no floor (-1); otherwise the floor is the lowest cell of the gas run that reaches
// the top: one above the highest non-gas cell, 0 when every cell is gas.  One warp per column
// scans 32 cells at a time from the top; the first chunk holding a non-gas cell ends the scan.
// A column index outside the grid gives -2.
__global__ void k_column_floors(const float* __restrict__ phi, int nx, int ny, int nz,
                                const int* __restrict__ cols, int n_cols, int* __restrict__ k_out) {
    const int lane = threadIdx.x & 31;
    const int c = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    if (c >= n_cols) return;
    const int i = cols[2 * c], j = cols[2 * c + 1];
    if (i < 0 || i >= nx || j < 0 || j >= ny) {
        if (lane == 0) k_out[c] = -2;
        return;
    }
    const float* col = phi + ((long long)i * ny + j) * nz;
    if (!(col[nz - 1] < 0.0f)) {
        if (lane == 0) k_out[c] = -1;
        return;
    }
    int k = 0;
    for (int start = nz - 1; start >= 0; start -= 32) {
        const int idx = start - lane;
        const bool solid = idx >= 0 && !(col[idx] < 0.0f);
        const unsigned m = __ballot_sync(0xffffffffu, solid);
        if (m) {
            k = start - (__ffs(m) - 1) + 1;
            break;
        }
    }
    if (lane == 0) k_out[c] = k;
}

}  // namespace

using namespace petch;

extern "C" int petch_column_floors(const float* phi, int nx, int ny, int nz, const int* cols,
                                   int n_cols, int* k_out, void* stream) {
    PETCH_REQUIRE(phi && (n_cols == 0 || (cols && k_out)), "petch_column_floors: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && n_cols >= 0, "petch_column_floors: bad size");
    if (n_cols == 0) return PETCH_OK;
    const long long threads = 32LL * n_cols;
    k_column_floors<<<(unsigned)((threads + 255) / 256), 256, 0, as_stream(stream)>>>(
        phi, nx, ny, nz, cols, n_cols, k_out);
    PETCH_LAUNCH_CHECK("k_column_floors");
    return PETCH_OK;
}

extern "C" int petch_reinit_pde(const float* phi_in, float* phi_out, float* phi0, float* tmp,
                                int nx, int ny, int nz, double dx, int n_iter, void* stream) {
    PETCH_REQUIRE(phi_in && phi_out && phi0 && tmp, "petch_reinit_pde: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && dx > 0.0 && n_iter >= 0,
                  "petch_reinit_pde: bad grid or iteration count");
    PETCH_REQUIRE(phi_out != tmp && phi0 != tmp && phi0 != phi_out,
                  "petch_reinit_pde: phi_out, phi0 and tmp must be distinct");
    cudaStream_t st = as_stream(stream);
    const G3 g = make_g3(nx, ny, nz);
    const size_t bytes = sizeof(float) * (size_t)g.n;
    PETCH_CUDA(cudaMemcpyAsync(phi0, phi_in, bytes, cudaMemcpyDeviceToDevice, st), "copy phi0");
    if (n_iter == 0) {
        if (phi_out != phi_in)
            PETCH_CUDA(cudaMemcpyAsync(phi_out, phi_in, bytes, cudaMemcpyDeviceToDevice, st),
                       "copy phi");
        return PETCH_OK;
    }
    const float inv_dx = (float)(1.0 / dx), dtau = (float)(0.3 * dx);
    // ping-pong so that the last sweep lands in phi_out: sweep s reads src, writes dst
    const int blocks = grid_for(g.n, kLB);
    const float* src = phi0;
    for (int s = 0; s < n_iter; ++s) {
        float* dst = ((n_iter - 1 - s) % 2 == 0) ? phi_out : tmp;
        k_reinit_pde<<<blocks, kLB, 0, st>>>(src, phi0, dst, g, inv_dx, dtau);
        PETCH_LAUNCH_CHECK("k_reinit_pde");
        src = dst;
    }
    return PETCH_OK;
}

extern "C" int petch_gaussian_smooth(float* phi, float* tmp_a, float* tmp_b, const uint8_t* mask,
                                     const float* mask_phi, int nx, int ny, int nz, double sigma,
                                     double truncate, void* stream) {
    PETCH_REQUIRE(phi && tmp_a && tmp_b, "petch_gaussian_smooth: null pointer");
    PETCH_REQUIRE((mask == nullptr) == (mask_phi == nullptr),
                  "petch_gaussian_smooth: pass mask and mask_phi together");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && sigma > 0.0 && truncate > 0.0,
                  "petch_gaussian_smooth: bad grid or sigma");
    const int radius = (int)(truncate * sigma + 0.5);
    PETCH_REQUIRE(radius <= kMaxRadius, "petch_gaussian_smooth: truncate * sigma exceeds %d cells",
                  kMaxRadius);
    Taps taps;
    taps.radius = radius;
    double sum = 0.0;
    for (int t = -radius; t <= radius; ++t) {
        taps.w[t + radius] = std::exp(-0.5 / (sigma * sigma) * (double)t * (double)t);
        sum += taps.w[t + radius];
    }
    for (int t = 0; t <= 2 * radius; ++t) taps.w[t] /= sum;
    cudaStream_t st = as_stream(stream);
    const G3 g = make_g3(nx, ny, nz);
    const int blocks = grid_for(g.n, kLB);
    k_gauss_pass<<<blocks, kLB, 0, st>>>(phi, tmp_a, g, 0, taps, nullptr, nullptr);
    PETCH_LAUNCH_CHECK("k_gauss_pass");
    k_gauss_pass<<<blocks, kLB, 0, st>>>(tmp_a, tmp_b, g, 1, taps, nullptr, nullptr);
    PETCH_LAUNCH_CHECK("k_gauss_pass");
    k_gauss_pass<<<blocks, kLB, 0, st>>>(tmp_b, phi, g, 2, taps, mask, mask_phi);
    PETCH_LAUNCH_CHECK("k_gauss_pass");
    return PETCH_OK;
}
