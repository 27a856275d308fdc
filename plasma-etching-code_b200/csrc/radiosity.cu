// Deterministic radiosity neutral transport (mc_flux_3d_radiosity, petch/threed.py:923-991).
//
// The form-factor rays themselves are traced by the persistent tracer (petch_trace_ff in
// trace.cu); this file holds the rest of the path:
//   * the into-gas face normals the rays leave along (_gas_normals, threed.py:1553-1568);
//   * the sparse matrix A[i, j] = (rays from face j whose first hit is face i) / n_ff as a CSR
//     over rows i, built without host synchronisation: hit counts per row by integer atomics, an
//     exclusive scan for the row offsets, and a stable radix sort of (hit face, source face) so
//     the entries of a row keep the ray order -- the matrix, and every sum over it, is the same
//     bit for bit on every run;
//   * D[i] = escaping rays of face i / n_ff (the sky view);
//   * the Jacobi iteration G <- D + M G with M[i, j] = A[i, j] (1 - clip(bare_j beta, 0, 1)),
//     both species (betaE, betaO) at once because they share the coverage, in float64, one warp
//     per row, one launch per iteration.
#include <cub/cub.cuh>
#include "common.cuh"
#include "mesh.cuh"
#include "petch_b200.h"

namespace petch {
namespace {

constexpr int kRB = 256;

// _gas_normals: the winding normal normalize(cross(b - a, c - a)) (float32, as numpy computes it
// on the float32 vertices), flipped where it points against -grad(phi) sampled at the grid node
// nearest the centroid (np.gradient: central differences inside, one-sided at the faces; indices
// rounded half to even and clipped to the grid).
__global__ void k_gas_normals(MeshView m, const float* __restrict__ phi, int nx, int ny, int nz,
                              double dx, float* __restrict__ fn) {
    const int F = min(m.hdr[HDR_F], m.MT);
    const long long sy = nz, sx = (long long)ny * nz;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x) {
        const int a = m.faces[3 * f], b = m.faces[3 * f + 1], c = m.faces[3 * f + 2];
        const float ax = m.verts[3 * a], ay = m.verts[3 * a + 1], az = m.verts[3 * a + 2];
        const float e1x = __fsub_rn(m.verts[3 * b], ax), e1y = __fsub_rn(m.verts[3 * b + 1], ay),
                    e1z = __fsub_rn(m.verts[3 * b + 2], az);
        const float e2x = __fsub_rn(m.verts[3 * c], ax), e2y = __fsub_rn(m.verts[3 * c + 1], ay),
                    e2z = __fsub_rn(m.verts[3 * c + 2], az);
        float n0 = __fsub_rn(__fmul_rn(e1y, e2z), __fmul_rn(e1z, e2y));
        float n1 = __fsub_rn(__fmul_rn(e1z, e2x), __fmul_rn(e1x, e2z));
        float n2 = __fsub_rn(__fmul_rn(e1x, e2y), __fmul_rn(e1y, e2x));
        const float len = __fadd_rn(
            __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(n0, n0), __fmul_rn(n1, n1)), __fmul_rn(n2, n2))),
            1.0e-12f);
        n0 = __fdiv_rn(n0, len);
        n1 = __fdiv_rn(n1, len);
        n2 = __fdiv_rn(n2, len);
        int idx[3];
        const int ext[3] = {nx, ny, nz};
        for (int q = 0; q < 3; ++q) {
            double r = rint((double)m.centroid[3 * f + q] / dx);
            r = fmin(fmax(r, 0.0), (double)(ext[q] - 1));
            idx[q] = (int)r;
        }
        const long long base = idx[0] * sx + idx[1] * sy + idx[2];
        const long long str[3] = {sx, sy, 1};
        double g[3];
        for (int q = 0; q < 3; ++q) {
            const int i = idx[q], n = ext[q];
            if (n < 2) {
                g[q] = 0.0;
            } else if (i == 0) {
                g[q] = ((double)phi[base + str[q]] - (double)phi[base]) / dx;
            } else if (i == n - 1) {
                g[q] = ((double)phi[base] - (double)phi[base - str[q]]) / dx;
            } else {
                g[q] = ((double)phi[base + str[q]] - (double)phi[base - str[q]]) / (2.0 * dx);
            }
        }
        // into-gas = -grad(phi); flip where the normal points the other way
        const double dd = -((double)n0 * g[0] + (double)n1 * g[1] + (double)n2 * g[2]);
        if (dd < 0.0) {
            n0 = -n0;
            n1 = -n1;
            n2 = -n2;
        }
        fn[3 * f] = n0;
        fn[3 * f + 1] = n1;
        fn[3 * f + 2] = n2;
    }
}

// Per ray p (source face j = p / n_ff): sort key = hit face (F for an escape, MT past the live
// rays), value = j; row counts and escape counts by integer atomics.
__global__ void k_ff_keys(const int* __restrict__ hdr, int MT, const int* __restrict__ hit, int n_ff,
                          unsigned* __restrict__ keys, int* __restrict__ vals, int* __restrict__ cnt,
                          int* __restrict__ esc) {
    const int F = min(hdr[HDR_F], MT);
    const long long live = (long long)F * n_ff, n = (long long)MT * n_ff;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(p / n_ff);
        unsigned key = (unsigned)MT;
        if (p < live) {
            const int h = hit[p];
            if (h >= 0 && h < F) {
                key = (unsigned)h;
                atomicAdd(cnt + h, 1);
            } else {
                key = (unsigned)F;
                atomicAdd(esc + j, 1);
            }
        }
        keys[p] = key;
        vals[p] = j;
    }
}

__global__ void k_ff_sky(const int* __restrict__ hdr, int MT, const int* __restrict__ esc, int n_ff,
                         double* __restrict__ D) {
    const int F = min(hdr[HDR_F], MT);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
        D[i] = (double)esc[i] / (double)n_ff;
}

// One Jacobi iteration for both species, a group of kG lanes per row i (32 / kG rows per warp):
//   G_i = D_i + (1 / n_ff) * sum over the row's entries j of x_j,
// where x_j = (1 - s_j) G_j from the previous iteration (x = y_in), or (1 - s_j) D_j on the first
// (y_in == nullptr), s = clip(bare * beta, 0, 1).  The last iteration writes clip(G, 0, 8) as
// float; the others write x_i = (1 - s_i) G_i for the next.  Lane q of a group sums entries
// q, q + kG, q + 2 kG, ... and the group reduces with a fixed butterfly, so every run sums in the
// same order.
constexpr int kG = 8;

__global__ void __launch_bounds__(kRB) k_rad_iter(const int* __restrict__ hdr, int MT,
                                                  const int* __restrict__ row_ptr,
                                                  const int* __restrict__ col,
                                                  const double* __restrict__ D,
                                                  const float* __restrict__ bare, double betaE,
                                                  double betaO, double inv_nff,
                                                  const double2* __restrict__ y_in,
                                                  double2* __restrict__ y_out, float* __restrict__ gE,
                                                  float* __restrict__ gO) {
    const int F = min(hdr[HDR_F], MT);
    const int sub = threadIdx.x & (kG - 1);
    const int groups = (gridDim.x * blockDim.x) / kG;
    // every lane of a warp runs the same number of trips (the warp's groups share the loop
    // bound), so the butterfly below always has the full warp converged
    const int first = (blockIdx.x * blockDim.x + threadIdx.x) / kG;
    const int warp_first = first - ((threadIdx.x & 31) / kG);
    for (int base = warp_first; base < F; base += groups) {
        const int i = base + ((threadIdx.x & 31) / kG);
        double sE = 0.0, sO = 0.0;
        if (i < F) {
            const int e0 = row_ptr[i], e1 = row_ptr[i + 1];
            if (y_in) {
                for (int e = e0 + sub; e < e1; e += kG) {
                    const double2 x = y_in[__ldg(col + e)];
                    sE += x.x;
                    sO += x.y;
                }
            } else {
                for (int e = e0 + sub; e < e1; e += kG) {
                    const int j = __ldg(col + e);
                    const double b = (double)__ldg(bare + j), dj = __ldg(D + j);
                    sE += (1.0 - fmin(fmax(b * betaE, 0.0), 1.0)) * dj;
                    sO += (1.0 - fmin(fmax(b * betaO, 0.0), 1.0)) * dj;
                }
            }
        }
        for (int o = kG / 2; o > 0; o >>= 1) {
            sE += __shfl_xor_sync(0xffffffffu, sE, o);
            sO += __shfl_xor_sync(0xffffffffu, sO, o);
        }
        if (sub == 0 && i < F) {
            const double GE = D[i] + inv_nff * sE, GO = D[i] + inv_nff * sO;
            if (gE) {
                gE[i] = (float)fmin(fmax(GE, 0.0), 8.0);
                gO[i] = (float)fmin(fmax(GO, 0.0), 8.0);
            } else {
                const double b = (double)bare[i];
                y_out[i] = make_double2((1.0 - fmin(fmax(b * betaE, 0.0), 1.0)) * GE,
                                        (1.0 - fmin(fmax(b * betaO, 0.0), 1.0)) * GO);
            }
        }
    }
}

__global__ void k_rad_sky_only(const int* __restrict__ hdr, int MT, const double* __restrict__ D,
                               float* __restrict__ gE, float* __restrict__ gO) {
    const int F = min(hdr[HDR_F], MT);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x) {
        const float v = (float)fmin(fmax(D[i], 0.0), 8.0);
        gE[i] = v;
        gO[i] = v;
    }
}

int key_bits(int MT) {
    int b = 1;
    while (b < 31 && (1LL << b) <= (long long)MT) ++b;
    return b;
}

// Scratch of petch_ff_matrix: keys, sorted keys, values, row / escape counts, CUB temporaries.
struct FFScratch {
    unsigned* keys;
    unsigned* keys_out;
    int* vals;
    int* cnt;
    int* esc;
    void* cub_tmp;
    size_t cub_bytes;
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

int ff_layout(int MT, int n_ff, void* base, size_t* total, FFScratch* s) {
    const long long n = (long long)MT * n_ff;
    size_t sort_bytes = 0, scan_bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (unsigned*)nullptr,
                                                    (unsigned*)nullptr, (int*)nullptr, (int*)nullptr,
                                                    (int)n, 0, key_bits(MT));
    if (e != cudaSuccess) return cuda_fail(e, "petch_ff_matrix: sort size query");
    e = cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (int*)nullptr, (int*)nullptr, MT + 1);
    if (e != cudaSuccess) return cuda_fail(e, "petch_ff_matrix: scan size query");
    const size_t cub_bytes = sort_bytes > scan_bytes ? sort_bytes : scan_bytes;
    size_t off = 0;
    char* b = (char*)base;
    auto take = [&](size_t bytes) {
        char* p = b ? b + off : nullptr;
        off += align256(bytes);
        return (void*)p;
    };
    FFScratch t;
    t.keys = (unsigned*)take(sizeof(unsigned) * n);
    t.keys_out = (unsigned*)take(sizeof(unsigned) * n);
    t.vals = (int*)take(sizeof(int) * n);
    t.cnt = (int*)take(sizeof(int) * ((size_t)MT + 1));
    t.esc = (int*)take(sizeof(int) * (size_t)MT);
    t.cub_tmp = take(cub_bytes);
    t.cub_bytes = cub_bytes;
    *total = off;
    if (s) *s = t;
    return PETCH_OK;
}

}  // namespace
}  // namespace petch

using namespace petch;

extern "C" int petch_gas_normals(const void* mesh, int max_tris, int max_verts, const float* phi,
                                 int nx, int ny, int nz, double dx, float* fn, void* stream) {
    PETCH_REQUIRE(mesh && phi && fn, "petch_gas_normals: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && dx > 0.0, "petch_gas_normals: bad grid");
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    k_gas_normals<<<grid_for(max_tris, kRB), kRB, 0, as_stream(stream)>>>(m, phi, nx, ny, nz, dx, fn);
    PETCH_LAUNCH_CHECK("k_gas_normals");
    return PETCH_OK;
}

extern "C" int petch_ff_scratch_bytes(int max_tris, int n_ff, long long* bytes) {
    PETCH_REQUIRE(bytes, "petch_ff_scratch_bytes: null pointer");
    PETCH_REQUIRE(max_tris > 0 && n_ff >= 1 && (long long)max_tris * n_ff < (1LL << 31),
                  "petch_ff_scratch_bytes: max_tris * n_ff must be in [1, 2^31)");
    size_t total = 0;
    int rc = ff_layout(max_tris, n_ff, nullptr, &total, nullptr);
    if (rc) return rc;
    *bytes = (long long)total;
    return PETCH_OK;
}

extern "C" int petch_ff_matrix(const void* mesh, int max_tris, int max_verts, const int* hitface,
                               int n_ff, int* row_ptr, int* col, double* sky, void* scratch,
                               long long scratch_bytes, void* stream) {
    PETCH_REQUIRE(mesh && hitface && row_ptr && col && sky && scratch,
                  "petch_ff_matrix: null pointer");
    PETCH_REQUIRE(max_tris > 0 && n_ff >= 1 && (long long)max_tris * n_ff < (1LL << 31),
                  "petch_ff_matrix: max_tris * n_ff must be in [1, 2^31)");
    size_t need = 0;
    FFScratch s;
    int rc = ff_layout(max_tris, n_ff, scratch, &need, &s);
    if (rc) return rc;
    PETCH_REQUIRE((long long)need <= scratch_bytes, "petch_ff_matrix: scratch too small");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    const long long n = (long long)max_tris * n_ff;
    PETCH_CUDA(cudaMemsetAsync(s.cnt, 0, sizeof(int) * ((size_t)max_tris + 1), st), "memset counts");
    PETCH_CUDA(cudaMemsetAsync(s.esc, 0, sizeof(int) * (size_t)max_tris, st), "memset escapes");
    k_ff_keys<<<grid_for(n, kRB, 16), kRB, 0, st>>>(m.hdr, max_tris, hitface, n_ff, s.keys, s.vals,
                                                    s.cnt, s.esc);
    PETCH_LAUNCH_CHECK("k_ff_keys");
    k_ff_sky<<<grid_for(max_tris, kRB), kRB, 0, st>>>(m.hdr, max_tris, s.esc, n_ff, sky);
    PETCH_LAUNCH_CHECK("k_ff_sky");
    size_t cb = s.cub_bytes;
    PETCH_CUDA(cub::DeviceScan::ExclusiveSum(s.cub_tmp, cb, s.cnt, row_ptr, max_tris + 1, st),
               "row offsets scan");
    cb = s.cub_bytes;
    // stable: the entries of a row keep ascending ray (hence source face) order
    PETCH_CUDA(cub::DeviceRadixSort::SortPairs(s.cub_tmp, cb, s.keys, s.keys_out, s.vals, col,
                                               (int)n, 0, key_bits(max_tris), st),
               "sort by hit face");
    return PETCH_OK;
}

extern "C" int petch_radiosity_solve(const void* mesh, int max_tris, int max_verts,
                                     const int* row_ptr, const int* col, const double* sky,
                                     int n_ff, const float* bare, double betaE, double betaO,
                                     int n_iter, float* g_E, float* g_O, double* work2,
                                     void* stream) {
    PETCH_REQUIRE(mesh && row_ptr && col && sky && bare && g_E && g_O && work2,
                  "petch_radiosity_solve: null pointer");
    PETCH_REQUIRE(max_tris > 0 && n_ff >= 1 && n_iter >= 0, "petch_radiosity_solve: bad size");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    if (n_iter == 0) {
        k_rad_sky_only<<<grid_for(max_tris, kRB), kRB, 0, st>>>(m.hdr, max_tris, sky, g_E, g_O);
        PETCH_LAUNCH_CHECK("k_rad_sky_only");
        return PETCH_OK;
    }
    double2* ya = reinterpret_cast<double2*>(work2);
    double2* yb = ya + max_tris;
    const double2* yin = nullptr;
    const int blocks = grid_for((long long)max_tris * kG, kRB);
    for (int it = 0; it < n_iter; ++it) {
        const bool last = it == n_iter - 1;
        double2* yout = (it & 1) ? yb : ya;
        k_rad_iter<<<blocks, kRB, 0, st>>>(m.hdr, max_tris, row_ptr, col, sky, bare, betaE, betaO,
                                           1.0 / n_ff, yin, last ? nullptr : yout,
                                           last ? g_E : nullptr, last ? g_O : nullptr);
        PETCH_LAUNCH_CHECK("k_rad_iter");
        yin = yout;
    }
    return PETCH_OK;
}
