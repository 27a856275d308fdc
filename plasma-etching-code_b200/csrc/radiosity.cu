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
// same order; products and sums are rounded explicitly (no contraction), so the tangent kernel's
// primal below gives the same bits.
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
                    sE = __dadd_rn(sE, __dmul_rn(1.0 - fmin(fmax(b * betaE, 0.0), 1.0), dj));
                    sO = __dadd_rn(sO, __dmul_rn(1.0 - fmin(fmax(b * betaO, 0.0), 1.0), dj));
                }
            }
        }
        for (int o = kG / 2; o > 0; o >>= 1) {
            sE += __shfl_xor_sync(0xffffffffu, sE, o);
            sO += __shfl_xor_sync(0xffffffffu, sO, o);
        }
        if (sub == 0 && i < F) {
            const double GE = __dadd_rn(D[i], __dmul_rn(inv_nff, sE));
            const double GO = __dadd_rn(D[i], __dmul_rn(inv_nff, sO));
            if (gE) {
                gE[i] = (float)fmin(fmax(GE, 0.0), 8.0);
                gO[i] = (float)fmin(fmax(GO, 0.0), 8.0);
            } else {
                const double b = (double)bare[i];
                y_out[i] = make_double2(__dmul_rn(1.0 - fmin(fmax(b * betaE, 0.0), 1.0), GE),
                                        __dmul_rn(1.0 - fmin(fmax(b * betaO, 0.0), 1.0), GO));
            }
        }
    }
}

// k_rad_iter with the three recipe tangents (direction-major dbare [3][MT]): the primal exactly
// as k_rad_iter computes it (the same entries, lanes and butterfly, so the same bits), and
//   dx_j = -ds_j G_j + (1 - s_j) dG_j   (first iteration: -ds_j D_j),   dG_i = sum_j dx_j / n_ff,
// with ds = beta dbare where 0 < bare beta < 1 (the clip's derivative, 0 at its bounds); the sky
// view D does not depend on the recipe.  The last iteration writes clip(G, 0, 8) and its tangent
// (0 where the clip holds).  y / dy hold x and dx: [MT] and [3][MT] double2 (E, O).
constexpr int kND = 3;

__device__ __forceinline__ double clip_ds(double b, double beta, double db) {
    const double s = b * beta;
    return (s > 0.0 && s < 1.0) ? beta * db : 0.0;
}

__global__ void __launch_bounds__(kRB) k_rad_iter_tan(const int* __restrict__ hdr, int MT,
                                                      const int* __restrict__ row_ptr,
                                                      const int* __restrict__ col,
                                                      const double* __restrict__ D,
                                                      const float* __restrict__ bare,
                                                      const float* __restrict__ dbare,
                                                      double betaE, double betaO, double inv_nff,
                                                      const double2* __restrict__ y_in,
                                                      const double2* __restrict__ dy_in,
                                                      double2* __restrict__ y_out,
                                                      double2* __restrict__ dy_out,
                                                      float* __restrict__ gE, float* __restrict__ gO,
                                                      float* __restrict__ dgE,
                                                      float* __restrict__ dgO) {
    const int F = min(hdr[HDR_F], MT);
    const int sub = threadIdx.x & (kG - 1);
    const int groups = (gridDim.x * blockDim.x) / kG;
    const int first = (blockIdx.x * blockDim.x + threadIdx.x) / kG;
    const int warp_first = first - ((threadIdx.x & 31) / kG);
    for (int base = warp_first; base < F; base += groups) {
        const int i = base + ((threadIdx.x & 31) / kG);
        double sE = 0.0, sO = 0.0;
        double tE[kND] = {0.0, 0.0, 0.0}, tO[kND] = {0.0, 0.0, 0.0};
        if (i < F) {
            const int e0 = row_ptr[i], e1 = row_ptr[i + 1];
            if (y_in) {
                for (int e = e0 + sub; e < e1; e += kG) {
                    const int j = __ldg(col + e);
                    const double2 x = y_in[j];
                    sE += x.x;
                    sO += x.y;
#pragma unroll
                    for (int k = 0; k < kND; ++k) {
                        const double2 dx = dy_in[(long long)k * MT + j];
                        tE[k] += dx.x;
                        tO[k] += dx.y;
                    }
                }
            } else {
                for (int e = e0 + sub; e < e1; e += kG) {
                    const int j = __ldg(col + e);
                    const double b = (double)__ldg(bare + j), dj = __ldg(D + j);
                    sE = __dadd_rn(sE, __dmul_rn(1.0 - fmin(fmax(b * betaE, 0.0), 1.0), dj));
                    sO = __dadd_rn(sO, __dmul_rn(1.0 - fmin(fmax(b * betaO, 0.0), 1.0), dj));
#pragma unroll
                    for (int k = 0; k < kND; ++k) {
                        const double db = (double)__ldg(dbare + (long long)k * MT + j);
                        tE[k] -= clip_ds(b, betaE, db) * dj;
                        tO[k] -= clip_ds(b, betaO, db) * dj;
                    }
                }
            }
        }
        for (int o = kG / 2; o > 0; o >>= 1) {
            sE += __shfl_xor_sync(0xffffffffu, sE, o);
            sO += __shfl_xor_sync(0xffffffffu, sO, o);
#pragma unroll
            for (int k = 0; k < kND; ++k) {
                tE[k] += __shfl_xor_sync(0xffffffffu, tE[k], o);
                tO[k] += __shfl_xor_sync(0xffffffffu, tO[k], o);
            }
        }
        if (sub == 0 && i < F) {
            const double GE = __dadd_rn(D[i], __dmul_rn(inv_nff, sE));
            const double GO = __dadd_rn(D[i], __dmul_rn(inv_nff, sO));
            if (gE) {
                gE[i] = (float)fmin(fmax(GE, 0.0), 8.0);
                gO[i] = (float)fmin(fmax(GO, 0.0), 8.0);
#pragma unroll
                for (int k = 0; k < kND; ++k) {
                    dgE[(long long)k * MT + i] = (GE > 0.0 && GE < 8.0) ? (float)(inv_nff * tE[k]) : 0.0f;
                    dgO[(long long)k * MT + i] = (GO > 0.0 && GO < 8.0) ? (float)(inv_nff * tO[k]) : 0.0f;
                }
            } else {
                const double b = (double)bare[i];
                const double cE = 1.0 - fmin(fmax(b * betaE, 0.0), 1.0);
                const double cO = 1.0 - fmin(fmax(b * betaO, 0.0), 1.0);
                y_out[i] = make_double2(__dmul_rn(cE, GE), __dmul_rn(cO, GO));
#pragma unroll
                for (int k = 0; k < kND; ++k) {
                    const double db = (double)dbare[(long long)k * MT + i];
                    dy_out[(long long)k * MT + i] =
                        make_double2(cE * inv_nff * tE[k] - clip_ds(b, betaE, db) * GE,
                                     cO * inv_nff * tO[k] - clip_ds(b, betaO, db) * GO);
                }
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

extern "C" int petch_radiosity_solve_tangent(const void* mesh, int max_tris, int max_verts,
                                             const int* row_ptr, const int* col,
                                             const double* sky, int n_ff, const float* bare,
                                             const float* dbare, double betaE, double betaO,
                                             int n_iter, float* g_E, float* g_O, float* dg_E,
                                             float* dg_O, double* work, void* stream) {
    PETCH_REQUIRE(mesh && row_ptr && col && sky && bare && dbare && g_E && g_O && dg_E && dg_O &&
                      work,
                  "petch_radiosity_solve_tangent: null pointer");
    PETCH_REQUIRE(max_tris > 0 && n_ff >= 1 && n_iter >= 1,
                  "petch_radiosity_solve_tangent: bad size");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    double2* ya = reinterpret_cast<double2*>(work);
    double2* yb = ya + max_tris;
    double2* dya = yb + max_tris;
    double2* dyb = dya + (long long)kND * max_tris;
    const double2 *yin = nullptr, *dyin = nullptr;
    const int blocks = grid_for((long long)max_tris * kG, kRB);
    for (int it = 0; it < n_iter; ++it) {
        const bool last = it == n_iter - 1;
        double2* yout = (it & 1) ? yb : ya;
        double2* dyout = (it & 1) ? dyb : dya;
        k_rad_iter_tan<<<blocks, kRB, 0, st>>>(m.hdr, max_tris, row_ptr, col, sky, bare, dbare,
                                               betaE, betaO, 1.0 / n_ff, yin, dyin,
                                               last ? nullptr : yout, last ? nullptr : dyout,
                                               last ? g_E : nullptr, last ? g_O : nullptr,
                                               last ? dg_E : nullptr, last ? dg_O : nullptr);
        PETCH_LAUNCH_CHECK("k_rad_iter_tan");
        yin = yout;
        dyin = dyout;
    }
    return PETCH_OK;
}

// ---------------------------------------------------------------------------------------------
// Restarted GMRES on (I - M) G = D (radiosity_solver = 'gmres', threed.py:972-982): the
// reference's scipy gmres(rtol, atol 0, restart, maxiter) with its Jacobi fallback on failure.
// Host-driven: each Arnoldi step is a few kernels (mat-vec, modified Gram-Schmidt dot / axpy
// pairs with the coefficients left on the device, norm, Givens rotation), and one 8-byte read of
// the residual estimate decides whether the cycle goes on; every reduction sums in a fixed order,
// so a solve is reproducible bit for bit.  Float64 throughout.
// ---------------------------------------------------------------------------------------------
namespace petch {
namespace {

constexpr int kGB = 256;
constexpr int kGBlocks = 296;   // dot-product partial blocks (2 per SM)

struct GmScratch {
    double* V;        // [(restart + 1) * MT] Krylov basis
    double* w;        // [MT]
    double* x;        // [MT]
    double* t;        // [MT]
    double* a;        // [MT] 1 - clip(bare beta, 0, 1)
    double* part;     // [kGBlocks]
    double* H;        // [(restart + 1) * restart], column-major
    double* cs;       // [restart]
    double* sn;       // [restart]
    double* g;        // [restart + 1]
    double* y;        // [restart]
    double* scal;     // [4]: [0] last dot / norm, [1] residual estimate
};

int gm_layout(int MT, int restart, void* base, size_t* total, GmScratch* out) {
    size_t off = 0;
    char* b = (char*)base;
    auto take = [&](size_t n) {
        char* p = b ? b + off : nullptr;
        off += (sizeof(double) * n + 255) & ~(size_t)255;
        return (double*)p;
    };
    GmScratch s;
    s.V = take((size_t)(restart + 1) * MT);
    s.w = take(MT);
    s.x = take(MT);
    s.t = take(MT);
    s.a = take(MT);
    s.part = take(kGBlocks);
    s.H = take((size_t)(restart + 1) * restart);
    s.cs = take(restart);
    s.sn = take(restart);
    s.g = take(restart + 1);
    s.y = take(restart);
    s.scal = take(4);
    *total = off;
    if (out) *out = s;
    return PETCH_OK;
}

__global__ void k_gm_alpha(const int* hdr, int MT, const float* __restrict__ bare, double beta,
                           double* __restrict__ a) {
    const int F = min(hdr[HDR_F], MT);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
        a[i] = 1.0 - fmin(fmax((double)bare[i] * beta, 0.0), 1.0);
}

// out = in - (1 / n_ff) sum over row i's entries j of a_j in_j  (row entries in ascending order)
__global__ void k_gm_matvec(const int* hdr, int MT, const int* __restrict__ row_ptr,
                            const int* __restrict__ col, const double* __restrict__ a,
                            double inv_nff, const double* __restrict__ in,
                            double* __restrict__ out) {
    const int F = min(hdr[HDR_F], MT);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
            const int j = __ldg(col + e);
            s += a[j] * in[j];
        }
        out[i] = in[i] - inv_nff * s;
    }
}

// partial[b] = sum over this block's fixed slice of u . v; then dest = sum of the partials
__global__ void __launch_bounds__(kGB) k_gm_dot_part(const int* hdr, int MT,
                                                      const double* __restrict__ u,
                                                      const double* __restrict__ v,
                                                      double* __restrict__ part) {
    __shared__ double sh[kGB];
    const int F = min(hdr[HDR_F], MT);
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
        acc += u[i] * v[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kGB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// dest = sum(part); sqrt_it: dest = sqrt(sum)
__global__ void __launch_bounds__(kGB) k_gm_dot_final(const double* __restrict__ part, int n,
                                                       double* __restrict__ dest, int sqrt_it) {
    __shared__ double sh[kGB];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += part[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kGB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *dest = sqrt_it ? sqrt(sh[0]) : sh[0];
}

// y = x * (*num) / (*den) elementwise factor read on the device (den <= 0: y = 0)
__global__ void k_gm_scale(const int* hdr, int MT, const double* __restrict__ x,
                           const double* __restrict__ den, double* __restrict__ y) {
    const int F = min(hdr[HDR_F], MT);
    const double d = *den;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
        y[i] = d > 0.0 ? x[i] / d : 0.0;
}

// w -= (*h) v
__global__ void k_gm_axpy(const int* hdr, int MT, const double* __restrict__ h,
                          const double* __restrict__ v, double* __restrict__ w) {
    const int F = min(hdr[HDR_F], MT);
    const double c = *h;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
        w[i] -= c * v[i];
}

// r = b - t
__global__ void k_gm_resid(const int* hdr, int MT, const double* __restrict__ b,
                           const double* __restrict__ t, double* __restrict__ r) {
    const int F = min(hdr[HDR_F], MT);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
        r[i] = b[i] - t[i];
}

// Start of a cycle: g = (beta0, 0, ...), beta0 = scal[0].
__global__ void k_gm_start(GmScratch s, int restart) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i <= restart; ++i) s.g[i] = 0.0;
    s.g[0] = s.scal[0];
}

// Column j of H (rows 0..j+1 in place): apply the previous rotations, form the new one, rotate g;
// scal[1] = |g[j + 1]|, the residual norm of the current iterate.
__global__ void k_gm_givens(GmScratch s, int j, int restart) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int m1 = restart + 1;
    double* h = s.H + (size_t)j * m1;
    for (int i = 0; i < j; ++i) {
        const double t = s.cs[i] * h[i] + s.sn[i] * h[i + 1];
        h[i + 1] = -s.sn[i] * h[i] + s.cs[i] * h[i + 1];
        h[i] = t;
    }
    const double a = h[j], b = h[j + 1];
    double c = 1.0, sn = 0.0;
    if (b != 0.0) {
        if (fabs(b) > fabs(a)) {
            const double t = a / b;
            sn = 1.0 / sqrt(1.0 + t * t);
            c = t * sn;
        } else {
            const double t = b / a;
            c = 1.0 / sqrt(1.0 + t * t);
            sn = t * c;
        }
    }
    s.cs[j] = c;
    s.sn[j] = sn;
    h[j] = c * a + sn * b;
    h[j + 1] = 0.0;
    s.g[j + 1] = -sn * s.g[j];
    s.g[j] = c * s.g[j];
    s.scal[1] = fabs(s.g[j + 1]);
}

// y = R^-1 g over the first k columns (zero pivots give 0).
__global__ void k_gm_backsolve(GmScratch s, int k, int restart) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int m1 = restart + 1;
    for (int i = k - 1; i >= 0; --i) {
        double v = s.g[i];
        for (int l = i + 1; l < k; ++l) v -= s.H[i + (size_t)l * m1] * s.y[l];
        const double d = s.H[i + (size_t)i * m1];
        s.y[i] = d != 0.0 ? v / d : 0.0;
    }
}

// x += sum_k y_k V_k
__global__ void k_gm_xupdate(const int* hdr, int MT, GmScratch s, int k) {
    const int F = min(hdr[HDR_F], MT);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x) {
        double v = s.x[i];
        for (int q = 0; q < k; ++q) v += s.y[q] * s.V[(size_t)q * MT + i];
        s.x[i] = v;
    }
}

__global__ void k_gm_out(const int* hdr, int MT, const double* __restrict__ x,
                         float* __restrict__ out) {
    const int F = min(hdr[HDR_F], MT);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x)
        out[i] = (float)fmin(fmax(x[i], 0.0), 8.0);
}

}  // namespace
}  // namespace petch

extern "C" int petch_radiosity_gmres_scratch_bytes(int max_tris, int restart, long long* bytes) {
    PETCH_REQUIRE(bytes, "petch_radiosity_gmres_scratch_bytes: null pointer");
    PETCH_REQUIRE(max_tris > 0 && restart >= 1 && restart <= 256,
                  "petch_radiosity_gmres_scratch_bytes: bad size");
    size_t total = 0;
    gm_layout(max_tris, restart, nullptr, &total, nullptr);
    *bytes = (long long)total;
    return PETCH_OK;
}

extern "C" int petch_radiosity_gmres(const void* mesh, int max_tris, int max_verts,
                                     const int* row_ptr, const int* col, const double* sky,
                                     int n_ff, const float* bare, double beta, double rtol,
                                     int restart, int maxiter, float* g_out, void* scratch,
                                     long long scratch_bytes, int* info, void* stream) {
    PETCH_REQUIRE(mesh && row_ptr && col && sky && bare && g_out && scratch && info,
                  "petch_radiosity_gmres: null pointer");
    PETCH_REQUIRE(max_tris > 0 && n_ff >= 1 && restart >= 1 && restart <= 256 && maxiter >= 0 &&
                      rtol >= 0.0,
                  "petch_radiosity_gmres: bad size");
    size_t need = 0;
    GmScratch s;
    gm_layout(max_tris, restart, scratch, &need, &s);
    PETCH_REQUIRE((long long)need <= scratch_bytes, "petch_radiosity_gmres: scratch too small");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    const int* hdr = m.hdr;
    const int MT = max_tris;
    const int gb = grid_for(MT, kGB);
    const double inv_nff = 1.0 / n_ff;
    auto dot = [&](const double* u, const double* v, double* dest, int sqrt_it) -> int {
        k_gm_dot_part<<<kGBlocks, kGB, 0, st>>>(hdr, MT, u, v, s.part);
        PETCH_LAUNCH_CHECK("k_gm_dot_part");
        k_gm_dot_final<<<1, kGB, 0, st>>>(s.part, kGBlocks, dest, sqrt_it);
        PETCH_LAUNCH_CHECK("k_gm_dot_final");
        return PETCH_OK;
    };
    auto read = [&](const double* p, double* h) -> int {
        PETCH_CUDA(cudaMemcpyAsync(h, p, sizeof(double), cudaMemcpyDeviceToHost, st),
                   "petch_radiosity_gmres: read scalar");
        PETCH_CUDA(cudaStreamSynchronize(st), "petch_radiosity_gmres: sync");
        return PETCH_OK;
    };
    int rc;
    k_gm_alpha<<<gb, kGB, 0, st>>>(hdr, MT, bare, beta, s.a);
    PETCH_LAUNCH_CHECK("k_gm_alpha");
    PETCH_CUDA(cudaMemsetAsync(s.x, 0, sizeof(double) * MT, st), "petch_radiosity_gmres: memset");
    if ((rc = dot(sky, sky, s.scal + 2, 1))) return rc;
    double bnorm = 0.0;
    if ((rc = read(s.scal + 2, &bnorm))) return rc;
    const double tol = rtol * bnorm;          // atol 0: the reference's threshold
    int status = 1;
    if (bnorm == 0.0) status = 0;
    const int m1 = restart + 1;
    for (int cycle = 0; cycle < maxiter && status; ++cycle) {
        // r = b - A x into V_0, beta0 = |r|
        k_gm_matvec<<<gb, kGB, 0, st>>>(hdr, MT, row_ptr, col, s.a, inv_nff, s.x, s.t);
        PETCH_LAUNCH_CHECK("k_gm_matvec");
        k_gm_resid<<<gb, kGB, 0, st>>>(hdr, MT, sky, s.t, s.w);
        PETCH_LAUNCH_CHECK("k_gm_resid");
        if ((rc = dot(s.w, s.w, s.scal, 1))) return rc;
        double beta0 = 0.0;
        if ((rc = read(s.scal, &beta0))) return rc;
        if (beta0 <= tol) {
            status = 0;
            break;
        }
        k_gm_scale<<<gb, kGB, 0, st>>>(hdr, MT, s.w, s.scal, s.V);
        PETCH_LAUNCH_CHECK("k_gm_scale");
        k_gm_start<<<1, 32, 0, st>>>(s, restart);
        PETCH_LAUNCH_CHECK("k_gm_start");
        int k = 0;
        for (int j = 0; j < restart; ++j) {
            double* vj = s.V + (size_t)j * MT;
            k_gm_matvec<<<gb, kGB, 0, st>>>(hdr, MT, row_ptr, col, s.a, inv_nff, vj, s.w);
            PETCH_LAUNCH_CHECK("k_gm_matvec");
            double* hj = s.H + (size_t)j * m1;
            for (int i = 0; i <= j; ++i) {         // modified Gram-Schmidt
                if ((rc = dot(s.w, s.V + (size_t)i * MT, hj + i, 0))) return rc;
                k_gm_axpy<<<gb, kGB, 0, st>>>(hdr, MT, hj + i, s.V + (size_t)i * MT, s.w);
                PETCH_LAUNCH_CHECK("k_gm_axpy");
            }
            if ((rc = dot(s.w, s.w, hj + j + 1, 1))) return rc;
            k_gm_scale<<<gb, kGB, 0, st>>>(hdr, MT, s.w, hj + j + 1, s.V + (size_t)(j + 1) * MT);
            PETCH_LAUNCH_CHECK("k_gm_scale");
            k_gm_givens<<<1, 32, 0, st>>>(s, j, restart);
            PETCH_LAUNCH_CHECK("k_gm_givens");
            k = j + 1;
            double est = 0.0;
            if ((rc = read(s.scal + 1, &est))) return rc;
            if (est <= tol) break;
        }
        k_gm_backsolve<<<1, 32, 0, st>>>(s, k, restart);
        PETCH_LAUNCH_CHECK("k_gm_backsolve");
        k_gm_xupdate<<<gb, kGB, 0, st>>>(hdr, MT, s, k);
        PETCH_LAUNCH_CHECK("k_gm_xupdate");
    }
    if (status) {   // the iterate after the last cycle may have converged: check it as scipy does
        k_gm_matvec<<<gb, kGB, 0, st>>>(hdr, MT, row_ptr, col, s.a, inv_nff, s.x, s.t);
        PETCH_LAUNCH_CHECK("k_gm_matvec");
        k_gm_resid<<<gb, kGB, 0, st>>>(hdr, MT, sky, s.t, s.w);
        PETCH_LAUNCH_CHECK("k_gm_resid");
        if ((rc = dot(s.w, s.w, s.scal, 1))) return rc;
        double r = 0.0;
        if ((rc = read(s.scal, &r))) return rc;
        if (r <= tol) status = 0;
    }
    k_gm_out<<<gb, kGB, 0, st>>>(hdr, MT, s.x, g_out);
    PETCH_LAUNCH_CHECK("k_gm_out");
    *info = status;
    return PETCH_OK;
}
