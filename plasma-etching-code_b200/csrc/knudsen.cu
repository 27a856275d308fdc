// Knudsen 1-D conductance tail for the deep-feature neutral flux (petch/knudsen.py, wired as
// mc_flux_3d_knudsen, petch/threed.py:1149-1208).
//
// The open feature is a vertical duct: per z-slice below sub_top the gas area a and sidewall
// perimeter p (slice_geometry, knudsen.py:29-68) give a free-molecular conductance
// (2/3) max(2a/p, dx) a / dx; adjacent slices are linked by the harmonic mean, the opening is held
// at unit concentration, and the floor faces of each slice consume 0.25 s A; a Thomas solve down the
// chain gives the concentration profile, and every face below sub_top takes its slice's value
// (knudsen_face_flux, knudsen.py:188-241).
//
// petch_knudsen_prepare does the geometry once per level set / mesh: slice counts from phi by
// integer warp reductions, the chain of valid slices and the nearest-valid-slice table (one thread:
// a few hundred slices), each face's slice, and the floor faces grouped by slice with a stable sort
// so every slice sums its faces in ascending face order (np.add.at's order).  petch_knudsen_solve
// runs both sticking fields of one coverage round: sink sums, the two Thomas chains (one warp
// each), the per-face values.  petch_knudsen_profile solves the chain for a caller's sink.
#include <cub/cub.cuh>
#include "common.cuh"
#include "petch_b200.h"

namespace petch {
namespace {

constexpr int kKB = 256;

struct KnParams {
    double dx, sub_top;
    int nz, trench, m;   // m: valid slices in the chain
    int pad;
};

struct KnScratch {
    KnParams* prm;      // [1]
    int* cnt_a;         // [nz]  hole: gas cells; trench: summed open-row counts
    int* cnt_b;         // [nz]  hole: gas / solid cell faces; trench: rows with gas
    double* area;       // [nz]
    double* perim;      // [nz]
    int* chain;         // [nz]  valid slices, opening first
    double* cond;       // [nz]  conductance of chain entry i
    int* snap;          // [nz]  nearest valid slice of each slice, -1 without any
    unsigned* key;      // [MF]  slice of a selected floor face, nz otherwise
    unsigned* key_s;    // [MF]
    int* fid;           // [MF]
    int* fid_s;         // [MF]
    int* take;          // [MF]  slice whose value the face takes, -1: value 1
    unsigned char* fld; // [MF]  open-field face (the 'field' sink's mean)
    int* seg;           // [nz + 1] first sorted face of each slice
    double* loss;       // [2 * nz]
    double* work;       // [4 * nz] Thomas diagonal / right-hand side, per species
    double* prof;       // [2 * nz]
    double* fmean;      // [2]   field mean of bare, field faces
    int* nfaces;        // [1]
    void* cub_tmp;
    size_t cub_bytes;
};

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

int slice_bits(int nz) {
    int b = 1;
    while (b < 31 && (1LL << b) <= (long long)nz) ++b;
    return b;
}

int kn_layout(int MF, int nz, void* base, size_t* total, KnScratch* out) {
    size_t sort_bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (unsigned*)nullptr,
                                                    (unsigned*)nullptr, (int*)nullptr, (int*)nullptr,
                                                    MF, 0, slice_bits(nz));
    if (e != cudaSuccess) return cuda_fail(e, "petch_knudsen: sort size query");
    size_t off = 0;
    char* b = (char*)base;
    auto take = [&](size_t bytes) {
        char* p = b ? b + off : nullptr;
        off += al256(bytes);
        return (void*)p;
    };
    KnScratch s;
    s.prm = (KnParams*)take(sizeof(KnParams));
    s.cnt_a = (int*)take(sizeof(int) * nz);
    s.cnt_b = (int*)take(sizeof(int) * nz);
    s.area = (double*)take(sizeof(double) * nz);
    s.perim = (double*)take(sizeof(double) * nz);
    s.chain = (int*)take(sizeof(int) * nz);
    s.cond = (double*)take(sizeof(double) * nz);
    s.snap = (int*)take(sizeof(int) * nz);
    s.key = (unsigned*)take(sizeof(unsigned) * MF);
    s.key_s = (unsigned*)take(sizeof(unsigned) * MF);
    s.fid = (int*)take(sizeof(int) * MF);
    s.fid_s = (int*)take(sizeof(int) * MF);
    s.take = (int*)take(sizeof(int) * MF);
    s.fld = (unsigned char*)take(MF);
    s.seg = (int*)take(sizeof(int) * ((size_t)nz + 1));
    s.loss = (double*)take(sizeof(double) * 2 * nz);
    s.work = (double*)take(sizeof(double) * 4 * nz);
    s.prof = (double*)take(sizeof(double) * 2 * nz);
    s.fmean = (double*)take(sizeof(double) * 2);
    s.nfaces = (int*)take(sizeof(int));
    s.cub_bytes = sort_bytes;
    s.cub_tmp = take(sort_bytes);
    *total = off;
    if (out) *out = s;
    return PETCH_OK;
}

__device__ __forceinline__ bool gas_at(const float* phi, int ny, int nz, int i, int j, int k) {
    return __ldg(phi + ((long long)i * ny + j) * nz + k) < 0.0f;
}

// Hole slices: per column (i, j) down k, gas cells and gas / solid faces towards i + 1 and j + 1,
// summed over the warp's columns with integer reductions (exact, order-free).
__global__ void k_kn_count_hole(const float* __restrict__ phi, int nx, int ny, int nz,
                                KnScratch s) {
    const long long ncol = (long long)nx * ny;
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * 32; base < ncol; base += nwarp * 32) {
        const long long col = base + lane;
        const bool live = col < ncol;
        const int i = live ? (int)(col / ny) : 0, j = live ? (int)(col % ny) : 0;
        for (int k = 0; k < nz; ++k) {
            int a = 0, f = 0;
            if (live) {
                const bool g = gas_at(phi, ny, nz, i, j, k);
                a = g;
                if (i + 1 < nx) f += g != gas_at(phi, ny, nz, i + 1, j, k);
                if (j + 1 < ny) f += g != gas_at(phi, ny, nz, i, j + 1, k);
            }
            a = __reduce_add_sync(0xffffffffu, a);
            f = __reduce_add_sync(0xffffffffu, f);
            if (lane == 0 && (a | f)) {
                if (a) atomicAdd(s.cnt_a + k, a);
                if (f) atomicAdd(s.cnt_b + k, f);
            }
        }
    }
}

// Trench slices: per (row j, slice k), the open cells along x; summed counts and open rows.
__global__ void k_kn_count_trench(const float* __restrict__ phi, int nx, int ny, int nz,
                                  KnScratch s) {
    const long long n = (long long)ny * nz;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(p / nz), k = (int)(p % nz);
        int c = 0;
        for (int i = 0; i < nx; ++i) c += gas_at(phi, ny, nz, i, j, k);
        if (c) {
            atomicAdd(s.cnt_a + k, c);
            atomicAdd(s.cnt_b + k, 1);
        }
    }
}

// One thread: slice area / perimeter, the chain of valid slices (opening first) with their
// conductances, and the nearest valid slice of every slice (ties to the lower, as
// _nearest_valid_slice).
__global__ void k_kn_chain(double dx, double sub_top, int nz, int trench, KnScratch s) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int k = 0; k < nz; ++k) {
        double a = 0.0, p = 0.0;
        const bool below = __dmul_rn((double)k, dx) < sub_top;
        if (below && s.cnt_a[k] > 0) {
            if (trench) {
                a = __dmul_rn((double)s.cnt_a[k], dx) / (double)s.cnt_b[k];
                p = 2.0;
            } else {
                a = __dmul_rn(__dmul_rn((double)s.cnt_a[k], dx), dx);
                p = fmax(__dmul_rn((double)s.cnt_b[k], dx), dx);
            }
        }
        s.area[k] = a;
        s.perim[k] = p;
    }
    int m = 0;
    for (int k = nz - 1; k >= 0; --k) {
        if (__dmul_rn((double)k, dx) < sub_top && s.area[k] > 0.0 && s.perim[k] > 0.0) {
            const double a = s.area[k], p = s.perim[k];
            const double r = fmax(__dmul_rn(2.0, a) / fmax(p, 1.0e-30), dx);
            s.chain[m] = k;
            s.cond[m] = __dmul_rn(__dmul_rn(2.0 / 3.0, r), a) / dx;
            ++m;
        }
    }
    // nearest valid slice: the chain lists them descending
    int lo = -1;  // highest valid slice <= k
    int ci = m - 1;
    for (int k = 0; k < nz; ++k) {
        while (ci >= 0 && s.chain[ci] <= k) lo = s.chain[ci--];
        const int hi = ci >= 0 ? s.chain[ci] : -1;  // lowest valid slice > k
        int v;
        if (m == 0) v = -1;
        else if (lo < 0) v = hi;
        else if (hi < 0) v = lo;
        else v = (hi - k) < (k - lo) ? hi : lo;
        s.snap[k] = v;
    }
    KnParams q;
    q.dx = dx;
    q.sub_top = sub_top;
    q.nz = nz;
    q.trench = trench;
    q.m = m;
    q.pad = 0;
    *s.prm = q;
}

// Per face: its slice (np.round of the centroid height, snapped), whether it takes the slice's
// value (below sub_top), whether it sinks (a floor face, n_z > 0.7, inside the footprint), whether
// it is an open-field face (z > sub_top - 0.5 dx).
__global__ void k_kn_faces(const int* __restrict__ n_faces, int MF, const float* __restrict__ cen,
                           const float* __restrict__ nrm, double cx, double cy, double half_width,
                           KnScratch s) {
    const int F = min(max(*n_faces, 0), MF);
    const KnParams q = *s.prm;
    const double band = half_width + 2.0 * q.dx;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < MF; f += gridDim.x * blockDim.x) {
        s.fid[f] = f;
        if (f == 0) *s.nfaces = F;
        if (f >= F) {
            s.key[f] = (unsigned)q.nz;
            continue;
        }
        const double x = cen[3 * f], y = cen[3 * f + 1], z = cen[3 * f + 2];
        int iz = (int)fmin(fmax(rint(z / q.dx), 0.0), (double)(q.nz - 1));
        const int sn = s.snap[iz];
        const bool below = z < q.sub_top;
        bool inside = true;
        if (half_width >= 0.0)
            inside = q.trench ? fabs(x - cx) <= band : hypot(x - cx, y - cy) <= band;
        const bool sel = below && inside && sn >= 0 && (double)nrm[3 * f + 2] > 0.7;
        s.key[f] = sel ? (unsigned)sn : (unsigned)q.nz;
        s.take[f] = (sn >= 0 && below) ? sn : -1;
        s.fld[f] = z > q.sub_top - 0.5 * q.dx;
    }
}

__global__ void k_kn_segments(int MF, KnScratch s) {
    const int nz = s.prm->nz;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= nz; k += gridDim.x * blockDim.x) {
        int lo = 0, hi = MF;  // first sorted position with key >= k
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (s.key_s[mid] < (unsigned)k) lo = mid + 1;
            else hi = mid;
        }
        s.seg[k] = lo;
    }
}

// Mean of bare over the open-field faces (one block, fixed-order reduction); fmean[1] = count.
__global__ void __launch_bounds__(kKB) k_kn_field_mean(const float* __restrict__ bare, KnScratch s) {
    __shared__ double sh[kKB];
    __shared__ double shc[kKB];
    const int F = *s.nfaces;
    double a = 0.0, c = 0.0;
    for (int f = threadIdx.x; f < F; f += blockDim.x)
        if (s.fld[f]) {
            a += (double)bare[f];
            c += 1.0;
        }
    sh[threadIdx.x] = a;
    shc[threadIdx.x] = c;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sh[threadIdx.x] += sh[threadIdx.x + w];
            shc[threadIdx.x] += shc[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        s.fmean[0] = shc[0] > 0.0 ? sh[0] / shc[0] : 0.0;
        s.fmean[1] = shc[0];
    }
}

// Per slice, both species: sum over its floor faces (ascending) of 0.25 clip(s, 0, 1) A with
// s = clip(bare' beta, 0, 1), bare' = min(bare, field mean) for the 'field' sink; per unit trench
// length for a trench.
__global__ void k_kn_loss(const float* __restrict__ bare, const float* __restrict__ area,
                          double betaE, double betaO, int sink_field, double Ly, KnScratch s) {
    const KnParams q = *s.prm;
    const bool clamp = sink_field && s.fmean[1] > 0.0;
    const double fm = s.fmean[0];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < q.nz; k += gridDim.x * blockDim.x) {
        double lE = 0.0, lO = 0.0;
        for (int p = s.seg[k]; p < s.seg[k + 1]; ++p) {
            const int f = s.fid_s[p];
            double b = (double)bare[f];
            if (clamp) b = fmin(b, fm);
            const double A = (double)area[f];
            const double sE = fmin(fmax(fmin(fmax(__dmul_rn(b, betaE), 0.0), 1.0), 0.0), 1.0);
            const double sO = fmin(fmax(fmin(fmax(__dmul_rn(b, betaO), 0.0), 1.0), 0.0), 1.0);
            lE = __dadd_rn(lE, __dmul_rn(0.25, __dmul_rn(sE, A)));
            lO = __dadd_rn(lO, __dmul_rn(0.25, __dmul_rn(sO, A)));
        }
        if (q.trench) {
            const double L = fmax(Ly, 1.0e-30);
            lE /= L;
            lO /= L;
        }
        s.loss[k] = lE;
        s.loss[q.nz + k] = lO;
    }
}

struct LossScale {
    const double* arr;   // per-slice scale, or null
    double wls;          // scalar scale
    int front;           // passivation-linked front loss (knudsen.py:165-185)
    double W, band_W, pass_frac, ar_pass;
};

__device__ double loss_scale(const LossScale& ls, const KnParams& q, int k) {
    if (ls.arr) return fmax(ls.arr[k], 0.0);
    if (!ls.front) return fmax(ls.wls, 0.0);
    const double zc = __dmul_rn((double)k, q.dx);
    const double ar = fmax((q.sub_top - zc) / fmax(ls.W, 1.0e-9), 0.0);
    const double g = exp(-fmax(ar - ls.band_W, 0.0) / fmax(ls.ar_pass, 1.0e-9));
    return fmax(ls.wls, 0.0) * __dadd_rn(ls.pass_frac, __dmul_rn(1.0 - ls.pass_frac, g));
}

// The tridiagonal chain of species `sp` (conductance_profile, knudsen.py:91-150) by the guarded
// Thomas algorithm (knudsen.py:71-88), one thread per species; prof = clip(conc, 0, 1) on the
// chain's slices, 1 elsewhere.
__global__ void k_kn_thomas(int n_species, LossScale ls, KnScratch s) {
    const KnParams q = *s.prm;
    const int sp = threadIdx.x >> 5;
    if (sp >= n_species) return;
    double* prof = s.prof + (size_t)sp * q.nz;
    const int lane = threadIdx.x & 31;
    for (int k = lane; k < q.nz; k += 32) prof[k] = 1.0;
    __syncwarp();
    if (lane != 0 || q.m == 0) return;
    const double* loss = s.loss + (size_t)sp * q.nz;
    double* b = s.work + (size_t)sp * 2 * q.nz;  // diagonal, then eliminated
    double* d = b + q.nz;                         // right-hand side
    const int m = q.m;
    // link i joins chain entries i, i + 1 when their slices are adjacent
    auto link = [&](int i) {
        if (abs(s.chain[i + 1] - s.chain[i]) != 1) return 0.0;
        const double c0 = s.cond[i], c1 = s.cond[i + 1];
        return __dmul_rn(__dmul_rn(2.0, c0), c1) / fmax(__dadd_rn(c0, c1), 1.0e-30);
    };
    for (int i = 0; i < m; ++i) {
        const int k = s.chain[i];
        double di = __dmul_rn(loss_scale(ls, q, k), fmax(loss[k], 0.0));
        double ri = 0.0;
        if (i == 0) {
            di = __dadd_rn(di, s.cond[0]);
            ri = __dadd_rn(ri, s.cond[0]);
        }
        if (i > 0) di = __dadd_rn(di, link(i - 1));
        if (i < m - 1) di = __dadd_rn(di, link(i));
        b[i] = fmax(di, 1.0e-30);
        d[i] = ri;
    }
    // forward elimination: lower = upper = -link
    for (int i = 1; i < m; ++i) {
        const double g = link(i - 1);
        const double w = (-g) / fmax(b[i - 1], 1.0e-30);
        b[i] = __dsub_rn(b[i], __dmul_rn(w, -g));
        d[i] = __dsub_rn(d[i], __dmul_rn(w, d[i - 1]));
    }
    double x = d[m - 1] / fmax(b[m - 1], 1.0e-30);
    prof[s.chain[m - 1]] = fmin(fmax(x, 0.0), 1.0);
    for (int i = m - 2; i >= 0; --i) {
        const double g = link(i);
        x = __dsub_rn(d[i], __dmul_rn(-g, x)) / fmax(b[i], 1.0e-30);
        prof[s.chain[i]] = fmin(fmax(x, 0.0), 1.0);
    }
}

__global__ void k_kn_out(int MF, KnScratch s, float* __restrict__ gE, float* __restrict__ gO) {
    const int F = *s.nfaces;
    const int nz = s.prm->nz;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x) {
        const int t = s.take[f];
        const double vE = t >= 0 ? s.prof[t] : 1.0;
        const double vO = t >= 0 ? s.prof[nz + t] : 1.0;
        gE[f] = (float)fmin(fmax(vE, 0.0), 8.0);
        gO[f] = (float)fmin(fmax(vO, 0.0), 8.0);
    }
}

int kn_bind(int MF, int nz, void* scratch, long long bytes, KnScratch* s, const char* who) {
    size_t need = 0;
    int rc = kn_layout(MF, nz, scratch, &need, s);
    if (rc) return rc;
    PETCH_REQUIRE((long long)need <= bytes, "%s: scratch too small", who);
    return PETCH_OK;
}

}  // namespace
}  // namespace petch

using namespace petch;

extern "C" int petch_knudsen_scratch_bytes(int max_faces, int nz, long long* bytes) {
    PETCH_REQUIRE(bytes, "petch_knudsen_scratch_bytes: null pointer");
    PETCH_REQUIRE(max_faces > 0 && nz > 0, "petch_knudsen_scratch_bytes: bad size");
    size_t total = 0;
    const int rc = kn_layout(max_faces, nz, nullptr, &total, nullptr);
    if (rc) return rc;
    *bytes = (long long)total;
    return PETCH_OK;
}

extern "C" int petch_knudsen_prepare(const float* phi, int nx, int ny, int nz, double dx,
                                     double sub_top, int trench, const int* n_faces,
                                     int max_faces, const float* centroids, const float* normals,
                                     double cx, double cy, double half_width, void* scratch,
                                     long long scratch_bytes, void* stream) {
    PETCH_REQUIRE(phi && n_faces && centroids && normals && scratch,
                  "petch_knudsen_prepare: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && (long long)nx * ny * nz < (1LL << 31) && dx > 0.0,
                  "petch_knudsen_prepare: bad grid");
    PETCH_REQUIRE(max_faces > 0, "petch_knudsen_prepare: bad face capacity");
    KnScratch s;
    int rc = kn_bind(max_faces, nz, scratch, scratch_bytes, &s, "petch_knudsen_prepare");
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    PETCH_CUDA(cudaMemsetAsync(s.cnt_a, 0, sizeof(int) * nz, st), "petch_knudsen_prepare: memset");
    PETCH_CUDA(cudaMemsetAsync(s.cnt_b, 0, sizeof(int) * nz, st), "petch_knudsen_prepare: memset");
    if (trench) {
        k_kn_count_trench<<<grid_for((long long)ny * nz, kKB), kKB, 0, st>>>(phi, nx, ny, nz, s);
        PETCH_LAUNCH_CHECK("k_kn_count_trench");
    } else {
        k_kn_count_hole<<<grid_for((long long)nx * ny, kKB, 4), kKB, 0, st>>>(phi, nx, ny, nz, s);
        PETCH_LAUNCH_CHECK("k_kn_count_hole");
    }
    k_kn_chain<<<1, 32, 0, st>>>(dx, sub_top, nz, trench ? 1 : 0, s);
    PETCH_LAUNCH_CHECK("k_kn_chain");
    k_kn_faces<<<grid_for(max_faces, kKB), kKB, 0, st>>>(n_faces, max_faces, centroids, normals,
                                                        cx, cy, half_width, s);
    PETCH_LAUNCH_CHECK("k_kn_faces");
    size_t cb = s.cub_bytes;
    // stable: the faces of a slice stay in ascending order
    PETCH_CUDA(cub::DeviceRadixSort::SortPairs(s.cub_tmp, cb, s.key, s.key_s, s.fid, s.fid_s,
                                               max_faces, 0, slice_bits(nz), st),
               "petch_knudsen_prepare: sort by slice");
    k_kn_segments<<<grid_for(nz + 1LL, kKB), kKB, 0, st>>>(max_faces, s);
    PETCH_LAUNCH_CHECK("k_kn_segments");
    return PETCH_OK;
}

extern "C" int petch_knudsen_solve(int max_faces, int nz, const float* bare, const float* areas,
                                   double betaE, double betaO, int sink_field, double Ly,
                                   double wall_loss_scale, int front_loss, double W, double band_W,
                                   double pass_frac, double ar_pass, void* scratch,
                                   long long scratch_bytes, float* flux_E, float* flux_O,
                                   void* stream) {
    PETCH_REQUIRE(bare && areas && scratch && flux_E && flux_O, "petch_knudsen_solve: null pointer");
    PETCH_REQUIRE(max_faces > 0 && nz > 0, "petch_knudsen_solve: bad size");
    KnScratch s;
    int rc = kn_bind(max_faces, nz, scratch, scratch_bytes, &s, "petch_knudsen_solve");
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    if (sink_field) {
        k_kn_field_mean<<<1, kKB, 0, st>>>(bare, s);
        PETCH_LAUNCH_CHECK("k_kn_field_mean");
    }
    k_kn_loss<<<grid_for(nz, 64), 64, 0, st>>>(bare, areas, betaE, betaO, sink_field ? 1 : 0, Ly, s);
    PETCH_LAUNCH_CHECK("k_kn_loss");
    LossScale ls{nullptr, wall_loss_scale, front_loss ? 1 : 0, W, band_W, pass_frac, ar_pass};
    k_kn_thomas<<<1, 64, 0, st>>>(2, ls, s);
    PETCH_LAUNCH_CHECK("k_kn_thomas");
    k_kn_out<<<grid_for(max_faces, kKB), kKB, 0, st>>>(max_faces, s, flux_E, flux_O);
    PETCH_LAUNCH_CHECK("k_kn_out");
    return PETCH_OK;
}

extern "C" int petch_knudsen_profile(int max_faces, int nz, const double* slice_loss,
                                     const double* loss_scale_arr, double wall_loss_scale,
                                     void* scratch, long long scratch_bytes, double* profile,
                                     void* stream) {
    PETCH_REQUIRE(slice_loss && scratch && profile, "petch_knudsen_profile: null pointer");
    PETCH_REQUIRE(max_faces > 0 && nz > 0, "petch_knudsen_profile: bad size");
    KnScratch s;
    int rc = kn_bind(max_faces, nz, scratch, scratch_bytes, &s, "petch_knudsen_profile");
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    PETCH_CUDA(cudaMemcpyAsync(s.loss, slice_loss, sizeof(double) * nz, cudaMemcpyDeviceToDevice, st),
               "petch_knudsen_profile: copy sink");
    LossScale ls{loss_scale_arr, wall_loss_scale, 0, 0.0, 0.0, 0.0, 0.0};
    k_kn_thomas<<<1, 32, 0, st>>>(1, ls, s);
    PETCH_LAUNCH_CHECK("k_kn_thomas");
    PETCH_CUDA(cudaMemcpyAsync(profile, s.prof, sizeof(double) * nz, cudaMemcpyDeviceToDevice, st),
               "petch_knudsen_profile: copy profile");
    return PETCH_OK;
}

extern "C" int petch_knudsen_slices(int max_faces, int nz, const void* scratch,
                                    long long scratch_bytes, double* area, double* perimeter,
                                    void* stream) {
    PETCH_REQUIRE(scratch && area && perimeter, "petch_knudsen_slices: null pointer");
    PETCH_REQUIRE(max_faces > 0 && nz > 0, "petch_knudsen_slices: bad size");
    KnScratch s;
    int rc = kn_bind(max_faces, nz, const_cast<void*>(scratch), scratch_bytes, &s,
                     "petch_knudsen_slices");
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    PETCH_CUDA(cudaMemcpyAsync(area, s.area, sizeof(double) * nz, cudaMemcpyDeviceToDevice, st),
               "petch_knudsen_slices: copy");
    PETCH_CUDA(cudaMemcpyAsync(perimeter, s.perim, sizeof(double) * nz, cudaMemcpyDeviceToDevice, st),
               "petch_knudsen_slices: copy");
    return PETCH_OK;
}
