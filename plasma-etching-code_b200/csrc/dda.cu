// Deterministic discrete-ordinates (DDA) neutral transport (dda_neutral_flux, petch/dda.py:132-188,
// wired as mc_flux_3d_dda, petch/threed.py:1211-1244).
//
// The reference marches every (surface point, direction) ray through the occupancy grid once per
// gather: 13 gathers per dda_neutral_flux call (the direct view and n_reemit = 12 re-emission
// passes), two calls per coverage round, four rounds per step.  Where a ray ends depends only on
// the geometry, which is fixed within a step, so here each ray is marched ONCE (petch_dda_prepare)
// and its end recorded as a code: the solid cell whose re-emission it picks up, or escape, or
// nothing.  Every gather afterwards is a read of those codes and of the re-emission field
// (petch_dda_solve), both species at once because they share the geometry and the coverage.
//
// Arithmetic follows the reference's types: the march and the per-face gather sums in float32
// (its Warp kernel), the cell re-emission, dilation and Aitken extrapolation in float64 (its numpy
// host code), every operation rounded explicitly so no multiply-add is fused and the results do not
// depend on the compiler; each sum runs in the reference's order (directions ascending, the faces of
// a cell ascending, the six neighbours in np.roll order), so the whole solve is reproducible bit for
// bit and matches a float32 evaluation of the reference's algorithm exactly.
#include <cub/cub.cuh>
#include "common.cuh"
#include "petch_b200.h"

namespace petch {
namespace {

constexpr int kDB = 256;
constexpr int CODE_ESCAPE = -1;    // reached z >= z_top: carries the source (1 direct, 0 re-emission)
constexpr int CODE_NONE = -2;      // still marching after max_steps: carries 0
constexpr int CODE_INACTIVE = -3;  // acc = max(n . d, 0) <= 1e-6: not part of the sum

struct Grid {
    const float* phi;
    int nx, ny, nz;
    float dx, z_top;
    int max_steps, periodic_y;
};

__device__ __forceinline__ float ld_phi(const Grid& g, int i, int j, int k) {
    return __ldg(g.phi + ((long long)i * g.ny + j) * g.nz + k);
}

// clamp(int(q / dx + 0.5), 0, n - 1) with int() truncating toward zero
__device__ __forceinline__ int round_cell(float q, float dx, int n) {
    const int c = (int)__fadd_rn(__fdiv_rn(q, dx), 0.5f);
    return c < 0 ? 0 : (c > n - 1 ? n - 1 : c);
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

__device__ __forceinline__ float lerp_rn(float a, float b, float t) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
}

// acc = max(n . d, 0), the dot product summed x, y, z
__device__ __forceinline__ float cos_weight(float n0, float n1, float n2, float d0, float d1,
                                            float d2) {
    const float dot = __fadd_rn(__fadd_rn(__fmul_rn(n0, d0), __fmul_rn(n1, d1)), __fmul_rn(n2, d2));
    return dot > 0.0f ? dot : 0.0f;
}

// The march of one ray (_dda_gather_kernel, dda.py:44-94): from o + 1.01 dx d, one dx per step;
// escape at z >= z_top; where the trilinear phi turns positive, the first solid rounded cell of up
// to six half-cell steps forward, else the rounded cell of the position itself.
__device__ int march(const Grid& g, float ox, float oy, float oz, float d0, float d1, float d2) {
    const float dx = g.dx;
    const float sx = __fmul_rn(d0, dx), sy = __fmul_rn(d1, dx), sz = __fmul_rn(d2, dx);
    float px = __fadd_rn(ox, __fmul_rn(sx, 1.01f));
    float py = __fadd_rn(oy, __fmul_rn(sy, 1.01f));
    float pz = __fadd_rn(oz, __fmul_rn(sz, 1.01f));
    const float umax = __fsub_rn((float)g.nx, 1.001f), vmax = __fsub_rn((float)g.ny, 1.001f),
                wmax = __fsub_rn((float)g.nz, 1.001f);
    const float Ly = __fmul_rn((float)g.ny, dx);
    const float hx = __fmul_rn(sx, 0.5f), hy = __fmul_rn(sy, 0.5f), hz = __fmul_rn(sz, 0.5f);
    for (int s = 0; s < g.max_steps; ++s) {
        if (pz >= g.z_top) return CODE_ESCAPE;
        const float u = clampf(__fdiv_rn(px, dx), 0.0f, umax);
        const float v = clampf(__fdiv_rn(py, dx), 0.0f, vmax);
        const float w = clampf(__fdiv_rn(pz, dx), 0.0f, wmax);
        const int i0 = (int)u, j0 = (int)v, k0 = (int)w;
        const float fu = __fsub_rn(u, (float)i0), fv = __fsub_rn(v, (float)j0),
                    fw = __fsub_rn(w, (float)k0);
        const float p00 = lerp_rn(ld_phi(g, i0, j0, k0), ld_phi(g, i0 + 1, j0, k0), fu);
        const float p10 = lerp_rn(ld_phi(g, i0, j0 + 1, k0), ld_phi(g, i0 + 1, j0 + 1, k0), fu);
        const float p01 = lerp_rn(ld_phi(g, i0, j0, k0 + 1), ld_phi(g, i0 + 1, j0, k0 + 1), fu);
        const float p11 =
            lerp_rn(ld_phi(g, i0, j0 + 1, k0 + 1), ld_phi(g, i0 + 1, j0 + 1, k0 + 1), fu);
        const float pv = lerp_rn(lerp_rn(p00, p10, fv), lerp_rn(p01, p11, fv), fw);
        if (pv > 0.0f) {
            float qx = px, qy = py, qz = pz;
            for (int e = 0; e < 6; ++e) {
                const int ix = round_cell(qx, dx, g.nx), iy = round_cell(qy, dx, g.ny),
                          iz = round_cell(qz, dx, g.nz);
                if (ld_phi(g, ix, iy, iz) > 0.0f) return (ix * g.ny + iy) * g.nz + iz;
                qx = __fadd_rn(qx, hx);
                qy = __fadd_rn(qy, hy);
                qz = __fadd_rn(qz, hz);
            }
            const int ix = round_cell(px, dx, g.nx), iy = round_cell(py, dx, g.ny),
                      iz = round_cell(pz, dx, g.nz);
            return (ix * g.ny + iy) * g.nz + iz;
        }
        px = __fadd_rn(px, sx);
        py = __fadd_rn(py, sy);
        pz = __fadd_rn(pz, sz);
        if (g.periodic_y == 1) {
            if (py < 0.0f) py = __fadd_rn(py, Ly);
            if (py >= Ly) py = __fsub_rn(py, Ly);
        }
    }
    return CODE_NONE;
}

// Scratch of one prepared geometry (sizes from max_faces MF, cells NC, directions D).
struct DDAScratch {
    int* code;        // [D * MF] ray end of direction k of face f at k * MF + f
    float* den;       // [MF]     sum over directions of w acc
    double2* vf0;     // [MF]     the direct view (both components)
    double2* ring;    // [2 * MF] iterates of the re-emission passes
    float* nrm;       // [3 * MF] normals, copied
    double* area;     // [MF]     face areas as float64, copied
    float4* dirw;     // [D]      direction xyz, weight
    unsigned* key;    // [MF]     wall cell per face (NC past the live faces)
    unsigned* key_s;  // [MF]     sorted
    int* fid;         // [MF]     0..MF-1
    int* fid_s;       // [MF]     faces in (wall cell, face) order
    int* head;        // [MF + 1] 1 at the first face of each wall cell
    int* slot_at;     // [MF + 1] exclusive scan of head: the slot of each wall cell
    int* seg;         // [MF + 1] first sorted face of each slot
    int* slot_cell;   // [MF]     cell of each slot
    double* cell_area;// [MF]     summed face area of each slot
    double2* R;       // [MF]     re-emission of each slot, both species (float64)
    int* slot_of;     // [NC]     slot of each cell, -1 where no face deposits
    int* fill;        // [FC]     unseeded solid cells next to a seeded one
    int* cnt;         // [4]      faces, slots, fill cells, fill overflow
    float2* remit;    // [NC]     re-emission field as the gather reads it (float32)
    void* cub_tmp;
    size_t cub_bytes;
    int fill_cap;
};

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

int cell_bits(long long ncell) {
    int b = 1;
    while (b < 31 && (1LL << b) <= ncell) ++b;
    return b;
}

int dda_layout(int MF, long long NC, int D, void* base, size_t* total, DDAScratch* out) {
    size_t sort_bytes = 0, scan_bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (unsigned*)nullptr,
                                                    (unsigned*)nullptr, (int*)nullptr, (int*)nullptr,
                                                    MF, 0, cell_bits(NC));
    if (e != cudaSuccess) return cuda_fail(e, "petch_dda: sort size query");
    e = cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (int*)nullptr, (int*)nullptr, MF + 1);
    if (e != cudaSuccess) return cuda_fail(e, "petch_dda: scan size query");
    size_t off = 0;
    char* b = (char*)base;
    auto take = [&](size_t bytes) {
        char* p = b ? b + off : nullptr;
        off += al256(bytes);
        return (void*)p;
    };
    DDAScratch s;
    const long long fc = NC < 6LL * MF ? NC : 6LL * MF;
    s.fill_cap = (int)fc;
    s.code = (int*)take(sizeof(int) * (size_t)D * MF);
    s.den = (float*)take(sizeof(float) * MF);
    s.vf0 = (double2*)take(sizeof(double2) * MF);
    s.ring = (double2*)take(sizeof(double2) * 2 * (size_t)MF);
    s.nrm = (float*)take(sizeof(float) * 3 * (size_t)MF);
    s.area = (double*)take(sizeof(double) * MF);
    s.dirw = (float4*)take(sizeof(float4) * D);
    s.key = (unsigned*)take(sizeof(unsigned) * MF);
    s.key_s = (unsigned*)take(sizeof(unsigned) * MF);
    s.fid = (int*)take(sizeof(int) * MF);
    s.fid_s = (int*)take(sizeof(int) * MF);
    s.head = (int*)take(sizeof(int) * ((size_t)MF + 1));
    s.slot_at = (int*)take(sizeof(int) * ((size_t)MF + 1));
    s.seg = (int*)take(sizeof(int) * ((size_t)MF + 1));
    s.slot_cell = (int*)take(sizeof(int) * MF);
    s.cell_area = (double*)take(sizeof(double) * MF);
    s.R = (double2*)take(sizeof(double2) * MF);
    s.slot_of = (int*)take(sizeof(int) * (size_t)NC);
    s.fill = (int*)take(sizeof(int) * (size_t)fc);
    s.cnt = (int*)take(sizeof(int) * 4);
    s.remit = (float2*)take(sizeof(float2) * (size_t)NC);
    s.cub_bytes = sort_bytes > scan_bytes ? sort_bytes : scan_bytes;
    s.cub_tmp = take(s.cub_bytes);
    *total = off;
    if (out) *out = s;
    return PETCH_OK;
}

__device__ __forceinline__ int live_faces(const int* n_faces, int MF) {
    const int F = *n_faces;
    return F < 0 ? 0 : (F > MF ? MF : F);
}

// Copies of the per-face inputs the solve needs again, the directions, and the face count.
__global__ void k_dda_copy(const int* __restrict__ n_faces, int MF, const float* __restrict__ nrm,
                           const float* __restrict__ area, const float* __restrict__ dirs,
                           const float* __restrict__ wts, int D, DDAScratch s) {
    const int F = live_faces(n_faces, MF);
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    if (t0 == 0) s.cnt[0] = F;
    for (int k = t0; k < D; k += st)
        s.dirw[k] = make_float4(dirs[3 * k], dirs[3 * k + 1], dirs[3 * k + 2], wts[k]);
    for (int f = t0; f < F; f += st) {
        s.nrm[3 * f] = nrm[3 * f];
        s.nrm[3 * f + 1] = nrm[3 * f + 1];
        s.nrm[3 * f + 2] = nrm[3 * f + 2];
        s.area[f] = (double)area[f];
    }
}

// One thread per (direction k, face f), f fastest so a warp marches one direction from 32
// neighbouring faces (marching-cubes order keeps them close in space and in normal).
__global__ void __launch_bounds__(kDB) k_dda_march(Grid g, const float* __restrict__ org, int MF,
                                                   int D, DDAScratch s) {
    const int F = s.cnt[0];
    const long long n = (long long)F * D;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(p / F), f = (int)(p - (long long)k * F);
        const float4 d = s.dirw[k];
        const float acc = cos_weight(s.nrm[3 * f], s.nrm[3 * f + 1], s.nrm[3 * f + 2], d.x, d.y, d.z);
        int code = CODE_INACTIVE;
        if (acc > 1.0e-6f) code = march(g, org[3 * f], org[3 * f + 1], org[3 * f + 2], d.x, d.y, d.z);
        s.code[(long long)k * MF + f] = code;
    }
}

// Per face: den = sum(w acc), the direct view num / max(den, 1e-12) with num the escapes' w acc
// (a hit adds w acc * 0 on this pass), and the solid-side wall cell round(c - 0.7 dx n) in float64
// (dda.py:143-149) as the sort key.
__global__ void k_dda_direct(Grid g, const float* __restrict__ cen, int MF, int D, long long NC,
                             double dxd, DDAScratch s) {
    const int F = s.cnt[0];
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < MF; f += gridDim.x * blockDim.x) {
        s.fid[f] = f;
        if (f >= F) {
            s.key[f] = (unsigned)NC;
            continue;
        }
        const float n0 = s.nrm[3 * f], n1 = s.nrm[3 * f + 1], n2 = s.nrm[3 * f + 2];
        float den = 0.0f, num = 0.0f;
        for (int k = 0; k < D; ++k) {
            const float4 d = s.dirw[k];
            const float wa = __fmul_rn(d.w, cos_weight(n0, n1, n2, d.x, d.y, d.z));
            den = __fadd_rn(den, wa);
            if (s.code[(long long)k * MF + f] == CODE_ESCAPE) num = __fadd_rn(num, wa);
        }
        s.den[f] = den;
        const double dir = (double)__fdiv_rn(num, fmaxf(den, 1.0e-12f));
        s.vf0[f] = make_double2(dir, dir);
        const double inv = 1.0 / dxd, off = __dmul_rn(0.7, dxd);
        const int ext[3] = {g.nx, g.ny, g.nz};
        long long c[3];
        for (int q = 0; q < 3; ++q) {
            const double sp = __dsub_rn((double)cen[3 * f + q], __dmul_rn(off, (double)s.nrm[3 * f + q]));
            long long i = (long long)__dadd_rn(__dmul_rn(sp, inv), 0.5);
            c[q] = i < 0 ? 0 : (i > ext[q] - 1 ? ext[q] - 1 : i);
        }
        s.key[f] = (unsigned)((c[0] * g.ny + c[1]) * g.nz + c[2]);
    }
}

__global__ void k_dda_heads(int MF, DDAScratch s) {
    const int F = s.cnt[0];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= MF; p += gridDim.x * blockDim.x)
        s.head[p] = (p < F && (p == 0 || s.key_s[p] != s.key_s[p - 1])) ? 1 : 0;
}

__global__ void k_dda_segments(int MF, DDAScratch s) {
    const int F = s.cnt[0];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= MF; p += gridDim.x * blockDim.x) {
        if (p == MF) {
            s.cnt[1] = s.slot_at[MF];
            s.seg[s.slot_at[MF]] = F;
        } else if (s.head[p]) {
            const int slot = s.slot_at[p];
            const int cell = (int)s.key_s[p];
            s.seg[slot] = p;
            s.slot_cell[slot] = cell;
            s.slot_of[cell] = slot;
        }
    }
}

// Summed area of each wall cell's faces, ascending face order (np.add.at).
__global__ void k_dda_cell_area(int MF, DDAScratch s) {
    const int ns = s.cnt[1];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ns; q += gridDim.x * blockDim.x) {
        double a = 0.0;
        for (int p = s.seg[q]; p < s.seg[q + 1]; ++p) a = __dadd_rn(a, s.area[s.fid_s[p]]);
        s.cell_area[q] = a;
    }
}

// Neighbour j (0..5) of a cell in the order the dilation sums them: np.roll(., +1) then (., -1)
// along x, y, z, i.e. (i - 1, i + 1) periodic on each axis.
__device__ __forceinline__ long long roll_nbr(int ix, int iy, int iz, int j, int nx, int ny, int nz) {
    int a[3] = {ix, iy, iz};
    const int n[3] = {nx, ny, nz};
    const int ax = j >> 1;
    a[ax] = (j & 1) ? (a[ax] + 1) % n[ax] : (a[ax] - 1 + n[ax]) % n[ax];
    return ((long long)a[0] * ny + a[1]) * nz + a[2];
}

// Unseeded solid cells with at least one seeded neighbour (the one-cell dilation's support).
__global__ void k_dda_fill_list(Grid g, long long NC, DDAScratch s) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < NC;
         c += (long long)gridDim.x * blockDim.x) {
        if (!(__ldg(g.phi + c) > 0.0f) || s.slot_of[c] >= 0) continue;
        const int iz = (int)(c % g.nz), iy = (int)((c / g.nz) % g.ny), ix = (int)(c / ((long long)g.nz * g.ny));
        bool any = false;
        for (int j = 0; j < 6 && !any; ++j)
            any = s.slot_of[roll_nbr(ix, iy, iz, j, g.nx, g.ny, g.nz)] >= 0;
        if (!any) continue;
        const int i = atomicAdd(s.cnt + 2, 1);
        if (i < s.fill_cap) s.fill[i] = (int)c;
        else atomicOr(s.cnt + 3, 1);
    }
}

// Re-emission of each seeded cell: sum over its faces (ascending) of A (1 - s) max(vf, 0), over
// max(cell area, 1e-12); s = clip(bare beta, 0, 1), alpha = clip(1 - s, 0, 1) (dda.py:163-165).
__global__ void k_dda_remit(const double2* __restrict__ vf, const float* __restrict__ bare,
                            double betaE, double betaO, DDAScratch s) {
    const int ns = s.cnt[1];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ns; q += gridDim.x * blockDim.x) {
        double aE = 0.0, aO = 0.0;
        for (int p = s.seg[q]; p < s.seg[q + 1]; ++p) {
            const int f = s.fid_s[p];
            const double b = (double)bare[f], A = s.area[f];
            const double sE = fmin(fmax(__dmul_rn(b, betaE), 0.0), 1.0);
            const double sO = fmin(fmax(__dmul_rn(b, betaO), 0.0), 1.0);
            const double alE = fmin(fmax(__dsub_rn(1.0, sE), 0.0), 1.0);
            const double alO = fmin(fmax(__dsub_rn(1.0, sO), 0.0), 1.0);
            const double2 v = vf[f];
            aE = __dadd_rn(aE, __dmul_rn(__dmul_rn(A, alE), fmax(v.x, 0.0)));
            aO = __dadd_rn(aO, __dmul_rn(__dmul_rn(A, alO), fmax(v.y, 0.0)));
        }
        const double ca = fmax(s.cell_area[q], 1.0e-12);
        const double2 r = make_double2(aE / ca, aO / ca);
        s.R[q] = r;
        s.remit[s.slot_cell[q]] = make_float2((float)r.x, (float)r.y);
    }
}

// Dilation: an unseeded solid cell next to seeded ones takes their mean (dda.py:170-178).
__global__ void k_dda_fill(int nx, int ny, int nz, DDAScratch s) {
    const int nf = min(s.cnt[2], s.fill_cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x) {
        const long long c = s.fill[i];
        const int iz = (int)(c % nz), iy = (int)((c / nz) % ny), ix = (int)(c / ((long long)nz * ny));
        double nE = 0.0, nO = 0.0, cnt = 0.0;
        for (int j = 0; j < 6; ++j) {
            const int q = s.slot_of[roll_nbr(ix, iy, iz, j, nx, ny, nz)];
            if (q >= 0) {
                const double2 r = s.R[q];
                nE = __dadd_rn(nE, r.x);
                nO = __dadd_rn(nO, r.y);
                cnt = __dadd_rn(cnt, 1.0);
            }
        }
        s.remit[c] = make_float2((float)(nE / cnt), (float)(nO / cnt));
    }
}

// One re-emission pass for both species: vf = direct + num / max(den, 1e-12), num summing w acc
// remit over the directions that hit a cell (escapes carry 0 here).  The last pass extrapolates
// (Aitken, dda.py:182-187) from the two previous iterates p1, p2 (p2 null: none) and writes
// clip(max(vf, 0), 0, 8).
__global__ void __launch_bounds__(kDB) k_dda_gather(int MF, int D, DDAScratch s,
                                                    double2* __restrict__ out,
                                                    const double2* __restrict__ p1,
                                                    const double2* __restrict__ p2,
                                                    float* __restrict__ gE, float* __restrict__ gO) {
    const int F = s.cnt[0];
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x) {
        const float n0 = s.nrm[3 * f], n1 = s.nrm[3 * f + 1], n2 = s.nrm[3 * f + 2];
        float numE = 0.0f, numO = 0.0f;
        for (int k = 0; k < D; ++k) {
            const int code = __ldg(s.code + (long long)k * MF + f);
            if (code < 0) continue;
            const float4 d = s.dirw[k];
            const float wa = __fmul_rn(d.w, cos_weight(n0, n1, n2, d.x, d.y, d.z));
            const float2 r = __ldg(s.remit + code);
            numE = __fadd_rn(numE, __fmul_rn(wa, r.x));
            numO = __fadd_rn(numO, __fmul_rn(wa, r.y));
        }
        const float den = fmaxf(s.den[f], 1.0e-12f);
        const double dir = s.vf0[f].x;
        double vE = __dadd_rn(dir, (double)__fdiv_rn(numE, den));
        double vO = __dadd_rn(dir, (double)__fdiv_rn(numO, den));
        if (!gE) {
            out[f] = make_double2(vE, vO);
            continue;
        }
        if (p2) {
            const double2 a = p1[f], b = p2[f];
            double v[2] = {vE, vO};
            const double q1[2] = {a.x, a.y}, q2[2] = {b.x, b.y};
            for (int c = 0; c < 2; ++c) {
                const double d1 = __dsub_rn(v[c], q1[c]), d0 = __dsub_rn(q1[c], q2[c]);
                double r = fabs(d0) > 1.0e-12 ? d1 / d0 : 0.0;
                r = fmin(fmax(r, 0.0), 0.995);
                v[c] = __dadd_rn(v[c], __dmul_rn(d1, r) / __dsub_rn(1.0, r));
            }
            vE = v[0];
            vO = v[1];
        }
        gE[f] = (float)fmin(fmax(fmax(vE, 0.0), 0.0), 8.0);
        gO[f] = (float)fmin(fmax(fmax(vO, 0.0), 0.0), 8.0);
    }
}

}  // namespace
}  // namespace petch

using namespace petch;

extern "C" int petch_dda_scratch_bytes(int max_faces, int nx, int ny, int nz, int n_dirs,
                                       long long* bytes) {
    PETCH_REQUIRE(bytes, "petch_dda_scratch_bytes: null pointer");
    PETCH_REQUIRE(max_faces > 0 && n_dirs > 0 && (long long)max_faces * n_dirs < (1LL << 31),
                  "petch_dda_scratch_bytes: max_faces * n_dirs must be in [1, 2^31)");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && (long long)nx * ny * nz < (1LL << 31),
                  "petch_dda_scratch_bytes: grid must have 1 .. 2^31 - 1 cells");
    size_t total = 0;
    const int rc = dda_layout(max_faces, (long long)nx * ny * nz, n_dirs, nullptr, &total, nullptr);
    if (rc) return rc;
    *bytes = (long long)total;
    return PETCH_OK;
}

extern "C" int petch_dda_prepare(const float* phi, int nx, int ny, int nz, double dx, double z_top,
                                 int max_steps, int periodic_y, const int* n_faces, int max_faces,
                                 const float* origins, const float* normals, const float* areas,
                                 const float* dirs, const float* weights, int n_dirs,
                                 void* scratch, long long scratch_bytes, void* stream) {
    PETCH_REQUIRE(phi && n_faces && origins && normals && areas && dirs && weights && scratch,
                  "petch_dda_prepare: null pointer");
    // the trilinear test reads nodes i0 and i0 + 1 on every axis
    PETCH_REQUIRE(nx >= 2 && ny >= 2 && nz >= 2 && (long long)nx * ny * nz < (1LL << 31) && dx > 0.0,
                  "petch_dda_prepare: the grid needs at least 2 nodes per axis and < 2^31 cells");
    PETCH_REQUIRE(max_faces > 0 && n_dirs > 0 && (long long)max_faces * n_dirs < (1LL << 31),
                  "petch_dda_prepare: max_faces * n_dirs must be in [1, 2^31)");
    PETCH_REQUIRE(max_steps >= 0, "petch_dda_prepare: max_steps must be >= 0");
    const long long NC = (long long)nx * ny * nz;
    size_t need = 0;
    DDAScratch s;
    int rc = dda_layout(max_faces, NC, n_dirs, scratch, &need, &s);
    if (rc) return rc;
    PETCH_REQUIRE((long long)need <= scratch_bytes, "petch_dda_prepare: scratch too small");
    cudaStream_t st = as_stream(stream);
    Grid g{phi, nx, ny, nz, (float)dx, (float)z_top, max_steps, periodic_y};
    PETCH_CUDA(cudaMemsetAsync(s.cnt, 0, sizeof(int) * 4, st), "petch_dda_prepare: memset");
    PETCH_CUDA(cudaMemsetAsync(s.slot_of, 0xff, sizeof(int) * (size_t)NC, st),
               "petch_dda_prepare: memset");
    PETCH_CUDA(cudaMemsetAsync(s.remit, 0, sizeof(float2) * (size_t)NC, st),
               "petch_dda_prepare: memset");
    k_dda_copy<<<grid_for(max_faces, kDB), kDB, 0, st>>>(n_faces, max_faces, normals, areas, dirs,
                                                         weights, n_dirs, s);
    PETCH_LAUNCH_CHECK("k_dda_copy");
    k_dda_march<<<grid_for((long long)max_faces * n_dirs, kDB, 16), kDB, 0, st>>>(
        g, origins, max_faces, n_dirs, s);
    PETCH_LAUNCH_CHECK("k_dda_march");
    k_dda_direct<<<grid_for(max_faces, kDB), kDB, 0, st>>>(g, origins, max_faces, n_dirs, NC, dx, s);
    PETCH_LAUNCH_CHECK("k_dda_direct");
    size_t cb = s.cub_bytes;
    // stable: the faces of one wall cell stay in ascending order
    PETCH_CUDA(cub::DeviceRadixSort::SortPairs(s.cub_tmp, cb, s.key, s.key_s, s.fid, s.fid_s,
                                               max_faces, 0, cell_bits(NC), st),
               "petch_dda_prepare: sort by wall cell");
    k_dda_heads<<<grid_for(max_faces + 1LL, kDB), kDB, 0, st>>>(max_faces, s);
    PETCH_LAUNCH_CHECK("k_dda_heads");
    cb = s.cub_bytes;
    PETCH_CUDA(cub::DeviceScan::ExclusiveSum(s.cub_tmp, cb, s.head, s.slot_at, max_faces + 1, st),
               "petch_dda_prepare: slot scan");
    k_dda_segments<<<grid_for(max_faces + 1LL, kDB), kDB, 0, st>>>(max_faces, s);
    PETCH_LAUNCH_CHECK("k_dda_segments");
    k_dda_cell_area<<<grid_for(max_faces, kDB), kDB, 0, st>>>(max_faces, s);
    PETCH_LAUNCH_CHECK("k_dda_cell_area");
    k_dda_fill_list<<<grid_for(NC, kDB), kDB, 0, st>>>(g, NC, s);
    PETCH_LAUNCH_CHECK("k_dda_fill_list");
    return PETCH_OK;
}

extern "C" int petch_dda_solve(int max_faces, int nx, int ny, int nz, int n_dirs,
                               const float* bare, double betaE, double betaO, int n_reemit,
                               void* scratch, long long scratch_bytes, float* flux_E,
                               float* flux_O, void* stream) {
    PETCH_REQUIRE(bare && scratch && flux_E && flux_O, "petch_dda_solve: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && (long long)nx * ny * nz < (1LL << 31),
                  "petch_dda_solve: bad grid");
    PETCH_REQUIRE(max_faces > 0 && n_dirs > 0 && (long long)max_faces * n_dirs < (1LL << 31),
                  "petch_dda_solve: max_faces * n_dirs must be in [1, 2^31)");
    const long long NC = (long long)nx * ny * nz;
    size_t need = 0;
    DDAScratch s;
    int rc = dda_layout(max_faces, NC, n_dirs, scratch, &need, &s);
    if (rc) return rc;
    PETCH_REQUIRE((long long)need <= scratch_bytes, "petch_dda_solve: scratch too small");
    cudaStream_t st = as_stream(stream);
    const int n = n_reemit > 1 ? n_reemit : 1;
    const int gf = grid_for(max_faces, kDB);
    // iterate i (1..n) reads V(i-1) and writes V(i); V(0) = direct, V(i) in ring[(i - 1) & 1]
    auto V = [&](int i) -> double2* { return i == 0 ? s.vf0 : s.ring + (size_t)((i - 1) & 1) * max_faces; };
    for (int i = 1; i <= n; ++i) {
        k_dda_remit<<<gf, kDB, 0, st>>>(V(i - 1), bare, betaE, betaO, s);
        PETCH_LAUNCH_CHECK("k_dda_remit");
        k_dda_fill<<<grid_for(s.fill_cap, kDB), kDB, 0, st>>>(nx, ny, nz, s);
        PETCH_LAUNCH_CHECK("k_dda_fill");
        const bool last = i == n;
        k_dda_gather<<<gf, kDB, 0, st>>>(max_faces, n_dirs, s, last ? nullptr : V(i), V(i - 1),
                                         (last && i >= 2) ? V(i - 2) : nullptr,
                                         last ? flux_E : nullptr, last ? flux_O : nullptr);
        PETCH_LAUNCH_CHECK("k_dda_gather");
    }
    return PETCH_OK;
}
