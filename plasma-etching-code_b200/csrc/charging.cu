// Charging hooks on the per-face ion results: the Hwang-Giapis closure
// (_apply_hg_charging, petch/threed.py:1046-1110) and the deep-AR floor throttle
// (_apply_floor_charge_throttle, petch/threed.py:1112-1147), and the electron-shadowing factor of
// mc_flux_3d_coupled (threed.py:847-868; k_electron_shadow below).
//
// The first two act on the same face classes: inside the feature footprint (within half the
// feature width + 2 dx of its axis), below sub_top, and either facing up (into-gas n_z > 0.7: the
// floor) or not (the sidewall; the HG "foot" is the part within foot_h of the deepest floor
// face).  The aspect-ratio tables they interpolate are host arithmetic on four numbers; the device
// gives those numbers (petch_charging_floor_stats, one block, fixed-order reductions) and applies
// the result to every face (petch_charging_apply).
#include "common.cuh"
#include "petch_b200.h"

namespace petch {
namespace {

constexpr int kCB = 1024;

struct FaceClass {
    double cx, cy, band, sub_top;
    int hole;
};

__device__ __forceinline__ bool in_feature(const FaceClass& c, const float* cen, int f) {
    const double x = cen[3 * f], y = cen[3 * f + 1], z = cen[3 * f + 2];
    const bool inside = c.hole ? hypot(x - c.cx, y - c.cy) <= c.band : fabs(x - c.cx) <= c.band;
    return inside && z < c.sub_top;
}

// stats: [0] floor faces, [1] min floor centroid z, [2] sum of m_i A over the floor,
//        [3] foot faces, [4] summed foot area (foot: in feature, n_z <= 0.7, z <= z_floor + foot_h)
__global__ void __launch_bounds__(kCB) k_floor_stats(const int* __restrict__ n_faces, int MF,
                                                     const float* __restrict__ cen,
                                                     const float* __restrict__ nrm,
                                                     const float* __restrict__ area,
                                                     const float* __restrict__ m_i, FaceClass c,
                                                     double foot_h, double* __restrict__ stats) {
    __shared__ float zmin_s[kCB];
    __shared__ double a_s[kCB], b_s[kCB], n_s[kCB], m_s[kCB];
    const int F = min(max(*n_faces, 0), MF);
    float zmin = INFINITY;
    double nfl = 0.0, ma = 0.0;
    for (int f = threadIdx.x; f < F; f += blockDim.x) {
        if (in_feature(c, cen, f) && (double)nrm[3 * f + 2] > 0.7) {
            zmin = fminf(zmin, cen[3 * f + 2]);
            nfl += 1.0;
            ma += (double)(m_i ? m_i[f] : 0.0f) * (double)area[f];
        }
    }
    zmin_s[threadIdx.x] = zmin;
    n_s[threadIdx.x] = nfl;
    m_s[threadIdx.x] = ma;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            zmin_s[threadIdx.x] = fminf(zmin_s[threadIdx.x], zmin_s[threadIdx.x + w]);
            n_s[threadIdx.x] += n_s[threadIdx.x + w];
            m_s[threadIdx.x] += m_s[threadIdx.x + w];
        }
        __syncthreads();
    }
    const double ztop = (double)zmin_s[0] + foot_h;
    double nfo = 0.0, fa = 0.0;
    for (int f = threadIdx.x; f < F; f += blockDim.x) {
        if (in_feature(c, cen, f) && !((double)nrm[3 * f + 2] > 0.7) && (double)cen[3 * f + 2] <= ztop) {
            nfo += 1.0;
            fa += (double)area[f];
        }
    }
    a_s[threadIdx.x] = nfo;
    b_s[threadIdx.x] = fa;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            a_s[threadIdx.x] += a_s[threadIdx.x + w];
            b_s[threadIdx.x] += b_s[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        stats[0] = n_s[0];
        stats[1] = (double)zmin_s[0];
        stats[2] = m_s[0];
        stats[3] = a_s[0];
        stats[4] = b_s[0];
    }
}

// floor: m_i *= q[0], y_sp *= q[1], y_ie *= q[2], y_p *= q[3];
// sidewall faces with z <= z_foot: y_sp += add[0], y_ie += add[1], y_p += add[2].
struct ChargeApply {
    double q[4];
    double add[3];
    double z_foot;
};

__global__ void k_charge_apply(const int* __restrict__ n_faces, int MF,
                               const float* __restrict__ cen, const float* __restrict__ nrm,
                               FaceClass c, ChargeApply a, float* __restrict__ m_i,
                               float* __restrict__ y_sp, float* __restrict__ y_ie,
                               float* __restrict__ y_p) {
    const int F = min(max(*n_faces, 0), MF);
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x) {
        if (!in_feature(c, cen, f)) continue;
        if ((double)nrm[3 * f + 2] > 0.7) {
            if (m_i) m_i[f] = (float)((double)m_i[f] * a.q[0]);
            if (y_sp) y_sp[f] = (float)((double)y_sp[f] * a.q[1]);
            if (y_ie) y_ie[f] = (float)((double)y_ie[f] * a.q[2]);
            if (y_p) y_p[f] = (float)((double)y_p[f] * a.q[3]);
        } else if ((double)cen[3 * f + 2] <= a.z_foot) {
            if (y_sp) y_sp[f] = (float)((double)y_sp[f] + a.add[0]);
            if (y_ie) y_ie[f] = (float)((double)y_ie[f] + a.add[1]);
            if (y_p) y_p[f] = (float)((double)y_p[f] + a.add[2]);
        }
    }
}

__global__ void k_zero_below(const int* __restrict__ n_faces, int MF, const float* __restrict__ cen,
                             double z_top, float* __restrict__ v) {
    const int F = min(max(*n_faces, 0), MF);
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x)
        if ((double)cen[3 * f + 2] <= z_top) v[f] = 0.0f;
}

// The electron-shadowing factor (threed.py:862-867): each flux is taken relative to its own
// open-field level (ref: the 90th percentile of its faces above 1e-6), clipped to [0, 1]; the ion
// result of a face is scaled by f = 1 - alpha clip(1 - sh_e / max(sh_i, 1e-3), 0, 1).  Float64,
// every product and difference rounded on its own (no contraction), as numpy evaluates it.
__global__ void k_electron_shadow(const int* __restrict__ n_faces, int MF,
                                  const float* __restrict__ m_e, double ref_i, double ref_e,
                                  double alpha, float* __restrict__ m_i) {
    const int F = min(max(*n_faces, 0), MF);
    const double ri = fmax(ref_i, 1e-6), re = fmax(ref_e, 1e-6);
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x) {
        const double mi = m_i[f];
        const double sh_e = fmin(fmax((double)m_e[f] / re, 0.0), 1.0);
        const double sh_i = fmin(fmax(mi / ri, 0.0), 1.0);
        const double gap = fmin(fmax(__dsub_rn(1.0, sh_e / fmax(sh_i, 1e-3)), 0.0), 1.0);
        const double fc = __dsub_rn(1.0, __dmul_rn(alpha, gap));
        m_i[f] = (float)__dmul_rn(mi, fc);
    }
}

}  // namespace
}  // namespace petch

using namespace petch;

extern "C" int petch_electron_shadow(const int* n_faces, int max_faces, const float* m_e,
                                     double ref_i, double ref_e, double alpha, float* m_i,
                                     void* stream) {
    PETCH_REQUIRE(n_faces && m_e && m_i, "petch_electron_shadow: null pointer");
    PETCH_REQUIRE(max_faces > 0, "petch_electron_shadow: bad face capacity");
    k_electron_shadow<<<grid_for(max_faces, 256), 256, 0, as_stream(stream)>>>(
        n_faces, max_faces, m_e, ref_i, ref_e, alpha, m_i);
    PETCH_LAUNCH_CHECK("k_electron_shadow");
    return PETCH_OK;
}

extern "C" int petch_zero_below(const int* n_faces, int max_faces, const float* centroids,
                                double z_top, float* values, void* stream) {
    PETCH_REQUIRE(n_faces && centroids && values, "petch_zero_below: null pointer");
    PETCH_REQUIRE(max_faces > 0, "petch_zero_below: bad face capacity");
    k_zero_below<<<grid_for(max_faces, 256), 256, 0, as_stream(stream)>>>(n_faces, max_faces,
                                                                          centroids, z_top, values);
    PETCH_LAUNCH_CHECK("k_zero_below");
    return PETCH_OK;
}

extern "C" int petch_charging_floor_stats(const int* n_faces, int max_faces,
                                          const float* centroids, const float* normals,
                                          const float* areas, const float* m_i, double cx,
                                          double cy, double band, int hole, double sub_top,
                                          double foot_h, double* stats, void* stream) {
    PETCH_REQUIRE(n_faces && centroids && normals && areas && stats,
                  "petch_charging_floor_stats: null pointer");
    PETCH_REQUIRE(max_faces > 0, "petch_charging_floor_stats: bad face capacity");
    FaceClass c{cx, cy, band, sub_top, hole ? 1 : 0};
    k_floor_stats<<<1, kCB, 0, as_stream(stream)>>>(n_faces, max_faces, centroids, normals, areas,
                                                   m_i, c, foot_h, stats);
    PETCH_LAUNCH_CHECK("k_floor_stats");
    return PETCH_OK;
}

extern "C" int petch_charging_apply(const int* n_faces, int max_faces, const float* centroids,
                                    const float* normals, double cx, double cy, double band,
                                    int hole, double sub_top, const double* q4, const double* add3,
                                    double z_foot, float* m_i, float* y_sp, float* y_ie,
                                    float* y_p, void* stream) {
    PETCH_REQUIRE(n_faces && centroids && normals && q4 && add3,
                  "petch_charging_apply: null pointer");
    PETCH_REQUIRE(max_faces > 0, "petch_charging_apply: bad face capacity");
    FaceClass c{cx, cy, band, sub_top, hole ? 1 : 0};
    ChargeApply a;
    for (int i = 0; i < 4; ++i) a.q[i] = q4[i];
    for (int i = 0; i < 3; ++i) a.add[i] = add3[i];
    a.z_foot = z_foot;
    k_charge_apply<<<grid_for(max_faces, 256), 256, 0, as_stream(stream)>>>(
        n_faces, max_faces, centroids, normals, c, a, m_i, y_sp, y_ie, y_p);
    PETCH_LAUNCH_CHECK("k_charge_apply");
    return PETCH_OK;
}
