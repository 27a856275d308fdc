// Per-face flux post-processing and surface chemistry, all on the device:
//   * normalisation (_norm_clip threed.py:165-170, the ion yields of mc_flux_3d_coupled
//     threed.py:814-823) and the 1-neighbour normal-weighted smoothing (smooth_flux /
//     smooth_flux_dev, threed.py:129-214) in gather form: each face sums over its three edge
//     neighbours, which is the pair scatter of the reference regrouped per face (no atomics);
//   * Belen coupled F/O coverages (_belen_coverages threed.py:715-737) -> bare coverage;
//   * surface rate (surface_rate_belen belen.py:26-63, surface_rate_langmuir
//     chemistry.py:96-114) with the mask zeroing, the non-finite guard of run_etch_3d
//     (threed.py:1723-1728) and the CFL maximum (threed.py:1750).
// Chemistry runs in float64 like the reference's numpy host code; flux arrays are float32.
#include "common.cuh"
#include "dual.cuh"
#include "levelset.cuh"
#include "mesh.cuh"

namespace petch {
namespace {

constexpr int kSB = 256;

// Smoothing of a normalised per-face field: out_i = (m_i + sum_j w_ij m_j) / (1 + sum_j w_ij),
// then out = (1 - alpha) * raw + alpha * out when alpha < 1.
__global__ void __launch_bounds__(kSB) k_smooth(MeshView m, const float* __restrict__ src,
                                                const float* __restrict__ raw, float alpha,
                                                float* __restrict__ out) {
    const int F = min(m.hdr[HDR_F], m.MT);
    for (int f = blockIdx.x * kSB + threadIdx.x; f < F; f += gridDim.x * kSB) {
        float num = src[f], den = 1.0f;
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            int j = m.nbr[3 * f + e];
            if (j >= 0) {
                float w = m.nbrw[3 * f + e];
                num += src[j] * w;
                den += w;
            }
        }
        float v = num / fmaxf(den, 1.0e-12f);
        if (alpha < 1.0f) v = (1.0f - alpha) * raw[f] + alpha * v;
        out[f] = v;
    }
}

// clamp((fl / A) * scale, lo, hi) (clip == 0: no clamp)
__global__ void __launch_bounds__(kSB) k_norm(MeshView m, const float* __restrict__ fl, float scale,
                                              float lo, float hi, int clip, float* __restrict__ out) {
    const int F = min(m.hdr[HDR_F], m.MT);
    for (int f = blockIdx.x * kSB + threadIdx.x; f < F; f += gridDim.x * kSB) {
        float v = (fl[f] / m.area[f]) * scale;
        if (clip) v = fminf(fmaxf(v, lo), hi);
        out[f] = v;
    }
}

// Ion tallies -> normalised (sp, ie, ip, m_i) (unsmoothed) and cos_i.
__global__ void __launch_bounds__(kSB) k_ion_norm(MeshView m, const float4* __restrict__ tal4,
                                                  const float* __restrict__ ang, float norm,
                                                  float* __restrict__ nsp, float* __restrict__ nie,
                                                  float* __restrict__ nip, float* __restrict__ nmi,
                                                  float* __restrict__ cos_i) {
    const int F = min(m.hdr[HDR_F], m.MT);
    for (int f = blockIdx.x * kSB + threadIdx.x; f < F; f += gridDim.x * kSB) {
        float4 t = tal4[f];
        float A = m.area[f];
        nsp[f] = (t.x / A) * norm;
        nie[f] = (t.y / A) * norm;
        nip[f] = (t.z / A) * norm;
        nmi[f] = (t.w / A) * norm;
        float fi = t.w;
        cos_i[f] = fi > 0.0f ? ang[f] / fmaxf(fi, 1.0e-9f) : 0.0f;
    }
}

struct Chem {
    double ionFlux, Fflux, Oflux, k_sigma, beta_sigma, rho, rate_scale, fnorm_E, fnorm_O, s_F,
        s_O, Yie, Ysp, Yp, B_sp;
    int viennaps, belen;
};

__device__ __forceinline__ void angular(double cos_i, const Chem& c, double& f_ie, double& f_sp) {
    double x = fmin(fmax(cos_i, 0.0), 1.0);
    if (c.viennaps) {
        f_sp = fmax((1.0 + c.B_sp * (1.0 - x * x)) * x, 0.0);
        double th = acos(x);
        f_ie = x >= 0.5 ? 1.0 : fmax(3.0 - 6.0 * th / 3.141592653589793, 0.0);
    } else {
        f_ie = x;
        f_sp = x;
    }
}

// _belen_coverages + bare = clip(1 - thF - thO, 0, 1)
__global__ void __launch_bounds__(kSB) k_belen_bare(MeshView m, Chem c, const float* __restrict__ m_i,
                                                    const float* __restrict__ m_F,
                                                    const float* __restrict__ m_O,
                                                    const float* __restrict__ cos_i,
                                                    const float* __restrict__ y_ie,
                                                    const float* __restrict__ y_ip,
                                                    float* __restrict__ bare) {
    const int F = min(m.hdr[HDR_F], m.MT);
    const double eps = 1e-9;
    for (int f = blockIdx.x * kSB + threadIdx.x; f < F; f += gridDim.x * kSB) {
        double GY_ie, GY_p;
        if (y_ie) {
            GY_ie = c.ionFlux * (double)y_ie[f];
            GY_p = c.ionFlux * (double)y_ip[f];
        } else {
            double f_ie, f_sp;
            angular(cos_i[f], c, f_ie, f_sp);
            double Fi = c.ionFlux * (double)m_i[f];
            GY_ie = c.Yie * f_ie * Fi;
            GY_p = c.Yp * f_ie * Fi;
        }
        double GbE = c.Fflux * (double)m_F[f] + eps;
        double GbP = c.Oflux * (double)m_O[f] + eps;
        double a = (c.k_sigma + 2.0 * GY_ie) / GbE;
        double b = (c.beta_sigma + GY_p) / GbP;
        double thF = 1.0 / (1.0 + a * (1.0 + 1.0 / (b + eps)));
        double thO = 1.0 / (1.0 + b * (1.0 + 1.0 / (a + eps)));
        bare[f] = (float)fmin(fmax(1.0 - thF - thO, 0.0), 1.0);
    }
}

// surface_rate_{belen,langmuir}: V per face (float32 of the float64 rate), 0 on mask faces;
// non-finite values are zeroed and counted in stats[0]; max(V) lands in stats[1] (float bits).
__global__ void __launch_bounds__(kSB) k_rate(MeshView m, Chem c, const float* __restrict__ m_i,
                                              const float* __restrict__ m_F,
                                              const float* __restrict__ m_O,
                                              const float* __restrict__ cos_i,
                                              const float* __restrict__ y_sp,
                                              const float* __restrict__ y_ie,
                                              const float* __restrict__ y_ip,
                                              float* __restrict__ V, int* stats) {
    const int F = min(m.hdr[HDR_F], m.MT);
    const double eps = 1e-9;
    int bad = 0;
    float vmax = 0.0f;
    for (int f = blockIdx.x * kSB + threadIdx.x; f < F; f += gridDim.x * kSB) {
        double f_ie, f_sp;
        angular(cos_i[f], c, f_ie, f_sp);
        double Fi = c.ionFlux * (double)m_i[f];
        double Yie_a = c.Yie * f_ie, Ysp_a = c.Ysp * f_sp, Yp_a = c.Yp * f_ie;
        double v;
        if (c.belen) {
            double GY_ie, GY_p, sputter, ion_enh;
            if (y_ie) {
                GY_ie = c.ionFlux * (double)y_ie[f];
                GY_p = c.ionFlux * (double)y_ip[f];
                sputter = c.ionFlux * (double)y_sp[f];
                ion_enh = GY_ie;
            } else {
                GY_ie = Yie_a * Fi;
                GY_p = Yp_a * Fi;
                sputter = Ysp_a * Fi;
                ion_enh = Yie_a * Fi;
            }
            double GbE = c.Fflux * (double)m_F[f] / c.fnorm_E + eps;
            double GbP = c.Oflux * (double)m_O[f] / c.fnorm_O + eps;
            double a = (c.k_sigma + 2.0 * GY_ie) / GbE;
            double b = (c.beta_sigma + GY_p) / GbP;
            double thF = 1.0 / (1.0 + a * (1.0 + 1.0 / (b + eps)));
            double rate = c.k_sigma * thF / 4.0 + sputter + thF * ion_enh;
            v = (1.0 / c.rho) * rate * c.rate_scale;
        } else {
            double Fev = c.Fflux * (double)m_F[f], Fp = c.Oflux * (double)m_O[f];
            double rF = c.s_F * Fev / (Yie_a * Fi + eps);
            double rO = c.s_O * Fp / (Yp_a * Fi + eps);
            double bare = 1.0 / (1.0 + rF + rO);
            double thF = rF * bare;
            v = (1.0 / c.rho) * (Yie_a * Fi * thF + Ysp_a * Fi * bare);
            v = v * c.rate_scale;
        }
        if (m.fmask[f]) v = 0.0;
        float vf = (float)v;
        if (!isfinite(v) || !isfinite(vf)) {
            ++bad;
            vf = 0.0f;
        }
        V[f] = vf;
        vmax = fmaxf(vmax, vf);
    }
    // block reduce then one atomic per block
    for (int o = 16; o > 0; o >>= 1) {
        vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicAdd(stats, bad);
        atomicMax(stats + 1, __float_as_int(fmaxf(vmax, 0.0f)));
    }
}

// ---- tangent (forward-mode) versions for the recipe gradient: the primal values bit for bit,
// plus N = 3 directional derivatives; tangent arrays are direction-major ([3][MT]) ----
constexpr int kND = 3;
using DD = Dual<double, kND>;

__device__ __forceinline__ DD ddload(const float* v, const float* d, int f, long long MT) {
    DD r;
    r.v = (double)v[f];
#pragma unroll
    for (int k = 0; k < kND; ++k) r.d[k] = d ? (double)d[f + k * MT] : 0.0;
    return r;
}

struct ParamTan {
    double dOflux[kND];      // d Oflux / d theta_k
    double drate[kND];       // d rate_scale / d theta_k
};

__device__ __forceinline__ DD dparam(double v, const double* d) {
    DD r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < kND; ++k) r.d[k] = d[k];
    return r;
}

// k_belen_bare with the faithful-ion yields, in dual arithmetic.
__global__ void __launch_bounds__(kSB) k_belen_bare_tan(MeshView m, Chem c, ParamTan pt,
                                                        const float* __restrict__ m_F,
                                                        const float* __restrict__ dm_F,
                                                        const float* __restrict__ m_O,
                                                        const float* __restrict__ dm_O,
                                                        const float* __restrict__ y_ie,
                                                        const float* __restrict__ dy_ie,
                                                        const float* __restrict__ y_ip,
                                                        const float* __restrict__ dy_ip,
                                                        float* __restrict__ bare,
                                                        float* __restrict__ dbare) {
    const int F = min(m.hdr[HDR_F], m.MT);
    const long long MT = m.MT;
    const double eps = 1e-9;
    const DD Oflux = dparam(c.Oflux, pt.dOflux);
    for (int f = blockIdx.x * kSB + threadIdx.x; f < F; f += gridDim.x * kSB) {
        const DD GY_ie = c.ionFlux * ddload(y_ie, dy_ie, f, MT);
        const DD GY_p = c.ionFlux * ddload(y_ip, dy_ip, f, MT);
        const DD GbE = c.Fflux * ddload(m_F, dm_F, f, MT) + eps;
        const DD GbP = Oflux * ddload(m_O, dm_O, f, MT) + eps;
        const DD a = (c.k_sigma + 2.0 * GY_ie) / GbE;
        const DD b = (c.beta_sigma + GY_p) / GbP;
        const DD thF = 1.0 / (1.0 + a * (1.0 + 1.0 / (b + eps)));
        const DD thO = 1.0 / (1.0 + b * (1.0 + 1.0 / (a + eps)));
        const DD x = 1.0 - thF - thO;
        const bool inside = x.v > 0.0 && x.v < 1.0;
        bare[f] = (float)fmin(fmax(x.v, 0.0), 1.0);
#pragma unroll
        for (int k = 0; k < kND; ++k) dbare[f + k * MT] = inside ? (float)x.d[k] : 0.0f;
    }
}

// k_rate (Belen chemistry, faithful-ion yields) in dual arithmetic; stats as k_rate.
__global__ void __launch_bounds__(kSB) k_rate_tan(MeshView m, Chem c, ParamTan pt,
                                                  const float* __restrict__ m_F,
                                                  const float* __restrict__ dm_F,
                                                  const float* __restrict__ m_O,
                                                  const float* __restrict__ dm_O,
                                                  const float* __restrict__ y_sp,
                                                  const float* __restrict__ dy_sp,
                                                  const float* __restrict__ y_ie,
                                                  const float* __restrict__ dy_ie,
                                                  const float* __restrict__ y_ip,
                                                  const float* __restrict__ dy_ip,
                                                  float* __restrict__ V, float* __restrict__ dV,
                                                  int* stats) {
    const int F = min(m.hdr[HDR_F], m.MT);
    const long long MT = m.MT;
    const double eps = 1e-9;
    const DD Oflux = dparam(c.Oflux, pt.dOflux);
    const DD rs = dparam(c.rate_scale, pt.drate);
    int bad = 0;
    float vmax_ = 0.0f;
    for (int f = blockIdx.x * kSB + threadIdx.x; f < F; f += gridDim.x * kSB) {
        const DD GY_ie = c.ionFlux * ddload(y_ie, dy_ie, f, MT);
        const DD GY_p = c.ionFlux * ddload(y_ip, dy_ip, f, MT);
        const DD sputter = c.ionFlux * ddload(y_sp, dy_sp, f, MT);
        const DD ion_enh = GY_ie;
        const DD GbE = c.Fflux * ddload(m_F, dm_F, f, MT) / c.fnorm_E + eps;
        const DD GbP = Oflux * ddload(m_O, dm_O, f, MT) / c.fnorm_O + eps;
        const DD a = (c.k_sigma + 2.0 * GY_ie) / GbE;
        const DD b = (c.beta_sigma + GY_p) / GbP;
        const DD thF = 1.0 / (1.0 + a * (1.0 + 1.0 / (b + eps)));
        const DD rate = c.k_sigma * thF / 4.0 + sputter + thF * ion_enh;
        DD v = (1.0 / c.rho) * rate * rs;
        if (m.fmask[f]) v = dconst<double, kND>(0.0);
        float vf = (float)v.v;
        bool ok = isfinite(v.v) && isfinite(vf);
        if (!ok) {
            ++bad;
            vf = 0.0f;
        }
        V[f] = vf;
#pragma unroll
        for (int k = 0; k < kND; ++k) dV[f + k * MT] = ok ? (float)v.d[k] : 0.0f;
        vmax_ = fmaxf(vmax_, vf);
    }
    for (int o = 16; o > 0; o >>= 1) {
        vmax_ = fmaxf(vmax_, __shfl_xor_sync(0xffffffffu, vmax_, o));
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicAdd(stats, bad);
        atomicMax(stats + 1, __float_as_int(fmaxf(vmax_, 0.0f)));
    }
}

// Tangent of clamp((fl / A) * scale, lo, hi): d(out) = (d fl / A) * scale inside the clamp.
__global__ void __launch_bounds__(kSB) k_norm_tan(MeshView m, const float* __restrict__ fl,
                                                  const float* __restrict__ dfl, float scale,
                                                  float lo, float hi, int clip,
                                                  float* __restrict__ dout) {
    const int F = min(m.hdr[HDR_F], m.MT);
    for (int f = blockIdx.x * kSB + threadIdx.x; f < F; f += gridDim.x * kSB) {
        const float A = m.area[f];
        const float v = (fl[f] / A) * scale;
        const bool inside = !clip || (v > lo && v < hi);
        dout[f] = inside ? (dfl[f] / A) * scale : 0.0f;
    }
}

Chem to_chem(const petch_chem_params* p) {
    Chem c;
    c.ionFlux = p->ionFlux;
    c.Fflux = p->Fflux;
    c.Oflux = p->Oflux;
    c.k_sigma = p->k_sigma;
    c.beta_sigma = p->beta_sigma;
    c.rho = p->rho;
    c.rate_scale = p->rate_scale;
    c.fnorm_E = p->fnorm_E;
    c.fnorm_O = p->fnorm_O;
    c.s_F = p->s_F;
    c.s_O = p->s_O;
    c.Yie = p->Yie;
    c.Ysp = p->Ysp;
    c.Yp = p->Yp;
    c.B_sp = p->B_sp;
    c.viennaps = p->yield_angular;
    c.belen = p->chemistry;
    return c;
}

// ---- sparse narrow-band advection -----------------------------------------------------------
struct AGrid {
    int nx, ny, nz;
    long long plane;
};

__global__ void __launch_bounds__(kSB) k_pin(float* __restrict__ dst, const int* __restrict__ idx,
                                             int n, const float* __restrict__ mask_phi) {
    for (int s = blockIdx.x * kSB + threadIdx.x; s < n; s += gridDim.x * kSB) {
        int c = idx[s];
        dst[c] = mask_phi[c];
    }
}

// One substep over the listed cells only (threed.py:1262-1292 restricted to F > 0 cells; all
// other cells are constant or pinned and identical in both buffers).
__global__ void __launch_bounds__(kSB) k_advect_list(const float* __restrict__ phi,
                                                     float* __restrict__ out,
                                                     const float* __restrict__ F,
                                                     const int* __restrict__ idx, int n, AGrid g,
                                                     float inv_dx, float dt) {
    const LGrid lg = make_lgrid(g.nx, g.ny, g.nz);
    for (int s = blockIdx.x * kSB + threadIdx.x; s < n; s += gridDim.x * kSB) {
        long long c = idx[s];
        out[c] = advect_cell(phi, c, lg, inv_dx, F[c], dt);
    }
}

__global__ void __launch_bounds__(kSB) k_copy_list(float* __restrict__ dst, const float* __restrict__ src,
                                                   const int* __restrict__ idx, int n) {
    for (int s = blockIdx.x * kSB + threadIdx.x; s < n; s += gridDim.x * kSB) dst[idx[s]] = src[idx[s]];
}

}  // namespace
}  // namespace petch

using namespace petch;

extern "C" int petch_norm_smooth(const void* mesh, int max_tris, int max_verts, const float* fl,
                                 float scale, float lo, float hi, int clip, int n_smooth,
                                 float alpha, float* out, float* tmp_a, float* tmp_b, void* stream) {
    PETCH_REQUIRE(mesh && fl && out && tmp_a && tmp_b, "petch_norm_smooth: null pointer");
    PETCH_REQUIRE(n_smooth >= 0, "petch_norm_smooth: n_smooth must be >= 0");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    int b = grid_for(max_tris, kSB);
    if (n_smooth == 0 || alpha <= 0.0f) {
        k_norm<<<b, kSB, 0, st>>>(m, fl, scale, lo, hi, clip, out);
        PETCH_LAUNCH_CHECK("k_norm");
        return PETCH_OK;
    }
    k_norm<<<b, kSB, 0, st>>>(m, fl, scale, lo, hi, clip, tmp_a);
    PETCH_LAUNCH_CHECK("k_norm");
    // smooth_flux_dev applied n_smooth times, each blending against its own input
    const float* src = tmp_a;
    for (int it = 0; it < n_smooth; ++it) {
        float* dst = (it == n_smooth - 1) ? out : (src == tmp_a ? tmp_b : tmp_a);
        k_smooth<<<b, kSB, 0, st>>>(m, src, src, alpha, dst);
        PETCH_LAUNCH_CHECK("k_smooth");
        src = dst;
    }
    return PETCH_OK;
}

extern "C" int petch_ion_post(const void* mesh, int max_tris, int max_verts, const float* tally4,
                              const float* ang, float norm, int n_smooth, float alpha,
                              float* y_sp, float* y_ie, float* y_ip, float* m_i, float* cos_i,
                              float* tmp, void* stream) {
    PETCH_REQUIRE(mesh && tally4 && ang && y_sp && y_ie && y_ip && m_i && cos_i && tmp,
                  "petch_ion_post: null pointer");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    int b = grid_for(max_tris, kSB);
    float* nrm = tmp;  // 5 * max_tris floats: normalised sp, ie, ip, m_i + one ping buffer
    float* outs[4] = {y_sp, y_ie, y_ip, m_i};
    bool smooth = n_smooth > 0 && alpha > 0.0f;
    float* dst0 = smooth ? nrm : y_sp;
    float* dst1 = smooth ? nrm + max_tris : y_ie;
    float* dst2 = smooth ? nrm + 2LL * max_tris : y_ip;
    float* dst3 = smooth ? nrm + 3LL * max_tris : m_i;
    k_ion_norm<<<b, kSB, 0, st>>>(m, (const float4*)tally4, ang, norm, dst0, dst1, dst2, dst3, cos_i);
    PETCH_LAUNCH_CHECK("k_ion_norm");
    if (!smooth) return PETCH_OK;
    // smooth_flux_gpu: n_smooth passes, each on the previous pass, blended with the raw field once
    // at the end.  Destinations alternate between the output and tmp[4*MT..5*MT) so the last pass
    // lands in the output and no pass reads what it writes.
    float* ping = nrm + 4LL * max_tris;
    for (int q = 0; q < 4; ++q) {
        const float* raw = nrm + (long long)q * max_tris;
        const float* src = raw;
        for (int it = 0; it < n_smooth; ++it) {
            bool last = it == n_smooth - 1;
            float* dst = ((n_smooth - 1 - it) % 2 == 0) ? outs[q] : ping;
            k_smooth<<<b, kSB, 0, st>>>(m, src, raw, last ? alpha : 1.0f, dst);
            PETCH_LAUNCH_CHECK("k_smooth");
            src = dst;
        }
    }
    return PETCH_OK;
}

extern "C" int petch_belen_bare(const void* mesh, int max_tris, int max_verts,
                                const petch_chem_params* p, const float* m_i, const float* m_F,
                                const float* m_O, const float* cos_i, const float* y_ie,
                                const float* y_ip, float* bare, void* stream) {
    PETCH_REQUIRE(mesh && p && m_i && m_F && m_O && cos_i && bare, "petch_belen_bare: null pointer");
    PETCH_REQUIRE((y_ie == nullptr) == (y_ip == nullptr), "petch_belen_bare: pass both yields or neither");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    k_belen_bare<<<grid_for(max_tris, kSB), kSB, 0, st>>>(m, to_chem(p), m_i, m_F, m_O, cos_i, y_ie,
                                                          y_ip, bare);
    PETCH_LAUNCH_CHECK("k_belen_bare");
    return PETCH_OK;
}

extern "C" int petch_surface_rate(const void* mesh, int max_tris, int max_verts,
                                  const petch_chem_params* p, const float* m_i, const float* m_F,
                                  const float* m_O, const float* cos_i, const float* y_sp,
                                  const float* y_ie, const float* y_ip, float* V, int* stats,
                                  void* stream) {
    PETCH_REQUIRE(mesh && p && m_i && m_F && m_O && cos_i && V && stats,
                  "petch_surface_rate: null pointer");
    PETCH_REQUIRE((y_sp == nullptr) == (y_ie == nullptr) && (y_ie == nullptr) == (y_ip == nullptr),
                  "petch_surface_rate: pass all three yields or none");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    PETCH_CUDA(cudaMemsetAsync(stats, 0, 2 * sizeof(int), st), "memset stats");
    k_rate<<<grid_for(max_tris, kSB), kSB, 0, st>>>(m, to_chem(p), m_i, m_F, m_O, cos_i, y_sp, y_ie,
                                                    y_ip, V, stats);
    PETCH_LAUNCH_CHECK("k_rate");
    return PETCH_OK;
}

__global__ void __launch_bounds__(kSB) k_cos_ratio(MeshView m, const float* __restrict__ fl,
                                                   const float* __restrict__ ang,
                                                   float* __restrict__ out) {
    const int F = min(m.hdr[HDR_F], m.MT);
    for (int f = blockIdx.x * kSB + threadIdx.x; f < F; f += gridDim.x * kSB)
        out[f] = fl[f] > 0.0f ? ang[f] / fl[f] : 0.0f;
}

extern "C" int petch_cos_ratio(const void* mesh, int max_tris, int max_verts, const float* fl,
                               const float* ang, float* out, void* stream) {
    PETCH_REQUIRE(mesh && fl && ang && out, "petch_cos_ratio: null pointer");
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    k_cos_ratio<<<grid_for(max_tris, kSB), kSB, 0, as_stream(stream)>>>(m, fl, ang, out);
    PETCH_LAUNCH_CHECK("k_cos_ratio");
    return PETCH_OK;
}

extern "C" int petch_advect_sparse(float* phi, float* tmp, const float* F, const float* mask_phi,
                                   const int* mask_idx, int n_mask, const int* active, int n_active,
                                   int nx, int ny, int nz, float inv_dx, float dt_sub, int nsub,
                                   void* stream) {
    PETCH_REQUIRE(phi && tmp && F && mask_phi && (n_mask == 0 || mask_idx) &&
                      (n_active == 0 || active),
                  "petch_advect_sparse: null pointer");
    PETCH_REQUIRE(nx > 0 && ny > 0 && nz > 0 && nsub >= 0 && n_mask >= 0 && n_active >= 0,
                  "petch_advect_sparse: bad size");
    PETCH_REQUIRE(phi != tmp, "petch_advect_sparse: phi and tmp must differ");
    if (nsub == 0) return PETCH_OK;
    cudaStream_t st = as_stream(stream);
    long long n = (long long)nx * ny * nz;
    AGrid g{nx, ny, nz, (long long)ny * nz};
    PETCH_CUDA(cudaMemcpyAsync(tmp, phi, sizeof(float) * n, cudaMemcpyDeviceToDevice, st),
               "petch_advect_sparse copy");
    int bm = grid_for(n_mask, kSB), ba = grid_for(n_active, kSB);
    if (n_mask) {
        k_pin<<<bm, kSB, 0, st>>>(tmp, mask_idx, n_mask, mask_phi);
        PETCH_LAUNCH_CHECK("k_pin");
    }
    float* a = phi;
    float* b = tmp;
    for (int s = 0; s < nsub; ++s) {
        if (n_active) {
            k_advect_list<<<ba, kSB, 0, st>>>(a, b, F, active, n_active, g, inv_dx, dt_sub);
            PETCH_LAUNCH_CHECK("k_advect_list");
        }
        if (s == 0 && n_mask) {
            k_pin<<<bm, kSB, 0, st>>>(phi, mask_idx, n_mask, mask_phi);
            PETCH_LAUNCH_CHECK("k_pin");
        }
        float* t = a;
        a = b;
        b = t;
    }
    if (a != phi && n_active) {
        k_copy_list<<<ba, kSB, 0, st>>>(phi, a, active, n_active);
        PETCH_LAUNCH_CHECK("k_copy_list");
    }
    return PETCH_OK;
}

static ParamTan param_tan(const double* dOflux, const double* drate) {
    ParamTan pt;
    for (int k = 0; k < kND; ++k) {
        pt.dOflux[k] = dOflux ? dOflux[k] : 0.0;
        pt.drate[k] = drate ? drate[k] : 0.0;
    }
    return pt;
}

extern "C" int petch_norm_smooth_tangent(const void* mesh, int max_tris, int max_verts,
                                         const float* fl, const float* dfl, float scale, float lo,
                                         float hi, int clip, int n_smooth, float alpha,
                                         int blend_last_only, float* dout, float* tmp_a,
                                         float* tmp_b, void* stream) {
    PETCH_REQUIRE(mesh && fl && dfl && dout && tmp_a && tmp_b,
                  "petch_norm_smooth_tangent: null pointer");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    const int b = grid_for(max_tris, kSB);
    const long long MT = max_tris;
    for (int k = 0; k < kND; ++k) {
        float* out = dout + k * MT;
        const bool smooth = n_smooth > 0 && alpha > 0.0f;
        k_norm_tan<<<b, kSB, 0, st>>>(m, fl, dfl + k * MT, scale, lo, hi, clip, smooth ? tmp_a : out);
        PETCH_LAUNCH_CHECK("k_norm_tan");
        if (!smooth) continue;
        // the primal's smoothing passes on the tangent (the smoothing is linear): each pass
        // blended with its own input (petch_norm_smooth) or only the last pass blended with the
        // raw field (petch_ion_post, blend_last_only)
        const float* raw = tmp_a;
        const float* src = tmp_a;
        for (int it = 0; it < n_smooth; ++it) {
            const bool last = it == n_smooth - 1;
            float* dst;
            if (blend_last_only)      // as petch_ion_post: the raw field stays intact to the end
                dst = ((n_smooth - 1 - it) % 2 == 0) ? out : tmp_b;
            else                      // as petch_norm_smooth
                dst = last ? out : (src == tmp_a ? tmp_b : tmp_a);
            const float* blend = blend_last_only ? raw : src;
            const float a = blend_last_only ? (last ? alpha : 1.0f) : alpha;
            k_smooth<<<b, kSB, 0, st>>>(m, src, blend, a, dst);
            PETCH_LAUNCH_CHECK("k_smooth");
            src = dst;
        }
    }
    return PETCH_OK;
}

extern "C" int petch_belen_bare_tangent(const void* mesh, int max_tris, int max_verts,
                                        const petch_chem_params* p, const double* dOflux,
                                        const float* m_F, const float* dm_F, const float* m_O,
                                        const float* dm_O, const float* y_ie, const float* dy_ie,
                                        const float* y_ip, const float* dy_ip, float* bare,
                                        float* dbare, void* stream) {
    PETCH_REQUIRE(mesh && p && m_F && m_O && y_ie && y_ip && bare && dbare,
                  "petch_belen_bare_tangent: null pointer");
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    k_belen_bare_tan<<<grid_for(max_tris, kSB), kSB, 0, as_stream(stream)>>>(
        m, to_chem(p), param_tan(dOflux, nullptr), m_F, dm_F, m_O, dm_O, y_ie, dy_ie, y_ip, dy_ip,
        bare, dbare);
    PETCH_LAUNCH_CHECK("k_belen_bare_tan");
    return PETCH_OK;
}

extern "C" int petch_surface_rate_tangent(const void* mesh, int max_tris, int max_verts,
                                          const petch_chem_params* p, const double* dOflux,
                                          const double* drate, const float* m_F, const float* dm_F,
                                          const float* m_O, const float* dm_O, const float* y_sp,
                                          const float* dy_sp, const float* y_ie,
                                          const float* dy_ie, const float* y_ip,
                                          const float* dy_ip, float* V, float* dV, int* stats,
                                          void* stream) {
    PETCH_REQUIRE(mesh && p && m_F && m_O && y_sp && y_ie && y_ip && V && dV && stats,
                  "petch_surface_rate_tangent: null pointer");
    PETCH_REQUIRE(p->chemistry == 1, "petch_surface_rate_tangent: Belen chemistry only");
    cudaStream_t st = as_stream(stream);
    MeshView m = mesh_view(const_cast<void*>(mesh), max_tris, max_verts);
    PETCH_CUDA(cudaMemsetAsync(stats, 0, 2 * sizeof(int), st), "memset stats");
    k_rate_tan<<<grid_for(max_tris, kSB), kSB, 0, st>>>(m, to_chem(p), param_tan(dOflux, drate), m_F,
                                                        dm_F, m_O, dm_O, y_sp, dy_sp, y_ie, dy_ie,
                                                        y_ip, dy_ip, V, dV, stats);
    PETCH_LAUNCH_CHECK("k_rate_tan");
    return PETCH_OK;
}
