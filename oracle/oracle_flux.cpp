// ORACLE -- test infrastructure only.  FP64 CPU restatement of petch's Monte-Carlo flux kernels:
//   source                : _gen_source            petch/threed.py:441-458
//   lateral wrap          : _apply_bc              petch/threed.py:289-349
//   Russian-roulette neut.: _trace3d_cov_rr        petch/threed.py:549-596
//   faithful ion          : _trace3d_ion_yield     petch/threed.py:599-712
//   legacy species        : _trace3d               petch/threed.py:352-406
//   form-factor rays      : _trace_ff + emission   petch/threed.py:908-920, 947-956, 1571-1579
//   redeposition          : mc_redep_3d            petch/threed.py:1582-1605
// The random stream is this file's own (SplitMix64 counter hash per (seed, domain, ray)), not the
// device's Philox and not Warp's: these are oracles of the same estimator, checked statistically.
// Parity pin: tests/golden/flux.npz holds per-face means of the reference's own kernels (executed
// through tests/golden/warp_shim.py) on small meshes.
#include <cmath>
#include <cstdint>
#include <vector>

namespace orc {
struct HitD {
    double t;
    int f;
};
}  // namespace orc

// provided by oracle_mesh.cpp (same library)
struct Mesh;
namespace orc {
HitD closest_hit(const Mesh* m, const double o[3], const double d[3], double tmax);
void face_normal(const Mesh* m, int f, double n[3]);
}  // namespace orc

namespace {

struct Rng {
    uint64_t s;
    double spare;
    bool has;
    Rng(uint64_t seed, uint64_t domain, uint64_t ray) : has(false) {
        s = seed * 0x9E3779B97F4A7C15ULL ^ (domain + 0x632BE59BD9B4E019ULL) * 0xBF58476D1CE4E5B9ULL ^
            (ray + 1) * 0x94D049BB133111EBULL;
        next();
        next();
    }
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    double normal() {
        if (has) {
            has = false;
            return spare;
        }
        double u1 = 1.0 - uniform(), u2 = uniform();
        double r = std::sqrt(-2.0 * std::log(u1));
        spare = r * std::sin(6.283185307179586 * u2);
        has = true;
        return r * std::cos(6.283185307179586 * u2);
    }
};

struct Dom {
    double lx, ly, lz, z_src;
    int periodic;
};

double dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
void cross(const double* a, const double* b, double* r) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
void normalize(double* v) {
    double l = std::sqrt(dot(v, v));
    if (l > 0)
        for (int q = 0; q < 3; ++q) v[q] /= l;
}

// _apply_bc + the kernel's own query.
orc::HitD query(const Mesh* m, double o[3], const double d[3], const Dom& D) {
    if (!D.periodic) return orc::closest_hit(m, o, d, 1.0e6);
    for (int w = 0; w < 256; ++w) {
        orc::HitD h = orc::closest_hit(m, o, d, 1.0e6);
        if (h.f >= 0) return h;
        double tx = 1e30, ty = 1e30, tz = 1e30;
        if (d[0] > 1e-9) tx = (D.lx - o[0]) / d[0];
        if (d[0] < -1e-9) tx = (0.0 - o[0]) / d[0];
        if (d[1] > 1e-9) ty = (D.ly - o[1]) / d[1];
        if (d[1] < -1e-9) ty = (0.0 - o[1]) / d[1];
        if (d[2] > 1e-9) tz = (D.lz - o[2]) / d[2];
        if (tx < tz && tx < ty && tx > 1e-7) {
            double hy = o[1] + tx * d[1], hz = o[2] + tx * d[2];
            o[0] = d[0] < 0 ? D.lx - 1e-4 : 1e-4;
            o[1] = hy;
            o[2] = hz;
        } else if (ty < tz && ty < 1e29 && ty > 1e-7) {
            double hx = o[0] + ty * d[0], hz = o[2] + ty * d[2];
            o[0] = hx;
            o[1] = d[1] < 0 ? D.ly - 1e-4 : 1e-4;
            o[2] = hz;
        } else {
            return h;
        }
    }
    return orc::closest_hit(m, o, d, 1.0e6);
}

void source(Rng& g, bool ion, double sigma, const Dom& D, double o[3], double d[3]) {
    o[0] = g.uniform() * D.lx;
    o[1] = g.uniform() * D.ly;
    o[2] = D.z_src;
    if (ion) {
        double ax = g.normal() * sigma, ay = g.normal() * sigma;
        d[0] = std::sin(ax);
        d[1] = std::sin(ay);
        d[2] = -std::cos(ax) * std::cos(ay);
    } else {
        double r1 = g.uniform(), r2 = g.uniform();
        double ct = std::sqrt(r1), s = std::sqrt(1 - r1), ph = 6.2831853 * r2;
        d[0] = s * std::cos(ph);
        d[1] = s * std::sin(ph);
        d[2] = -ct;
    }
    normalize(d);
}

void cosine_emit(Rng& g, const double n[3], double d[3]) {
    double a[3] = {1, 0, 0};
    if (std::fabs(n[0]) > 0.9) {
        a[0] = 0;
        a[1] = 1;
    }
    double t[3], b[3];
    cross(a, n, t);
    normalize(t);
    cross(n, t, b);
    double r1 = g.uniform(), r2 = g.uniform();
    double ct = std::sqrt(r1), st = std::sqrt(1 - r1), ph = 6.2831853 * r2;
    for (int q = 0; q < 3; ++q) d[q] = st * std::cos(ph) * t[q] + st * std::sin(ph) * b[q] + ct * n[q];
}

void oriented_normal(const Mesh* m, int f, const double d[3], double n[3]) {
    orc::face_normal(m, f, n);
    if (dot(n, d) > 0)
        for (int q = 0; q < 3; ++q) n[q] = -n[q];
}

void add(double* a, int i, double v) {
#pragma omp atomic
    a[i] += v;
}

}  // namespace

extern "C" {

// tallies: double[5*F] = (sp, ie, ip, arr, ang) per face, accumulated (caller zeroes).
// prm: meanE sigmaE A_sp Eth_sp B_sp A_ie Eth_ie A_p Eth_p inflect minang n_l A_en minE thrmin
//      thrmax sigma ; dom: lx ly lz z_src periodic
void orc_trace_ions(void* mesh, const double* prm, const double* dom, uint64_t seed, int n,
                    double* tal) {
    const Mesh* m = (const Mesh*)mesh;
    Dom D{dom[0], dom[1], dom[2], dom[3], (int)dom[4]};
    const double meanE = prm[0], sigmaE = prm[1], A_sp = prm[2], Eth_sp = prm[3], B_sp = prm[4],
                 A_ie = prm[5], Eth_ie = prm[6], A_p = prm[7], Eth_p = prm[8], inflect = prm[9],
                 minang = prm[10], n_l = prm[11], A_en = prm[12], minE = prm[13], thrmin = prm[14],
                 thrmax = prm[15], sigma = prm[16];
    const double PI_2 = 1.5707963;
    const double sEsp = std::sqrt(Eth_sp), sEie = std::sqrt(Eth_ie), sEp = std::sqrt(Eth_p);
#pragma omp parallel for schedule(dynamic, 64)
    for (int p = 0; p < n; ++p) {
        Rng g(seed, 0x696f6e73, (uint64_t)p);
        double o[3], d[3];
        source(g, true, sigma, D, o, d);
        double E = meanE + sigmaE * g.normal();
        if (E < 0) E = 0;
        double w = 1.0;
        for (int bounce = 0; bounce < 1024; ++bounce) {
            orc::HitD h = query(m, o, d, D);
            if (h.f < 0) break;
            double nr[3];
            oriented_normal(m, h.f, d, nr);
            double cosT = -dot(d, nr);
            cosT = std::min(std::max(cosT, 0.0), 1.0);
            double incAng = std::acos(cosT);
            double sqrtE = std::sqrt(E);
            double f_sp = std::max((1.0 + B_sp * (1.0 - cosT * cosT)) * cosT, 0.0);
            double f_ie = 1.0;
            if (cosT < 0.5) f_ie = std::max(3.0 - 6.0 * incAng / 3.14159265, 0.0);
            int f = h.f;
            add(tal, 5 * f + 0, A_sp * std::max(sqrtE - sEsp, 0.0) * f_sp * w);
            add(tal, 5 * f + 1, A_ie * std::max(sqrtE - sEie, 0.0) * f_ie * w);
            add(tal, 5 * f + 2, A_p * std::max(sqrtE - sEp, 0.0) * f_ie * w);
            add(tal, 5 * f + 3, w);
            add(tal, 5 * f + 4, cosT * w);
            double stick = 1.0;
            if (incAng > thrmin) {
                double rr = std::min(std::max((incAng - thrmin) / (thrmax - thrmin), 0.0), 1.0);
                stick = 1.0 - rr;
            }
            if (stick >= 1.0) break;
            double Eref = incAng >= inflect ? 1.0 - (1.0 - A_en) * (PI_2 - incAng) / (PI_2 - inflect)
                                            : A_en * std::pow(incAng / inflect, n_l);
            double newE = Eref * E;
            for (int e = 0; e < 4; ++e) {
                double cand = Eref * E + 0.1 * E * g.normal();
                if (cand >= 0 && cand <= E) {
                    newE = cand;
                    break;
                }
            }
            newE = std::min(std::max(newE, 0.0), E);
            if (newE <= minE) break;
            E = newE;
            w = w - w * stick;
            if (w <= 1e-4) break;
            double hit[3] = {o[0] + h.t * d[0], o[1] + h.t * d[1], o[2] + h.t * d[2]};
            double dn = dot(d, nr);
            double axis[3] = {d[0] - 2 * dn * nr[0], d[1] - 2 * dn * nr[1], d[2] - 2 * dn * nr[2]};
            normalize(axis);
            double tt[3], bb[3];
            if (axis[2] < -0.9999999) {
                tt[0] = 0; tt[1] = -1; tt[2] = 0;
                bb[0] = -1; bb[1] = 0; bb[2] = 0;
            } else {
                double aa = 1.0 / (1.0 + axis[2]), cc = -axis[0] * axis[1] * aa;
                tt[0] = 1 - axis[0] * axis[0] * aa; tt[1] = cc; tt[2] = -axis[0];
                bb[0] = cc; bb[1] = 1 - axis[1] * axis[1] * aa; bb[2] = -axis[1];
            }
            double maxcone = PI_2 - std::min(incAng, minang);
            double theta = 0.0;
            for (int q = 0; q < 64; ++q) {
                double uu = std::sqrt(g.uniform());
                double ss = std::sqrt(std::max(1.0 - uu, 0.0));
                theta = maxcone * ss;
                if (g.uniform() * theta * uu <= std::cos(PI_2 * ss) * std::sin(theta)) break;
            }
            double ph = 6.2831853 * g.uniform();
            double nd[3];
            for (int q = 0; q < 3; ++q)
                nd[q] = std::sin(theta) * (std::cos(ph) * tt[q] + std::sin(ph) * bb[q]) + std::cos(theta) * axis[q];
            normalize(nd);
            double nn = dot(nd, nr);
            if (nn <= 0)
                for (int q = 0; q < 3; ++q) nd[q] -= 2 * nn * nr[q];
            for (int q = 0; q < 3; ++q) {
                d[q] = nd[q];
                o[q] = hit[q] + 1e-4 * nr[q];
            }
        }
    }
}

// flux: double[F] arriving weight (caller zeroes).  bare may be NULL (=1).
void orc_trace_neutrals(void* mesh, const double* dom, const double* bare, double beta,
                        uint64_t seed, uint64_t domain, int n, double* flux) {
    const Mesh* m = (const Mesh*)mesh;
    Dom D{dom[0], dom[1], dom[2], dom[3], (int)dom[4]};
#pragma omp parallel for schedule(dynamic, 64)
    for (int p = 0; p < n; ++p) {
        Rng g(seed, 0x6e657500ULL ^ domain, (uint64_t)p);
        double o[3], d[3];
        source(g, false, 0.0, D, o, d);
        double w = 1.0;
        for (int bounce = 0; bounce < 1024; ++bounce) {
            orc::HitD h = query(m, o, d, D);
            if (h.f < 0) break;
            double nr[3];
            oriented_normal(m, h.f, d, nr);
            add(flux, h.f, w);
            double S = (bare ? bare[h.f] : 1.0) * beta;
            w = w - w * S;
            if (w <= 1e-6) break;
            if (w < 0.1) {
                if (g.uniform() < (1.0 - w / 0.3)) break;
                w = 0.3;
            }
            double hit[3] = {o[0] + h.t * d[0], o[1] + h.t * d[1], o[2] + h.t * d[2]};
            cosine_emit(g, nr, d);
            for (int q = 0; q < 3; ++q) o[q] = hit[q] + 1e-4 * nr[q];
        }
    }
}

// The electron trace of mc_flux_3d_coupled's charging block (threed.py:852-856): the ion-type
// source with tilt sigma, _trace3d_cov_rr with bare = 1 and beta = 1 -> weight 1 on the first face
// reached, with the domain's lateral wrap.  flux double[F] (caller zeroes).
void orc_trace_electrons(void* mesh, const double* dom, double sigma, uint64_t seed, int n,
                         double* flux) {
    const Mesh* m = (const Mesh*)mesh;
    Dom D{dom[0], dom[1], dom[2], dom[3], (int)dom[4]};
#pragma omp parallel for schedule(dynamic, 64)
    for (int p = 0; p < n; ++p) {
        Rng g(seed, 0x656c6563ULL, (uint64_t)p);
        double o[3], d[3];
        source(g, true, sigma, D, o, d);
        orc::HitD h = query(m, o, d, D);
        if (h.f >= 0) add(flux, h.f, 1.0);
    }
}

// _trace3d: flux, angacc double[F] (caller zeroes); no lateral wrap.
void orc_trace_legacy(void* mesh, const double* dom, int ion, double sigma, double sticking,
                      int n_reemit, int specular, double cos_thr, double eta, uint64_t seed, int n,
                      double* flux, double* angacc) {
    const Mesh* m = (const Mesh*)mesh;
    Dom D{dom[0], dom[1], dom[2], dom[3], 0};
#pragma omp parallel for schedule(dynamic, 64)
    for (int p = 0; p < n; ++p) {
        Rng g(seed, ion ? 0x6c696f6eULL : 0x6c6e6575ULL, (uint64_t)p);
        double o[3], d[3];
        source(g, ion != 0, sigma, D, o, d);
        double w = 1.0;
        for (int bounce = 0; bounce < n_reemit + 1; ++bounce) {
            orc::HitD h = orc::closest_hit(m, o, d, 1.0e6);
            if (h.f < 0) break;
            double nr[3];
            oriented_normal(m, h.f, d, nr);
            double cosang = std::max(-dot(d, nr), 0.0);
            double hit[3] = {o[0] + h.t * d[0], o[1] + h.t * d[1], o[2] + h.t * d[2]};
            if (specular == 1) {
                if (cosang >= cos_thr || bounce == n_reemit) {
                    add(flux, h.f, w);
                    add(angacc, h.f, w * cosang);
                    break;
                }
                double R = (cos_thr - cosang) / cos_thr, dep = w * (1 - R);
                add(flux, h.f, dep);
                add(angacc, h.f, dep * cosang);
                w = w * R * eta;
                double dn = dot(d, nr);
                for (int q = 0; q < 3; ++q) {
                    d[q] = d[q] - 2 * dn * nr[q];
                    o[q] = hit[q] + 1e-4 * nr[q];
                }
            } else {
                if (g.uniform() < sticking || bounce == n_reemit) {
                    add(flux, h.f, w);
                    add(angacc, h.f, w * cosang);
                    break;
                }
                cosine_emit(g, nr, d);
                for (int q = 0; q < 3; ++q) o[q] = hit[q] + 1e-4 * nr[q];
            }
        }
    }
}

// mc_flux_3d_radiosity's form-factor cast: ray k of face j leaves centroid_j + 1e-3 * fn_j in a
// cosine direction about fn_j (the _cosine_dirs tangent frame), wraps laterally like _apply_bc,
// and hit[j * n_ff + k] = its first hit face or -1.  fn, centroid: double[3 * F].
void orc_trace_ff(void* mesh, const double* dom, const double* fn, const double* centroid, int F,
                  int n_ff, uint64_t seed, int* hit) {
    const Mesh* m = (const Mesh*)mesh;
    Dom D{dom[0], dom[1], dom[2], dom[3], (int)dom[4]};
    const long long n = (long long)F * n_ff;
#pragma omp parallel for schedule(dynamic, 256)
    for (long long p = 0; p < n; ++p) {
        const int j = (int)(p / n_ff);
        Rng g(seed, 0x66666600ULL, (uint64_t)p);
        double o[3], d[3];
        for (int q = 0; q < 3; ++q) o[q] = centroid[3 * j + q] + 1e-3 * fn[3 * j + q];
        cosine_emit(g, fn + 3 * j, d);
        orc::HitD h = query(m, o, d, D);
        hit[p] = h.f;
    }
}

// mc_redep_3d's emission + trace: particle p leaves face j with probability cdf-weighted
// (cdf: inclusive prefix of w = max(V * area, 0), double[F]) from centroid_j + 1e-3 fn_j in a
// cosine direction about fn_j, then moves like _trace3d_cov_rr with bare = 1, beta = s_redep and
// no lateral wrap.  flux: double[F] deposited weight (caller zeroes).
void orc_trace_redep(void* mesh, const double* fn, const double* centroid, const double* cdf,
                     int F, double s_redep, uint64_t seed, int n, double* flux) {
    const Mesh* m = (const Mesh*)mesh;
    if (F <= 0 || !(cdf[F - 1] > 0.0)) return;
    Dom D{1.0, 1.0, 1.0, 0.0, 0};
#pragma omp parallel for schedule(dynamic, 64)
    for (int p = 0; p < n; ++p) {
        Rng g(seed, 0x72656470ULL, (uint64_t)p);
        const double target = g.uniform() * cdf[F - 1];
        int lo = 0, hi = F - 1;
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            if (cdf[mid] > target) hi = mid;
            else lo = mid + 1;
        }
        const int j = lo;
        double o[3], d[3];
        for (int q = 0; q < 3; ++q) o[q] = centroid[3 * j + q] + 1e-3 * fn[3 * j + q];
        cosine_emit(g, fn + 3 * j, d);
        double w = 1.0;
        for (int bounce = 0; bounce < 1024; ++bounce) {
            orc::HitD h = query(m, o, d, D);
            if (h.f < 0) break;
            double nr[3];
            oriented_normal(m, h.f, d, nr);
            add(flux, h.f, w);
            w = w - w * s_redep;
            if (w <= 1e-6) break;
            if (w < 0.1) {
                if (g.uniform() < (1.0 - w / 0.3)) break;
                w = 0.3;
            }
            double hit[3] = {o[0] + h.t * d[0], o[1] + h.t * d[1], o[2] + h.t * d[2]};
            cosine_emit(g, nr, d);
            for (int q = 0; q < 3; ++q) o[q] = hit[q] + 1e-4 * nr[q];
        }
    }
}

}  // extern "C"
