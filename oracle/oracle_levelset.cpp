// ORACLE -- test infrastructure only (tests/, __graft_entry__.smoke() and bench.py's CPU baseline
// may call it; the product path never does).  FP64 CPU restatement of petch's level-set stages.
//
// Follows, line by line (paths within the reference project):
//   orc_seed    : make_trench_3d CSG field + mask              petch/threed.py:32-55
//   orc_advect  : _advect_iter + advect_3d_gpu ping-pong       petch/threed.py:1262-1307
//   orc_reinit  : _eik_solve/_eik_init/_eik_jacobi/reinit_fsm  petch/threed.py:1421-1537
// Parity pin: tests/golden/levelset.npz holds outputs of the reference's own kernel and host code
// (executed through tests/golden/warp_shim.py); tests/test_oracle_golden.py checks these functions
// against it.  skfmm.distance (make_trench_3d's last line) is not restated: parity unpinned there.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {

struct G {
    int nx, ny, nz;
    long long plane, n;
    G(int a, int b, int c) : nx(a), ny(b), nz(c), plane((long long)b * c), n((long long)a * b * c) {}
    long long at(int i, int j, int k) const { return (long long)i * plane + (long long)j * nz + k; }
};

double eik_solve(double a1, double a2, double a3, double dx) {
    double t;
    if (a1 > a2) { t = a1; a1 = a2; a2 = t; }
    if (a2 > a3) { t = a2; a2 = a3; a3 = t; }
    if (a1 > a2) { t = a1; a1 = a2; a2 = t; }
    double x = a1 + dx;
    if (x <= a2) return x;
    double d2 = 2.0 * dx * dx - (a1 - a2) * (a1 - a2);
    if (d2 < 0.0) d2 = 0.0;
    x = 0.5 * (a1 + a2 + std::sqrt(d2));
    if (x <= a3) return x;
    double s1 = a1 + a2 + a3;
    double s2 = a1 * a1 + a2 * a2 + a3 * a3;
    double d3 = s1 * s1 - 3.0 * (s2 - dx * dx);
    if (d3 < 0.0) d3 = 0.0;
    return (s1 + std::sqrt(d3)) / 3.0;
}

}  // namespace

extern "C" {

void orc_seed(double* phi, uint8_t* mask, int nx, int ny, int nz, double dx, double Lx, double Ly,
              double sub_top, double mask_th, double width, int hole) {
    G g(nx, ny, nz);
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                double X = i * dx, Y = j * dx, Z = k * dx;
                double ddx = X - Lx / 2.0, ddy = Y - Ly / 2.0;
                double r;
                bool opening;
                if (hole) {
                    opening = ddx * ddx + ddy * ddy < (width / 2.0) * (width / 2.0);
                    r = std::sqrt(ddx * ddx + ddy * ddy);
                } else {
                    opening = std::fabs(ddx) < width / 2.0;
                    r = std::fabs(ddx);
                }
                bool band = (Z >= sub_top) && (Z < sub_top + mask_th);
                double d_sub = sub_top - Z;
                double d_slab = std::min(Z - sub_top, sub_top + mask_th - Z);
                double d_mask = std::min(d_slab, r - width / 2.0);
                long long c = g.at(i, j, k);
                phi[c] = std::max(d_sub, d_mask);
                mask[c] = (band && !opening) ? 1 : 0;
            }
}

// nsub substeps; mask may be NULL (then F < 0 marks mask cells).
void orc_advect(double* phi, const double* F, const uint8_t* mask, const double* mask_phi, int nx,
                int ny, int nz, double inv_dx, double dt, int nsub) {
    G g(nx, ny, nz);
    std::vector<double> out((size_t)g.n);
    for (int s = 0; s < nsub; ++s) {
#pragma omp parallel for collapse(2)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) {
                    long long c = g.at(i, j, k);
                    bool pinned = mask ? (mask[c] != 0) : (F[c] < 0.0);
                    if (pinned) {
                        out[c] = mask_phi[c];
                        continue;
                    }
                    double v = phi[c], gg = 0.0, dm, dp;
                    dm = (i >= 1) ? (v - phi[c - g.plane]) * inv_dx : 0.0;
                    dp = (i <= nx - 2) ? (phi[c + g.plane] - v) * inv_dx : 0.0;
                    gg += std::max(dm, 0.0) * std::max(dm, 0.0) + std::min(dp, 0.0) * std::min(dp, 0.0);
                    dm = (j >= 1) ? (v - phi[c - nz]) * inv_dx : 0.0;
                    dp = (j <= ny - 2) ? (phi[c + nz] - v) * inv_dx : 0.0;
                    gg += std::max(dm, 0.0) * std::max(dm, 0.0) + std::min(dp, 0.0) * std::min(dp, 0.0);
                    dm = (k >= 1) ? (v - phi[c - 1]) * inv_dx : 0.0;
                    dp = (k <= nz - 2) ? (phi[c + 1] - v) * inv_dx : 0.0;
                    gg += std::max(dm, 0.0) * std::max(dm, 0.0) + std::min(dp, 0.0) * std::min(dp, 0.0);
                    out[c] = v - dt * F[c] * std::sqrt(gg);
                }
        std::memcpy(phi, out.data(), sizeof(double) * (size_t)g.n);
    }
}

// reinit_fsm(phi, dx, band, n_iter): big = band + 4dx, cap = band + dx.
// seed != 0: the skfmm.distance stand-in for the seed field (phi == 0 nodes frozen at 0 and kept
// at 0).
void orc_reinit_mode(const double* phi0, double* phi_out, int nx, int ny, int nz, double dx,
                     double band, int n_iter, int seed);

void orc_reinit(const double* phi0, double* phi_out, int nx, int ny, int nz, double dx,
                double band, int n_iter) {
    orc_reinit_mode(phi0, phi_out, nx, ny, nz, dx, band, n_iter, 0);
}

void orc_reinit_mode(const double* phi0, double* phi_out, int nx, int ny, int nz, double dx,
                     double band, int n_iter, int seed) {
    G g(nx, ny, nz);
    const double big = band + 4.0 * dx, cap = band + dx, inv_dx = 1.0 / dx;
    std::vector<double> U((size_t)g.n), B((size_t)g.n);
    std::vector<uint8_t> fz((size_t)g.n);
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                long long c = g.at(i, j, k);
                double v = phi0[c];
                double oxm = phi0[g.at(std::max(i - 1, 0), j, k)], oxp = phi0[g.at(std::min(i + 1, nx - 1), j, k)];
                double oym = phi0[g.at(i, std::max(j - 1, 0), k)], oyp = phi0[g.at(i, std::min(j + 1, ny - 1), k)];
                double ozm = phi0[g.at(i, j, std::max(k - 1, 0))], ozp = phi0[g.at(i, j, std::min(k + 1, nz - 1))];
                bool iface = v * oxm < 0 || v * oxp < 0 || v * oym < 0 || v * oyp < 0 || v * ozm < 0 || v * ozp < 0;
                if (seed && v == 0.0) {
                    U[c] = 0.0;
                    fz[c] = 1;
                } else if (iface) {
                    double gx = (oxp - oxm) * 0.5 * inv_dx, gy = (oyp - oym) * 0.5 * inv_dx,
                           gz = (ozp - ozm) * 0.5 * inv_dx;
                    double grad0 = std::max(std::sqrt(gx * gx + gy * gy + gz * gz), 0.5);
                    double dxl = 1.0 / inv_dx;
                    U[c] = std::min(std::fabs(v) / grad0, 1.8 * dxl);
                    fz[c] = 1;
                } else {
                    U[c] = big;
                    fz[c] = 0;
                }
            }
    for (int it = 0; it < n_iter; ++it) {
#pragma omp parallel for collapse(2)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) {
                    long long c = g.at(i, j, k);
                    if (fz[c]) {
                        B[c] = U[c];
                        continue;
                    }
                    double um = (i >= 1) ? U[c - g.plane] : big, up = (i <= nx - 2) ? U[c + g.plane] : big;
                    double ax = std::min(um, up);
                    um = (j >= 1) ? U[c - nz] : big;
                    up = (j <= ny - 2) ? U[c + nz] : big;
                    double ay = std::min(um, up);
                    um = (k >= 1) ? U[c - 1] : big;
                    up = (k <= nz - 2) ? U[c + 1] : big;
                    double az = std::min(um, up);
                    B[c] = std::min(U[c], eik_solve(ax, ay, az, dx));
                }
        std::swap(U, B);
    }
#pragma omp parallel for
    for (long long c = 0; c < g.n; ++c) {
        double s = phi0[c] < 0.0 ? -1.0 : (seed && phi0[c] == 0.0 ? 0.0 : 1.0);
        phi_out[c] = s * std::min(U[c], cap) + 0.0;
    }
}

}  // extern "C"
