// ORACLE -- test infrastructure only (never linked into the product).
//
// CPU restatement of the DDA gather of petch's deterministic discrete-ordinates neutral
// transport: _dda_gather_kernel, petch/dda.py:26-96.  One surface point at a time, every
// direction of the fixed quadrature marched cell by cell through the occupancy grid from the
// point stepped 1.01 dx off the surface: a ray reaching z >= z_top carries src_top, a ray whose
// trilinear phi turns positive carries the re-emission value of the first solid cell found by up
// to six half-cell steps forward (else of the nearest cell), a ray still marching after max_steps
// carries 0.  The arriving flux is the cosine-weighted mean sum(w acc contrib) / max(sum(w acc),
// 1e-12), acc = max(n . d, 0), over the directions with acc > 1e-6.
//
// Templated on the arithmetic type T: T = double evaluates the kernel the way the golden fixture
// ran it (float32 arrays read into float64, float64 scalars); T = float evaluates every operation
// in float32 in the kernel's order, the same IEEE operations as the device gather.  Built with
// -ffp-contract=off so no multiply-add is fused.
#include <algorithm>
#include <cmath>
#include <cstdint>

namespace {

template <typename T>
T trilinear(const float* phi, int ny, int nz, int i0, int j0, int k0, T fu, T fv, T fw) {
    auto at = [&](int i, int j, int k) {
        return (T)phi[((long long)i * ny + j) * nz + k];
    };
    const T one = (T)1.0;
    const T p00 = at(i0, j0, k0) * (one - fu) + at(i0 + 1, j0, k0) * fu;
    const T p10 = at(i0, j0 + 1, k0) * (one - fu) + at(i0 + 1, j0 + 1, k0) * fu;
    const T p01 = at(i0, j0, k0 + 1) * (one - fu) + at(i0 + 1, j0, k0 + 1) * fu;
    const T p11 = at(i0, j0 + 1, k0 + 1) * (one - fu) + at(i0 + 1, j0 + 1, k0 + 1) * fu;
    return (p00 * (one - fv) + p10 * fv) * (one - fw) + (p01 * (one - fv) + p11 * fv) * fw;
}

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

template <typename T>
T clampt(T v, T lo, T hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Rounded cell of a position: clamp(int(q / dx + 0.5), 0, n - 1), int() truncating.
template <typename T>
int rcell(T q, T dx, int n) { return clampi((int)(q / dx + (T)0.5), 0, n - 1); }

template <typename T>
void gather(const float* phi, int nx, int ny, int nz, const double* origins, const double* normals,
            const double* dirs, const double* weights, int D, const double* remit, double dx_in,
            double z_top_in, double src_in, int max_steps, int periodic_y, int N, double* out) {
    const T dx = (T)dx_in, z_top = (T)z_top_in, src_top = (T)src_in;
    const T umax = (T)nx - (T)1.001, vmax = (T)ny - (T)1.001, wmax = (T)nz - (T)1.001;
    const T Ly = (T)ny * dx;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < N; ++i) {
        const T o[3] = {(T)origins[3 * i], (T)origins[3 * i + 1], (T)origins[3 * i + 2]};
        const T n[3] = {(T)normals[3 * i], (T)normals[3 * i + 1], (T)normals[3 * i + 2]};
        T num = (T)0.0, den = (T)0.0;
        for (int k = 0; k < D; ++k) {
            const T d[3] = {(T)dirs[3 * k], (T)dirs[3 * k + 1], (T)dirs[3 * k + 2]};
            const T wk = (T)weights[k];
            const T dot = n[0] * d[0] + n[1] * d[1] + n[2] * d[2];
            const T acc = std::max(dot, (T)0.0);
            den += wk * acc;
            if (!(acc > (T)1.0e-6)) continue;
            T px = o[0] + d[0] * dx * (T)1.01;
            T py = o[1] + d[1] * dx * (T)1.01;
            T pz = o[2] + d[2] * dx * (T)1.01;
            T contrib = (T)0.0;
            bool done = false;
            for (int s = 0; s < max_steps && !done; ++s) {
                if (pz >= z_top) {
                    contrib = src_top;
                    done = true;
                } else {
                    const T u = clampt(px / dx, (T)0.0, umax);
                    const T v = clampt(py / dx, (T)0.0, vmax);
                    const T w = clampt(pz / dx, (T)0.0, wmax);
                    const int i0 = (int)u, j0 = (int)v, k0 = (int)w;
                    const T pv = trilinear<T>(phi, ny, nz, i0, j0, k0, u - (T)i0, v - (T)j0,
                                              w - (T)k0);
                    if (pv > (T)0.0) {
                        T qx = px, qy = py, qz = pz;
                        for (int e = 0; e < 6 && !done; ++e) {
                            const int ix = rcell(qx, dx, nx), iy = rcell(qy, dx, ny),
                                      iz = rcell(qz, dx, nz);
                            if (phi[((long long)ix * ny + iy) * nz + iz] > 0.0f) {
                                contrib = (T)remit[((long long)ix * ny + iy) * nz + iz];
                                done = true;
                            } else {
                                qx += d[0] * dx * (T)0.5;
                                qy += d[1] * dx * (T)0.5;
                                qz += d[2] * dx * (T)0.5;
                            }
                        }
                        if (!done) {
                            const int ix = rcell(px, dx, nx), iy = rcell(py, dx, ny),
                                      iz = rcell(pz, dx, nz);
                            contrib = (T)remit[((long long)ix * ny + iy) * nz + iz];
                            done = true;
                        }
                    }
                }
                px += d[0] * dx;
                py += d[1] * dx;
                pz += d[2] * dx;
                if (periodic_y == 1) {
                    if (py < (T)0.0) py += Ly;
                    if (py >= Ly) py -= Ly;
                }
            }
            num += wk * acc * contrib;
        }
        out[i] = (double)(num / std::max(den, (T)1.0e-12));
    }
}

}  // namespace

extern "C" void orc_dda_gather(const float* phi, int nx, int ny, int nz, const double* origins,
                               const double* normals, const double* dirs, const double* weights,
                               int D, const double* remit, double dx, double z_top, double src_top,
                               int max_steps, int periodic_y, int N, int f32, double* out) {
    if (f32)
        gather<float>(phi, nx, ny, nz, origins, normals, dirs, weights, D, remit, dx, z_top,
                      src_top, max_steps, periodic_y, N, out);
    else
        gather<double>(phi, nx, ny, nz, origins, normals, dirs, weights, D, remit, dx, z_top,
                       src_top, max_steps, periodic_y, N, out);
}
