/*
 * petch-b200 C ABI: the per-step 3D etch loop of petch (level set -> marching-cubes surface ->
 * Monte-Carlo ion / neutral flux -> SF6/O2 coverage fixed point -> upwind advection -> Eikonal
 * reinit) as sm_100a CUDA kernels behind plain C entry points.
 *
 * Conventions for every entry point:
 *   - all array arguments are DEVICE pointers owned by the caller; the library never allocates,
 *     frees or keeps them (scratch buffers are passed in too);
 *   - grids are (nx, ny, nz) C-order, z fastest: cell (i, j, k) is at (i * ny + j) * nz + k, node
 *     coordinates x = i * dx, y = j * dx, z = k * dx (as petch's make_trench_3d);
 *   - `stream` is a cudaStream_t (NULL = legacy default stream); work is enqueued, not waited on;
 *   - the return value is a PETCH_* status; on failure petch_last_error() gives a message.
 *
 * Each declaration names the petch function it replaces as `petch/<file>:<line>` (paths within
 * the reference project's src/ tree).
 */
#ifndef PETCH_B200_H
#define PETCH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PETCH_OK = 0,
    PETCH_E_INVALID = 1,   /* bad argument (null pointer, non-positive size, ...) */
    PETCH_E_CUDA = 2,      /* a CUDA runtime call or kernel launch failed */
    PETCH_E_OVERFLOW = 3,  /* a caller-sized device buffer was too small (output truncated) */
    PETCH_E_NONFINITE = 4, /* non-finite values met where the reference raises */
    PETCH_E_LIMIT = 5      /* a bounded device loop hit its iteration limit */
};

/* ABI version (bumped on any signature change). */
int petch_abi_version(void);

/* Copies the last error message of the calling host thread into buf (NUL-terminated, <= n bytes).
 * Returns the message length. */
int petch_last_error(char* buf, int n);

/* ------------------------------------------------------------------------------------------ */
/* Level set                                                                                   */
/* ------------------------------------------------------------------------------------------ */

/* Replaces make_trench_3d (petch/threed.py:32-59): writes the analytic CSG field
 * max(sub_top - z, min(min(z - sub_top, sub_top + mask_th - z), r - width/2)) with
 * r = hypot(x - Lx/2, y - Ly/2) (hole) or |x - Lx/2| (trench), and the mask flag
 * (z in [sub_top, sub_top + mask_th) and outside the opening), evaluated in double.
 * The reference then calls skfmm.distance; callers redistance with petch_reinit_eik. */
int petch_seed_level_set(float* phi, uint8_t* mask, int nx, int ny, int nz, double dx,
                         double Lx, double Ly, double sub_top, double mask_th, double width,
                         int hole, void* stream);

/* Replaces advect_3d_gpu + _advect_iter (petch/threed.py:1262-1307): `nsub` first-order
 * Godunov upwind substeps phi <- phi - dt_sub * F * sqrt(g), with a zero one-sided difference at
 * the domain faces; cells with mask != 0 are re-pinned to mask_phi every substep.
 * phi (in/out) and tmp are ping-pong buffers of nx*ny*nz floats; the result lands in phi.
 * If mask is NULL, cells with F < 0 are treated as mask cells (the engine's folded encoding).
 * inv_dx and dt_sub are the float32 values the reference passes (1/dx and dt/nsub). */
int petch_advect(float* phi, float* tmp, const float* F, const uint8_t* mask,
                 const float* mask_phi, int nx, int ny, int nz, float inv_dx, float dt_sub,
                 int nsub, void* stream);

/* Replaces reinit_fsm + _eik_init + _eik_jacobi + _eik_solve (petch/threed.py:1421-1537):
 * Russo-Smereka frozen interface distance, n_iter Jacobi Godunov-Eikonal sweeps, then
 * phi_out = sign(phi_in) * min(U, cap) with sign(0) = +1.  big = band + 4 dx and
 * cap = band + dx as the reference computes them (float64, rounded to float32); dx is taken in
 * double so that 1/dx is rounded once, as the reference's host does; n_iter >= 1.
 * phi_in may alias phi_out.  u_a, u_b: scratch of nx*ny*nz floats each. */
int petch_reinit_eik(const float* phi_in, float* phi_out, float* u_a, float* u_b, int nx,
                     int ny, int nz, double dx, float big, float cap, int n_iter, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PETCH_B200_H */
