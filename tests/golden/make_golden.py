"""Generates the golden fixtures in this folder by running the REFERENCE's own code (petch's
threed.py / belen.py / chemistry.py, unmodified) on small seeded inputs, with the third-party
warp-lang replaced by warp_shim.py (a CPU stand-in: see its docstring for what it restates).

Run in a checkout that has the reference at /root/reference (or $PETCH_REFERENCE):

    python tests/golden/make_golden.py [group ...]      # groups: levelset surface flux

The fixtures are committed; tests read only the .npz files, never the reference.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("PETCH_REFERENCE", "/root/reference")
sys.path.insert(0, HERE)
import warp_shim  # noqa: E402

t3 = warp_shim.install(os.path.join(REF, "src", "petch"))


def _csg(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole):
    """make_trench_3d's analytic field and mask (threed.py:34-55), before skfmm."""
    xs, ys, zs = np.arange(nx) * dx, np.arange(ny) * dx, np.arange(nz) * dx
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    mask_band = (Z >= sub_top) & (Z < sub_top + mask_th)
    if hole:
        opening = (X - Lx / 2) ** 2 + (Y - Ly / 2) ** 2 < (width / 2) ** 2
        r = np.sqrt((X - Lx / 2) ** 2 + (Y - Ly / 2) ** 2)
    else:
        opening = np.abs(X - Lx / 2) < width / 2
        r = np.abs(X - Lx / 2)
    d_sub = sub_top - Z
    d_slab = np.minimum(Z - sub_top, sub_top + mask_th - Z)
    d_mask = np.minimum(d_slab, r - width / 2.0)
    return np.maximum(d_sub, d_mask), mask_band & ~opening


def levelset():
    out = {}
    rng = np.random.default_rng(1234)
    cases = [
        # name, nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole
        ("hole", 14, 14, 20, 0.25, 3.5, 3.5, 3.0, 0.75, 1.5, True),
        ("trench", 16, 6, 18, 0.15, 2.4, 0.9, 1.8, 0.3, 0.9, False),
    ]
    for name, nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole in cases:
        phi_a, mask = _csg(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole)
        phi_a = phi_a.astype(np.float32)
        out[f"{name}_seed_args"] = np.array([nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width,
                                             float(hole)])
        out[f"{name}_csg"] = phi_a
        out[f"{name}_mask"] = mask
        band = 4 * dx + 2.0 * dx                         # run_etch_3d: reinit_fsm(phi, dx, band + 2dx)
        t0 = time.time()
        phi_r = t3.reinit_fsm(phi_a.astype(np.float64), dx, band)
        print(f"  reinit_fsm {name}: {time.time() - t0:.1f}s", flush=True)
        out[f"{name}_reinit_band"] = np.array([band])
        out[f"{name}_reinit"] = phi_r
        # advection on the redistanced field: F > 0 in the narrow band (as extend_velocity), a
        # sprinkle of exact zeros, mask cells re-pinned to the CSG field (mask_phi)
        phi1 = phi_r.astype(np.float32)
        F = np.where(np.abs(phi1) < 4 * dx, rng.uniform(0.0, 3.0, phi1.shape), 0.0)
        F[rng.random(phi1.shape) < 0.1] = 0.0
        F = F.astype(np.float32)
        dt, nsub = 0.02, 3
        t0 = time.time()
        adv = t3.advect_3d_gpu(phi1.astype(np.float64), F, mask, phi_a, dx, dt / nsub, nsub)
        print(f"  advect_3d_gpu {name}: {time.time() - t0:.1f}s", flush=True)
        out[f"{name}_F"] = F
        out[f"{name}_adv_args"] = np.array([dx, dt / nsub, nsub])
        out[f"{name}_advect"] = adv
        # the numpy twin (no mask) on the same input, one substep
        out[f"{name}_advect_np"] = t3.advect_3d(phi1.astype(np.float64), F.astype(np.float64),
                                                dx, dt / nsub)
    # a noisy field with exact zeros on nodes (sign(0) = +1, zero never an interface partner)
    nx, ny, nz, dx = 9, 8, 10, 0.2
    X, Y, Z = np.meshgrid(np.arange(nx) * dx, np.arange(ny) * dx, np.arange(nz) * dx, indexing="ij")
    phi = np.sqrt((X - 0.8) ** 2 + (Y - 0.7) ** 2 + (Z - 0.9) ** 2) - 0.55
    phi += rng.normal(0, 0.03, phi.shape)
    phi[rng.random(phi.shape) < 0.05] = 0.0
    phi = phi.astype(np.float32)
    out["noisy_phi"] = phi
    out["noisy_args"] = np.array([dx, 5 * dx, 3])
    out["noisy_reinit"] = t3.reinit_fsm(phi.astype(np.float64), dx, 5 * dx, n_iter=3)
    np.savez_compressed(os.path.join(HERE, "levelset.npz"), **out)


GROUPS = {"levelset": levelset}

if __name__ == "__main__":
    for g in (sys.argv[1:] or list(GROUPS)):
        print(g, flush=True)
        GROUPS[g]()
