"""The depth metrics (center_depth_3d / max_depth_3d, threed.py:1798-1869) on host arrays: the
column scan is vectorised, so it is checked against the oracle's per-column loop (depth3d) and a
plain loop for the 5th-percentile metric on random fields with buried pockets, all-gas columns
and columns whose top cell is solid.  CPU only."""
import numpy as np
import pytest

import oracle.oracle as orc
from petch_b200 import threed as t3


def _field(rng, nx, ny, nz, dx):
    z = np.arange(nz) * dx
    floor = rng.uniform(0.0, nz * dx, (nx, ny))
    phi = (floor[:, :, None] - z[None, None, :]).copy()          # gas above the floor
    pockets = rng.random((nx, ny, nz)) < 0.05                    # isolated gas below the floor
    phi[pockets] = -0.1
    phi[rng.random((nx, ny)) < 0.1, :] = -1.0                    # columns that are all gas
    phi[rng.random((nx, ny)) < 0.1, nz - 1] = 0.5                # columns with a solid top
    phi[rng.random((nx, ny, nz)) < 0.01] = 0.0                   # exact zeros count as solid
    return phi


def _loop_floors(phi, cols, zs):
    out = []
    for i, j in cols:
        col = phi[i, j, :] < 0
        k = len(col) - 1
        if not col[k]:
            continue
        while k > 0 and col[k - 1]:
            k -= 1
        out.append(zs[k])
    return out


@pytest.mark.parametrize("hole", [True, False])
@pytest.mark.parametrize("seed", range(4))
def test_vectorised_metrics_equal_the_column_loop(hole, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz, dx = 24, 20, 40, 0.25
    phi = _field(rng, nx, ny, nz, dx)
    g = dict(Lx=nx * dx, Ly=ny * dx, dx=dx, sub_top=8.0, trench_width=3.0, hole=hole,
             xs=np.arange(nx) * dx, ys=np.arange(ny) * dx, zs=np.arange(nz) * dx, phi=phi)
    for half in (1.0, 0.4, 3.0):
        assert t3.center_depth_3d(g, half) == orc.depth3d(g, phi, half)
    xs, ys, zs = g['xs'], g['ys'], g['zs']
    cx, cy, r = g['Lx'] / 2, g['Ly'] / 2, 1.5
    if hole:
        ii, jj = np.where((xs[:, None] - cx) ** 2 + (ys[None, :] - cy) ** 2 <= (r + dx) ** 2)
        cols = list(zip(ii, jj))
    else:
        cols = [(i, j) for i in np.where(np.abs(xs - cx) <= r + dx)[0] for j in range(ny)]
    fl = _loop_floors(phi, cols, zs)
    want = 0.0 if not fl else float(8.0 - np.percentile(fl, 5))
    assert t3.max_depth_3d(g) == want


def test_no_gas_column_gives_zero():
    nx, ny, nz, dx = 8, 8, 10, 0.5
    g = dict(Lx=4.0, Ly=4.0, dx=dx, sub_top=4.0, trench_width=2.0, hole=True,
             xs=np.arange(nx) * dx, ys=np.arange(ny) * dx, zs=np.arange(nz) * dx,
             phi=np.ones((nx, ny, nz)))
    assert t3.center_depth_3d(g) == 0.0 and t3.max_depth_3d(g) == 0.0
