"""The FP64 oracle against golden vectors produced by the reference's own code (see
tests/golden/make_golden.py).  CPU only."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
import oracle.oracle as orc


@pytest.fixture(scope="module")
def lv():
    return np.load(os.path.join(GOLDEN, "levelset.npz"))


@pytest.mark.parametrize("name", ["hole", "trench"])
def test_seed_matches_reference_csg(lv, name):
    nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole = lv[f"{name}_seed_args"]
    phi, mask = orc.seed(int(nx), int(ny), int(nz), dx, Lx, Ly, sub_top, mask_th, width, bool(hole))
    np.testing.assert_array_equal(mask, lv[f"{name}_mask"])
    np.testing.assert_array_equal(phi.astype(np.float32), lv[f"{name}_csg"])


@pytest.mark.parametrize("name", ["hole", "trench"])
def test_reinit_matches_reference(lv, name):
    dx = float(lv[f"{name}_seed_args"][3])
    band = float(lv[f"{name}_reinit_band"][0])
    out = orc.reinit(lv[f"{name}_csg"], dx, band)
    np.testing.assert_allclose(out, lv[f"{name}_reinit"], rtol=0, atol=1e-12)


def test_reinit_zero_nodes_and_short_sweeps(lv):
    dx, band, n_iter = lv["noisy_args"]
    out = orc.reinit(lv["noisy_phi"], dx, band, int(n_iter))
    np.testing.assert_allclose(out, lv["noisy_reinit"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", ["hole", "trench"])
def test_advect_matches_reference(lv, name):
    dx, dt_sub, nsub = lv[f"{name}_adv_args"]
    phi1 = lv[f"{name}_reinit"].astype(np.float32)
    out = orc.advect(phi1, lv[f"{name}_F"], lv[f"{name}_mask"], lv[f"{name}_csg"], 1.0 / dx, dt_sub,
                     int(nsub))
    np.testing.assert_allclose(out, lv[f"{name}_advect"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", ["hole", "trench"])
def test_advect_numpy_twin_without_mask(lv, name):
    """advect_3d (numpy, no mask) == one masked substep with an all-false mask."""
    dx, dt_sub, _ = lv[f"{name}_adv_args"]
    phi1 = lv[f"{name}_reinit"].astype(np.float32)
    F = lv[f"{name}_F"]
    out = orc.advect(phi1, F, np.zeros(F.shape, bool), phi1, 1.0 / dx, dt_sub, 1)
    np.testing.assert_allclose(out, lv[f"{name}_advect_np"], rtol=0, atol=1e-12)
