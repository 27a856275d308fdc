"""The oracle's run_etch_3d options against tests/golden/options.npz, made by the reference's own
reinit_gpu (threed.py:1399-1418) and extend_velocity_3d (threed.py:1310-1321).  CPU only."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
import oracle.oracle as orc


@pytest.fixture(scope="module")
def op():
    return np.load(os.path.join(GOLDEN, "options.npz"))


@pytest.mark.parametrize("name", ["hole", "trench"])
def test_reinit_pde_matches_reference(op, name):
    """float32 restatement vs the reference kernel (run in float64 by the fixture shim)."""
    dx = float(op[f"{name}_pde_dx"][0])
    out = orc.reinit_pde(op[f"{name}_pde_in"], dx)
    np.testing.assert_allclose(out, op[f"{name}_pde_out"], rtol=2e-5, atol=2e-6 * dx)


def test_reinit_pde_pins_the_front(op):
    """Interface cells are driven to phi0/|grad phi0|: the sign pattern of the input survives."""
    phi = op["hole_pde_in"]
    out = orc.reinit_pde(phi, float(op["hole_pde_dx"][0]))
    assert np.mean(np.sign(out) == np.sign(phi)) > 0.999


def test_extend_nearest_centroid_matches_reference(op):
    dx, band = op["ext_args"]
    Fs = orc.extend_nearest_centroid(op["ext_V"], op["ext_centroids"], op["ext_phi"].astype(np.float64),
                                     dx, band)
    np.testing.assert_array_equal(Fs, op["ext_Fs"])


def test_gaussian_smooth_repins_mask():
    rng = np.random.default_rng(5)
    phi = rng.normal(size=(9, 7, 11))
    mask = rng.random(phi.shape) < 0.2
    mp = rng.normal(size=phi.shape)
    out = orc.gaussian_smooth(phi, 0.8, mask, mp)
    np.testing.assert_array_equal(out[mask], mp[mask])
    assert abs(out[~mask].std() - phi.std()) > 0.1            # actually smoothed
