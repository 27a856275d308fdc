"""The oracle's DDA neutral transport against tests/golden/dda.npz, produced by the reference's
own petch/dda.py (_dda_gather_kernel, fib_sphere, dda_neutral_flux) and mc_flux_3d_dda
(threed.py:1211-1244).  CPU only.

Pins: the direction set and the float64 gather exactly (a direct view, a pass over a random
re-emission field); dda_neutral_flux exactly at four direction / pass counts (1 and 2 passes
included: no extrapolation, extrapolation from the direct view); the coverage <-> DDA fixed point
from the reference's recorded ion results.  The float32 evaluation (the device's arithmetic) is
bounded against the same fixture."""
import os
import types

import numpy as np
import pytest

from conftest import GOLDEN
import oracle.oracle as orc
import petch_b200.params as P
from petch_b200 import dda as pdda

KEYS = ["hole", "trench"]
RUNS = [(16, 12), (8, 1), (8, 2), (8, 5)]


@pytest.fixture(scope="module")
def dd():
    return np.load(os.path.join(GOLDEN, "dda.npz"))


def case(dd, key):
    phi = dd[f"{key}_phi"]
    Lx, Ly, Lz, dx, periodic = dd[f"{key}_geo"]
    nz = phi.shape[2]
    zs = np.arange(nz) * dx
    z_top = zs[-1] - 0.5 * dx
    max_steps = (int((z_top - zs[0]) / dx) + 4) * (3 if periodic else 1)
    return (phi, float(dx), zs, int(periodic), dd[f"{key}_centroids"], dd[f"{key}_gas_normals"],
            dd[f"{key}_areas"], z_top, max_steps)


def test_direction_sets_match_reference(dd):
    d, w = orc.fib_sphere(128)
    np.testing.assert_array_equal(d, dd["hole_dirs"])
    assert np.all(w == 1.0)
    d2, w2 = pdda.fib_sphere(128)                       # the product's host copy
    np.testing.assert_array_equal(d2, dd["hole_dirs"])
    np.testing.assert_array_equal(w2, w)
    h, hw = pdda.fib_hemisphere(64)
    assert np.all(h[:, 2] > 0) and np.allclose(np.linalg.norm(h, axis=1), 1.0)
    np.testing.assert_array_equal(hw, h[:, 2])


@pytest.mark.parametrize("key", KEYS)
def test_march_bounds_follow_reference(dd, key):
    phi, dx, zs, per, *_, z_top, max_steps = case(dd, key)
    assert pdda.march_bounds(len(zs), dx, per) == (z_top, max_steps)


@pytest.mark.parametrize("key", KEYS)
def test_gather_float64_is_exact(dd, key):
    phi, dx, zs, per, c, fn, A, z_top, ms = case(dd, key)
    dirs, w = orc.fib_sphere(128)
    direct = orc.dda_gather(phi, dx, c, fn, dirs, w, np.zeros(phi.size), z_top, 1.0, ms, per)
    np.testing.assert_array_equal(direct, dd[f"{key}_direct"])
    rp = orc.dda_gather(phi, dx, c, fn, dirs, w, dd[f"{key}_remit"], z_top, 0.0, ms, per)
    np.testing.assert_array_equal(rp, dd[f"{key}_remit_pass"])
    # the cases reach every outcome: escapes, wall hits, open faces and buried ones
    assert direct.max() > 0.9 and direct.min() < 0.3 and rp.max() > 0.3


@pytest.mark.parametrize("key", KEYS)
@pytest.mark.parametrize("n_dir,n_re", RUNS)
def test_dda_neutral_flux_float64_is_exact(dd, key, n_dir, n_re):
    phi, dx, zs, per, c, fn, A, *_ = case(dd, key)
    v = orc.dda_neutral_flux(phi, dx, zs, c, fn, dd[f"{key}_s_face"], n_dir, n_re,
                             face_areas=np.maximum(A, 1e-9), periodic_y=per)
    np.testing.assert_array_equal(v, dd[f"{key}_flux_{n_dir}_{n_re}"])


@pytest.mark.parametrize("key", KEYS)
@pytest.mark.parametrize("n_dir,n_re", RUNS)
def test_dda_neutral_flux_float32_bounded(dd, key, n_dir, n_re):
    """float32 arithmetic against the float64 fixture: the march takes the same decisions for
    all but a handful of rays; the extrapolation from two iterates amplifies rounding (its ratio
    r / (1 - r) reaches 199), so that case gets a looser bound."""
    phi, dx, zs, per, c, fn, A, *_ = case(dd, key)
    v = orc.dda_neutral_flux(phi, dx, zs, c, fn, dd[f"{key}_s_face"], n_dir, n_re,
                             face_areas=np.maximum(A, 1e-9), periodic_y=per, f32=True)
    ref = dd[f"{key}_flux_{n_dir}_{n_re}"]
    err = np.abs(v - ref)
    if n_re == 2:
        assert np.mean(err > 1e-5) < 0.05 and err.max() < 1e-3
    else:
        assert err.max() < 2e-6


@pytest.mark.parametrize("key", KEYS)
def test_fixed_point_replays_reference_ions(dd, key):
    """mc_flux_3d_dda's coverage rounds from the reference's recorded ion results (dda_n_dir 8,
    12 passes, 4 rounds) -> its m_F, m_O."""
    phi, dx, zs, per, c, fn, A, *_ = case(dd, key)
    par = dict(P.PAR, periodic_y=per, dda_n_dir=8, dda_n_reemit=12)
    flags = types.SimpleNamespace(chemistry="belen", yield_angular="viennaps", ion_reflection=True)
    m_F, m_O = orc.dda_fixed_point(phi, dx, zs, c, fn, A, dd[f"{key}_m_i"], dd[f"{key}_cos_i"],
                                   tuple(dd[f"{key}_ion_yield"]), par, flags)
    np.testing.assert_allclose(m_F, dd[f"{key}_m_F"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(m_O, dd[f"{key}_m_O"], rtol=1e-10, atol=1e-12)


def test_wall_cells_are_solid_side(dd):
    """The re-emission cell of a face lies on the solid side: phi > 0 there for most faces."""
    for key in KEYS:
        phi, dx, zs, per, c, fn, *_ = case(dd, key)
        cells = orc.dda_wall_cells(c, fn, dx, phi.shape)
        assert np.mean(phi.ravel()[cells] > 0) > 0.9
