"""The oracle's Knudsen conductance tail and charging hooks against tests/golden/knudsen.npz,
produced by the reference's own petch/knudsen.py, mc_flux_3d_knudsen (threed.py:1149-1208),
_apply_hg_charging (threed.py:1046-1110) and _apply_floor_charge_throttle (threed.py:1112-1147).
CPU only.  Every comparison is exact: the reference is numpy float64 and so is the oracle."""
import os
import types

import numpy as np
import pytest

from conftest import GOLDEN
import oracle.oracle as orc
import petch_b200.params as P

KEYS = ["hole", "trench", "hole_deep", "trench_deep"]
RUNS = (("local", {}, {}), ("field", dict(knudsen_sink='field'), {}),
        ("front", dict(knudsen_front_band_W=1.0, knudsen_passive_frac=0.3,
                       knudsen_front_ar_pass=0.7), dict(knudsen_front_loss=True)),
        ("hg", {}, {}), ("petch", {}, {}))


@pytest.fixture(scope="module")
def kd():
    return np.load(os.path.join(GOLDEN, "knudsen.npz"))


def case(kd, key):
    phi = kd[f"{key}_phi"].astype(np.float64)
    Lx, Ly, Lz, dx, per, sub_top, W = kd[f"{key}_geo"]
    geo = dict(Lx=float(Lx), Ly=float(Ly), Lz=float(Lz), dx=float(dx), sub_top=float(sub_top),
               trench_width=float(W), hole="hole" in key)
    zs = np.arange(phi.shape[2]) * dx
    return (phi, geo, zs, int(per), "trench" in key, kd[f"{key}_centroids"],
            kd[f"{key}_gas_normals"], np.maximum(kd[f"{key}_areas"], 1e-9))


@pytest.mark.parametrize("key", KEYS)
def test_slice_geometry_and_profiles(kd, key):
    phi, geo, zs, per, trench, *_ = case(kd, key)
    a, p = orc.kn_slice_geometry(phi, zs, geo['dx'], geo['sub_top'], trench)
    np.testing.assert_array_equal(a, kd[f"{key}_slice_area"])
    np.testing.assert_array_equal(p, kd[f"{key}_slice_perim"])
    for name, ls in (("scalar", 1.85), ("array", kd[f"{key}_ls"])):
        pr = orc.kn_profile(phi, zs, geo['dx'], geo['sub_top'], trench, kd[f"{key}_loss"], ls)
        np.testing.assert_array_equal(pr, kd[f"{key}_profile_{name}"])
    assert kd[f"{key}_profile_scalar"].min() < (0.1 if "deep" in key else 0.9)


@pytest.mark.parametrize("key", KEYS)
def test_face_flux(kd, key):
    phi, geo, zs, per, trench, c, fn, A = case(kd, key)
    s = kd[f"{key}_s_face"]
    kw = dict(center=(0.5 * geo['Lx'], 0.5 * geo['Ly']), half_width=0.5 * geo['trench_width'])
    args = (phi, zs, geo['dx'], geo['sub_top'], trench, c, fn[:, 2], A, geo['Ly'], s)
    np.testing.assert_array_equal(orc.kn_face_flux(*args, 2.9), kd[f"{key}_kff_plain"])
    np.testing.assert_array_equal(orc.kn_face_flux(*args, 2.9, **kw), kd[f"{key}_kff_foot"])
    np.testing.assert_array_equal(
        orc.kn_face_flux(*args, 2.0, front_loss=True, band_W=1.0, pass_frac=0.3, ar_pass=0.7,
                         **kw), kd[f"{key}_kff_front"])


@pytest.mark.parametrize("key", KEYS)
@pytest.mark.parametrize("run", RUNS, ids=[r[0] for r in RUNS])
def test_fixed_point_replays_reference_ions(kd, key, run):
    name, pkw, fkw = run
    phi, geo, zs, per, trench, c, fn, A = case(kd, key)
    par = dict(P.PAR, periodic_y=per, **pkw)
    fl = types.SimpleNamespace(chemistry="belen", yield_angular="viennaps", ion_reflection=True,
                               **fkw)
    m_F, m_O = orc.knudsen_fixed_point(phi, geo, c, fn, A, kd[f"{key}_{name}_m_i"],
                                       kd[f"{key}_{name}_cos_i"],
                                       tuple(kd[f"{key}_{name}_ion_yield"]), par, fl)
    np.testing.assert_array_equal(m_F, kd[f"{key}_{name}_m_F"])
    np.testing.assert_array_equal(m_O, kd[f"{key}_{name}_m_O"])


@pytest.mark.parametrize("key", KEYS)
def test_charging_hooks(kd, key):
    phi, geo, zs, per, trench, c, fn, A = case(kd, key)
    m_i, iy = kd[f"{key}_hook_m_i"], tuple(kd[f"{key}_hook_iy"])
    for mode in ("hg", "petch"):
        m2, iy2 = orc.hg_charging(m_i, iy, dict(P.PAR), mode, c, fn[:, 2], A, geo)
        np.testing.assert_array_equal(m2, kd[f"{key}_{mode}_hook_m_i"])
        np.testing.assert_array_equal(np.stack(iy2), kd[f"{key}_{mode}_hook_iy"])
        assert np.any(m2 != m_i)
    c32 = kd[f"{key}_verts"][kd[f"{key}_faces"]].mean(axis=1)
    m2, iy2 = orc.floor_throttle(m_i, iy, c32, fn[:, 2], geo)
    np.testing.assert_array_equal(m2, kd[f"{key}_throttle_m_i"])
    np.testing.assert_array_equal(np.stack(iy2), kd[f"{key}_throttle_iy"])


def test_hooks_leave_non_floor_faces_alone(kd):
    """Only floor faces (and, for the HG closure, the sidewall foot) change; a mode other than
    hg / petch, or no yields, is a no-op."""
    phi, geo, zs, per, trench, c, fn, A = case(kd, "hole_deep")
    m_i, iy = kd["hole_deep_hook_m_i"], tuple(kd["hole_deep_hook_iy"])
    _, floor = orc._footprint_floor(c, fn[:, 2], geo)
    m2, _ = orc.hg_charging(m_i, iy, dict(P.PAR), "hg", c, fn[:, 2], A, geo)
    np.testing.assert_array_equal(m2[~floor], m_i[~floor])
    assert np.all(m2[floor] < m_i[floor])
    m3, iy3 = orc.hg_charging(m_i, iy, dict(P.PAR), "other", c, fn[:, 2], A, geo)
    assert m3 is m_i and iy3 is iy
    m4, iy4 = orc.hg_charging(m_i, None, dict(P.PAR), "hg", c, fn[:, 2], A, geo)
    assert m4 is m_i and iy4 is None
