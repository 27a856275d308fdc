"""Knudsen conductance tail and floor-charging hooks on the device (petch_knudsen_*,
petch_charging_*, petch_zero_below) against tests/golden/knudsen.npz (the reference's own
knudsen.py, mc_flux_3d_knudsen and charging hooks) and the oracle."""
import ctypes
import os
import types

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_helpers import cuda_mesh, stream
from test_knudsen_oracle import KEYS, RUNS, case
import oracle.oracle as orc
import petch_b200 as petch
from petch_b200 import _lib
from petch_b200 import charging as pch
from petch_b200 import knudsen as pkn
from petch_b200 import threed as t3

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kd():
    return np.load(os.path.join(GOLDEN, "knudsen.npz"))


def shape_of(key):
    return "trench" if "trench" in key else "via"


@pytest.mark.parametrize("key", KEYS)
def test_slice_geometry_and_profile_drop_ins(kd, key):
    phi, geo, zs, per, trench, *_ = case(kd, key)
    a, p = pkn.slice_geometry(phi, zs, geo['dx'], geo['sub_top'], shape_of(key))
    np.testing.assert_allclose(a, kd[f"{key}_slice_area"], rtol=1e-14, atol=0)
    np.testing.assert_array_equal(p, kd[f"{key}_slice_perim"])
    for name, ls in (("scalar", 1.85), ("array", kd[f"{key}_ls"])):
        pr = pkn.conductance_profile(phi, zs, geo['dx'], geo['sub_top'], shape_of(key),
                                     kd[f"{key}_loss"], ls)
        np.testing.assert_allclose(pr, kd[f"{key}_profile_{name}"], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("key", KEYS)
def test_face_flux_drop_in(kd, key):
    """knudsen_face_flux on the fixture's host arrays (float64 centroids and normals); the
    sticking field travels as float32."""
    phi, geo, zs, per, trench, c, fn, A = case(kd, key)
    s = kd[f"{key}_s_face"]
    kw = dict(center=(0.5 * geo['Lx'], 0.5 * geo['Ly']), half_width=0.5 * geo['trench_width'])
    args = (phi, zs, geo['dx'], geo['sub_top'], shape_of(key), c, fn[:, 2], A, geo['Ly'], s)
    for name, extra in (("plain", dict(wall_loss_scale=2.9)),
                        ("foot", dict(wall_loss_scale=2.9, **kw)),
                        ("front", dict(wall_loss_scale=2.0, front_loss=True, band_W=1.0,
                                       pass_frac=0.3, ar_pass=0.7, **kw))):
        got = pkn.knudsen_face_flux(*args, **extra)
        np.testing.assert_allclose(got, kd[f"{key}_kff_{name}"], rtol=2e-6, atol=1e-7,
                                   err_msg=name)


def device_case(kd, key):
    phi, geo, zs, per, trench, c, fn, A = case(kd, key)
    m = cuda_mesh(phi.astype(np.float32), geo['dx'], dict(geo, mask_th=0.75))
    np.testing.assert_array_equal(m.faces[:m.F].cpu().numpy(), kd[f"{key}_faces"])
    par = dict(petch.PAR, periodic_y=per)
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", ion_reflection=True,
                     coverage_sticking=True, neutral_transport="knudsen")
    fe = t3.FluxEngine(geo, par, fl, m.MT)
    fe.mesh = m
    phid = torch.from_numpy(phi.astype(np.float32)).cuda()
    fnd = fe.gas_normals(phid)
    return m, fe, phi, phid, fnd, geo, zs, per


def load_ions(fe, m, mi, cos_i, iy):
    F = m.F
    fe.m_i[:F] = torch.from_numpy(np.asarray(mi, np.float32)).cuda()
    fe.cos_i[:F] = torch.from_numpy(np.asarray(cos_i, np.float32)).cuda()
    for q in range(3):
        fe.y[q, :F] = torch.from_numpy(np.asarray(iy[q], np.float32)).cuda()
    fe.yields = tuple(fe.y[q].data_ptr() for q in range(3))
    return fe.yields


@pytest.mark.parametrize("key", KEYS)
@pytest.mark.parametrize("run", RUNS, ids=[r[0] for r in RUNS])
def test_fixed_point_matches_oracle_and_reference(kd, key, run):
    """The engine's coverage rounds from the reference's recorded ions: against the oracle on the
    device's own float32 mesh data (float32 coverage vs float64: 1e-5), and against the
    reference's run on its float64 mesh data."""
    name, pkw, fkw = run
    m, fe, phi, phid, fnd, geo, zs, per = device_case(kd, key)
    F = m.F
    fe.par = dict(fe.par, **pkw)
    fe.flags = petch.Flags(chemistry="belen", yield_angular="viennaps", ion_reflection=True,
                           coverage_sticking=True, neutral_transport="knudsen", **fkw)
    mi, ci, iy = (kd[f"{key}_{name}_m_i"], kd[f"{key}_{name}_cos_i"],
                  kd[f"{key}_{name}_ion_yield"])
    yields = load_ions(fe, m, mi, ci, iy)
    fe.knudsen_prepare(phid, fnd)
    fe.knudsen_fixed_point(yields)
    c = m.centroid[:F].double().cpu().numpy()
    n = fnd[:F].double().cpu().numpy()
    A = m.area[:F].double().cpu().numpy()
    f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    flags = types.SimpleNamespace(chemistry="belen", yield_angular="viennaps", ion_reflection=True,
                                  **fkw)
    rF, rO = orc.knudsen_fixed_point(phi, geo, c, n, A, f32(mi), f32(ci),
                                     tuple(f32(a) for a in iy), fe.par, flags)
    for got, ref, refk in ((fe.m_F, rF, "m_F"), (fe.m_O, rO, "m_O")):
        g = got[:F].double().cpu().numpy()
        np.testing.assert_allclose(g, ref, rtol=1e-5, atol=1e-6, err_msg=refk)
        np.testing.assert_allclose(g, kd[f"{key}_{name}_{refk}"], rtol=1e-4, atol=1e-5,
                                   err_msg=refk)


@pytest.mark.parametrize("key", KEYS)
def test_charging_hooks_match_oracle_and_reference(kd, key):
    m, fe, phi, phid, fnd, geo, zs, per = device_case(kd, key)
    F = m.F
    mi, iy = kd[f"{key}_hook_m_i"], kd[f"{key}_hook_iy"]
    c = m.centroid[:F].double().cpu().numpy()
    n = fnd[:F].double().cpu().numpy()
    A = m.area[:F].double().cpu().numpy()
    for mode in ("hg", "petch"):
        load_ions(fe, m, mi, np.ones(F), iy)
        info = pch.apply_hg_charging(fe, fnd, mode)
        assert info is not None and info['n_floor'] > 0
        om, oy = orc.hg_charging(np.asarray(mi, np.float32).astype(np.float64),
                                 tuple(np.asarray(a, np.float32).astype(np.float64) for a in iy),
                                 dict(fe.par), mode, c, n[:, 2], A, geo)
        got_m = fe.m_i[:F].double().cpu().numpy()
        got_y = fe.y[:, :F].double().cpu().numpy()
        np.testing.assert_allclose(got_m, om, rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(got_y, np.stack(oy), rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(got_m, kd[f"{key}_{mode}_hook_m_i"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(got_y, kd[f"{key}_{mode}_hook_iy"], rtol=1e-5, atol=1e-5)
    load_ions(fe, m, mi, np.ones(F), iy)
    info = pch.apply_floor_throttle(fe, fnd)
    c32 = m.centroid[:F].cpu().numpy()
    om, oy = orc.floor_throttle(np.asarray(mi, np.float32).astype(np.float64),
                                tuple(np.asarray(a, np.float32).astype(np.float64) for a in iy),
                                c32, n[:, 2], geo)
    np.testing.assert_allclose(fe.m_i[:F].double().cpu().numpy(), om, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(fe.y[:, :F].double().cpu().numpy(), np.stack(oy), rtol=1e-6,
                               atol=1e-6)
    np.testing.assert_allclose(fe.m_i[:F].double().cpu().numpy(), kd[f"{key}_throttle_m_i"],
                               rtol=1e-5, atol=1e-6)
    assert 0.0 < info['Q'] <= 1.0


def test_tables_match_oracle():
    ar = np.linspace(-1.0, 30.0, 311)
    for a, b in zip(pch.charging_floor_profile(ar), (np.interp(ar, orc.HG_AR, t)
                                                     for t in (orc.HG_Q, orc.HG_VF, orc.HG_E))):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(pch.petch_floor_profile(ar), (np.interp(ar, orc.PT_AR, t)
                                                  for t in (orc.PT_Q, orc.PT_VF, orc.PT_E))):
        np.testing.assert_array_equal(a, b)
    q = pch.floor_charge_throttle_profile(ar)
    assert q[0] == 1.0 and q[-1] == 0.5 and np.all((q >= 0) & (q <= 1))


@pytest.mark.parametrize("key", ["hole_deep", "trench_deep"])
@pytest.mark.parametrize("run", RUNS, ids=[r[0] for r in RUNS])
def test_mc_flux_3d_knudsen_drop_in(kd, key, run):
    """The drop-in with the device's own ions: equal to the oracle's hooks + fixed point on the
    same ion results (before the hook: the hook is re-applied by the oracle)."""
    name, pkw, fkw = run
    phi, geo, zs, per, trench, c, fn, A = case(kd, key)
    m = cuda_mesh(phi.astype(np.float32), geo['dx'], dict(geo, mask_th=0.75))
    F = m.F
    par = dict(petch.PAR, periodic_y=per, **pkw)
    mode = {"hg": "hg", "petch": "petch"}.get(name, False)
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", ion_reflection=True,
                     coverage_sticking=True, neutral_transport="knudsen", surface_charging=mode,
                     **fkw)
    p = dict(par)
    m_i, m_F, m_O, cos_i = petch.mc_flux_3d_knudsen(m, None, None, None, None,
                                                    dict(geo, phi=phi), p, n_ion=20000, seed=3,
                                                    flags=fl)
    assert np.all(np.isfinite(m_F)) and 0.0 <= m_F.min() and m_F.max() <= 8.0
    assert m_F.min() < 0.9                              # the deep floor is starved
    phid = torch.from_numpy(phi.astype(np.float32)).cuda()
    fe = t3.FluxEngine(geo, par, fl, m.MT)
    fe.mesh = m
    n = fe.gas_normals(phid)[:F].double().cpu().numpy()
    cc = m.centroid[:F].double().cpu().numpy()
    AA = m.area[:F].double().cpu().numpy()
    flags = types.SimpleNamespace(chemistry="belen", yield_angular="viennaps", ion_reflection=True,
                                  knudsen_front_loss=fkw.get('knudsen_front_loss', False))
    rF, rO = orc.knudsen_fixed_point(phi, geo, cc, n, AA, m_i, cos_i, p['_ion_yield'], par, flags)
    np.testing.assert_allclose(m_F, rF, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(m_O, rO, rtol=1e-5, atol=1e-6)


def test_zero_below_and_bad_arguments(kd):
    phi, geo, zs, per, trench, *_ = case(kd, "hole_deep")
    m = cuda_mesh(phi.astype(np.float32), geo['dx'], dict(geo, mask_th=0.75))
    v = torch.ones(m.MT, device="cuda")
    _lib.call("petch_zero_below", m.id, m.MT, m.centroid.data_ptr(), 1.0, v.data_ptr(), stream())
    z = m.centroid[:m.F, 2]
    assert torch.equal(v[:m.F] == 0, z.double() <= 1.0) and bool((v[:m.F] == 0).any())
    assert torch.all(v[m.F:] == 1.0)
    nb = ctypes.c_longlong()
    _lib.call("petch_knudsen_scratch_bytes", m.MT, phi.shape[2], ctypes.byref(nb))
    small = torch.empty(int(nb.value) // 2, dtype=torch.uint8, device="cuda")
    phid = torch.from_numpy(phi.astype(np.float32)).cuda()
    with pytest.raises(_lib.PetchError, match="scratch too small"):
        _lib.call("petch_knudsen_prepare", phid.data_ptr(), *phi.shape, geo['dx'],
                  geo['sub_top'], 0, m.id, m.MT, m.centroid.data_ptr(), m.normal.data_ptr(),
                  0.0, 0.0, -1.0, small.data_ptr(), small.numel(), stream())
    with pytest.raises(_lib.PetchError, match="null pointer"):
        _lib.call("petch_charging_apply", m.id, m.MT, m.centroid.data_ptr(), None, 0.0, 0.0, 1.0,
                  1, 1.0, None, None, 0.0, None, None, None, None, stream())


@pytest.mark.parametrize("hole", [True, False])
def test_knudsen_loop_depth_matches_oracle_loop(hole):
    """run_etch_3d with neutral_transport='knudsen' (and the HG closure on the hole) on the device
    and in the oracle loop (independent ion streams): centre depth within one grid cell."""
    dx = 0.25
    cfg = dict(Lx=5.0, Ly=5.0 if hole else 2.5, Lz=8.0, dx=dx, trench_width=2.0, mask_th=1.0,
               sub_top=6.0, t_end=1.2, n_steps=12, hole=hole)
    par = dict(petch.PAR, rate_scale=0.3, periodic_y=0 if hole else 1)
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     ion_reflection=True, neutral_transport="knudsen",
                     surface_charging="hg" if hole else False)
    n = 60000
    geo = t3.run_etch_3d(**cfg, par=par, flags=fl, n_ion=n, n_neu=n, reinit_method="fsm",
                         verbose=False, record_depth_every=3)
    dev_hist = dict(geo['depth_history'])
    _, hist, _ = orc.run_etch_3d(cfg['Lx'], cfg['Ly'], cfg['Lz'], dx, cfg['trench_width'],
                                 cfg['mask_th'], cfg['sub_top'], cfg['t_end'], cfg['n_steps'],
                                 hole, par, fl, n, n, record_depth_every=3)
    orc_hist = dict(hist)
    assert set(dev_hist) == set(orc_hist)
    for s in sorted(orc_hist):
        assert abs(dev_hist[s] - orc_hist[s]) <= dx + 1e-9, (s, dev_hist[s], orc_hist[s])
    assert max(orc_hist.values()) > 2 * dx


def test_throttled_mc_loop_depth_matches_oracle_loop():
    """floor_charge_throttle on the Monte-Carlo coverage path: device loop against the oracle
    loop, and shallower than the same run without the throttle."""
    dx = 0.25
    cfg = dict(Lx=5.0, Ly=5.0, Lz=8.0, dx=dx, trench_width=2.0, mask_th=1.0, sub_top=6.0,
               t_end=1.2, n_steps=12, hole=True)
    par = dict(petch.PAR, rate_scale=0.3)
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     ion_reflection=True, floor_charge_throttle=True)
    n = 60000
    geo = t3.run_etch_3d(**cfg, par=par, flags=fl, n_ion=n, n_neu=n, reinit_method="fsm",
                         verbose=False, record_depth_every=3)
    dev_hist = dict(geo['depth_history'])
    _, hist, _ = orc.run_etch_3d(cfg['Lx'], cfg['Ly'], cfg['Lz'], dx, cfg['trench_width'],
                                 cfg['mask_th'], cfg['sub_top'], cfg['t_end'], cfg['n_steps'],
                                 True, par, fl, n, n, record_depth_every=3)
    orc_hist = dict(hist)
    for s in sorted(orc_hist):
        assert abs(dev_hist[s] - orc_hist[s]) <= dx + 1e-9, (s, dev_hist[s], orc_hist[s])
    fl0 = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                      ion_reflection=True)
    g0 = t3.run_etch_3d(**cfg, par=par, flags=fl0, n_ion=n, n_neu=n, reinit_method="fsm",
                        verbose=False)
    assert t3.center_depth_3d(geo) <= t3.center_depth_3d(g0) + 1e-9


def test_redeposition_foot_cleaning_runs():
    """surface_charging + etch_stop_z + redeposition: the foot band gets no redeposit (the run
    completes and stops at the etch stop)."""
    dx = 0.25
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     ion_reflection=True, neutral_transport="knudsen", surface_charging="hg",
                     redeposition=True)
    geo = t3.run_etch_3d(Lx=5.0, Ly=5.0, Lz=8.0, dx=dx, trench_width=2.0, mask_th=1.0,
                         sub_top=6.0, t_end=0.6, n_steps=6, hole=True,
                         par=dict(petch.PAR, rate_scale=0.3), flags=fl, n_ion=40000,
                         n_neu=40000, reinit_method="fsm", verbose=False, etch_stop_z=5.0)
    assert np.isfinite(geo['phi']).all()
    assert t3.max_depth_3d(geo) <= 6.0 - 5.0 + 2 * dx
