"""DDA neutral transport on the device (petch_dda_prepare, petch_dda_solve) against the oracle and
tests/golden/dda.npz (the reference's own dda_neutral_flux and mc_flux_3d_dda).

The device marches each ray once and replays its end in every pass; the oracle re-marches every
pass as the reference does.  On the same float32 inputs the two agree bit for bit (float32 march
and gather sums, float64 re-emission, dilation and extrapolation, the same summation orders)."""
import ctypes
import os
import types

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_helpers import cuda_mesh, small_feature, stream
from test_dda_oracle import KEYS, RUNS, case
import oracle.oracle as orc
import petch_b200 as petch
from petch_b200 import _lib
from petch_b200 import dda as pdda
from petch_b200 import threed as t3

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dd():
    return np.load(os.path.join(GOLDEN, "dda.npz"))


def device_case(dd, key):
    phi, dx, zs, per, *_ = case(dd, key)
    phi2, g = small_feature(key == "hole", nx=10, ny=10, nz=14, dx=0.3)
    np.testing.assert_array_equal(phi2, phi)
    m = cuda_mesh(phi, dx, g)
    np.testing.assert_array_equal(m.faces[:m.F].cpu().numpy(), dd[f"{key}_faces"])
    Lx, Ly, Lz = dd[f"{key}_geo"][:3]
    g = dict(g, Lx=Lx, Ly=Ly, Lz=Lz)
    phid = torch.from_numpy(phi).cuda()
    fn = torch.empty((m.MT, 3), device="cuda")
    nx, ny, nz = phi.shape
    _lib.call("petch_gas_normals", m.id, m.MT, m.MV, phid.data_ptr(), nx, ny, nz, dx,
              fn.data_ptr(), stream())
    return m, g, phi, phid, fn, dx, zs, per


def run_device(m, phid, fn, dx, per, n_dir, n_re, bare, betaE, betaO):
    solver = pdda.DDASolver(m.MT, tuple(phid.shape), n_dir)
    solver.prepare(phid, dx, m.id, m.centroid, fn, m.area, per)
    b = torch.ones(m.MT, device="cuda")
    b[:m.F] = torch.from_numpy(bare).cuda()
    oE = torch.full((m.MT,), -1.0, device="cuda")
    oO = torch.full((m.MT,), -1.0, device="cuda")
    solver.solve(b, betaE, betaO, n_re, oE, oO)
    return solver, oE, oO


@pytest.mark.parametrize("key", KEYS)
@pytest.mark.parametrize("n_dir,n_re", [(64, 12), (8, 1), (8, 2), (8, 5), (16, 30)])
def test_device_matches_oracle_float32_exactly(dd, key, n_dir, n_re):
    m, g, phi, phid, fn, dx, zs, per = device_case(dd, key)
    F = m.F
    rng = np.random.default_rng(n_dir * 100 + n_re)
    bare = rng.uniform(0.0, 1.0, F).astype(np.float32)
    bare[:10] = [0.0, 1.0, 0.5, 1.0, 1.0, 0.0, 0.25, 1.0, 0.9, 0.1]
    _, oE, oO = run_device(m, phid, fn, dx, per, n_dir, n_re, bare, 0.7, 1.0)
    c = m.centroid[:F].double().cpu().numpy()
    n = fn[:F].double().cpu().numpy()
    A = m.area[:F].double().cpu().numpy()
    b64 = bare.astype(np.float64)
    for beta, out in ((0.7, oE), (1.0, oO)):
        ref = orc.dda_neutral_flux(phi, dx, zs, c, n, np.clip(b64 * beta, 0.0, 1.0), n_dir, n_re,
                                   face_areas=A, periodic_y=per, f32=True)
        got = out[:F].cpu().numpy()
        bad = np.flatnonzero(got != ref.astype(np.float32))
        assert bad.size == 0, (beta, bad[:10], got[bad[:5]], ref[bad[:5]])
    assert torch.all(oE[F:] == -1.0)                     # nothing written past the live faces


@pytest.mark.parametrize("key", KEYS)
@pytest.mark.parametrize("n_dir,n_re", RUNS)
def test_drop_in_matches_reference(dd, key, n_dir, n_re):
    """petch_b200.dda_neutral_flux on the fixture's own host arrays (float64 centroids, normals,
    sticking) against the reference's float64 run."""
    phi, dx, zs, per, c, fn, A, *_ = case(dd, key)
    v = petch.dda_neutral_flux(phi, dx, zs, c, fn, dd[f"{key}_s_face"], n_dir, n_re,
                               face_areas=np.maximum(A, 1e-9), periodic_y=per)
    ref = dd[f"{key}_flux_{n_dir}_{n_re}"]
    err = np.abs(v - ref)
    if n_re == 2:
        assert np.mean(err > 1e-5) < 0.05 and err.max() < 1e-3
    else:
        assert err.max() < 5e-6, err.max()


@pytest.mark.parametrize("key", KEYS)
def test_fixed_point_replays_reference_ions(dd, key):
    """The engine's coverage rounds on the device mesh from the reference's recorded ion results
    -> its mc_flux_3d_dda m_F, m_O (float32 march and coverage against the float64 run)."""
    m, g, phi, phid, fn, dx, zs, per = device_case(dd, key)
    F = m.F
    par = dict(petch.PAR, periodic_y=per, dda_n_dir=8, dda_n_reemit=12)
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", ion_reflection=True,
                     neutral_transport="dda")
    fe = t3.FluxEngine(g, par, fl, m.MT)
    fe.mesh = m
    fe.m_i[:F] = torch.from_numpy(dd[f"{key}_m_i"].astype(np.float32)).cuda()
    fe.cos_i[:F] = torch.from_numpy(dd[f"{key}_cos_i"].astype(np.float32)).cuda()
    iy = dd[f"{key}_ion_yield"]
    for q in range(3):
        fe.y[q, :F] = torch.from_numpy(iy[q].astype(np.float32)).cuda()
    yields = tuple(fe.y[q].data_ptr() for q in range(3))
    fe.dda_prepare(phid)
    fe.dda_fixed_point(yields)
    for name, t in (("m_F", fe.m_F), ("m_O", fe.m_O)):
        got = t[:F].double().cpu().numpy()
        ref = dd[f"{key}_{name}"]
        err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-3)
        assert np.mean(err > 1e-4) < 0.02 and err.max() < 1e-2, (name, err.max(), np.mean(err > 1e-4))


def test_solve_is_bitwise_reproducible_and_passes_clamp(dd):
    m, g, phi, phid, fn, dx, zs, per = device_case(dd, "trench")
    bare = np.full(m.F, 0.4, np.float32)
    solver, oE, oO = run_device(m, phid, fn, dx, per, 16, 12, bare, 0.7, 1.0)
    b = torch.ones(m.MT, device="cuda")
    b[:m.F] = 0.4
    outs = []
    for n_re in (12, 12, 0, 1):
        e = torch.empty(m.MT, device="cuda")
        o = torch.empty(m.MT, device="cuda")
        solver.solve(b, 0.7, 1.0, n_re, e, o)
        outs.append((e[:m.F].clone(), o[:m.F].clone()))
    assert torch.equal(outs[0][0], oE[:m.F]) and torch.equal(outs[0][1], oO[:m.F])
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    assert torch.equal(outs[2][0], outs[3][0])          # n_reemit < 1 runs one pass
    for e, o in outs:
        assert float(e.min()) >= 0.0 and float(e.max()) <= 8.0


def test_sticking_one_gives_the_direct_view(dd):
    """s = 1 everywhere: no re-emission, so every pass returns the direct view."""
    m, g, phi, phid, fn, dx, zs, per = device_case(dd, "hole")
    F = m.F
    _, oE, _ = run_device(m, phid, fn, dx, per, 64, 12, np.ones(F, np.float32), 1.0, 1.0)
    c = m.centroid[:F].double().cpu().numpy()
    n = fn[:F].double().cpu().numpy()
    dirs, w = orc.fib_sphere(128)
    zt, ms = pdda.march_bounds(phi.shape[2], dx, per)
    direct = orc.dda_gather(phi, dx, c, n, dirs, w, np.zeros(phi.size), zt, 1.0, ms, per, True)
    np.testing.assert_array_equal(oE[:F].cpu().numpy(), direct.astype(np.float32))


def test_bad_arguments_fail_without_launching(dd):
    m, g, phi, phid, fn, dx, zs, per = device_case(dd, "hole")
    nb = ctypes.c_longlong()
    _lib.call("petch_dda_scratch_bytes", m.MT, *phi.shape, 16, ctypes.byref(nb))
    small = torch.empty(int(nb.value) // 2, dtype=torch.uint8, device="cuda")
    dirs = torch.zeros((16, 3), device="cuda")
    w = torch.ones(16, device="cuda")
    with pytest.raises(_lib.PetchError, match="scratch too small"):
        _lib.call("petch_dda_prepare", phid.data_ptr(), *phi.shape, dx, 3.0, 20, 0, m.id, m.MT,
                  m.centroid.data_ptr(), fn.data_ptr(), m.area.data_ptr(), dirs.data_ptr(),
                  w.data_ptr(), 16, small.data_ptr(), small.numel(), stream())
    with pytest.raises(_lib.PetchError, match="null pointer"):
        _lib.call("petch_dda_prepare", None, *phi.shape, dx, 3.0, 20, 0, m.id, m.MT,
                  m.centroid.data_ptr(), fn.data_ptr(), m.area.data_ptr(), dirs.data_ptr(),
                  w.data_ptr(), 16, small.data_ptr(), small.numel(), stream())
    with pytest.raises(_lib.PetchError):
        _lib.call("petch_dda_scratch_bytes", 0, *phi.shape, 16, ctypes.byref(nb))


@pytest.mark.parametrize("key", KEYS)
def test_mc_flux_3d_dda_drop_in(dd, key):
    """The drop-in on a device mesh: ions from the device tracer, DDA neutrals; equal to the
    oracle's coverage <-> DDA fixed point on the same ion results."""
    m, g, phi, phid, fn, dx, zs, per = device_case(dd, key)
    F = m.F
    par = dict(petch.PAR, periodic_y=per, dda_n_dir=16, dda_n_reemit=12)
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", ion_reflection=True,
                     coverage_sticking=True, neutral_transport="dda")
    p = dict(par)
    m_i, m_F, m_O, cos_i = petch.mc_flux_3d_dda(m, None, None, None, None, dict(g, phi=phi), p,
                                                n_ion=20000, seed=5, flags=fl)
    assert '_ion_yield' in p and len(p['_ion_yield'][0]) == F
    assert np.all(np.isfinite(m_F)) and m_F.min() >= 0 and m_F.max() <= 8.0
    flags = types.SimpleNamespace(chemistry="belen", yield_angular="viennaps", ion_reflection=True)
    c = m.centroid[:F].double().cpu().numpy()
    n = fn[:F].double().cpu().numpy()
    A = m.area[:F].double().cpu().numpy()
    rF, rO = orc.dda_fixed_point(phi, dx, zs, c, n, A, m_i, cos_i, p['_ion_yield'], par, flags,
                                 f32=True)
    for got, ref in ((m_F, rF), (m_O, rO)):
        err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-3)
        assert np.mean(err > 1e-4) < 0.02 and err.max() < 1e-2


@pytest.mark.parametrize("hole", [True, False])
def test_dda_loop_depth_matches_oracle_loop(hole):
    """run_etch_3d with neutral_transport='dda' on the device and in the oracle loop (independent
    ion streams): centre depth within one grid cell at every recorded step."""
    dx = 0.25
    cfg = dict(Lx=5.0, Ly=5.0 if hole else 2.5, Lz=8.0, dx=dx, trench_width=2.0, mask_th=1.0,
               sub_top=6.0, t_end=1.2, n_steps=12, hole=hole)
    par = dict(petch.PAR, rate_scale=0.3, periodic_y=0 if hole else 1, dda_n_dir=16)
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     ion_reflection=True, neutral_transport="dda")
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
