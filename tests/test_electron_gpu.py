"""The electron-shadowing charge model of mc_flux_3d_coupled (threed.py:847-868) on the device:
the electron trace (petch_trace_electrons) against the reference kernel's per-face means
(tests/golden/electron.npz) with a chi-square test; the charging factor (petch_electron_shadow)
bit for bit against the oracle; its wiring into the coverage-coupled flux (deterministic tallies:
the charged ion result equals the oracle's factor applied to the uncharged one); and the whole
loop against the oracle's loop."""
import ctypes
import os

import numpy as np
import pytest
import torch

import oracle.oracle as orc
import petch_b200 as petch
from conftest import GOLDEN
from gpu_helpers import cuda_mesh, domain, small_feature, stream
from petch_b200 import _lib
from petch_b200 import charging as pch
from petch_b200 import threed as t3

pytestmark = pytest.mark.gpu

FLAGS = dict(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
             ion_reflection=True)


@pytest.fixture(scope="module")
def ed():
    return np.load(os.path.join(GOLDEN, "electron.npz"))


def _mesh(key, ed):
    phi, geo = small_feature(key == "hole", nx=10, ny=10, nz=14, dx=0.3)
    m = cuda_mesh(phi, geo['dx'], geo)
    np.testing.assert_array_equal(m.faces[:m.F].cpu().numpy(), ed[f"{key}_faces"])
    return m, geo, phi


def cuda_electrons(m, geo, sigma, seed, n):
    flux = torch.zeros(m.MT, device="cuda")
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    _lib.call("petch_trace_electrons", m.id, m.MT, m.MV, ctypes.byref(domain(geo)), float(sigma),
              int(seed), int(n), flux.data_ptr(), work.data_ptr(), stream())
    assert work[1].item() == 0
    return flux[:m.F].double().cpu().numpy()


def _z2(x, g, sg):
    """z = (x - g) / sg is Student-t with 7 degrees of freedom without a systematic difference:
    E[z^2] = 1.4, median(z^2) = 0.49."""
    k = sg > 0
    z2 = (x[k] - g[k]) ** 2 / sg[k] ** 2
    return float(np.median(z2)), float(z2.mean())


@pytest.mark.parametrize("key", ["hole", "trench"])
def test_electron_trace_vs_reference_kernel(ed, key):
    m, geo, _ = _mesh(key, ed)
    n = 8_000_000
    x = cuda_electrons(m, geo, 0.5, 1, n) / n
    g, sg = ed[f"{key}_electron_mean"], ed[f"{key}_electron_se"]
    med, mean = _z2(x, g, sg)
    assert med < 0.75 and mean < 2.2, (med, mean)
    assert x.sum() == pytest.approx(g.sum(), rel=0.02)
    assert x.sum() <= 1.0 + 1e-6                   # one unit at most per electron


def test_electron_trace_vs_oracle_and_zero_rays():
    """Against the oracle's tracer at 4M rays each (per-face relative L2 within 2 %), and
    n = 0 zeroes the tally."""
    phi, geo = small_feature(False)
    m = cuda_mesh(phi, geo['dx'], geo)
    verts, faces, _, _ = m.host_arrays()
    om = orc.mesh_from_arrays(verts, faces)
    n = 4_000_000
    x = cuda_electrons(m, geo, 0.5, 3, n) / n
    y = orc.trace_electrons(om, geo, dict(periodic_y=1), 0.5, 3, n) / n
    assert np.linalg.norm(x - y) / np.linalg.norm(y) < 0.02
    assert cuda_electrons(m, geo, 0.5, 3, 0).max() == 0.0


def test_electron_shadow_kernel_is_exact():
    """petch_electron_shadow == the oracle's factor on the same float32 inputs, rounded once to
    float32; faces past the live count stay as they are."""
    phi, geo = small_feature(True)
    m = cuda_mesh(phi, geo['dx'], geo)
    F, MT = m.F, m.MT
    rng = np.random.default_rng(8)
    mi = rng.uniform(0.0, 1.4, MT).astype(np.float32)
    me = rng.uniform(0.0, 3.0, MT).astype(np.float32)
    mi[:F:7] = 0.0
    me[:F:5] = 0.0
    mi[1:F:11] = 5e-7
    for alpha in (0.0, 0.35, 1.0):
        ref_i = pch.open_field_level(mi[:F])
        ref_e = pch.open_field_level(me[:F])
        want, oi, oe = orc.electron_shadow(mi[:F].astype(np.float64), me[:F].astype(np.float64),
                                           alpha)
        assert (oi, oe) == (ref_i, ref_e)
        d_i = torch.from_numpy(mi.copy()).cuda()
        d_e = torch.from_numpy(me).cuda()
        _lib.call("petch_electron_shadow", m.id, MT, d_e.data_ptr(), ref_i, ref_e, alpha,
                  d_i.data_ptr(), stream())
        got = d_i.cpu().numpy()
        np.testing.assert_array_equal(got[:F], want.astype(np.float32))
        np.testing.assert_array_equal(got[F:], mi[F:])
        if alpha > 0:
            assert np.any(got[:F] < 0.9 * mi[:F])
    with pytest.raises(_lib.PetchError, match="null pointer"):
        _lib.call("petch_electron_shadow", m.id, MT, None, 1.0, 1.0, 0.5, d_i.data_ptr(), stream())


@pytest.mark.parametrize("faithful", [True, False])
def test_coupled_flux_applies_the_charging_factor(faithful):
    """With deterministic tallies the ion trace of the charged and the uncharged run is the same;
    the charged m_i is the oracle's factor (levels from the device's own m_i and m_e) applied to
    the uncharged one, bit for bit; the yields are left alone."""
    phi, geo = small_feature(False, nx=12, ny=8, nz=20, dx=0.25)
    m = cuda_mesh(phi, geo['dx'], geo)
    F = m.F
    par = dict(petch.PAR, periodic_y=1, charge_alpha=0.6, eFlux=1.3)
    _lib.set_deterministic(64 << 20)
    try:
        out = {}
        for charged in (False, True):
            fl = petch.Flags(**dict(FLAGS, ion_reflection=faithful, surface_charging=charged))
            fe = t3._flux_engine(m, geo, dict(par), fl)
            fe.flux_coupled(20000, 20000, 7, False)
            out[charged] = (fe.m_i[:F].cpu().numpy().copy(), fe.y[:, :F].cpu().numpy().copy(),
                            None if not charged else fe.m_e[:F].cpu().numpy().copy(),
                            getattr(fe, "electron", None))
    finally:
        _lib.set_deterministic(0)
    mi0, y0, _, _ = out[False]
    mi1, y1, me, info = out[True]
    want, ri, re_ = orc.electron_shadow(mi0.astype(np.float64), me.astype(np.float64), 0.6)
    assert info['ref_i'] == ri and info['ref_e'] == re_
    np.testing.assert_array_equal(mi1, want.astype(np.float32))
    if faithful:
        np.testing.assert_array_equal(y1, y0)
    # the trench floor sees fewer electrons than ions, relative to the field: it loses ions
    assert np.sum(mi1 < 0.95 * mi0) > 0 and np.all(mi1 <= mi0)
    assert me.max() <= 8.0 and me.min() >= 0.0


def test_charged_mc_loop_depth_matches_oracle_loop():
    """surface_charging with charge_alpha > 0 on the Monte-Carlo coverage path: device loop
    against the oracle loop (centre depth within one cell at every recorded step), and not
    deeper than the same run without charging."""
    dx = 0.25
    cfg = dict(Lx=5.0, Ly=2.5, Lz=8.0, dx=dx, trench_width=1.5, mask_th=1.0, sub_top=6.0,
               t_end=1.2, n_steps=12, hole=False)
    par = dict(petch.PAR, rate_scale=0.3, periodic_y=1, charge_alpha=0.8)
    fl = petch.Flags(**FLAGS, surface_charging=True)
    n = 60000
    geo = t3.run_etch_3d(**cfg, par=par, flags=fl, n_ion=n, n_neu=n, reinit_method="fsm",
                         verbose=False, record_depth_every=3)
    dev_hist = dict(geo['depth_history'])
    _, hist, _ = orc.run_etch_3d(cfg['Lx'], cfg['Ly'], cfg['Lz'], dx, cfg['trench_width'],
                                 cfg['mask_th'], cfg['sub_top'], cfg['t_end'], cfg['n_steps'],
                                 False, par, fl, n, n, record_depth_every=3)
    orc_hist = dict(hist)
    assert set(dev_hist) == set(orc_hist)
    for s in sorted(orc_hist):
        assert abs(dev_hist[s] - orc_hist[s]) <= dx + 1e-9, (s, dev_hist[s], orc_hist[s])
    assert max(orc_hist.values()) > 2 * dx
    g0 = t3.run_etch_3d(**cfg, par=par, flags=petch.Flags(**FLAGS), n_ion=n, n_neu=n,
                        reinit_method="fsm", verbose=False)
    assert t3.center_depth_3d(geo) <= t3.center_depth_3d(g0) + dx


def test_drop_in_with_charging(ed):
    """The drop-in mc_flux_3d_coupled with surface_charging on a fixture mesh: finite, charged
    (smaller floor ion flux than without) and the yields set."""
    m, geo, phi = _mesh("trench", ed)
    F = m.F
    par = dict(petch.PAR, periodic_y=1, charge_alpha=0.6)
    g = dict(geo, phi=phi)
    outs = []
    for charged in (False, True):
        p = dict(par)
        fl = petch.Flags(**FLAGS, surface_charging=charged)
        r = t3.mc_flux_3d_coupled(m, None, None, None, g, p, n_ion=200000, n_neu=200000, seed=3,
                                  flags=fl)
        assert all(np.isfinite(a).all() and a.shape == (F,) for a in r)
        assert '_ion_yield' in p
        outs.append(r)
    assert outs[1][0].sum() < outs[0][0].sum()
