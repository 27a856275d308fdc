"""GMRES radiosity solve on the device (petch_radiosity_gmres, radiosity_solver='gmres') against
the oracle (scipy's gmres, as the reference calls it) and tests/golden/gmres.npz (the reference's
own mc_flux_3d_radiosity with the GMRES solver)."""
import ctypes
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_helpers import cuda_mesh, small_feature, stream
import oracle.oracle as orc
import petch_b200 as petch
from petch_b200 import _lib
from petch_b200 import threed as t3

pytestmark = pytest.mark.gpu

CASES = [(k, t) for k in ("hole", "trench") for t in ("a", "b")]


@pytest.fixture(scope="module")
def gd():
    return np.load(os.path.join(GOLDEN, "gmres.npz"))


def setup(gd, key, tag):
    hole = key == "hole"
    phi, geo = small_feature(hole, nx=10, ny=10, nz=14, dx=0.3)
    np.testing.assert_array_equal(phi, gd[f"{key}_phi"])
    m = cuda_mesh(phi, geo['dx'], geo)
    np.testing.assert_array_equal(m.faces[:m.F].cpu().numpy(), gd[f"{key}_faces"])
    par = dict(petch.PAR, periodic_y=0 if hole else 1, radiosity_solver="gmres",
               betaE=float(gd[f"{key}_{tag}_betaE"][0]))
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", ion_reflection=True,
                     neutral_transport="radiosity")
    fe = t3.FluxEngine(geo, par, fl, m.MT)
    fe.mesh = m
    F = m.F
    hit = torch.full((m.MT * 64,), -1, dtype=torch.int32, device="cuda")
    hit[:F * 64] = torch.from_numpy(gd[f"{key}_{tag}_hit"]).cuda()
    r = fe._radiosity_buffers(64)
    _lib.call("petch_ff_matrix", m.id, m.MT, m.MV, hit.data_ptr(), 64, r['row_ptr'].data_ptr(),
              r['col'].data_ptr(), r['sky'].data_ptr(), r['scratch'].data_ptr(),
              r['scratch'].numel(), stream())
    return m, fe, r, hit, F


def gmres(m, fe, r, bare_t, beta, maxiter=40, restart=12):
    out = torch.full((m.MT,), -1.0, device="cuda")
    nb = ctypes.c_longlong()
    _lib.call("petch_radiosity_gmres_scratch_bytes", m.MT, restart, ctypes.byref(nb))
    scr = torch.empty(int(nb.value), dtype=torch.uint8, device="cuda")
    info = ctypes.c_int(-5)
    _lib.call("petch_radiosity_gmres", m.id, m.MT, m.MV, r['row_ptr'].data_ptr(),
              r['col'].data_ptr(), r['sky'].data_ptr(), 64, bare_t.data_ptr(), float(beta), 1e-3,
              restart, maxiter, out.data_ptr(), scr.data_ptr(), scr.numel(), ctypes.byref(info),
              stream())
    return out, info.value


@pytest.mark.parametrize("key,tag", CASES)
def test_solve_meets_the_tolerance_and_matches_scipy(gd, key, tag):
    m, fe, r, hit, F = setup(gd, key, tag)
    rng = np.random.default_rng(3)
    bare = rng.uniform(0.0, 1.0, F).astype(np.float32)
    bt = torch.ones(m.MT, device="cuda")
    bt[:F] = torch.from_numpy(bare).cuda()
    D, Aff = orc.ff_matrix(gd[f"{key}_{tag}_hit"], F, 64)
    for beta in (0.7, 0.05):
        out, info = gmres(m, fe, r, bt, beta)
        assert info == 0
        G = out[:F].double().cpu().numpy()
        assert G.min() >= 0.0 and G.max() <= 8.0
        s = np.clip(bare.astype(np.float64) * beta, 0.0, 1.0)
        M = Aff.multiply((1.0 - s)[None, :]).tocsr()
        res = np.linalg.norm(D - (G - M.dot(G)))
        assert res <= 1e-3 * np.linalg.norm(D) * 1.0001 + 1e-6, (res, np.linalg.norm(D))
        ref = orc.radiosity_solve(Aff, D, bare.astype(np.float64), beta, 40, "gmres")
        exact = np.clip(np.linalg.solve(np.eye(F) - M.toarray(), D), 0.0, 8.0)
        # both iterates are within the tolerance of the exact solution, not of each other
        err_dev = np.linalg.norm(G - exact) / np.linalg.norm(exact)
        err_ref = np.linalg.norm(ref - exact) / np.linalg.norm(exact)
        assert err_dev <= max(5.0 * err_ref, 2e-3), (err_dev, err_ref)


@pytest.mark.parametrize("key,tag", CASES)
def test_fixed_point_replays_reference(gd, key, tag):
    m, fe, r, hit, F = setup(gd, key, tag)
    fe.m_i[:F] = torch.from_numpy(gd[f"{key}_{tag}_m_i"].astype(np.float32)).cuda()
    fe.cos_i[:F] = torch.from_numpy(gd[f"{key}_{tag}_cos_i"].astype(np.float32)).cuda()
    iy = gd[f"{key}_{tag}_ion_yield"]
    for q in range(3):
        fe.y[q, :F] = torch.from_numpy(iy[q].astype(np.float32)).cuda()
    yields = tuple(fe.y[q].data_ptr() for q in range(3))
    fe.radiosity_from_hits(hit, 64, yields)
    for name, t in (("m_F", fe.m_F), ("m_O", fe.m_O)):
        got = t[:F].double().cpu().numpy()
        ref = gd[f"{key}_{tag}_{name}"]
        np.testing.assert_allclose(got, ref, rtol=5e-3, atol=2e-3, err_msg=name)


def test_reproducible_and_reports_non_convergence(gd):
    m, fe, r, hit, F = setup(gd, "trench", "b")
    bt = torch.full((m.MT,), 0.3, device="cuda")
    a, ia = gmres(m, fe, r, bt, 0.05)
    b, ib = gmres(m, fe, r, bt, 0.05)
    assert ia == ib == 0 and torch.equal(a, b)
    _, i0 = gmres(m, fe, r, bt, 0.05, maxiter=0)
    assert i0 == 1
    _, i1 = gmres(m, fe, r, bt, 0.05, maxiter=1, restart=1)
    assert i1 == 1
    with pytest.raises(_lib.PetchError, match="scratch too small"):
        info = ctypes.c_int()
        small = torch.empty(256, dtype=torch.uint8, device="cuda")
        _lib.call("petch_radiosity_gmres", m.id, m.MT, m.MV, r['row_ptr'].data_ptr(),
                  r['col'].data_ptr(), r['sky'].data_ptr(), 64, bt.data_ptr(), 0.05, 1e-3, 12, 40,
                  a.data_ptr(), small.data_ptr(), small.numel(), ctypes.byref(info), stream())


def test_radiosity_loop_with_gmres_runs():
    """run_etch_3d with the GMRES radiosity solver: finite, etches, and differs from the Jacobi
    run only through the solver."""
    cfg = dict(Lx=5.0, Ly=5.0, Lz=8.0, dx=0.25, trench_width=2.0, mask_th=1.0, sub_top=6.0,
               t_end=0.6, n_steps=6, hole=True)
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     ion_reflection=True, neutral_transport="radiosity")
    depths = {}
    for solver in ("gmres", "jacobi"):
        par = dict(petch.PAR, rate_scale=0.3, radiosity_solver=solver)
        g = t3.run_etch_3d(**cfg, par=par, flags=fl, n_ion=30000, n_neu=30000,
                           reinit_method="fsm", verbose=False)
        assert np.isfinite(g['phi']).all()
        depths[solver] = t3.center_depth_3d(g)
    assert depths["gmres"] > 0.25 and abs(depths["gmres"] - depths["jacobi"]) <= 0.5
