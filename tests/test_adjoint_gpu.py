"""Recipe-gradient (forward-mode tangent) kernels against finite differences of the primal kernels
they mirror, stage by stage, plus the tangent loop's primal against the plain engine and the
torch.autograd.Function wrapper.

Deterministic stages (advection, reinit, chemistry) are compared with central differences
directly; Monte-Carlo stages (ion energy, neutral coverage) through face totals, where the rare
decision flips a finite step causes average out."""
import ctypes

import numpy as np
import pytest
import torch

from gpu_helpers import cuda_mesh, domain, small_feature, stream
import petch_b200 as petch
from petch_b200 import _lib
from petch_b200 import threed as t3
from petch_b200.adjoint import (EtchProfile, apply_theta, profile_loss, radial_profile,
                                run_etch_3d_tangent)

pytestmark = pytest.mark.gpu


def _field(seed, n=(24, 22, 26), dx=0.25):
    rng = np.random.default_rng(seed)
    X, Y, Z = np.meshgrid(*(np.arange(k) * dx for k in n), indexing="ij")
    phi = 1.6 - np.sqrt((X - 3.0) ** 2 + (Y - 2.7) ** 2 + (Z - 3.2) ** 2)
    phi += 0.05 * np.sin(3 * X) * np.cos(2 * Y)
    mask = (Z > 5.6) & (rng.random(phi.shape) < 0.3)
    return phi.astype(np.float32), mask.astype(np.uint8), dx, rng


def _close_fraction(t, fd, rtol, atol):
    ok = np.abs(t - fd) <= atol + rtol * np.abs(fd)
    return ok.mean()


def test_advect_tangent_matches_finite_differences():
    phi, mask, dx, rng = _field(1)
    n = phi.size
    F = np.where(np.abs(phi) < 1.0, rng.uniform(0.2, 2.0, phi.shape), 0.0).astype(np.float32)
    F[mask.astype(bool)] = -1.0
    dphi = rng.normal(0, 0.05, (3,) + phi.shape).astype(np.float32)
    dF = (rng.normal(0, 0.3, (3,) + phi.shape) * (F > 0)).astype(np.float32)
    mp = phi.copy()
    # every device input is held in a name for the duration of the calls that read it
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    P, T, dP = g(phi), torch.empty(phi.shape, device="cuda"), g(dphi)
    dT = torch.empty_like(dP)
    Fd, dFd, Md, MPd = g(F), g(dF), g(mask), g(mp)
    nx, ny, nz = phi.shape
    dt, nsub = 0.05, 3
    _lib.call("petch_advect_tangent", P.data_ptr(), T.data_ptr(), dP.data_ptr(), dT.data_ptr(),
              Fd.data_ptr(), dFd.data_ptr(), Md.data_ptr(), MPd.data_ptr(), nx, ny, nz,
              float(1 / dx), dt, nsub, stream())
    # primal equal to petch_advect
    Q, Qt = g(phi), torch.empty(phi.shape, device="cuda")
    _lib.call("petch_advect", Q.data_ptr(), Qt.data_ptr(), Fd.data_ptr(), Md.data_ptr(),
              MPd.data_ptr(), nx, ny, nz, float(1 / dx), dt, nsub, stream())
    assert torch.equal(P, Q)
    eps = 1e-3
    for k in range(3):
        outs = []
        for sgn in (1, -1):
            A = g(phi + sgn * eps * dphi[k])
            Fk = g(np.where(mask.astype(bool), -1.0, F + sgn * eps * dF[k]).astype(np.float32))
            _lib.call("petch_advect", A.data_ptr(), Qt.data_ptr(), Fk.data_ptr(), Md.data_ptr(),
                      MPd.data_ptr(), nx, ny, nz, float(1 / dx), dt, nsub, stream())
            outs.append(A.double().cpu().numpy())
        fd = (outs[0] - outs[1]) / (2 * eps)
        t = dP[k].double().cpu().numpy()
        assert _close_fraction(t, fd, 2e-2, 2e-3) > 0.995, k


def test_reinit_tangent_matches_finite_differences():
    phi, mask, dx, rng = _field(2)
    phi = (phi * 1.3).astype(np.float32)               # |grad| != 1: the reinit changes values
    dphi = rng.normal(0, 0.05, (3,) + phi.shape).astype(np.float32)
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    nx, ny, nz = phi.shape
    n = phi.size
    band = 6 * dx
    big, cap, n_iter = band + 4 * dx, band + dx, int(np.ceil(band / dx)) + 4
    P, dP = g(phi), g(dphi)
    scr = [torch.empty(n, device="cuda") for _ in range(2)] + \
          [torch.empty(3 * n, device="cuda") for _ in range(2)]
    _lib.call("petch_reinit_tangent", P.data_ptr(), dP.data_ptr(), *[x.data_ptr() for x in scr],
              nx, ny, nz, dx, big, cap, n_iter, stream())
    Q, ua, ub = g(phi), torch.empty(n, device="cuda"), torch.empty(n, device="cuda")
    _lib.call("petch_reinit_eik", Q.data_ptr(), Q.data_ptr(), ua.data_ptr(), ub.data_ptr(), nx, ny,
              nz, dx, big, cap, n_iter, 0, stream())
    assert torch.equal(P, Q)
    eps = 1e-3
    for k in range(3):
        outs = []
        for sgn in (1, -1):
            A = g(phi + sgn * eps * dphi[k])
            _lib.call("petch_reinit_eik", A.data_ptr(), A.data_ptr(), ua.data_ptr(), ub.data_ptr(),
                      nx, ny, nz, dx, big, cap, n_iter, 0, stream())
            outs.append(A.double().cpu().numpy())
        fd = (outs[0] - outs[1]) / (2 * eps)
        t = dP[k].double().cpu().numpy()
        assert _close_fraction(t, fd, 2e-2, 2e-3) > 0.99, k


def _chem_case():
    phi, geo = small_feature(True)
    m = cuda_mesh(phi, geo['dx'], geo)
    rng = np.random.default_rng(9)
    MT = m.MT
    par = dict(petch.PAR)
    flags = petch.Flags(chemistry="belen", yield_angular="viennaps", ion_reflection=True)
    fields = {k: rng.uniform(0.2, 2.0, MT).astype(np.float32) for k in
              ("m_F", "m_O", "y_sp", "y_ie", "y_ip")}
    tans = {k: rng.normal(0, 0.1, (3, MT)).astype(np.float32) for k in fields}
    return m, par, flags, fields, tans


def test_chemistry_tangents_match_finite_differences():
    m, par, flags, fields, tans = _chem_case()
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dOflux = (ctypes.c_double * 3)(0.0, float(par['Fflux']), 0.0)
    drate = (ctypes.c_double * 3)(0.0, 0.0, 1.0)
    MT, F = m.MT, m.F
    bare, dbare = torch.empty(MT, device="cuda"), torch.empty(3 * MT, device="cuda")
    V, dV = torch.empty(MT, device="cuda"), torch.empty(3 * MT, device="cuda")
    stats = torch.zeros(2, dtype=torch.int32, device="cuda")
    d = {k: g(v) for k, v in fields.items()}
    dd = {k: g(v) for k, v in tans.items()}
    chem = t3.chem_params(par, flags)
    _lib.call("petch_belen_bare_tangent", m.id, MT, m.MV, ctypes.byref(chem), dOflux,
              d['m_F'].data_ptr(), dd['m_F'].data_ptr(), d['m_O'].data_ptr(), dd['m_O'].data_ptr(),
              d['y_ie'].data_ptr(), dd['y_ie'].data_ptr(), d['y_ip'].data_ptr(),
              dd['y_ip'].data_ptr(), bare.data_ptr(), dbare.data_ptr(), stream())
    _lib.call("petch_surface_rate_tangent", m.id, MT, m.MV, ctypes.byref(chem), dOflux, drate,
              d['m_F'].data_ptr(), dd['m_F'].data_ptr(), d['m_O'].data_ptr(), dd['m_O'].data_ptr(),
              d['y_sp'].data_ptr(), dd['y_sp'].data_ptr(), d['y_ie'].data_ptr(),
              dd['y_ie'].data_ptr(), d['y_ip'].data_ptr(), dd['y_ip'].data_ptr(), V.data_ptr(),
              dV.data_ptr(), stats.data_ptr(), stream())

    def primal(h, k):
        p = dict(par)
        if k == 1:
            p['Oflux'] = par['Oflux'] + h * par['Fflux']
        if k == 2:
            p['rate_scale'] = par['rate_scale'] + h
        c = t3.chem_params(p, flags)
        x = {kk: g(fields[kk].astype(np.float64) + h * tans[kk][k]) for kk in fields}
        x = {kk: v.float() for kk, v in x.items()}
        b, v = torch.empty(MT, device="cuda"), torch.empty(MT, device="cuda")
        mi = torch.ones(MT, device="cuda")
        _lib.call("petch_belen_bare", m.id, MT, m.MV, ctypes.byref(c), mi.data_ptr(),
                  x['m_F'].data_ptr(), x['m_O'].data_ptr(), mi.data_ptr(), x['y_ie'].data_ptr(),
                  x['y_ip'].data_ptr(), b.data_ptr(), stream())
        _lib.call("petch_surface_rate", m.id, MT, m.MV, ctypes.byref(c), mi.data_ptr(),
                  x['m_F'].data_ptr(), x['m_O'].data_ptr(), mi.data_ptr(), x['y_sp'].data_ptr(),
                  x['y_ie'].data_ptr(), x['y_ip'].data_ptr(), v.data_ptr(),
                  torch.zeros(2, dtype=torch.int32, device="cuda").data_ptr(), stream())
        return b[:F].double().cpu().numpy(), v[:F].double().cpu().numpy()

    b0, v0 = primal(0.0, 0)
    np.testing.assert_array_equal(b0, bare[:F].double().cpu().numpy())
    np.testing.assert_array_equal(v0, V[:F].double().cpu().numpy())
    h = 1e-3
    for k in range(3):
        bp, vp = primal(h, k)
        bm, vm = primal(-h, k)
        for fd, t in (((bp - bm) / (2 * h), dbare[k * MT:k * MT + F]),
                      ((vp - vm) / (2 * h), dV[k * MT:k * MT + F])):
            t = t.double().cpu().numpy()
            scale = np.abs(fd).max() + 1e-30
            assert _close_fraction(t, fd, 2e-2, 1e-3 * scale) > 0.99, k


def test_ion_energy_tangent_matches_finite_differences():
    phi, geo = small_feature(True)
    m = cuda_mesh(phi, geo['dx'], geo)
    par = dict(petch.PAR, periodic_y=0)
    MT, n = m.MT, 2_000_000
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    tal, ang = torch.zeros((MT, 4), device="cuda"), torch.zeros(MT, device="cuda")
    dtal = torch.zeros(3 * MT, device="cuda")
    E0 = 120.0
    _lib.call("petch_trace_ions_tangent", m.id, MT, m.MV, ctypes.byref(domain(geo)),
              ctypes.byref(t3.ion_params(dict(par, Emean=E0))), 11, n, tal.data_ptr(),
              ang.data_ptr(), dtal.data_ptr(), work.data_ptr(), stream())
    base = tal[:m.F].double().sum(0).cpu().numpy()
    ref = torch.zeros_like(tal)
    _lib.call("petch_trace_ions", m.id, MT, m.MV, ctypes.byref(domain(geo)),
              ctypes.byref(t3.ion_params(dict(par, Emean=E0))), 11, n, ref.data_ptr(),
              ang.data_ptr(), work.data_ptr(), stream())
    np.testing.assert_allclose(ref[:m.F].double().sum(0).cpu().numpy(), base, rtol=1e-5)
    h = 2.0
    sums = []
    for E in (E0 + h, E0 - h):
        _lib.call("petch_trace_ions", m.id, MT, m.MV, ctypes.byref(domain(geo)),
                  ctypes.byref(t3.ion_params(dict(par, Emean=E))), 11, n, ref.data_ptr(),
                  ang.data_ptr(), work.data_ptr(), stream())
        sums.append(ref[:m.F].double().sum(0).cpu().numpy())
    fd = (sums[0] - sums[1]) / (2 * h)
    t = dtal.view(3, MT)[:, :m.F].double().sum(1).cpu().numpy()
    np.testing.assert_allclose(t, fd[:3], rtol=0.05)


def test_neutral_coverage_tangent_matches_finite_differences():
    phi, geo = small_feature(False)
    m = cuda_mesh(phi, geo['dx'], geo)
    MT, F, n = m.MT, m.F, 2_000_000
    rng = np.random.default_rng(3)
    bare = rng.uniform(0.3, 0.9, MT).astype(np.float32)
    dbare = np.zeros((3, MT), np.float32)
    dbare[0] = 0.2
    dbare[1, :F] = rng.uniform(-0.2, 0.2, F)
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    flux, dflux = torch.zeros(MT, device="cuda"), torch.zeros(3 * MT, device="cuda")
    bare_d, dbare_d = g(bare), g(dbare)
    # roulette decisions that a finite step flips make the difference quotient noisy (about
    # 1 / sqrt(h)): a wide step, two seeds
    h = 0.05
    for k in (0, 1):
        fd = t = 0.0
        for seed in (5, 6):
            _lib.call("petch_trace_neutrals_tangent", m.id, MT, m.MV, ctypes.byref(domain(geo)),
                      bare_d.data_ptr(), dbare_d.data_ptr(), 0.7, seed, 0, n, flux.data_ptr(),
                      dflux.data_ptr(), work.data_ptr(), stream())
            t += dflux[k * MT:k * MT + F].double().sum().item()
            tot = []
            for sgn in (1, -1):
                f2 = torch.zeros(MT, device="cuda")
                bk = g(bare + sgn * h * dbare[k])
                _lib.call("petch_trace_neutrals", m.id, MT, m.MV, ctypes.byref(domain(geo)),
                          bk.data_ptr(), 0.7, seed, 0, n, f2.data_ptr(), work.data_ptr(), stream())
                tot.append(f2[:F].double().sum().item())
            fd += (tot[0] - tot[1]) / (2 * h)
        assert abs(t - fd) <= 0.05 * abs(fd), (k, t, fd)


def test_tangent_loop_primal_follows_the_plain_loop():
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     warm_start_coverage=True, ion_reflection=True)
    cfg = dict(Lx=6.0, Ly=6.0, Lz=10.0, dx=0.25, trench_width=3.0, mask_th=1.0, sub_top=7.0,
               t_end=0.4, n_steps=4, hole=True)
    theta = (110.0, 0.15, 0.05)
    phi, dphi, geo, _ = run_etch_3d_tangent(theta, flags=fl, n_ion=40000, n_neu=40000,
                                            seed_offset=2, **cfg)
    ref = t3.run_etch_3d(**cfg, par=apply_theta(dict(petch.PAR), theta), flags=fl, n_ion=40000,
                         n_neu=40000, reinit_method="fsm", verbose=False, seed_offset=2)
    assert abs(t3.center_depth_3d(dict(geo, phi=phi)) - t3.center_depth_3d(ref)) <= 0.25 + 1e-9
    assert np.isfinite(dphi).all()
    p, J = radial_profile(phi, geo, dphi)
    ok = np.isfinite(p)
    assert ok.sum() >= 8
    assert np.all(J[ok, 2] >= 0.0)                 # a higher rate_scale never etches less here


def test_autograd_function_returns_the_jacobian_product():
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     warm_start_coverage=True, ion_reflection=True)
    cfg = dict(Lx=6.0, Ly=6.0, Lz=10.0, dx=0.25, trench_width=3.0, mask_th=1.0, sub_top=7.0,
               t_end=0.3, n_steps=3, hole=True, flags=fl, n_ion=30000, n_neu=30000,
               seed_offset=4, n_bins=16)
    theta = torch.tensor([110.0, 0.15, 0.05], dtype=torch.float64, requires_grad=True)
    prof = EtchProfile.apply(theta, cfg)
    w = torch.linspace(0.5, 1.5, prof.numel(), dtype=torch.float64)
    ok = torch.isfinite(prof)
    (prof[ok] * w[ok]).sum().backward()
    kw = {k: v for k, v in cfg.items() if k != 'n_bins'}
    phi, dphi, geo, _ = run_etch_3d_tangent(theta.detach().tolist(), **kw)
    p2, J = radial_profile(phi, geo, dphi, 16)
    want = (np.nan_to_num(J) * np.where(np.isfinite(p2), w.numpy(), 0.0)[:, None]).sum(0)
    np.testing.assert_allclose(theta.grad.numpy(), want, rtol=0.1, atol=1e-6)
    loss = profile_loss(theta.detach().requires_grad_(True), cfg, np.nan_to_num(p2) + 0.1)
    assert torch.isfinite(loss)


_HOLE = dict(Lx=8.0, Ly=8.0, Lz=12.0, dx=0.25, trench_width=4.0, mask_th=1.0, sub_top=8.0,
             hole=True)
_FLAGS = dict(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
              ion_reflection=True, warm_start_coverage=True)


def _crn_slope(cfg, theta, k, h_rel, seeds, **kw):
    """Seed-mean tangent and central difference (common random numbers) of the radial profile
    along theta_k, averaged over the bins every run defines."""
    tan, fd = [], []
    for s in seeds:
        phi, dphi, geo, _ = run_etch_3d_tangent(theta, seed_offset=s, **cfg, **kw)
        p, J = radial_profile(phi, geo, dphi)
        h = h_rel * theta[k]
        tp, tm = np.array(theta, float), np.array(theta, float)
        tp[k] += h
        tm[k] -= h
        pp = radial_profile(run_etch_3d_tangent(tp, seed_offset=s, **cfg, **kw)[0], geo)[0]
        pm = radial_profile(run_etch_3d_tangent(tm, seed_offset=s, **cfg, **kw)[0], geo)[0]
        ok = np.isfinite(p) & np.isfinite(pp) & np.isfinite(pm) & (p > -0.5)
        tan.append(J[ok, k].mean())
        fd.append(((pp - pm)[ok] / (2 * h)).mean())
    return np.array(tan), np.array(fd)


def test_loop_tangent_with_a_uniform_rate_matches_central_differences(monkeypatch):
    """The level-set half of the loop tangent (extension, advection, reinit, the profile) over 6
    steps: with every face's velocity set to rate_scale * 24 um/min (no tracing), the profile's
    rate_scale tangent equals its central difference, and both equal depth / rate_scale (the
    front moves about half a cell per step)."""
    from petch_b200 import adjoint

    class UniformRate(adjoint.TangentEngine):
        def flux_tangent(self, n_ion, n_neu, seed, warm):
            pass

        def rate_extend_tangent(self, band):
            rs = float(self.par['rate_scale'])
            self.V.fill_(24.0 * rs)
            self.dV.zero_()
            self.dV[2].fill_(24.0)
            self.small[6:8].zero_()
            self.small[7:8].view(torch.float32).fill_(24.0 * rs)
            m = self.mesh
            nx, ny, nz = self.shape
            _lib.call("petch_extend_velocity_dual", m.id, m.MT, m.MV, self.phi.data_ptr(),
                      self.mask.data_ptr(), nx, ny, nz, self.dx, float(band), self.V.data_ptr(),
                      self.dV.data_ptr(), self.F.data_ptr(), self.dF.data_ptr(), 1,
                      self.active.data_ptr(), self.small[8:9].data_ptr(), self.ncell,
                      self.small[0:6].data_ptr(), t3._sp())

    monkeypatch.setattr(adjoint, "TangentEngine", UniformRate)
    fl = petch.Flags(**_FLAGS)
    flat = dict(_HOLE, Lx=4.0, Ly=4.0, trench_width=8.0, hole=False)
    for geo_kw in (_HOLE, dict(_HOLE, Lx=16.0, Ly=16.0, trench_width=12.0), flat):
        cfg = dict(geo_kw, t_end=0.6, n_steps=6, flags=fl, n_ion=1000, n_neu=1000)
        theta = np.array([100.0, 0.1, 0.05])
        tan, fd = _crn_slope(cfg, theta, 2, 0.01, [0])
        phi, _, geo, _ = run_etch_3d_tangent(theta, seed_offset=0, **cfg)
        p = radial_profile(phi, geo)[0]
        etched = p[np.isfinite(p) & (p > -0.5)].mean()
        assert abs(tan[0] - fd[0]) <= 0.03 * abs(fd[0]), (geo_kw, tan, fd)
        assert abs(tan[0] * theta[2] - etched) <= 0.03 * etched, (geo_kw, tan, etched)


def test_one_step_loop_tangent_matches_the_seed_averaged_difference():
    """The first step's mesh does not depend on theta, so holding it fixed is exact there: the
    one-step profile tangent equals the common-random-number central difference (16 seeds,
    30000 rays) along mean ion energy and rate_scale, within 3 % plus three standard errors."""
    fl = petch.Flags(**_FLAGS)
    cfg = dict(_HOLE, t_end=0.1, n_steps=1, flags=fl, n_ion=30000, n_neu=30000)
    _lib.set_deterministic(8 * 16 * 131072)
    try:
        for k in (0, 2):
            tan, fd = _crn_slope(cfg, np.array([100.0, 0.1, 0.05]), k, 0.02, range(300, 316))
            se = fd.std(ddof=1) / np.sqrt(len(fd))
            assert abs(tan.mean() - fd.mean()) <= 0.03 * abs(fd.mean()) + 3 * se, (k, tan, fd)
    finally:
        _lib.set_deterministic(0)


def test_one_step_radiosity_loop_tangent_matches_the_seed_averaged_difference():
    """The recipe gradient on the radiosity path (ion energy tangents through the unsmoothed ion
    yields, coverage tangents through the Jacobi solve): one step, where holding the mesh fixed
    is exact, against the common-random-number central difference (16 seeds)."""
    fl = petch.Flags(**_FLAGS, neutral_transport="radiosity")
    cfg = dict(_HOLE, t_end=0.1, n_steps=1, flags=fl, n_ion=30000, n_neu=30000)
    _lib.set_deterministic(8 * 16 * 131072)
    try:
        for k in (0, 2):
            tan, fd = _crn_slope(cfg, np.array([100.0, 0.1, 0.05]), k, 0.02, range(300, 316))
            se = fd.std(ddof=1) / np.sqrt(len(fd))
            assert abs(tan.mean() - fd.mean()) <= 0.03 * abs(fd.mean()) + 3 * se, (k, tan, fd)
    finally:
        _lib.set_deterministic(0)
