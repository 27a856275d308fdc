"""Recipe gradients of the etch loop: d(etch profile) / d(theta) for theta = (mean ion energy,
O/F flux ratio, rate_scale), computed in forward mode alongside the simulation.

No reference counterpart: the reference's only wp.Tape use differentiates a chemistry kernel on
frozen fluxes (scripts/inverse_design.py:20-45); its run_etch_3d is not differentiable.

What is differentiated, and what is held fixed.  Every stage of the step (threed.py:1643-1795)
runs its primal computation unchanged and carries three tangent directions:
  * ions: d(sputter, ion-enhanced, passivation tallies) / d(mean energy) along the same Philox
    paths (hits, sticking and energy-acceptance decisions fixed);
  * neutrals: the weight tangents of every Russian-roulette path given the coverage tangents
    (roulette decisions fixed; a survivor carries dw / p, p = w / 0.3 its survival probability,
    which keeps the tangent an unbiased estimate of the derivative of the expected deposits);
  * normalisation / smoothing (linear), Belen coverages and surface rate (float64 duals), the
    coverage fixed point and its warm start, the velocity extension (nearest face fixed);
  * the narrow-band advection (upwind choices fixed) and the Eikonal reinit (branches fixed);
  * on the radiosity path (neutral_transport="radiosity", Jacobi solve): the unsmoothed ion
    yields' energy tangents and the coverage tangents through every Jacobi sweep (the form
    factors and sky view are geometry).
Held fixed: the surface mesh and hit topology — the fluxes' dependence on the shape of the
surface is not differentiated (a pathwise derivative of a ray tally with respect to the surface
would need visibility-boundary terms, which are out of scope), and the CFL substep count.
Forward mode is used because theta has three components: the cost is one tangent-carrying run
(no reverse sweep, no level-set checkpoints; memory independent of the number of steps).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .params import DEFAULT_FLAGS, PAR
from .threed import (MESH_ERR_HASH_FULL, MESH_ERR_TRI_OVERFLOW, MESH_ERR_VERT_OVERFLOW, EtchEngine,
                     _sp, make_trench_3d)

ND = 3
THETA_NAMES = ("Emean", "O_F_ratio", "rate_scale")


def apply_theta(par, theta):
    """PAR with the recipe parameters theta = (mean ion energy eV, Oflux / Fflux, rate_scale)."""
    E, r, rs = (float(t) for t in theta)
    return dict(par, Emean=E, Oflux=r * par['Fflux'], rate_scale=rs)


class TangentEngine(EtchEngine):
    """EtchEngine that also carries the three theta-tangents of its state."""

    def __init__(self, geo, par, flags, max_tris=None):
        super().__init__(geo, par, flags, max_tris=max_tris)
        n = self.ncell
        dev = dict(device="cuda", dtype=torch.float32)
        self.dphi = torch.zeros((ND,) + self.shape, **dev)
        self.dtmp = torch.empty_like(self.dphi)
        self.dF = torch.zeros((ND, n), **dev)
        self.du_a = torch.empty((ND, n), **dev)
        self.du_b = torch.empty((ND, n), **dev)
        self.mask_u8 = self.mask.to(torch.uint8).contiguous()
        self.dOflux = (ctypes.c_double * ND)(0.0, float(par['Fflux']), 0.0)
        self.drate = (ctypes.c_double * ND)(0.0, 0.0, 1.0)
        self.prev_dbare = None

    def _alloc_faces(self, MT):
        super()._alloc_faces(MT)
        dev = dict(device="cuda", dtype=torch.float32)
        self.dtal = torch.empty((ND, MT), **dev)
        self.dtal_in = torch.zeros((ND, MT), **dev)       # [dtal_q, 0, 0] staging
        self.dy = torch.zeros((3, ND, MT), **dev)          # d(y_sp, y_ie, y_ip)
        self.dm_F = torch.zeros((ND, MT), **dev)
        self.dm_O = torch.zeros((ND, MT), **dev)
        self.dbare = torch.zeros((ND, MT), **dev)
        self.dflux = torch.empty((ND, MT), **dev)
        self.dflux_o = torch.empty((ND, MT), **dev)      # the O species of a paired round
        self.dV = torch.zeros((ND, MT), **dev)
        self.ttmp = torch.empty((2, MT), **dev)

    def end_step(self, warm):
        if warm:
            old = self.prev
            old_d = self.prev_dbare
            self.prev = (self.mesh, self.bare)
            self.prev_dbare = self.dbare
            if old is not None and old[0].MT == self.MT:
                self.mesh, self.bare = old
                self.dbare = old_d
            else:
                from .threed import DeviceMesh
                self.mesh = DeviceMesh(self.MT)
                self.bare = torch.empty(self.MT, device="cuda")
                self.dbare = torch.zeros((ND, self.MT), device="cuda")

    def grow(self, need):
        super().grow(need)
        self.prev = None
        self.prev_dbare = None

    def flux_tangent(self, n_ion, n_neu, seed, warm):
        """mc_flux_3d_coupled (faithful ions) with tangents."""
        par, m = self.par, self.mesh
        s = _sp()
        A_src = float(self.geo['Lx'] * self.geo['Ly'])
        n_smooth = int(par.get('flux_smooth', 1))
        alpha = float(par.get('flux_smooth_alpha', 1.0))
        work = self.small[0:6]
        MT = m.MT
        seeded = False
        if warm and self.prev is not None:
            pm, pb = self.prev
            _lib.call("petch_warmstart_dual", pm.id, pm.MT, pm.MV, pb.data_ptr(),
                      self.prev_dbare.data_ptr(), m.id, m.MT, m.MV, self.bare.data_ptr(),
                      self.dbare.data_ptr(), work.data_ptr(), s)
            seeded = True
        _lib.call("petch_trace_ions_tangent", m.id, m.MT, m.MV, ctypes.byref(self.dom),
                  ctypes.byref(self.ionp), int(seed * 9 + 1) & 0xffffffff, int(n_ion),
                  self.tal4.data_ptr(), self.ang.data_ptr(), self.dtal.data_ptr(),
                  work.data_ptr(), s)
        norm = float(A_src / n_ion)
        _lib.call("petch_ion_post", m.id, m.MT, m.MV, self.tal4.data_ptr(), self.ang.data_ptr(),
                  norm, n_smooth, alpha, self.y[0].data_ptr(), self.y[1].data_ptr(),
                  self.y[2].data_ptr(), self.m_i.data_ptr(), self.cos_i.data_ptr(),
                  self.tmp5.data_ptr(), s)
        for q in range(3):                     # d y_q: direction 0 only (ion energy)
            self.dtal_in[0].copy_(self.dtal[q])
            _lib.call("petch_norm_smooth_tangent", m.id, m.MT, m.MV, self.dtal_in.data_ptr(),
                      self.dtal_in.data_ptr(), norm, 0.0, 0.0, 0, n_smooth, alpha, 1,
                      self.dy[q].data_ptr(), self.ttmp[0].data_ptr(), self.ttmp[1].data_ptr(), s)
        n_fp = int(par.get('n_fp', 1 if seeded else 4))
        if not seeded:
            self.bare.fill_(1.0)
            self.dbare.zero_()
        betaE, betaO = float(par.get('betaE', 0.7)), float(par.get('betaO', 1.0))
        flux_o = self.tmp5[2 * MT:3 * MT]
        for it in range(n_fp):
            # both species of the round in one launch (F: betaE, seed*9+2+2it; O: betaO, +3+2it)
            _lib.call("petch_trace_neutral_pair_tangent", m.id, m.MT, m.MV, ctypes.byref(self.dom),
                      self.bare.data_ptr(), self.dbare.data_ptr(), betaE, betaO,
                      int(seed * 9 + 2 + 2 * it) & 0xffffffff,
                      int(seed * 9 + 3 + 2 * it) & 0xffffffff, 0, int(n_neu),
                      self.flux.data_ptr(), self.dflux.data_ptr(), flux_o.data_ptr(),
                      self.dflux_o.data_ptr(), work.data_ptr(), s)
            for fl, dfl, out, dout in ((self.flux, self.dflux, self.m_F, self.dm_F),
                                       (flux_o, self.dflux_o, self.m_O, self.dm_O)):
                _lib.call("petch_norm_smooth", m.id, m.MT, m.MV, fl.data_ptr(),
                          float(A_src / n_neu), 0.0, 8.0, 1, n_smooth, alpha, out.data_ptr(),
                          self.tmp5.data_ptr(), self.tmp5[MT:].data_ptr(), s)
                _lib.call("petch_norm_smooth_tangent", m.id, m.MT, m.MV, fl.data_ptr(),
                          dfl.data_ptr(), float(A_src / n_neu), 0.0, 8.0, 1, n_smooth,
                          alpha, 0, dout.data_ptr(), self.ttmp[0].data_ptr(),
                          self.ttmp[1].data_ptr(), s)
            _lib.call("petch_belen_bare_tangent", m.id, m.MT, m.MV, ctypes.byref(self.chem),
                      self.dOflux, self.m_F.data_ptr(), self.dm_F.data_ptr(), self.m_O.data_ptr(),
                      self.dm_O.data_ptr(), self.y[1].data_ptr(), self.dy[1].data_ptr(),
                      self.y[2].data_ptr(), self.dy[2].data_ptr(), self.bare.data_ptr(),
                      self.dbare.data_ptr(), s)
        self.yields = (self.y[0].data_ptr(), self.y[1].data_ptr(), self.y[2].data_ptr())

    def flux_radiosity_tangent(self, phi, n_ion, seed, n_ff=64, n_fp=4, n_iter=40):
        """mc_flux_3d_radiosity (threed.py:923-991) with tangents: the faithful ions of
        _ions_deterministic (unsmoothed yields) with their energy tangents, the form factors and
        the sky view as geometry (held fixed), then n_fp rounds of the two-species Jacobi solve
        with the coverage tangents (petch_radiosity_solve_tangent) and the Belen coverage
        update with its tangents, from bare = 1."""
        par, m = self.par, self.mesh
        s = _sp()
        A_src = float(self.geo['Lx'] * self.geo['Ly'])
        work = self.small[0:6]
        _lib.call("petch_trace_ions_tangent", m.id, m.MT, m.MV, ctypes.byref(self.dom),
                  ctypes.byref(self.ionp), int(seed * 9 + 1) & 0xffffffff, int(n_ion),
                  self.tal4.data_ptr(), self.ang.data_ptr(), self.dtal.data_ptr(),
                  work.data_ptr(), s)
        norm = float(A_src / n_ion)
        _lib.call("petch_ion_post", m.id, m.MT, m.MV, self.tal4.data_ptr(), self.ang.data_ptr(),
                  norm, 0, 1.0, self.y[0].data_ptr(), self.y[1].data_ptr(), self.y[2].data_ptr(),
                  self.m_i.data_ptr(), self.cos_i.data_ptr(), self.tmp5.data_ptr(), s)
        for q in range(3):                     # d y_q: direction 0 only (ion energy)
            self.dtal_in[0].copy_(self.dtal[q])
            _lib.call("petch_norm_smooth_tangent", m.id, m.MT, m.MV, self.dtal_in.data_ptr(),
                      self.dtal_in.data_ptr(), norm, 0.0, 0.0, 0, 0, 1.0, 1,
                      self.dy[q].data_ptr(), self.ttmp[0].data_ptr(), self.ttmp[1].data_ptr(), s)
        r = self._radiosity_buffers(n_ff)
        if r.get('work_tan') is None or r['work_tan'].numel() < 16 * m.MT:
            r['work_tan'] = torch.empty(16 * m.MT, device="cuda", dtype=torch.float64)
        nx, ny, nz = phi.shape
        _lib.call("petch_gas_normals", m.id, m.MT, m.MV, phi.data_ptr(), nx, ny, nz,
                  float(self.geo['dx']), r['fn'].data_ptr(), s)
        _lib.call("petch_trace_ff", m.id, m.MT, m.MV, ctypes.byref(self.dom), r['fn'].data_ptr(),
                  int(seed) & 0xffffffff, int(n_ff), r['hit'].data_ptr(), work.data_ptr(), s)
        _lib.call("petch_ff_matrix", m.id, m.MT, m.MV, r['hit'].data_ptr(), int(n_ff),
                  r['row_ptr'].data_ptr(), r['col'].data_ptr(), r['sky'].data_ptr(),
                  r['scratch'].data_ptr(), r['scratch'].numel(), s)
        self.bare.fill_(1.0)
        self.dbare.zero_()
        betaE, betaO = float(par.get('betaE', 0.7)), float(par.get('betaO', 1.0))
        for _ in range(n_fp):
            _lib.call("petch_radiosity_solve_tangent", m.id, m.MT, m.MV, r['row_ptr'].data_ptr(),
                      r['col'].data_ptr(), r['sky'].data_ptr(), int(n_ff), self.bare.data_ptr(),
                      self.dbare.data_ptr(), betaE, betaO, int(n_iter), self.m_F.data_ptr(),
                      self.m_O.data_ptr(), self.dm_F.data_ptr(), self.dm_O.data_ptr(),
                      r['work_tan'].data_ptr(), s)
            _lib.call("petch_belen_bare_tangent", m.id, m.MT, m.MV, ctypes.byref(self.chem),
                      self.dOflux, self.m_F.data_ptr(), self.dm_F.data_ptr(), self.m_O.data_ptr(),
                      self.dm_O.data_ptr(), self.y[1].data_ptr(), self.dy[1].data_ptr(),
                      self.y[2].data_ptr(), self.dy[2].data_ptr(), self.bare.data_ptr(),
                      self.dbare.data_ptr(), s)
        self.yields = (self.y[0].data_ptr(), self.y[1].data_ptr(), self.y[2].data_ptr())

    def rate_extend_tangent(self, band):
        m = self.mesh
        s = _sp()
        _lib.call("petch_surface_rate_tangent", m.id, m.MT, m.MV, ctypes.byref(self.chem),
                  self.dOflux, self.drate, self.m_F.data_ptr(), self.dm_F.data_ptr(),
                  self.m_O.data_ptr(), self.dm_O.data_ptr(), self.y[0].data_ptr(),
                  self.dy[0].data_ptr(), self.y[1].data_ptr(), self.dy[1].data_ptr(),
                  self.y[2].data_ptr(), self.dy[2].data_ptr(), self.V.data_ptr(),
                  self.dV.data_ptr(), self.small[6:8].data_ptr(), s)
        nx, ny, nz = self.shape
        _lib.call("petch_extend_velocity_dual", m.id, m.MT, m.MV, self.phi.data_ptr(),
                  self.mask.data_ptr(), nx, ny, nz, self.dx, float(band), self.V.data_ptr(),
                  self.dV.data_ptr(), self.F.data_ptr(), self.dF.data_ptr(), 1,
                  self.active.data_ptr(), self.small[8:9].data_ptr(), self.ncell,
                  self.small[0:6].data_ptr(), s)

    def advect_tangent(self, dt_sub, nsub):
        nx, ny, nz = self.shape
        _lib.call("petch_advect_tangent", self.phi.data_ptr(), self.tmp.data_ptr(),
                  self.dphi.data_ptr(), self.dtmp.data_ptr(), self.F.data_ptr(),
                  self.dF.data_ptr(), self.mask_u8.data_ptr(), self.mask_phi.data_ptr(), nx, ny,
                  nz, float(1.0 / self.dx), float(dt_sub), int(nsub), _sp())

    def reinit_tangent(self, band_r):
        nx, ny, nz = self.shape
        n_iter = int(np.ceil(band_r / self.dx)) + 4
        _lib.call("petch_reinit_tangent", self.phi.data_ptr(), self.dphi.data_ptr(),
                  self.ua.data_ptr(), self.ub.data_ptr(), self.du_a.data_ptr(),
                  self.du_b.data_ptr(), nx, ny, nz, float(self.dx),
                  float(band_r + 4.0 * self.dx), float(band_r + self.dx), n_iter, _sp())


def run_etch_3d_tangent(theta, Lx, Ly, Lz, dx, trench_width, mask_th, sub_top, t_end=3.0,
                        n_steps=20, hole=True, par=None, flags=None, n_ion=30000, n_neu=30000,
                        seed_offset=0, max_tris=None):
    """run_etch_3d (FSM reinit, nearest-face extension, coverage-coupled SF6/O2 flux with
    faithful ions; Monte-Carlo or radiosity neutrals) at recipe theta, carrying d/dtheta.  Returns (phi, dphi[3], geo) as numpy
    float64 (phi: (nx, ny, nz); dphi: (3, nx, ny, nz)) plus timings (device seconds)."""
    par = apply_theta(dict(par or PAR), theta)
    flags = flags or DEFAULT_FLAGS
    if not (getattr(flags, "ion_reflection", False) and getattr(flags, "coverage_sticking", False)
            and getattr(flags, "chemistry", "langmuir") == "belen"):
        raise NotImplementedError("the recipe gradient follows the coverage-coupled SF6/O2 path "
                                  "with faithful ions (belen, ion_reflection, coverage_sticking)")
    transport = getattr(flags, "neutral_transport", "mc")
    if transport not in ("mc", "radiosity") or getattr(flags, "redeposition", False):
        raise NotImplementedError("the recipe gradient follows Monte-Carlo or radiosity neutrals "
                                  "without redeposition")
    if transport == "radiosity" and par.get('radiosity_solver', 'jacobi') == 'gmres':
        raise NotImplementedError("the recipe gradient follows the radiosity path's Jacobi solve")
    if getattr(flags, "floor_charge_throttle", False):
        raise NotImplementedError("the recipe gradient does not include the floor-charging throttle")
    if getattr(flags, "surface_charging", False) and float(par.get('charge_alpha', 0.0)) > 0.0:
        raise NotImplementedError("the recipe gradient does not include the electron-shadowing "
                                  "charge model")
    torch.cuda.init()
    geo = make_trench_3d(Lx, Ly, Lz, dx, trench_width, mask_th, sub_top, hole=hole, host=False)
    geo['mask_th'] = mask_th
    geo['mask_phi_dev'] = geo['phi_dev'].clone()
    dt = t_end / n_steps
    band = 4 * dx
    warm = getattr(flags, "warm_start_coverage", False)
    eng = TangentEngine(geo, par, flags, max_tris=max_tris)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    step = 0
    while step < n_steps:
        seed = step + seed_offset
        eng.small.zero_()
        eng.build_mesh()
        if transport == "radiosity":
            eng.flux_radiosity_tangent(eng.phi, n_ion, seed)
        else:
            eng.flux_tangent(n_ion, n_neu, seed, warm)
        eng.rate_extend_tangent(band)
        st = eng.sync_status()
        if st['mesh_err'] & (MESH_ERR_TRI_OVERFLOW | MESH_ERR_VERT_OVERFLOW | MESH_ERR_HASH_FULL):
            raise RuntimeError(f"mesh capacity {eng.MT} exceeded; pass a larger max_tris")
        if st['trace_err']:
            raise RuntimeError(f"step {step}: device traversal limit hit ({st['trace_err']})")
        vmx = st['vmax'] if st['F'] > 0 else 0.0
        Vmax = max(vmx if np.isfinite(vmx) else 0.0, 1e-6)
        nsub = max(1, min(int(np.ceil(Vmax * dt / (0.4 * dx))), 160))
        eng.advect_tangent(dt / nsub, nsub)
        eng.reinit_tangent(band + 2.0 * dx)
        eng.end_step(warm)
        step += 1
    e1.record()
    torch.cuda.synchronize()
    out_geo = dict(xs=geo['xs'], ys=geo['ys'], zs=geo['zs'], dx=dx, Lx=Lx, Ly=Ly, Lz=Lz,
                   sub_top=sub_top, trench_width=trench_width, hole=hole)
    return (eng.phi.double().cpu().numpy(), eng.dphi.double().cpu().numpy(), out_geo,
            e0.elapsed_time(e1) / 1e3)


def radial_profile(phi, geo, dphi=None, n_bins=32):
    """Zero-level-set depth profile of a hole (geo['hole'] true or absent) or a trench: per column
    (i, j), the depth below sub_top of the lowest zero crossing of the gas run connected to the top
    of the grid (linear interpolation between the last gas node and the solid node under it; the
    grid floor if the run reaches it), averaged over n_bins equal bins of the column's distance
    from the hole axis (out to min(Lx, Ly) / 2) or from the trench's mid-plane x = Lx / 2 (out to
    Lx / 2).  Returns (profile[n_bins], jac[n_bins, 3] or None); empty bins are NaN."""
    phi = np.asarray(phi, np.float64)
    dx = geo['dx']
    nx, ny, nz = phi.shape
    xs, ys = np.arange(nx) * dx, np.arange(ny) * dx
    cx, cy = geo['Lx'] / 2.0, geo['Ly'] / 2.0
    hole = geo.get('hole', True)
    rmax = min(geo['Lx'], geo['Ly']) / 2.0 if hole else geo['Lx'] / 2.0
    gas = phi < 0
    # lowest gas node of the top-connected run: cumulative "all gas from the top"
    run = np.flip(np.cumprod(np.flip(gas, axis=2), axis=2), axis=2).astype(bool)
    has = run[:, :, -1]
    kg = np.where(has, nz - run.sum(axis=2), -1)          # lowest gas index of the run
    prof = np.zeros(n_bins)
    cnt = np.zeros(n_bins)
    jac = np.zeros((n_bins, ND)) if dphi is not None else None
    X, Y = np.meshgrid(xs - cx, ys - cy, indexing="ij")
    R = np.hypot(X, Y) if hole else np.abs(X)
    b = np.floor(R / rmax * n_bins).astype(int)
    for i in range(nx):
        for j in range(ny):
            if not has[i, j] or b[i, j] >= n_bins:
                continue
            k = kg[i, j]
            if k <= 0:
                z, dz = 0.0, np.zeros(ND)
            else:
                pa, pb = phi[i, j, k - 1], phi[i, j, k]      # solid (>= 0), gas (< 0)
                den = pa - pb
                t = pa / den
                z = (k - 1 + t) * dx
                if dphi is not None:
                    da, db = dphi[:, i, j, k - 1], dphi[:, i, j, k]
                    dz = dx * (pa * db - pb * da) / den ** 2
            prof[b[i, j]] += geo['sub_top'] - z
            cnt[b[i, j]] += 1
            if dphi is not None:
                jac[b[i, j]] -= dz
    with np.errstate(invalid="ignore"):
        prof = np.where(cnt > 0, prof / np.maximum(cnt, 1), np.nan)
        if jac is not None:
            jac = np.where(cnt[:, None] > 0, jac / np.maximum(cnt, 1)[:, None], np.nan)
    return prof, jac


class EtchProfile(torch.autograd.Function):
    """profile = EtchProfile.apply(theta, cfg): the radial depth profile after cfg's run at
    recipe theta (a float64 tensor (Emean, O/F, rate_scale)); backward returns J^T grad with J
    the forward-mode Jacobian d profile / d theta of the same run.  cfg: keyword arguments of
    run_etch_3d_tangent (geometry, steps, rays, seed_offset, par, flags) plus n_bins."""

    @staticmethod
    def forward(ctx, theta, cfg):
        kw = dict(cfg)
        n_bins = kw.pop('n_bins', 32)
        phi, dphi, geo, _ = run_etch_3d_tangent(theta.detach().cpu().tolist(), **kw)
        prof, jac = radial_profile(phi, geo, dphi, n_bins)
        ctx.save_for_backward(torch.from_numpy(np.nan_to_num(jac)).to(theta))
        return torch.from_numpy(prof).to(theta)

    @staticmethod
    def backward(ctx, grad):
        (jac,) = ctx.saved_tensors
        return jac.t() @ torch.nan_to_num(grad), None


def profile_loss(theta, cfg, target):
    """MSE between the radial profile at theta and `target` over the bins both define."""
    prof = EtchProfile.apply(theta, cfg)
    t = torch.as_tensor(target).to(prof)
    ok = torch.isfinite(prof) & torch.isfinite(t)
    return ((prof[ok] - t[ok]) ** 2).mean()
