"""Batched inverse design: recipe gradients of many etch runs at once, and an Adam loop on them.

No reference counterpart (the reference has neither batching nor an end-to-end gradient).  Each
instance follows run_etch_3d_tangent (the forward-mode recipe gradient of the coverage-coupled
SF6/O2 loop, petch/threed.py:1643-1795 with faithful ions, warm-started coverage, nearest-face
extension and the FSM reinit); the instances advance together as BatchEngine's do:

    per instance: marching cubes + BVH, warm start of the coverage and its tangents (one
        nearest-face query per face)
    ions of ALL instances with energy tangents: one persistent launch (petch_trace_batch_tangent)
    per instance: ion normalisation + smoothing, the yields' tangents
    coverage fixed point: F and O neutrals of all instances with weight tangents, one launch;
        per instance normalisation + smoothing (+ tangents), Belen coverage update with duals
    per instance: surface rate with duals, velocity extension and its tangent (one nearest-face
        query per band cell)
    all instances: CFL substeps on the device and the dual advection (petch_batch_advect_tangent),
        the dual Eikonal reinit (petch_batch_reinit_tangent), the step counter
No host synchronisation inside a step, so each step is captured in a CUDA graph and replayed.
Instance b's rays draw the Philox streams of its own run_etch_3d_tangent(seed_offset = its
seed), so with deterministic tallies (petch_set_deterministic) the batched run equals the
per-instance runs bit for bit, gradients included.

The Adam loop (configs: 32 periodic trenches, per-instance recipes and targets) shards instances
over ranks when torch.distributed is initialised, with one all-gather of the per-instance losses
and recipes per iteration.
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib
from .adjoint import ND, apply_theta, radial_profile, run_etch_3d_tangent
from .batch import LANES, on_lanes
from .params import PAR
from .threed import (MESH_ERR_HASH_FULL, MESH_ERR_TRI_OVERFLOW, MESH_ERR_VERT_OVERFLOW, DeviceMesh,
                     FluxEngine, _sp, chem_params, default_capacity, ion_params, make_trench_3d,
                     mesh_scratch_bytes)

MAX_BATCH = 64


def trench_batch_specs(n=32, seed=0, dx=0.125, aspect=10.0, mask=1.0, Ly_cells=8, margin=2.0,
                       headroom=1.0):
    """The inverse-design batch: periodic trenches of width ~ U[1, 4] um with a 1 um mask, the
    substrate deep enough for aspect ratio `aspect` (sub_top = aspect * width + 1 um), x extent
    width + 2 margin, Ly = Ly_cells * dx (periodic along y); per instance ion energy log-uniform
    in [50, 500] eV, F / ion flux ratio log-uniform in [10, 1000], O / F ratio ~ U[0, 0.5] (the
    ragged forward batch's draws, seeded torch.Generator).  Returns (specs, theta0[n, 3]) with
    theta = (ion energy, O/F ratio, rate_scale = 1)."""
    g = torch.Generator().manual_seed(seed)
    u = torch.rand((n, 4), generator=g, dtype=torch.float64).numpy()
    specs, theta = [], []
    for k in range(n):
        w = 1.0 + 3.0 * u[k, 0]
        E = float(np.exp(np.log(50.0) + (np.log(500.0) - np.log(50.0)) * u[k, 1]))
        rF = float(np.exp(np.log(10.0) + (np.log(1000.0) - np.log(10.0)) * u[k, 2]))
        rO = 0.5 * u[k, 3]
        Lx = round((w + 2.0 * margin) / dx) * dx
        sub_top = round((aspect * w + 1.0) / dx) * dx
        Lz = sub_top + mask + headroom
        par = dict(Fflux=rF * PAR['ionFlux'], periodic_y=1)
        specs.append(dict(Lx=Lx, Ly=Ly_cells * dx, Lz=Lz, dx=dx, trench_width=w, mask_th=mask,
                          sub_top=sub_top, hole=False, par=par))
        theta.append((E, rO, 1.0))
    return specs, np.array(theta)


class _TInst:
    """Device state of one instance (the TangentEngine buffers, double-buffered warm start)."""

    def __init__(self, spec, flags, MT):
        self.spec = spec
        self.base_par = dict(PAR, **spec.get('par', {}))
        geo = make_trench_3d(spec['Lx'], spec['Ly'], spec['Lz'], spec['dx'],
                             spec['trench_width'], spec['mask_th'], spec['sub_top'],
                             hole=spec.get('hole', True), host=False)
        geo['mask_th'] = spec['mask_th']
        self.geo = geo
        self.phi = geo['phi_dev']
        self.phi0 = self.phi.clone()
        self.mask = geo['mask_dev']
        self.mask_u8 = self.mask.to(torch.uint8).contiguous()
        self.mask_phi = self.phi.clone()
        self.shape = tuple(self.phi.shape)
        self.ncell = int(np.prod(self.shape))
        self.dx = float(spec['dx'])
        dev = dict(device="cuda", dtype=torch.float32)
        self.tmp = torch.empty_like(self.phi)
        self.ua = torch.empty_like(self.phi)
        self.ub = torch.empty_like(self.phi)
        self.F = torch.zeros_like(self.phi)
        self.active = torch.empty(self.ncell, dtype=torch.int32, device="cuda")
        self.dphi = torch.zeros((ND,) + self.shape, **dev)
        self.dtmp = torch.empty_like(self.dphi)
        self.dF = torch.zeros((ND, self.ncell), **dev)
        self.du_a = torch.empty((ND, self.ncell), **dev)
        self.du_b = torch.empty((ND, self.ncell), **dev)
        self.sub = torch.zeros(2, dtype=torch.int32, device="cuda")
        self.fe = FluxEngine(geo, dict(self.base_par), flags, MT)
        self.meshes = (self.fe.mesh, DeviceMesh(MT))
        self.bares = (self.fe.bare, torch.empty(MT, device="cuda"))
        self.dbares = (torch.zeros((ND, MT), **dev), torch.zeros((ND, MT), **dev))
        self.dtal = torch.empty((ND, MT), **dev)
        self.dtal_in = torch.zeros((ND, MT), **dev)
        self.dy = torch.zeros((3, ND, MT), **dev)
        self.dm_F = torch.zeros((ND, MT), **dev)
        self.dm_O = torch.zeros((ND, MT), **dev)
        self.dflux = torch.empty((ND, MT), **dev)
        self.dflux_o = torch.empty((ND, MT), **dev)      # the O species of a paired round
        self.dV = torch.zeros((ND, MT), **dev)
        self.ttmp = torch.empty((2, MT), **dev)
        self.scratch = torch.empty(mesh_scratch_bytes(self.shape, MT), dtype=torch.uint8,
                                   device="cuda")
        self.set_theta((float(self.base_par['Emean']),
                        float(self.base_par['Oflux'] / self.base_par['Fflux']),
                        float(self.base_par['rate_scale'])))

    def set_theta(self, theta):
        self.theta = tuple(float(t) for t in theta)
        par = apply_theta(self.base_par, self.theta)
        fe = self.fe
        fe.par = par
        fe.chem = chem_params(par, fe.flags)
        fe.ionp = ion_params(par)
        self.dOflux = (ctypes.c_double * ND)(0.0, float(par['Fflux']), 0.0)
        self.drate = (ctypes.c_double * ND)(0.0, 0.0, 1.0)

    def reset(self):
        self.phi.copy_(self.phi0)
        self.dphi.zero_()


class BatchTangentEngine:
    """B <= 64 tangent-carrying etch runs in lock step (see the module docstring).

    specs: run_etch_3d geometries + 'par' overrides (trench_batch_specs); every instance shares
    the flags, ray counts, t_end, n_steps and dx; seed_offset: each instance's Philox seed offset
    (as run_etch_3d_tangent's)."""

    def __init__(self, specs, flags, n_ion=1 << 16, n_neu=1 << 16, t_end=0.5, n_steps=20,
                 max_tris=None, seed_offset=0):
        B = len(specs)
        if not 1 <= B <= MAX_BATCH:
            raise ValueError(f"a batch holds 1..{MAX_BATCH} instances")
        if not (getattr(flags, "ion_reflection", False) and getattr(flags, "coverage_sticking", False)
                and getattr(flags, "chemistry", "langmuir") == "belen"):
            raise NotImplementedError("the batched gradient follows the coverage-coupled SF6/O2 "
                                      "path with faithful ions (belen, ion_reflection, "
                                      "coverage_sticking)")
        for flag in ("redeposition", "floor_charge_throttle"):
            if getattr(flags, flag, False):
                raise NotImplementedError(f"{flag} is not part of the batched gradient")
        if getattr(flags, "neutral_transport", "mc") != "mc":
            raise NotImplementedError("the batched gradient follows Monte-Carlo neutrals")
        alphas = [float(dict(PAR, **sp.get('par', {})).get('charge_alpha', 0.0)) for sp in specs]
        if getattr(flags, "surface_charging", False) and max(alphas) > 0.0:
            raise NotImplementedError("the electron-shadowing charge model is not part of the "
                                      "batched gradient")
        dxs = {float(s['dx']) for s in specs}
        if len(dxs) != 1:
            raise ValueError("all instances need the same dx")
        torch.cuda.init()
        _lib.call("petch_prepare_device")
        from .levelset import grid_shape
        shapes = [grid_shape(s['Lx'], s['Ly'], s['Lz'], s['dx']) for s in specs]
        self.MT = int(max_tris or max(default_capacity(sh) for sh in shapes))
        self.flags, self.n_ion, self.n_neu = flags, int(n_ion), int(n_neu)
        self.warm = bool(getattr(flags, "warm_start_coverage", False))
        self.t_end, self.n_steps, self.seed_offset = float(t_end), int(n_steps), int(seed_offset)
        self.dt = self.t_end / self.n_steps
        self.dx = dxs.pop()
        self.band = 4 * self.dx
        self.inst = [_TInst(s, flags, self.MT) for s in specs]
        p0 = self.inst[0].base_par
        for x in self.inst[1:]:
            for k in ('betaE', 'betaO', 'flux_smooth', 'flux_smooth_alpha'):
                if x.base_par.get(k, PAR.get(k)) != p0.get(k, PAR.get(k)):
                    raise ValueError(f"PAR['{k}'] must be the same for every instance")
        self.betaE, self.betaO = float(p0.get('betaE', 0.7)), float(p0.get('betaO', 1.0))
        self.n_smooth = int(p0.get('flux_smooth', 1))
        self.alpha = float(p0.get('flux_smooth_alpha', 1.0))
        self.step_dev = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.work = torch.zeros(8, dtype=torch.int32, device="cuda")
        self.lanes = [torch.cuda.Stream() for _ in range(min(LANES, len(self.inst)))]
        self.graphs = None
        self.steps_done = 0

    # ---- recipes ----
    def set_thetas(self, thetas):
        """Per-instance recipes theta = (ion energy, O/F ratio, rate_scale); the captured graphs
        hold the recipe constants, so they are re-captured on the next run."""
        for x, th in zip(self.inst, thetas):
            x.set_theta(th)
        self.graphs = None

    def reset(self):
        """Back to the initial level sets (zero tangents) at step 0."""
        for x in self.inst:
            x.reset()
        self.step_dev.zero_()
        self.work.zero_()
        self.steps_done = 0

    # ---- one step (launches only; capturable) ----
    def _items(self, ion, cur):
        B = len(self.inst)
        items = (_lib.BatchItem * B)()
        tans = (_lib.BatchTangent * B)()
        for b, x in enumerate(self.inst):
            it = items[b]
            it.mesh = x.meshes[cur].id
            it.dom = x.fe.dom
            it.ion = x.fe.ionp
            it.bare = x.bares[cur].data_ptr()
            it.out = (x.fe.tal4 if ion else x.fe.flux).data_ptr()
            it.ang = x.fe.ang.data_ptr() if ion else None
            it.n_rays = self.n_ion if ion else self.n_neu
            it.seed = self.seed_offset & 0xffffffff
            tans[b].dout = (x.dtal if ion else x.dflux).data_ptr()
            tans[b].dbare = None if ion else x.dbares[cur].data_ptr()
        return items, tans

    def _grids(self, cur):
        B = len(self.inst)
        g = (_lib.BatchGrid * B)()
        t = (_lib.BatchTangentGrid * B)()
        for b, x in enumerate(self.inst):
            q = g[b]
            q.phi, q.tmp, q.ua, q.ub = (x.phi.data_ptr(), x.tmp.data_ptr(), x.ua.data_ptr(),
                                        x.ub.data_ptr())
            q.F, q.mask_phi = x.F.data_ptr(), x.mask_phi.data_ptr()
            q.mask_idx, q.n_mask = None, 0
            q.active, q.n_active = x.active.data_ptr(), x.fe.small[8:9].data_ptr()
            q.max_active = x.ncell
            q.nx, q.ny, q.nz = x.shape
            q.dx, q.dt = self.dx, self.dt
            q.stats = x.fe.small[6:8].data_ptr()
            q.hdr = x.meshes[cur].hdr.data_ptr()
            q.sub = x.sub.data_ptr()
            d = t[b]
            d.dphi, d.dtmp, d.dF = x.dphi.data_ptr(), x.dtmp.data_ptr(), x.dF.data_ptr()
            d.mask, d.du_a, d.du_b = x.mask_u8.data_ptr(), x.du_a.data_ptr(), x.du_b.data_ptr()
        return g, t

    def _each(self, fn):
        on_lanes(self.lanes, self.inst, fn)

    def _step(self, cold, cur):
        s = _sp()
        prev = 1 - cur
        B = len(self.inst)
        MT = self.MT
        MV = self.inst[0].meshes[cur].MV
        n_fp = int(self.inst[0].base_par.get('n_fp', 4 if cold else 1))

        def surface(x):
            x.fe.small.zero_()
            x.meshes[cur].build(x.phi, x.dx, x.geo, x.scratch)
            if not cold:
                pm, cm = x.meshes[prev], x.meshes[cur]
                _lib.call("petch_warmstart_dual", pm.id, pm.MT, pm.MV, x.bares[prev].data_ptr(),
                          x.dbares[prev].data_ptr(), cm.id, cm.MT, cm.MV,
                          x.bares[cur].data_ptr(), x.dbares[cur].data_ptr(),
                          x.fe.small.data_ptr(), _sp())
            else:
                x.bares[cur].fill_(1.0)
                x.dbares[cur].zero_()

        def ion_post(x):
            m, fe = x.meshes[cur], x.fe
            norm = float(x.geo['Lx'] * x.geo['Ly'] / self.n_ion)
            _lib.call("petch_ion_post", m.id, m.MT, m.MV, fe.tal4.data_ptr(), fe.ang.data_ptr(),
                      norm, self.n_smooth, self.alpha, fe.y[0].data_ptr(), fe.y[1].data_ptr(),
                      fe.y[2].data_ptr(), fe.m_i.data_ptr(), fe.cos_i.data_ptr(),
                      fe.tmp5.data_ptr(), _sp())
            for q in range(3):                  # d y_q: direction 0 only (ion energy)
                x.dtal_in[0].copy_(x.dtal[q])
                _lib.call("petch_norm_smooth_tangent", m.id, m.MT, m.MV, x.dtal_in.data_ptr(),
                          x.dtal_in.data_ptr(), norm, 0.0, 0.0, 0, self.n_smooth, self.alpha, 1,
                          x.dy[q].data_ptr(), x.ttmp[0].data_ptr(), x.ttmp[1].data_ptr(), _sp())

        def coverage(x):
            m, fe = x.meshes[cur], x.fe
            norm = float(x.geo['Lx'] * x.geo['Ly'] / self.n_neu)
            for fl, dfl, out, dout in ((fe.flux, x.dflux, fe.m_F, x.dm_F),
                                       (fe.tmp5[2 * MT:3 * MT], x.dflux_o, fe.m_O, x.dm_O)):
                _lib.call("petch_norm_smooth", m.id, m.MT, m.MV, fl.data_ptr(), norm, 0.0,
                          8.0, 1, self.n_smooth, self.alpha, out.data_ptr(),
                          fe.tmp5.data_ptr(), fe.tmp5[MT:].data_ptr(), _sp())
                _lib.call("petch_norm_smooth_tangent", m.id, m.MT, m.MV, fl.data_ptr(),
                          dfl.data_ptr(), norm, 0.0, 8.0, 1, self.n_smooth, self.alpha, 0,
                          dout.data_ptr(), x.ttmp[0].data_ptr(), x.ttmp[1].data_ptr(), _sp())
            _lib.call("petch_belen_bare_tangent", m.id, m.MT, m.MV, ctypes.byref(fe.chem),
                      x.dOflux, fe.m_F.data_ptr(), x.dm_F.data_ptr(), fe.m_O.data_ptr(),
                      x.dm_O.data_ptr(), fe.y[1].data_ptr(), x.dy[1].data_ptr(),
                      fe.y[2].data_ptr(), x.dy[2].data_ptr(), x.bares[cur].data_ptr(),
                      x.dbares[cur].data_ptr(), _sp())

        def rate_extend(x):
            m, fe = x.meshes[cur], x.fe
            _lib.call("petch_surface_rate_tangent", m.id, m.MT, m.MV, ctypes.byref(fe.chem),
                      x.dOflux, x.drate, fe.m_F.data_ptr(), x.dm_F.data_ptr(), fe.m_O.data_ptr(),
                      x.dm_O.data_ptr(), fe.y[0].data_ptr(), x.dy[0].data_ptr(),
                      fe.y[1].data_ptr(), x.dy[1].data_ptr(), fe.y[2].data_ptr(),
                      x.dy[2].data_ptr(), fe.V.data_ptr(), x.dV.data_ptr(),
                      fe.small[6:8].data_ptr(), _sp())
            nx, ny, nz = x.shape
            _lib.call("petch_extend_velocity_dual", m.id, m.MT, m.MV, x.phi.data_ptr(),
                      x.mask.data_ptr(), nx, ny, nz, x.dx, float(self.band), fe.V.data_ptr(),
                      x.dV.data_ptr(), x.F.data_ptr(), x.dF.data_ptr(), 1, x.active.data_ptr(),
                      fe.small[8:9].data_ptr(), x.ncell, fe.small[0:6].data_ptr(), _sp())

        self._each(surface)
        items, tans = self._items(True, cur)
        _lib.call("petch_trace_batch_tangent", 0, items, tans, B, MT, MV, 0.0,
                  self.step_dev.data_ptr(), 9, 1, self.work.data_ptr(), s)
        self._each(ion_post)
        for it in range(n_fp):
            # both species of the round with their tangents in one launch: F (betaE, +2+2it) into
            # fe.flux / x.dflux, O (betaO, +3+2it) into fe.tmp5's third slice / x.dflux_o
            items, tans = self._items(False, cur)
            tans_o = (_lib.BatchTangent * B)()
            for b, x in enumerate(self.inst):
                items[b].ang = x.fe.tmp5[2 * MT:3 * MT].data_ptr()
                tans_o[b].dout = x.dflux_o.data_ptr()
            _lib.call("petch_trace_batch_pair_tangent", items, tans, tans_o, B, MT, MV,
                      self.betaE, self.betaO, self.step_dev.data_ptr(), 9, 2 + 2 * it, 3 + 2 * it,
                      self.work.data_ptr(), s)
            self._each(coverage)
        self._each(rate_extend)
        grids, tg = self._grids(cur)
        _lib.call("petch_batch_advect_tangent", grids, tg, B, s)
        _lib.call("petch_batch_reinit_tangent", grids, tg, B, float(self.band + 2.0 * self.dx), s)
        _lib.call("petch_batch_step_advance", self.step_dev.data_ptr(), s)

    # ---- capture and run ----
    def capture(self):
        """Capture the cold first step and the two warm steps into CUDA graphs; returns the
        kernel launches per step."""
        graphs, launches = {}, {}
        keys = (("cold", True, 0), ("warm1", False, 1), ("warm0", False, 0))
        if not self.warm:
            keys = (("cold", True, 0), ("cold1", True, 1))
        for key, cold, cur in keys:
            g = torch.cuda.CUDAGraph()
            n0 = _lib.launch_count()
            with torch.cuda.graph(g):
                self._step(cold, cur)
            launches[key] = _lib.launch_count() - n0
            graphs[key] = g
        torch.cuda.synchronize()
        self.graphs = graphs
        self.launches_per_step = launches
        return launches

    def step(self, use_graph=True):
        k = self.steps_done
        cold = k == 0 or not self.warm
        cur = k % 2
        if use_graph:
            if self.graphs is None:
                self.capture()
            key = ("cold" if k == 0 else f"warm{cur}") if self.warm else ("cold" if cur == 0 else "cold1")
            self.graphs[key].replay()
        else:
            self._step(cold, cur)
        self.steps_done += 1

    def run(self, use_graph=True):
        """Reset, then the whole schedule; returns device seconds (events around the steps)."""
        self.reset()
        if use_graph and self.graphs is None:
            self.capture()
            self.reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(self.n_steps):
            self.step(use_graph)
        e1.record()
        torch.cuda.synchronize()
        self.check()
        return e0.elapsed_time(e1) / 1e3

    def check(self):
        err = int(self.work[1].item())
        if err:
            raise RuntimeError(f"batched tangent trace: device error bits {err}")
        for b, x in enumerate(self.inst):
            for m in x.meshes:
                e = int(m.hdr[3].item())
                if e & (MESH_ERR_TRI_OVERFLOW | MESH_ERR_VERT_OVERFLOW | MESH_ERR_HASH_FULL):
                    raise RuntimeError(f"instance {b}: mesh capacity {self.MT} exceeded "
                                       f"(error bits {e}); pass a larger max_tris")
            if int(x.fe.small[1].item()):
                raise RuntimeError(f"instance {b}: device error bits {int(x.fe.small[1].item())}")

    def results(self):
        """[(phi, dphi, geo)] as numpy float64 per instance (geo: what radial_profile reads)."""
        out = []
        for x in self.inst:
            s = x.spec
            geo = dict(dx=s['dx'], Lx=s['Lx'], Ly=s['Ly'], Lz=s['Lz'], sub_top=s['sub_top'],
                       trench_width=s['trench_width'], hole=s.get('hole', True))
            out.append((x.phi.double().cpu().numpy(), x.dphi.double().cpu().numpy(), geo))
        return out


# ---------------------------------------------------------------------------------------------
# the inverse-design loop
# ---------------------------------------------------------------------------------------------
def loss_and_grad(prof, jac, target):
    """MSE over the bins both profiles define, and its gradient J^T (2 / n)(prof - target)."""
    ok = np.isfinite(prof) & np.isfinite(target)
    if not ok.any():
        return float("nan"), np.zeros(ND)
    r = prof[ok] - target[ok]
    J = np.nan_to_num(jac[ok])
    return float(np.mean(r * r)), 2.0 / ok.sum() * (J.T @ r)


class Adam:
    """Adam on theta / theta_scale (per instance, per component)."""

    def __init__(self, theta0, lr=0.05, b1=0.9, b2=0.999, eps=1e-8):
        self.scale = np.abs(np.asarray(theta0, float)) + 1e-12
        self.u = np.asarray(theta0, float) / self.scale
        self.m = np.zeros_like(self.u)
        self.v = np.zeros_like(self.u)
        self.t = 0
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps

    @property
    def theta(self):
        return self.u * self.scale

    def step(self, grad_theta):
        g = np.asarray(grad_theta, float) * self.scale
        self.t += 1
        self.m = self.b1 * self.m + (1 - self.b1) * g
        self.v = self.b2 * self.v + (1 - self.b2) * g * g
        mh = self.m / (1 - self.b1 ** self.t)
        vh = self.v / (1 - self.b2 ** self.t)
        self.u = self.u - self.lr * mh / (np.sqrt(vh) + self.eps)
        # keep the recipe physical: energy above 1 eV, ratios and rate scale non-negative
        self.u = np.maximum(self.u, np.array([1.0, 0.0, 0.0]) / self.scale)


def shard(B, world, rank):
    """Instances of rank `rank`: b = rank, rank + world, ..."""
    return list(range(rank, B, world))


def gather_rows(rows, B, world, rank, group=None):
    """All-gather per-instance rows (float64 [len(shard), k]) into [B, k] in instance order."""
    rows = np.asarray(rows, np.float64)
    if world == 1:
        return rows
    import torch.distributed as dist
    k = rows.shape[1]
    n_max = (B + world - 1) // world
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    buf = torch.zeros((n_max, k), dtype=torch.float64, device=dev)
    buf[:len(rows)] = torch.from_numpy(rows).to(dev)
    out = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    full = np.zeros((B, k))
    for r in range(world):
        idx = shard(B, world, r)
        full[idx] = out[r][:len(idx)].cpu().numpy()
    return full


def batched_inverse_design(specs, theta0, targets, flags, n_iter=50, lr=0.05, n_bins=32,
                           n_ion=1 << 16, n_neu=1 << 16, t_end=0.5, n_steps=20, max_tris=None,
                           seed_offset=0, world=1, rank=0, group=None, callback=None):
    """Adam on every instance's recipe against its target profile, all instances of this rank's
    shard advanced by one BatchTangentEngine per iteration.  Returns dict(theta [B, 3],
    loss [n_iter, B], seconds, forward_seconds) with the rows of all ranks gathered."""
    B = len(specs)
    mine = shard(B, world, rank)
    eng = BatchTangentEngine([specs[b] for b in mine], flags, n_ion, n_neu, t_end, n_steps,
                             max_tris, seed_offset)
    opt = Adam(np.asarray(theta0)[mine], lr=lr)
    losses = []
    t_fwd = 0.0
    t0 = time.time()
    for it in range(n_iter):
        eng.set_thetas(opt.theta)
        t_fwd += eng.run()
        rows, grads = [], []
        for k, (phi, dphi, geo) in enumerate(eng.results()):
            prof, jac = radial_profile(phi, geo, dphi, n_bins)
            L, g = loss_and_grad(prof, jac, targets[mine[k]])
            rows.append([L])
            grads.append(g)
        opt.step(np.array(grads))
        losses.append(gather_rows(rows, B, world, rank, group)[:, 0])
        if callback:
            callback(it, losses[-1])
    theta = gather_rows(opt.theta, B, world, rank, group)
    return dict(theta=theta, loss=np.array(losses), seconds=time.time() - t0,
                forward_seconds=t_fwd)


def plain_inverse_design(spec, theta0, target, flags, n_iter=50, lr=0.05, n_bins=32,
                         n_ion=1 << 16, n_neu=1 << 16, t_end=0.5, n_steps=20, max_tris=None,
                         seed_offset=0):
    """The same loop for one instance with run_etch_3d_tangent (the per-instance baseline)."""
    opt = Adam(np.asarray(theta0)[None, :], lr=lr)
    losses, grads = [], []
    base = dict(PAR, **spec.get('par', {}))
    geo_kw = {k: spec[k] for k in ('Lx', 'Ly', 'Lz', 'dx', 'trench_width', 'mask_th', 'sub_top')}
    t0 = time.time()
    for it in range(n_iter):
        phi, dphi, geo, _ = run_etch_3d_tangent(opt.theta[0], **geo_kw, t_end=t_end,
                                                n_steps=n_steps, hole=spec.get('hole', True),
                                                par=base, flags=flags, n_ion=n_ion, n_neu=n_neu,
                                                seed_offset=seed_offset, max_tris=max_tris)
        prof, jac = radial_profile(phi, geo, dphi, n_bins)
        L, g = loss_and_grad(prof, jac, target)
        losses.append(L)
        grads.append(g)
        opt.step(g[None, :])
    return dict(theta=opt.theta[0], loss=np.array(losses), grads=np.array(grads),
                seconds=time.time() - t0)


def target_profiles(specs, theta_t, flags, n_bins=32, n_ion=1 << 16, n_neu=1 << 16, t_end=0.5,
                    n_steps=20, max_tris=None, seed_offset=1):
    """Per-instance target profiles from the same simulator at recipes theta_t (one batched
    run, seed offset 1)."""
    eng = BatchTangentEngine(specs, flags, n_ion, n_neu, t_end, n_steps, max_tris, seed_offset)
    eng.set_thetas(theta_t)
    eng.run()
    return np.array([radial_profile(phi, geo, None, n_bins)[0]
                     for phi, _, geo in eng.results()])
