"""Batched forward: many independent etch runs (features x recipes, grids of different sizes)
advanced together, each step captured in a CUDA graph.

No single reference counterpart: the reference runs one feature per run_etch_3d call
(petch/threed.py:1643-1795).  Every instance here follows that loop with the coverage-coupled
SF6/O2 flux (mc_flux_3d_coupled, threed.py:740-905, faithful ions, warm-started coverage) and the
FSM reinit, with the instance's own geometry and PAR overrides (ion energy, flux ratios, ...).

One step, all on one stream, no host synchronisation:
    per instance: marching cubes + BVH into the instance's mesh buffer (all buffers share one
        capacity, so the batched tracer addresses any of them with one layout), warm start
    ions of ALL instances: one persistent launch, one global ray queue (petch_trace_batch)
    per instance: ion normalisation + smoothing
    coverage fixed point: F and O neutrals of all instances, one launch each; per instance
        normalisation + smoothing and the Belen coverage update
    per instance: surface rate, velocity extension into the band
    all instances: CFL substep counts on the device and the narrow-band advection
        (petch_batch_advect), the Eikonal reinit (petch_batch_reinit), the step counter
Ray r of instance b draws the Philox stream it would draw in its own run_etch_3d with
seed_offset = the instance's seed, so a batched run follows the per-instance runs' paths (up to
the summation order of float atomics).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .params import DEFAULT_FLAGS, PAR
from .threed import (MESH_ERR_HASH_FULL, MESH_ERR_TRI_OVERFLOW, MESH_ERR_VERT_OVERFLOW, DeviceMesh,
                     FluxEngine, _depth3d, _sp, default_capacity, make_trench_3d,
                     mesh_scratch_bytes)

MAX_BATCH = 64
LANES = 8          # side streams for the per-instance kernels of a batched step


def on_lanes(lanes, insts, fn):
    """fn(x) for every instance, instance b on side stream b % len(lanes), forked from and joined
    back into the current stream: the small per-instance kernels of different instances overlap
    (parallel branches of a captured step graph).  Each instance's chain must touch only its own
    buffers."""
    main = torch.cuda.current_stream()
    for ln in lanes:
        ln.wait_stream(main)
    for b, x in enumerate(insts):
        with torch.cuda.stream(lanes[b % len(lanes)]):
            fn(x)
    for ln in lanes:
        main.wait_stream(ln)


class _Instance:
    """Device state of one instance."""

    def __init__(self, spec, flags, MT):
        par = dict(PAR, **spec.get('par', {}))
        geo = make_trench_3d(spec['Lx'], spec['Ly'], spec['Lz'], spec['dx'],
                             spec['trench_width'], spec['mask_th'], spec['sub_top'],
                             hole=spec.get('hole', True), host=False)
        geo['mask_th'] = spec['mask_th']
        self.spec, self.par, self.geo = spec, par, geo
        self.phi = geo['phi_dev']
        self.mask = geo['mask_dev']
        self.mask_phi = self.phi.clone()
        self.shape = tuple(self.phi.shape)
        self.ncell = int(np.prod(self.shape))
        self.dx = float(spec['dx'])
        self.tmp = torch.empty_like(self.phi)
        self.ua = torch.empty_like(self.phi)
        self.ub = torch.empty_like(self.phi)
        self.F = torch.zeros_like(self.phi)
        self.mask_idx = torch.nonzero(self.mask.view(-1)).view(-1).to(torch.int32)
        self.active = torch.empty(self.ncell, dtype=torch.int32, device="cuda")
        self.fe = FluxEngine(geo, par, flags, MT)
        self.meshes = (self.fe.mesh, DeviceMesh(MT))
        self.bares = (self.fe.bare, torch.empty(MT, device="cuda"))
        self.scratch = torch.empty(mesh_scratch_bytes(self.shape, MT), dtype=torch.uint8,
                                   device="cuda")
        self.sub = torch.zeros(2, dtype=torch.int32, device="cuda")


class BatchEngine:
    """B <= 64 etch runs advanced in lock step.

    specs: list of dicts with the run_etch_3d geometry (Lx, Ly, Lz, dx, trench_width, mask_th,
    sub_top, hole) and 'par' (PAR overrides); all instances share flags, ray counts, t_end,
    n_steps and dx.  seed_offset: the Philox seed offset of every instance (as run_etch_3d's)."""

    def __init__(self, specs, flags=None, n_ion=1 << 20, n_neu=1 << 20, t_end=3.0, n_steps=30,
                 max_tris=None, seed_offset=0):
        flags = flags or DEFAULT_FLAGS
        B = len(specs)
        if not 1 <= B <= MAX_BATCH:
            raise ValueError(f"a batch holds 1..{MAX_BATCH} instances")
        if not (getattr(flags, "ion_reflection", False) and getattr(flags, "coverage_sticking", False)
                and getattr(flags, "chemistry", "langmuir") == "belen"):
            raise NotImplementedError("the batched step runs the coverage-coupled SF6/O2 path with "
                                      "faithful ions (belen, ion_reflection, coverage_sticking)")
        for flag in ("redeposition", "floor_charge_throttle"):
            if getattr(flags, flag, False):
                raise NotImplementedError(f"{flag} is not part of the batched step")
        if getattr(flags, "neutral_transport", "mc") != "mc":
            raise NotImplementedError("the batched step runs Monte-Carlo neutrals")
        alphas = [float(dict(PAR, **sp.get('par', {})).get('charge_alpha', 0.0)) for sp in specs]
        if getattr(flags, "surface_charging", False) and max(alphas) > 0.0:
            raise NotImplementedError("the electron-shadowing charge model is not part of the "
                                      "batched step")
        dxs = {float(s['dx']) for s in specs}
        if len(dxs) != 1:
            raise ValueError("all instances need the same dx")
        torch.cuda.init()
        _lib.call("petch_prepare_device")
        from .levelset import grid_shape
        shapes = [grid_shape(s['Lx'], s['Ly'], s['Lz'], s['dx']) for s in specs]
        self.MT = int(max_tris or max(default_capacity(sh) for sh in shapes))
        self.flags, self.n_ion, self.n_neu = flags, int(n_ion), int(n_neu)
        self.t_end, self.n_steps, self.seed_offset = float(t_end), int(n_steps), int(seed_offset)
        self.dt = self.t_end / self.n_steps
        self.dx = dxs.pop()
        self.band = 4 * self.dx
        self.inst = [_Instance(s, flags, self.MT) for s in specs]
        p0 = self.inst[0].par
        for x in self.inst[1:]:
            for k in ('betaE', 'betaO', 'flux_smooth', 'flux_smooth_alpha'):
                if x.par.get(k, PAR.get(k)) != p0.get(k, PAR.get(k)):
                    raise ValueError(f"PAR['{k}'] must be the same for every instance")
        self.betaE, self.betaO = float(p0.get('betaE', 0.7)), float(p0.get('betaO', 1.0))
        self.n_smooth = int(p0.get('flux_smooth', 1))
        self.alpha = float(p0.get('flux_smooth_alpha', 1.0))
        self.step_dev = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.work = torch.zeros(8, dtype=torch.int32, device="cuda")
        self.lanes = [torch.cuda.Stream() for _ in range(min(LANES, B))]
        self.graphs = None
        self.steps_done = 0
        self.depth_history = [[] for _ in self.inst]

    # ---- one step (launches only; capturable) ----
    def _items(self, kind, cur):
        B = len(self.inst)
        items = (_lib.BatchItem * B)()
        for b, x in enumerate(self.inst):
            it = items[b]
            it.mesh = x.meshes[cur].id
            it.dom = x.fe.dom
            it.ion = x.fe.ionp
            it.bare = x.bares[cur].data_ptr()
            it.out = (x.fe.tal4 if kind == 0 else x.fe.flux).data_ptr()
            it.ang = x.fe.ang.data_ptr() if kind == 0 else None
            it.n_rays = self.n_ion if kind == 0 else self.n_neu
            it.seed = self.seed_offset & 0xffffffff
        return items

    def _grids(self, cur):
        B = len(self.inst)
        g = (_lib.BatchGrid * B)()
        for b, x in enumerate(self.inst):
            t = g[b]
            t.phi, t.tmp, t.ua, t.ub = (x.phi.data_ptr(), x.tmp.data_ptr(), x.ua.data_ptr(),
                                        x.ub.data_ptr())
            t.F, t.mask_phi = x.F.data_ptr(), x.mask_phi.data_ptr()
            t.mask_idx, t.n_mask = x.mask_idx.data_ptr(), int(x.mask_idx.numel())
            t.active, t.n_active = x.active.data_ptr(), x.fe.small[8:9].data_ptr()
            t.max_active = x.ncell
            t.nx, t.ny, t.nz = x.shape
            t.dx, t.dt = self.dx, self.dt
            t.stats = x.fe.small[6:8].data_ptr()
            t.hdr = x.meshes[cur].hdr.data_ptr()
            t.sub = x.sub.data_ptr()
        return g

    def _each(self, fn):
        on_lanes(self.lanes, self.inst, fn)

    def _step(self, cold, cur):
        s = _sp()
        prev = 1 - cur
        MT = self.MT
        B = len(self.inst)
        MV = self.inst[0].meshes[cur].MV
        n_fp = int(self.inst[0].par.get('n_fp', 4 if cold else 1))

        def surface(x):
            x.fe.small.zero_()
            x.meshes[cur].build(x.phi, x.dx, x.geo, x.scratch)
            if not cold:
                pm, cm = x.meshes[prev], x.meshes[cur]
                _lib.call("petch_warmstart", pm.id, pm.MT, pm.MV, x.bares[prev].data_ptr(), cm.id,
                          cm.MT, cm.MV, x.bares[cur].data_ptr(), x.fe.small.data_ptr(), _sp())
            else:
                x.bares[cur].fill_(1.0)

        def ion_post(x):
            m, fe = x.meshes[cur], x.fe
            A_src = float(x.geo['Lx'] * x.geo['Ly'])
            _lib.call("petch_ion_post", m.id, m.MT, m.MV, fe.tal4.data_ptr(), fe.ang.data_ptr(),
                      float(A_src / self.n_ion), self.n_smooth, self.alpha, fe.y[0].data_ptr(),
                      fe.y[1].data_ptr(), fe.y[2].data_ptr(), fe.m_i.data_ptr(),
                      fe.cos_i.data_ptr(), fe.tmp5.data_ptr(), _sp())

        def coverage(x):
            m, fe = x.meshes[cur], x.fe
            A_src = float(x.geo['Lx'] * x.geo['Ly'])
            for fl, out in ((fe.flux, fe.m_F), (fe.tmp5[2 * MT:3 * MT], fe.m_O)):
                _lib.call("petch_norm_smooth", m.id, m.MT, m.MV, fl.data_ptr(),
                          float(A_src / self.n_neu), 0.0, 8.0, 1, self.n_smooth, self.alpha,
                          out.data_ptr(), fe.tmp5.data_ptr(), fe.tmp5[m.MT:].data_ptr(), _sp())
            _lib.call("petch_belen_bare", m.id, m.MT, m.MV, ctypes.byref(fe.chem),
                      fe.m_i.data_ptr(), fe.m_F.data_ptr(), fe.m_O.data_ptr(),
                      fe.cos_i.data_ptr(), fe.y[1].data_ptr(), fe.y[2].data_ptr(),
                      x.bares[cur].data_ptr(), _sp())

        def rate_extend(x):
            m, fe = x.meshes[cur], x.fe
            _lib.call("petch_surface_rate", m.id, m.MT, m.MV, ctypes.byref(fe.chem),
                      fe.m_i.data_ptr(), fe.m_F.data_ptr(), fe.m_O.data_ptr(), fe.cos_i.data_ptr(),
                      fe.y[0].data_ptr(), fe.y[1].data_ptr(), fe.y[2].data_ptr(), fe.V.data_ptr(),
                      fe.small[6:8].data_ptr(), _sp())
            nx, ny, nz = x.shape
            _lib.call("petch_extend_velocity", m.id, m.MT, m.MV, x.phi.data_ptr(),
                      x.mask.data_ptr(), nx, ny, nz, x.dx, float(self.band), fe.V.data_ptr(),
                      x.F.data_ptr(), 1, x.active.data_ptr(), fe.small[8:9].data_ptr(), x.ncell,
                      fe.small[0:6].data_ptr(), _sp())

        self._each(surface)
        _lib.call("petch_trace_batch", 0, self._items(0, cur), B, MT, MV, 0.0,
                  self.step_dev.data_ptr(), 9, 1, self.work.data_ptr(), s)
        self._each(ion_post)
        for it in range(n_fp):
            # both species of the round in one launch: F (betaE, +2+2it) into fe.flux, O (betaO,
            # +3+2it) into the third slice of fe.tmp5
            items = self._items(1, cur)
            for b, x in enumerate(self.inst):
                items[b].ang = x.fe.tmp5[2 * MT:3 * MT].data_ptr()
            _lib.call("petch_trace_batch_pair", items, B, MT, MV, self.betaE, self.betaO,
                      self.step_dev.data_ptr(), 9, 2 + 2 * it, 3 + 2 * it, self.work.data_ptr(), s)
            self._each(coverage)
        self._each(rate_extend)
        grids = self._grids(cur)
        _lib.call("petch_batch_advect", grids, B, s)
        _lib.call("petch_batch_reinit", grids, B, float(self.band + 2.0 * self.dx), s)
        _lib.call("petch_batch_step_advance", self.step_dev.data_ptr(), s)

    # ---- capture and run ----
    def capture(self):
        """Capture the cold first step and the two warm steps (mesh / coverage buffers swap
        roles every step) into CUDA graphs.  Returns the kernel launches per warm step."""
        graphs = {}
        launches = {}
        for key, cold, cur in (("cold", True, 0), ("warm1", False, 1), ("warm0", False, 0)):
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
        cold = k == 0
        cur = k % 2
        if use_graph:
            if self.graphs is None:
                self.capture()
            self.graphs["cold" if cold else f"warm{cur}"].replay()
        else:
            self._step(cold, cur)
        self.steps_done += 1

    def run(self, n_steps=None, use_graph=True, record_depth_every=0):
        """Advance n_steps (default: the rest of the schedule); returns seconds of device time
        (CUDA events around the whole run)."""
        n = self.n_steps - self.steps_done if n_steps is None else int(n_steps)
        if use_graph and self.graphs is None:
            self.capture()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            self.step(use_graph)
            if record_depth_every and (self.steps_done % record_depth_every == 0
                                       or self.steps_done == self.n_steps):
                self._record_depths()
        e1.record()
        torch.cuda.synchronize()
        self.check()
        return e0.elapsed_time(e1) / 1e3

    def _record_depths(self):
        for b, x in enumerate(self.inst):
            self.depth_history[b].append((self.steps_done, _depth3d(dict(x.geo, phi=x.phi))))

    def check(self):
        """Raise on device-side errors (mesh capacity, traversal limits) after a run."""
        err = int(self.work[1].item())
        if err:
            raise RuntimeError(f"batched trace: device error bits {err}")
        for b, x in enumerate(self.inst):
            for m in x.meshes:
                e = int(m.hdr[3].item())
                if e & (MESH_ERR_TRI_OVERFLOW | MESH_ERR_VERT_OVERFLOW | MESH_ERR_HASH_FULL):
                    raise RuntimeError(f"instance {b}: mesh capacity {self.MT} exceeded "
                                       f"(error bits {e}); pass a larger max_tris")
            if int(x.fe.small[1].item()):
                raise RuntimeError(f"instance {b}: device error bits {int(x.fe.small[1].item())}")

    def depths(self):
        """Centre depth (_depth3d) of every instance now."""
        return [_depth3d(dict(x.geo, phi=x.phi)) for x in self.inst]

    def phis(self):
        return [x.phi.double().cpu().numpy() for x in self.inst]


def hole_batch_specs(n=64, seed=0, dx=0.25, Lz=24.0, headroom=4.0):
    """The ragged hole batch: diameter ~ U[2, 8] um, mask thickness ~ U[1, 3] um, extent =
    diameter + 8 um, grid height Lz; per instance ion energy log-uniform in [50, 500] eV,
    F / ion flux ratio log-uniform in [10, 1000], O / F ratio ~ U[0, 0.5] (drawn with a seeded
    torch.Generator).  The substrate top sits `headroom` + mask below the top of the grid."""
    g = torch.Generator().manual_seed(seed)
    u = torch.rand((n, 5), generator=g, dtype=torch.float64).numpy()
    specs = []
    for k in range(n):
        d = 2.0 + 6.0 * u[k, 0]
        mask = 1.0 + 2.0 * u[k, 1]
        E = float(np.exp(np.log(50.0) + (np.log(500.0) - np.log(50.0)) * u[k, 2]))
        rF = float(np.exp(np.log(10.0) + (np.log(1000.0) - np.log(10.0)) * u[k, 3]))
        rO = 0.5 * u[k, 4]
        ext = round((d + 8.0) / dx) * dx
        sub_top = Lz - headroom - mask
        par = dict(Emean=E, Fflux=rF * PAR['ionFlux'], Oflux=rO * rF * PAR['ionFlux'])
        specs.append(dict(Lx=ext, Ly=ext, Lz=Lz, dx=dx, trench_width=d, mask_th=mask,
                          sub_top=sub_top, hole=True, par=par))
    return specs
