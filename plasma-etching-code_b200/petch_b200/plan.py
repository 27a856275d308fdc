"""The fused etch step from Python: petch_plan / petch_step / petch_plan_status / petch_destroy.

One C call per step of run_etch_3d's coverage-coupled Monte-Carlo loop (petch/threed.py:
1671-1792 with mc_flux_3d_coupled), on a workspace the library plans once.  A step enqueues only
stream-ordered work with every step-dependent quantity on the device, so steps are captured into
CUDA graphs and replayed: one graph for the cold first step, one for a pair of warm steps and
one for a single warm step (the warm start's mesh / coverage buffers alternate).  With deterministic tallies a plan's steps equal
run_etch_3d's bit for bit.

    plan = StepPlan(Lx=8, Ly=4, Lz=40, dx=0.0625, trench_width=2, mask_th=1, sub_top=35,
                    hole=False, t_end=2.0, n_steps=100, par=par, flags=flags,
                    n_ion=1 << 22, n_neu=1 << 22)
    plan.run(100)           # graph replays
    plan.status()           # one synchronising read: faces, substeps, errors
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .levelset import grid_shape
from .params import DEFAULT_FLAGS, PAR
from .threed import _sp, chem_params, default_capacity, domain_params, ion_params


def supported(flags, par):
    """True if (flags, par) select the path the fused step runs: faithful ions with Belen
    coverages and coverage-dependent sticking, Monte-Carlo neutrals, no redeposition or
    charging models."""
    f = flags or DEFAULT_FLAGS
    return (getattr(f, "chemistry", "langmuir") == "belen"
            and getattr(f, "ion_reflection", False) and getattr(f, "coverage_sticking", False)
            and getattr(f, "neutral_transport", "mc") == "mc"
            and not getattr(f, "redeposition", False)
            and not getattr(f, "floor_charge_throttle", False)
            and not (getattr(f, "surface_charging", False)
                     and float(par.get('charge_alpha', 0.0)) > 0.0)
            and par.get('cov_transport', 'rr') == 'rr')


class StepPlan:
    """A planned run of the fused step on a device level set (float32, caller-visible as
    `self.phi`).  phi_init: initial level set (host or device array); None writes the seed field
    (make_trench_3d's CSG field, redistanced).  dt: the step length, when not t_end / n_steps
    (a plan that continues another run)."""

    def __init__(self, Lx, Ly, Lz, dx, trench_width, mask_th, sub_top, hole, t_end, n_steps,
                 par=None, flags=None, n_ion=20000, n_neu=20000, seed_offset=0, max_tris=None,
                 phi_init=None, dt=None):
        par = dict(PAR if par is None else par)
        flags = flags or DEFAULT_FLAGS
        if not supported(flags, par):
            raise NotImplementedError("the fused step runs the coverage-coupled SF6/O2 path "
                                      "(belen, ion_reflection, coverage_sticking, mc neutrals)")
        torch.cuda.init()
        nx, ny, nz = grid_shape(Lx, Ly, Lz, dx)
        geo = dict(Lx=Lx, Ly=Ly, Lz=Lz, dx=dx)
        c = _lib.StepConfig()
        c.nx, c.ny, c.nz = nx, ny, nz
        c.dx, c.Lx, c.Ly, c.Lz = float(dx), float(Lx), float(Ly), float(Lz)
        c.sub_top, c.mask_th, c.trench_width = float(sub_top), float(mask_th), float(trench_width)
        c.hole = int(bool(hole))
        c.dt = float(t_end) / int(n_steps) if dt is None else float(dt)
        c.n_ion, c.n_neu = int(n_ion), int(n_neu)
        c.seed_offset = int(seed_offset)
        c.max_tris = int(max_tris or default_capacity((nx, ny, nz)))
        c.n_fp = int(par['n_fp']) if 'n_fp' in par else 0
        c.warm_start = int(bool(getattr(flags, "warm_start_coverage", False)))
        c.n_smooth = int(par.get('flux_smooth', 1))
        c.smooth_alpha = float(par.get('flux_smooth_alpha', 1.0))
        c.betaE, c.betaO = float(par.get('betaE', 0.7)), float(par.get('betaO', 1.0))
        c.dom = domain_params(geo, par)
        c.ion = ion_params(par)
        c.chem = chem_params(par, flags)
        self.cfg = c
        self.shape = (nx, ny, nz)
        self.n_steps = int(n_steps)
        if phi_init is None:
            self.phi = torch.empty(self.shape, dtype=torch.float32, device="cuda")
        else:
            src = phi_init if isinstance(phi_init, torch.Tensor) else torch.from_numpy(
                np.ascontiguousarray(phi_init))
            self.phi = src.to("cuda", torch.float32).contiguous().view(self.shape).clone()
        h = ctypes.c_void_p()
        _lib.call("petch_plan", ctypes.byref(c), self.phi.data_ptr(), int(phi_init is None),
                  ctypes.byref(h), _sp())
        self.h = h
        self.steps_done = 0
        self.graphs = None
        self.graph_launches = {}
        self._cap_stream = None

    def step(self):
        """Enqueue one step on the current stream."""
        _lib.call("petch_plan_seek", self.h, self.steps_done)
        _lib.call("petch_step", self.h, _sp())
        self.steps_done += 1

    # graph key -> (the step it is captured at, steps it holds)
    _GRAPH_STEPS = {"cold": (0, 1), "warm2": (1, 2), "warm1": (1, 1), "warm0": (2, 1)}

    def _capture_graph(self, key):
        """Capture one graph on a side stream.  Capturing is host work only and waits for
        nothing, so it overlaps the steps the device is still running."""
        first, n = self._GRAPH_STEPS[key]
        if self._cap_stream is None:
            _lib.call("petch_prepare_device")
            self._cap_stream = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        _lib.call("petch_plan_seek", self.h, first)
        n0 = _lib.launch_count()
        try:
            with torch.cuda.stream(self._cap_stream):
                g.capture_begin()
                try:
                    for _ in range(n):
                        _lib.call("petch_step", self.h, _sp())
                finally:
                    g.capture_end()
        finally:
            _lib.call("petch_plan_seek", self.h, self.steps_done)
        if self.graphs is None:
            self.graphs = {}
        self.graphs[key] = g
        self.graph_launches[key] = _lib.launch_count() - n0
        return g

    def capture(self, pair=True):
        """Capture the cold first step, a pair of warm steps (pair=True) and a single odd and a
        single even warm step into CUDA graphs (capturing enqueues nothing: the graphs run on
        replay).  A warm step s uses mesh buffer s % 2, so the pair graph starts on an odd step:
        run() replays cold, pairs, and a single step when the remaining count is odd;
        replay_step() replays one step at a time."""
        self.graphs, self.graph_launches = {}, {}
        for key in ("cold", "warm2", "warm1", "warm0"):
            if pair or key != "warm2":
                self._capture_graph(key)
        return self.graphs

    def run(self, n=None, use_graph=True):
        """Advance n steps (default: the rest of the schedule) by graph replays, or eagerly."""
        n = self.n_steps - self.steps_done if n is None else int(n)
        if not use_graph:
            for _ in range(n):
                self.step()
            return
        if self.graphs is None or "warm2" not in self.graphs:
            self.capture()
        warm = bool(self.cfg.warm_start)
        while n > 0:
            s = self.steps_done
            if s == 0 or not warm:
                g, k = self.graphs["cold"], 1
            elif s % 2 == 1:
                g, k = (self.graphs["warm2"], 2) if n >= 2 else (self.graphs["warm1"], 1)
            else:                          # an even warm step (after eager steps): run it eagerly
                self.step()
                n -= 1
                continue
            g.replay()
            self.steps_done += k
            n -= k

    def replay_step(self):
        """Advance one step by replaying its graph (cold, odd or even warm step); returns the
        library kernel launches it holds.  Without captured graphs the plan's first step runs
        eagerly, and each graph is captured at its first use, while the device still runs the
        steps before it (a run that replays step by step then never waits for a capture)."""
        s = self.steps_done
        if self.graphs is None and s == 0:
            self.graphs = {}
            n0 = _lib.launch_count()
            self.step()
            return _lib.launch_count() - n0
        key = "cold" if s == 0 or not self.cfg.warm_start else ("warm1" if s % 2 else "warm0")
        g = (self.graphs or {}).get(key) or self._capture_graph(key)
        g.replay()
        self.steps_done += 1
        return self.graph_launches[key]

    def mask_host(self):
        """The plan's mask (the pinned, un-etched mask cells) as a host bool array."""
        out = np.empty(self.shape, dtype=np.uint8)
        _lib.call("petch_plan_mask", self.h, out.ctypes.data, _sp())
        return out.view(np.bool_)

    def timing(self, on=True):
        """Record CUDA events around each step's neutral-pair trace launches (enable before
        capture(): the graphs then record them on every replay)."""
        _lib.call("petch_plan_timing", self.h, int(bool(on)))

    def trace_ms(self):
        """Device milliseconds of the last step's neutral-pair trace launches (waits for them)."""
        ms = ctypes.c_float()
        _lib.call("petch_plan_trace_ms", self.h, ctypes.byref(ms))
        return float(ms.value)

    def status(self, check=True):
        """The plan's accumulated status (one synchronising read); raises on device errors."""
        st = _lib.StepStatus()
        rc = _lib.lib().petch_plan_status(self.h, ctypes.byref(st), _sp())
        out = {k: getattr(st, k) for k, _ in _lib.StepStatus._fields_}
        if check and rc != 0:
            raise _lib.PetchError(rc, "petch_plan_status", _lib.last_error())
        out['status'] = rc
        return out

    def close(self):
        if getattr(self, "h", None):
            torch.cuda.synchronize()
            self.graphs = None
            _lib.call("petch_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
