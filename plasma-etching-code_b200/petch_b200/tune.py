"""The tuner: picks the settings of the persistent tracer and of the level-set stencils by timing
candidates on the run's own surface, once per (device, size bucket), and caches the choice in
memory and in a JSON file so later runs (and later steps in the same bucket) just apply it.

Tracer knobs (petch_tracer_config, petch_tally_aggregation, petch_tracer_grouping):
    bvh_width     2 (binary LBVH) or 8 (quantised 8-wide BVH, top levels in shared memory)
    steps         traversal steps a warp runs for its open queries between shading rounds
    keep          lanes that may still be traversing when a warp stops to shade and refill
    aggregate     warp-aggregated deposits (tried against the fastest candidates)
    grouping      leaf grouping of the traversal (0 off, or the 1/g share of open lanes
                  at a leaf that switches a warp iteration to triangle tests)
Stencil knob (petch_stencil_config): the block shape (threads along z x grid rows) of the
row-mapped Eikonal passes.

The tracer trial is the step's dominant launch: both neutral species of a coverage round
(petch_trace_neutral_pair) on the current mesh with the coverage warm-started from the previous
step's, as the loop runs it; the stencil trial is the reinit of the current level set.  A coarse
pass times every candidate, a fine pass (larger trials, more timings) the few fastest, and the
fastest of the fine pass is chosen; every timing is the minimum over repeats (CUDA events), each
after an untimed run of the same candidate.  Buckets: face count (tracer) and cell count
(stencil) by powers of two.

Enable in run_etch_3d with tune=True (or a Tuner); the cache file is $PETCH_TUNE_CACHE, else
~/.cache/petch_b200/tune.json.
"""
import ctypes
import json
import math
import os

import numpy as np
import torch

from . import _lib

# tracer settings: (bvh_width, steps, keep, aggregate, grouping)
TRACER_GRID = (tuple((2, s, k, 0, g) for s in (32, 64, 128) for k in (8, 12, 16) for g in (2, 3))
               + ((2, 32, 16, 0, 0), (8, 32, 16, 0, 2), (8, 64, 12, 0, 2), (8, 32, 16, 0, 0)))
STENCIL_GRID = ((32, 8), (64, 4), (128, 2), (256, 1), (64, 2), (128, 1))
TRACER_DEFAULT = (2, 32, 16, 0, 2)
STENCIL_DEFAULT = (128, 2)


def default_cache_path():
    return os.environ.get("PETCH_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "petch_b200", "tune.json")


def apply_tracer(cfg):
    w, s, k, a, g = (int(v) for v in cfg)
    _lib.call("petch_tracer_config", w, s, k)
    _lib.call("petch_tally_aggregation", a)
    _lib.call("petch_tracer_grouping", g)


def apply_stencil(cfg):
    _lib.call("petch_stencil_config", int(cfg[0]), int(cfg[1]))


def bucket(n):
    """Power-of-two size bucket of a face or cell count."""
    return int(math.floor(math.log2(max(int(n), 1))))


class Tuner:
    """rays: rays per species of a fine tracer trial (coarse trials take half), best the run's
    own count, since the launch tail depends on it; reps: timings per candidate in the coarse
    pass (three times as many in the fine pass); top: candidates of the fine pass; path: cache
    file (None: the default; False: memory only)."""

    def __init__(self, rays=1 << 20, reps=2, path=None, tracer_grid=TRACER_GRID,
                 stencil_grid=STENCIL_GRID, top=4):
        self.rays, self.reps, self.top = int(rays), int(reps), int(top)
        self.path = default_cache_path() if path is None else path
        self.tracer_grid, self.stencil_grid = tuple(tracer_grid), tuple(stencil_grid)
        self.cache = self._load()
        self.chosen = {}       # bucket key -> config applied in this process (for reports)
        self.trials = {}       # bucket key -> {config: median ms} measured in this process
        self.frozen = False    # True: never measure; an uncached bucket takes the nearest one
        p = torch.cuda.get_device_properties(torch.cuda.current_device())
        self.device = f"{p.name}/{p.multi_processor_count}sm"

    # ---- cache ----
    def _load(self):
        if self.path and os.path.exists(self.path):
            try:
                return json.load(open(self.path))
            except (OSError, ValueError):
                return {}
        return {}

    def _store(self):
        if not self.path:
            return
        os.makedirs(os.path.dirname(self.path) or ".", exist_ok=True)
        tmp = self.path + f".{os.getpid()}"
        with open(tmp, "w") as fh:
            json.dump(self.cache, fh, indent=1, sort_keys=True)
        os.replace(tmp, self.path)

    def key(self, what, n):
        return f"{self.device}|{what}|{bucket(n)}"

    def _nearest(self, what, n):
        """The cached key of this device and kind with the bucket nearest n's (None if none)."""
        pre = f"{self.device}|{what}|"
        have = [int(k[len(pre):]) for k in self.cache if k.startswith(pre)]
        if not have:
            return None
        b = min(have, key=lambda v: (abs(v - bucket(n)), v))
        return pre + str(b)

    # ---- measurement ----
    @staticmethod
    def _time(fns, reps):
        """fns: {config: callable enqueueing one trial on the current stream}.  The fastest of
        `reps` timings per config (CUDA events); each timing follows an untimed run of the same
        config, so it does not inherit another config's cache state, and the configs take turns
        (order reversed every round)."""
        out = {c: [] for c in fns}
        order = list(fns)
        for r in range(reps):
            evs = []
            for c in (order if r % 2 == 0 else order[::-1]):
                fns[c]()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                fns[c]()
                e1.record()
                evs.append((c, e0, e1))
            torch.cuda.synchronize()
            for c, e0, e1 in evs:
                out[c].append(e0.elapsed_time(e1))
        return {c: float(np.min(v)) for c, v in out.items()}

    def _search(self, trial, grid, reps, top, twin=None):
        """Coarse pass (every config, `reps` timings at half the trial size), then a fine pass on
        the `top` fastest -- and on twin(c) of the two fastest, when given: a setting the coarse
        grid leaves at one value -- with three times the timings at the full trial size, then a
        duel of the fine pass's two fastest (alternating, six times the timings), whose times
        replace theirs.  Settings a few per cent apart can swap places between passes of a few
        timings; the duel settles the choice between the two that matter.  Returns ({config: ms}
        of the coarse pass, {config: ms} of the fine pass and the duel, which decides)."""
        coarse = self._time({c: trial(c, 1) for c in grid}, reps)
        best = sorted(coarse, key=coarse.get)[:max(1, top)]
        if twin is not None:
            best += [t for t in (twin(c) for c in best[:2]) if t is not None and t not in best]
        fine = self._time({c: trial(c, 2) for c in best}, 3 * reps)
        pair = sorted(fine, key=fine.get)[:2]
        if len(pair) == 2:
            fine.update(self._time({c: trial(c, 2) for c in pair}, 6 * reps))
        return coarse, fine

    def tracer_trials(self, eng, grid=None, reps=None, exhaustive=False):
        """Timings (ms) of the neutral-pair trial for the tracer configs of `grid` on eng's
        current level set (meshes rebuilt here: binary and, for width 8, with the wide tree),
        coverage warm-started from eng's previous mesh when it has one: (coarse, fine) of
        _search, or with exhaustive=True the fine timing of every config."""
        from .threed import DeviceMesh, _sp
        grid = tuple(grid or self.tracer_grid)
        meshes, bares = {}, {}
        for w in sorted({c[0] for c in grid}):
            _lib.call("petch_tracer_config", w, 64, 12)
            m = DeviceMesh(eng.MT)
            m.build(eng.phi, eng.dx, eng.geo, eng.scratch)
            b = torch.ones(eng.MT, device="cuda")
            if eng.prev is not None:
                pm, pb = eng.prev
                _lib.call("petch_warmstart", pm.id, pm.MT, pm.MV, pb.data_ptr(), m.id, m.MT, m.MV,
                          b.data_ptr(), eng.small[0:6].data_ptr(), _sp())
            meshes[w], bares[w] = m, b
        flux_a = torch.empty(eng.MT, device="cuda")
        flux_b = torch.empty(eng.MT, device="cuda")
        work = torch.zeros(6, dtype=torch.int32, device="cuda")
        betaE = float(eng.par.get('betaE', 0.7))
        betaO = float(eng.par.get('betaO', 1.0))

        def trial(cfg, scale):
            def run():
                apply_tracer(cfg)
                m = meshes[cfg[0]]
                _lib.call("petch_trace_neutral_pair", m.id, m.MT, m.MV, ctypes.byref(eng.dom),
                          bares[cfg[0]].data_ptr(), betaE, betaO, 7, 8, 0, scale * self.rays // 2,
                          flux_a.data_ptr(), flux_b.data_ptr(), work.data_ptr(), _sp())
            return run

        try:
            if exhaustive:
                res = self._time({c: trial(c, 2) for c in grid}, 3 * (reps or self.reps))
            else:
                res = self._search(trial, grid, reps or self.reps, self.top,
                                   twin=lambda c: (c[0], c[1], c[2], 1 - c[3], c[4]))
        finally:
            apply_tracer(TRACER_DEFAULT)
        if int(work[1].item()):
            raise RuntimeError(f"tuner trial: tracer error bits {int(work[1].item())}")
        return res

    def stencil_trials(self, eng, grid=None, reps=None, exhaustive=False):
        """Timings (ms) of the reinit of eng's level set (into scratch) for the block shapes:
        (coarse, fine) of _search, or with exhaustive=True the fine timing of every shape."""
        from .levelset import reinit_fsm_dev
        grid = tuple(grid or self.stencil_grid)
        out = torch.empty_like(eng.phi)
        band = 6.0 * eng.dx

        def trial(cfg, scale):
            def run():
                apply_stencil(cfg)
                for _ in range(scale):
                    reinit_fsm_dev(eng.phi, eng.dx, band, out=out, scratch=(eng.ua, eng.ub))
            return run

        try:
            if exhaustive:
                return self._time({c: trial(c, 2) for c in grid}, 3 * (reps or self.reps))
            return self._search(trial, grid, reps or self.reps, self.top)
        finally:
            apply_stencil(STENCIL_DEFAULT)

    def _record(self, key, coarse, fine):
        self.trials[key] = {"coarse": {str(list(c)): round(v, 4) for c, v in coarse.items()},
                            "fine": {str(list(c)): round(v, 4) for c, v in fine.items()}}
        self.cache[key] = list(min(fine, key=fine.get))

    # ---- choose and apply ----
    def ensure(self, eng, n_faces):
        """Apply the cached settings of eng's buckets, measuring those not cached yet.  Returns
        True if the tracer's BVH width changed (the caller rebuilds its mesh)."""
        before = tracer_settings()[0]
        changed = False
        kt = self.key("tracer", n_faces)
        ks = self.key("stencil", eng.ncell)
        if self.frozen:
            kt = kt if kt in self.cache else self._nearest("tracer", n_faces)
            ks = ks if ks in self.cache else self._nearest("stencil", eng.ncell)
            if kt is None or ks is None:
                raise RuntimeError("frozen tuner without a cached choice for this device")
        if kt not in self.cache:
            coarse, fine = self.tracer_trials(eng)
            self._record(kt, coarse, fine)
            changed = True
        if ks not in self.cache:
            coarse, fine = self.stencil_trials(eng)
            self._record(ks, coarse, fine)
            changed = True
        if changed:
            self._store()
        apply_tracer(self.cache[kt])
        apply_stencil(self.cache[ks])
        self.chosen[kt] = self.cache[kt]
        self.chosen[ks] = self.cache[ks]
        return self.cache[kt][0] != before


def tracer_settings():
    """(bvh_width, steps, keep, aggregate, grouping) in force in the library."""
    out = (ctypes.c_int * 5)()
    _lib.call("petch_tracer_settings", out)
    return tuple(out)


def reset():
    """Back to the library's default settings."""
    apply_tracer(TRACER_DEFAULT)
    apply_stencil(STENCIL_DEFAULT)
