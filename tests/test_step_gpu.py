"""The fused step (petch_plan / petch_step / petch_plan_status / petch_destroy) through the C ABI:
N steps of petch_step alone equal run_etch_3d's steps bit for bit with deterministic tallies
(the same kernels in the same order, seeds and substep counts read on the device), graph-replayed
steps equal eager ones, and a capacity overflow is reported, not hidden."""
import ctypes

import numpy as np
import pytest
import torch

from petch_b200 import _lib, params
from petch_b200 import threed as t3
from petch_b200.levelset import grid_shape
from petch_b200.plan import StepPlan

pytestmark = pytest.mark.gpu

SF6O2 = params.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     warm_start_coverage=True, sampling="sobol", ion_reflection=True)

HOLE = dict(Lx=8.0, Ly=8.0, Lz=12.0, dx=0.25, trench_width=4.0, mask_th=1.0, sub_top=8.0,
            hole=True)
TRENCH = dict(Lx=4.0, Ly=2.0, Lz=10.0, dx=0.125, trench_width=2.0, mask_th=1.0, sub_top=7.0,
              hole=False)


def _par(hole, rate_scale=0.3):
    return dict(params.PAR, rate_scale=rate_scale, periodic_y=0 if hole else 1)


def _config(g, par, t_end, n_steps, n, seed_offset=0, max_tris=None):
    """A petch_step_config filled field by field through the ctypes structure (as a C caller
    would), from run_etch_3d's arguments."""
    nx, ny, nz = grid_shape(g['Lx'], g['Ly'], g['Lz'], g['dx'])
    c = _lib.StepConfig()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.dx, c.Lx, c.Ly, c.Lz = g['dx'], g['Lx'], g['Ly'], g['Lz']
    c.sub_top, c.mask_th, c.trench_width, c.hole = (g['sub_top'], g['mask_th'],
                                                     g['trench_width'], int(g['hole']))
    c.dt = t_end / n_steps
    c.n_ion = c.n_neu = n
    c.seed_offset = seed_offset
    c.max_tris = max_tris or t3.default_capacity((nx, ny, nz))
    c.n_fp = 0
    c.warm_start = 1
    c.n_smooth, c.smooth_alpha = 1, 1.0
    c.betaE, c.betaO = par['betaE'], par['betaO']
    c.dom = t3.domain_params(g, par)
    c.ion = t3.ion_params(par)
    c.chem = t3.chem_params(par, SF6O2)
    return c, (nx, ny, nz)


@pytest.mark.parametrize("g", [HOLE, TRENCH], ids=["hole", "trench"])
def test_petch_step_equals_run_etch_3d(g):
    """Seven steps through the C ABI alone (plan with the seed field, petch_step x 7, status,
    destroy) against run_etch_3d's stage-by-stage engine with the same arguments: level sets
    equal bit for bit."""
    par = _par(g['hole'])
    n, steps, t_end = 30000, 7, 0.7
    c, shape = _config(g, par, t_end, steps, n, seed_offset=5)
    s = torch.cuda.current_stream().cuda_stream
    _lib.set_deterministic(16 * c.max_tris)
    try:
        phi = torch.empty(shape, dtype=torch.float32, device="cuda")
        h = ctypes.c_void_p()
        _lib.call("petch_plan", ctypes.byref(c), phi.data_ptr(), 1, ctypes.byref(h), s)
        try:
            for _ in range(steps):
                _lib.call("petch_step", h, s)
            st = _lib.StepStatus()
            _lib.call("petch_plan_status", h, ctypes.byref(st), s)
        finally:
            torch.cuda.synchronize()
            _lib.call("petch_destroy", h)
        geo = t3.run_etch_3d(**g, t_end=t_end, n_steps=steps, par=par, flags=SF6O2, n_ion=n,
                             n_neu=n, reinit_method="fsm", verbose=False, seed_offset=5,
                             engine="stages")
    finally:
        _lib.set_deterministic(0)
    assert st.steps == steps and st.trace_errors == 0 and st.mesh_errors & 7 == 0
    assert st.faces > 0 and st.max_faces >= st.faces
    np.testing.assert_array_equal(phi.double().cpu().numpy(), geo['phi'])
    assert (geo['phi'] < 0).sum() > 0


def test_graph_replay_equals_eager_steps():
    """The plan's CUDA graphs replayed over 8 steps -- cold step, warm pairs and an odd single,
    or one step at a time -- equal 8 eager petch_step calls bit for bit (deterministic
    tallies)."""
    par = _par(True)
    kw = dict(**HOLE, t_end=0.8, n_steps=8, par=par, flags=SF6O2, n_ion=30000, n_neu=30000)
    _lib.set_deterministic(16 * t3.default_capacity(grid_shape(8.0, 8.0, 12.0, 0.25)))
    try:
        eager = StepPlan(**kw)
        eager.run(use_graph=False)
        st_e = eager.status()
        graph = StepPlan(**kw)
        graph.run()                       # cold, 3 warm pairs, 1 warm single
        st_g = graph.status()
        single = StepPlan(**kw)
        for _ in range(8):
            single.replay_step()          # cold, then odd / even single-step graphs
        st_s = single.status()
        a, b, c = eager.phi.clone(), graph.phi.clone(), single.phi.clone()
        for p in (eager, graph, single):
            p.close()
    finally:
        _lib.set_deterministic(0)
    assert st_e['steps'] == st_g['steps'] == st_s['steps'] == 8
    assert torch.equal(a, b) and torch.equal(a, c)


def test_trace_timing_events_in_eager_steps_and_graph_replays():
    """petch_plan_timing: the events around a step's neutral-pair launch are recorded by eager
    steps and by every replay of a captured graph (external event nodes), and bracket less than
    the whole step; timing leaves the results unchanged (bit-equal level sets)."""
    par = _par(True)
    kw = dict(**HOLE, t_end=0.6, n_steps=6, par=par, flags=SF6O2, n_ion=1 << 18, n_neu=1 << 18)
    _lib.set_deterministic(16 * t3.default_capacity(grid_shape(8.0, 8.0, 12.0, 0.25)))
    try:
        plain = StepPlan(**kw)
        plain.run(use_graph=False)
        timed = StepPlan(**kw)
        timed.timing(True)
        timed.step()
        assert timed.trace_ms() > 0.0                    # the cold step, eager
        timed.capture()
        ms = []
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            timed.replay_step()
            e1.record()
            torch.cuda.synchronize()
            ms.append((timed.trace_ms(), e0.elapsed_time(e1)))
        a, b = plain.phi.clone(), timed.phi.clone()
        for p in (plain, timed):
            p.close()
    finally:
        _lib.set_deterministic(0)
    assert torch.equal(a, b)
    for t, step in ms:
        assert 0.0 < t < step, ms


def test_capacity_overflow_is_reported():
    par = _par(True)
    plan = StepPlan(**HOLE, t_end=0.2, n_steps=2, par=par, flags=SF6O2, n_ion=1000, n_neu=1000,
                    max_tris=256)
    plan.run(1, use_graph=False)
    st = plan.status(check=False)
    plan.close()
    assert st['status'] == 3                     # PETCH_E_OVERFLOW
    assert st['mesh_errors'] & 1


def test_run_etch_3d_fused_equals_stages_with_depth_history():
    """run_etch_3d's two engines (the fused step, the default for these arguments, and the
    stage-by-stage composition) give the same level set and depth history bit for bit."""
    par = _par(False)
    kw = dict(**TRENCH, t_end=0.6, n_steps=6, par=par, flags=SF6O2, n_ion=30000, n_neu=30000,
              reinit_method="fsm", verbose=False, record_depth_every=1)
    _lib.set_deterministic(1 << 22)
    try:
        a = t3.run_etch_3d(**kw, engine="fused")
        b = t3.run_etch_3d(**kw, engine="stages")
        c = t3.run_etch_3d(**kw)
    finally:
        _lib.set_deterministic(0)
    assert a['timings'].get('fused') and not b['timings'].get('fused') and c['timings'].get('fused')
    np.testing.assert_array_equal(a['phi'], b['phi'])
    np.testing.assert_array_equal(a['mask'], b['mask'])
    assert a['depth_history'] == b['depth_history'] and len(a['depth_history']) == 6


def test_fused_run_regrows_capacity():
    """A fused run whose mesh outgrows max_tris holds the step on the device, plans again with
    more capacity from the held level set and finishes: the depth follows the stage engine's
    (which regrows in place) within one cell."""
    par = _par(True)
    kw = dict(**HOLE, t_end=0.6, n_steps=6, par=par, flags=SF6O2, n_ion=30000, n_neu=30000,
              reinit_method="fsm", verbose=False, record_depth_every=1, max_tris=2048)
    a = t3.run_etch_3d(**kw, engine="fused")
    b = t3.run_etch_3d(**kw, engine="stages")
    assert [s for s, _ in a['depth_history']] == list(range(1, 7))
    for (s, da), (_, db) in zip(a['depth_history'], b['depth_history']):
        assert abs(da - db) <= HOLE['dx'] + 1e-9, (s, da, db)


@pytest.mark.parametrize("g", [HOLE, TRENCH], ids=["hole", "trench"])
def test_plan_mask_equals_the_seed_mask(g):
    """petch_plan_mask hands back the mask the plan pinned (make_trench_3d's), the one
    run_etch_3d's fused engine returns as geo['mask']."""
    from petch_b200.levelset import seed_field
    plan = StepPlan(**g, t_end=0.2, n_steps=2, par=_par(g['hole']), flags=SF6O2, n_ion=1000,
                    n_neu=1000)
    try:
        got = plan.mask_host()
    finally:
        plan.close()
    nx, ny, nz = grid_shape(g['Lx'], g['Ly'], g['Lz'], g['dx'])
    _, mask = seed_field(nx, ny, nz, g['dx'], g['Lx'], g['Ly'], g['sub_top'], g['mask_th'],
                         g['trench_width'], g['hole'])
    want = mask.bool().cpu().numpy()
    assert got.dtype == np.bool_ and got.shape == want.shape and want.any()
    np.testing.assert_array_equal(got, want)
