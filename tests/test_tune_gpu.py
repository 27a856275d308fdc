"""The tuner picks, per size bucket, the fastest tracer and stencil settings of its candidate
grid: re-timing every candidate on the same surface, the chosen one is within 2 % of the best.
Settings are speed knobs only: a run with the tuner on gives the same etch (deterministic
tallies) as with the defaults."""
import numpy as np
import pytest

from petch_b200 import _lib, params
from petch_b200 import threed as t3
from petch_b200 import tune

pytestmark = pytest.mark.gpu

SF6O2 = params.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     warm_start_coverage=True, sampling="sobol", ion_reflection=True)
TRENCH = dict(Lx=8.0, Ly=4.0, Lz=40.0, dx=0.0625, trench_width=2.0, mask_th=1.0, sub_top=35.0,
              hole=False)


@pytest.fixture(scope="module")
def deep_trench():
    """The headline trench after 40 steps of its 100-step schedule (~10 um deep)."""
    par = dict(params.PAR, periodic_y=1)
    geo = t3.run_etch_3d(**TRENCH, t_end=0.8, n_steps=40, par=par, flags=SF6O2, n_ion=1 << 18,
                         n_neu=1 << 18, reinit_method="fsm", verbose=False, max_tris=1 << 20,
                         engine="stages")
    return geo['engine']


def test_tuner_choice_within_2pct_of_exhaustive_sweep(deep_trench):
    """The tuner's pick against an exhaustive sweep of its candidate grid (every candidate timed
    with the fine trial), then the pick and the sweep's best timed head to head (alternating, 8
    rounds): the pick is within 2 % of the best."""
    eng = deep_trench
    F = eng.prev[0].n_faces()
    tuner = tune.Tuner(rays=1 << 20, path=False)
    try:
        tuner.ensure(eng, F)
        chosen_t = tuple(tuner.cache[tuner.key("tracer", F)])
        chosen_s = tuple(tuner.cache[tuner.key("stencil", eng.ncell)])
        sweep_t = tuner.tracer_trials(eng, exhaustive=True)
        sweep_s = tuner.stencil_trials(eng, exhaustive=True)
        best_t = min(sweep_t, key=sweep_t.get)
        best_s = min(sweep_s, key=sweep_s.get)
        duel_t = tuner.tracer_trials(eng, grid=[chosen_t, best_t], reps=8, exhaustive=True)
        duel_s = tuner.stencil_trials(eng, grid=[chosen_s, best_s], reps=8, exhaustive=True)
    finally:
        tune.reset()
    print("tracer chosen", chosen_t, "sweep best", best_t, "duel", duel_t)
    print("stencil chosen", chosen_s, "sweep best", best_s, "duel", duel_s)
    assert len(sweep_t) == len(tune.TRACER_GRID) and len(sweep_s) == len(tune.STENCIL_GRID)
    assert duel_t[chosen_t] <= 1.02 * duel_t[best_t]
    assert duel_s[chosen_s] <= 1.02 * duel_s[best_s] + 0.002      # + 2 us: sub-ms launches


def test_tuned_run_equals_default_run(tmp_path):
    """With deterministic tallies a run under the tuner etches exactly as the default settings
    do: steps per round, keep lanes, aggregation and the stencil block shape change the speed,
    not the results.  (The 8-wide tree may break an exact tie between coincident faces the other
    way; tests/test_flux_gpu.py::test_tracer_configs_agree compares the widths.)"""
    kw = dict(Lx=4.0, Ly=2.0, Lz=10.0, dx=0.125, trench_width=2.0, mask_th=1.0, sub_top=7.0,
              hole=False, t_end=0.5, n_steps=5, par=dict(params.PAR, periodic_y=1, rate_scale=0.3),
              flags=SF6O2, n_ion=30000, n_neu=30000, reinit_method="fsm", verbose=False)
    _lib.set_deterministic(1 << 22)
    try:
        a = t3.run_etch_3d(**kw)
        tuner = tune.Tuner(rays=1 << 16, reps=1, path=str(tmp_path / "tune.json"),
                           tracer_grid=[c for c in tune.TRACER_GRID if c[0] == 2])
        b = t3.run_etch_3d(**kw, tune=tuner)
    finally:
        tune.reset()
        _lib.set_deterministic(0)
    assert b['tuning'] and (tmp_path / "tune.json").exists()
    np.testing.assert_array_equal(a['phi'], b['phi'])
