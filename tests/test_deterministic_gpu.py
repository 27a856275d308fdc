"""Deterministic tallies (petch_set_deterministic): with the Philox streams fixed, traces and
whole etch runs are reproducible bit for bit, batched launches equal per-instance calls exactly,
and the values agree with the float-atomic tallies to rounding."""
import ctypes

import numpy as np
import pytest
import torch

from gpu_helpers import cuda_mesh, domain, small_feature, stream
import petch_b200 as petch
from petch_b200 import _lib
from petch_b200 import threed as t3

pytestmark = pytest.mark.gpu


@pytest.fixture
def det():
    _lib.set_deterministic(8 * 4 * 65536 * 8)
    yield
    _lib.set_deterministic(0)


def _trace(m, geo, kind, seed, n):
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    if kind == "ions":
        tal, ang = torch.zeros((m.MT, 4), device="cuda"), torch.zeros(m.MT, device="cuda")
        _lib.call("petch_trace_ions", m.id, m.MT, m.MV, ctypes.byref(domain(geo)),
                  ctypes.byref(t3.ion_params(dict(petch.PAR))), seed, n, tal.data_ptr(),
                  ang.data_ptr(), work.data_ptr(), stream())
        return torch.cat([tal, ang[:, None]], 1)[:m.F]
    flux = torch.zeros(m.MT, device="cuda")
    _lib.call("petch_trace_neutrals", m.id, m.MT, m.MV, ctypes.byref(domain(geo)), None, 0.7, seed,
              0, n, flux.data_ptr(), work.data_ptr(), stream())
    return flux[:m.F]


@pytest.mark.parametrize("kind", ["ions", "neutrals"])
def test_traces_are_bit_reproducible_and_match_float_tallies(det, kind):
    phi, geo = small_feature(False)
    m = cuda_mesh(phi, geo['dx'], geo, MT=65536)
    a = _trace(m, geo, kind, 5, 500_000)
    b = _trace(m, geo, kind, 5, 500_000)
    assert torch.equal(a, b)
    _lib.set_deterministic(0)
    c = _trace(m, geo, kind, 5, 500_000)
    np.testing.assert_allclose(a.double().cpu().numpy(), c.double().cpu().numpy(), rtol=2e-5,
                               atol=1e-4)


def test_etch_runs_are_bit_reproducible(det):
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     warm_start_coverage=True, ion_reflection=True)
    kw = dict(Lx=5.0, Ly=2.5, Lz=8.0, dx=0.25, trench_width=2.0, mask_th=1.0, sub_top=6.0,
              t_end=0.6, n_steps=6, par=dict(petch.PAR, rate_scale=0.2, periodic_y=1), flags=fl,
              n_ion=50000, n_neu=50000, reinit_method="fsm", verbose=False, max_tris=65536)
    a = t3.run_etch_3d(**kw)['phi']
    b = t3.run_etch_3d(**kw)['phi']
    assert np.array_equal(a, b)


def test_batched_run_equals_per_instance_runs_exactly(det):
    from petch_b200.batch import BatchEngine
    from test_batch_gpu import FLAGS, plain_run, small_specs
    specs = small_specs()[:3]
    _lib.set_deterministic(5 * len(specs) * 65536 + 16 * 65536)
    eng = BatchEngine(specs, petch.Flags(**FLAGS), n_ion=60_000, n_neu=60_000, t_end=0.8,
                      n_steps=4, seed_offset=9, max_tris=65536)
    eng.run()
    for b, spec in enumerate(specs):
        geo = plain_run(spec, 60_000, 4, 0.8, 9)
        assert np.array_equal(eng.inst[b].phi.double().cpu().numpy(), geo['phi']), b
