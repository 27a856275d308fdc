"""Batched recipe gradients on the device (petch_trace_batch_tangent, petch_batch_advect_tangent,
petch_batch_reinit_tangent through inverse.BatchTangentEngine) against the per-instance tangent
runs (run_etch_3d_tangent): with deterministic tallies the level sets and their tangents are
identical bit for bit, from CUDA-graph replays and from direct launches."""
import numpy as np
import pytest
import torch

import petch_b200 as petch
from petch_b200 import _lib, adjoint, inverse

pytestmark = pytest.mark.gpu

FLAGS = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                    ion_reflection=True, warm_start_coverage=True)
RUN = dict(n_ion=1 << 14, n_neu=1 << 14, t_end=0.2, n_steps=4)


def small_batch(n=3, seed=5):
    specs, th = inverse.trench_batch_specs(n, seed=seed, aspect=3.0)
    return specs, th


@pytest.fixture
def deterministic():
    _lib.set_deterministic(8 * 4 * 65536 * 4)
    yield
    _lib.set_deterministic(0)


@pytest.mark.parametrize("use_graph", [True, False])
def test_batched_tangents_equal_per_instance_runs(deterministic, use_graph):
    specs, th = small_batch()
    eng = inverse.BatchTangentEngine(specs, FLAGS, seed_offset=2, **RUN)
    eng.set_thetas(th)
    eng.run(use_graph=use_graph)
    res = eng.results()
    for b, sp in enumerate(specs):
        phi, dphi, geo, _ = adjoint.run_etch_3d_tangent(
            th[b], sp['Lx'], sp['Ly'], sp['Lz'], sp['dx'], sp['trench_width'], sp['mask_th'],
            sp['sub_top'], hole=False, par=dict(petch.PAR, **sp['par']), flags=FLAGS,
            seed_offset=2, max_tris=eng.MT, **RUN)
        assert np.array_equal(res[b][0], phi), b
        assert np.array_equal(res[b][1], dphi), b
        assert np.abs(dphi).max() > 0.0                   # the tangents are not trivially zero


def test_reset_and_recapture_reproduce(deterministic):
    """Runs are repeatable; a new recipe changes the result, and the old one comes back."""
    specs, th = small_batch(2, seed=9)
    eng = inverse.BatchTangentEngine(specs, FLAGS, **RUN)
    eng.set_thetas(th)
    eng.run()
    a = [r[0].copy() for r in eng.results()]
    eng.run()
    b = [r[0] for r in eng.results()]
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    th2 = th.copy()
    th2[:, 2] *= 1.5
    eng.set_thetas(th2)
    eng.run()
    c = [r[0] for r in eng.results()]
    assert not np.array_equal(a[0], c[0])
    eng.set_thetas(th)
    eng.run()
    d = [r[0] for r in eng.results()]
    assert all(np.array_equal(x, y) for x, y in zip(a, d))


def test_inverse_design_loop_runs_and_matches_the_plain_gradient(deterministic):
    """Two Adam iterations of the batched loop; iteration 0's gradient of instance 0 equals the
    per-instance loop's."""
    specs, th = small_batch(3, seed=1)
    rng = np.random.default_rng(0)
    th_t = th * (1.0 + rng.uniform(-0.2, 0.2, th.shape))
    targets = inverse.target_profiles(specs, th_t, FLAGS, **RUN)
    assert np.isfinite(targets).any()
    grads = []
    orig = inverse.loss_and_grad

    def spy(prof, jac, target):
        L, g = orig(prof, jac, target)
        grads.append(g)
        return L, g

    inverse.loss_and_grad = spy
    try:
        out = inverse.batched_inverse_design(specs, th, targets, FLAGS, n_iter=2, **RUN)
    finally:
        inverse.loss_and_grad = orig
    assert out['loss'].shape == (2, 3) and np.all(np.isfinite(out['loss']))
    assert out['theta'].shape == (3, 3) and not np.allclose(out['theta'], th)
    plain = inverse.plain_inverse_design(specs[0], th[0], targets[0], FLAGS, n_iter=1, **RUN)
    assert np.array_equal(plain['grads'][0], grads[0])
    assert plain['loss'][0] == out['loss'][0, 0]


def test_bad_tables_fail_loudly():
    specs, th = small_batch(1)
    eng = inverse.BatchTangentEngine(specs, FLAGS, **RUN)
    g, t = eng._grids(0)
    t[0].dF = None
    with pytest.raises(_lib.PetchError, match="incomplete"):
        _lib.call("petch_batch_advect_tangent", g, t, 1, torch.cuda.current_stream().cuda_stream)
    items, tans = eng._items(True, 0)
    with pytest.raises(_lib.PetchError, match="null tangent table"):
        _lib.call("petch_trace_batch_tangent", 0, items, None, 1, eng.MT, eng.MT, 0.0, None, 9, 1,
                  eng.work.data_ptr(), torch.cuda.current_stream().cuda_stream)
    with pytest.raises(NotImplementedError):
        inverse.BatchTangentEngine(specs, petch.Flags(chemistry="belen", coverage_sticking=True))


def test_fused_extension_and_warm_start_equal_the_separate_calls():
    """petch_extend_velocity_dual / petch_warmstart_dual give the same numbers as the primal call
    followed by its tangent call."""
    from gpu_helpers import cuda_mesh, small_feature, stream
    phi, geo = small_feature(True, nx=12, ny=12, nz=16, dx=0.25)
    m1 = cuda_mesh(phi, 0.25, geo)
    phi2 = phi.copy()
    phi2[:, :, 6:] -= 0.05
    m2 = cuda_mesh(phi2, 0.25, geo, MT=m1.MT)
    MT = m1.MT
    rng = np.random.default_rng(0)
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
    V = g(rng.uniform(0, 2, MT))
    dV = g(rng.normal(size=(3, MT)))
    phid = g(phi2)
    nx, ny, nz = phi.shape
    n = phi.size
    mask = torch.zeros(n, dtype=torch.uint8, device="cuda")
    pb = g(rng.uniform(-0.2, 1.2, MT))                   # coverages outside [0, 1] included
    pdb = g(rng.normal(size=(3, MT)))
    outs = []
    for dual in (False, True):
        Fs = torch.full((n,), 7.0, device="cuda")
        dF = torch.full((3, n), 7.0, device="cuda")
        act = torch.zeros(n, dtype=torch.int32, device="cuda")
        na = torch.zeros(1, dtype=torch.int32, device="cuda")
        work = torch.zeros(6, dtype=torch.int32, device="cuda")
        if dual:
            _lib.call("petch_extend_velocity_dual", m2.id, MT, m2.MV, phid.data_ptr(),
                      mask.data_ptr(), nx, ny, nz, 0.25, 1.0, V.data_ptr(), dV.data_ptr(),
                      Fs.data_ptr(), dF.data_ptr(), 1, act.data_ptr(), na.data_ptr(), n,
                      work.data_ptr(), stream())
        else:
            _lib.call("petch_extend_velocity", m2.id, MT, m2.MV, phid.data_ptr(), mask.data_ptr(),
                      nx, ny, nz, 0.25, 1.0, V.data_ptr(), Fs.data_ptr(), 1, act.data_ptr(),
                      na.data_ptr(), n, work.data_ptr(), stream())
            _lib.call("petch_extend_tangent", m2.id, MT, m2.MV, phid.data_ptr(), nx, ny, nz, 0.25,
                      1.0, dV.data_ptr(), dF.data_ptr(), work.data_ptr(), stream())
        bare = torch.full((MT,), 7.0, device="cuda")
        dbare = torch.full((3, MT), 7.0, device="cuda")
        if dual:
            _lib.call("petch_warmstart_dual", m1.id, MT, m1.MV, pb.data_ptr(), pdb.data_ptr(),
                      m2.id, MT, m2.MV, bare.data_ptr(), dbare.data_ptr(), work.data_ptr(),
                      stream())
        else:
            _lib.call("petch_warmstart", m1.id, MT, m1.MV, pb.data_ptr(), m2.id, MT, m2.MV,
                      bare.data_ptr(), work.data_ptr(), stream())
            _lib.call("petch_warmstart_tangent", m1.id, MT, m1.MV, pb.data_ptr(), pdb.data_ptr(),
                      m2.id, MT, m2.MV, dbare.data_ptr(), work.data_ptr(), stream())
        F2 = m2.F
        outs.append((Fs.clone(), dF.clone(), bare[:F2].clone(), dbare[:, :F2].clone(),
                     int(na.item())))
        assert int(work[1].item()) == 0
    a, b = outs
    for x, y in zip(a[:4], b[:4]):
        assert torch.equal(x, y)
    assert a[4] == b[4] and a[4] > 0
