"""The batched forward (petch_b200.batch.BatchEngine: petch_trace_batch, petch_batch_advect,
petch_batch_reinit, whole steps replayed from CUDA graphs) against the plain per-instance loop
(run_etch_3d with the same per-instance parameters and seeds).  A batched ray draws the Philox
stream of the same ray in its instance's own run, so the two differ only by the summation order
of float atomics."""
import ctypes

import numpy as np
import pytest
import torch

from gpu_helpers import cuda_mesh, domain, small_feature, stream
import petch_b200 as petch
from petch_b200 import _lib
from petch_b200 import threed as t3
from petch_b200.batch import BatchEngine, hole_batch_specs

pytestmark = pytest.mark.gpu

FLAGS = dict(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
             warm_start_coverage=True, ion_reflection=True)


def small_specs():
    """Four small ragged holes with different recipes (a scaled-down hole batch)."""
    specs = hole_batch_specs(n=4, seed=3, dx=0.25, Lz=8.0, headroom=2.0)
    for s in specs:
        d = 1.0 + s['trench_width'] / 4.0
        s['trench_width'] = d
        s['Lx'] = s['Ly'] = round((d + 3.0) / 0.25) * 0.25
        s['mask_th'] = 0.5 + s['mask_th'] / 6.0
        s['sub_top'] = 8.0 - 2.0 - s['mask_th']
        s['par']['rate_scale'] = 0.2
    return specs


def plain_run(spec, n_rays, n_steps, t_end, seed_offset):
    par = dict(petch.PAR, **spec['par'])
    geo = t3.run_etch_3d(Lx=spec['Lx'], Ly=spec['Ly'], Lz=spec['Lz'], dx=spec['dx'],
                         trench_width=spec['trench_width'], mask_th=spec['mask_th'],
                         sub_top=spec['sub_top'], hole=True, t_end=t_end, n_steps=n_steps,
                         par=par, flags=petch.Flags(**FLAGS), n_ion=n_rays, n_neu=n_rays,
                         reinit_method="fsm", verbose=False, seed_offset=seed_offset,
                         record_depth_every=1)
    return geo


def test_batched_steps_follow_the_per_instance_runs():
    specs = small_specs()
    n_rays, n_steps, t_end = 100_000, 5, 1.0
    eng = BatchEngine(specs, petch.Flags(**FLAGS), n_ion=n_rays, n_neu=n_rays, t_end=t_end,
                      n_steps=n_steps, seed_offset=7)
    launches = eng.capture()
    assert launches["warm0"] > 0
    eng.run(record_depth_every=1)
    assert int(eng.work[2].item()) + (int(eng.work[3].item()) << 32) > 0   # BVH queries made
    for b, spec in enumerate(specs):
        geo = plain_run(spec, n_rays, n_steps, t_end, 7)
        dev = dict(eng.depth_history[b])
        ref = dict(geo['depth_history'])
        assert set(dev) == set(ref)
        for s in sorted(ref):
            assert abs(dev[s] - ref[s]) <= spec['dx'] + 1e-9, (b, s, dev[s], ref[s])
    # With float-atomic tallies the two runs part after the first coverage round: the per-face
    # sums differ in rounding, the coverage feeds the Russian-roulette decisions, and from then
    # on the paths differ at Monte-Carlo noise level.  That the batch draws exactly the streams
    # of the per-instance runs is checked with deterministic tallies
    # (test_deterministic_gpu.py::test_batched_run_equals_per_instance_runs_exactly).


def test_batched_trace_equals_per_instance_traces():
    """One petch_trace_batch launch over three meshes (a common capacity) against the
    single-instance tracers with the seeds the batch derives: identical per-face tallies up to
    the order of float atomic additions."""
    par = dict(petch.PAR)
    feats = [small_feature(True), small_feature(False), small_feature(True, nx=12, ny=12, nz=16)]
    MT = 65536
    meshes = [cuda_mesh(phi, geo['dx'], geo, MT=MT) for phi, geo in feats]
    rng = np.random.default_rng(4)
    step = torch.tensor([3], dtype=torch.int32, device="cuda")
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    n = 200_000
    for kind in (0, 1):
        items = (_lib.BatchItem * 3)()
        outs, angs, bares = [], [], []
        for b, (m, (phi, geo)) in enumerate(zip(meshes, feats)):
            out = torch.zeros((MT, 4) if kind == 0 else MT, device="cuda")
            ang = torch.zeros(MT, device="cuda")
            bare = torch.from_numpy(rng.uniform(0.2, 1.0, MT).astype(np.float32)).cuda()
            it = items[b]
            it.mesh, it.dom, it.ion = m.id, domain(geo), t3.ion_params(dict(par, Emean=80.0 + 40 * b))
            it.bare, it.out, it.ang = bare.data_ptr(), out.data_ptr(), ang.data_ptr()
            it.n_rays, it.seed = n + 1000 * b, 10 * b
            outs.append(out)
            angs.append(ang)
            bares.append(bare)
        _lib.call("petch_trace_batch", kind, items, 3, MT, MT, 0.7, step.data_ptr(), 9, 2,
                  work.data_ptr(), stream())
        assert work[1].item() == 0
        for b, (m, (phi, geo)) in enumerate(zip(meshes, feats)):
            seed = (3 + 10 * b) * 9 + 2
            if kind == 0:
                tal = torch.zeros((MT, 4), device="cuda")
                ang = torch.zeros(MT, device="cuda")
                _lib.call("petch_trace_ions", m.id, m.MT, m.MV, ctypes.byref(domain(geo)),
                          ctypes.byref(t3.ion_params(dict(par, Emean=80.0 + 40 * b))), seed,
                          n + 1000 * b, tal.data_ptr(), ang.data_ptr(), work.data_ptr(), stream())
                got = torch.cat([outs[b][:m.F], angs[b][:m.F, None]], 1)
                want = torch.cat([tal[:m.F], ang[:m.F, None]], 1)
            else:
                flux = torch.zeros(MT, device="cuda")
                _lib.call("petch_trace_neutrals", m.id, m.MT, m.MV, ctypes.byref(domain(geo)),
                          bares[b].data_ptr(), 0.7, seed, 0, n + 1000 * b, flux.data_ptr(),
                          work.data_ptr(), stream())
                got, want = outs[b][:m.F], flux[:m.F]
            got, want = got.double().cpu().numpy(), want.double().cpu().numpy()
            scale = np.abs(want).max()
            np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-5 * scale)


def test_graph_replay_equals_eager_launches():
    specs = small_specs()[:2]
    kw = dict(n_ion=50_000, n_neu=50_000, t_end=0.6, n_steps=3, seed_offset=2)
    a = BatchEngine(specs, petch.Flags(**FLAGS), **kw)
    a.run(use_graph=True)
    b = BatchEngine(specs, petch.Flags(**FLAGS), **kw)
    b.run(use_graph=False)
    for x, y in zip(a.inst, b.inst):
        d = (x.phi - y.phi).abs()
        band = y.phi.abs() < 1.0
        assert float(d[band].median()) < 1e-4


def test_batch_rejects_unsupported_configurations():
    specs = small_specs()[:1]
    with pytest.raises(NotImplementedError):
        BatchEngine(specs, petch.Flags(chemistry="langmuir"))
    bad = [dict(specs[0]), dict(specs[0], dx=0.2)]
    with pytest.raises(ValueError):
        BatchEngine(bad, petch.Flags(**FLAGS))


def test_batched_pair_equals_per_instance_single_launches():
    """petch_trace_batch_pair (both neutral species of every instance in one launch) against the
    per-instance single-species tracers with the seeds the batch derives: bit-equal with
    deterministic tallies."""
    feats = [small_feature(True), small_feature(False), small_feature(True, nx=12, ny=12, nz=16)]
    MT = 65536
    meshes = [cuda_mesh(phi, geo['dx'], geo, MT=MT) for phi, geo in feats]
    rng = np.random.default_rng(6)
    step = torch.tensor([5], dtype=torch.int32, device="cuda")
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    n = 100_000
    bares = [torch.from_numpy(rng.uniform(0.2, 1.0, MT).astype(np.float32)).cuda() for _ in meshes]
    fa = [torch.full((MT,), 3.0, device="cuda") for _ in meshes]
    fb = [torch.full((MT,), 3.0, device="cuda") for _ in meshes]
    items = (_lib.BatchItem * 3)()
    for b, (m, (phi, geo)) in enumerate(zip(meshes, feats)):
        it = items[b]
        it.mesh, it.dom, it.ion = m.id, domain(geo), t3.ion_params(dict(petch.PAR))
        it.bare, it.out, it.ang = bares[b].data_ptr(), fa[b].data_ptr(), fb[b].data_ptr()
        it.n_rays, it.seed = n + 500 * b, 7 * b
    _lib.set_deterministic(64 << 20)
    try:
        _lib.call("petch_trace_batch_pair", items, 3, MT, MT, 0.7, 1.0, step.data_ptr(), 9, 2, 3,
                  work.data_ptr(), stream())
        assert work[1].item() == 0
        for b, (m, (phi, geo)) in enumerate(zip(meshes, feats)):
            for beta, add, got in ((0.7, 2, fa[b]), (1.0, 3, fb[b])):
                flux = torch.zeros(MT, device="cuda")
                _lib.call("petch_trace_neutrals", m.id, m.MT, m.MV, ctypes.byref(domain(geo)),
                          bares[b].data_ptr(), beta, (5 + 7 * b) * 9 + add, 0, n + 500 * b,
                          flux.data_ptr(), work.data_ptr(), stream())
                assert torch.equal(got[:m.F], flux[:m.F]), (b, beta)
                assert flux[:m.F].abs().max().item() > 0.0
    finally:
        _lib.set_deterministic(0)
    items[0].ang = items[0].out
    with pytest.raises(_lib.PetchError, match="second flux"):
        _lib.call("petch_trace_batch_pair", items, 3, MT, MT, 0.7, 1.0, None, 9, 2, 3,
                  work.data_ptr(), stream())
