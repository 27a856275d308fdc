"""Both neutral species of a coverage round with their weight tangents in one launch:
petch_trace_neutral_pair_tangent (single instance) and petch_trace_batch_pair_tangent (batched)
against the one-species tangent tracer per species, bit for bit with deterministic tallies."""
import ctypes

import numpy as np
import pytest
import torch

import petch_b200 as petch
from gpu_helpers import cuda_mesh, domain, small_feature, stream
from petch_b200 import _lib
from petch_b200 import threed as t3

pytestmark = pytest.mark.gpu


def _single(m, geo, bare, dbare, beta, seed, n):
    flux = torch.zeros(m.MT, device="cuda")
    dflux = torch.zeros((3, m.MT), device="cuda")
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    _lib.call("petch_trace_neutrals_tangent", m.id, m.MT, m.MV, ctypes.byref(domain(geo)),
              bare.data_ptr(), dbare.data_ptr(), beta, seed, 0, n, flux.data_ptr(),
              dflux.data_ptr(), work.data_ptr(), stream())
    assert work[1].item() == 0
    return flux[:m.F].clone(), dflux[:, :m.F].clone()


@pytest.fixture
def det():
    _lib.set_deterministic(64 << 20)
    yield
    _lib.set_deterministic(0)


def _inputs(m, seed):
    rng = np.random.default_rng(seed)
    bare = torch.from_numpy(rng.uniform(0.1, 1.0, m.MT).astype(np.float32)).cuda()
    dbare = torch.from_numpy(rng.normal(0.0, 0.2, (3, m.MT)).astype(np.float32)).cuda()
    return bare, dbare


@pytest.mark.parametrize("hole", [True, False])
def test_pair_tangent_equals_single_tangent_launches(det, hole):
    phi, geo = small_feature(hole)
    m = cuda_mesh(phi, geo['dx'], geo)
    bare, dbare = _inputs(m, 1)
    n = 200_000
    fa = torch.zeros(m.MT, device="cuda")
    fb = torch.zeros(m.MT, device="cuda")
    da = torch.zeros((3, m.MT), device="cuda")
    db = torch.zeros((3, m.MT), device="cuda")
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    _lib.call("petch_trace_neutral_pair_tangent", m.id, m.MT, m.MV, ctypes.byref(domain(geo)),
              bare.data_ptr(), dbare.data_ptr(), 0.7, 1.0, 21, 22, 0, n, fa.data_ptr(),
              da.data_ptr(), fb.data_ptr(), db.data_ptr(), work.data_ptr(), stream())
    assert work[1].item() == 0
    for beta, seed, f, d in ((0.7, 21, fa, da), (1.0, 22, fb, db)):
        sf, sd = _single(m, geo, bare, dbare, beta, seed, n)
        assert torch.equal(f[:m.F], sf) and torch.equal(d[:, :m.F], sd), beta
        assert sd.abs().max().item() > 0.0
    with pytest.raises(_lib.PetchError, match="must differ"):
        _lib.call("petch_trace_neutral_pair_tangent", m.id, m.MT, m.MV, ctypes.byref(domain(geo)),
                  bare.data_ptr(), dbare.data_ptr(), 0.7, 1.0, 21, 22, 0, 10, fa.data_ptr(),
                  da.data_ptr(), fb.data_ptr(), da.data_ptr(), work.data_ptr(), stream())


def test_batched_pair_tangent_equals_single_tangent_launches(det):
    feats = [small_feature(True), small_feature(False)]
    MT = 65536
    meshes = [cuda_mesh(phi, geo['dx'], geo, MT=MT) for phi, geo in feats]
    step = torch.tensor([4], dtype=torch.int32, device="cuda")
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    n = 80_000
    items = (_lib.BatchItem * 2)()
    ta = (_lib.BatchTangent * 2)()
    tb = (_lib.BatchTangent * 2)()
    keep = []
    for b, (m, (phi, geo)) in enumerate(zip(meshes, feats)):
        bare, dbare = _inputs(m, 10 + b)
        fa, fb = torch.zeros(MT, device="cuda"), torch.zeros(MT, device="cuda")
        da, db = torch.zeros((3, MT), device="cuda"), torch.zeros((3, MT), device="cuda")
        it = items[b]
        it.mesh, it.dom, it.ion = m.id, domain(geo), t3.ion_params(dict(petch.PAR))
        it.bare, it.out, it.ang = bare.data_ptr(), fa.data_ptr(), fb.data_ptr()
        it.n_rays, it.seed = n + 300 * b, 5 * b
        ta[b].dout, ta[b].dbare = da.data_ptr(), dbare.data_ptr()
        tb[b].dout = db.data_ptr()
        keep.append((bare, dbare, fa, fb, da, db))
    _lib.call("petch_trace_batch_pair_tangent", items, ta, tb, 2, MT, MT, 0.7, 1.0,
              step.data_ptr(), 9, 2, 3, work.data_ptr(), stream())
    assert work[1].item() == 0
    for b, (m, (phi, geo)) in enumerate(zip(meshes, feats)):
        bare, dbare, fa, fb, da, db = keep[b]
        for beta, add, f, d in ((0.7, 2, fa, da), (1.0, 3, fb, db)):
            sf, sd = _single(m, geo, bare, dbare, beta, (4 + 5 * b) * 9 + add, n + 300 * b)
            assert torch.equal(f[:m.F], sf) and torch.equal(d[:, :m.F], sd), (b, beta)
    with pytest.raises(_lib.PetchError, match="second tangent"):
        _lib.call("petch_trace_batch_pair_tangent", items, ta, None, 2, MT, MT, 0.7, 1.0, None, 9,
                  2, 3, work.data_ptr(), stream())
