"""Monte-Carlo flux kernels on the device against (a) the reference's own kernels' per-face means
(tests/golden/flux.npz, shim-executed) with a chi-square test on the per-face differences, and
(b) the FP64 oracle at high ray counts with the criterion per-face relative L2 <= 2% (plus the
measured noise floor).  Different random streams on all three sides: estimator parity."""
import ctypes
import os

import numpy as np
import pytest
import torch

import oracle.oracle as orc
from conftest import GOLDEN
from gpu_helpers import (cuda_ions, cuda_legacy, cuda_mesh, cuda_neutrals, domain, small_feature,
                         stream)
from petch_b200 import params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLDEN, "flux.npz"))


def _mesh(key, gold):
    phi, geo = small_feature(key == "hole", nx=10, ny=10, nz=14, dx=0.3)
    m = cuda_mesh(phi, geo['dx'], geo)
    np.testing.assert_array_equal(m.faces[:m.F].cpu().numpy(), gold[f"{key}_faces"])
    return m, geo, phi


def _z2(x, g, sg):
    """x: a high-ray-count device estimate; g, sg: the reference kernel's 8-seed mean and
    standard error.  Without a systematic difference z = (x - g) / sg is Student-t with 7 degrees
    of freedom: E[z^2] = 1.4, median(z^2) = 0.49."""
    k = sg > 0
    z2 = (x[k] - g[k]) ** 2 / sg[k] ** 2
    return float(np.median(z2)), float(z2.mean())


@pytest.mark.parametrize("key", ["hole", "trench"])
def test_neutral_vs_reference_kernel(gold, key):
    m, geo, _ = _mesh(key, gold)
    n = 8_000_000
    x = cuda_neutrals(m, geo, gold[f"{key}_bare"], 0.7, 1, n) / n
    med, mean = _z2(x, gold[f"{key}_neutral_mean"], gold[f"{key}_neutral_se"])
    assert med < 0.75 and mean < 2.2, (med, mean)
    assert x.sum() == pytest.approx(gold[f"{key}_neutral_mean"].sum(), rel=0.03)


@pytest.mark.parametrize("key", ["hole", "trench"])
def test_ion_vs_reference_kernel(gold, key):
    m, geo, _ = _mesh(key, gold)
    n = 8_000_000
    par = dict(params.PAR)
    x = cuda_ions(m, geo, par, 1, n).T / n
    g, sg = gold[f"{key}_ion_mean"], gold[f"{key}_ion_se"]
    for q in range(5):
        med, mean = _z2(x[q], g[q], sg[q])
        assert med < 0.75 and mean < 2.2, (q, med, mean)
        assert x[q].sum() == pytest.approx(g[q].sum(), rel=0.03)


@pytest.mark.parametrize("key", ["hole", "trench"])
def test_legacy_vs_reference_kernel(gold, key):
    m, geo, _ = _mesh(key, gold)
    n = 8_000_000
    x = np.stack(cuda_legacy(m, dict(geo, periodic_y=0), 0, 0.0, 0.2, 12, 0, 1, n)) / n
    g, sg = gold[f"{key}_legacy_mean"], gold[f"{key}_legacy_se"]
    for q in range(2):
        med, mean = _z2(x[q], g[q], sg[q])
        assert med < 0.75 and mean < 2.2, (q, med, mean)


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("hole", [True, False])
def test_neutral_vs_oracle_rel_l2(hole):
    """Per-face relative L2 <= 2% against the FP64 oracle at high ray counts (noise measured
    from two independent device runs and subtracted in quadrature)."""
    phi, geo = small_feature(hole)
    m = cuda_mesh(phi, geo['dx'], geo)
    o = orc.mesh_build(phi, geo['dx'], geo)
    rng = np.random.default_rng(0)
    bare = rng.uniform(0.1, 1.0, m.F)
    n = 4_000_000
    a = cuda_neutrals(m, geo, bare, 0.7, 11, n)
    b = cuda_neutrals(m, geo, bare, 0.7, 12, n)
    r = orc.trace_neutrals(o, geo, geo, bare, 0.7, 5, n)
    noise = _rel_l2(a, b) / np.sqrt(2)
    err = _rel_l2(0.5 * (a + b), r)
    assert np.sqrt(max(err ** 2 - 1.5 * noise ** 2, 0.0)) <= 0.02, (err, noise)


def test_neutral_wraps_above_the_surface_vs_oracle():
    """Rays that start high above a periodic trench (a gas column more than twice the lateral
    period above the mask) cross the lateral faces several times before they come down to the
    surface: the device takes those wraps in one step, the oracle one query at a time.  Per-face
    relative L2 <= 2% at high ray counts, as for the plain trench."""
    phi, geo = small_feature(False, nz=48)
    assert geo['Lz'] - (geo['sub_top'] + geo['mask_th']) > 2.0 * geo['Lx']
    m = cuda_mesh(phi, geo['dx'], geo)
    o = orc.mesh_build(phi, geo['dx'], geo)
    rng = np.random.default_rng(1)
    bare = rng.uniform(0.1, 1.0, m.F)
    n = 4_000_000
    a = cuda_neutrals(m, geo, bare, 0.7, 31, n)
    b = cuda_neutrals(m, geo, bare, 0.7, 32, n)
    r = orc.trace_neutrals(o, geo, geo, bare, 0.7, 9, n)
    noise = _rel_l2(a, b) / np.sqrt(2)
    err = _rel_l2(0.5 * (a + b), r)
    assert np.sqrt(max(err ** 2 - 1.5 * noise ** 2, 0.0)) <= 0.02, (err, noise)
    # the same share of the rays reaches the surface on both sides
    assert abs(0.5 * (a.sum() + b.sum()) / r.sum() - 1.0) < 3 * noise + 0.005, (a.sum(), r.sum())


@pytest.mark.parametrize("hole", [True, False])
def test_ion_vs_oracle_rel_l2(hole):
    phi, geo = small_feature(hole)
    m = cuda_mesh(phi, geo['dx'], geo)
    o = orc.mesh_build(phi, geo['dx'], geo)
    par = dict(params.PAR, periodic_y=geo['periodic_y'])
    n = 4_000_000
    a = cuda_ions(m, geo, par, 21, n)
    b = cuda_ions(m, geo, par, 22, n)
    r = orc.trace_ions(o, geo, par, 7, n)
    for q in range(5):
        noise = _rel_l2(a[:, q], b[:, q]) / np.sqrt(2)
        err = _rel_l2(0.5 * (a[:, q] + b[:, q]), r[:, q])
        assert np.sqrt(max(err ** 2 - 1.5 * noise ** 2, 0.0)) <= 0.02, (q, err, noise)


@pytest.mark.parametrize("width,steps,keep", [(2, 2, 0), (2, 8, 0), (2, 16, 24), (8, 4, 0),
                                              (8, 64, 12), (8, 8, 31)])
def test_tracer_configs_agree(width, steps, keep):
    """Every BVH width / steps-per-round / keep-lanes setting is the same estimator (same Philox
    paths up to float rounding of the traversal order): totals within noise, per-face within
    1 %."""
    phi, geo = small_feature(False)
    from petch_b200 import _lib
    try:
        _lib.call("petch_tracer_config", width, steps, keep)
        m = cuda_mesh(phi, geo['dx'], geo)      # the 8-wide tree is built only when configured
        x = cuda_neutrals(m, geo, None, 0.7, 7, 1_000_000)
    finally:
        _lib.call("petch_tracer_config", *_lib.TRACER_DEFAULT)
    ref = cuda_neutrals(m, geo, None, 0.7, 7, 1_000_000)
    assert _rel_l2(x, ref) < 0.01
    assert x.sum() == pytest.approx(ref.sum(), rel=1e-3)


def test_wide_traversal_without_wide_tree_fails_loudly():
    """A mesh built under the default (binary) configuration has no 8-wide tree: tracing it with
    width 8 sets error bit 8 instead of silently missing every face."""
    phi, geo = small_feature(False)
    m = cuda_mesh(phi, geo['dx'], geo)
    from petch_b200 import _lib
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    flux = torch.zeros(m.MT, device="cuda")
    try:
        _lib.call("petch_tracer_config", 8, 8, 0)
        _lib.call("petch_trace_neutrals", m.id, m.MT, m.MV, ctypes.byref(domain(geo)), None, 0.7,
                  1, 0, 1000, flux.data_ptr(), work.data_ptr(), stream())
    finally:
        _lib.call("petch_tracer_config", *_lib.TRACER_DEFAULT)
    assert work[1].item() & 8


def test_replay_same_seed_same_paths():
    """Philox streams are keyed by (seed, ray): the same seed reproduces every path; the
    per-face tallies then differ only by float-atomic summation order."""
    phi, geo = small_feature(True)
    m = cuda_mesh(phi, geo['dx'], geo)
    a = cuda_neutrals(m, geo, None, 0.7, 3, 200_000)
    b = cuda_neutrals(m, geo, None, 0.7, 3, 200_000)
    c = cuda_neutrals(m, geo, None, 0.7, 4, 200_000)
    np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-3)
    assert np.abs(a - c).max() > 1.0


@pytest.mark.parametrize("hole", [True, False])
def test_neutral_pair_equals_two_single_launches(hole):
    """petch_trace_neutral_pair (both species of a coverage round in one launch) gives each
    species exactly the tally of its own petch_trace_neutrals launch with deterministic tallies
    (same Philox paths), and the same up to float summation order without them."""
    from petch_b200 import _lib
    phi, geo = small_feature(hole)
    m = cuda_mesh(phi, geo['dx'], geo)
    rng = np.random.default_rng(2)
    bare = torch.from_numpy(rng.uniform(0.1, 1.0, m.MT).astype(np.float32)).cuda()
    n = 300_000
    dom = domain(geo)

    def single(beta, seed):
        flux = torch.zeros(m.MT, device="cuda")
        work = torch.zeros(6, dtype=torch.int32, device="cuda")
        _lib.call("petch_trace_neutrals", m.id, m.MT, m.MV, ctypes.byref(dom), bare.data_ptr(),
                  beta, seed, 0, n, flux.data_ptr(), work.data_ptr(), stream())
        assert work[1].item() == 0
        return flux[:m.F].cpu().numpy()

    def pair(count=n):
        fa = torch.full((m.MT,), 5.0, device="cuda")
        fb = torch.full((m.MT,), 5.0, device="cuda")
        work = torch.zeros(6, dtype=torch.int32, device="cuda")
        _lib.call("petch_trace_neutral_pair", m.id, m.MT, m.MV, ctypes.byref(dom),
                  bare.data_ptr(), 0.7, 1.0, 11, 12, 0, count, fa.data_ptr(), fb.data_ptr(),
                  work.data_ptr(), stream())
        assert work[1].item() == 0
        return fa[:m.F].cpu().numpy(), fb[:m.F].cpu().numpy()

    _lib.set_deterministic(64 << 20)
    try:
        a, b = single(0.7, 11), single(1.0, 12)
        pa, pb = pair()
    finally:
        _lib.set_deterministic(0)
    np.testing.assert_array_equal(pa, a)
    np.testing.assert_array_equal(pb, b)
    assert np.abs(a - b).max() > 1.0                      # two different species
    qa, qb = pair()
    np.testing.assert_allclose(qa, a, rtol=1e-5, atol=1e-3)
    np.testing.assert_allclose(qb, b, rtol=1e-5, atol=1e-3)
    za, zb = pair(0)
    assert za.max() == 0.0 and zb.max() == 0.0
    with pytest.raises(_lib.PetchError, match="must differ"):
        f = torch.zeros(m.MT, device="cuda")
        _lib.call("petch_trace_neutral_pair", m.id, m.MT, m.MV, ctypes.byref(dom), None, 0.7, 1.0,
                  1, 2, 0, 10, f.data_ptr(), f.data_ptr(), torch.zeros(6, dtype=torch.int32,
                                                                    device="cuda").data_ptr(),
                  stream())


@pytest.mark.parametrize("group", [0, 3, 4])
def test_leaf_grouping_is_bit_exact(group):
    """Leaf grouping only reorders which lanes of a warp step when; every lane's traversal is
    unchanged, so with deterministic tallies the ion and neutral tallies equal the default's
    (grouping 2) bit for bit."""
    phi, geo = small_feature(False)
    m = cuda_mesh(phi, geo['dx'], geo)
    from petch_b200 import _lib
    par = dict(params.PAR, periodic_y=1)
    bare = np.random.default_rng(5).uniform(0.05, 1.0, m.F)
    _lib.set_deterministic(8 * m.MT + (1 << 16))
    try:
        ref_n = cuda_neutrals(m, geo, bare, 0.7, 3, 400_000)
        ref_i = cuda_ions(m, geo, par, 4, 400_000)
        _lib.call("petch_tracer_grouping", group)
        got_n = cuda_neutrals(m, geo, bare, 0.7, 3, 400_000)
        got_i = cuda_ions(m, geo, par, 4, 400_000)
    finally:
        _lib.call("petch_tracer_grouping", _lib.TRACER_GROUPING_DEFAULT)
        _lib.set_deterministic(0)
    np.testing.assert_array_equal(got_n, ref_n)
    np.testing.assert_array_equal(got_i, ref_i)


def test_leaf_grouping_on_the_wide_tree_is_bit_exact():
    """The 8-wide traversal with leaf grouping (2 and 3) equals the 8-wide traversal without it,
    bit for bit with deterministic tallies."""
    from petch_b200 import _lib
    phi, geo = small_feature(False)
    par = dict(params.PAR, periodic_y=1)
    _lib.call("petch_tracer_config", 8, 32, 16)
    try:
        m = cuda_mesh(phi, geo['dx'], geo)
        bare = np.random.default_rng(6).uniform(0.05, 1.0, m.F)
        _lib.set_deterministic(8 * m.MT + (1 << 16))
        _lib.call("petch_tracer_grouping", 0)
        ref_n = cuda_neutrals(m, geo, bare, 0.7, 3, 400_000)
        ref_i = cuda_ions(m, geo, par, 4, 400_000)
        for group in (2, 3):
            _lib.call("petch_tracer_grouping", group)
            np.testing.assert_array_equal(cuda_neutrals(m, geo, bare, 0.7, 3, 400_000), ref_n)
            np.testing.assert_array_equal(cuda_ions(m, geo, par, 4, 400_000), ref_i)
    finally:
        _lib.call("petch_tracer_grouping", _lib.TRACER_GROUPING_DEFAULT)
        _lib.call("petch_tracer_config", *_lib.TRACER_DEFAULT)
        _lib.set_deterministic(0)
