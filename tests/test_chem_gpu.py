"""Device per-face post-processing and chemistry (normalisation, smoothing, ion yields, Belen
coverages, surface rates) against the oracle's numpy restatement, on a device mesh.  Float32
flux arrays and float64 chemistry: relative tolerance 1e-5."""
import ctypes

import numpy as np
import pytest
import torch

import oracle.oracle as orc
from gpu_helpers import cuda_mesh, small_feature, stream
from petch_b200 import _lib, params
from petch_b200 import threed as t3

pytestmark = pytest.mark.gpu
RT = 1e-5


@pytest.fixture(scope="module")
def mesh():
    phi, geo = small_feature(True)
    m = cuda_mesh(phi, geo['dx'], geo)
    o = orc.mesh_build(phi, geo['dx'], geo)
    return m, o


def dev(a, n):
    t = torch.zeros(n, device="cuda")
    t[:len(a)] = torch.from_numpy(np.asarray(a, np.float32))
    return t


@pytest.mark.parametrize("n_smooth,alpha", [(1, 1.0), (2, 1.0), (1, 0.5), (0, 1.0)])
def test_norm_smooth(mesh, n_smooth, alpha):
    m, o = mesh
    rng = np.random.default_rng(1)
    fl = rng.uniform(0, 50, m.F)
    scale = 0.37
    out = torch.zeros(m.MT, device="cuda")
    ta, tb = torch.zeros(m.MT, device="cuda"), torch.zeros(m.MT, device="cuda")
    _lib.call("petch_norm_smooth", m.id, m.MT, m.MV, dev(fl, m.MT).data_ptr(), scale, 0.0, 8.0, 1,
              n_smooth, alpha, out.data_ptr(), ta.data_ptr(), tb.data_ptr(), stream())
    ref = np.clip((fl / o.area) * scale, 0, 8)
    for _ in range(n_smooth):                       # smooth_flux_dev applied n_smooth times
        ref = orc.smooth(ref, o.normal, o.pairs(), 1, alpha)
    np.testing.assert_allclose(out[:m.F].cpu().numpy(), ref, rtol=RT, atol=1e-6)


@pytest.mark.parametrize("n_smooth,alpha", [(1, 1.0), (2, 0.5)])
def test_ion_post(mesh, n_smooth, alpha):
    m, o = mesh
    rng = np.random.default_rng(2)
    tal = rng.uniform(0, 20, (m.F, 5))
    tal[::7, 3] = 0.0                              # faces no ion reached
    t4 = torch.zeros((m.MT, 4), device="cuda")
    t4[:m.F] = torch.from_numpy(tal[:, :4].astype(np.float32))
    ang = dev(tal[:, 4], m.MT)
    outs = [torch.zeros(m.MT, device="cuda") for _ in range(5)]
    tmp = torch.zeros(5 * m.MT, device="cuda")
    norm = 0.123
    _lib.call("petch_ion_post", m.id, m.MT, m.MV, t4.data_ptr(), ang.data_ptr(), norm, n_smooth,
              alpha, *[x.data_ptr() for x in outs], tmp.data_ptr(), stream())
    tal32 = tal.astype(np.float32).astype(np.float64)
    for q in range(4):
        ref = orc.smooth((tal32[:, q] / o.area) * norm, o.normal, o.pairs(), n_smooth, alpha)
        np.testing.assert_allclose(outs[q][:m.F].cpu().numpy(), ref, rtol=RT, atol=1e-6)
    fi, ai = tal32[:, 3], tal32[:, 4]
    cos_ref = np.where(fi > 0, ai / np.maximum(fi, 1e-9), 0.0)
    np.testing.assert_allclose(outs[4][:m.F].cpu().numpy(), cos_ref, rtol=RT, atol=1e-6)


@pytest.mark.parametrize("chem", ["belen", "langmuir"])
@pytest.mark.parametrize("ya", ["viennaps", "cosine"])
@pytest.mark.parametrize("with_yields", [True, False])
def test_coverage_and_rate(mesh, chem, ya, with_yields):
    if chem == "langmuir" and with_yields:
        pytest.skip("the faithful-ion yields only enter the Belen model")
    m, o = mesh
    rng = np.random.default_rng(4)
    F = m.F
    arrs = dict(m_i=rng.uniform(0, 1.5, F), m_F=rng.uniform(0, 3, F), m_O=rng.uniform(0, 3, F),
                cos_i=rng.uniform(0, 1, F))
    arrs = {k: v.astype(np.float32).astype(np.float64) for k, v in arrs.items()}
    iy = tuple(rng.uniform(0, 4, F).astype(np.float32).astype(np.float64) for _ in range(3))
    par = dict(params.PAR, ied_mode="gauss", rate_scale=0.9)
    flags = params.Flags(chemistry=chem, yield_angular=ya)
    cp = t3.chem_params(par, flags)
    d = {k: dev(v, m.MT) for k, v in arrs.items()}
    y = [dev(a, m.MT) for a in iy] if with_yields else [None, None, None]
    yp = [None if a is None else a.data_ptr() for a in y]
    bare = torch.zeros(m.MT, device="cuda")
    _lib.call("petch_belen_bare", m.id, m.MT, m.MV, ctypes.byref(cp), d['m_i'].data_ptr(),
              d['m_F'].data_ptr(), d['m_O'].data_ptr(), d['cos_i'].data_ptr(), yp[1], yp[2],
              bare.data_ptr(), stream())
    thF, thO = orc.belen_coverages(arrs['m_i'], arrs['m_F'], arrs['m_O'], arrs['cos_i'], par, ya,
                                   iy if with_yields else None)
    np.testing.assert_allclose(bare[:F].cpu().numpy(), np.clip(1 - thF - thO, 0, 1), rtol=RT,
                               atol=1e-6)
    V = torch.zeros(m.MT, device="cuda")
    stats = torch.zeros(2, dtype=torch.int32, device="cuda")
    _lib.call("petch_surface_rate", m.id, m.MT, m.MV, ctypes.byref(cp), d['m_i'].data_ptr(),
              d['m_F'].data_ptr(), d['m_O'].data_ptr(), d['cos_i'].data_ptr(), *yp,
              V.data_ptr(), stats.data_ptr(), stream())
    ref = orc.surface_rate(arrs['m_i'], arrs['m_F'], arrs['m_O'], arrs['cos_i'], o.fmask, par, chem,
                           ya, iy if with_yields else None)
    np.testing.assert_allclose(V[:F].cpu().numpy(), ref, rtol=RT, atol=1e-7)
    s = stats.cpu().numpy()
    assert s[0] == 0
    vmax = np.array([s[1]], np.int32).view(np.float32)[0]
    assert vmax == pytest.approx(ref.max(), rel=RT)
    assert o.fmask.any() and (V[:F].cpu().numpy()[o.fmask] == 0).all()


def test_nonfinite_guard(mesh):
    """A non-finite rate is zeroed and counted (run_etch_3d's warn-and-zero guard)."""
    m, _ = mesh
    F = m.F
    par = dict(params.PAR)
    cp = t3.chem_params(par, params.Flags(chemistry="belen", yield_angular="viennaps"))
    m_i = np.full(F, 0.5, np.float32)
    m_i[3] = np.nan
    d = [dev(m_i, m.MT)] + [dev(np.full(F, 0.5), m.MT) for _ in range(3)]
    V = torch.zeros(m.MT, device="cuda")
    stats = torch.zeros(2, dtype=torch.int32, device="cuda")
    _lib.call("petch_surface_rate", m.id, m.MT, m.MV, ctypes.byref(cp), *[x.data_ptr() for x in d],
              None, None, None, V.data_ptr(), stats.data_ptr(), stream())
    s = stats.cpu().numpy()
    fm = m.fmask[:F].bool().cpu().numpy()
    assert s[0] == (0 if fm[3] else 1)
    assert V[3].item() == 0.0 and torch.isfinite(V[:F]).all()
