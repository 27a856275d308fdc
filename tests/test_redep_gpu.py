"""Redeposition on the device (petch_trace_redep + petch_redep_apply) against
tests/golden/redep.npz (the reference's mc_redep_3d over 8 seeds) and the oracle loop."""
import ctypes
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_helpers import cuda_mesh, domain, small_feature, stream
from test_redep_oracle import check_redep
import oracle.oracle as orc
import petch_b200 as petch
from petch_b200 import _lib
from petch_b200 import threed as t3

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rp():
    return np.load(os.path.join(GOLDEN, "redep.npz"))


def _setup(rp, key):
    phi, geo = small_feature(key == "hole", nx=10, ny=10, nz=14, dx=0.3)
    np.testing.assert_array_equal(phi, rp[f"{key}_phi"])
    m = cuda_mesh(phi, geo['dx'], geo)
    np.testing.assert_array_equal(m.faces[:m.F].cpu().numpy(), rp[f"{key}_faces"])
    fn = torch.empty((m.MT, 3), device="cuda")
    nx, ny, nz = phi.shape
    phid = torch.from_numpy(phi).cuda()
    _lib.call("petch_gas_normals", m.id, m.MT, m.MV, phid.data_ptr(), nx, ny, nz,
              float(geo['dx']), fn.data_ptr(), stream())
    np.testing.assert_allclose(fn[:m.F].double().cpu().numpy(), rp[f"{key}_gas_normals"],
                               atol=2e-7)
    nb = ctypes.c_longlong()
    _lib.call("petch_redep_scratch_bytes", m.MT, ctypes.byref(nb))
    bufs = dict(fn=fn, cdf=torch.empty(m.MT, dtype=torch.float64, device="cuda"),
                scratch=torch.empty(max(nb.value, 1), dtype=torch.uint8, device="cuda"),
                flux=torch.empty(m.MT, device="cuda"), Rf=torch.empty(m.MT, device="cuda"),
                work=torch.zeros(6, dtype=torch.int32, device="cuda"),
                stats=torch.zeros(2, dtype=torch.int32, device="cuda"))
    return m, geo, bufs


def _redep(m, geo, b, V, n, seed, k_redep=0.0):
    Vd = torch.zeros(m.MT, device="cuda")
    Vd[:m.F] = torch.from_numpy(np.asarray(V, np.float32)).cuda()
    _lib.call("petch_trace_redep", m.id, m.MT, m.MV, ctypes.byref(domain(geo)),
              b['fn'].data_ptr(), Vd.data_ptr(), 0.5, int(seed), int(n), b['flux'].data_ptr(),
              b['cdf'].data_ptr(), b['scratch'].data_ptr(), b['scratch'].numel(),
              b['work'].data_ptr(), stream())
    _lib.call("petch_redep_apply", m.id, m.MT, m.MV, b['flux'].data_ptr(), b['cdf'].data_ptr(),
              int(n), float(k_redep), Vd.data_ptr(), b['Rf'].data_ptr(), b['stats'].data_ptr(),
              stream())
    assert b['work'][1].item() == 0
    return b['Rf'][:m.F].double().cpu().numpy(), Vd[:m.F].double().cpu().numpy()


@pytest.mark.parametrize("key", ["hole", "trench"])
def test_device_redep_matches_reference(rp, key):
    m, geo, b = _setup(rp, key)
    n = int(rp[f"{key}_n"][0])
    runs = np.stack([_redep(m, geo, b, rp[f"{key}_V"], n, 500 + s)[0] for s in range(32)])
    check_redep(runs, rp[f"{key}_mean"], rp[f"{key}_se"], rp[f"{key}_verts"], rp[f"{key}_faces"])


def test_redep_apply_updates_rate_and_max(rp):
    m, geo, b = _setup(rp, "hole")
    V = rp["hole_V"]
    Rf, Vn = _redep(m, geo, b, V, 20000, 3, k_redep=1.7)
    want = np.maximum(V.astype(np.float32) - np.float32(1.7) * Rf.astype(np.float32), 0.0)
    np.testing.assert_allclose(Vn, want, rtol=1e-6, atol=1e-6)
    vmax = np.array([b['stats'][1].item()], np.int32).view(np.float32)[0]
    assert vmax == np.float32(Vn.max())
    Rf0, V0 = _redep(m, geo, b, np.zeros(m.F), 20000, 3, k_redep=1.7)
    assert np.all(Rf0 == 0.0) and np.all(V0 == 0.0)


def test_redep_loop_depth_matches_oracle_loop():
    """With redeposition a single small-trench run scatters by several cells between seeds, so
    the centre depth averaged over 16 seeds is compared at every recorded step: device vs oracle
    (independent random streams) within one cell, or within three standard errors of the
    difference of the two means where the seed scatter is larger than that."""
    dx = 0.25
    cfg = dict(Lx=5.0, Ly=2.5, Lz=8.0, dx=dx, trench_width=2.0, mask_th=1.0, sub_top=6.0,
               t_end=1.2, n_steps=12, hole=False)
    par = dict(petch.PAR, rate_scale=0.1, periodic_y=1, k_redep=2.0)
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     ion_reflection=True, warm_start_coverage=True, redeposition=True)
    n = 60000
    dev, orc_h = [], []
    for off in range(0, 1600, 100):
        geo = t3.run_etch_3d(**cfg, par=par, flags=fl, n_ion=n, n_neu=n, reinit_method="fsm",
                             verbose=False, record_depth_every=3, seed_offset=off)
        dev.append(dict(geo['depth_history']))
        _, hist, _ = orc.run_etch_3d(cfg['Lx'], cfg['Ly'], cfg['Lz'], dx, cfg['trench_width'],
                                     cfg['mask_th'], cfg['sub_top'], cfg['t_end'],
                                     cfg['n_steps'], False, par, fl, n, n, seed_offset=off,
                                     record_depth_every=3)
        orc_h.append(dict(hist))
    steps = sorted(orc_h[0])
    for s in steps:
        a = np.array([h[s] for h in dev])
        b = np.array([h[s] for h in orc_h])
        se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
        assert abs(a.mean() - b.mean()) <= max(dx, 3.0 * se) + 1e-9, (s, a.mean(), b.mean(), se)
    assert np.mean([h[steps[-1]] for h in orc_h]) > 2 * dx
