"""run_etch_3d's non-default level-set options on the device: petch_reinit_pde
(reinit_method='gpu'), petch_gaussian_smooth (surf_smooth) and petch_extend_velocity_centroid
(extend != 'gpu'), against tests/golden/options.npz (the reference's own functions), scipy's
gaussian_filter (the reference's own call) and the oracle loop."""
import ctypes
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_helpers import cuda_mesh, small_feature, stream
import oracle.oracle as orc
import petch_b200 as petch
from petch_b200 import _lib
from petch_b200 import threed as t3
from petch_b200.levelset import gaussian_smooth_dev, reinit_pde_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def op():
    return np.load(os.path.join(GOLDEN, "options.npz"))


@pytest.mark.parametrize("name", ["hole", "trench"])
def test_reinit_pde_matches_reference(op, name):
    dx = float(op[f"{name}_pde_dx"][0])
    phi = torch.from_numpy(op[f"{name}_pde_in"]).cuda()
    out = reinit_pde_dev(phi, dx).double().cpu().numpy()
    np.testing.assert_allclose(out, op[f"{name}_pde_out"], rtol=2e-5, atol=2e-6 * dx)
    np.testing.assert_allclose(out, orc.reinit_pde(op[f"{name}_pde_in"], dx), rtol=1e-5,
                               atol=1e-6 * dx)


def test_reinit_pde_in_place_and_zero_iterations(op):
    dx = float(op["hole_pde_dx"][0])
    phi = torch.from_numpy(op["hole_pde_in"]).cuda()
    ref = reinit_pde_dev(phi.clone(), dx, n_iter=5)
    p2 = phi.clone()
    reinit_pde_dev(p2, dx, n_iter=5, out=p2)
    assert torch.equal(p2, ref)
    assert torch.equal(reinit_pde_dev(phi, dx, n_iter=0), phi)


@pytest.mark.parametrize("sigma,shape", [(0.5, (20, 16, 24)), (1.0, (17, 9, 33)),
                                         (2.3, (12, 5, 40))])
def test_gaussian_smooth_matches_scipy(sigma, shape):
    """Includes an axis shorter than the filter radius (reflection past both ends)."""
    rng = np.random.default_rng(int(10 * sigma))
    phi = rng.normal(size=shape).astype(np.float32)
    mask = rng.random(shape) < 0.1
    mp = rng.normal(size=shape).astype(np.float32)
    d = torch.from_numpy(phi).cuda()
    gaussian_smooth_dev(d, sigma, torch.from_numpy(mask.astype(np.uint8)).cuda(),
                        torch.from_numpy(mp).cuda())
    ref = orc.gaussian_smooth(phi, sigma, mask, mp)
    np.testing.assert_allclose(d.double().cpu().numpy(), ref, rtol=0, atol=2e-6)


def test_gaussian_smooth_rejects_oversized_radius():
    d = torch.zeros((4, 4, 4), device="cuda")
    with pytest.raises(_lib.PetchError):
        gaussian_smooth_dev(d, 40.0)


def test_extend_nearest_centroid_matches_reference(op):
    phi, geo = small_feature(True)
    np.testing.assert_array_equal(phi, op["ext_phi"])
    m = cuda_mesh(phi, geo['dx'], geo)
    np.testing.assert_array_equal(m.faces[:m.F].cpu().numpy(), op["ext_faces"])
    dx, band = op["ext_args"]
    nx, ny, nz = phi.shape
    V = torch.zeros(m.MT, device="cuda")
    V[:m.F] = torch.from_numpy(op["ext_V"].astype(np.float32)).cuda()
    Fs = torch.empty(phi.shape, device="cuda")
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    phid = torch.from_numpy(phi).cuda()
    _lib.call("petch_extend_velocity_centroid", m.id, m.MT, m.MV, phid.data_ptr(), None, nx, ny,
              nz, float(dx), float(band), V.data_ptr(), Fs.data_ptr(), 0, None, None, 0,
              work.data_ptr(), stream())
    got = Fs.double().cpu().numpy()
    want = op["ext_Fs"].astype(np.float32).astype(np.float64)
    diff = np.argwhere(got != want)
    # where the two disagree the two centroids must be equidistant (a float32 tie)
    c = op["ext_centroids"]
    for i, j, k in diff:
        p = np.array([i, j, k]) * dx
        d = np.linalg.norm(c - p, axis=1)
        cand = np.flatnonzero(np.abs(d - d.min()) < 1e-5)
        assert got[i, j, k] in op["ext_V"][cand].astype(np.float32), (i, j, k)
    # the symmetric hole has many exactly equidistant centroids (cKDTree and the device break
    # such ties differently); every disagreement above was checked to be one
    assert len(diff) <= 0.05 * np.count_nonzero(want)


def test_loop_with_options_matches_oracle_loop():
    """reinit_method='gpu', extend='cpu' (nearest centroid) and surf_smooth=0.6 together, through
    the device engine and the oracle loop: centre depth within one grid cell."""
    dx = 0.25
    cfg = dict(Lx=5.0, Ly=5.0, Lz=8.0, dx=dx, trench_width=2.0, mask_th=1.0, sub_top=6.0,
               t_end=1.2, n_steps=12, hole=True)
    par = dict(petch.PAR, rate_scale=0.3, periodic_y=0)
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     ion_reflection=True, warm_start_coverage=True)
    n = 60000
    geo = t3.run_etch_3d(**cfg, par=par, flags=fl, n_ion=n, n_neu=n, reinit_method="gpu",
                         extend="cpu", surf_smooth=0.6, verbose=False, record_depth_every=3)
    dev_hist = dict(geo['depth_history'])
    _, hist, _ = orc.run_etch_3d(cfg['Lx'], cfg['Ly'], cfg['Lz'], dx, cfg['trench_width'],
                                 cfg['mask_th'], cfg['sub_top'], cfg['t_end'], cfg['n_steps'],
                                 True, par, fl, n, n, record_depth_every=3, reinit_method="gpu",
                                 extend="cpu", surf_smooth=0.6)
    orc_hist = dict(hist)
    assert set(dev_hist) == set(orc_hist)
    for s in sorted(orc_hist):
        assert abs(dev_hist[s] - orc_hist[s]) <= dx + 1e-9, (s, dev_hist[s], orc_hist[s])
    assert max(orc_hist.values()) > 2 * dx
