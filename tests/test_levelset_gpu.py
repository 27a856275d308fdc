"""CUDA level-set stages (through the C ABI) against the FP64 oracle and the reference's golden
vectors.  Deterministic stages: |cuda - oracle| <= 1e-5 * scale (FP32 arithmetic vs FP64)."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
import oracle.oracle as orc
from petch_b200 import levelset as ls

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def lv():
    return np.load(os.path.join(GOLDEN, "levelset.npz"))


def cuda(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


@pytest.mark.parametrize("name", ["hole", "trench"])
def test_seed_field_bitwise(lv, name):
    nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole = lv[f"{name}_seed_args"]
    phi, mask = ls.seed_field(int(nx), int(ny), int(nz), dx, Lx, Ly, sub_top, mask_th, width,
                              bool(hole))
    np.testing.assert_array_equal(phi.cpu().numpy(), lv[f"{name}_csg"])
    np.testing.assert_array_equal(mask.bool().cpu().numpy(), lv[f"{name}_mask"])


@pytest.mark.parametrize("name", ["hole", "trench"])
def test_reinit_vs_reference_golden(lv, name):
    dx = float(lv[f"{name}_seed_args"][3])
    band = float(lv[f"{name}_reinit_band"][0])
    out = ls.reinit_fsm_dev(cuda(lv[f"{name}_csg"]), dx, band).cpu().numpy()
    ref = lv[f"{name}_reinit"]
    np.testing.assert_allclose(out, ref, rtol=TOL, atol=TOL * (band + dx))


def test_reinit_short_sweeps_with_zero_nodes(lv):
    dx, band, n_iter = lv["noisy_args"]
    out = ls.reinit_fsm_dev(cuda(lv["noisy_phi"]), dx, band, int(n_iter)).cpu().numpy()
    np.testing.assert_allclose(out, lv["noisy_reinit"], rtol=TOL, atol=TOL * (band + dx))


@pytest.mark.parametrize("name", ["hole", "trench"])
def test_advect_vs_reference_golden(lv, name):
    dx, dt_sub, nsub = lv[f"{name}_adv_args"]
    phi = cuda(lv[f"{name}_reinit"])
    ls.advect_dev(phi, cuda(lv[f"{name}_F"]), cuda(lv[f"{name}_mask"], torch.uint8),
                  cuda(lv[f"{name}_csg"]), dx, dt_sub, int(nsub))
    np.testing.assert_allclose(phi.cpu().numpy(), lv[f"{name}_advect"], rtol=TOL, atol=TOL * 2.0)


def _c0_field():
    """Config-0 hole grid (56 x 56 x 96, dx 0.25) seeded and redistanced by the oracle."""
    dx = 0.25
    phi, mask = orc.seed(56, 56, 96, dx, 14.0, 14.0, 18.0, 2.0, 6.0, True)
    phi = orc.reinit(phi.astype(np.float32), dx, 24 * dx, 28)
    return phi.astype(np.float32), mask, dx


def test_reinit_config0_grid_vs_oracle():
    phi, _, dx = _c0_field()
    band = 4 * dx + 2.0 * dx
    rng = np.random.default_rng(0)
    phi = (phi + rng.normal(0, 0.05 * dx, phi.shape)).astype(np.float32)   # a perturbed front
    ref = orc.reinit(phi, dx, band)
    out = ls.reinit_fsm_dev(cuda(phi), dx, band).cpu().numpy()
    np.testing.assert_allclose(out, ref, rtol=TOL, atol=TOL * (band + dx))


@pytest.mark.parametrize("nsub", [1, 4, 7])
def test_advect_config0_grid_vs_oracle(nsub):
    phi, mask, dx = _c0_field()
    rng = np.random.default_rng(nsub)
    F = np.where(np.abs(phi) < 4 * dx, rng.uniform(0.0, 40.0, phi.shape), 0.0).astype(np.float32)
    dt_sub = 0.4 * dx / 40.0
    ref = orc.advect(phi, F, mask, phi, 1.0 / dx, dt_sub, nsub)
    p = cuda(phi)
    ls.advect_dev(p, cuda(F), cuda(mask, torch.uint8), cuda(phi), dx, dt_sub, nsub)
    np.testing.assert_allclose(p.cpu().numpy(), ref, rtol=TOL, atol=TOL * 8 * dx)
    # folded encoding: F < 0 marks the mask cells, no mask array
    Ff = np.where(mask, -1.0, F).astype(np.float32)
    p2 = cuda(phi)
    ls.advect_dev(p2, cuda(Ff), None, cuda(phi), dx, dt_sub, nsub)
    np.testing.assert_array_equal(p2.cpu().numpy(), p.cpu().numpy())
