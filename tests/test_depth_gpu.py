"""The depth metrics on the engine's device level set (petch_column_floors: the column scan on
the device, only the floor indices read back) against the host scan of the same float32 field."""
import numpy as np
import pytest
import torch

from petch_b200 import _lib
from petch_b200 import threed as t3
from test_depth_metrics import _field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("hole", [True, False])
@pytest.mark.parametrize("shape", [(24, 20, 40), (16, 12, 200), (10, 10, 33)])
def test_device_scan_equals_host_scan(hole, shape):
    rng = np.random.default_rng(sum(shape))
    nx, ny, nz = shape
    dx = 0.25
    phi = _field(rng, nx, ny, nz, dx).astype(np.float32)
    g = dict(Lx=nx * dx, Ly=ny * dx, dx=dx, sub_top=nz * dx * 0.8, trench_width=2.0, hole=hole,
             xs=np.arange(nx) * dx, ys=np.arange(ny) * dx, zs=np.arange(nz) * dx)
    host = dict(g, phi=phi.astype(np.float64))
    dev = dict(g, phi=torch.from_numpy(phi).cuda())
    for half in (1.0, 0.4):
        assert t3.center_depth_3d(dev, half) == t3.center_depth_3d(host, half)
    assert t3.max_depth_3d(dev) == t3.max_depth_3d(host)
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    np.testing.assert_array_equal(t3._floor_indices(dev['phi'], ii, jj),
                                  t3._floor_indices(host['phi'], ii, jj))


def test_out_of_grid_column_raises():
    phi = torch.zeros((4, 4, 8), device="cuda")
    with pytest.raises(ValueError, match="outside the grid"):
        t3._floor_indices(phi, [0, 4], [0, 0])
    with pytest.raises(_lib.PetchError, match="bad size"):
        _lib.call("petch_column_floors", phi.data_ptr(), 0, 4, 8, None, 0, None,
                  torch.cuda.current_stream().cuda_stream)
