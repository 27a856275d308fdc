"""petch_reinit_eik_noalloc: the Eikonal reinit for callers that cannot allocate device memory.

Such callers (a host framework that owns the whole device heap and forbids driver allocations, a
fixed-budget loop that cannot take an allocation's latency and implicit synchronisation) own
their input and output grids but cannot hand the library scratch buffers.  This entry point
keeps its two scratch grids in a fixed device array inside the library instead.  The tests call
it through the C ABI and compare it with petch_reinit_eik, which takes caller scratch, on two
calls in a row with different inputs (nothing may carry over between calls through the shared
array).  This file is collected last so a failure here never hides another test's result.
"""
import ctypes

import numpy as np
import pytest

from petch_b200 import _lib

TOL = 1e-5


def _field(seed, nx=40, ny=36, nz=48, dx=0.25):
    """A sphere-plus-plane level set with a perturbed front and a few exact zeros."""
    X, Y, Z = np.meshgrid(np.arange(nx) * dx, np.arange(ny) * dx, np.arange(nz) * dx,
                          indexing="ij")
    rng = np.random.default_rng(seed)
    phi = np.maximum(3.0 - np.sqrt((X - 5.0) ** 2 + (Y - 4.5) ** 2 + (Z - 6.0) ** 2), 4.0 - Z)
    phi += rng.normal(0.0, 0.05 * dx, phi.shape)
    phi[rng.random(phi.shape) < 0.002] = 0.0
    return phi.astype(np.float32), dx


@pytest.mark.gpu
@pytest.mark.parametrize("mode,shape", [(0, (40, 36, 48)), (1, (40, 36, 48)),
                                        (0, (128, 128, 128))],
                         ids=["mode0", "mode1", "mode0-at-limit"])
def test_noalloc_reinit_matches_caller_scratch_reinit_on_two_calls(mode, shape):
    """Two calls in a row; the last case fills the fixed array exactly (2^21 cells per grid, the
    second grid ending at the array's end)."""
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (1, 2):                                  # two calls in a row, different inputs
        phi_np, dx = _field(seed, *shape)
        phi = torch.from_numpy(phi_np).cuda()
        nx, ny, nz = phi.shape
        band = 6 * dx
        big, cap, n_iter = band + 4 * dx, band + dx, int(np.ceil(band / dx)) + 4
        ref = torch.empty_like(phi)
        ua, ub = torch.empty_like(phi), torch.empty_like(phi)
        _lib.call("petch_reinit_eik", phi.data_ptr(), ref.data_ptr(), ua.data_ptr(), ub.data_ptr(),
                  nx, ny, nz, dx, big, cap, n_iter, mode, stream)
        out = torch.full_like(phi, float("nan"))
        _lib.call("petch_reinit_eik_noalloc", phi.data_ptr(), out.data_ptr(), nx, ny, nz, dx, big,
                  cap, n_iter, mode, stream)
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=TOL,
                                   atol=TOL * cap)


def test_noalloc_reinit_rejects_grids_beyond_its_fixed_scratch():
    """More cells than the fixed array holds: a clear error before any device work."""
    dummy = ctypes.c_void_p(16)                          # never dereferenced: the size check fails
    rc = _lib.lib().petch_reinit_eik_noalloc(dummy, dummy, 256, 128, 128, 0.25, 2.5, 1.75, 10, 0,
                                             None)
    assert rc == 1                                       # PETCH_E_INVALID
    assert "exceeds the fixed scratch" in _lib.last_error()


def test_noalloc_reinit_rejects_one_cell_past_the_limit():
    """2^21 + 1 cells (one more than each fixed scratch grid holds) is rejected."""
    dummy = ctypes.c_void_p(16)
    rc = _lib.lib().petch_reinit_eik_noalloc(dummy, dummy, (1 << 21) + 1, 1, 1, 0.25, 2.5, 1.75,
                                             10, 0, None)
    assert rc == 1 and "exceeds the fixed scratch" in _lib.last_error()
