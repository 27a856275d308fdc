"""Level-set stages on the device: the seed field (make_trench_3d), upwind advection
(advect_3d_gpu) and the Jacobi Godunov-Eikonal reinit (reinit_fsm).

Each function mirrors the reference signature (petch/threed.py) and accepts either numpy arrays
(then returns float64 numpy, as the reference does) or CUDA tensors (then stays on the device and
returns float32 tensors).  All arithmetic runs in the CUDA library; nothing is computed on the host
except the scalar parameters, which follow the reference's float64 host formulas.
"""
import numpy as np
import torch

from . import _lib


def _dev(x, dtype=torch.float32):
    if isinstance(x, torch.Tensor):
        return x.to(device="cuda", dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(x)).to(device="cuda", dtype=dtype)


def grid_shape(Lx, Ly, Lz, dx):
    """make_trench_3d's node counts (threed.py:34)."""
    return int(round(Lx / dx)), int(round(Ly / dx)), int(round(Lz / dx))


def seed_field(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole, stream=None):
    """Analytic CSG field (float32) and uint8 mask on the device (threed.py:34-55)."""
    phi = torch.empty((nx, ny, nz), dtype=torch.float32, device="cuda")
    mask = torch.empty((nx, ny, nz), dtype=torch.uint8, device="cuda")
    _lib.call("petch_seed_level_set", _lib.ptr(phi), _lib.ptr(mask), nx, ny, nz, float(dx),
              float(Lx), float(Ly), float(sub_top), float(mask_th), float(width), int(bool(hole)),
              _lib.stream_ptr(stream))
    return phi, mask


def reinit_fsm_dev(phi, dx, band, n_iter=None, out=None, scratch=None, stream=None, mode=0):
    """reinit_fsm on a CUDA float32 grid (threed.py:1515-1537); returns the redistanced grid.
    mode=1: the seed-field variant (zero nodes frozen on the front, see petch_reinit_eik)."""
    if n_iter is None:
        n_iter = int(np.ceil(band / dx)) + 4
    big = float(band + 4.0 * dx)
    cap = float(band + dx)
    nx, ny, nz = phi.shape
    if out is None:
        out = torch.empty_like(phi)
    if scratch is None:
        scratch = (torch.empty_like(phi), torch.empty_like(phi))
    _lib.call("petch_reinit_eik", _lib.ptr(phi), _lib.ptr(out), _lib.ptr(scratch[0]),
              _lib.ptr(scratch[1]), nx, ny, nz, float(dx), big, cap, int(n_iter), int(mode),
              _lib.stream_ptr(stream))
    return out


def advect_dev(phi, F, mask, mask_phi, dx, dt_sub, nsub, tmp=None, stream=None):
    """In-place advect_3d_gpu on CUDA float32 grids (threed.py:1295-1307).  mask: uint8 grid or
    None (then F < 0 marks the mask cells)."""
    nx, ny, nz = phi.shape
    if tmp is None:
        tmp = torch.empty_like(phi)
    _lib.call("petch_advect", _lib.ptr(phi), _lib.ptr(tmp), _lib.ptr(F), _lib.ptr(mask),
              _lib.ptr(mask_phi), nx, ny, nz, float(1.0 / dx), float(dt_sub), int(nsub),
              _lib.stream_ptr(stream))
    return phi


# ---- reference-signature wrappers (numpy in -> numpy float64 out) ----
def reinit_fsm(phi_np, dx, band, n_iter=None):
    """Drop-in for threed.reinit_fsm."""
    host = not isinstance(phi_np, torch.Tensor)
    out = reinit_fsm_dev(_dev(phi_np), dx, band, n_iter)
    return out.double().cpu().numpy() if host else out


def advect_3d_gpu(phi, Fspeed, mask, mask_phi, dx, dt, nsub):
    """Drop-in for threed.advect_3d_gpu (dt is the substep size, as the reference passes it)."""
    host = not isinstance(phi, torch.Tensor)
    p = _dev(phi).clone() if not host else _dev(phi)
    m = _dev(mask, torch.uint8)
    out = advect_dev(p, _dev(Fspeed), m, _dev(mask_phi), dx, dt, nsub)
    return out.double().cpu().numpy() if host else out


def reinit_pde_dev(phi, dx, n_iter=24, out=None, scratch=None, stream=None):
    """reinit_gpu on a CUDA float32 grid (threed.py:1399-1418): n_iter Russo-Smereka PDE sweeps."""
    nx, ny, nz = phi.shape
    if out is None:
        out = torch.empty_like(phi)
    if scratch is None:
        scratch = (torch.empty_like(phi), torch.empty_like(phi))
    _lib.call("petch_reinit_pde", _lib.ptr(phi), _lib.ptr(out), _lib.ptr(scratch[0]),
              _lib.ptr(scratch[1]), nx, ny, nz, float(dx), int(n_iter), _lib.stream_ptr(stream))
    return out


def gaussian_smooth_dev(phi, sigma, mask=None, mask_phi=None, truncate=4.0, scratch=None,
                        stream=None):
    """In place: scipy.ndimage.gaussian_filter(phi, sigma) then phi[mask] = mask_phi[mask]
    (run_etch_3d's surf_smooth, threed.py:1779-1782) on a CUDA float32 grid."""
    nx, ny, nz = phi.shape
    if scratch is None:
        scratch = (torch.empty_like(phi), torch.empty_like(phi))
    _lib.call("petch_gaussian_smooth", _lib.ptr(phi), _lib.ptr(scratch[0]), _lib.ptr(scratch[1]),
              _lib.ptr(mask), _lib.ptr(mask_phi), nx, ny, nz, float(sigma), float(truncate),
              _lib.stream_ptr(stream))
    return phi


def reinit_gpu(phi_np, dx, n_iter=24):
    """Drop-in for threed.reinit_gpu (numpy in -> float64 numpy out; tensors stay on the device)."""
    host = not isinstance(phi_np, torch.Tensor)
    out = reinit_pde_dev(_dev(phi_np), dx, n_iter)
    return out.double().cpu().numpy() if host else out
