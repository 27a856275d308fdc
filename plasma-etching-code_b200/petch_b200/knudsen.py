"""Knudsen 1-D conductance tail on the device (drop-in for petch/knudsen.py,
neutral_transport="knudsen").

The open feature is modelled as a vertical duct: per z-slice the gas area and sidewall perimeter
from the level set give a free-molecular conductance, slices are linked in series, the opening is
held at unit concentration and the floor faces of each slice are its sink; a tridiagonal solve
gives the neutral concentration down the feature, which every face below the substrate top takes
as its arrival multiplier.  The geometry is prepared once per mesh (petch_knudsen_prepare) and each
coverage round solves both sticking fields (petch_knudsen_solve).
"""
import ctypes

import numpy as np
import torch

from . import _lib


def _stream():
    return torch.cuda.current_stream().cuda_stream


class KnudsenSolver:
    """Device buffers of the Knudsen tail for one face capacity and slice count."""

    def __init__(self, max_faces, nz):
        self.MF, self.nz = int(max_faces), int(nz)
        nb = ctypes.c_longlong()
        _lib.call("petch_knudsen_scratch_bytes", self.MF, self.nz, ctypes.byref(nb))
        self.scratch = torch.empty(int(nb.value), dtype=torch.uint8, device="cuda")

    def fits(self, max_faces, nz):
        return self.MF == int(max_faces) and self.nz == int(nz)

    def prepare(self, phi, dx, sub_top, trench, n_faces_ptr, centroids, normals, center=None,
                half_width=None, stream=None):
        """Slice geometry of phi (device float32) and the per-face slice data of the mesh."""
        nx, ny, nz = phi.shape
        cx, cy = center if center is not None else (0.0, 0.0)
        hw = -1.0 if half_width is None or center is None else float(half_width)
        _lib.call("petch_knudsen_prepare", phi.data_ptr(), nx, ny, nz, float(dx), float(sub_top),
                  int(bool(trench)), n_faces_ptr, self.MF, centroids.data_ptr(),
                  normals.data_ptr(), float(cx), float(cy), hw, self.scratch.data_ptr(),
                  self.scratch.numel(), _stream() if stream is None else stream)

    def solve(self, bare, areas, betaE, betaO, Ly, wall_loss_scale, out_E, out_O,
              sink_field=False, front=None, stream=None):
        """One coverage round: flux for s = clip(bare' betaE, 0, 1) -> out_E, betaO -> out_O.
        front = (W, band_W, pass_frac, ar_pass) for the passivation-linked loss scale."""
        fr = (0, 0.0, 0.0, 0.0, 0.0) if front is None else (1,) + tuple(float(v) for v in front)
        _lib.call("petch_knudsen_solve", self.MF, self.nz, bare.data_ptr(), areas.data_ptr(),
                  float(betaE), float(betaO), int(bool(sink_field)), float(Ly),
                  float(wall_loss_scale), *fr, self.scratch.data_ptr(), self.scratch.numel(),
                  out_E.data_ptr(), out_O.data_ptr(), _stream() if stream is None else stream)


def _prepared(phi, zs, dx, sub_top, feature_shape, centroids=None, normals=None, center=None,
              half_width=None):
    phi_t = phi if isinstance(phi, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(phi))
    phi_t = phi_t.to("cuda", torch.float32).contiguous()
    nz = phi_t.shape[2]
    if len(zs) != nz or abs(float(zs[0])) > 1e-12 * dx:
        raise ValueError("zs must be arange(nz) * dx of the grid")
    if feature_shape not in ("via", "trench"):
        raise ValueError(f"unknown feature_shape {feature_shape!r}")
    F = 0 if centroids is None else len(centroids)
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
    cen = f32(np.zeros((1, 3)) if F == 0 else np.reshape(centroids, (F, 3)))
    nrm = f32(np.zeros((1, 3)) if F == 0 else np.reshape(normals, (F, 3)))
    nf = torch.tensor([F], dtype=torch.int32, device="cuda")
    sol = KnudsenSolver(max(F, 1), nz)
    sol.prepare(phi_t, dx, sub_top, feature_shape == "trench", nf.data_ptr(), cen, nrm, center,
                half_width)
    return sol, F, nf


def slice_geometry(phi, zs, dx, sub_top, feature_shape):
    """slice_geometry (knudsen.py:61-68): per-slice gas area and sidewall perimeter (numpy)."""
    sol, _, _ = _prepared(phi, zs, dx, sub_top, feature_shape)
    a = torch.empty(sol.nz, dtype=torch.float64, device="cuda")
    p = torch.empty(sol.nz, dtype=torch.float64, device="cuda")
    _lib.call("petch_knudsen_slices", sol.MF, sol.nz, sol.scratch.data_ptr(), sol.scratch.numel(),
              a.data_ptr(), p.data_ptr(), _stream())
    return a.cpu().numpy(), p.cpu().numpy()


def conductance_profile(phi, zs, dx, sub_top, feature_shape, slice_loss, wall_loss_scale=1.85):
    """conductance_profile (knudsen.py:91-150): the neutral concentration per slice (numpy)."""
    sol, _, _ = _prepared(phi, zs, dx, sub_top, feature_shape)
    nz = sol.nz
    loss = torch.from_numpy(np.ascontiguousarray(slice_loss, np.float64)).cuda()
    ls = np.asarray(wall_loss_scale, float)
    arr = None if ls.ndim == 0 else torch.from_numpy(np.ascontiguousarray(ls[:nz])).cuda()
    out = torch.empty(nz, dtype=torch.float64, device="cuda")
    _lib.call("petch_knudsen_profile", sol.MF, nz, loss.data_ptr(),
              None if arr is None else arr.data_ptr(), float(ls) if ls.ndim == 0 else 0.0,
              sol.scratch.data_ptr(), sol.scratch.numel(), out.data_ptr(), _stream())
    return out.cpu().numpy()


def knudsen_face_flux(phi, zs, dx, sub_top, feature_shape, centroids, gas_nz, face_areas, Ly,
                      s_face, wall_loss_scale=1.85, center=None, half_width=None,
                      front_loss=False, band_W=8.0, pass_frac=0.5, ar_pass=15.0):
    """knudsen_face_flux (knudsen.py:188-241) with the reference's arguments (host arrays):
    the per-face arrival multiplier (numpy float64).  The sticking field is carried in float32."""
    F = len(centroids)
    if F == 0:
        return np.zeros(0)
    normals = np.zeros((F, 3))
    normals[:, 2] = np.asarray(gas_nz, float)
    sol, _, nf = _prepared(phi, zs, dx, sub_top, feature_shape, centroids, normals, center,
                           half_width)
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
    s = f32(s_face)
    A = f32(face_areas)
    out, out2 = torch.empty(F, device="cuda"), torch.empty(F, device="cuda")
    front = None
    if front_loss:
        W = 2.0 * float(half_width) if half_width is not None else dx
        front = (W, band_W, pass_frac, ar_pass)
    sol.solve(s, A, 1.0, 1.0, Ly, wall_loss_scale, out, out2, front=front)
    return out.double().cpu().numpy()
