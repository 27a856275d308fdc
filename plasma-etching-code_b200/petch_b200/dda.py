"""Deterministic discrete-ordinates (DDA) neutral transport on the device (drop-in for
petch/dda.py, neutral_transport="dda").

Same method as the reference: for each surface point, the cosine-weighted mean over a fixed set of
Fibonacci directions of what a ray marched cell by cell through the occupancy grid picks up (the
source at the top, a wall cell's re-emitted flux otherwise), iterated for diffuse re-emission
Gamma = direct + K (1 - s) Gamma and finished by Aitken extrapolation.  On the device each ray is
marched once per geometry (petch_dda_prepare) and every re-emission pass only reads where the rays
ended (petch_dda_solve), both sticking fields at once.
"""
import ctypes

import numpy as np
import torch

from . import _lib


def fib_hemisphere(n):
    """fib_hemisphere (dda.py:98-113): n upper-hemisphere directions, cosine weights."""
    i = np.arange(n) + 0.5
    polar = np.arccos(1.0 - i / n)
    theta = np.pi * (1.0 + 5.0 ** 0.5) * i
    dz = np.cos(polar)
    r = np.sin(polar)
    d = np.stack([r * np.cos(theta), r * np.sin(theta), dz], axis=1)
    return d.astype(np.float64), np.clip(dz, 0.0, None).astype(np.float64)


def fib_sphere(n):
    """fib_sphere (dda.py:116-129): n directions on the full sphere (Fibonacci lattice), unit
    weights; the gather weighs each by max(n_face . d, 0)."""
    i = np.arange(n) + 0.5
    z = 1.0 - 2.0 * i / n
    r = np.sqrt(np.maximum(1.0 - z * z, 0.0))
    gold = np.pi * (1.0 + 5.0 ** 0.5)
    theta = gold * i
    d = np.stack([r * np.cos(theta), r * np.sin(theta), z], axis=1)
    return d.astype(np.float64), np.ones(n)


def march_bounds(nz, dx, periodic_y, z_top=None):
    """(z_top, max_steps) as dda_neutral_flux derives them (dda.py:137-151) for zs = arange(nz) dx."""
    zs0, zs_last = 0.0, float(np.arange(nz)[-1] * dx)
    if z_top is None:
        z_top = zs_last - 0.5 * dx
    max_steps = (int((z_top - zs0) / dx) + 4) * (3 if periodic_y else 1)
    return float(z_top), int(max_steps)


class DDASolver:
    """Device buffers of the DDA transport for one face capacity, grid and direction count."""

    def __init__(self, max_faces, shape, n_dir):
        self.MF = int(max_faces)
        self.shape = tuple(int(s) for s in shape)
        self.n_dir = int(n_dir)
        dirs, w = fib_sphere(2 * self.n_dir)
        self.D = len(w)
        self.dirs = torch.from_numpy(dirs.astype(np.float32)).cuda().contiguous()
        self.weights = torch.from_numpy(w.astype(np.float32)).cuda()
        nb = ctypes.c_longlong()
        _lib.call("petch_dda_scratch_bytes", self.MF, *self.shape, self.D, ctypes.byref(nb))
        self.scratch = torch.empty(int(nb.value), dtype=torch.uint8, device="cuda")

    def fits(self, max_faces, shape, n_dir):
        return (self.MF == int(max_faces) and self.shape == tuple(shape)
                and self.n_dir == int(n_dir))

    def prepare(self, phi, dx, n_faces_ptr, origins, normals, areas, periodic_y, z_top=None,
                stream=None):
        """March every (face, direction) ray of the level set phi (device float32)."""
        nx, ny, nz = self.shape
        zt, ms = march_bounds(nz, dx, periodic_y, z_top)
        s = torch.cuda.current_stream().cuda_stream if stream is None else stream
        _lib.call("petch_dda_prepare", phi.data_ptr(), nx, ny, nz, float(dx), zt, ms,
                  int(periodic_y), n_faces_ptr, self.MF, origins.data_ptr(), normals.data_ptr(),
                  areas.data_ptr(), self.dirs.data_ptr(), self.weights.data_ptr(), self.D,
                  self.scratch.data_ptr(), self.scratch.numel(), s)

    def solve(self, bare, betaE, betaO, n_reemit, out_E, out_O, stream=None):
        """dda_neutral_flux for s = clip(bare * betaE, 0, 1) -> out_E and betaO -> out_O."""
        s = torch.cuda.current_stream().cuda_stream if stream is None else stream
        _lib.call("petch_dda_solve", self.MF, *self.shape, self.D, bare.data_ptr(), float(betaE),
                  float(betaO), int(n_reemit), self.scratch.data_ptr(), self.scratch.numel(),
                  out_E.data_ptr(), out_O.data_ptr(), s)


def dda_neutral_flux(phi, dx, zs, centroids, into_gas_normals, s_face, n_dir=64, n_reemit=12,
                     z_top=None, face_areas=None, periodic_y=0):
    """dda_neutral_flux (dda.py:132-188) with the reference's arguments (host arrays); returns the
    per-face arrival multiplier (numpy float64).  zs must be the grid's node heights
    arange(nz) * dx.  The sticking field is carried in float32."""
    phi_t = phi if isinstance(phi, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(phi))
    phi_t = phi_t.to("cuda", torch.float32).contiguous()
    nz = phi_t.shape[2]
    if len(zs) != nz or abs(float(zs[0])) > 1e-12 * dx:
        raise ValueError("zs must be arange(nz) * dx of the grid")
    F = len(centroids)
    if F == 0:
        return np.zeros(0)
    if z_top is None:
        z_top = float(zs[-1]) - 0.5 * dx
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
    org = f32(centroids).reshape(F, 3)
    nrm = f32(into_gas_normals).reshape(F, 3)
    area = f32(np.ones(F) if face_areas is None else face_areas)
    s = f32(s_face)
    nf = torch.tensor([F], dtype=torch.int32, device="cuda")
    solver = DDASolver(F, tuple(phi_t.shape), n_dir)
    solver.prepare(phi_t, dx, nf.data_ptr(), org, nrm, area, periodic_y, z_top)
    out = torch.empty(F, device="cuda")
    out2 = torch.empty(F, device="cuda")
    solver.solve(s, 1.0, 1.0, n_reemit, out, out2)
    return out.double().cpu().numpy()
