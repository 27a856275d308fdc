"""Shared helpers for the GPU parity tests: fixture geometries, device meshes, C-ABI calls."""
import ctypes

import numpy as np
import torch

import oracle.oracle as orc
from petch_b200 import _lib
from petch_b200 import threed as t3


def stream():
    return torch.cuda.current_stream().cuda_stream


def small_feature(hole, nx=14, ny=14, nz=18, dx=0.25):
    """The etched-pit feature of tests/golden/make_golden.py::_small_mesh (same construction):
    a masked hole or trench with a pit down to z = 1.6.  Returns (phi float32, geo)."""
    Lx, Ly, Lz = nx * dx, ny * dx, nz * dx
    sub_top, mask_th, width = 3.0, 0.75, 1.5
    phi_a, _ = orc.seed(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole)
    X, Y, Z = np.meshgrid(np.arange(nx) * dx, np.arange(ny) * dx, np.arange(nz) * dx, indexing="ij")
    r = np.sqrt((X - Lx / 2) ** 2 + (Y - Ly / 2) ** 2) if hole else np.abs(X - Lx / 2)
    phi_a = np.minimum(phi_a, np.maximum(r - width / 2, 1.6 - Z))
    phi = orc.reinit(phi_a.astype(np.float32), dx, 6 * dx).astype(np.float32)
    geo = dict(Lx=Lx, Ly=Ly, Lz=Lz, dx=dx, sub_top=sub_top, mask_th=mask_th, trench_width=width,
               hole=hole, periodic_y=0 if hole else 1)
    return phi, geo


def hole_seed(nx=56, ny=56, nz=96, dx=0.25, Lx=14.0, Ly=14.0, sub_top=18.0, mask_th=2.0, width=6.0):
    """Config-0 hole seed field (CSG + the oracle's seed distance)."""
    phi_a, mask = orc.seed(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, True)
    phi = orc.seed_distance(phi_a.astype(np.float32), dx).astype(np.float32)
    geo = dict(Lx=Lx, Ly=Ly, Lz=nz * dx, dx=dx, sub_top=sub_top, mask_th=mask_th,
               trench_width=width, hole=True)
    return phi, mask, geo


def cuda_mesh(phi, dx, geo, MT=None):
    phid = torch.from_numpy(np.ascontiguousarray(phi, np.float32)).cuda()
    MT = MT or t3.default_capacity(phid.shape)
    m = t3.DeviceMesh(MT)
    scr = torch.empty(t3.mesh_scratch_bytes(phid.shape, MT), dtype=torch.uint8, device="cuda")
    m.build(phid, dx, geo, scr)
    c = m.counts()
    assert (c['err'] & ~t3.MESH_ERR_NONMANIFOLD) == 0, c
    m.F, m.V = c['F'], c['V']
    return m


def domain(geo):
    d = _lib.Domain()
    d.lx, d.ly, d.lz = geo['Lx'], geo['Ly'], geo['Lz']
    d.z_src = geo['Lz'] - geo['dx']
    d.periodic = int(geo.get('periodic_y', 0))
    return d


def cuda_neutrals(m, geo, bare, beta, seed, n):
    flux = torch.zeros(m.MT, device="cuda")
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    b = None if bare is None else torch.from_numpy(np.asarray(bare, np.float32)).cuda()
    _lib.call("petch_trace_neutrals", m.id, m.MT, m.MV, ctypes.byref(domain(geo)),
              None if b is None else b.data_ptr(), float(beta), int(seed), 0, int(n),
              flux.data_ptr(), work.data_ptr(), stream())
    assert work[1].item() == 0
    return flux[:m.F].double().cpu().numpy()


def cuda_ions(m, geo, par, seed, n):
    tal = torch.zeros((m.MT, 4), device="cuda")
    ang = torch.zeros(m.MT, device="cuda")
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    _lib.call("petch_trace_ions", m.id, m.MT, m.MV, ctypes.byref(domain(geo)),
              ctypes.byref(t3.ion_params(par)), int(seed), int(n), tal.data_ptr(), ang.data_ptr(),
              work.data_ptr(), stream())
    assert work[1].item() == 0
    out = torch.cat([tal[:m.F], ang[:m.F, None]], dim=1)
    return out.double().cpu().numpy()


def cuda_legacy(m, geo, ion, sigma, sticking, n_reemit, specular, seed, n):
    fl = torch.zeros(m.MT, device="cuda")
    ang = torch.zeros(m.MT, device="cuda")
    work = torch.zeros(6, dtype=torch.int32, device="cuda")
    _lib.call("petch_trace_legacy", m.id, m.MT, m.MV, ctypes.byref(domain(geo)), int(ion),
              float(sigma), float(sticking), int(n_reemit), int(specular), 0.34, 0.8, int(seed),
              int(n), fl.data_ptr(), ang.data_ptr(), work.data_ptr(), stream())
    assert work[1].item() == 0
    return fl[:m.F].double().cpu().numpy(), ang[:m.F].double().cpu().numpy()
