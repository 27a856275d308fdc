"""The per-step 3D etch loop on the device (drop-in for petch/threed.py's run_etch_3d,
mc_flux_3d_coupled, mc_flux_3d and helpers).

One step, all in libpetchb200.so kernels on one CUDA stream:

    mesh build (marching cubes -> faces, geometry, adjacency, BVH)
    -> warm-start coverage (nearest face of the previous mesh)
    -> ions (faithful ViennaPS reflection) -> yields / m_i / cos_i (normalised + smoothed)
    -> coverage fixed point: F and O Russian-roulette neutrals -> Belen coverages -> bare
    -> surface rate V -> velocity extension into the band (+ active-cell list)
    -- one small device->host read: max V, band size, counts and error bits --
    -> nsub CFL substeps of upwind advection on the band -> Jacobi Godunov-Eikonal reinit

Host code only derives scalars (seeds, CFL substep count, float64 constants) the way the
reference's host code does; no per-face or per-cell arithmetic happens on the CPU.
"""
import ctypes
import threading
import time
import warnings

import numpy as np
import torch

from . import _lib
from .chemistry import _yields
from .levelset import (gaussian_smooth_dev, grid_shape, reinit_fsm_dev, reinit_pde_dev,
                       seed_field)
from .params import DEFAULT_FLAGS, PAR

SEGMENTS = ("hdr", "vnode", "verts", "faces", "tri", "area", "normal", "centroid", "fmask", "nbr",
            "nbrw", "leaf_code", "leaf_start", "nodes", "parent", "flags")

MESH_ERR_TRI_OVERFLOW, MESH_ERR_VERT_OVERFLOW, MESH_ERR_HASH_FULL, MESH_ERR_NONMANIFOLD = 1, 2, 4, 8


def _sp():
    return torch.cuda.current_stream().cuda_stream


class EventTimer:
    """CUDA-event intervals on the current stream, grouped by name; read once at the end of a run
    (no per-interval synchronisation).  Each interval is also an NVTX range of the same name (a
    start / end range, so intervals of different names may overlap), for a profiler's
    timeline."""

    def __init__(self):
        self.open = {}
        self.pairs = {}
        self.pool = []

    def _ev(self):
        return self.pool.pop() if self.pool else torch.cuda.Event(enable_timing=True)

    def start(self, name):
        e = self._ev()
        e.record()
        self.open[name] = (e, torch.cuda.nvtx.range_start(name))

    def stop(self, name):
        e = self._ev()
        e.record()
        e0, rid = self.open.pop(name)
        torch.cuda.nvtx.range_end(rid)
        self.pairs.setdefault(name, []).append((e0, e))

    def totals_ms(self):
        torch.cuda.current_stream().synchronize()
        out = {k: [a.elapsed_time(b) for a, b in v] for k, v in self.pairs.items()}
        for v in self.pairs.values():
            for a, b in v:
                self.pool += [a, b]
        self.pairs = {}
        return out


class _NoTimer:
    def start(self, name):
        pass

    def stop(self, name):
        pass


class DeviceMesh:
    """Surface mesh + BVH in one device buffer (the role of wp.Mesh plus extract_mesh_3d's
    arrays).  Counts live on the device in `hdr`; `n_faces()` reads them (a sync)."""

    def __init__(self, max_tris, max_verts=None):
        self.MT = int(max_tris)
        self.MV = int(max_verts if max_verts is not None else max_tris)
        offs = (ctypes.c_longlong * len(SEGMENTS))()
        total = ctypes.c_longlong()
        _lib.call("petch_mesh_layout", self.MT, self.MV, offs, len(SEGMENTS), ctypes.byref(total))
        self.off = list(offs)
        self.buf = torch.empty(int(total.value), dtype=torch.uint8, device="cuda")
        MT, MV = self.MT, self.MV
        self.hdr = self._view(0, torch.int32, 16)
        self.vnode = self._view(1, torch.float32, 3 * MV).view(MV, 3)
        self.verts = self._view(2, torch.float32, 3 * MV).view(MV, 3)
        self.faces = self._view(3, torch.int32, 3 * MT).view(MT, 3)
        self.area = self._view(5, torch.float32, MT)
        self.normal = self._view(6, torch.float32, 3 * MT).view(MT, 3)
        self.centroid = self._view(7, torch.float32, 3 * MT).view(MT, 3)
        self.fmask = self._view(8, torch.uint8, MT)
        self.nbr = self._view(9, torch.int32, 3 * MT).view(MT, 3)
        self.nbrw = self._view(10, torch.float32, 3 * MT).view(MT, 3)
        self.hdr.zero_()

    def _view(self, seg, dtype, n):
        item = torch.empty((), dtype=dtype).element_size()
        a = self.off[seg]
        return self.buf[a:a + n * item].view(dtype)

    @property
    def id(self):
        return self.buf.data_ptr()

    def counts(self):
        h = self.hdr[:8].cpu().numpy()
        return dict(F=int(h[0]), V=int(h[1]), L=int(h[2]), err=int(h[3]))

    def n_faces(self):
        return min(int(self.hdr[0].item()), self.MT)

    def build(self, phi, dx, geo, scratch):
        nx, ny, nz = phi.shape
        _lib.call("petch_mesh_build", phi.data_ptr(), nx, ny, nz, float(dx), float(geo['Lx']),
                  float(geo['Ly']), float(geo['sub_top']), float(geo['mask_th']),
                  float(geo['trench_width']), int(bool(geo['hole'])), self.id, self.MT, self.MV,
                  scratch.data_ptr(), scratch.numel(), _sp())

    # host copies trimmed to the live counts (for the drop-in API / tests)
    def host_arrays(self):
        c = self.counts()
        F, V = min(c['F'], self.MT), min(c['V'], self.MV)
        return (self.verts[:V].cpu().numpy(), self.faces[:F].cpu().numpy(),
                self.centroid[:F].double().cpu().numpy(), self.area[:F].double().cpu().numpy())


def mesh_scratch_bytes(shape, max_tris):
    b = ctypes.c_longlong()
    _lib.call("petch_mesh_scratch_bytes", *shape, int(max_tris), ctypes.byref(b))
    return int(b.value)


def default_capacity(shape):
    """Starting face capacity: ~4 faces per boundary cell of the domain box (grown on demand)."""
    nx, ny, nz = shape
    return int(max(65536, 8 * (nx * ny + ny * nz + nx * nz)))


# --------------------------------------------------------------------------------------------
# parameters
# --------------------------------------------------------------------------------------------
def domain_params(geo, par):
    d = _lib.Domain()
    d.lx, d.ly, d.lz = float(geo['Lx']), float(geo['Ly']), float(geo['Lz'])
    d.z_src = float(geo['Lz'] - geo['dx'])
    d.periodic = int(par.get('periodic_y', 0))
    return d


def ion_params(par):
    """The float arguments of _trace3d_ion_yield as mc_flux_3d_coupled computes them
    (threed.py:800-812)."""
    p = _lib.IonParams()
    inflect = float(par.get('inflectAngle', 1.55334303))
    minang = float(par.get('minAngle', 1.3962634))
    n_l = float(par.get('n_l', 10.0))
    A_en = 1.0 / (1.0 + n_l * (1.5707963 / inflect - 1.0))
    p.meanE, p.sigmaE = float(par['Emean']), float(par['Esig'])
    p.A_sp, p.Eth_sp, p.B_sp = float(par['A_sp']), float(par['Eth_sp']), float(par['B_sp'])
    p.A_ie, p.Eth_ie = float(par['A_ie']), float(par['Eth_ie'])
    p.A_p, p.Eth_p = float(par['A_p']), float(par['Eth_p'])
    p.inflect, p.minang, p.n_l, p.A_en = inflect, minang, n_l, float(A_en)
    p.minE = float(min(par['Eth_ie'], par['Eth_sp']))
    p.thrmin = float(par.get('thetaRMin', 1.2217305))
    p.thrmax = float(par.get('thetaRMax', 1.5707963))
    p.sigma = float(par['ion_ang_sigma'])
    return p


def chem_params(par, flags):
    c = _lib.ChemParams()
    for k in ("ionFlux", "Fflux", "Oflux", "k_sigma", "beta_sigma", "rho", "rate_scale", "s_F",
              "s_O", "B_sp"):
        setattr(c, k, float(par.get(k, PAR.get(k, 0.0))))
    c.fnorm_E = float(par.get('fnorm_E', 1.0))
    c.fnorm_O = float(par.get('fnorm_O', 1.0))
    c.Yie, c.Ysp, c.Yp = _yields(par)
    mode = "cosine" if flags is None else getattr(flags, "yield_angular", "cosine")
    c.yield_angular = 1 if mode == "viennaps" else 0
    chem = "langmuir" if flags is None else getattr(flags, "chemistry", "langmuir")
    if chem not in ("langmuir", "belen"):
        raise ValueError(f"unknown chemistry model: {chem}")
    c.chemistry = 1 if chem == "belen" else 0
    return c


def _unsupported(flags, par):
    if par.get('cov_transport', 'rr') != 'rr':
        raise NotImplementedError("only the Russian-roulette coverage transport (cov_transport='rr')")


# --------------------------------------------------------------------------------------------
# the engine: all buffers of one run
# --------------------------------------------------------------------------------------------
class FluxEngine:
    """Per-face device buffers and the flux stages of one mesh capacity (the part of the loop
    between the mesh and the surface rate): mc_flux_3d_coupled, mc_flux_3d and
    mc_flux_3d_radiosity on a DeviceMesh."""

    def __init__(self, geo, par, flags, max_tris):
        self.geo, self.par, self.flags = geo, par, flags
        dev = dict(device="cuda")
        # small[0:6] tracer work words (ray counter, error bits, u64 queries, u64 visits),
        # small[6:8] rate stats, small[8] band size
        self.small = torch.zeros(16, dtype=torch.int32, **dev)
        self.host = torch.zeros(32, dtype=torch.int32).pin_memory()
        self.dom = domain_params(geo, par)
        self.ionp = ion_params(par)
        self.chem = chem_params(par, flags)
        self._alloc_faces(max_tris)
        self.prev = None          # (mesh, bare) of the previous step for the warm start
        self.ktimer = _NoTimer()  # set to an EventTimer to time individual trace launches

    def _alloc_faces(self, MT):
        self.MT = int(MT)
        dev = dict(device="cuda", dtype=torch.float32)
        self.mesh = DeviceMesh(self.MT)
        MT = self.MT
        self.tal4 = torch.empty((MT, 4), **dev)
        self.ang = torch.empty(MT, **dev)
        self.flux = torch.empty(MT, **dev)
        self.m_i = torch.empty(MT, **dev)
        self.m_F = torch.empty(MT, **dev)
        self.m_O = torch.empty(MT, **dev)
        self.cos_i = torch.empty(MT, **dev)
        self.y = torch.empty((3, MT), **dev)
        self.bare = torch.empty(MT, **dev)
        self.V = torch.empty(MT, **dev)
        self.tmp5 = torch.empty(5 * MT, **dev)
        self.rad = None           # radiosity buffers, allocated on first use
        self.dda = None           # DDA solver, allocated on first use
        self.kn = None            # Knudsen solver, allocated on first use
        self.fn = None            # into-gas normals, allocated on first use

    def grow(self, need):
        MT = max(int(need * 1.5), 2 * self.MT)
        self._alloc_faces(MT)

    # ---- flux stages ----
    def flux_coupled(self, n_ion, n_neu, seed, warm, bare_init=None, phi=None):
        """mc_flux_3d_coupled (threed.py:740-905) on the device.  The coverage starts from the
        previous step's (warm, nearest face) or from bare_init (a device float[F] the caller
        supplies), else cold at 1.  With flags.surface_charging and charge_alpha > 0 the
        electron-shadowing factor scales m_i (threed.py:847-868); flags.floor_charge_throttle
        then scales the floor's ion results (_apply_floor_charge_throttle; it needs the level
        set phi, the engine's own when not given).  Each coverage round traces both neutral
        species in one launch (petch_trace_neutral_pair)."""
        par, flags, m = self.par, self.flags, self.mesh
        s = _sp()
        A_src = float(self.geo['Lx'] * self.geo['Ly'])
        n_smooth = int(par.get('flux_smooth', 1))
        alpha = float(par.get('flux_smooth_alpha', 1.0))
        work = self.small[0:6]
        faithful = (flags is not None and getattr(flags, "ion_reflection", False)
                    and getattr(flags, "chemistry", "langmuir") == "belen")
        seeded = False
        if bare_init is not None:
            F = int(bare_init.numel())
            self.bare[:F].copy_(bare_init.clamp(0.0, 1.0))
            seeded = True
        elif warm and self.prev is not None:
            pm, pb = self.prev
            _lib.call("petch_warmstart", pm.id, pm.MT, pm.MV, pb.data_ptr(), m.id, m.MT, m.MV,
                      self.bare.data_ptr(), work.data_ptr(), s)
            seeded = True
        if faithful:
            self.ktimer.start("k_ions")
            _lib.call("petch_trace_ions", m.id, m.MT, m.MV, ctypes.byref(self.dom),
                      ctypes.byref(self.ionp), int(seed * 9 + 1) & 0xffffffff, int(n_ion),
                      self.tal4.data_ptr(), self.ang.data_ptr(), work.data_ptr(), s)
            self.ktimer.stop("k_ions")
            _lib.call("petch_ion_post", m.id, m.MT, m.MV, self.tal4.data_ptr(), self.ang.data_ptr(),
                      float(A_src / n_ion), n_smooth, alpha, self.y[0].data_ptr(),
                      self.y[1].data_ptr(), self.y[2].data_ptr(), self.m_i.data_ptr(),
                      self.cos_i.data_ptr(), self.tmp5.data_ptr(), s)
            yields = (self.y[0].data_ptr(), self.y[1].data_ptr(), self.y[2].data_ptr())
        else:
            # legacy first-hit ion (threed.py:825-840): m_i normalised, clipped at 1.5, smoothed
            _lib.call("petch_trace_legacy", m.id, m.MT, m.MV, ctypes.byref(self.dom), 1,
                      float(par['ion_ang_sigma']), 1.0, 0, 0, 0.34, 0.8,
                      int(seed * 9 + 1) & 0xffffffff, int(n_ion), self.flux.data_ptr(),
                      self.ang.data_ptr(), work.data_ptr(), s)
            _lib.call("petch_cos_ratio", m.id, m.MT, m.MV, self.flux.data_ptr(),
                      self.ang.data_ptr(), self.cos_i.data_ptr(), s)
            _lib.call("petch_norm_smooth", m.id, m.MT, m.MV, self.flux.data_ptr(),
                      float(A_src / n_ion), 0.0, 1.5, 1, n_smooth, alpha, self.m_i.data_ptr(),
                      self.tmp5.data_ptr(), self.tmp5[m.MT:].data_ptr(), s)
            yields = (None, None, None)
        if (flags is not None and getattr(flags, "surface_charging", False)
                and float(par.get('charge_alpha', 0.0)) > 0.0):
            from .charging import apply_electron_shadow
            self.electron = apply_electron_shadow(self, n_neu, seed)
        if flags is not None and getattr(flags, "floor_charge_throttle", False):
            from .charging import apply_floor_throttle
            phi = phi if phi is not None else getattr(self, "phi", None)
            if phi is None:
                raise ValueError("floor_charge_throttle needs the level set the mesh came from")
            self.yields = yields
            self.charging = apply_floor_throttle(self, self.gas_normals(phi))
        n_fp = int(par.get('n_fp', 1 if seeded else 4))
        if not seeded:
            self.bare.fill_(1.0)
        betaE, betaO = float(par.get('betaE', 0.7)), float(par.get('betaO', 1.0))
        flux_o = self.tmp5[2 * m.MT:3 * m.MT]
        for it in range(n_fp):
            # both species of the round in one launch (F: betaE, seed*9+2+2it; O: betaO, +3+2it)
            self.ktimer.start("k_neutrals")
            _lib.call("petch_trace_neutral_pair", m.id, m.MT, m.MV, ctypes.byref(self.dom),
                      self.bare.data_ptr(), betaE, betaO, int(seed * 9 + 2 + 2 * it) & 0xffffffff,
                      int(seed * 9 + 3 + 2 * it) & 0xffffffff, 0, int(n_neu),
                      self.flux.data_ptr(), flux_o.data_ptr(), work.data_ptr(), s)
            self.ktimer.stop("k_neutrals")
            for fl, out in ((self.flux, self.m_F), (flux_o, self.m_O)):
                _lib.call("petch_norm_smooth", m.id, m.MT, m.MV, fl.data_ptr(),
                          float(A_src / n_neu), 0.0, 8.0, 1, n_smooth, alpha, out.data_ptr(),
                          self.tmp5.data_ptr(), self.tmp5[m.MT:].data_ptr(), s)
            _lib.call("petch_belen_bare", m.id, m.MT, m.MV, ctypes.byref(self.chem),
                      self.m_i.data_ptr(), self.m_F.data_ptr(), self.m_O.data_ptr(),
                      self.cos_i.data_ptr(), yields[1], yields[2], self.bare.data_ptr(), s)
        self.yields = yields
        return n_fp

    def flux_legacy(self, n_ion, n_neu, seed, ion_reflection):
        """mc_flux_3d (threed.py:472-507): legacy species, no smoothing, clipped fluxes."""
        par, m = self.par, self.mesh
        s = _sp()
        A_src = float(self.geo['Lx'] * self.geo['Ly'])
        work = self.small[0:6]
        sF = float(par['s_F'])
        sO = float(par['s_O'])
        if getattr(self.flags, "chemistry", "langmuir") == "belen":
            sF, sO = float(par['betaE']), float(par['betaO'])
        spec, nre = (1, 3) if ion_reflection else (0, 0)
        _lib.call("petch_trace_legacy", m.id, m.MT, m.MV, ctypes.byref(self.dom), 1,
                  float(par['ion_ang_sigma']), 1.0, nre, spec, 0.34, 0.8,
                  int(seed * 9 + 1) & 0xffffffff, int(n_ion), self.flux.data_ptr(),
                  self.ang.data_ptr(), work.data_ptr(), s)
        _lib.call("petch_cos_ratio", m.id, m.MT, m.MV, self.flux.data_ptr(), self.ang.data_ptr(),
                  self.cos_i.data_ptr(), s)
        _lib.call("petch_norm_smooth", m.id, m.MT, m.MV, self.flux.data_ptr(), float(A_src / n_ion),
                  0.0, 1.5, 1, 0, 1.0, self.m_i.data_ptr(), self.tmp5.data_ptr(),
                  self.tmp5[m.MT:].data_ptr(), s)
        for stick, out, sd in ((sF, self.m_F, seed * 9 + 2), (sO, self.m_O, seed * 9 + 3)):
            _lib.call("petch_trace_legacy", m.id, m.MT, m.MV, ctypes.byref(self.dom), 0, 0.0,
                      stick, 12, 0, 0.34, 0.8, int(sd) & 0xffffffff, int(n_neu),
                      self.flux.data_ptr(), self.ang.data_ptr(), work.data_ptr(), s)
            _lib.call("petch_norm_smooth", m.id, m.MT, m.MV, self.flux.data_ptr(),
                      float(A_src / n_neu), 0.0, 4.0, 1, 0, 1.0, out.data_ptr(),
                      self.tmp5.data_ptr(), self.tmp5[m.MT:].data_ptr(), s)
        self.yields = (None, None, None)

    def _radiosity_buffers(self, n_ff):
        r = self.rad
        if r is None or r['n_ff'] != n_ff:
            MT = self.MT
            nb = ctypes.c_longlong()
            _lib.call("petch_ff_scratch_bytes", MT, int(n_ff), ctypes.byref(nb))
            i32 = dict(device="cuda", dtype=torch.int32)
            f64 = dict(device="cuda", dtype=torch.float64)
            r = dict(n_ff=int(n_ff), fn=torch.empty((MT, 3), device="cuda"),
                     hit=torch.empty(MT * n_ff, **i32), col=torch.empty(MT * n_ff, **i32),
                     row_ptr=torch.empty(MT + 1, **i32), sky=torch.empty(MT, **f64),
                     work2=torch.empty(4 * MT, **f64),
                     scratch=torch.empty(int(nb.value), dtype=torch.uint8, device="cuda"))
            self.rad = r
        return r

    def _ions_deterministic(self, n_ion, seed):
        """_ions_deterministic (threed.py:994-1029), the ion launch of the deterministic-neutral
        paths (radiosity, DDA): faithful ViennaPS reflection (yields, m_i, cos_i, unsmoothed) or
        the legacy first-hit ion (m_i clipped at 1.5).  Returns the yield pointers (or Nones)."""
        par, flags, m = self.par, self.flags, self.mesh
        s = _sp()
        A_src = float(self.geo['Lx'] * self.geo['Ly'])
        work = self.small[0:6]
        faithful = (flags is not None and getattr(flags, "ion_reflection", False)
                    and getattr(flags, "chemistry", "langmuir") == "belen")
        self.ktimer.start("k_ions")
        if faithful:
            _lib.call("petch_trace_ions", m.id, m.MT, m.MV, ctypes.byref(self.dom),
                      ctypes.byref(self.ionp), int(seed * 9 + 1) & 0xffffffff, int(n_ion),
                      self.tal4.data_ptr(), self.ang.data_ptr(), work.data_ptr(), s)
            _lib.call("petch_ion_post", m.id, m.MT, m.MV, self.tal4.data_ptr(), self.ang.data_ptr(),
                      float(A_src / n_ion), 0, 1.0, self.y[0].data_ptr(), self.y[1].data_ptr(),
                      self.y[2].data_ptr(), self.m_i.data_ptr(), self.cos_i.data_ptr(),
                      self.tmp5.data_ptr(), s)
            yields = (self.y[0].data_ptr(), self.y[1].data_ptr(), self.y[2].data_ptr())
        else:
            _lib.call("petch_trace_legacy", m.id, m.MT, m.MV, ctypes.byref(self.dom), 1,
                      float(par['ion_ang_sigma']), 1.0, 0, 0, 0.34, 0.8,
                      int(seed * 9 + 1) & 0xffffffff, int(n_ion), self.flux.data_ptr(),
                      self.ang.data_ptr(), work.data_ptr(), s)
            _lib.call("petch_cos_ratio", m.id, m.MT, m.MV, self.flux.data_ptr(),
                      self.ang.data_ptr(), self.cos_i.data_ptr(), s)
            _lib.call("petch_norm_smooth", m.id, m.MT, m.MV, self.flux.data_ptr(),
                      float(A_src / n_ion), 0.0, 1.5, 1, 0, 1.0, self.m_i.data_ptr(),
                      self.tmp5.data_ptr(), self.tmp5[m.MT:].data_ptr(), s)
            yields = (None, None, None)
        self.ktimer.stop("k_ions")
        return yields

    def flux_radiosity(self, phi, n_ion, seed, n_ff=64, n_fp=4, n_iter=40):
        """mc_flux_3d_radiosity (threed.py:923-991) on the device: ions as _ions_deterministic
        (unsmoothed), into-gas normals from phi, n_ff form-factor rays per face, the CSR form
        factor matrix, then n_fp rounds of the two-species Jacobi solve and the Belen coverage
        update, starting from bare = 1; par['radiosity_solver'] 'gmres' solves each species by
        restarted GMRES (anything else: the Jacobi sweeps, as the reference)."""
        par, flags, m = self.par, self.flags, self.mesh
        s = _sp()
        work = self.small[0:6]
        yields = self._ions_deterministic(n_ion, seed)
        r = self._radiosity_buffers(n_ff)
        nx, ny, nz = phi.shape
        _lib.call("petch_gas_normals", m.id, m.MT, m.MV, phi.data_ptr(), nx, ny, nz,
                  float(self.geo['dx']), r['fn'].data_ptr(), s)
        self.ktimer.start("k_ff")
        _lib.call("petch_trace_ff", m.id, m.MT, m.MV, ctypes.byref(self.dom), r['fn'].data_ptr(),
                  int(seed) & 0xffffffff, int(n_ff), r['hit'].data_ptr(), work.data_ptr(), s)
        self.ktimer.stop("k_ff")
        self.radiosity_from_hits(r['hit'], n_ff, yields, n_fp, n_iter)
        self.yields = yields

    def radiosity_from_hits(self, hit, n_ff, yields, n_fp=4, n_iter=40):
        """The deterministic part of mc_flux_3d_radiosity from form-factor hits already on the
        device (int[MT * n_ff]): matrix assembly, then the coverage <-> radiosity fixed point
        into m_F, m_O and bare (m_i, cos_i and the yields must be in place)."""
        m = self.mesh
        s = _sp()
        r = self._radiosity_buffers(n_ff)
        _lib.call("petch_ff_matrix", m.id, m.MT, m.MV, hit.data_ptr(), int(n_ff),
                  r['row_ptr'].data_ptr(), r['col'].data_ptr(), r['sky'].data_ptr(),
                  r['scratch'].data_ptr(), r['scratch'].numel(), s)
        self.bare.fill_(1.0)
        betaE, betaO = float(self.par.get('betaE', 0.7)), float(self.par.get('betaO', 1.0))
        gmres = self.par.get('radiosity_solver', 'jacobi') == 'gmres'
        for _ in range(n_fp):
            self.ktimer.start("k_rad_solve")
            if gmres:
                for beta, out in ((betaE, self.m_F), (betaO, self.m_O)):
                    self._radiosity_gmres(r, n_ff, beta, n_iter, out)
            else:
                _lib.call("petch_radiosity_solve", m.id, m.MT, m.MV, r['row_ptr'].data_ptr(),
                          r['col'].data_ptr(), r['sky'].data_ptr(), int(n_ff),
                          self.bare.data_ptr(), betaE, betaO, int(n_iter), self.m_F.data_ptr(),
                          self.m_O.data_ptr(), r['work2'].data_ptr(), s)
            self.ktimer.stop("k_rad_solve")
            _lib.call("petch_belen_bare", m.id, m.MT, m.MV, ctypes.byref(self.chem),
                      self.m_i.data_ptr(), self.m_F.data_ptr(), self.m_O.data_ptr(),
                      self.cos_i.data_ptr(), yields[1], yields[2], self.bare.data_ptr(), s)


    def _radiosity_gmres(self, r, n_ff, beta, n_iter, out, rtol=1e-3, restart=12, maxiter=40):
        """One species of solve() with radiosity_solver='gmres' (threed.py:972-982): restarted
        GMRES on (I - M) G = D into out; the Jacobi sweeps when it does not converge."""
        m = self.mesh
        s = _sp()
        if r.get('gm') is None or r['gm'][0] != restart:
            nb = ctypes.c_longlong()
            _lib.call("petch_radiosity_gmres_scratch_bytes", m.MT, int(restart), ctypes.byref(nb))
            r['gm'] = (restart, torch.empty(int(nb.value), dtype=torch.uint8, device="cuda"))
        scr = r['gm'][1]
        info = ctypes.c_int(0)
        _lib.call("petch_radiosity_gmres", m.id, m.MT, m.MV, r['row_ptr'].data_ptr(),
                  r['col'].data_ptr(), r['sky'].data_ptr(), int(n_ff), self.bare.data_ptr(),
                  float(beta), float(rtol), int(restart), int(maxiter), out.data_ptr(),
                  scr.data_ptr(), scr.numel(), ctypes.byref(info), s)
        if info.value != 0:
            _lib.call("petch_radiosity_solve", m.id, m.MT, m.MV, r['row_ptr'].data_ptr(),
                      r['col'].data_ptr(), r['sky'].data_ptr(), int(n_ff), self.bare.data_ptr(),
                      float(beta), float(beta), int(n_iter), out.data_ptr(),
                      self.tmp5.data_ptr(), r['work2'].data_ptr(), s)
        return info.value

    def flux_dda(self, phi, n_ion, seed, n_fp=4):
        """mc_flux_3d_dda (threed.py:1211-1244) on the device: ions as _ions_deterministic, the
        into-gas normals, the DDA rays marched once for this mesh, then n_fp rounds of the
        two-species DDA solve (par dda_n_dir directions per hemisphere, dda_n_reemit passes) and
        the Belen coverage update, starting from bare = 1."""
        yields = self._ions_deterministic(n_ion, seed)
        self.dda_prepare(phi)
        self.dda_fixed_point(yields, n_fp)
        self.yields = yields

    def gas_normals(self, phi):
        """_gas_normals (threed.py:1553-1568) of the current mesh on the level set phi, into a
        [MT, 3] device buffer of the engine."""
        m = self.mesh
        if self.fn is None or self.fn.shape[0] != m.MT:
            self.fn = torch.empty((m.MT, 3), device="cuda")
        nx, ny, nz = phi.shape
        _lib.call("petch_gas_normals", m.id, m.MT, m.MV, phi.data_ptr(), nx, ny, nz,
                  float(self.geo['dx']), self.fn.data_ptr(), _sp())
        return self.fn

    def dda_prepare(self, phi):
        """Into-gas normals and the DDA march for the current mesh on the level set phi."""
        from .dda import DDASolver
        m = self.mesh
        s = _sp()
        n_dir = int(self.par.get('dda_n_dir', 64))
        shape = tuple(phi.shape)
        if self.dda is None or not self.dda.fits(m.MT, shape, n_dir):
            self.dda = DDASolver(m.MT, shape, n_dir)
        solver = self.dda
        fn = self.gas_normals(phi)
        dx = float(self.geo['dx'])
        self.ktimer.start("k_dda_march")
        solver.prepare(phi, dx, m.id, m.centroid, fn, m.area, int(self.par.get('periodic_y', 0)),
                       stream=s)
        self.ktimer.stop("k_dda_march")

    def dda_fixed_point(self, yields, n_fp=4):
        """The coverage <-> DDA fixed point (threed.py:1234-1243) on the prepared rays (m_i,
        cos_i and the yields must be in place)."""
        m = self.mesh
        s = _sp()
        solver = self.dda
        n_re = int(self.par.get('dda_n_reemit', 12))
        betaE, betaO = float(self.par.get('betaE', 0.7)), float(self.par.get('betaO', 1.0))
        self.bare.fill_(1.0)
        for _ in range(n_fp):
            self.ktimer.start("k_dda_solve")
            solver.solve(self.bare, betaE, betaO, n_re, self.m_F, self.m_O, stream=s)
            self.ktimer.stop("k_dda_solve")
            _lib.call("petch_belen_bare", m.id, m.MT, m.MV, ctypes.byref(self.chem),
                      self.m_i.data_ptr(), self.m_F.data_ptr(), self.m_O.data_ptr(),
                      self.cos_i.data_ptr(), yields[1], yields[2], self.bare.data_ptr(), s)


    def flux_knudsen(self, phi, n_ion, seed, n_fp=4):
        """mc_flux_3d_knudsen (threed.py:1149-1208) on the device: ions as _ions_deterministic,
        the floor-charging closure for flags.surface_charging = "hg" / "petch" (_apply_hg_charging),
        then n_fp rounds of the two-species Knudsen solve and the Belen coverage update, starting
        from bare = 1."""
        from .charging import apply_hg_charging
        yields = self._ions_deterministic(n_ion, seed)
        self.yields = yields
        fn = self.gas_normals(phi)
        self.charging = apply_hg_charging(self, fn, getattr(self.flags, "surface_charging", False))
        self.knudsen_prepare(phi, fn)
        self.knudsen_fixed_point(yields, n_fp)

    def knudsen_prepare(self, phi, fn):
        """Slice geometry of phi and the per-face slice data of the current mesh."""
        from .knudsen import KnudsenSolver
        m, geo = self.mesh, self.geo
        nz = phi.shape[2]
        if self.kn is None or not self.kn.fits(m.MT, nz):
            self.kn = KnudsenSolver(m.MT, nz)
        hw = 0.5 * float(geo.get('trench_width', geo['Lx']))
        self.ktimer.start("k_kn_prepare")
        self.kn.prepare(phi, float(geo['dx']), float(geo['sub_top']), not geo.get('hole', False),
                        m.id, m.centroid, fn, center=(0.5 * geo['Lx'], 0.5 * geo['Ly']),
                        half_width=hw, stream=_sp())
        self.ktimer.stop("k_kn_prepare")

    def knudsen_fixed_point(self, yields, n_fp=4):
        """The coverage <-> Knudsen fixed point (threed.py:1184-1207) on the prepared geometry
        (m_i, cos_i and the yields must be in place)."""
        m, par, geo = self.mesh, self.par, self.geo
        s = _sp()
        betaE, betaO = float(par.get('betaE', 0.7)), float(par.get('betaO', 1.0))
        wls = float(par.get('knudsen_wall_loss_scale', 1.85))
        front = None
        if getattr(self.flags, 'knudsen_front_loss', False):
            W = 2.0 * 0.5 * float(geo.get('trench_width', geo['Lx']))
            front = (W, float(par.get('knudsen_front_band_W', 8.0)),
                     float(par.get('knudsen_passive_frac', 0.5)),
                     float(par.get('knudsen_front_ar_pass', 15.0)))
        field = par.get('knudsen_sink', 'local') == 'field'
        self.bare.fill_(1.0)
        for _ in range(n_fp):
            self.ktimer.start("k_kn_solve")
            self.kn.solve(self.bare, m.area, betaE, betaO, float(geo['Ly']), wls, self.m_F,
                          self.m_O, sink_field=field, front=front, stream=s)
            self.ktimer.stop("k_kn_solve")
            _lib.call("petch_belen_bare", m.id, m.MT, m.MV, ctypes.byref(self.chem),
                      self.m_i.data_ptr(), self.m_F.data_ptr(), self.m_O.data_ptr(),
                      self.cos_i.data_ptr(), yields[1], yields[2], self.bare.data_ptr(), s)


class EtchEngine(FluxEngine):
    """Device state of one etch run on an (nx, ny, nz) grid."""

    def __init__(self, geo, par, flags, max_tris=None):
        self.shape = tuple(int(s) for s in geo['phi_dev'].shape)
        self.ncell = int(np.prod(self.shape))
        self.dx = float(geo['dx'])
        dev = dict(device="cuda")
        self.phi = geo['phi_dev']
        self.tmp = torch.empty_like(self.phi)
        self.ua = torch.empty_like(self.phi)
        self.ub = torch.empty_like(self.phi)
        self.F = torch.zeros_like(self.phi)
        self.mask = geo['mask_dev']
        self.mask_phi = geo['mask_phi_dev']
        self.mask_idx = torch.nonzero(self.mask.view(-1)).view(-1).to(torch.int32)
        self.active = torch.empty(self.ncell, dtype=torch.int32, **dev)
        super().__init__(geo, par, flags, max_tris or default_capacity(self.shape))

    def _alloc_faces(self, MT):
        super()._alloc_faces(MT)
        self.scratch = torch.empty(mesh_scratch_bytes(self.shape, self.MT), dtype=torch.uint8,
                                   device="cuda")

    def build_mesh(self):
        self.mesh.build(self.phi, self.dx, self.geo, self.scratch)

    def rate_and_extend(self, band, centroid=False, redep=None):
        """surface_rate, the optional redeposition correction (redep = (n particles, seed) or
        (n, seed, z_clean): no redeposit on faces with centroid z <= z_clean), then the velocity
        extension into the band: nearest face (extend_velocity_gpu) or nearest centroid
        (extend_velocity_3d, centroid=True)."""
        m = self.mesh
        s = _sp()
        y = self.yields
        stats = self.small[6:8]
        _lib.call("petch_surface_rate", m.id, m.MT, m.MV, ctypes.byref(self.chem),
                  self.m_i.data_ptr(), self.m_F.data_ptr(), self.m_O.data_ptr(),
                  self.cos_i.data_ptr(), y[0], y[1], y[2], self.V.data_ptr(), stats.data_ptr(), s)
        if redep is not None:
            self.redeposition(*redep)
        nx, ny, nz = self.shape
        fn = "petch_extend_velocity_centroid" if centroid else "petch_extend_velocity"
        _lib.call(fn, m.id, m.MT, m.MV, self.phi.data_ptr(),
                  self.mask.data_ptr(), nx, ny, nz, self.dx, float(band), self.V.data_ptr(),
                  self.F.data_ptr(), 1, self.active.data_ptr(), self.small[8:9].data_ptr(),
                  self.ncell, self.small[0:6].data_ptr(), s)

    def redeposition(self, n, seed, z_clean=None):
        """mc_redep_3d + run_etch_3d's V = max(V - k_redep * Rf, 0) (threed.py:1582-1605,
        1730-1743), with the into-gas normals of the current level set; Rf = 0 on faces with
        centroid z <= z_clean (the charging foot cleaning, threed.py:1733-1741)."""
        m, par = self.mesh, self.par
        s = _sp()
        if getattr(self, "redep", None) is None or self.redep['MT'] != self.MT:
            nb = ctypes.c_longlong()
            _lib.call("petch_redep_scratch_bytes", self.MT, ctypes.byref(nb))
            self.redep = dict(MT=self.MT, fn=torch.empty((self.MT, 3), device="cuda"),
                              cdf=torch.empty(self.MT, dtype=torch.float64, device="cuda"),
                              Rf=torch.empty(self.MT, device="cuda"),
                              scratch=torch.empty(max(int(nb.value), 1), dtype=torch.uint8,
                                                  device="cuda"))
        r = self.redep
        nx, ny, nz = self.shape
        _lib.call("petch_gas_normals", m.id, m.MT, m.MV, self.phi.data_ptr(), nx, ny, nz, self.dx,
                  r['fn'].data_ptr(), s)
        self.ktimer.start("k_redep")
        _lib.call("petch_trace_redep", m.id, m.MT, m.MV, ctypes.byref(self.dom), r['fn'].data_ptr(),
                  self.V.data_ptr(), float(par.get('s_redep', 0.5)), int(seed) & 0xffffffff,
                  int(n), self.flux.data_ptr(), r['cdf'].data_ptr(), r['scratch'].data_ptr(),
                  r['scratch'].numel(), self.small[0:6].data_ptr(), s)
        self.ktimer.stop("k_redep")
        if z_clean is not None:
            _lib.call("petch_zero_below", m.id, m.MT, m.centroid.data_ptr(), float(z_clean),
                      self.flux.data_ptr(), s)
        _lib.call("petch_redep_apply", m.id, m.MT, m.MV, self.flux.data_ptr(), r['cdf'].data_ptr(),
                  int(n), float(par.get('k_redep', 1.0)), self.V.data_ptr(), r['Rf'].data_ptr(),
                  self.small[6:8].data_ptr(), s)

    def sync_status(self):
        """The step's single device->host read: mesh counts/errors + rate stats + band size."""
        self.host[0:8].copy_(self.mesh.hdr[0:8], non_blocking=True)
        self.host[8:17].copy_(self.small[0:9], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        h = self.host.numpy()
        q = h[10:14].view(np.uint64)
        return dict(F=int(h[0]), V=int(h[1]), L=int(h[2]), mesh_err=int(h[3]),
                    trace_err=int(h[9]), queries=int(q[0]), visits=int(q[1]),
                    nonfinite=int(h[14]),
                    vmax=float(np.array([h[15]], np.int32).view(np.float32)[0]),
                    n_active=int(h[16]))

    def advect(self, dt_sub, nsub, n_active):
        nx, ny, nz = self.shape
        _lib.call("petch_advect_sparse", self.phi.data_ptr(), self.tmp.data_ptr(),
                  self.F.data_ptr(), self.mask_phi.data_ptr(), self.mask_idx.data_ptr(),
                  int(self.mask_idx.numel()), self.active.data_ptr(), int(n_active), nx, ny, nz,
                  float(1.0 / self.dx), float(dt_sub), int(nsub), _sp())

    def reinit(self, band_r, method="fsm"):
        if method == "gpu":
            reinit_pde_dev(self.phi, self.dx, out=self.phi, scratch=(self.ua, self.ub))
        else:
            reinit_fsm_dev(self.phi, self.dx, band_r, out=self.phi, scratch=(self.ua, self.ub))

    def smooth(self, sigma):
        gaussian_smooth_dev(self.phi, sigma, self.mask, self.mask_phi, scratch=(self.ua, self.ub))

    def end_step(self, warm):
        """Keep this step's mesh + coverage for the next step's warm start."""
        if warm:
            old = self.prev
            self.prev = (self.mesh, self.bare)
            if old is not None and old[0].MT == self.MT:
                self.mesh, self.bare = old
            else:
                self.mesh = DeviceMesh(self.MT)
                self.bare = torch.empty(self.MT, device="cuda", dtype=torch.float32)


# --------------------------------------------------------------------------------------------
# drop-in functions
# --------------------------------------------------------------------------------------------
def make_trench_3d(Lx, Ly, Lz, dx, trench_width, mask_th, sub_top, hole=False, seed_cells=24,
                   host=True):
    """make_trench_3d (threed.py:32-59): the CSG field and mask, redistanced on the device.
    skfmm.distance is replaced by the Jacobi Godunov-Eikonal solve out to `seed_cells` cells
    (the etch loop reads nothing but the sign beyond the narrow band)."""
    nx, ny, nz = grid_shape(Lx, Ly, Lz, dx)
    phi_a, mask = seed_field(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, trench_width, hole)
    phi = reinit_fsm_dev(phi_a, dx, seed_cells * dx, n_iter=seed_cells + 4, mode=1)
    xs, ys, zs = np.arange(nx) * dx, np.arange(ny) * dx, np.arange(nz) * dx
    geo = dict(xs=xs, ys=ys, zs=zs, dx=dx, Lx=Lx, Ly=Ly, Lz=Lz, sub_top=sub_top,
               trench_width=trench_width, hole=hole, phi_dev=phi, mask_dev=mask)
    if host:
        geo['phi'] = phi.double().cpu().numpy()
        geo['mask'] = mask.bool().cpu().numpy()
    return geo


def run_etch_3d(Lx=10.0, Ly=4.0, Lz=14.0, dx=0.4, trench_width=4.0, mask_th=2.0,
                sub_top=10.0, t_end=2.0, n_steps=20, hole=False, par=None, flags=None,
                n_ion=20000, n_neu=20000, reinit_every=1, extend="gpu",
                reinit_method="skfmm", verbose=True, record_depth_every=0, seed_offset=0,
                rays_per_point=None, record_frames=False, surf_smooth=0.0,
                etch_stop_z=None, max_tris=None, phi_init=None, hooks=None, tune=False,
                engine="auto"):
    """run_etch_3d (threed.py:1643-1795) on the device.  Same arguments and the same returned
    `geo` dict (numpy phi / mask, `timings` per stage from CUDA events, optional depth_history /
    frames).

    reinit_method: 'gpu' runs the Russo-Smereka PDE reinit (reinit_gpu); every other method runs
    the Jacobi Godunov-Eikonal reinit ('fsm'; the reference's skfmm variants are CPU paths).
    extend: 'gpu' takes V of the nearest face (extend_velocity_gpu), anything else V of the
    nearest centroid (extend_velocity_3d).  surf_smooth > 0 applies the Gaussian smoothing and
    mask re-pin after each reinit.
    Extensions: phi_init (host or device initial level set, replacing the seed field; the mask
    and mask_phi still come from the geometry), max_tris (initial face capacity, grown on
    demand), hooks (dict of callables: before_step(step, eng), after_step(step, eng, status)),
    tune (True or a petch_b200.tune.Tuner: pick the tracer and stencil settings per size bucket
    by timing them on this run's surfaces, cached; geo['tuning'] lists the choices), engine:
    "fused" runs every step as one call of the library's fused step (petch_plan / petch_step:
    no host work or synchronisation inside a step; the coverage-coupled Monte-Carlo path with
    FSM reinit, nearest-face extension, reinit every step, no surface smoothing, etch stop,
    rays_per_point, hooks or tuner), "stages" composes each step from the stage calls here
    (every option), "auto" (default) the fused step whenever the arguments allow it."""
    if par is None:
        par = PAR
    if flags is None:
        flags = DEFAULT_FLAGS
    _unsupported(flags, par)
    if reinit_method in ("skfmm", "skfmm_full"):
        warnings.warn(f"reinit_method={reinit_method!r} (scikit-fmm's fast marching, "
                      "threed.py:1538-1549) runs as the device Jacobi Godunov-Eikonal reinit "
                      "('fsm'): pass reinit_method='fsm' to silence this", UserWarning,
                      stacklevel=2)
    if engine not in ("auto", "fused", "stages"):
        raise ValueError(f"engine must be 'auto', 'fused' or 'stages', not {engine!r}")
    if engine != "stages":
        from .plan import supported
        fusable = (supported(flags, par) and reinit_method != "gpu" and extend == "gpu"
                   and reinit_every == 1 and not surf_smooth and rays_per_point is None
                   and etch_stop_z is None and not hooks and not tune)
        if engine == "fused" and not fusable:
            raise ValueError("engine='fused' runs the coverage-coupled MC path with the default "
                             "level-set options, without hooks or tuner")
        if fusable:
            return _run_fused(Lx, Ly, Lz, dx, trench_width, mask_th, sub_top, t_end, n_steps,
                              hole, par, flags, n_ion, n_neu, verbose, record_depth_every,
                              seed_offset, record_frames, max_tris, phi_init)
    nt = getattr(flags, "neutral_transport", "mc")
    hooks = hooks or {}
    mc_par = par
    if getattr(flags, "chemistry", "langmuir") == "belen":
        mc_par = dict(par)
        mc_par['s_F'] = par['betaE']
        mc_par['s_O'] = par['betaO']
    torch.cuda.init()
    t_wall = time.time()
    geo = make_trench_3d(Lx, Ly, Lz, dx, trench_width, mask_th, sub_top, hole=hole, host=False)
    if phi_init is not None:
        src = phi_init if isinstance(phi_init, torch.Tensor) else torch.from_numpy(
            np.ascontiguousarray(phi_init))
        geo['phi_dev'] = src.to("cuda", torch.float32).contiguous().view(geo['phi_dev'].shape)
    geo['mask_th'] = mask_th
    geo['mask_phi_dev'] = geo['phi_dev'].clone()
    dt = t_end / n_steps
    band = 4 * dx
    timings = dict(flux=0.0, extend=0.0, reinit=0.0, mesh=0.0, advect=0.0, rate=0.0, total=0.0,
                   nsub_max=0)
    warm = getattr(flags, "warm_start_coverage", False)
    coupled = getattr(flags, "coverage_sticking", False)
    redepo = getattr(flags, "redeposition", False)
    eng = EtchEngine(geo, par, flags, max_tris=max_tris)
    tuner = None
    if tune:
        from .tune import Tuner
        tuner = tune if isinstance(tune, Tuner) else Tuner()
    st_timer = EventTimer()
    step = 0
    while step < n_steps:
        seed = step + seed_offset
        if 'before_step' in hooks:
            hooks['before_step'](step, eng)
        eng.small.zero_()
        st_timer.start("mesh")
        eng.build_mesh()
        if tuner is not None and tuner.ensure(eng, eng.mesh.n_faces()):
            eng.build_mesh()              # the chosen BVH width needs its own tree
        st_timer.stop("mesh")
        if rays_per_point is not None:
            F_now = eng.mesh.n_faces()
            n_eff = max(int(rays_per_point) * F_now, 1000)
            n_ion_s, n_neu_s = n_eff, n_eff
        else:
            n_ion_s, n_neu_s = n_ion, n_neu
        st_timer.start("flux")
        if nt == "radiosity":
            eng.flux_radiosity(eng.phi, n_ion_s, seed)
        elif nt == "dda":
            eng.flux_dda(eng.phi, n_ion_s, seed)
        elif nt == "knudsen":
            eng.flux_knudsen(eng.phi, n_ion_s, seed)
        elif coupled:
            eng.flux_coupled(n_ion_s, n_neu_s, seed, warm)
        else:
            eng.par = mc_par
            eng.flux_legacy(n_ion_s, n_neu_s, seed, getattr(flags, "ion_reflection", False))
            eng.par = par
        st_timer.stop("flux")
        st_timer.start("extend")
        redep = None
        if redepo:
            redep = (n_neu, step)
            if getattr(flags, "surface_charging", False) and etch_stop_z is not None:
                foot_h = max(0.3 * trench_width, 2.0 * dx)
                redep = (n_neu, step, float(etch_stop_z) + foot_h)
        eng.rate_and_extend(band, centroid=extend != "gpu", redep=redep)
        st_timer.stop("extend")
        st = eng.sync_status()
        if st['mesh_err'] & (MESH_ERR_TRI_OVERFLOW | MESH_ERR_VERT_OVERFLOW | MESH_ERR_HASH_FULL):
            eng.grow(max(st['F'], st['V']))       # redo this step with larger buffers
            continue
        if st['trace_err']:
            raise RuntimeError(f"step {step}: device traversal limit hit (error bits {st['trace_err']})")
        if st['nonfinite']:
            warnings.warn(f"step {step}: {st['nonfinite']} non-finite surface velocities (NaN/inf) "
                          "zeroed; check flux normalization / coverage if this persists.",
                          RuntimeWarning)
        vmx = st['vmax'] if st['F'] > 0 else 0.0
        Vmax = max(vmx if np.isfinite(vmx) else 0.0, 1e-6)
        nsub = max(1, min(int(np.ceil(Vmax * dt / (0.4 * dx))), 160))
        timings['nsub_max'] = max(timings['nsub_max'], nsub)
        if etch_stop_z is not None:
            below = torch.from_numpy(geo['zs'] < float(etch_stop_z)).to("cuda")
            Fv = eng.F.view(eng.shape)
            Fv[:, :, below] = torch.where(Fv[:, :, below] < 0, Fv[:, :, below], 0.0)
        st_timer.start("advect")
        eng.advect(dt / nsub, nsub, min(st['n_active'], eng.ncell))
        st_timer.stop("advect")
        if (step + 1) % reinit_every == 0 or step == n_steps - 1:
            st_timer.start("reinit")
            eng.reinit(band + 2.0 * dx, "gpu" if reinit_method == "gpu" else "fsm")
            st_timer.stop("reinit")
        if surf_smooth and surf_smooth > 0.0:
            eng.smooth(float(surf_smooth))
        eng.end_step(warm and coupled and nt == "mc")
        st['nsub'] = nsub
        if record_depth_every and (step % record_depth_every == 0 or step == n_steps - 1):
            d_now = _depth3d(dict(geo, phi=eng.phi))
            geo.setdefault('depth_history', []).append((step + 1, d_now))
            if record_frames:
                jc = eng.shape[1] // 2
                geo.setdefault('frames', []).append(
                    dict(step=step + 1, t=(step + 1) / n_steps * t_end, depth=d_now,
                         phi_xz=eng.phi[:, jc, :].double().cpu().numpy()))
        if verbose and step % 5 == 0:
            print(f"  step {step:3d}/{n_steps}  faces {st['F']:5d}  "
                  f"depth ~ {_depth3d(dict(geo, phi=eng.phi)):5.2f}  Vmax {Vmax:.3f}")
        if 'after_step' in hooks:
            hooks['after_step'](step, eng, st)
        step += 1
    ms = st_timer.totals_ms()
    for k, v in ms.items():
        timings[k] = float(np.sum(v)) / 1e3
    geo['phi'] = _to_host_f64(eng.phi)
    geo['mask'] = eng.mask.bool().cpu().numpy()
    timings['total'] = time.time() - t_wall
    geo['timings'] = timings
    geo['engine'] = eng
    if tuner is not None:
        geo['tuning'] = dict(tuner.chosen)
    for k in ('phi_dev', 'mask_dev', 'mask_phi_dev'):
        geo.pop(k, None)
    return geo


FUSED_GRAPH_MIN_STEPS = 6


def _run_fused(Lx, Ly, Lz, dx, trench_width, mask_th, sub_top, t_end, n_steps, hole, par, flags,
               n_ion, n_neu, verbose, record_depth_every, seed_offset, record_frames, max_tris,
               phi_init):
    """run_etch_3d on the fused step (plan.StepPlan): steps are enqueued without host work in
    between (from captured CUDA graphs for runs of FUSED_GRAPH_MIN_STEPS steps or more) and the
    plan's status is read once per chunk of steps (every step when the depth, frames or progress
    are recorded).  A mesh that outgrows the capacity holds its step on the
    device; the run then plans again from the held level set with twice the capacity (or 1.5x
    the largest mesh seen) and repeats the step, the new plan starting its coverage cold."""
    from .plan import StepPlan
    torch.cuda.init()
    t_wall = time.time()
    nx, ny, nz = grid_shape(Lx, Ly, Lz, dx)
    geo = dict(xs=np.arange(nx) * dx, ys=np.arange(ny) * dx, zs=np.arange(nz) * dx, dx=dx, Lx=Lx,
               Ly=Ly, Lz=Lz, sub_top=sub_top, trench_width=trench_width, hole=hole,
               mask_th=mask_th)
    dt = t_end / n_steps
    MT = int(max_tris or default_capacity((nx, ny, nz)))
    kw = dict(Lx=Lx, Ly=Ly, Lz=Lz, dx=dx, trench_width=trench_width, mask_th=mask_th,
              sub_top=sub_top, hole=hole, par=par, flags=flags, n_ion=n_ion, n_neu=n_neu)
    per_step = bool(record_frames or verbose)
    chunk = 1 if per_step else 16
    # depths without frames or progress: each step's centre-column floors are scanned on the
    # device right after it (into one slot per step of the chunk) and read back with the chunk's
    # status, so recording depths adds no host synchronisation
    floors_dev = None
    if record_depth_every and not per_step:
        I, J = center_columns(geo)
        if len(I):
            cols_dev = torch.from_numpy(np.stack([I, J], axis=1).astype(np.int32)).cuda()
            floors_dev = torch.empty((chunk, len(I)), dtype=torch.int32, device="cuda")
    # runs of a few steps or more replay each step from a captured CUDA graph (one launch per
    # step instead of ~200; the capture costs a few milliseconds once per plan)
    use_graph = n_steps >= FUSED_GRAPH_MIN_STEPS
    done, issued, nsub_max, nonfinite = 0, 0, 0, 0
    plan = StepPlan(**kw, t_end=t_end, n_steps=n_steps, seed_offset=seed_offset, max_tris=MT,
                    phi_init=phi_init, dt=dt)
    base = 0                              # steps completed before the current plan
    while done < n_steps:
        k = min(chunk, n_steps - done)
        first = done
        for i in range(k):
            if use_graph:
                plan.replay_step()
            else:
                plan.step()
            if floors_dev is not None:
                _lib.call("petch_column_floors", plan.phi.data_ptr(), nx, ny, nz,
                          cols_dev.data_ptr(), cols_dev.shape[0], floors_dev[i].data_ptr(), _sp())
        st = plan.status(check=False)
        if record_depth_every and not per_step and st['status'] in (0, 3):
            fl = floors_dev[:k].cpu().numpy() if floors_dev is not None else None
            for s_ in range(first, base + st['steps']):   # the steps that completed
                if s_ % record_depth_every == 0 or s_ == n_steps - 1:
                    d_now = _depth_from_floors(geo, fl[s_ - first] if fl is not None else None)
                    geo.setdefault('depth_history', []).append((s_ + 1, d_now))
        if st['status'] == 3:             # PETCH_E_OVERFLOW: the held steps are repeated
            done = base + st['steps']
            MT = max(2 * MT, int(1.5 * st['max_faces']))
            phi_now = plan.phi
            plan.close()
            geo['depth_history'] = [h for h in geo.get('depth_history', []) if h[0] <= done]
            geo['frames'] = [f for f in geo.get('frames', []) if f['step'] <= done]
            plan = StepPlan(**kw, t_end=dt * (n_steps - done), n_steps=n_steps - done,
                            seed_offset=seed_offset + done, max_tris=MT, phi_init=phi_now, dt=dt)
            base = done
            continue
        if st['status'] != 0:
            plan.close()
            raise _lib.PetchError(st['status'], "run_etch_3d (fused step)", _lib.last_error())
        done = base + st['steps']
        nsub_max = max(nsub_max, st['nsub_max'])
        if st['nonfinite'] > nonfinite:
            warnings.warn(f"steps up to {done}: {st['nonfinite'] - nonfinite} non-finite surface "
                          "velocities (NaN/inf) zeroed; check flux normalization / coverage if "
                          "this persists.", RuntimeWarning)
            nonfinite = st['nonfinite']
        step = done - 1
        if per_step and record_depth_every and (step % record_depth_every == 0
                                                or step == n_steps - 1):
            d_now = _depth3d(dict(geo, phi=plan.phi))
            geo.setdefault('depth_history', []).append((step + 1, d_now))
            if record_frames:
                geo.setdefault('frames', []).append(
                    dict(step=step + 1, t=(step + 1) / n_steps * t_end, depth=d_now,
                         phi_xz=plan.phi[:, ny // 2, :].double().cpu().numpy()))
        if verbose and step % 5 == 0:
            print(f"  step {step:3d}/{n_steps}  faces {st['faces']:5d}  "
                  f"depth ~ {_depth3d(dict(geo, phi=plan.phi)):5.2f}  Vmax {st['vmax']:.3f}")
    geo['mask'] = plan.mask_host()
    plan.close()
    geo['phi'] = _to_host_f64(plan.phi)
    geo['timings'] = dict(flux=0.0, extend=0.0, reinit=0.0, mesh=0.0, advect=0.0, rate=0.0,
                          total=time.time() - t_wall, nsub_max=nsub_max, fused=True)
    geo['engine'] = plan
    return geo


_STAGE = {}
_STAGE_LOCK = threading.Lock()


def _to_host_f64(t):
    """A device float32 array as a float64 numpy array: the float32 copy goes through pinned
    memory (half the bytes of a float64 copy, at the pinned rate) and is widened on the host.
    The pinned staging buffer is kept for the next call of the same size (allocating pinned
    memory took 20-35 ms a call, the copy and the widening ~3 ms)."""
    with _STAGE_LOCK:
        key = (t.dtype, t.numel())
        host = _STAGE.get(key)
        if host is None:
            _STAGE.clear()
            host = _STAGE[key] = torch.empty(t.numel(), dtype=t.dtype, pin_memory=True)
        h = host.view(t.shape)
        h.copy_(t, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return h.double().numpy()


# ---- depth metrics (threed.py:1798-1869) ----
def _floor_indices(phi, ii, jj):
    """For each column (ii[c], jj[c]) of phi: the index of the lowest cell of the gas run
    (phi < 0) that reaches the top cell, -1 when the top cell is not gas (threed.py:1822-1830).
    A device phi is scanned on the device (petch_column_floors) and only the indices come back;
    a host phi is scanned with numpy."""
    ii = np.asarray(ii, np.int64).ravel()
    jj = np.asarray(jj, np.int64).ravel()
    if isinstance(phi, torch.Tensor):
        nx, ny, nz = phi.shape
        if len(ii) == 0:
            return np.zeros(0, np.int64)
        # the scan tests phi < 0; a float64 field is reduced to its sign first (a float32 cast
        # would turn negatives smaller than the float32 subnormals into -0.0, i.e. solid)
        src = phi if phi.dtype == torch.float32 else torch.where(phi < 0, -1.0, 1.0).float()
        src = src.contiguous()
        cols = torch.from_numpy(np.stack([ii, jj], axis=1).astype(np.int32)).to(src.device)
        out = torch.empty(len(ii), dtype=torch.int32, device=src.device)
        _lib.call("petch_column_floors", src.data_ptr(), nx, ny, nz, cols.data_ptr(), len(ii),
                  out.data_ptr(), _sp())
        k = out.cpu().numpy().astype(np.int64)
        if (k == -2).any():
            raise ValueError("depth metric: a column index lies outside the grid")
        return k
    phi = np.asarray(phi)
    nz = phi.shape[2]
    gas = phi[ii, jj, :] < 0
    solid = ~gas
    k = np.where(solid.any(axis=1), nz - np.argmax(solid[:, ::-1], axis=1), 0)
    return np.where(gas[:, nz - 1], k, -1)


def center_columns(geo, half=1.0):
    """The columns (i, j) center_depth_3d samples: inside the opening, within `half` of the axis
    (threed.py:1805-1820)."""
    xs, ys = geo['xs'], geo['ys']
    cx, cy = geo['Lx'] / 2, geo['Ly'] / 2
    r_feat = geo.get('trench_width', 2.0) / 2.0 - geo['dx']
    hx = max(min(half, r_feat), geo['dx'])
    ic = np.where(np.abs(xs - cx) <= hx)[0]
    if geo.get('hole', False):
        jc = np.where(np.abs(ys - cy) <= hx)[0]
    else:
        jc = np.where(np.abs(ys - cy) <= half)[0]
    I, J = np.meshgrid(ic, jc, indexing="ij")
    I, J = I.ravel(), J.ravel()
    if geo.get('hole', False):
        keep = (xs[I] - cx) ** 2 + (ys[J] - cy) ** 2 <= r_feat ** 2
        I, J = I[keep], J[keep]
    return I, J


def _depth3d(geo, half=1.0):
    """center_depth_3d: sub_top - median floor over the central columns inside the opening.
    geo['phi'] may be a host array or the engine's device level set."""
    I, J = center_columns(geo, half)
    return _depth_from_floors(geo, _floor_indices(geo['phi'], I, J))


def _depth_from_floors(geo, k):
    """sub_top - the median of the floors zs[k] of the columns whose top cell is gas (k >= 0);
    0 when there are none."""
    if k is None:
        return 0.0
    k = np.asarray(k, np.int64)
    if (k == -2).any():
        raise ValueError("depth metric: a column index lies outside the grid")
    floors = geo['zs'][k[k >= 0]]
    if floors.size == 0:
        return 0.0
    return float(geo['sub_top'] - np.median(floors))


def center_depth_3d(geo, half=1.0):
    return _depth3d(geo, half)


def max_depth_3d(geo):
    """max_depth_3d: sub_top - 5th-percentile floor over the feature footprint."""
    phi, xs, ys, zs = geo['phi'], geo['xs'], geo['ys'], geo['zs']
    cx, cy = geo['Lx'] / 2.0, geo['Ly'] / 2.0
    r = geo.get('trench_width', 4.0) / 2.0
    if geo.get('hole', False):
        ii, jj = np.where((xs[:, None] - cx) ** 2 + (ys[None, :] - cy) ** 2 <= (r + geo['dx']) ** 2)
    else:
        ix = np.where(np.abs(xs - cx) <= r + geo['dx'])[0]
        ii, jj = np.meshgrid(ix, np.arange(len(ys)), indexing="ij")
    k = _floor_indices(phi, ii, jj)
    floors = zs[k[k >= 0]]
    if floors.size == 0:
        return 0.0
    return float(geo['sub_top'] - np.percentile(floors, 5))


def extract_mesh_3d(phi, dx, geo=None):
    """extract_mesh_3d (threed.py:62-69): (verts f32, faces i32, centroids f64, areas f64) from
    the device marching cubes."""
    return extract_mesh_3d_device(phi, dx, geo)[1]


# --------------------------------------------------------------------------------------------
# drop-in flux functions on a DeviceMesh
# --------------------------------------------------------------------------------------------
def _flux_engine(mesh, geo, par, flags):
    fe = FluxEngine(geo, par, flags, mesh.MT)
    fe.mesh = mesh                       # the caller's mesh (same face capacity)
    return fe


def _host(t, F):
    return t[:F].double().cpu().numpy()


def mc_flux_3d_coupled(mesh, verts, faces, areas, geo, par, n_ion=20000, n_neu=20000, seed=0,
                       sampling="pseudo", flags=None, n_fp=4, bare_init=None):
    """mc_flux_3d_coupled (threed.py:740-905) on a DeviceMesh (from extract_mesh_3d_device):
    returns numpy (m_i, m_F, m_O, cos_i, bare) and, on the faithful-ion path, sets
    par['_ion_yield'] like the reference.  Sources are device Philox streams whatever `sampling`
    says (the reference's CUDA path also generates them on the device); n_fp is unused there too
    (4 rounds cold, 1 from bare_init).  verts / faces / areas describe the same mesh and are not
    read."""
    F = mesh.n_faces()
    fe = _flux_engine(mesh, geo, par, flags)
    b0 = None
    if bare_init is not None:
        b0 = torch.as_tensor(np.asarray(bare_init, np.float32), device="cuda")
    phi = None
    if flags is not None and getattr(flags, "floor_charge_throttle", False):
        phi = geo['phi']
        phi = (phi if isinstance(phi, torch.Tensor)
               else torch.from_numpy(np.ascontiguousarray(phi)))
        phi = phi.to("cuda", torch.float32).contiguous()
    fe.flux_coupled(int(n_ion), int(n_neu), int(seed), False, bare_init=b0, phi=phi)
    _raise_trace_errors(fe)
    _set_ion_yield(fe, par, F)
    return (_host(fe.m_i, F), _host(fe.m_F, F), _host(fe.m_O, F), _host(fe.cos_i, F),
            _host(fe.bare, F))


def mc_flux_3d_radiosity(mesh, verts, faces, centroids, areas, geo, par, n_ion=20000, n_ff=64,
                         seed=0, flags=None, n_fp=4):
    """mc_flux_3d_radiosity (threed.py:923-991) on a DeviceMesh: returns numpy
    (m_i, m_F, m_O, cos_i) and sets or clears par['_ion_yield'] like the reference.  geo['phi']
    (host or device) is the level set the mesh was extracted from (for the into-gas normals)."""
    F = mesh.n_faces()
    fe = _flux_engine(mesh, geo, par, flags)
    phi = geo['phi']
    phi = (phi if isinstance(phi, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(phi)))
    phi = phi.to("cuda", torch.float32).contiguous()
    fe.flux_radiosity(phi, int(n_ion), int(seed), n_ff=int(n_ff), n_fp=int(n_fp))
    _raise_trace_errors(fe)
    _set_ion_yield(fe, par, F)
    return _host(fe.m_i, F), _host(fe.m_F, F), _host(fe.m_O, F), _host(fe.cos_i, F)


def mc_flux_3d_dda(mesh, verts, faces, centroids, areas, geo, par, n_ion=20000, seed=0,
                   flags=None, n_fp=4):
    """mc_flux_3d_dda (threed.py:1211-1244) on a DeviceMesh: returns numpy (m_i, m_F, m_O,
    cos_i) and sets or clears par['_ion_yield'] like the reference.  geo['phi'] (host or device)
    is the level set the mesh was extracted from; verts / faces / centroids / areas describe the
    same mesh and are not read."""
    F = mesh.n_faces()
    fe = _flux_engine(mesh, geo, par, flags)
    phi = geo['phi']
    phi = (phi if isinstance(phi, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(phi)))
    phi = phi.to("cuda", torch.float32).contiguous()
    fe.flux_dda(phi, int(n_ion), int(seed), n_fp=int(n_fp))
    _raise_trace_errors(fe)
    _set_ion_yield(fe, par, F)
    return _host(fe.m_i, F), _host(fe.m_F, F), _host(fe.m_O, F), _host(fe.cos_i, F)


def mc_flux_3d_knudsen(mesh, verts, faces, centroids, areas, geo, par, n_ion=20000, seed=0,
                       flags=None, n_fp=4):
    """mc_flux_3d_knudsen (threed.py:1149-1208) on a DeviceMesh: returns numpy (m_i, m_F, m_O,
    cos_i) and sets or clears par['_ion_yield'] like the reference.  geo carries phi (host or
    device), Lx, Ly, Lz, dx, sub_top, trench_width and hole; verts / faces / centroids / areas
    describe the same mesh and are not read."""
    F = mesh.n_faces()
    fe = _flux_engine(mesh, geo, par, flags)
    phi = geo['phi']
    phi = (phi if isinstance(phi, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(phi)))
    phi = phi.to("cuda", torch.float32).contiguous()
    fe.flux_knudsen(phi, int(n_ion), int(seed), n_fp=int(n_fp))
    _raise_trace_errors(fe)
    _set_ion_yield(fe, par, F)
    return _host(fe.m_i, F), _host(fe.m_F, F), _host(fe.m_O, F), _host(fe.cos_i, F)


def _raise_trace_errors(fe):
    err = int(fe.small[1].item())
    if err:
        raise RuntimeError(f"device traversal limit hit (error bits {err})")


def _set_ion_yield(fe, par, F):
    if fe.yields[0] is None:
        par.pop('_ion_yield', None)
    else:
        par['_ion_yield'] = tuple(_host(fe.y[q], F) for q in range(3))


def extract_mesh_3d_device(phi, dx, geo=None):
    """extract_mesh_3d_gpu + wp.Mesh (threed.py:75-100, 1674-1675) in one: the DeviceMesh (the
    handle every flux function takes as `mesh`) and its host arrays (verts f32, faces i32,
    centroids f64, areas f64)."""
    phi_t = phi if isinstance(phi, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(phi))
    phi_t = phi_t.to("cuda", torch.float32).contiguous()
    shape = tuple(phi_t.shape)
    g = geo or dict(Lx=0.0, Ly=0.0, sub_top=-1e30, mask_th=0.0, trench_width=0.0, hole=False)
    MT = default_capacity(shape)
    while True:
        mesh = DeviceMesh(MT)
        scratch = torch.empty(mesh_scratch_bytes(shape, MT), dtype=torch.uint8, device="cuda")
        mesh.build(phi_t, dx, dict(g, mask_th=g.get('mask_th', 0.0)), scratch)
        c = mesh.counts()
        if c['err'] & (MESH_ERR_TRI_OVERFLOW | MESH_ERR_VERT_OVERFLOW | MESH_ERR_HASH_FULL):
            MT = 2 * max(MT, c['F'], c['V'])
            continue
        return mesh, mesh.host_arrays()
