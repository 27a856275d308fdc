"""ORACLE -- test infrastructure only.  ctypes wrapper around liboracle.so (the FP64 C++
restatement in oracle_*.cpp) plus the numpy restatement of the per-face host arithmetic, and the
oracle etch loop.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
leg use this module; the product (plasma-etching-code_b200/petch_b200) never imports it.

Reference lines followed (paths within the reference project):
  mc_flux_3d_coupled   petch/threed.py:740-905     normalisation, smoothing, fixed point
  smooth_flux          petch/threed.py:129-148     pair scatter, np.add.at
  _belen_coverages     petch/threed.py:715-737
  surface_rate_belen   petch/belen.py:26-63 ; surface_rate_langmuir petch/chemistry.py:96-114
  angular_factors / _yields / _ied_yield   petch/chemistry.py:10-59
  run_etch_3d          petch/threed.py:1643-1795   CFL, band, seeds, warm start
  extend_velocity_gpu  petch/threed.py:1333-1346 ; faces_in_mask :1608-1616
  extend_velocity_3d   petch/threed.py:1310-1321   nearest centroid (the same cKDTree call)
  reinit_gpu           petch/threed.py:1349-1418   Russo-Smereka PDE sweeps
  surf_smooth          petch/threed.py:1779-1782   the same scipy gaussian_filter call
  mc_flux_3d_radiosity petch/threed.py:923-1029    _gas_normals :1553-1568, _cosine_dirs :1571-1579
                       (radiosity_solver 'gmres': the same scipy gmres call, :972-982)
  mc_redep_3d          petch/threed.py:1582-1605   wired as run_etch_3d :1730-1743
  dda_neutral_flux     petch/dda.py:26-188         gather kernel (oracle_dda.cpp), fib_sphere,
                       wall cells, dilation, Aitken; mc_flux_3d_dda petch/threed.py:1211-1244
  _depth3d / max_depth_3d petch/threed.py:1798-1869
Parity pinning: level-set stages and the per-face arithmetic against tests/golden/*.npz made by
running the reference's own code (tests/golden/make_golden.py); Monte-Carlo stages statistically
against the reference kernels' per-face means (tests/golden/flux.npz, radiosity.npz); the
radiosity fixed point exactly from the reference's recorded form-factor hits; the DDA gather
and dda_neutral_flux exactly against tests/golden/dda.npz (float64 evaluation, as the fixture
ran).  Marching cubes and the seed distance (skfmm) are third-party in the reference: parity
unpinned there.
"""
import ctypes
import glob
import os
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_U64 = ctypes.c_uint64

_SIGS = {
    "orc_seed": ([_P, _P, _I, _I, _I, _D, _D, _D, _D, _D, _D, _I], None),
    "orc_advect": ([_P, _P, _P, _P, _I, _I, _I, _D, _D, _I], None),
    "orc_reinit": ([_P, _P, _I, _I, _I, _D, _D, _I], None),
    "orc_reinit_mode": ([_P, _P, _I, _I, _I, _D, _D, _I, _I], None),
    "orc_mesh_build": ([_P, _I, _I, _I, _D, _D, _D, _D, _D, _D, _I], _P),
    "orc_mesh_from_arrays": ([_P, _I, _P, _I], _P),
    "orc_mesh_free": ([_P], None),
    "orc_mesh_counts": ([_P, _P], None),
    "orc_mesh_get": ([_P, _I, _P], None),
    "orc_mesh_raycast": ([_P, _P, _P, _I, _P, _P], None),
    "orc_mesh_nearest": ([_P, _P, _I, _P], None),
    "orc_trace_ions": ([_P, _P, _P, _U64, _I, _P], None),
    "orc_trace_neutrals": ([_P, _P, _P, _D, _U64, _U64, _I, _P], None),
    "orc_trace_legacy": ([_P, _P, _I, _D, _D, _I, _I, _D, _D, _U64, _I, _P, _P], None),
    "orc_trace_electrons": ([_P, _P, _D, _U64, _I, _P], None),
    "orc_trace_ff": ([_P, _P, _P, _P, _I, _I, _U64, _P], None),
    "orc_trace_redep": ([_P, _P, _P, _P, _I, _D, _U64, _I, _P], None),
    "orc_dda_gather": ([_P, _I, _I, _I, _P, _P, _P, _P, _I, _P, _D, _D, _D, _I, _I, _I, _I, _P],
                       None),
}


def build(force=False):
    """Compile every oracle_*.cpp into liboracle.so (skipped when up to date)."""
    srcs = sorted(glob.glob(os.path.join(HERE, "oracle_*.cpp")))
    newest = max(os.path.getmtime(s) for s in srcs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + f".{os.getpid()}.tmp"
        cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
               "-o", tmp, *srcs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + r.stderr)
        os.replace(tmp, LIB)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB)
        for name, (args, res) in _SIGS.items():
            f = getattr(_lib, name)
            f.argtypes = args
            f.restype = res
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ------------------------------- level set -------------------------------
def seed(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole):
    """make_trench_3d's analytic CSG field and mask (before skfmm)."""
    phi = np.empty((nx, ny, nz), np.float64)
    mask = np.empty((nx, ny, nz), np.uint8)
    lib().orc_seed(_p(phi), _p(mask), nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, int(hole))
    return phi, mask.astype(bool)


def advect(phi, F, mask, mask_phi, inv_dx, dt_sub, nsub):
    """advect_3d_gpu: nsub upwind substeps with mask re-pin (mask=None: F<0 marks mask cells)."""
    out = _f64(phi).copy()
    F = _f64(F)
    mp = _f64(mask_phi)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    nx, ny, nz = out.shape
    lib().orc_advect(_p(out), _p(F), None if m is None else _p(m), _p(mp), nx, ny, nz,
                     float(inv_dx), float(dt_sub), int(nsub))
    return out


def reinit(phi, dx, band, n_iter=None):
    """reinit_fsm(phi, dx, band, n_iter)."""
    phi = _f64(phi)
    if n_iter is None:
        n_iter = int(np.ceil(band / dx)) + 4
    out = np.empty_like(phi)
    nx, ny, nz = phi.shape
    lib().orc_reinit(_p(phi), _p(out), nx, ny, nz, float(dx), float(band), int(n_iter))
    return out


def seed_distance(phi_a, dx, cells=24):
    """Stand-in for skfmm.distance on the seed field: nodes with phi == 0 stay on the front at
    distance 0, the rest are redistanced from the front out to `cells` cells."""
    phi = _f64(phi_a)
    out = np.empty_like(phi)
    nx, ny, nz = phi.shape
    lib().orc_reinit_mode(_p(phi), _p(out), nx, ny, nz, float(dx), float(cells * dx),
                          int(cells + 4), 1)
    return out


def seed_distance_numpy(phi_a, dx, cells=24):
    """The same seed distance in plain numpy (cross-check of the C++ path)."""
    return _zero_front_distance(_f64(phi_a), dx, cells * dx, cells + 4)


def _zero_front_distance(phi_a, dx, band, n_iter):
    """Jacobi sweeps with zero nodes frozen at 0 plus the sign-change interface of reinit_fsm,
    in numpy."""
    big = band + 4 * dx
    nx, ny, nz = phi_a.shape
    U = np.full(phi_a.shape, big)
    fz = np.zeros(phi_a.shape, bool)
    # interface cells (reinit_fsm's _eik_init) + zero nodes
    pad = np.pad(phi_a, 1, mode="edge")
    c = phi_a
    nb = [pad[2:, 1:-1, 1:-1], pad[:-2, 1:-1, 1:-1], pad[1:-1, 2:, 1:-1], pad[1:-1, :-2, 1:-1],
          pad[1:-1, 1:-1, 2:], pad[1:-1, 1:-1, :-2]]
    iface = np.zeros_like(fz)
    for o in nb:
        iface |= (c * o) < 0
    gx = (nb[0] - nb[1]) * 0.5 / dx
    gy = (nb[2] - nb[3]) * 0.5 / dx
    gz = (nb[4] - nb[5]) * 0.5 / dx
    grad0 = np.maximum(np.sqrt(gx * gx + gy * gy + gz * gz), 0.5)
    D = np.minimum(np.abs(c) / grad0, 1.8 * dx)
    U[iface] = D[iface]
    fz |= iface
    U[c == 0] = 0.0
    fz |= c == 0
    for _ in range(n_iter):
        P = np.pad(U, 1, mode="constant", constant_values=big)
        ax = np.minimum(P[2:, 1:-1, 1:-1], P[:-2, 1:-1, 1:-1])
        ay = np.minimum(P[1:-1, 2:, 1:-1], P[1:-1, :-2, 1:-1])
        az = np.minimum(P[1:-1, 1:-1, 2:], P[1:-1, 1:-1, :-2])
        a = np.sort(np.stack([ax, ay, az]), axis=0)
        x = a[0] + dx
        d2 = np.maximum(2 * dx * dx - (a[0] - a[1]) ** 2, 0)
        x2 = 0.5 * (a[0] + a[1] + np.sqrt(d2))
        s1 = a[0] + a[1] + a[2]
        s2 = a[0] ** 2 + a[1] ** 2 + a[2] ** 2
        x3 = (s1 + np.sqrt(np.maximum(s1 * s1 - 3 * (s2 - dx * dx), 0))) / 3
        cand = np.where(x <= a[1], x, np.where(x2 <= a[2], x2, x3))
        U = np.where(fz, U, np.minimum(U, cand))
    sg = np.sign(phi_a)
    return sg * np.minimum(U, band + dx)


# ------------------------------- mesh -------------------------------
class Mesh:
    """Oracle mesh (marching cubes + geometry + adjacency + CPU BVH)."""

    def __init__(self, handle):
        self.h = handle
        c = np.zeros(2, np.int32)
        lib().orc_mesh_counts(self.h, _p(c))
        self.F, self.V = int(c[0]), int(c[1])
        F, V = self.F, self.V

        def get(which, shape, dt):
            a = np.empty(shape, dt)
            if a.size:
                lib().orc_mesh_get(self.h, which, _p(a))
            return a

        self.vnode = get(0, (V, 3), np.float64)
        self.verts = get(1, (V, 3), np.float64)
        self.faces = get(2, (F, 3), np.int32)
        self.area = get(3, (F,), np.float64)
        self.normal = get(4, (F, 3), np.float64)
        self.centroid = get(5, (F, 3), np.float64)
        self.fmask = get(6, (F,), np.uint8).astype(bool)
        self.nbr = get(7, (F, 3), np.int32)
        self.nbrw = get(8, (F, 3), np.float64)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_mesh_free(self.h)
            self.h = None

    def raycast(self, o, d):
        o, d = _f64(o), _f64(d)
        n = len(o)
        f = np.empty(n, np.int32)
        t = np.empty(n, np.float64)
        lib().orc_mesh_raycast(self.h, _p(o), _p(d), n, _p(f), _p(t))
        return f, t

    def nearest(self, p):
        p = _f64(p)
        f = np.empty(len(p), np.int32)
        if len(p):
            lib().orc_mesh_nearest(self.h, _p(p), len(p), _p(f))
        return f

    def pairs(self):
        """Edge-neighbour face pairs (i < j), the set _edge_adjacency produces."""
        i = np.repeat(np.arange(self.F), 3)
        j = self.nbr.reshape(-1)
        k = (j >= 0) & (i < j)
        return np.stack([i[k], j[k]], axis=1)


def mesh_build(phi, dx, geo):
    phi = np.ascontiguousarray(phi, dtype=np.float32)
    nx, ny, nz = phi.shape
    h = lib().orc_mesh_build(_p(phi), nx, ny, nz, float(dx), float(geo['Lx']), float(geo['Ly']),
                             float(geo['sub_top']), float(geo['mask_th']),
                             float(geo['trench_width']), int(bool(geo['hole'])))
    return Mesh(h)


def mesh_from_arrays(verts, faces):
    v = _f64(verts)
    f = np.ascontiguousarray(faces, dtype=np.int32)
    return Mesh(lib().orc_mesh_from_arrays(_p(v), len(v), _p(f), len(f)))


# ------------------------------- flux -------------------------------
def _dom(geo, par):
    return np.array([geo['Lx'], geo['Ly'], geo['Lz'], geo['Lz'] - geo['dx'],
                     float(par.get('periodic_y', 0))], np.float64)


def ion_prm(par):
    inflect = float(par.get('inflectAngle', 1.55334303))
    minang = float(par.get('minAngle', 1.3962634))
    n_l = float(par.get('n_l', 10.0))
    A_en = 1.0 / (1.0 + n_l * (1.5707963 / inflect - 1.0))
    return np.array([par['Emean'], par['Esig'], par['A_sp'], par['Eth_sp'], par['B_sp'],
                     par['A_ie'], par['Eth_ie'], par['A_p'], par['Eth_p'], inflect, minang, n_l,
                     A_en, min(par['Eth_ie'], par['Eth_sp']), par.get('thetaRMin', 1.2217305),
                     par.get('thetaRMax', 1.5707963), par['ion_ang_sigma']], np.float64)


def trace_ions(mesh, geo, par, seed, n):
    tal = np.zeros(5 * mesh.F, np.float64)
    lib().orc_trace_ions(mesh.h, _p(ion_prm(par)), _p(_dom(geo, par)), int(seed) & (2**64 - 1),
                         int(n), _p(tal))
    return tal.reshape(mesh.F, 5)


def trace_neutrals(mesh, geo, par, bare, beta, seed, n, domain=0):
    fl = np.zeros(mesh.F, np.float64)
    b = None if bare is None else _f64(bare)
    lib().orc_trace_neutrals(mesh.h, _p(_dom(geo, par)), None if b is None else _p(b),
                             float(beta), int(seed) & (2**64 - 1), int(domain), int(n), _p(fl))
    return fl


def trace_legacy(mesh, geo, par, ion, sigma, sticking, n_reemit, specular, cos_thr, eta, seed, n):
    fl = np.zeros(mesh.F, np.float64)
    ang = np.zeros(mesh.F, np.float64)
    lib().orc_trace_legacy(mesh.h, _p(_dom(geo, par)), int(ion), float(sigma), float(sticking),
                           int(n_reemit), int(specular), float(cos_thr), float(eta),
                           int(seed) & (2**64 - 1), int(n), _p(fl), _p(ang))
    return fl, ang


def trace_electrons(mesh, geo, par, sigma, seed, n):
    """The electron trace of mc_flux_3d_coupled's charging block (threed.py:852-856)."""
    fl = np.zeros(mesh.F, np.float64)
    lib().orc_trace_electrons(mesh.h, _p(_dom(geo, par)), float(sigma), int(seed) & (2**64 - 1),
                              int(n), _p(fl))
    return fl


# ------------------------------- per-face arithmetic (numpy) -------------------------------
def smooth(flux, normals, pairs, n_iter=1, alpha=1.0):
    """smooth_flux (threed.py:129-148), np.add.at pair scatter."""
    if len(pairs) == 0 or n_iter <= 0 or alpha <= 0.0:
        return flux
    raw = np.asarray(flux, np.float64)
    out = raw.copy()
    i, j = pairs[:, 0], pairs[:, 1]
    w = np.maximum(0.0, np.sum(normals[i] * normals[j], axis=1))
    for _ in range(n_iter):
        num = out.copy()
        den = np.ones(len(out))
        np.add.at(num, i, out[j] * w)
        np.add.at(den, i, w)
        np.add.at(num, j, out[i] * w)
        np.add.at(den, j, w)
        out = num / den
    return out if alpha >= 1.0 else (1.0 - alpha) * raw + alpha * out


def _ied_yield(A, Eth, par):
    mode = par.get('ied_mode', 'mean')
    Em = float(par['Emean'])
    sEth = np.sqrt(max(Eth, 0.0))
    if mode == 'mean':
        return float(A * max(np.sqrt(max(Em, 0.0)) - sEth, 0.0))
    if mode == 'gauss':
        Es = float(par.get('Esig', 10.0))
        z = np.linspace(-3.5, 3.5, 25)
        w = np.exp(-0.5 * z * z)
        w /= w.sum()
        E = np.clip(Em + Es * z, 0.0, None)
        return float((w * A * np.maximum(np.sqrt(E) - sEth, 0.0)).sum())
    dE = float(par.get('ied_dE', 40.0))
    ph = np.linspace(0.0, np.pi, 49)
    E = np.clip(Em + 0.5 * dE * np.cos(ph), 0.0, None)
    return float(np.mean(A * np.maximum(np.sqrt(E) - sEth, 0.0)))


def yields(par):
    return (_ied_yield(par['A_ie'], par['Eth_ie'], par), _ied_yield(par['A_sp'], par['Eth_sp'], par),
            _ied_yield(par['A_p'], par['Eth_p'], par))


def angular_factors(cos_i, par, mode):
    c = np.clip(cos_i, 0.0, 1.0)
    if mode == "viennaps":
        B = par.get('B_sp', 9.3)
        f_sp = np.maximum((1.0 + B * (1.0 - c * c)) * c, 0.0)
        th = np.arccos(c)
        f_ie = np.where(c >= 0.5, 1.0, np.maximum(3.0 - 6.0 * th / np.pi, 0.0))
        return f_ie, f_sp
    return c, c


def belen_coverages(m_i, m_F, m_O, cos_i, par, yield_angular, ion_yield=None):
    Yie, Ysp, Yp = yields(par)
    f_ie, _ = angular_factors(cos_i, par, yield_angular)
    Fi = par['ionFlux'] * m_i
    eps = 1e-9
    if ion_yield is not None:
        GY_ie = par['ionFlux'] * ion_yield[1]
        GY_p = par['ionFlux'] * ion_yield[2]
    else:
        GY_ie = Yie * f_ie * Fi
        GY_p = Yp * f_ie * Fi
    Gb_E = par['Fflux'] * m_F + eps
    Gb_P = par['Oflux'] * m_O + eps
    a = (par['k_sigma'] + 2.0 * GY_ie) / Gb_E
    b = (par['beta_sigma'] + GY_p) / Gb_P
    thF = 1.0 / (1.0 + a * (1.0 + 1.0 / (b + eps)))
    thO = 1.0 / (1.0 + b * (1.0 + 1.0 / (a + eps)))
    return thF, thO


def surface_rate(m_i, m_F, m_O, cos_i, is_mask, par, chemistry, yield_angular, ion_yield=None):
    Yie, Ysp, Yp = yields(par)
    f_ie, f_sp = angular_factors(cos_i, par, yield_angular)
    Fi = par['ionFlux'] * m_i
    Yie_a, Ysp_a, Yp_a = Yie * f_ie, Ysp * f_sp, Yp * f_ie
    eps = 1e-9
    if chemistry == "belen":
        if ion_yield is not None:
            sp, ie, ip = ion_yield
            GY_ie, GY_p = par['ionFlux'] * ie, par['ionFlux'] * ip
            sputter, ion_enh = par['ionFlux'] * sp, par['ionFlux'] * ie
        else:
            GY_ie, GY_p = Yie_a * Fi, Yp_a * Fi
            sputter, ion_enh = Ysp_a * Fi, Yie_a * Fi
        Gb_E = par['Fflux'] * m_F / par.get('fnorm_E', 1.0) + eps
        Gb_P = par['Oflux'] * m_O / par.get('fnorm_O', 1.0) + eps
        a = (par['k_sigma'] + 2.0 * GY_ie) / Gb_E
        b = (par['beta_sigma'] + GY_p) / Gb_P
        thF = 1.0 / (1.0 + a * (1.0 + 1.0 / (b + eps)))
        rate = par['k_sigma'] * thF / 4.0 + sputter + thF * ion_enh
        V = (1.0 / par['rho']) * rate * par['rate_scale']
    else:
        Fev, Fp = par['Fflux'] * m_F, par['Oflux'] * m_O
        rF = par['s_F'] * Fev / (Yie_a * Fi + eps)
        rO = par['s_O'] * Fp / (Yp_a * Fi + eps)
        bare = 1.0 / (1.0 + rF + rO)
        thF = rF * bare
        V = (1.0 / par['rho']) * (Yie_a * Fi * thF + Ysp_a * Fi * bare) * par['rate_scale']
    V = np.array(V, dtype=np.float64)
    V[is_mask] = 0.0
    return V


def open_field_level(x):
    """np.percentile(x[x > 1e-6], 90), 1.0 when no face is above 1e-6 (threed.py:862-863)."""
    x = np.asarray(x, np.float64)
    live = x[x > 1e-6]
    return float(np.percentile(live, 90)) if live.size else 1.0


def electron_shadow(m_i, m_e, alpha):
    """The charging factor of mc_flux_3d_coupled (threed.py:862-868): each flux relative to its
    open-field level, clipped to [0, 1]; m_i times 1 - alpha clip(1 - sh_e / max(sh_i, 1e-3), 0, 1).
    Returns (m_i scaled, ref_i, ref_e)."""
    m_i = np.asarray(m_i, np.float64)
    m_e = np.asarray(m_e, np.float64)
    ref_i, ref_e = open_field_level(m_i), open_field_level(m_e)
    sh_e = np.clip(m_e / max(ref_e, 1e-6), 0.0, 1.0)
    sh_i = np.clip(m_i / max(ref_i, 1e-6), 0.0, 1.0)
    f = 1.0 - alpha * np.clip(1.0 - sh_e / np.maximum(sh_i, 1e-3), 0.0, 1.0)
    return m_i * f, ref_i, ref_e


def electron_flux(fe, A, A_src, n_neu, par, sm):
    """m_e of the charging block (threed.py:857-859): the normalised electron arrival times eFlux,
    clipped to [0, 8], smoothed like the other fluxes."""
    return sm(np.clip((fe / A) / (n_neu / A_src) * par.get('eFlux', 1.0), 0.0, 8.0))


def flux_coupled(mesh, geo, par, flags, n_ion, n_neu, seed, bare_init=None, tt=None, phi=None):
    """mc_flux_3d_coupled (faithful-ion / legacy-ion branches, the optional electron-shadowing
    charge model, RR neutrals, the optional floor throttle) on the oracle mesh.  Returns (m_i,
    m_F, m_O, cos_i, bare, ion_yield-or-None).  tt: optional dict that accumulates the seconds
    spent in the ray tracers under key 'trace'; phi: the level set (for the throttle's into-gas
    normals)."""
    tt = {} if tt is None else tt
    tt.setdefault('trace', 0.0)

    def timed(fn, *a):
        t0 = time.time()
        r = fn(*a)
        tt['trace'] += time.time() - t0
        return r

    A_src = geo['Lx'] * geo['Ly']
    A = np.maximum(mesh.area, 1e-9)
    n_smooth = int(par.get('flux_smooth', 1))
    alpha = float(par.get('flux_smooth_alpha', 1.0))
    pairs = mesh.pairs()
    sm = (lambda x: smooth(x, mesh.normal, pairs, n_smooth, alpha)) if n_smooth > 0 else (lambda x: x)
    faithful = getattr(flags, "ion_reflection", False) and getattr(flags, "chemistry", "langmuir") == "belen"
    iy = None
    if faithful:
        tal = timed(trace_ions, mesh, geo, par, seed * 9 + 1, n_ion)
        norm = A_src / n_ion
        iy = tuple(sm((tal[:, q] / A) * norm) for q in range(3))
        fi, ai = tal[:, 3], tal[:, 4]
        m_i = sm((fi / A) * norm)
        cos_i = np.where(fi > 0, ai / np.maximum(fi, 1e-9), 0.0)
    else:
        fi, ai = timed(trace_legacy, mesh, geo, par, 1, par['ion_ang_sigma'], 1.0, 0, 0, 0.34,
                       0.8, seed * 9 + 1, n_ion)
        cos_i = np.where(fi > 0, ai / np.where(fi > 0, fi, 1.0), 0.0)
        m_i = sm(np.clip((fi / A) * (A_src / n_ion), 0.0, 1.5))
    alpha_c = float(par.get('charge_alpha', 0.0))
    if getattr(flags, "surface_charging", False) and alpha_c > 0.0:
        fe = timed(trace_electrons, mesh, geo, par, par.get('e_ang_sigma', 0.5), seed * 9 + 7,
                   n_neu)
        m_i, _, _ = electron_shadow(m_i, electron_flux(fe, A, A_src, n_neu, par, sm), alpha_c)
    if getattr(flags, "floor_charge_throttle", False):
        fn = gas_normals(mesh.verts, mesh.faces, mesh.centroid, phi, geo['dx'])
        c32 = np.asarray(mesh.verts, np.float32)[mesh.faces].mean(axis=1)
        m_i, iy = floor_throttle(m_i, iy, c32, fn[:, 2], geo)
    n_fp = int(par.get('n_fp', 1 if bare_init is not None else 4))
    bare = np.ones(mesh.F) if bare_init is None else np.clip(np.asarray(bare_init, float), 0.0, 1.0)
    betaE, betaO = par.get('betaE', 0.7), par.get('betaO', 1.0)
    m_F = m_O = np.zeros(mesh.F)
    ya = getattr(flags, "yield_angular", "cosine")
    for it in range(n_fp):
        fF = timed(trace_neutrals, mesh, geo, par, bare, betaE, seed * 9 + 2 + 2 * it, n_neu)
        m_F = sm(np.clip((fF / A) * (A_src / n_neu), 0.0, 8.0))
        fO = timed(trace_neutrals, mesh, geo, par, bare, betaO, seed * 9 + 3 + 2 * it, n_neu)
        m_O = sm(np.clip((fO / A) * (A_src / n_neu), 0.0, 8.0))
        thF, thO = belen_coverages(m_i, m_F, m_O, cos_i, par, ya, iy)
        bare = np.clip(1.0 - thF - thO, 0.0, 1.0)
    return m_i, m_F, m_O, cos_i, bare, iy


# ------------------------------- run_etch_3d options -------------------------------
def reinit_pde(phi, dx, n_iter=24):
    """reinit_gpu / _reinit_iter (threed.py:1349-1418) in float32 numpy: n_iter forward-Euler
    sweeps of step 0.3 dx, Russo-Smereka sub-cell target at interface cells."""
    f = np.float32
    a = np.asarray(phi, np.float32).copy()
    phi0 = a.copy()
    inv = f(1.0 / dx)
    dtau = f(0.3 * dx)

    def nb(x):
        p = np.pad(x, 1, mode="edge")
        return (p[:-2, 1:-1, 1:-1], p[2:, 1:-1, 1:-1], p[1:-1, :-2, 1:-1], p[1:-1, 2:, 1:-1],
                p[1:-1, 1:-1, :-2], p[1:-1, 1:-1, 2:])

    o_xm, o_xp, o_ym, o_yp, o_zm, o_zp = nb(phi0)
    s0 = phi0
    interface = ((s0 * o_xm < 0) | (s0 * o_xp < 0) | (s0 * o_ym < 0) | (s0 * o_yp < 0)
                 | (s0 * o_zm < 0) | (s0 * o_zp < 0))
    gx0 = (o_xp - o_xm) * f(0.5) * inv
    gy0 = (o_yp - o_ym) * f(0.5) * inv
    gz0 = (o_zp - o_zm) * f(0.5) * inv
    grad0 = np.maximum(np.sqrt(gx0 * gx0 + gy0 * gy0 + gz0 * gz0), f(0.5))
    dxl = f(1.0) / inv
    D = np.clip(s0 / grad0, f(-1.8) * dxl, f(1.8) * dxl)
    sgn0 = np.where(s0 < 0, f(-1.0), f(1.0))
    sgn = s0 / np.sqrt(s0 * s0 + f(0.25) / (inv * inv))
    for _ in range(n_iter):
        xm, xp, ym, yp, zm, zp = nb(a)
        Dxm, Dxp = (a - xm) * inv, (xp - a) * inv
        Dym, Dyp = (a - ym) * inv, (yp - a) * inv
        Dzm, Dzp = (a - zm) * inv, (zp - a) * inv
        pos = sgn > 0
        gx = np.where(pos, np.maximum(np.maximum(Dxm, 0), -np.minimum(Dxp, 0)),
                      np.maximum(-np.minimum(Dxm, 0), np.maximum(Dxp, 0)))
        gy = np.where(pos, np.maximum(np.maximum(Dym, 0), -np.minimum(Dyp, 0)),
                      np.maximum(-np.minimum(Dym, 0), np.maximum(Dyp, 0)))
        gz = np.where(pos, np.maximum(np.maximum(Dzm, 0), -np.minimum(Dzp, 0)),
                      np.maximum(-np.minimum(Dzm, 0), np.maximum(Dzp, 0)))
        G = np.sqrt(gx * gx + gy * gy + gz * gz)
        bulk = a - dtau * sgn * (G - f(1.0))
        front = a - dtau * inv * (sgn0 * np.abs(a) - D)
        a = np.where(interface, front, bulk).astype(np.float32)
    return a


def gaussian_smooth(phi, sigma, mask=None, mask_phi=None):
    """run_etch_3d's surf_smooth step (threed.py:1779-1782): the same scipy call, then the mask
    re-pin."""
    from scipy.ndimage import gaussian_filter
    out = gaussian_filter(np.asarray(phi, np.float64), sigma)
    if mask is not None:
        out[mask] = np.asarray(mask_phi, np.float64)[mask]
    return out


def extend_nearest_centroid(V, centroids, phi, dx, band):
    """extend_velocity_3d (threed.py:1310-1321): band cells take V of the nearest centroid."""
    from scipy.spatial import cKDTree
    Fs = np.zeros(phi.shape)
    bm = np.abs(phi) < band
    ii, jj, kk = np.where(bm)
    if len(centroids) == 0 or len(ii) == 0:
        return Fs
    pts = np.stack([ii * dx, jj * dx, kk * dx], axis=1)
    _, idx = cKDTree(centroids).query(pts)
    Fs[ii, jj, kk] = np.asarray(V)[idx]
    return Fs


# ------------------------------- redeposition -------------------------------
def redep(mesh, fn, src_flux, n_redep, s_redep, seed):
    """mc_redep_3d (threed.py:1582-1605): redeposited flux density per face."""
    F = mesh.F
    if F == 0:
        return np.zeros(0)
    w = np.maximum(np.asarray(src_flux, np.float64) * mesh.area, 0.0)
    tot = float(w.sum())
    if tot <= 0.0:
        return np.zeros(F)
    cdf = np.cumsum(w)
    fl = np.zeros(F)
    lib().orc_trace_redep(mesh.h, _p(_f64(fn)), _p(_f64(mesh.centroid)), _p(cdf), F,
                          float(s_redep), int(seed) & (2**64 - 1), int(n_redep), _p(fl))
    return (fl * (tot / n_redep)) / np.maximum(mesh.area, 1e-9)


# ------------------------------- radiosity neutrals -------------------------------
def gas_normals(verts, faces, centroids, phi, dx):
    """_gas_normals (threed.py:1553-1568): float32 winding normals of the float32 vertices,
    flipped to agree with -np.gradient(phi) at the rounded, clipped centroid node."""
    vv = np.asarray(verts, np.float32)[np.asarray(faces)]
    fn = np.cross(vv[:, 1] - vv[:, 0], vv[:, 2] - vv[:, 0])
    fn = fn / (np.linalg.norm(fn, axis=1, keepdims=True) + np.float32(1e-12))
    gx, gy, gz = np.gradient(np.asarray(phi, np.float64), dx)
    c = np.asarray(centroids, np.float64)
    ix = np.clip((c[:, 0] / dx).round().astype(int), 0, gx.shape[0] - 1)
    iy = np.clip((c[:, 1] / dx).round().astype(int), 0, gx.shape[1] - 1)
    iz = np.clip((c[:, 2] / dx).round().astype(int), 0, gx.shape[2] - 1)
    into_gas = -np.stack([gx[ix, iy, iz], gy[ix, iy, iz], gz[ix, iy, iz]], axis=1)
    flip = np.sum(fn * into_gas, axis=1) < 0.0
    fn[flip] *= -1.0
    return fn


def trace_ff(mesh, geo, par, fn, centroids, n_ff, seed):
    """The form-factor cast (threed.py:947-956 + _trace_ff :908-920): int[F * n_ff] first-hit
    faces, -1 for escapes; ray k of face j at index j * n_ff + k."""
    F = len(fn)
    hit = np.empty(F * n_ff, np.int32)
    if F:
        lib().orc_trace_ff(mesh.h, _p(_dom(geo, par)), _p(_f64(fn)), _p(_f64(centroids)), F,
                           int(n_ff), int(seed) & (2**64 - 1), _p(hit))
    return hit


def ff_matrix(hit, F, n_ff):
    """D (sky view) and the CSR A[i, j] = F_{j->i} of mc_flux_3d_radiosity (threed.py:957-960)."""
    import scipy.sparse as sp
    hit = np.asarray(hit)
    src = np.repeat(np.arange(F), n_ff)
    esc = hit < 0
    D = np.bincount(src[esc], minlength=F).astype(np.float64) / n_ff
    j = src[~esc]
    i = hit[~esc]
    Aff = sp.coo_matrix((np.full(len(i), 1.0 / n_ff), (i, j)), shape=(F, F)).tocsr()
    return D, Aff


def radiosity_solve(Aff, D, bare, beta, n_iter=40, solver="jacobi"):
    """solve() of mc_flux_3d_radiosity (threed.py:966-985): n_iter Jacobi sweeps G = D + M G, or
    (solver 'gmres') scipy's restarted GMRES on (I - M) G = D with rtol 1e-3, restart 12, at most
    40 cycles, the Jacobi sweeps when it does not converge."""
    s = np.clip(bare * beta, 0.0, 1.0)
    M = Aff.multiply((1.0 - s)[None, :]).tocsr()

    def jacobi():
        G = D.copy()
        for _ in range(n_iter):
            G = D + M.dot(G)
        return G

    if solver == "gmres":
        from scipy.sparse.linalg import LinearOperator, gmres
        n = len(D)
        op = LinearOperator((n, n), matvec=lambda x: x - M.dot(x), dtype=float)
        G, info = gmres(op, D, rtol=1e-3, atol=0.0, restart=12, maxiter=40)
        if info != 0:
            G = jacobi()
    else:
        G = jacobi()
    return np.clip(G, 0.0, 8.0)


def radiosity_ions(mesh, geo, par, flags, n_ion, seed):
    """_ions_deterministic (threed.py:994-1029): (m_i, cos_i, ion_yield-or-None), unsmoothed."""
    A_src = geo['Lx'] * geo['Ly']
    A = np.maximum(mesh.area, 1e-9)
    faithful = getattr(flags, "ion_reflection", False) and getattr(flags, "chemistry", "langmuir") == "belen"
    if faithful:
        tal = trace_ions(mesh, geo, par, seed * 9 + 1, n_ion)
        norm = A_src / n_ion
        iy = tuple((tal[:, q] / A) * norm for q in range(3))
        fi, ai = tal[:, 3], tal[:, 4]
        m_i = (fi / A) * norm
    else:
        fi, ai = trace_legacy(mesh, geo, par, 1, par['ion_ang_sigma'], 1.0, 0, 0, 0.34, 0.8,
                              seed * 9 + 1, n_ion)
        iy = None
        m_i = np.clip((fi / A) / (n_ion / A_src), 0.0, 1.5)
    cos_i = np.where(fi > 0, ai / np.maximum(fi, 1e-9), 0.0)
    return m_i, cos_i, iy


def radiosity_fixed_point(D, Aff, m_i, cos_i, iy, par, flags, n_fp=4, n_iter=40):
    """The coverage <-> radiosity fixed point of mc_flux_3d_radiosity (threed.py:986-990), with
    par['radiosity_solver'] ('jacobi' or 'gmres')."""
    solver = par.get('radiosity_solver', 'jacobi')
    F = len(D)
    bare = np.ones(F)
    betaE, betaO = par.get('betaE', 0.7), par.get('betaO', 1.0)
    ya = getattr(flags, "yield_angular", "cosine")
    m_F = m_O = np.zeros(F)
    for _ in range(n_fp):
        m_F = radiosity_solve(Aff, D, bare, betaE, n_iter, solver)
        m_O = radiosity_solve(Aff, D, bare, betaO, n_iter, solver)
        thF, thO = belen_coverages(m_i, m_F, m_O, cos_i, par, ya, iy)
        bare = np.clip(1.0 - thF - thO, 0.0, 1.0)
    return m_F, m_O


def flux_radiosity(mesh, geo, phi, par, flags, n_ion, seed, n_ff=64, tt=None):
    """mc_flux_3d_radiosity (threed.py:923-991) on the oracle mesh: (m_i, m_F, m_O, cos_i,
    ion_yield-or-None)."""
    tt = {} if tt is None else tt
    tt.setdefault('trace', 0.0)
    t0 = time.time()
    m_i, cos_i, iy = radiosity_ions(mesh, geo, par, flags, n_ion, seed)
    fn = gas_normals(mesh.verts, mesh.faces, mesh.centroid, phi, geo['dx'])
    hit = trace_ff(mesh, geo, par, fn, mesh.centroid, n_ff, seed)
    tt['trace'] += time.time() - t0
    D, Aff = ff_matrix(hit, mesh.F, n_ff)
    m_F, m_O = radiosity_fixed_point(D, Aff, m_i, cos_i, iy, par, flags)
    return m_i, m_F, m_O, cos_i, iy


# ------------------------------- DDA neutrals -------------------------------
def fib_sphere(n):
    """fib_sphere (dda.py:120-129): n Fibonacci directions on the full sphere, unit weights."""
    i = np.arange(n) + 0.5
    z = 1.0 - 2.0 * i / n
    r = np.sqrt(np.maximum(1.0 - z * z, 0.0))
    gold = np.pi * (1.0 + 5.0 ** 0.5)
    theta = gold * i
    return np.stack([r * np.cos(theta), r * np.sin(theta), z], axis=1), np.ones(n)


def dda_gather(phi, dx, origins, normals, dirs, weights, remit, z_top, src_top, max_steps,
               periodic_y=0, f32=False):
    """One launch of _dda_gather_kernel (dda.py:26-96): the arriving flux per origin.  The
    arrays are rounded to float32 as the reference uploads them; f32 evaluates in float32 (the
    device's arithmetic), else in float64 (the golden fixture's)."""
    phi = np.ascontiguousarray(phi, np.float32)
    nx, ny, nz = phi.shape
    r32 = lambda a: np.ascontiguousarray(np.asarray(a, np.float32), np.float64)  # noqa: E731
    o, n, d, w = r32(origins), r32(normals), r32(dirs), r32(weights)
    rem = r32(np.ravel(remit))
    N = len(o)
    out = np.zeros(N)
    if N:
        lib().orc_dda_gather(_p(phi), nx, ny, nz, _p(o), _p(n), _p(d), _p(w), len(d), _p(rem),
                             float(dx), float(z_top), float(src_top), int(max_steps),
                             int(periodic_y), N, int(bool(f32)), _p(out))
    return out


def dda_wall_cells(centroids, normals, dx, shape):
    """The solid-side cell of each face (dda.py:143-149): round(centroid - 0.7 dx n)."""
    nx, ny, nz = shape
    spos = np.asarray(centroids, np.float64) - 0.7 * dx * np.asarray(normals, np.float64)
    inv = 1.0 / dx
    six = np.clip((spos[:, 0] * inv + 0.5).astype(np.int64), 0, nx - 1)
    siy = np.clip((spos[:, 1] * inv + 0.5).astype(np.int64), 0, ny - 1)
    siz = np.clip((spos[:, 2] * inv + 0.5).astype(np.int64), 0, nz - 1)
    return (six * ny + siy) * nz + siz


def dda_neutral_flux(phi, dx, zs, centroids, normals, s_face, n_dir=64, n_reemit=12, z_top=None,
                     face_areas=None, periodic_y=0, f32=False):
    """dda_neutral_flux (dda.py:132-188): the direct view, then n_reemit passes of
    vf = direct + gather(area-weighted cell re-emission (1 - s) vf, dilated once into unseeded
    solid neighbours), then Aitken extrapolation of the last three iterates."""
    phi = np.asarray(phi)
    nx, ny, nz = phi.shape
    F = len(centroids)
    if z_top is None:
        z_top = zs[-1] - 0.5 * dx
    dirs, weights = fib_sphere(2 * n_dir)
    wall_cell = dda_wall_cells(centroids, normals, dx, phi.shape)
    max_steps = (int((z_top - zs[0]) / dx) + 4) * (3 if periodic_y else 1)

    def gather(remit, src):
        return dda_gather(phi, dx, centroids, normals, dirs, weights, remit, z_top, src,
                          max_steps, periodic_y, f32)

    direct = gather(np.zeros(nx * ny * nz), 1.0)
    vf = direct.copy()
    alpha = np.clip(1.0 - np.asarray(s_face, float), 0.0, 1.0)
    A_face = np.asarray(face_areas, float) if face_areas is not None else np.ones(F)
    cell_area = np.zeros(nx * ny * nz)
    np.add.at(cell_area, wall_cell, A_face)
    solid = phi > 0.0
    seeded = np.zeros((nx, ny, nz), bool)
    seeded.ravel()[wall_cell] = True
    need = solid & ~seeded
    prev2 = prev1 = None
    for _ in range(max(1, n_reemit)):
        remit = np.zeros(nx * ny * nz)
        np.add.at(remit, wall_cell, A_face * alpha * np.maximum(vf, 0.0))
        remit /= np.maximum(cell_area, 1e-12)
        R = remit.reshape(nx, ny, nz)
        num = np.zeros_like(R)
        cnt = np.zeros_like(R)
        for ax in (0, 1, 2):
            for sh in (1, -1):
                num += np.where(np.roll(seeded, sh, axis=ax), np.roll(R, sh, axis=ax), 0.0)
                cnt += np.roll(seeded, sh, axis=ax)
        fill = need & (cnt > 0)
        R[fill] = num[fill] / cnt[fill]
        prev2, prev1 = prev1, vf
        vf = direct + gather(R.ravel(), 0.0)
    if prev2 is not None:
        d1 = vf - prev1
        d0 = prev1 - prev2
        big = np.abs(d0) > 1e-12
        r = np.where(big, d1 / np.where(big, d0, 1.0), 0.0)
        r = np.clip(r, 0.0, 0.995)
        vf = vf + d1 * r / (1.0 - r)
    return np.clip(np.maximum(vf, 0.0), 0.0, 8.0)


def dda_fixed_point(phi, dx, zs, centroids, fn, areas, m_i, cos_i, iy, par, flags, n_fp=4,
                    f32=False):
    """The coverage <-> DDA fixed point of mc_flux_3d_dda (threed.py:1234-1243)."""
    F = len(centroids)
    A = np.maximum(areas, 1e-9)
    betaE, betaO = par.get('betaE', 0.7), par.get('betaO', 1.0)
    n_dir, n_re = int(par.get('dda_n_dir', 64)), int(par.get('dda_n_reemit', 12))
    per = int(par.get('periodic_y', 0))
    ya = getattr(flags, "yield_angular", "cosine")
    bare = np.ones(F)
    m_F = m_O = np.zeros(F)
    for _ in range(n_fp):
        m_F = dda_neutral_flux(phi, dx, zs, centroids, fn, np.clip(bare * betaE, 0.0, 1.0), n_dir,
                               n_re, face_areas=A, periodic_y=per, f32=f32)
        m_O = dda_neutral_flux(phi, dx, zs, centroids, fn, np.clip(bare * betaO, 0.0, 1.0), n_dir,
                               n_re, face_areas=A, periodic_y=per, f32=f32)
        thF, thO = belen_coverages(m_i, m_F, m_O, cos_i, par, ya, iy)
        bare = np.clip(1.0 - thF - thO, 0.0, 1.0)
    return m_F, m_O


def flux_dda(mesh, geo, phi, par, flags, n_ion, seed, tt=None):
    """mc_flux_3d_dda (threed.py:1211-1244) on the oracle mesh: (m_i, m_F, m_O, cos_i,
    ion_yield-or-None); the DDA in float32 arithmetic (the device's)."""
    tt = {} if tt is None else tt
    tt.setdefault('trace', 0.0)
    t0 = time.time()
    m_i, cos_i, iy = radiosity_ions(mesh, geo, par, flags, n_ion, seed)
    tt['trace'] += time.time() - t0
    fn = gas_normals(mesh.verts, mesh.faces, mesh.centroid, phi, geo['dx'])
    zs = np.arange(np.asarray(phi).shape[2]) * geo['dx']
    m_F, m_O = dda_fixed_point(phi, geo['dx'], zs, mesh.centroid, fn, mesh.area, m_i, cos_i, iy,
                               par, flags, f32=True)
    return m_i, m_F, m_O, cos_i, iy


# ------------------------------- Knudsen tail -------------------------------
def kn_slice_geometry(phi, zs, dx, sub_top, trench):
    """slice_geometry (knudsen.py:29-68): per z-slice below sub_top, the gas area and the
    sidewall perimeter.  Hole: area = gas cells dx^2, perimeter = max(gas/solid cell faces in
    the slice, 1) dx.  Trench: area = mean open x-width over the y-rows with any gas,
    perimeter = 2."""
    gas = np.asarray(phi) < 0.0
    nz = gas.shape[2]
    area, perim = np.zeros(nz), np.zeros(nz)
    for k in np.flatnonzero(np.asarray(zs) < sub_top):
        g = gas[:, :, k]
        if trench:
            w = g.sum(axis=0) * dx
            w = w[w > 0.0]
            if w.size:
                area[k], perim[k] = float(w.mean()), 2.0
        elif g.any():
            area[k] = float(g.sum()) * dx * dx
            nf = np.count_nonzero(g[1:, :] != g[:-1, :]) + np.count_nonzero(g[:, 1:] != g[:, :-1])
            perim[k] = max(float(nf) * dx, dx)
    return area, perim


def kn_thomas(lower, diag, upper, rhs):
    """The guarded Thomas algorithm of knudsen.py:71-88."""
    n = len(diag)
    if n == 0:
        return np.zeros(0)
    b, d = np.array(diag, float), np.array(rhs, float)
    for i in range(1, n):
        w = lower[i - 1] / max(b[i - 1], 1.0e-30)
        b[i] -= w * upper[i - 1]
        d[i] -= w * d[i - 1]
    x = np.zeros(n)
    x[-1] = d[-1] / max(b[-1], 1.0e-30)
    for i in range(n - 2, -1, -1):
        x[i] = (d[i] - upper[i] * x[i + 1]) / max(b[i], 1.0e-30)
    return x


def kn_profile(phi, zs, dx, sub_top, trench, slice_loss, loss_scale):
    """conductance_profile (knudsen.py:91-150): the neutral concentration per slice from the
    chain of valid slices, opening first: conductance (2/3) r a / dx with r = max(2a/p, dx),
    harmonic-mean links between adjacent slices, unit concentration through the opening's own
    conductance, sink loss_scale * slice_loss.  1 outside the chain."""
    area, perim = kn_slice_geometry(phi, zs, dx, sub_top, trench)
    valid = (np.asarray(zs) < sub_top) & (area > 0.0) & (perim > 0.0)
    prof = np.ones(len(area))
    if not valid.any():
        return prof
    idx = np.flatnonzero(valid)[::-1]
    a, p = area[idx], perim[idx]
    r = np.maximum(2.0 * a / np.maximum(p, 1.0e-30), dx)
    cond = (2.0 / 3.0) * r * a / dx
    ls = np.asarray(loss_scale, float)
    scale = np.maximum(float(ls), 0.0) if ls.ndim == 0 else np.maximum(ls[idx], 0.0)
    sink = scale * np.maximum(np.asarray(slice_loss)[idx], 0.0)
    m = len(idx)
    diag = np.array(sink, float) * np.ones(m)
    lower, upper, rhs = np.zeros(max(m - 1, 0)), np.zeros(max(m - 1, 0)), np.zeros(m)
    diag[0] += cond[0]
    rhs[0] += cond[0]
    for i in range(m - 1):
        g = 0.0
        if abs(idx[i + 1] - idx[i]) == 1:
            g = 2.0 * cond[i] * cond[i + 1] / max(cond[i] + cond[i + 1], 1.0e-30)
        diag[i] += g
        diag[i + 1] += g
        upper[i] = -g
        lower[i] = -g
    prof[idx] = np.clip(kn_thomas(lower, np.maximum(diag, 1.0e-30), upper, rhs), 0.0, 1.0)
    return prof


def kn_front_scale(zs, sub_top, W, wls, band_W, pass_frac, ar_pass):
    """_front_loss_scale (knudsen.py:165-185): wls (f + (1 - f) exp(-max(AR - band, 0) / ar))
    per slice, AR = max(sub_top - z, 0) / W."""
    ar = np.maximum((sub_top - np.asarray(zs)) / max(W, 1.0e-9), 0.0)
    g = np.exp(-np.maximum(ar - band_W, 0.0) / max(ar_pass, 1.0e-9))
    return max(float(wls), 0.0) * (pass_frac + (1.0 - pass_frac) * g)


def kn_face_flux(phi, zs, dx, sub_top, trench, centroids, gas_nz, A, Ly, s_face, wls,
                 center=None, half_width=None, front_loss=False, band_W=8.0, pass_frac=0.5,
                 ar_pass=15.0):
    """knudsen_face_flux (knudsen.py:188-241): each face's slice (rounded centroid height,
    snapped to the nearest valid slice, ties to the lower), the floor faces (into-gas n_z > 0.7)
    below sub_top inside the footprint add 0.25 s A to their slice's sink (per unit trench
    length), and every face below sub_top takes its slice's concentration; 1 elsewhere."""
    zs = np.asarray(zs)
    nz = np.asarray(phi).shape[2]
    area, perim = kn_slice_geometry(phi, zs, dx, sub_top, trench)
    vz = np.flatnonzero((zs < sub_top) & (area > 0.0) & (perim > 0.0))
    c = np.asarray(centroids, float)
    iz = np.clip(np.round((c[:, 2] - zs[0]) / dx).astype(int), 0, nz - 1)
    if vz.size == 0:
        snap = np.full(len(c), -1)
    else:
        pos = np.searchsorted(vz, iz)
        hi, lo = vz[np.clip(pos, 0, vz.size - 1)], vz[np.clip(pos - 1, 0, vz.size - 1)]
        snap = np.where(np.abs(hi - iz) < np.abs(lo - iz), hi, lo)
    below = c[:, 2] < sub_top
    inside = np.ones(len(c), bool)
    if center is not None and half_width is not None:
        band = half_width + 2.0 * dx
        if trench:
            inside = np.abs(c[:, 0] - center[0]) <= band
        else:
            inside = np.hypot(c[:, 0] - center[0], c[:, 1] - center[1]) <= band
    loss = np.zeros(nz)
    sel = below & inside & (snap >= 0) & (np.asarray(gas_nz) > 0.7)
    if sel.any():
        np.add.at(loss, snap[sel], 0.25 * (np.clip(np.asarray(s_face, float)[sel], 0.0, 1.0)
                                           * np.asarray(A, float)[sel]))
        if trench:
            loss /= max(float(Ly), 1.0e-30)
    scale = wls
    if front_loss:
        W = 2.0 * float(half_width) if half_width is not None else dx
        scale = kn_front_scale(zs[:nz], sub_top, W, wls, band_W, pass_frac, ar_pass)
    prof = kn_profile(phi, zs, dx, sub_top, trench, loss, scale)
    m = np.ones(len(c))
    take = (snap >= 0) & below
    m[take] = prof[snap[take]]
    return np.clip(m, 0.0, 8.0)


# Floor-charging tables (the reference's data, restated): the Hwang-Giapis published values
# (charging2d.py:1511-1518), petch's own first-principles table (charging_general.py:1038-1041)
# and the de Boer deep-AR throttle (charging_general.py:1070-1071).
HG_AR = np.array([0.0, 1.0, 1.2, 1.6, 2.0, 2.6, 3.0, 3.6, 4.0])
HG_Q = np.array([1.0, 0.59, 0.55, 0.47, 0.40, 0.34, 0.30, 0.26, 0.22])
HG_VF = np.array([0.0, 8.0, 10.0, 15.0, 19.0, 25.0, 28.0, 31.0, 33.0])
HG_E = np.array([0.0, 15.0, 16.5, 17.5, 20.0, 23.0, 25.0, 26.5, 27.5])
PT_AR = np.array([1.0, 2.0, 3.0, 4.0])
PT_Q = np.array([0.704, 0.491, 0.406, 0.349])
PT_VF = np.array([9.5, 19.2, 27.7, 34.0])
PT_E = np.array([16.6, 14.2, 18.8, 21.6])
TH_AR = np.array([0.0, 1.0, 2.0, 3.0, 4.0, 8.0, 15.0, 25.0])
TH_Q = np.array([1.0, 0.704, 0.491, 0.406, 0.349, 0.25, 0.60, 0.50])


def _footprint_floor(centroids, gas_nz, geo):
    """The in-feature faces below sub_top (within half the width + 2 dx of the axis) and those
    of them facing up (n_z > 0.7)."""
    c = np.asarray(centroids, float)
    cx0, cy0 = 0.5 * geo['Lx'], 0.5 * geo['Ly']
    hw = 0.5 * geo['trench_width'] + 2.0 * geo['dx']
    if geo.get('hole', False):
        inside = np.hypot(c[:, 0] - cx0, c[:, 1] - cy0) <= hw
    else:
        inside = np.abs(c[:, 0] - cx0) <= hw
    below = c[:, 2] < geo['sub_top']
    return inside & below, inside & below & (np.asarray(gas_nz) > 0.7)


def hg_charging(m_i, iy, par, mode, centroids, gas_nz, A, geo):
    """_apply_hg_charging (threed.py:1046-1110): returns (m_i, (sp, ie, ip)).  The floor flux
    keeps the fraction Q(AR) with yields at Emean - V_f; the removed flux lands on the sidewall
    foot (0.3 W, at least 2 dx, above the deepest floor face) with the yields of E_defl."""
    if mode not in ("hg", "petch") or iy is None:
        return m_i, iy
    feat, floor = _footprint_floor(centroids, gas_nz, geo)
    if not floor.any():
        return m_i, iy
    c = np.asarray(centroids, float)
    W = geo['trench_width']
    AR = float(geo['sub_top'] - c[floor, 2].min()) / max(W, 1e-9)
    tab = (HG_AR, HG_Q, HG_VF, HG_E) if mode == "hg" else (PT_AR, PT_Q, PT_VF, PT_E)
    Q, Vf, Ed = (float(np.interp(AR, tab[0], t)) for t in tab[1:])
    sp, ie, ip = (np.array(a, float) for a in iy)
    y0 = yields(par)
    yv = yields(dict(par, Emean=max(par['Emean'] - Vf, 0.0)))
    r = [yv[q] / y0[q] if y0[q] > 0 else 0.0 for q in range(3)]      # (ie, sp, p)
    defl = float((m_i[floor] * A[floor]).sum()) * (1.0 - Q)
    ie[floor] *= Q * r[0]
    sp[floor] *= Q * r[1]
    ip[floor] *= Q * r[2]
    m_i = np.array(m_i, float)
    m_i[floor] *= Q
    zf = float(c[floor, 2].min())
    foot = feat & (np.asarray(gas_nz) <= 0.7) & (c[:, 2] <= zf + max(0.3 * W, 2.0 * geo['dx']))
    if foot.any() and defl > 0.0:
        fd = defl / max(float(A[foot].sum()), 1e-12)
        sE = np.sqrt(Ed)
        ie[foot] += fd * par['A_ie'] * max(sE - np.sqrt(par['Eth_ie']), 0.0)
        sp[foot] += fd * par['A_sp'] * max(sE - np.sqrt(par['Eth_sp']), 0.0)
        ip[foot] += fd * par['A_p'] * max(sE - np.sqrt(par['Eth_p']), 0.0)
    return m_i, (sp, ie, ip)


def floor_throttle(m_i, iy, centroids, gas_nz, geo):
    """_apply_floor_charge_throttle (threed.py:1112-1147): the floor faces' ion flux (and
    yields) times Q(AR) of the deep-AR throttle table (1 below AR 0, 0.5 above AR 25).  The
    reference averages the float32 vertices itself, so its depth sub_top - z_min is a float32
    subtraction (numpy's Python-scalar rule); `centroids` are those float32 means."""
    _, floor = _footprint_floor(centroids, gas_nz, geo)
    if not floor.any():
        return m_i, iy
    zmin = np.float32(np.asarray(centroids, np.float32)[floor, 2].min())
    AR = float(np.float32(geo['sub_top']) - zmin) / max(geo['trench_width'], 1e-9)
    Q = float(np.clip(np.interp(AR, TH_AR, TH_Q, left=1.0, right=float(TH_Q[-1])), 0.0, 1.0))
    m_i = np.array(m_i, float)
    m_i[floor] *= Q
    if iy is not None:
        iy = tuple(np.array(a, float) for a in iy)
        for a in iy:
            a[floor] *= Q
    return m_i, iy


def knudsen_fixed_point(phi, geo, centroids, fn, A, m_i, cos_i, iy, par, flags, n_fp=4):
    """The coverage <-> Knudsen fixed point of mc_flux_3d_knudsen (threed.py:1184-1207),
    starting from bare = 1; 'field' sinks clamp bare at the open-field faces' mean."""
    dx, sub_top = geo['dx'], geo['sub_top']
    zs = np.arange(np.asarray(phi).shape[2]) * dx
    trench = not geo.get('hole', False)
    c = np.asarray(centroids, float)
    gas_nz = np.asarray(fn)[:, 2]
    A = np.maximum(A, 1e-9)
    betaE, betaO = par.get('betaE', 0.7), par.get('betaO', 1.0)
    wls = float(par.get('knudsen_wall_loss_scale', 1.85))
    kw = dict(center=(0.5 * geo['Lx'], 0.5 * geo['Ly']),
              half_width=0.5 * float(geo.get('trench_width', geo['Lx'])),
              front_loss=bool(getattr(flags, 'knudsen_front_loss', False)),
              band_W=float(par.get('knudsen_front_band_W', 8.0)),
              pass_frac=float(par.get('knudsen_passive_frac', 0.5)),
              ar_pass=float(par.get('knudsen_front_ar_pass', 15.0)))
    ya = getattr(flags, "yield_angular", "cosine")
    field = c[:, 2] > sub_top - 0.5 * dx
    bare = np.ones(len(c))
    m_F = m_O = np.zeros(len(c))
    for _ in range(n_fp):
        sb = bare
        if par.get('knudsen_sink', 'local') == 'field' and field.any():
            sb = np.minimum(bare, float(np.mean(bare[field])))
        m_F = kn_face_flux(phi, zs, dx, sub_top, trench, c, gas_nz, A, geo['Ly'],
                           np.clip(sb * betaE, 0.0, 1.0), wls, **kw)
        m_O = kn_face_flux(phi, zs, dx, sub_top, trench, c, gas_nz, A, geo['Ly'],
                           np.clip(sb * betaO, 0.0, 1.0), wls, **kw)
        thF, thO = belen_coverages(m_i, m_F, m_O, cos_i, par, ya, iy)
        bare = np.clip(1.0 - thF - thO, 0.0, 1.0)
    return m_F, m_O


def flux_knudsen(mesh, geo, phi, par, flags, n_ion, seed, tt=None):
    """mc_flux_3d_knudsen (threed.py:1149-1208) on the oracle mesh: (m_i, m_F, m_O, cos_i,
    ion_yield-or-None), with the floor-charging closure for surface_charging hg / petch."""
    tt = {} if tt is None else tt
    tt.setdefault('trace', 0.0)
    t0 = time.time()
    m_i, cos_i, iy = radiosity_ions(mesh, geo, par, flags, n_ion, seed)
    tt['trace'] += time.time() - t0
    fn = gas_normals(mesh.verts, mesh.faces, mesh.centroid, phi, geo['dx'])
    A = np.maximum(mesh.area, 1e-9)
    m_i, iy = hg_charging(m_i, iy, par, getattr(flags, "surface_charging", False),
                          mesh.centroid, fn[:, 2], A, geo)
    m_F, m_O = knudsen_fixed_point(phi, geo, mesh.centroid, fn, A, m_i, cos_i, iy, par, flags)
    return m_i, m_F, m_O, cos_i, iy


# ------------------------------- the loop -------------------------------
def depth3d(geo, phi, half=1.0):
    """_depth3d (threed.py:1798-1834)."""
    xs, ys, zs = geo['xs'], geo['ys'], geo['zs']
    cx, cy = geo['Lx'] / 2, geo['Ly'] / 2
    r_feat = geo.get('trench_width', 2.0) / 2.0 - geo['dx']
    hx = max(min(half, r_feat), geo['dx'])
    ic = np.where(np.abs(xs - cx) <= hx)[0]
    if geo.get('hole', False):
        jc = np.where(np.abs(ys - cy) <= hx)[0]
    else:
        jc = np.where(np.abs(ys - cy) <= half)[0]
    floors = []
    for i in ic:
        for j in jc:
            if geo.get('hole', False) and (xs[i] - cx) ** 2 + (ys[j] - cy) ** 2 > r_feat ** 2:
                continue
            col = phi[i, j, :] < 0
            k = len(col) - 1
            if not col[k]:
                continue
            while k > 0 and col[k - 1]:
                k -= 1
            floors.append(zs[k])
    return 0.0 if not floors else float(geo['sub_top'] - np.median(floors))


def run_etch_3d(Lx, Ly, Lz, dx, trench_width, mask_th, sub_top, t_end, n_steps, hole, par, flags,
                n_ion, n_neu, seed_offset=0, record_depth_every=0, max_seconds=None, steps=None,
                stage_times=None, reinit_method="fsm", extend="gpu", surf_smooth=0.0,
                phi_init=None, bare_init=None):
    """run_etch_3d (threed.py:1643-1795) with the oracle's stages (coverage-coupled MC path,
    radiosity or DDA neutrals, FSM reinit, nearest-face extension).  Runs `steps` (default n_steps) steps of the n_steps
    schedule.  Returns (phi, depth_history, stats); stage_times (list) receives one dict of stage
    seconds per step.  phi_init: start from this level set instead of the seed field (mask and
    mask level set as run_etch_3d's phi_init); bare_init: the first step's starting coverage on
    phi_init's mesh (then that step runs the warm-start round count)."""
    nx, ny, nz = int(round(Lx / dx)), int(round(Ly / dx)), int(round(Lz / dx))
    phi_a, mask = seed(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, trench_width, hole)
    if phi_init is None:
        phi = seed_distance(phi_a.astype(np.float32), dx).astype(np.float32)
    else:
        phi = np.ascontiguousarray(phi_init, np.float32).reshape(nx, ny, nz).copy()
    mask_phi = phi.copy()
    geo = dict(Lx=Lx, Ly=Ly, Lz=Lz, dx=dx, sub_top=sub_top, mask_th=mask_th,
               trench_width=trench_width, hole=hole, xs=np.arange(nx) * dx,
               ys=np.arange(ny) * dx, zs=np.arange(nz) * dx)
    dt = t_end / n_steps
    band = 4 * dx
    warm = getattr(flags, "warm_start_coverage", False)
    prev = None
    hist = []
    t0 = time.time()
    steps_done = 0
    for step in range(n_steps if steps is None else min(steps, n_steps)):
        st = dict(trace=0.0)
        ta = time.time()
        mesh = mesh_build(phi, dx, geo)
        st['mesh'] = time.time() - ta
        ta = time.time()
        if getattr(flags, "neutral_transport", "mc") == "radiosity":
            m_i, m_F, m_O, cos_i, iy = flux_radiosity(mesh, geo, phi, par, flags, n_ion,
                                                      step + seed_offset, tt=st)
        elif getattr(flags, "neutral_transport", "mc") == "dda":
            m_i, m_F, m_O, cos_i, iy = flux_dda(mesh, geo, phi, par, flags, n_ion,
                                                step + seed_offset, tt=st)
        elif getattr(flags, "neutral_transport", "mc") == "knudsen":
            m_i, m_F, m_O, cos_i, iy = flux_knudsen(mesh, geo, phi, par, flags, n_ion,
                                                    step + seed_offset, tt=st)
        else:
            bi = None
            if step == 0 and bare_init is not None:
                bi = np.asarray(bare_init, np.float64)
            elif warm and prev is not None:
                pm, pb = prev
                q = pm.nearest(mesh.centroid.astype(np.float32).astype(np.float64))
                bi = np.where(q >= 0, pb[np.maximum(q, 0)], 1.0)
            m_i, m_F, m_O, cos_i, bare, iy = flux_coupled(mesh, geo, par, flags, n_ion, n_neu,
                                                          step + seed_offset, bi, tt=st, phi=phi)
            prev = (mesh, bare)
        V = surface_rate(m_i, m_F, m_O, cos_i, mesh.fmask, par,
                         getattr(flags, "chemistry", "langmuir"),
                         getattr(flags, "yield_angular", "cosine"), iy)
        V = np.nan_to_num(V, nan=0.0, posinf=0.0, neginf=0.0).astype(np.float32).astype(np.float64)
        if getattr(flags, "redeposition", False):
            fn = gas_normals(mesh.verts, mesh.faces, mesh.centroid, phi, dx)
            Rf = redep(mesh, fn, V, n_neu, par.get('s_redep', 0.5), step)
            V = np.maximum(V - par.get('k_redep', 1.0) * Rf, 0.0)
        st['flux_rate'] = time.time() - ta
        ta = time.time()
        bandm = np.abs(phi.astype(np.float64)) < band
        ii, jj, kk = np.nonzero(bandm)
        pts = np.stack([geo['xs'][ii], geo['ys'][jj], geo['zs'][kk]], axis=1)
        pts = pts.astype(np.float32).astype(np.float64)
        Fs = np.zeros(phi.shape)
        if extend != "gpu":
            Fs = extend_nearest_centroid(V, mesh.centroid, phi.astype(np.float64), dx, band)
        elif len(pts) and mesh.F:
            q = mesh.nearest(pts)
            Fs[ii, jj, kk] = np.where(q >= 0, V[np.maximum(q, 0)], 0.0)
        st['extend'] = time.time() - ta
        vmx = float(np.max(V)) if V.size else 0.0
        Vmax = max(vmx if np.isfinite(vmx) else 0.0, 1e-6)
        nsub = max(1, min(int(np.ceil(Vmax * dt / (0.4 * dx))), 160))
        ta = time.time()
        phi = advect(phi, Fs.astype(np.float32), mask, mask_phi, 1.0 / dx, dt / nsub, nsub)
        st['advect'] = time.time() - ta
        ta = time.time()
        if reinit_method == "gpu":
            phi = reinit_pde(phi.astype(np.float32), dx)
        else:
            phi = reinit(phi.astype(np.float32), dx, band + 2.0 * dx).astype(np.float32)
        if surf_smooth and surf_smooth > 0.0:
            phi = gaussian_smooth(phi, surf_smooth, mask, mask_phi).astype(np.float32)
        st['reinit'] = time.time() - ta
        st['nsub'] = nsub
        if stage_times is not None:
            stage_times.append(st)
        steps_done += 1
        if record_depth_every and (step % record_depth_every == 0 or step == n_steps - 1):
            hist.append((step + 1, depth3d(geo, phi)))
        if max_seconds is not None and time.time() - t0 > max_seconds:
            break
    return phi, hist, dict(seconds=time.time() - t0, steps=steps_done)


def timed_steps(workload, t_end, n_steps, par, flags, n_rays, n_rays_full, steps, budget_s):
    """The oracle loop on `workload` at n_rays rays per species for up to `steps` steps (stopping
    once budget_s seconds have passed); per step, the measured stage seconds and the full step
    time with the tracing time scaled linearly to n_rays_full."""
    st = []
    _, _, info = run_etch_3d(workload['Lx'], workload['Ly'], workload['Lz'], workload['dx'],
                             workload['trench_width'], workload['mask_th'], workload['sub_top'],
                             t_end, n_steps, workload['hole'], par, flags, n_rays, n_rays,
                             steps=steps, max_seconds=budget_s, stage_times=st)
    scale = n_rays_full / n_rays
    full = []
    for s in st:
        tot = s['mesh'] + s['flux_rate'] + s['extend'] + s['advect'] + s['reinit']
        full.append(tot + s['trace'] * (scale - 1.0))
    keys = ('mesh', 'trace', 'flux_rate', 'extend', 'advect', 'reinit')
    mean = {k: round(float(np.mean([s[k] for s in st])), 3) for k in keys}
    return dict(steps=info['steps'], full_step_seconds=full, stage_seconds=mean)
