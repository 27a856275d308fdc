"""ORACLE -- test infrastructure only.  ctypes wrapper around liboracle.so, the FP64 CPU
restatement of petch's per-step 3D etch loop (oracle_*.cpp; each function cites the reference
lines it follows).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product (plasma-etching-code_b200/petch_b200) never does.

    import oracle.oracle as orc
    orc.build()                     # g++ -O2 -fopenmp (no GPU needed)
    phi = orc.reinit(phi, dx, band)
"""
import ctypes
import glob
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_L = ctypes.c_longlong

_SIGS = {
    "orc_seed": [_P, _P, _I, _I, _I, _D, _D, _D, _D, _D, _D, _I],
    "orc_advect": [_P, _P, _P, _P, _I, _I, _I, _D, _D, _I],
    "orc_reinit": [_P, _P, _I, _I, _I, _D, _D, _I],
}


def build(force=False):
    """Compile every oracle_*.cpp into liboracle.so (skipped when up to date)."""
    srcs = sorted(glob.glob(os.path.join(HERE, "oracle_*.cpp")))
    hdrs = glob.glob(os.path.join(HERE, "*.h"))
    newest = max(os.path.getmtime(s) for s in srcs + hdrs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", LIB, *srcs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + r.stderr)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB)
        for name, args in _SIGS.items():
            f = getattr(_lib, name)
            f.argtypes = args
            f.restype = None
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
