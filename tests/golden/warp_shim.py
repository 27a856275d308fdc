"""CPU stand-in for the third-party `warp-lang` package (and the two CPU libraries the reference
imports at module level), used ONLY to execute the reference's own Python/Warp source in this
container when generating golden fixtures.

Test infrastructure, never shipped: `make_golden.py` installs these fakes into `sys.modules`, then
imports `petch/threed.py`, `petch/belen.py` and `petch/chemistry.py` from the reference checkout and
calls its kernels and host functions unmodified. Each Warp kernel body then runs as plain Python,
one thread index at a time, in float64.

What is restated here (warp-lang is unpinned in the reference's pyproject, `warp-lang>=1.13`):
  * `mesh_query_ray(mesh, o, d, tmax)`: closest triangle hit with 0 <= t <= tmax; `normal` is the
    unit geometric normal normalize(cross(b-a, c-a)), `face` the triangle index.  Brute force over
    all triangles (Moller-Trumbore in float64) -- the same closest-hit contract the Warp BVH gives.
  * `mesh_query_point_no_sign(mesh, p, dmax)`: closest point on the mesh; ties go to the lowest
    face index.
  * `rand_init/randf/randn`: an independent numpy PCG64 stream per (seed, thread).  Warp's own bit
    stream is not reproduced, so Monte-Carlo fixtures are statistical (means + standard errors).
  * `skfmm.distance` and `skimage.measure.marching_cubes` are NOT restated (they raise); fixtures
    that need a level set build it analytically and pass it through the reference's own reinit.
"""
import builtins
import math
import sys
import types

import numpy as np

_TID = [0]
_MESHES = {}


class _Arr(np.ndarray):
    """numpy array with Warp's `.numpy()` accessor."""

    def numpy(self):
        return np.asarray(self).copy()

    def zero_(self):
        self[...] = 0


def _as_arr(a, dtype=None):
    vec = dtype is vec3
    dt = np.int64 if dtype in (int, int32, uint64) else np.float64
    out = np.array(a, dtype=dt)
    if vec:
        out = out.reshape(-1, 3)
    return out.view(_Arr)


# ---- types (used in kernel annotations) ----
class uint64:  # noqa: N801
    pass


class int32:  # noqa: N801
    pass


class float32:  # noqa: N801
    pass


def vec3(x=0.0, y=0.0, z=0.0):
    return np.array([x, y, z], dtype=np.float64)


def array(data=None, dtype=None, device=None, **kw):
    if data is None:
        return None                       # annotation use: wp.array(dtype=float)
    return _as_arr(data, dtype)


def array3d(data=None, dtype=None, **kw):
    if data is None:
        return None
    return _as_arr(data, dtype)


def zeros(shape, dtype=float, device=None):
    if dtype is vec3:
        return np.zeros((int(shape), 3)).view(_Arr)
    dt = np.int64 if dtype in (int, int32) else np.float64
    return np.zeros(shape, dtype=dt).view(_Arr)


def full(shape, value, dtype=float, device=None):
    return np.full(shape, value, dtype=np.float64).view(_Arr)


def zeros_like(a):
    return np.zeros_like(a).view(_Arr)


def clone(a):
    return np.array(a).view(_Arr)


def kernel(f):
    return f


def func(f):
    return f


def struct(c):
    return c


def init():
    pass


def synchronize():
    pass


def synchronize_device(*a, **k):
    pass


def tid():
    return _TID[0]


def launch(k, dim, device=None, inputs=()):
    if isinstance(dim, (tuple, list)):
        for idx in np.ndindex(*dim):
            _TID[0] = idx
            k(*inputs)
    else:
        for p in range(int(dim)):
            _TID[0] = p
            k(*inputs)


def atomic_add(arr, idx, val):
    arr[idx] += val


# ---- math builtins ----
sqrt = math.sqrt
sin = math.sin
cos = math.cos
acos = math.acos
abs = builtins.abs  # noqa: A001


def pow(a, b):  # noqa: A001
    return math.pow(a, b)


def min(a, b):  # noqa: A001
    return a if a < b else b


def max(a, b):  # noqa: A001
    return a if a > b else b


def clamp(x, lo, hi):
    return lo if x < lo else (hi if x > hi else x)


def dot(a, b):
    return float(a[0] * b[0] + a[1] * b[1] + a[2] * b[2])


def cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


def normalize(v):
    n = math.sqrt(dot(v, v))
    return v / n if n > 0.0 else np.zeros(3)


# ---- RNG (statistical stand-in, see module docstring) ----
def rand_init(seed, offset=0):
    return np.random.Generator(np.random.PCG64([int(seed) & 0xFFFFFFFF, int(offset)]))


def randf(state):
    return float(state.random())


def randn(state):
    return float(state.standard_normal())


# ---- meshes ----
class Mesh:
    def __init__(self, points, indices, **kw):
        self.points = np.asarray(points, dtype=np.float64).reshape(-1, 3)
        self.indices = np.asarray(indices, dtype=np.int64).reshape(-1, 3)
        tri = self.points[self.indices]
        self.a = tri[:, 0]
        self.e1 = tri[:, 1] - tri[:, 0]
        self.e2 = tri[:, 2] - tri[:, 0]
        n = np.cross(self.e1, self.e2)
        ln = np.linalg.norm(n, axis=1, keepdims=True)
        self.nrm = np.where(ln > 0, n / np.where(ln > 0, ln, 1.0), 0.0)
        self.id = len(_MESHES) + 1
        _MESHES[self.id] = self


class _Q:
    __slots__ = ("result", "t", "face", "normal", "u", "v", "sign")


def mesh_query_ray(mesh_id, o, d, tmax):
    m = _MESHES[int(mesh_id)]
    o = np.asarray(o, float)
    d = np.asarray(d, float)
    p = np.cross(d[None, :], m.e2)
    det = np.einsum("ij,ij->i", m.e1, p)
    ok = np.abs(det) > 1e-300
    inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
    s = o[None, :] - m.a
    u = np.einsum("ij,ij->i", s, p) * inv
    qv = np.cross(s, m.e1)
    v = (qv @ d) * inv
    t = np.einsum("ij,ij->i", m.e2, qv) * inv
    hit = ok & (u >= 0) & (v >= 0) & (u + v <= 1) & (t >= 0) & (t <= tmax)
    q = _Q()
    if not hit.any():
        q.result = False
        q.t = 0.0
        q.face = -1
        q.normal = np.zeros(3)
        q.u = q.v = 0.0
        q.sign = 0.0
        return q
    tt = np.where(hit, t, np.inf)
    f = int(np.argmin(tt))
    q.result = True
    q.t = float(t[f])
    q.face = f
    q.normal = m.nrm[f].copy()
    q.u = float(u[f])
    q.v = float(v[f])
    q.sign = 1.0 if dot(d, q.normal) < 0 else -1.0
    return q


def _closest_on_tris(p, a, e1, e2):
    """Closest point on each triangle (a, a+e1, a+e2) to p (Ericson, Real-Time Collision Det. 5.1.5)."""
    b = a + e1
    c = a + e2
    ab, ac = e1, e2
    ap = p - a
    d1 = np.einsum("ij,ij->i", ab, ap)
    d2 = np.einsum("ij,ij->i", ac, ap)
    bp = p - b
    d3 = np.einsum("ij,ij->i", ab, bp)
    d4 = np.einsum("ij,ij->i", ac, bp)
    cp = p - c
    d5 = np.einsum("ij,ij->i", ab, cp)
    d6 = np.einsum("ij,ij->i", ac, cp)
    va = d3 * d6 - d5 * d4
    vb = d5 * d2 - d1 * d6
    vc = d1 * d4 - d3 * d2
    res = np.empty_like(a)
    done = np.zeros(len(a), bool)

    def put(mask, val):
        nonlocal done
        m = mask & ~done
        res[m] = val[m] if val.ndim == 2 else val
        done |= m

    put((d1 <= 0) & (d2 <= 0), a)
    put((d3 >= 0) & (d4 <= d3), b)
    with np.errstate(divide="ignore", invalid="ignore"):
        v_ab = d1 / (d1 - d3)
        put((vc <= 0) & (d1 >= 0) & (d3 <= 0), a + v_ab[:, None] * ab)
        put((d6 >= 0) & (d5 <= d6), c)
        w_ac = d2 / (d2 - d6)
        put((vb <= 0) & (d2 >= 0) & (d6 <= 0), a + w_ac[:, None] * ac)
        w_bc = (d4 - d3) / ((d4 - d3) + (d5 - d6))
        put((va <= 0) & ((d4 - d3) >= 0) & ((d5 - d6) >= 0), b + w_bc[:, None] * (c - b))
        denom = 1.0 / (va + vb + vc)
        v_in = vb * denom
        w_in = vc * denom
        put(np.ones(len(a), bool), a + v_in[:, None] * ab + w_in[:, None] * ac)
    return res


def mesh_query_point_no_sign(mesh_id, p, max_dist):
    m = _MESHES[int(mesh_id)]
    p = np.asarray(p, float)
    cp = _closest_on_tris(p[None, :], m.a, m.e1, m.e2)
    d2 = np.sum((cp - p[None, :]) ** 2, axis=1)
    q = _Q()
    f = int(np.argmin(d2))
    q.result = bool(d2[f] <= max_dist * max_dist)
    q.face = f
    q.t = 0.0
    q.normal = m.nrm[f].copy()
    q.u = q.v = 0.0
    q.sign = 0.0
    return q


def install(reference_src):
    """Register the fakes and a bare `petch` package rooted at the reference's src/petch (its
    __init__ is NOT executed, so the out-of-scope 2D/charging modules are never imported)."""
    me = sys.modules[__name__]
    wp = types.ModuleType("warp")
    for name in ("uint64", "int32", "float32", "vec3", "array", "array3d", "zeros", "full",
                 "zeros_like", "clone", "kernel", "func", "struct", "init", "synchronize",
                 "synchronize_device", "tid", "launch", "atomic_add", "sqrt", "sin", "cos", "acos",
                 "abs", "pow", "min", "max", "clamp", "dot", "cross", "normalize", "rand_init",
                 "randf", "randn", "Mesh", "mesh_query_ray", "mesh_query_point_no_sign"):
        setattr(wp, name, getattr(me, name))
    wp.int = int
    sys.modules["warp"] = wp

    def _no(*a, **k):
        raise NotImplementedError("not restated in the golden shim")

    skfmm = types.ModuleType("skfmm")
    skfmm.distance = _no
    sys.modules["skfmm"] = skfmm
    ski = types.ModuleType("skimage")
    meas = types.ModuleType("skimage.measure")
    meas.marching_cubes = _no
    ski.measure = meas
    sys.modules["skimage"] = ski
    sys.modules["skimage.measure"] = meas

    pkg = types.ModuleType("petch")
    pkg.__path__ = [str(reference_src)]
    sys.modules["petch"] = pkg
    import importlib
    return importlib.import_module("petch.threed")
