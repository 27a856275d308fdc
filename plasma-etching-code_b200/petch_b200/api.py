"""High-level API, a drop-in for petch/api.py: Domain / SF6O2 / Process / Result.

    import petch_b200 as petch
    dom = petch.Domain.hole(extent=14, dx=0.25, diameter=6, mask=2, depth=18)
    res = petch.Process(dom, petch.SF6O2(), duration=3.0).run(steps=40)
    res.depth, res.max_depth, res.save("etch.vtk")

Same constructors, defaults and properties as the reference (petch/api.py:24-171); Process.run
drives run_etch_3d on the GPU engine with the reference's config (reinit_method="fsm").
"""
import io
import os
import time

import numpy as np

from . import threed as _t3
from .params import PAR, Flags

# friendly API name -> internal PAR key (petch/api.py:21)
_ALIASES = {"meanE": "Emean", "sigmaE": "Esig", "iedf": "ied_mode"}


class Domain:
    """Etch geometry: a circular hole or a line trench in a masked substrate (micrometres)."""

    def __init__(self, geo):
        self._geo = geo

    @classmethod
    def hole(cls, extent, dx, diameter, mask=2.0, depth=16.0, headroom=4.0):
        sub_top = float(depth)
        return cls(dict(Lx=extent, Ly=extent, Lz=sub_top + mask + headroom, dx=dx,
                        trench_width=diameter, mask_th=mask, sub_top=sub_top, hole=True))

    @classmethod
    def trench(cls, extent, dx, width, mask=2.0, depth=16.0, headroom=4.0):
        sub_top = float(depth)
        return cls(dict(Lx=extent, Ly=extent, Lz=sub_top + mask + headroom, dx=dx,
                        trench_width=width, mask_th=mask, sub_top=sub_top, hole=False))

    @property
    def feature_width(self):
        return self._geo['trench_width']


class SF6O2:
    """SF6/O2 process model (Belen coverages, ViennaPS angular yields, faithful ion reflection,
    coverage-dependent neutral sticking, warm-started coverage fixed point).  Plasma parameters
    are overridden by keyword, with the reference's aliases (meanE, sigmaE, iedf)."""

    def __init__(self, rate_scale=0.025, iedf="gauss", **overrides):
        self.par = dict(PAR)
        self.par['rate_scale'] = rate_scale
        self.par['ied_mode'] = iedf
        for k, v in overrides.items():
            self.par[_ALIASES.get(k, k)] = v
        self.flags = dict(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                          ion_reflection=True, warm_start_coverage=True, sampling="sobol")


class Result:
    """Outcome of Process.run(): etch metrics, the level set and the surface mesh."""

    def __init__(self, geo, wall_time):
        self._geo = geo
        self.wall_time = wall_time

    @property
    def depth(self):
        """Centre etch depth (um)."""
        return _t3.center_depth_3d(self._geo)

    @property
    def max_depth(self):
        return _t3.max_depth_3d(self._geo)

    @property
    def aspect_ratio(self):
        return self.max_depth / self._geo['trench_width']

    @property
    def phi(self):
        """The signed-distance level set (nx, ny, nz), numpy float64."""
        return self._geo['phi']

    @property
    def mesh(self):
        """Surface triangle mesh (verts, faces) from the device marching cubes."""
        v, f, _, _ = _t3.extract_mesh_3d(self._geo['phi'], self._geo['dx'])
        return v, f

    def plot(self, path=None, show=False):
        """The etch profile in the x-z plane through the feature centre: the gas region shaded,
        the front (phi = 0) in red, the fronts of recorded frames (run_etch_3d(record_frames=
        True)) in grey, the substrate top dotted.  Returns the matplotlib Axes; `path` writes a
        PNG, `show` opens a window."""
        import matplotlib
        if path is not None and not show:
            matplotlib.use("Agg")
        import matplotlib.pyplot as plt
        g = self._geo
        x, z = np.asarray(g['xs']), np.asarray(g['zs'])
        phi = np.asarray(g['phi'])
        xz = phi[:, phi.shape[1] // 2, :]
        aspect = (z[-1] - z[0]) / max(x[-1] - x[0], 1e-9)
        fig, ax = plt.subplots(figsize=(4.8, min(max(4.8 * aspect, 3.0), 9.0)))
        ax.imshow((xz < 0).T, origin="lower", extent=(x[0], x[-1], z[0], z[-1]), cmap="Blues",
                  vmin=0.0, vmax=2.5, interpolation="nearest", aspect="auto")
        for fr in g.get('frames', ()):
            ax.contour(x, z, np.asarray(fr['phi_xz']).T, levels=[0.0], colors="0.65",
                       linewidths=0.5)
        ax.contour(x, z, xz.T, levels=[0.0], colors="crimson", linewidths=1.0)
        ax.plot([x[0], x[-1]], [g['sub_top'], g['sub_top']], ":", color="0.35", lw=0.8)
        ax.set_xlabel("x [um]")
        ax.set_ylabel("z [um]")
        ax.set_title(f"centre depth {self.depth:.2f} um, max {self.max_depth:.2f} um, "
                     f"AR {self.aspect_ratio:.2f}", fontsize=9)
        if path is not None:
            fig.savefig(path, dpi=120, bbox_inches="tight")
        if show:
            plt.show()
        return ax

    def save(self, path):
        """Write the surface mesh to `path`: Wavefront OBJ for a .obj suffix, legacy ASCII VTK
        PolyData (readable by ParaView / ViennaPS) otherwise."""
        v, f = self.mesh
        writer = _MESH_WRITERS.get(os.path.splitext(str(path))[1].lower(), _vtk_polydata)
        with open(path, "w") as fh:
            fh.write(writer(np.asarray(v, np.float32), np.asarray(f, np.int64)))
        return path


def _table(rows, fmt):
    """Rows of a numeric array as text, one line each (numpy formatting)."""
    buf = io.StringIO()
    if len(rows):
        np.savetxt(buf, rows, fmt=fmt)
    return buf.getvalue()


def _vtk_polydata(v, f):
    """Legacy VTK PolyData: the points block, then one polygon record (3, i, j, k) per face."""
    head = "# vtk DataFile Version 3.0\npetch surface\nASCII\nDATASET POLYDATA\n"
    polys = np.column_stack([np.full(len(f), 3, np.int64), f]) if len(f) else f
    return (head + f"POINTS {len(v)} float\n" + _table(v, "%.9g")
            + f"POLYGONS {len(f)} {4 * len(f)}\n" + _table(polys, "%d"))


def _wavefront_obj(v, f):
    """Wavefront OBJ: vertex records, then faces with 1-based indices."""
    return _table(v, "v %.9g %.9g %.9g") + _table(f + 1, "f %d %d %d")


_MESH_WRITERS = {".obj": _wavefront_obj, ".vtk": _vtk_polydata}


class Process:
    """Run a process `model` on a `domain` for `duration` (minutes), `steps` etch steps."""

    def __init__(self, domain, model, duration, n_ion=30000, n_neu=30000, transport="mc"):
        self.domain = domain
        self.model = model
        self.duration = float(duration)
        self.n_ion = n_ion
        self.n_neu = n_neu
        self.transport = transport

    def run(self, steps=40, verbose=False):
        flags = Flags(neutral_transport=self.transport, **self.model.flags)
        t0 = time.time()
        geo = _t3.run_etch_3d(t_end=self.duration, n_steps=steps, par=dict(self.model.par),
                              flags=flags, n_ion=self.n_ion, n_neu=self.n_neu,
                              reinit_method="fsm", verbose=verbose, **self.domain._geo)
        return Result(geo, time.time() - t0)
