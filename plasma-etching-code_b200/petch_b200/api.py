"""High-level API, a drop-in for petch/api.py: Domain / SF6O2 / Process / Result.

    import petch_b200 as petch
    dom = petch.Domain.hole(extent=14, dx=0.25, diameter=6, mask=2, depth=18)
    res = petch.Process(dom, petch.SF6O2(), duration=3.0).run(steps=40)
    res.depth, res.max_depth, res.save("etch.vtk")

Same constructors, defaults and properties as the reference (petch/api.py:24-171); Process.run
drives run_etch_3d on the GPU engine with the reference's config (reinit_method="fsm").
"""
import time

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
        """Matplotlib x-z cross-section through the feature centre (if matplotlib is present)."""
        import matplotlib
        if path is not None and not show:
            matplotlib.use("Agg")
        import matplotlib.pyplot as plt
        g = self._geo
        jc = g['phi'].shape[1] // 2
        phi = g['phi'][:, jc, :].T
        fig, ax = plt.subplots(figsize=(5, 4))
        ax.contourf(g['xs'], g['zs'], (phi < 0).astype(float), levels=[0.5, 1.5], colors=["#cfe8ff"])
        ax.contour(g['xs'], g['zs'], phi, levels=[0.0], colors="k", linewidths=1.2)
        ax.axhline(g['sub_top'], color="0.6", lw=0.6, ls="--")
        ax.set_xlabel("x (um)")
        ax.set_ylabel("z (um)")
        ax.set_title(f"depth {self.depth:.1f} um  AR {self.aspect_ratio:.1f}  ({self.wall_time:.1f}s)")
        ax.set_aspect("equal")
        if path is not None:
            fig.tight_layout()
            fig.savefig(path, dpi=130)
        if show:
            plt.show()
        return ax

    def save(self, path):
        """Write the surface mesh to `path`: legacy ASCII VTK PolyData, or Wavefront .obj."""
        v, f = self.mesh
        with open(path, "w") as fh:
            if str(path).lower().endswith(".obj"):
                for p in v:
                    fh.write(f"v {p[0]} {p[1]} {p[2]}\n")
                for t in f:
                    fh.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")
            else:
                fh.write("# vtk DataFile Version 3.0\npetch surface\nASCII\nDATASET POLYDATA\n")
                fh.write(f"POINTS {len(v)} float\n")
                for p in v:
                    fh.write(f"{p[0]} {p[1]} {p[2]}\n")
                fh.write(f"POLYGONS {len(f)} {4 * len(f)}\n")
                for t in f:
                    fh.write(f"3 {int(t[0])} {int(t[1])} {int(t[2])}\n")
        return path


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
