"""The drop-in API's host parts on the CPU: the mesh writers (legacy VTK PolyData, Wavefront OBJ)
round-trip a mesh, and Result.plot draws a host level set."""
import os

import numpy as np
import pytest

from petch_b200 import api


def _mesh():
    rng = np.random.default_rng(0)
    return rng.uniform(0, 5, (7, 3)).astype(np.float32), rng.integers(0, 7, (4, 3))


def test_vtk_writer_round_trip():
    v, f = _mesh()
    lines = api._vtk_polydata(v, f).splitlines()
    assert lines[:4] == ["# vtk DataFile Version 3.0", "petch surface", "ASCII", "DATASET POLYDATA"]
    assert lines[4] == f"POINTS {len(v)} float"
    pts = np.array([[float(x) for x in ln.split()] for ln in lines[5:5 + len(v)]], np.float32)
    np.testing.assert_array_equal(pts, v)              # %.9g round-trips float32 exactly
    assert lines[5 + len(v)] == f"POLYGONS {len(f)} {4 * len(f)}"
    polys = np.array([[int(x) for x in ln.split()] for ln in lines[6 + len(v):]])
    np.testing.assert_array_equal(polys[:, 0], 3)
    np.testing.assert_array_equal(polys[:, 1:], f)


def test_obj_writer_round_trip():
    v, f = _mesh()
    lines = api._wavefront_obj(v, f).splitlines()
    vv = np.array([[float(x) for x in ln.split()[1:]] for ln in lines if ln.startswith("v ")],
                  np.float32)
    ff = np.array([[int(x) for x in ln.split()[1:]] for ln in lines if ln.startswith("f ")])
    np.testing.assert_array_equal(vv, v)
    np.testing.assert_array_equal(ff - 1, f)


def test_empty_mesh_writes_headers_only():
    v, f = np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int64)
    assert "POINTS 0 float" in api._vtk_polydata(v, f)
    assert api._wavefront_obj(v, f) == ""


def test_plot_writes_png(tmp_path):
    pytest.importorskip("matplotlib")
    dx = 0.25
    xs, ys, zs = np.arange(16) * dx, np.arange(16) * dx, np.arange(20) * dx
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    r = np.sqrt((X - 2.0) ** 2 + (Y - 2.0) ** 2)
    phi = np.maximum(3.0 - Z, np.minimum(Z - 1.5, 1.0 - r))   # a pit of radius 1 down to z 1.5
    geo = dict(phi=phi, xs=xs, ys=ys, zs=zs, dx=dx, Lx=4.0, Ly=4.0, sub_top=3.0, trench_width=2.0,
               hole=True, frames=[dict(phi_xz=np.maximum(3.0 - Z, 1.0 - r)[:, 8, :])])
    res = api.Result(geo, 0.1)
    p = str(tmp_path / "profile.png")
    ax = res.plot(path=p)
    assert os.path.getsize(p) > 1000
    assert "centre depth" in ax.get_title()


def test_depth_from_floors_matches_the_host_scan():
    """The fused engine's recorded depths come from device floor indices read back per chunk;
    turning indices into a depth is the host scan's last step (sub_top - median floor of the
    columns whose top cell is gas), checked here against center_depth_3d on a host level set."""
    from petch_b200 import threed as t3
    nx, ny, nz, dx = 12, 10, 40, 0.25
    geo = dict(xs=np.arange(nx) * dx, ys=np.arange(ny) * dx, zs=np.arange(nz) * dx, dx=dx,
               Lx=nx * dx, Ly=ny * dx, sub_top=6.0, trench_width=1.5, hole=True)
    rng = np.random.default_rng(3)
    floor = rng.integers(5, 30, (nx, ny))
    phi = np.ones((nx, ny, nz))
    for i in range(nx):
        for j in range(ny):
            phi[i, j, floor[i, j]:] = -1.0                 # gas from the floor to the top
    I, J = t3.center_columns(geo)
    k = t3._floor_indices(phi, I, J)
    assert t3._depth_from_floors(geo, k) == t3.center_depth_3d(dict(geo, phi=phi))
    assert t3._depth_from_floors(geo, k) == pytest.approx(
        geo['sub_top'] - np.median(geo['zs'][floor[I, J]]))
    assert t3._depth_from_floors(geo, None) == 0.0        # no centre columns
    assert t3._depth_from_floors(geo, np.full(4, -1)) == 0.0   # no column open to the top
    with pytest.raises(ValueError):
        t3._depth_from_floors(geo, np.array([3, -2]))     # a column outside the grid
