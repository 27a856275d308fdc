"""The oracle's redeposition (mc_redep_3d, threed.py:1582-1605) against tests/golden/redep.npz,
the reference's own function over 8 seeds.  CPU only."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from test_radiosity_oracle import _z2, binned_z
import oracle.oracle as orc


@pytest.fixture(scope="module")
def rp():
    return np.load(os.path.join(GOLDEN, "redep.npz"))


def check_redep(runs, g, sg, verts, faces):
    """runs: [seeds, F] redeposited flux density from one implementation; g, sg: the
    reference's 8-seed mean and standard error.  Per face, z^2 with combined standard errors:
    median < 0.75 and mean < 2.2 (Student-t with 7 d.o.f.: 0.49 / 1.4); area-weighted sums over
    height bands within 3 sigma; the total within 3 %."""
    x, sx = runs.mean(0), runs.std(0, ddof=1) / np.sqrt(len(runs))
    med, mean = _z2(x, sx, g, sg)
    assert med < 0.75 and mean < 2.2, (med, mean)
    zb = binned_z(x, sx, g, sg, verts, faces)
    assert np.all(np.abs(zb) < 3.0), zb
    v = verts.astype(np.float64)[faces]
    area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
    assert (x * area).sum() == pytest.approx((g * area).sum(), rel=0.03)


@pytest.mark.parametrize("key", ["hole", "trench"])
def test_oracle_redep_matches_reference(rp, key):
    verts, faces = rp[f"{key}_verts"], rp[f"{key}_faces"]
    m = orc.mesh_from_arrays(verts, faces)
    fn = rp[f"{key}_gas_normals"]
    n = int(rp[f"{key}_n"][0])
    runs = np.stack([orc.redep(m, fn, rp[f"{key}_V"], n, 0.5, 1000 + s) for s in range(32)])
    check_redep(runs, rp[f"{key}_mean"], rp[f"{key}_se"], verts, faces)


def test_oracle_redep_without_source_is_zero(rp):
    m = orc.mesh_from_arrays(rp["hole_verts"], rp["hole_faces"])
    out = orc.redep(m, rp["hole_gas_normals"], np.zeros(m.F), 1000, 0.5, 1)
    assert np.all(out == 0.0)
