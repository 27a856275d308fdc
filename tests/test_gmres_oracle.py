"""The oracle's GMRES radiosity solve against tests/golden/gmres.npz, made by the reference's own
mc_flux_3d_radiosity with radiosity_solver='gmres' (scipy gmres, threed.py:964-985).  CPU only:
from the recorded form-factor hits and ion results, the coverage <-> radiosity fixed point matches
exactly, including the high-albedo case where 40 Jacobi sweeps have not converged."""
import os
import types

import numpy as np
import pytest

from conftest import GOLDEN
import oracle.oracle as orc
import petch_b200.params as P

CASES = [(k, t) for k in ("hole", "trench") for t in ("a", "b")]


@pytest.fixture(scope="module")
def gd():
    return np.load(os.path.join(GOLDEN, "gmres.npz"))


def replay(gd, key, tag, solver):
    F = len(gd[f"{key}_faces"])
    D, Aff = orc.ff_matrix(gd[f"{key}_{tag}_hit"], F, 64)
    par = dict(P.PAR, periodic_y=0 if key == "hole" else 1, radiosity_solver=solver,
               betaE=float(gd[f"{key}_{tag}_betaE"][0]))
    fl = types.SimpleNamespace(chemistry="belen", yield_angular="viennaps", ion_reflection=True)
    return orc.radiosity_fixed_point(D, Aff, gd[f"{key}_{tag}_m_i"], gd[f"{key}_{tag}_cos_i"],
                                     tuple(gd[f"{key}_{tag}_ion_yield"]), par, fl)


@pytest.mark.parametrize("key,tag", CASES)
def test_gmres_fixed_point_replays_reference(gd, key, tag):
    m_F, m_O = replay(gd, key, tag, "gmres")
    np.testing.assert_array_equal(m_F, gd[f"{key}_{tag}_m_F"])
    np.testing.assert_array_equal(m_O, gd[f"{key}_{tag}_m_O"])


def test_high_albedo_separates_the_solvers(gd):
    """With betaE 0.05 the 40 Jacobi sweeps stop short of the solution that GMRES reaches."""
    g, _ = replay(gd, "hole", "b", "gmres")
    j, _ = replay(gd, "hole", "b", "jacobi")
    assert np.abs(g - j).max() > 1e-3
