"""The oracle's electron-shadowing charge model against tests/golden/electron.npz, produced by the
reference's own mc_flux_3d_coupled (threed.py:847-868) with surface_charging and charge_alpha > 0.
CPU only.

Pins: the electron trace (Gaussian-angle source with e_ang_sigma, unit sticking, the lateral wrap
for the trench) statistically against the reference kernel's 8-seed means; from the reference's
recorded trace tallies, the ion and electron normalisation, the open-field levels, the charging
factor and the coverage fixed point that follows it, to rounding."""
import os
import types

import numpy as np
import pytest

from conftest import GOLDEN
import oracle.oracle as orc
import petch_b200.params as P
from petch_b200 import charging as pch

KEYS = ["hole", "trench"]
N = 3000           # n_ion = n_neu of the recorded runs
ALPHA = 0.6


@pytest.fixture(scope="module")
def ed():
    return np.load(os.path.join(GOLDEN, "electron.npz"))


def case(ed, key):
    verts, faces = ed[f"{key}_verts"], ed[f"{key}_faces"]
    Lx, Ly, Lz, dx, periodic = ed[f"{key}_geo"]
    geo = dict(Lx=Lx, Ly=Ly, Lz=Lz, dx=dx)
    par = dict(P.PAR, periodic_y=int(periodic), charge_alpha=ALPHA, eFlux=1.3)
    m = orc.mesh_from_arrays(verts, faces)
    return m, verts, faces, ed[f"{key}_areas"], geo, par


def _edge_pairs(faces):
    """The face pairs that share an edge, for edges with exactly two faces (_edge_adjacency)."""
    edges = {}
    for f, tri in enumerate(faces.tolist()):
        for e in range(3):
            edges.setdefault(tuple(sorted((tri[e], tri[(e + 1) % 3]))), []).append(f)
    return np.array(sorted(tuple(v) for v in edges.values() if len(v) == 2), np.int64)


def _smoother(verts, faces):
    """The reference's host smoothing (threed.py:773-776): float32 face normals from the float32
    vertices, one pass at full strength over the edge pairs."""
    vv = verts[faces]
    fn = np.cross(vv[:, 1] - vv[:, 0], vv[:, 2] - vv[:, 0])
    fn = fn / (np.linalg.norm(fn, axis=1, keepdims=True) + 1e-12)
    pairs = _edge_pairs(faces)
    assert len(pairs) > len(faces)
    return lambda x: orc.smooth(x, fn, pairs, 1, 1.0)


def _z2(x, g, sg):
    k = sg > 0
    z2 = (x[k] - g[k]) ** 2 / sg[k] ** 2
    return float(np.median(z2)), float(z2.mean())


@pytest.mark.parametrize("key", KEYS)
def test_electron_trace_matches_reference_kernel(ed, key):
    """z = (x - g) / sg follows Student-t with 7 degrees of freedom without a systematic
    difference: E[z^2] = 1.4, median(z^2) = 0.49."""
    m, verts, faces, A, geo, par = case(ed, key)
    n = 1_000_000
    x = orc.trace_electrons(m, geo, par, 0.5, 5, n) / n
    g, sg = ed[f"{key}_electron_mean"], ed[f"{key}_electron_se"]
    med, mean = _z2(x, g, sg)
    assert med < 0.75 and mean < 2.2, (med, mean)
    assert x.sum() == pytest.approx(g.sum(), rel=0.02)
    assert x.sum() <= 1.0 + 1e-12                  # first-hit deposits: one unit per electron


@pytest.mark.parametrize("key", KEYS)
@pytest.mark.parametrize("tag", ["faithful", "legacy"])
def test_charging_replays_reference(ed, key, tag):
    """Recorded ion, electron and neutral tallies -> the reference's charged m_i and its
    coverage fixed point (4 cold rounds), to rounding."""
    m, verts, faces, areas, geo, par = case(ed, key)
    A = np.maximum(areas, 1e-9)
    A_src = geo['Lx'] * geo['Ly']
    sm = _smoother(verts, faces)
    raw = ed[f"{key}_{tag}_ion_raw"]
    if tag == "faithful":
        norm = A_src / N
        iy = tuple(sm((raw[q] / A) * norm) for q in range(3))
        fi, ai = raw[3], raw[4]
        m_i = sm((fi / A) * norm)
        cos_i = np.where(fi > 0, ai / np.maximum(fi, 1e-9), 0.0)
        np.testing.assert_allclose(np.stack(iy), ed[f"{key}_{tag}_ion_yield"], rtol=1e-12,
                                   atol=1e-14)
    else:
        iy = None
        fi, ai = raw
        m_i = sm(np.clip((fi / A) / (N / A_src), 0.0, 1.5))
        cos_i = np.where(fi > 0, ai / np.maximum(fi, 1e-9), 0.0)
    np.testing.assert_allclose(cos_i, ed[f"{key}_{tag}_cos_i"], rtol=1e-12, atol=1e-14)
    m_e = orc.electron_flux(ed[f"{key}_{tag}_electron_raw"], A, A_src, N, par, sm)
    m_i2, ref_i, ref_e = orc.electron_shadow(m_i, m_e, ALPHA)
    np.testing.assert_allclose(m_i2, ed[f"{key}_{tag}_m_i"], rtol=1e-12, atol=1e-14)
    # the charging acts: some faces lose more than 10 % of their ions, none gains
    assert np.all(m_i2 <= m_i + 1e-15) and np.any(m_i2 < 0.9 * m_i)
    assert ref_i > 0 and ref_e > 0
    assert pch.open_field_level(m_i) == ref_i and pch.open_field_level(m_e) == ref_e
    # the coverage fixed point from the recorded neutral tallies
    betas = ed[f"{key}_{tag}_neutral_beta"]
    seeds = ed[f"{key}_{tag}_neutral_seed"]
    nraw = ed[f"{key}_{tag}_neutral_raw"]
    assert len(nraw) == 8 and list(seeds) == [100 * 9 + 2 + k for k in range(8)]
    flags = types.SimpleNamespace(chemistry="belen", yield_angular="viennaps")
    bare = np.ones(len(faces))
    for it in range(4):
        assert betas[2 * it] == pytest.approx(par['betaE']) and betas[2 * it + 1] == par['betaO']
        m_F = sm(np.clip((nraw[2 * it] / A) / (N / A_src), 0.0, 8.0))
        m_O = sm(np.clip((nraw[2 * it + 1] / A) / (N / A_src), 0.0, 8.0))
        thF, thO = orc.belen_coverages(m_i2, m_F, m_O, cos_i, par, flags.yield_angular, iy)
        bare = np.clip(1.0 - thF - thO, 0.0, 1.0)
    np.testing.assert_allclose(m_F, ed[f"{key}_{tag}_m_F"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(m_O, ed[f"{key}_{tag}_m_O"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(bare, ed[f"{key}_{tag}_bare"], rtol=1e-12, atol=1e-14)


def test_open_field_level_edges():
    """No face above 1e-6 -> 1.0; numpy's linear percentile otherwise."""
    assert pch.open_field_level(np.zeros(5)) == 1.0
    assert orc.open_field_level(np.full(3, 1e-7)) == 1.0
    x = np.array([0.0, 2.0, 1.0, 3.0, 5.0])
    assert pch.open_field_level(x) == pytest.approx(np.percentile([1.0, 2.0, 3.0, 5.0], 90))


def test_electron_shadow_factor_limits():
    """alpha = 0 leaves m_i alone; electrons as exposed as the ions -> factor 1; no electrons on
    an exposed face -> 1 - alpha; faces without ions (sh_i floored at 1e-3) lose at most alpha."""
    rng = np.random.default_rng(4)
    m_i = rng.uniform(0.0, 1.0, 200)
    m_e = rng.uniform(0.0, 1.0, 200)
    out, _, _ = orc.electron_shadow(m_i, m_e, 0.0)
    np.testing.assert_array_equal(out, m_i)
    out, _, _ = orc.electron_shadow(m_i, m_i, 0.7)
    np.testing.assert_allclose(out, m_i, rtol=1e-15)
    me = m_e.copy()
    me[0] = 0.0
    mi = m_i.copy()
    mi[0] = np.percentile(mi[mi > 1e-6], 90) * 2.0
    out, _, _ = orc.electron_shadow(mi, me, 0.7)
    assert out[0] == pytest.approx(mi[0] * 0.3)
    assert np.all(out >= 0.3 * mi - 1e-15)
