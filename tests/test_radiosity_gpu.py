"""Radiosity neutral transport on the device (petch_gas_normals, petch_trace_ff,
petch_ff_matrix, petch_radiosity_solve) against tests/golden/radiosity.npz (the reference's own
mc_flux_3d_radiosity, threed.py:923-991) and the oracle.

The fixture meshes are the oracle marching cubes of small etched pits; the device marching
cubes of the same level set gives the same faces in the same order, so per-face results line up.
"""
import ctypes
import os
import types

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from gpu_helpers import cuda_mesh, small_feature, stream
from test_radiosity_oracle import case, check_estimate
import oracle.oracle as orc
import petch_b200 as petch
from petch_b200 import _lib
from petch_b200 import threed as t3

pytestmark = pytest.mark.gpu

KEYS = ["hole", "trench", "hole_legacy"]


@pytest.fixture(scope="module")
def rd():
    return np.load(os.path.join(GOLDEN, "radiosity.npz"))


def device_case(rd, key):
    verts, faces, phi, geo, par, flags = case(rd, key)
    hole = key != "trench"
    phi2, g = small_feature(hole, nx=10, ny=10, nz=14, dx=0.3)
    np.testing.assert_array_equal(phi2, phi)
    m = cuda_mesh(phi, g['dx'], g)
    assert m.F == len(faces)
    np.testing.assert_array_equal(m.faces[:m.F].cpu().numpy(), faces)
    g = dict(g, Lx=geo['Lx'], Ly=geo['Ly'], Lz=geo['Lz'])
    return m, g, phi, par, flags


def engine(m, geo, par, flags):
    fe = t3.FluxEngine(geo, par, petch.Flags(chemistry=flags.chemistry,
                                               yield_angular=flags.yield_angular,
                                               ion_reflection=flags.ion_reflection), m.MT)
    fe.mesh = m
    return fe


@pytest.mark.parametrize("key", KEYS)
def test_gas_normals_match_reference(rd, key):
    m, geo, phi, par, flags = device_case(rd, key)
    fn = torch.empty((m.MT, 3), device="cuda")
    nx, ny, nz = phi.shape
    phid = torch.from_numpy(phi).cuda()
    _lib.call("petch_gas_normals", m.id, m.MT, m.MV, phid.data_ptr(), nx, ny, nz,
              float(geo['dx']), fn.data_ptr(), stream())
    np.testing.assert_allclose(fn[:m.F].double().cpu().numpy(), rd[f"{key}_gas_normals"],
                               rtol=0, atol=2e-7)


@pytest.mark.parametrize("key", KEYS)
def test_ff_matrix_matches_oracle(rd, key):
    """Same hits -> the same sky view (exact) and the same matrix (exact: multiples of 1/64),
    each row's entries in ascending source-face order."""
    m, geo, phi, par, flags = device_case(rd, key)
    F, n_ff = m.F, 64
    fe = engine(m, geo, par, flags)
    r = fe._radiosity_buffers(n_ff)
    hit = torch.full((m.MT * n_ff,), -1, dtype=torch.int32, device="cuda")
    hit[:F * n_ff] = torch.from_numpy(rd[f"{key}_hit"]).cuda()
    _lib.call("petch_ff_matrix", m.id, m.MT, m.MV, hit.data_ptr(), n_ff, r['row_ptr'].data_ptr(),
              r['col'].data_ptr(), r['sky'].data_ptr(), r['scratch'].data_ptr(),
              r['scratch'].numel(), stream())
    D, Aff = orc.ff_matrix(rd[f"{key}_hit"], F, n_ff)
    np.testing.assert_array_equal(r['sky'][:F].cpu().numpy(), D)
    rp = r['row_ptr'][:F + 1].cpu().numpy()
    col = r['col'][:rp[-1]].cpu().numpy()
    assert rp[0] == 0 and np.all(np.diff(rp) >= 0)
    dense = np.zeros((F, F))
    rows = np.repeat(np.arange(F), np.diff(rp))
    np.add.at(dense, (rows, col), 1.0 / n_ff)
    np.testing.assert_array_equal(dense, Aff.toarray())
    for i in range(F):
        assert np.all(np.diff(col[rp[i]:rp[i + 1]]) >= 0)


def _load_ions(fe, rd, key, F):
    fe.m_i[:F] = torch.from_numpy(rd[f"{key}_m_i"].astype(np.float32)).cuda()
    fe.cos_i[:F] = torch.from_numpy(rd[f"{key}_cos_i"].astype(np.float32)).cuda()
    if key == "hole_legacy":
        return (None, None, None)
    iy = rd[f"{key}_ion_yield"]
    for q in range(3):
        fe.y[q, :F] = torch.from_numpy(iy[q].astype(np.float32)).cuda()
    return tuple(fe.y[q].data_ptr() for q in range(3))


@pytest.mark.parametrize("key", KEYS)
def test_fixed_point_replays_reference_hits(rd, key):
    """The reference's recorded form-factor hits and ion results -> its m_F, m_O within 1e-5
    (float32 inputs and outputs around float64 solves)."""
    m, geo, phi, par, flags = device_case(rd, key)
    F, n_ff = m.F, 64
    fe = engine(m, geo, par, flags)
    yields = _load_ions(fe, rd, key, F)
    hit = torch.full((m.MT * n_ff,), -1, dtype=torch.int32, device="cuda")
    hit[:F * n_ff] = torch.from_numpy(rd[f"{key}_hit"]).cuda()
    fe.radiosity_from_hits(hit, n_ff, yields)
    for name, t in (("m_F", fe.m_F), ("m_O", fe.m_O)):
        np.testing.assert_allclose(t[:F].double().cpu().numpy(), rd[f"{key}_{name}"], rtol=1e-5,
                                   atol=1e-6, err_msg=name)


def test_fixed_point_is_bitwise_reproducible(rd):
    m, geo, phi, par, flags = device_case(rd, "trench")
    F, n_ff = m.F, 64
    fe = engine(m, geo, par, flags)
    yields = _load_ions(fe, rd, "trench", F)
    hit = torch.full((m.MT * n_ff,), -1, dtype=torch.int32, device="cuda")
    hit[:F * n_ff] = torch.from_numpy(rd["trench_hit"]).cuda()
    outs = []
    for _ in range(2):
        fe.radiosity_from_hits(hit, n_ff, yields)
        outs.append((fe.m_F[:F].clone(), fe.m_O[:F].clone(), fe.bare[:F].clone()))
    for a, b in zip(*outs):
        assert torch.equal(a, b)


def test_trace_ff_replays_and_wraps(rd):
    """Same seed -> the same hits; a periodic trench wraps rays that a closed hole loses."""
    m, geo, phi, par, flags = device_case(rd, "trench")
    fe = engine(m, geo, par, flags)
    phid = torch.from_numpy(phi).cuda()
    hits = []
    for periodic in (1, 1, 0):
        fe.dom.periodic = periodic
        r = fe._radiosity_buffers(64)
        nx, ny, nz = phi.shape
        _lib.call("petch_gas_normals", m.id, m.MT, m.MV, phid.data_ptr(), nx, ny, nz,
                  float(geo['dx']), r['fn'].data_ptr(), stream())
        _lib.call("petch_trace_ff", m.id, m.MT, m.MV, ctypes.byref(fe.dom), r['fn'].data_ptr(), 7,
                  64, r['hit'].data_ptr(), fe.small.data_ptr(), stream())
        assert fe.small[1].item() == 0
        hits.append(r['hit'][:m.F * 64].cpu().numpy().copy())
        assert np.all(r['hit'][m.F * 64:].cpu().numpy() == -1)
    np.testing.assert_array_equal(hits[0], hits[1])
    assert np.mean(hits[0] < 0) < np.mean(hits[2] < 0)


def test_solve_without_iterations_is_the_sky_view(rd):
    m, geo, phi, par, flags = device_case(rd, "hole")
    F, n_ff = m.F, 64
    fe = engine(m, geo, par, flags)
    hit = torch.full((m.MT * n_ff,), -1, dtype=torch.int32, device="cuda")
    hit[:F * n_ff] = torch.from_numpy(rd["hole_hit"]).cuda()
    r = fe._radiosity_buffers(n_ff)
    _lib.call("petch_ff_matrix", m.id, m.MT, m.MV, hit.data_ptr(), n_ff, r['row_ptr'].data_ptr(),
              r['col'].data_ptr(), r['sky'].data_ptr(), r['scratch'].data_ptr(),
              r['scratch'].numel(), stream())
    fe.bare.fill_(0.3)
    D, Aff = orc.ff_matrix(rd["hole_hit"], F, n_ff)
    for n_iter in (0, 1, 7):
        _lib.call("petch_radiosity_solve", m.id, m.MT, m.MV, r['row_ptr'].data_ptr(),
                  r['col'].data_ptr(), r['sky'].data_ptr(), n_ff, fe.bare.data_ptr(), 0.7, 1.0,
                  n_iter, fe.m_F.data_ptr(), fe.m_O.data_ptr(), r['work2'].data_ptr(), stream())
        bare = np.full(F, np.float32(0.3), np.float64)
        for beta, t in ((0.7, fe.m_F), (1.0, fe.m_O)):
            ref = orc.radiosity_solve(Aff, D, bare, beta, n_iter)
            np.testing.assert_allclose(t[:F].double().cpu().numpy(), ref, rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("key", ["hole", "trench"])
def test_device_radiosity_estimator_matches_reference(rd, key):
    """The whole device path through the drop-in mc_flux_3d_radiosity over 24 seeds against the
    reference's 8-seed means (criteria in test_radiosity_oracle.check_estimate)."""
    m, geo, phi, par, flags = device_case(rd, key)
    verts, faces = rd[f"{key}_verts"], rd[f"{key}_faces"]
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", ion_reflection=True,
                     neutral_transport="radiosity")
    g = dict(geo, phi=phi)
    runs = []
    for sd in range(24):
        p = dict(par)
        m_i, m_F, m_O, cos_i = petch.mc_flux_3d_radiosity(m, None, None, None, None, g, p,
                                                          n_ion=3000, seed=300 + sd, flags=fl)
        assert '_ion_yield' in p
        runs.append(np.stack([m_i, m_F, m_O]))
    check_estimate(np.stack(runs), rd[f"{key}_mean"], rd[f"{key}_se"], verts, faces)


@pytest.mark.parametrize("hole", [True, False])
def test_radiosity_loop_depth_matches_oracle_loop(hole):
    """run_etch_3d with neutral_transport='radiosity' on the device and in the oracle loop
    (independent random streams): centre depth within one grid cell at every recorded step."""
    dx = 0.25
    cfg = dict(Lx=5.0, Ly=5.0 if hole else 2.5, Lz=8.0, dx=dx, trench_width=2.0, mask_th=1.0,
               sub_top=6.0, t_end=1.2, n_steps=12, hole=hole)
    par = dict(petch.PAR, rate_scale=0.3, periodic_y=0 if hole else 1)
    fl = petch.Flags(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                     ion_reflection=True, neutral_transport="radiosity")
    n = 60000
    geo = t3.run_etch_3d(**cfg, par=par, flags=fl, n_ion=n, n_neu=n, reinit_method="fsm",
                         verbose=False, record_depth_every=3)
    dev_hist = dict(geo['depth_history'])
    _, hist, _ = orc.run_etch_3d(cfg['Lx'], cfg['Ly'], cfg['Lz'], dx, cfg['trench_width'],
                                 cfg['mask_th'], cfg['sub_top'], cfg['t_end'], cfg['n_steps'],
                                 hole, par, fl, n, n, record_depth_every=3)
    orc_hist = dict(hist)
    assert set(dev_hist) == set(orc_hist)
    for s in sorted(orc_hist):
        assert abs(dev_hist[s] - orc_hist[s]) <= dx + 1e-9, (s, dev_hist[s], orc_hist[s])
    assert max(orc_hist.values()) > 2 * dx


def test_radiosity_solve_tangent_matches_finite_differences(rd):
    """petch_radiosity_solve_tangent: its primal equals petch_radiosity_solve bit for bit, and its
    tangents along three random coverage directions match central differences of the 40-sweep
    solve per face (the solve is deterministic given the form-factor hits)."""
    m, geo, phi, par, flags = device_case(rd, "hole")
    F, n_ff, n_iter, MT = m.F, 64, 40, m.MT
    fe = engine(m, geo, par, flags)
    hit = torch.full((MT * n_ff,), -1, dtype=torch.int32, device="cuda")
    hit[:F * n_ff] = torch.from_numpy(rd["hole_hit"]).cuda()
    r = fe._radiosity_buffers(n_ff)
    _lib.call("petch_ff_matrix", m.id, m.MT, m.MV, hit.data_ptr(), n_ff, r['row_ptr'].data_ptr(),
              r['col'].data_ptr(), r['sky'].data_ptr(), r['scratch'].data_ptr(),
              r['scratch'].numel(), stream())
    rng = np.random.default_rng(3)
    bare = torch.zeros(MT, device="cuda")
    bare[:F] = torch.from_numpy(rng.uniform(0.2, 0.9, F).astype(np.float32)).cuda()
    dbare = torch.zeros((3, MT), device="cuda")
    dbare[:, :F] = torch.from_numpy(rng.normal(0.0, 1.0, (3, F)).astype(np.float32)).cuda()
    f32 = dict(device="cuda", dtype=torch.float32)
    gE, gO = torch.zeros(MT, **f32), torch.zeros(MT, **f32)
    dgE, dgO = torch.zeros((3, MT), **f32), torch.zeros((3, MT), **f32)
    work = torch.empty(16 * MT, device="cuda", dtype=torch.float64)

    def solve(b):
        _lib.call("petch_radiosity_solve", m.id, m.MT, m.MV, r['row_ptr'].data_ptr(),
                  r['col'].data_ptr(), r['sky'].data_ptr(), n_ff, b.data_ptr(), 0.7, 1.0, n_iter,
                  fe.m_F.data_ptr(), fe.m_O.data_ptr(), r['work2'].data_ptr(), stream())
        return fe.m_F[:F].double().cpu().numpy(), fe.m_O[:F].double().cpu().numpy()

    _lib.call("petch_radiosity_solve_tangent", m.id, m.MT, m.MV, r['row_ptr'].data_ptr(),
              r['col'].data_ptr(), r['sky'].data_ptr(), n_ff, bare.data_ptr(), dbare.data_ptr(),
              0.7, 1.0, n_iter, gE.data_ptr(), gO.data_ptr(), dgE.data_ptr(), dgO.data_ptr(),
              work.data_ptr(), stream())
    pE, pO = solve(bare)
    np.testing.assert_array_equal(gE[:F].double().cpu().numpy(), pE)
    np.testing.assert_array_equal(gO[:F].double().cpu().numpy(), pO)
    h = 1e-2
    for k in range(3):
        ep, op = solve(bare + h * dbare[k])
        em, om = solve(bare - h * dbare[k])
        for fd, t in (((ep - em) / (2 * h), dgE[k, :F]), ((op - om) / (2 * h), dgO[k, :F])):
            t = t.double().cpu().numpy()
            scale = np.abs(fd).max()
            assert np.abs(t - fd).max() <= 2e-3 * scale, (k, np.abs(t - fd).max(), scale)
