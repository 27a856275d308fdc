"""Host logic of the batched inverse design and of the multi-rank paths, on the CPU: the trench
batch draws, the depth profile of a trench, the loss gradient, Adam, and -- as two gloo ranks --
the instance sharding with its per-iteration all-gather and bench.py's max-over-ranks reduction."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from petch_b200 import adjoint, inverse


def test_trench_batch_draws():
    specs, th = inverse.trench_batch_specs(32, seed=0)
    assert len(specs) == 32 and th.shape == (32, 3)
    w = np.array([s['trench_width'] for s in specs])
    assert w.min() >= 1.0 and w.max() <= 4.0
    assert np.all((th[:, 0] >= 50.0) & (th[:, 0] <= 500.0))
    assert np.all((th[:, 1] >= 0.0) & (th[:, 1] <= 0.5)) and np.all(th[:, 2] == 1.0)
    for s in specs:
        assert not s['hole'] and s['par']['periodic_y'] == 1 and s['dx'] == 0.125
        assert s['sub_top'] >= 10.0 * s['trench_width']           # room for aspect ratio 10
        assert abs(s['Lz'] - s['sub_top'] - 2.0) < 1e-9
        rF = s['par']['Fflux'] / inverse.PAR['ionFlux']
        assert 10.0 <= rF <= 1000.0
    specs2, th2 = inverse.trench_batch_specs(32, seed=0)
    assert np.array_equal(th, th2)


def test_trench_profile_and_jacobian():
    """A flat floor at z0 (phi = z0 - z above it): every column's depth is sub_top - z0, and a
    unit level-set tangent moves it by -1."""
    nx, ny, nz, dx = 24, 4, 40, 0.125
    z = np.arange(nz) * dx
    z0 = 2.3
    phi = np.broadcast_to(z0 - z, (nx, ny, nz)).copy()
    dphi = np.zeros((3, nx, ny, nz))
    dphi[0] = 1.0
    geo = dict(dx=dx, Lx=nx * dx, Ly=ny * dx, sub_top=4.0, hole=False)
    prof, jac = adjoint.radial_profile(phi, geo, dphi, n_bins=8)
    assert np.allclose(prof[np.isfinite(prof)], 4.0 - z0)
    assert np.isfinite(prof).sum() >= 7
    ok = np.isfinite(jac[:, 0])
    assert np.allclose(jac[ok, 0], -1.0) and np.allclose(jac[ok, 1:], 0.0)


def test_loss_gradient_matches_differences():
    rng = np.random.default_rng(3)
    J = rng.normal(size=(16, 3))
    target = rng.normal(size=16)
    target[[2, 9]] = np.nan
    p0 = rng.normal(size=16)

    def prof(th):
        return p0 + J @ th

    th = np.array([0.3, -0.2, 0.1])
    L, g = inverse.loss_and_grad(prof(th), J, target)
    for k in range(3):
        e = np.zeros(3)
        e[k] = 1e-6
        num = (inverse.loss_and_grad(prof(th + e), J, target)[0]
               - inverse.loss_and_grad(prof(th - e), J, target)[0]) / 2e-6
        assert abs(num - g[k]) < 1e-6 * max(1.0, abs(g[k]))


def test_adam_matches_the_update_rule():
    th0 = np.array([[100.0, 0.1, 1.0]])
    opt = inverse.Adam(th0, lr=0.05)
    g = np.array([[2.0, -0.5, 0.0]])
    opt.step(g)
    # first step: m_hat = g s, v_hat = (g s)^2 -> u moves by -lr * sign(g) (g != 0)
    expect = th0 * (1.0 - 0.05 * np.sign(g) * (np.abs(g * th0) > 0))
    assert np.allclose(opt.theta, expect, rtol=1e-6)
    opt2 = inverse.Adam(np.array([[1.5, 0.0, 0.5]]), lr=10.0)
    opt2.step(np.array([[1.0, 1.0, 1.0]]))
    assert np.all(opt2.theta >= np.array([1.0, 0.0, 0.0]) - 1e-12)   # physical bounds


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        B = 7
        mine = inverse.shard(B, world, rank)
        rows = np.array([[b, 10.0 * b] for b in mine], np.float64)
        full = inverse.gather_rows(rows, B, world, rank)
        import bench
        mx = bench.rank_reduce([1.0 + rank, 5.0 - rank], "max", dist, world)
        sm = bench.rank_reduce([1.0 + rank], "sum", dist, world)
        out[rank] = (mine, full.tolist(), mx, sm)
    finally:
        dist.destroy_process_group()


def test_shard_gather_and_rank_reduce_on_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == [0, 2, 4, 6] and res[1][0] == [1, 3, 5]
    expect = [[b, 10.0 * b] for b in range(7)]
    for r in range(world):
        assert res[r][1] == expect
        assert res[r][2] == [2.0, 5.0]       # max over ranks
        assert res[r][3] == [3.0]            # sum over ranks
