"""The y-slab decomposition's host side on CPU: slab geometry, the split and
merge of padded blocks, the halo exchange between gloo ranks (world sizes 2
and 3), the merge of per-rank diagnostics (gks_stats_reduce, a host function
of the library) and the oracle's multi-rank statistics.  No GPU is used."""

import os
import socket

import numpy as np
import pytest

import gks_slabs


def test_slab_geometry_and_block_round_trip():
    assert gks_slabs.slab_planes(32, 4, 3) == (8, 24)
    for nc, p in [(32, 3), (8, 4), (16, 0)]:
        with pytest.raises(ValueError):
            gks_slabs.slab_planes(nc, p, 0)
    nc, nt = 12, 18
    rng = np.random.default_rng(0)
    inner = rng.random((5, nc, nc, nc))
    W = np.pad(inner, ((0, 0), (3, 3), (3, 3), (3, 3)), mode="wrap")
    for p in (1, 2, 4):
        blocks = [gks_slabs.split_block(W, p, r) for r in range(p)]
        for r, b in enumerate(blocks):
            ny, y0 = gks_slabs.slab_planes(nc, p, r)
            assert b.shape == (5, ny + 6, nt, nt)
            # the ghost planes are the neighbours' planes, periodically
            for a in range(ny + 6):
                np.testing.assert_array_equal(b[:, a, 3:-3, 3:-3], inner[:, (y0 + a - 3) % nc])
        np.testing.assert_array_equal(gks_slabs.merge_blocks(blocks), W)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        n = 6
        bufs = [torch.full((n,), 100.0 * rank + 1), torch.full((n,), 100.0 * rank + 2),
                torch.zeros(n), torch.zeros(n)]
        gks_slabs.exchange_halo(bufs, rank, ws)
        q.put((rank, float(bufs[2][0]), float(bufs[3][0]), bool((bufs[2] == bufs[2][0]).all()),
               bool((bufs[3] == bufs[3][0]).all())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2, 3])
def test_halo_exchange_between_gloo_ranks(ws):
    pytest.importorskip("torch")
    import torch.multiprocessing as mp

    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_exchange_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(ws))
    for rank, south_ghost, north_ghost, u1, u2 in got:
        south, north = (rank - 1) % ws, (rank + 1) % ws
        assert south_ghost == 100.0 * south + 2  # the south neighbour's north planes
        assert north_ghost == 100.0 * north + 1  # the north neighbour's south planes
        assert u1 and u2


def _reduce_rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        dt = gks_slabs.min_over_ranks(1e-3 * (1 + 0.5 * ((rank + 1) % ws)), "cpu")
        part = np.full(28, float(rank))
        parts = gks_slabs.gather_parts(part, "cpu")
        q.put((rank, dt, parts.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2, 3])
def test_dt_and_statistics_parts_over_gloo_ranks(ws):
    """The slabs' dt is the minimum over ranks and every rank sees all ranks'
    statistics parts in rank order (SlabField.timestep / SlabField.stats)."""
    pytest.importorskip("torch")
    import torch.multiprocessing as mp

    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_reduce_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(ws))
    for rank, dt, parts in got:
        assert dt == 1e-3
        assert [row[0] for row in parts] == [float(r) for r in range(ws)]


def test_single_rank_exchange_is_a_local_copy():
    torch = pytest.importorskip("torch")
    bufs = [torch.full((4,), 1.0), torch.full((4,), 2.0), torch.zeros(4), torch.zeros(4)]
    gks_slabs.exchange_halo(bufs, 0, 1)
    assert bufs[2].tolist() == [2.0] * 4 and bufs[3].tolist() == [1.0] * 4


def _part(x, v2):
    """A gks_stats_part record of samples x (columns = the 18 summed quantities)
    and (p, T, 1/rho) samples v2, shifted by their first values."""
    rec = np.zeros(28)
    rec[:18] = x.mean(0)
    K = v2[0]
    for i in range(3):
        d = v2[:, i] - K[i]
        rec[18 + 2 * i] = d.mean()
        rec[19 + 2 * i] = (d * d).mean()
    rec[24:27] = K
    rec[27] = len(x)
    return rec


def test_stats_reduce_merges_parts_like_the_whole(gks):
    rng = np.random.default_rng(1)
    n = 4096
    x = rng.random((n, 18)) + 0.5
    v2 = np.stack([1 + 0.1 * rng.random(n), 0.003 + 1e-4 * rng.random(n), 1 + 0.05 * rng.random(n)], 1)
    phys = gks.Phys(nc=16, K=2, visc_law=0, reserved=0, gam=1.4, gas_r=287.0, T0=1 / (1.4 * 287.0), mu0=1e-3,
                    visc_exp=0.76, pr_factor=1 / 0.7, p0=1 / 1.4, den0=1.0, Mt=0.3, t0=1.0)
    whole = gks.stats_reduce(_part(x, v2)[None], phys)
    cuts = [0, 1000, 1024, 3000, n]  # uneven parts
    parts = np.stack([_part(x[a:b], v2[a:b]) for a, b in zip(cuts[:-1], cuts[1:])])
    merged = gks.stats_reduce(parts, phys)
    for k in gks.STATS_FIELDS:
        assert merged[k] == pytest.approx(whole[k], rel=1e-12), k
    # the reference's normalisation of the rms values (update.cpp:759-770)
    prms = np.sqrt(((v2[:, 0] - v2[:, 0].mean()) ** 2).mean()) / (phys.gam * phys.p0 * phys.Mt ** 2)
    assert merged["prms"] == pytest.approx(prms, rel=1e-10)
    assert merged["tke"] == pytest.approx(x[:, 0].mean(), rel=1e-13)
    with pytest.raises(gks.GksError):
        bad = parts.copy()
        bad[1, 27] = 0
        gks.stats_reduce(bad, phys)


def test_oracle_multi_rank_statistics(oracle):
    import gks_ic

    case = gks_ic.make_dhit(16, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=2)
    W = gks_ic.to_conservative_padded(case)
    prm = oracle.params(16, case.gam, case.mu0, case.p0, case.rho0, case.Mt, case.t0)
    one = oracle.stats(W, prm)
    np.testing.assert_array_equal(oracle.stats_ranks(W, prm, 1), one)
    # segments' own splines change the y-derivatives near the segment ends only
    for p in (2, 4):
        st = oracle.stats_ranks(W, prm, p)
        assert not np.array_equal(st, one)
        np.testing.assert_allclose(st, one, rtol=0.05, atol=1e-9)
        # quantities without derivatives do not depend on the split
        np.testing.assert_allclose(st[[0, 8, 9, 10, 12, 13]], one[[0, 8, 9, 10, 12, 13]], rtol=1e-13, atol=1e-10)
