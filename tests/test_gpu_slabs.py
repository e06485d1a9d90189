"""GPU tests of the y-slab decomposition (gks_create_slab + halo exchange).

A field split over P ranks along y must advance exactly as the whole field:
every slab runs the same kernels on the same cells, the ghost planes holding
the neighbours' planes of the same step, so the merged state after several
steps equals the periodic single-field run bit for bit, and dt (the minimum
over slabs) equals the whole field's.  The P slabs run here in one process on
one GPU (LocalSlabs: the exchange is a device copy); a one-rank NCCL process
group runs the SlabField path itself.  The diagnostics of a split field follow
the reference's multi-rank PrintStats (splines over each rank's padded
segment, sums reduced over ranks) and are checked against the oracle's
restatement of it to 1e-10.
"""

import os
import socket

import numpy as np
import pytest

import gks_ic
import gks_slabs

pytestmark = pytest.mark.gpu

STATS_RTOL = 1e-10


def dhit(nc, seed=3, Mt=0.4):
    case = gks_ic.make_dhit(nc, k0=4.0, Mt=Mt, Re_lambda=72.0, seed=seed)
    return case, gks_ic.to_conservative_padded(case)


def periodic_run(gks, case, W, prec, nsteps, flags=0):
    with gks.Solver(gks.phys_from_case(case), prec, flags) as s:
        s.upload(W)
        dt = s.timestep(0.5)
        s.step(nsteps)
        s.sync()
        return s.download(), dt, s.stats_array()


@pytest.mark.parametrize("nranks", [1, 2, 4])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_slabs_advance_exactly_as_the_whole_field(gks, nranks, prec):
    p = gks.FP64 if prec == "fp64" else gks.MIXED
    case, W = dhit(32)
    ref, dt_ref, _ = periodic_run(gks, case, W, p, 4)
    sl = gks_slabs.LocalSlabs(gks.phys_from_case(case), nranks, p)
    try:
        sl.upload(W)
        assert sl.timestep(0.5) == dt_ref
        sl.step(4)
        sl.sync()
        got = sl.download()
    finally:
        sl.close()
    np.testing.assert_array_equal(got, ref)


def test_slabs_with_zsweep_fix_and_odd_edge(gks):
    # nc = 36 over 3 ranks (12 planes each), the corrected z sweep
    case, W = dhit(36, seed=5)
    ref, dt_ref, _ = periodic_run(gks, case, W, gks.FP64, 3, gks.FIX_ZSWEEP)
    sl = gks_slabs.LocalSlabs(gks.phys_from_case(case), 3, gks.FP64, gks.FIX_ZSWEEP)
    try:
        sl.upload(W)
        assert sl.timestep(0.5) == dt_ref
        sl.step(3)
        got = sl.download()
    finally:
        sl.close()
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("nranks", [1, 2, 4])
def test_slab_stats_match_the_multi_rank_oracle(gks, oracle, nranks):
    case, W = dhit(32, seed=7, Mt=0.5)
    phys = gks.phys_from_case(case)
    sl = gks_slabs.LocalSlabs(phys, nranks, gks.FP64)
    try:
        sl.upload(W)
        sl.timestep(0.5)
        sl.step(2)
        st = sl.stats()
        Wn = sl.download()
    finally:
        sl.close()
    prm = oracle.params(32, case.gam, case.mu0, case.p0, case.rho0, case.Mt, case.t0)
    want = oracle.stats_ranks(Wn, prm, nranks)
    got = np.array([st[k] for k in gks.STATS_FIELDS])
    np.testing.assert_allclose(got, want, rtol=STATS_RTOL, atol=1e-14)
    if nranks == 1:
        # one rank: the whole field's diagnostics
        with gks.Solver(phys) as s:
            s.upload(Wn)
            np.testing.assert_allclose(s.stats_array(), got, rtol=1e-13, atol=1e-15)


def test_slab_host_evolve_takes_its_ghosts_from_the_host(gks):
    # the reference's per-rank evolve(W, dev, dt) on a slab block whose ghost
    # planes the caller's HaloTransfer filled: the interior planes advance as
    # the whole field's, the y ghosts come back as they went up
    case, W = dhit(24, seed=11)
    ref, dt, _ = periodic_run(gks, case, W, gks.FP64, 1)
    phys = gks.phys_from_case(case)
    for r in range(2):
        block = gks_slabs.split_block(W, 2, r)
        with gks.Solver(phys, gks.FP64, slab=gks_slabs.slab_planes(24, 2, r)) as s:
            s.set_dt(dt)
            out = s.evolve(block.copy())
        ny, y0 = gks_slabs.slab_planes(24, 2, r)
        np.testing.assert_array_equal(out[:, 3:3 + ny], ref[:, 3 + y0:3 + y0 + ny])
        np.testing.assert_array_equal(out[:, :3], block[:, :3])
        np.testing.assert_array_equal(out[:, -3:], block[:, -3:])


def test_slab_rejects_whole_field_launches_and_bad_geometry(gks):
    case, W = dhit(16)
    phys = gks.phys_from_case(case)
    for ny, y0 in [(2, 0), (17, 0), (8, 9), (8, -1)]:
        with pytest.raises(gks.GksError):
            gks.Solver(phys, gks.FP64, slab=(ny, y0))
    with gks.Solver(phys, gks.FP64, slab=(8, 8)) as s:
        s.upload(gks_slabs.split_block(W, 2, 1))
        s.timestep(0.5)
        with pytest.raises(gks.GksError):
            s.time_stages(1)
        with pytest.raises(gks.GksError):
            s.autotune(1)
        s.step(1)
        s.sync()
        # one step per call: more would read stale ghosts
        with pytest.raises(gks.GksError):
            s.step(2)
        with pytest.raises(gks.GksError):
            s.evolve(gks_slabs.split_block(W, 2, 1), nsteps=2)
    with gks.Solver(phys) as s:
        with pytest.raises(gks.GksError):
            s.halo_pack()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slab_field_over_a_one_rank_nccl_group(gks):
    import torch
    import torch.distributed as dist

    case, W = dhit(32, seed=13)
    ref, dt_ref, st_ref = periodic_run(gks, case, W, gks.FP64, 3)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        f = gks_slabs.SlabField(gks.phys_from_case(case), gks.FP64)
        f.upload(gks_slabs.split_block(W, 1, 0))
        assert f.timestep(0.5) == dt_ref
        f.step(3)
        f.sync()
        got = f.download()
        st = f.stats()
        f.close()
    finally:
        dist.destroy_process_group()
    np.testing.assert_array_equal(got[:, 3:-3], ref[:, 3:-3])
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(ref)
        want = s.stats()
    for k in gks.STATS_FIELDS:
        assert st[k] == pytest.approx(want[k], rel=1e-13, abs=1e-15)


@pytest.mark.parametrize("mode", [["--local-slabs", "2"], ["--slabs"]])
def test_bench_slab_modes_print_a_line(mode):
    import json
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ)
    env.pop("MASTER_PORT", None)
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), *mode, "--nc", "32", "--steps", "2",
                        "--warmup", "3", "--no-tune"], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    assert line["value"] > 0 and line["scaling"] == "strong"
    assert line["config"]["slabs"] == (2 if mode[0] == "--local-slabs" else 1)
