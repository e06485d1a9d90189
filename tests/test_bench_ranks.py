"""The multi-rank path of bench.py on CPU: world size 2 over gloo.

bench.py runs replicas only (one field per GPU, no data exchange); its ranks
meet only at the timing barriers and the max over ranks of each timing.  These
tests run those steps with two gloo ranks on 127.0.0.1, and check that the
reference arm's non-zero ranks leave without work.  No GPU is used."""

import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, ws: int, port: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    import bench

    d = bench.Dist(ws, rank, backend="gloo")
    d.barrier()
    # each rank's timing differs; every rank must see the slowest one
    slowest = d.max(10.0 + rank)
    rate = bench.whole_job_rate(ws, 256 ** 3, slowest)
    d.close()
    q.put((rank, slowest, rate))


def test_two_gloo_ranks_agree_on_the_slowest_time():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp

    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(ws))
    assert [g[1] for g in got] == [11.0, 11.0]
    assert got[0][2] == got[1][2] == pytest.approx(2 * 256 ** 3 / 11.0e-3)


def test_single_rank_needs_no_process_group():
    import bench

    d = bench.Dist(1, 0, backend="gloo")
    assert d.max(3.5) == 3.5
    d.barrier()
    d.close()
    assert bench.whole_job_rate(1, 1000, 2.0) == pytest.approx(5e5)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_reference_arm_times_the_whole_field():
    """bench.py --impl reference: one reference process per y-slab, the slabs
    together the whole field, ms_per_step the slowest process's measured time."""
    import json

    sys.path.insert(0, ROOT)
    import bench

    assert bench.reference_slabs(256, 16) == 16
    assert bench.reference_slabs(256, 6) == 4
    assert bench.reference_slabs(256, 200) == 64
    assert bench.reference_slabs(24, 16) == 8
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--nc", "16",
                        "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    if "unavailable" in line:
        pytest.skip(line["unavailable"])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["config"] == bench.bench_config(16, bench.MACH, bench.RE, 1)
    per = line["per_process_ms_per_step"]
    assert len(per) == line["cpu_baseline"]["cores"]
    assert abs(line["ms_per_step"] - max(per)) < 1e-9
    assert abs(line["value"] - 16 ** 3 / (line["ms_per_step"] * 1e-3)) < 1e-6 * line["value"]
