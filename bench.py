#!/usr/bin/env python
"""Benchmark of the GKM-DNS WENO-GKS step on B200.

Workload: one decaying-isotropic-turbulence field at 256^3 (k0 4, Mt 0.5,
Re_lambda 100, CFL 0.5, seeded synthetic initial field; the configuration the
headline metric is quoted on).  A step is one pass of the hot path: the three
reconstruction + flux sweeps and the conservative update.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours       K timed steps of the FP64 path (the parity path, `value`) and of the
           mixed FP32/FP64 path (`mixed`), state resident in HBM (671 MB per
           field, above the 126 MB L2, so no flush between steps); CUDA events
           on the library's stream; max over ranks.  `e2e` times the
           reference-facing call (upload from pinned host memory, one step,
           download) per step.  `roofline` is the dominant kernel (the flux
           sweep) timed live with CUDA events against the FP64 FMA peak
           measured live on the same GPU.  Under torchrun every rank advances
           its own replica (replicas: the default line).
           The line also carries the mixed path's accuracy against the FP64
           path on the same field run to t/t0 = 2 (statistics every 10 steps).
--slabs    one field split over the torchrun ranks along y (gks_slabs, NCCL
           halo exchange after every step; strong scaling); --local-slabs P
           runs P slabs of one field in one process on one GPU.
reference  the reference's own CPU implementation (oracle/_ref, compiled from
           its sources) on the host cores: the 256^3 field cut into P y-slabs
           (P the largest power of two up to the core count, at most 64), one
           process per slab, so that every timed step advances the whole
           field; ms_per_step is the slowest process's measured time per step.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gkm-dns_b200"))

METRIC = "cell-updates/s at 256³, FP64 vs mixed FP32/FP64 (err vs FP64); HBM GB/s"
UNIT = "cell-updates/s"
NC = 256
K0, MACH, RE = 4.0, 0.5, 100.0
CFL = 0.5
# Algorithmic work (reference operation counts of flux() and ApplyWENO(), one
# WENO per line and interface): FP64 operations per interface in the flux
# kernel (flux 8005 + slopes 90 + c2p/viscosity/tau 25) and in the
# reconstruction kernel (5-component WENO 1122); per cell-update 3 interfaces
# + 30 for the update.
OPS_FLUX = 8005 + 90 + 25
OPS_RECON = 1122
OPS_CELL = 3 * (OPS_FLUX + OPS_RECON) + 30
BYTES_CELL = 80  # 5 doubles read + 5 written per cell-update
# FP64 FMA lanes per SM of B200 (sm_100): the nominal FP64 rate is
# SMs x 64 x 2 flops x SM clock
FP64_LANES_PER_SM = 64


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Dist:
    """Ranks of a replicas-only run: one process per GPU over NCCL (the
    bench), or over gloo on CPU (tests).  Every rank takes the same
    collective steps: barriers around the timed regions and a max over ranks
    of each timing."""

    def __init__(self, ws, local, backend: str = "nccl"):
        self.ws = ws
        self.pg = None
        self.device = "cpu" if backend == "gloo" else "cuda"
        if ws > 1:
            import datetime

            import torch
            import torch.distributed as dist

            if backend == "nccl":
                torch.cuda.set_device(local)
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                        device_id=torch.device("cuda", local))
            else:
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()


def whole_job_rate(ws: int, cells_per_rank: int, max_ms: float) -> float:
    """Cell-updates/s of the whole job: every rank advances its own replica of
    `cells_per_rank` cells per step; the step time is the slowest rank's."""
    return ws * cells_per_rank / (max_ms * 1e-3)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, pw, reasons = [], None, [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
                pw.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "power_w_max": max(pw) if pw else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def gpu_uuid(local: int) -> str:
    try:
        import torch

        u = torch.cuda.get_device_properties(local).uuid
        return "GPU-" + str(u)
    except Exception:
        return str(local)


def read_profile(name: str, key: str):
    """A per-interface figure (`key = value ...` line) of a committed ncu summary."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith(key):
                    return float(line.split("=")[1].split()[0])
    except (OSError, ValueError, IndexError):
        pass
    return None


def read_traffic(nc: int):
    """DRAM bytes per flux launch from the committed ncu summary, scaled to nc^3 cells."""
    b = read_profile("flux_fp64_ncu.txt", "dram_bytes_per_interface")
    return None if b is None else b * nc ** 3


def bench_config(nc: int, mach: float, re: float, ws: int) -> dict:
    """The workload both arms time (identical keys and values in both lines)."""
    return {"workload": f"DHIT {nc}^3 WENO-GKS step, FP64 parity path", "nc": nc, "k0": K0, "mach_t": mach,
            "re_lambda": re, "cfl": CFL, "precision": "fp64", "parallelism": f"replicas x{ws}",
            "l2": f"working set {32 * 8 * nc ** 3 / 1e6:.0f} MB per field (state {40 * nc ** 3 / 1e6:.0f} MB)"
                  " vs 126 MB L2, no flush"}


def make_case(nc: int, seed: int, mach: float = MACH, re: float = RE):
    import gks_ic

    return gks_ic.make_dhit(nc, k0=K0, Mt=mach, Re_lambda=re, seed=seed)


def timed_steps(solver, steps: int, torch) -> float:
    """ms per step over `steps` graph launches, CUDA events on the library stream."""
    stream = torch.cuda.ExternalStream(solver.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    solver.step(steps)
    e1.record(stream)
    e1.synchronize()
    solver.sync()
    return e0.elapsed_time(e1) / steps


def cpu_baseline(nc: int, steps: int, warmup: int, planes: int = 8, procs: int = 1) -> dict | None:
    """The reference CPU step (oracle/_ref) on y-slabs of the same field."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gks_ic
    import pyoracle

    if not os.path.exists(pyoracle.REF_HARNESS_FAST):
        return None
    case = make_case(nc, 0)
    d = tempfile.mkdtemp(prefix="gks_cpu_")
    gks_ic.write_case(d, case, slab_planes=planes)
    cmd = pyoracle.ref_time_cmd(d, steps, nc // planes, CFL, warmup)
    ps = [subprocess.Popen(cmd, stdout=subprocess.PIPE, text=True) for _ in range(procs)]
    res = []
    for p in ps:
        out, _ = p.communicate()
        if p.returncode != 0:
            return None
        res.append(json.loads(out.strip().splitlines()[-1]))
    secs = max(r["seconds"] for r in res)
    cells = sum(r["cells"] for r in res)
    return {"value": cells * steps / secs, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"{steps} timed step(s) after {warmup} warm-up of the reference CPU step "
                      f"(update.cpp evolveEulerian + HaloTransfer, g++ -O3 -march=x86-64-v3) on a "
                      f"{planes}x{nc}x{nc} y-slab of the {nc}^3 field per process, {procs} process(es)"}


def particle_cpu_baseline(W, case, npart: int) -> dict:
    """The oracle's particle routine (orc_particle_props: natural cubic
    B-splines of the five primitives over the padded block, then value and
    gradient at every particle) on one host core, on the same field and number
    of particles as the GPU figure.  A port, not the reference: the
    reference's tracker needs einspline, which is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import pyoracle

    prm = pyoracle.params(case.nc, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    rng = np.random.default_rng(7)
    rec = np.zeros((pyoracle.PREC_FIELDS, npart))
    for q in range(3):
        rec[q] = rng.random(npart) * 2 * np.pi
    t0 = time.perf_counter()
    pyoracle.particle_props(W, prm, rec)
    ms = (time.perf_counter() - t0) * 1e3
    return {"props_ms": ms, "cores": 1, "kind": "port",
            "sample": f"one orc_particle_props call (gcc -O2) on the same {case.nc}^3 field with {npart} "
                      "particles"}


def reference_gpu(nc: int, steps: int, warmup: int) -> dict | None:
    """The reference's own GPU path on the same field: GPUupdate.cu and GPUAlloc.cu
    built for sm_100a (oracle/_ref/ref_gpu_harness).  Each of its steps is evolve()
    -- host-to-device copy of the padded field, its derivs/flip/flux/update
    kernels, device-to-host copy -- followed by HaloTransfer on the host; a
    separate process with its own CUDA context."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gks_ic
    import pyoracle

    if not pyoracle.have_ref_gpu():
        return None
    d = tempfile.mkdtemp(prefix="gks_refgpu_")
    gks_ic.write_case(d, make_case(nc, 0))
    try:
        r = pyoracle.ref_time(d, steps, 1, CFL, warmup, gpu=True, timeout=600)
    except (subprocess.SubprocessError, OSError, ValueError):
        return None
    return {"value": r["cells"] * steps / r["seconds"], "unit": UNIT, "ms_per_step": 1e3 * r["seconds"] / steps,
            "evolve_ms_per_step": 1e3 * r["step_seconds"] / steps, "steps": steps, "warmup": warmup,
            "what": "reference GPU path (GPUupdate.cu, nvcc -O3 for sm_100a): evolve() with its per-step "
                    "host<->device copies of the padded field + host HaloTransfer, wall clock"}


def ensemble_cases(n_each: int = 32):
    """96 realisations: n_each at 32^3, 48^3 and 64^3, own seeds, k0 in {3,4,5},
    Mt uniform in [0.2, 0.5], Re_lambda 72."""
    import gks_ic
    import numpy as np

    rng = np.random.default_rng(1234)
    cases = []
    seed = 0
    for nc in (32, 48, 64):
        for _ in range(n_each):
            k0 = float(rng.choice([3.0, 4.0, 5.0]))
            mt = float(rng.uniform(0.2, 0.5))
            cases.append(gks_ic.make_dhit(nc, k0=k0, Mt=mt, Re_lambda=72.0, seed=seed))
            seed += 1
    return cases


def run_ensemble(gks, gks_ic, torch, steps: int, warmup: int, local: int, tune: bool) -> dict:
    cases = ensemble_cases()
    cells = sum(c.nc ** 3 for c in cases)
    out = {"fields": len(cases), "sizes": "32x32^3 + 32x48^3 + 32x64^3", "cells_per_step": cells}
    for name, prec in (("fp64", gks.FP64), ("mixed", gks.MIXED)):
        s = gks.Solver([gks.phys_from_case(c) for c in cases], prec, device=local)
        for f, c in enumerate(cases):
            s.upload(gks_ic.to_conservative_padded(c), f)
            s.timestep(CFL, f)
        if tune:
            s.autotune(2)
        s.step(warmup)
        s.sync()
        ms = timed_steps(s, steps, torch)
        s.close()
        out[name] = {"value": cells / (ms * 1e-3), "ms_per_step": ms}
    out["unit"] = UNIT
    out["launches_per_step"] = 7
    return out


def accuracy_history(gks, torch, nc: int, mach: float, re: float, t_end: float, control: bool = False,
                     stats_every: int = 10) -> dict:
    """Mixed vs FP64 on the same field to t/t0 = t_end (statistics every
    `stats_every` steps): relative errors of the statistics at the end and their
    largest value over the history.  With control, the second run is the FP64
    path started from the initial field rounded to FP32 (no FP32 arithmetic),
    the size of difference any FP32-rounding perturbation grows into."""
    import numpy as np

    import gks_ic

    case = make_case(nc, 0, mach, re)
    W = gks_ic.to_conservative_padded(case)
    hist = {}
    W32 = W.astype(np.float32).astype(np.float64) if control else None
    runs = (("fp64", gks.FP64, W), ("mixed", gks.FP64 if control else gks.MIXED, W32 if control else W))
    nsteps = dt = None
    for name, prec, w0 in runs:
        with gks.Solver(gks.phys_from_case(case), prec) as s:
            s.upload(w0)
            dt = s.timestep(CFL)
            nsteps = int(np.ceil(t_end * case.t0 / dt))
            h = []
            for k in range(nsteps + 1):
                if k % stats_every == 0 or k == nsteps:
                    h.append(s.stats())
                if k < nsteps:
                    s.step(1)
            s.sync()
            hist[name] = h
    keys = ("tke", "diss", "skew_u", "skew_v", "skew_w")
    final = {k: abs(hist["mixed"][-1][k] - hist["fp64"][-1][k]) / abs(hist["fp64"][-1][k]) for k in keys}
    worst = {k: max(abs(a[k] - b[k]) / abs(b[k]) for a, b in zip(hist["mixed"], hist["fp64"])) for k in keys}
    return {"nc": nc, "mach_t": mach, "re_lambda": re, "t_over_t0": t_end, "steps": nsteps, "dt": dt,
            "stats_every": stats_every, "rel_err_final": final, "rel_err_max_over_history": worst,
            "tke_fp64_initial": hist["fp64"][0]["tke"], "tke_fp64_final": hist["fp64"][-1]["tke"],
            "diss_fp64_final": hist["fp64"][-1]["diss"]}


def run_accuracy(args):
    """Mixed vs FP64 on the same field to t/t0 = args.t_end, plus each
    precision's step time (CUDA events over 10 further steps)."""
    import torch

    import gks_b200 as gks

    acc = accuracy_history(gks, torch, args.nc, args.mach, args.re, args.t_end, args.control)
    case = make_case(args.nc, 0, args.mach, args.re)
    import gks_ic

    ms = {}
    for name, prec in (("fp64", gks.FP64), ("mixed", gks.MIXED)):
        with gks.Solver(gks.phys_from_case(case), prec) as s:
            s.upload(gks_ic.to_conservative_padded(case))
            s.timestep(CFL)
            s.step(3)
            s.sync()
            ms[name] = timed_steps(s, 10, torch)
    acc.update({"mode": "accuracy-control" if args.control else "accuracy", "ms_per_step": ms,
                "cell_updates_per_s": {k: args.nc ** 3 / (v * 1e-3) for k, v in ms.items()},
                "mixed_speedup": ms["fp64"] / ms["mixed"]})
    print(json.dumps(acc))
    return 0


def reference_slabs(nc: int, cores: int) -> int:
    """Processes of the reference arm: the largest power of two up to `cores`
    (at most 64) that divides nc, one y-slab each."""
    p = 1
    while p * 2 <= min(cores, 64) and nc % (p * 2) == 0:
        p *= 2
    return p


def run_reference(args):
    """The reference's own CPU step on the whole field: P processes, each
    advancing its own y-slab (Init<a>00, as rank a of a P x 1 x 1 grid reads
    it), all started together; a step is every slab's evolveEulerian +
    HaloTransfer, timed by each process, and the job's step time is the slowest
    process's."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gks_ic
    import pyoracle

    if not os.path.exists(pyoracle.REF_HARNESS_FAST):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness_fast is not built"}))
        return 0
    nc = args.nc
    cores = len(os.sched_getaffinity(0))
    P = reference_slabs(nc, cores)
    planes = nc // P
    warm, steps = max(0, args.warmup), max(1, args.steps)
    d = tempfile.mkdtemp(prefix="gks_refarm_")
    gks_ic.write_case(d, make_case(nc, 0, args.mach, args.re), slab_planes=planes, all_slabs=True)
    ps = [subprocess.Popen(pyoracle.ref_time_cmd(d, steps, P, CFL, warm) + [str(a)], stdout=subprocess.PIPE,
                           text=True) for a in range(P)]
    res = []
    for p in ps:
        out, _ = p.communicate()
        if p.returncode != 0:
            print(json.dumps({"impl": "reference", "unavailable": f"reference step process exited {p.returncode}"}))
            return 0
        res.append(json.loads(out.strip().splitlines()[-1]))
    secs = max(r["seconds"] for r in res)
    cells = sum(r["cells"] for r in res)
    assert cells == nc ** 3 and sorted(r["slab_index"] for r in res) == list(range(P))
    value = cells * steps / secs
    sample = (f"the whole {nc}^3 field every step: {P} reference processes (update.cpp evolveEulerian + "
              f"HaloTransfer, g++ -O3 -march=x86-64-v3), each on its own {planes}x{nc}x{nc} y-slab; "
              f"{steps} timed steps after {warm} warm-up; slowest process")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
        "steps": steps, "warmup": warm, "ms_per_step": 1e3 * secs / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(nc, args.mach, args.re, ws),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": P, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "per_process_ms_per_step": sorted(1e3 * r["seconds"] / steps for r in res),
    }
    print(json.dumps(line))
    return 0


def measure_peaks(gks, uuid: str) -> dict:
    """FP64 / FP32 FMA peaks measured here (no FP64 figure is supplied): a first
    short burst, then the FP64 probe repeated for about 1.5 s with the SM clock
    sampled, whose settled rate (median of the second half) is the sustained
    peak that a kernel timed inside the long step loop is compared with; the
    nominal rate (SMs x 64 FP64 FMA lanes x 2 flops x clock) is given at the
    probe's clock and at the maximum clock, to locate the probe's gap."""
    import torch

    burst = gks.peak_tflops(gks.FP64)
    sampler = ClockSampler(uuid)
    sampler.start()
    runs, t0 = [], time.perf_counter()
    while time.perf_counter() - t0 < 1.5:
        runs.append(gks.peak_tflops(gks.FP64))
    clk = sampler.stop()
    peak64 = statistics.median(runs[len(runs) // 2:])
    peak32 = gks.peak_tflops(gks.MIXED)
    nsm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    out = {"fp64": peak64, "fp64_burst": burst, "fp32": peak32, "sms": nsm, "probe_clocks": clk}
    if clk:
        at_probe = nsm * FP64_LANES_PER_SM * 2 * clk["sm_mhz"] * 1e6 / 1e12
        at_max = nsm * FP64_LANES_PER_SM * 2 * clk["sm_max_mhz"] * 1e6 / 1e12
        out["fp64_nominal_at_probe_clock"] = at_probe
        out["fp64_nominal_at_max_clock"] = at_max
        out["probe_frac_of_nominal_at_probe_clock"] = peak64 / at_probe
        out["probe_frac_of_nominal_at_max_clock"] = peak64 / at_max
    return out


def run_ours(args):
    import torch

    import gks_b200 as gks
    import gks_ic

    ws, rank, local = dist_env()
    dist = Dist(ws, local)
    torch.cuda.set_device(local)
    gks.select_device(local)
    nc = args.nc
    case = make_case(nc, rank, args.mach, args.re)
    W = gks_ic.to_conservative_padded(case)
    phys = gks.phys_from_case(case)
    uuid = gpu_uuid(local)

    peaks = measure_peaks(gks, uuid)
    peak64 = peaks["fp64"]
    hbm_peak, hbm_src = 6650.0, "fallback 6.65 TB/s (no MEASURED_PEAKS.json)"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            hbm_peak, hbm_src = float(json.load(fh)["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except (OSError, ValueError, KeyError, TypeError):
        pass

    results = {}
    solvers = {}
    for name, prec in (("fp64", gks.FP64), ("mixed", gks.MIXED)):
        s = gks.Solver(phys, prec, device=local)
        s.upload(W)
        dt = s.timestep(CFL)
        if not args.no_tune:
            s.autotune(2)
        s.step(args.warmup)
        s.sync()
        dist.barrier()
        sampler = ClockSampler(uuid) if name == "fp64" else None
        if sampler:
            sampler.start()
        ms = timed_steps(s, args.steps, torch)
        clocks = sampler.stop() if sampler else None
        ms = dist.max(ms)
        results[name] = {"ms": ms, "dt": dt, "clocks": clocks, "stats": s.stats(), "launch": s.launch_config()}
        solvers[name] = s

    # stage timing (CUDA events around every launch) on both paths: per stage
    # the fastest of three samples of 5 individually launched steps each
    stages = {}
    for name in solvers:
        best = None
        for _ in range(3):
            st = solvers[name].time_stages(5)
            best = st if best is None else {k: min(best[k], st[k]) for k in st}
        stages[name] = best
    for name in solvers:
        solvers[name].close()

    # cost of one diagnostics evaluation (PrintStats' quantities) on the FP64 field
    s = gks.Solver(phys, gks.FP64, device=local)
    s.upload(W)
    s.timestep(CFL)
    s.stats()
    t0s = time.perf_counter()
    for _ in range(3):
        s.stats()
    stats_ms = (time.perf_counter() - t0s) / 3 * 1e3
    # the Lagrangian particle tracker on the same field (generateSplines +
    # getParticleProp for every particle, then one track), CUDA events on the
    # solver's stream
    prt = None
    if not args.no_particles:
        import numpy as np

        npart = 1 << 20
        rng = np.random.default_rng(7)
        s.particles_locate(*(rng.random(npart) * 2 * np.pi for _ in range(3)))
        pst = torch.cuda.ExternalStream(s.stream())
        s.particles_props()  # allocates the spline coefficients
        s.particles_track(1e-3)
        s.sync()
        pe = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        pe[0].record(pst)
        for _ in range(3):
            s.particles_props()
        pe[1].record(pst)
        for _ in range(3):
            s.particles_track(1e-3)
        pe[2].record(pst)
        pe[2].synchronize()
        prt = {"particles": npart, "props_ms": pe[0].elapsed_time(pe[1]) / 3,
               "track_ms": pe[1].elapsed_time(pe[2]) / 3,
               "what": "gks_particles_props (natural cubic B-splines of den, u, v, w, p over the padded "
                       f"{nc + 6}^3 block + value and gradient at every particle) and gks_particles_track, "
                       "uniformly random positions"}
    s.close()

    ens = None
    if not args.no_ensemble:
        ens = run_ensemble(gks, gks_ic, torch, args.steps, args.warmup, local, not args.no_tune)
        ens["fp64"]["ms_per_step"] = dist.max(ens["fp64"]["ms_per_step"])
        ens["mixed"]["ms_per_step"] = dist.max(ens["mixed"]["ms_per_step"])
        for k in ("fp64", "mixed"):
            ens[k]["value"] = whole_job_rate(ws, ens["cells_per_step"], ens[k]["ms_per_step"])

    # e2e through the reference-facing call, evolve(W, dev, dt): gks_evolve on a
    # pinned host field per step (upload, step, download; the copies overlap
    # the step slab by slab)
    nt = nc + 6
    host = torch.empty((5, nt, nt, nt), dtype=torch.float64, pin_memory=True).numpy()
    host[...] = W
    s = gks.Solver(phys, gks.FP64, device=local)
    s.upload(host)
    s.timestep(CFL)
    stream = torch.cuda.ExternalStream(s.stream())
    e2e_steps = max(1, min(args.steps, 5))
    s.evolve(host)  # warm-up: allocates the pipeline buffers
    s.evolve(host)
    torch.cuda.synchronize()
    dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        s.evolve(host)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = dist.max(e0.elapsed_time(e1) / e2e_steps)
    # the unpipelined sequence on the same buffers, for comparison
    t0p = time.perf_counter()
    for _ in range(2):
        s.upload(host)
        s.step(1)
        s.download(out=host)
    e2e_plain_ms = (time.perf_counter() - t0p) / 2 * 1e3
    s.close()
    bytes_io = 5 * nt ** 3 * 8

    # the mixed path's accuracy against FP64 to t/t0 = 2 on the same field
    acc = None
    if not args.no_accuracy:
        acc = accuracy_history(gks, torch, nc, args.mach, args.re, 2.0)

    cells = nc ** 3
    value = whole_job_rate(ws, cells, results["fp64"]["ms"])
    mixed_value = whole_job_rate(ws, cells, results["mixed"]["ms"])
    flux_ms = statistics.mean(stages["fp64"][k] for k in ("flux_x", "flux_y", "flux_z"))
    recon_ms = statistics.mean(stages["fp64"][k] for k in ("recon_x", "recon_y", "recon_z"))
    flux_s = flux_ms * 1e-3
    traffic = read_traffic(nc)
    # this algorithm's FP64 arithmetic per interface (ncu op counts of the flux
    # kernel, committed summary: 2 flops per DFMA, 1 per DMUL / DADD)
    flops = read_profile("flux_fp64_ncu.txt", "fp64_flops_per_interface")
    inst = read_profile("flux_fp64_ncu.txt", "fp64_inst_per_interface")
    achieved = flops * cells / flux_s / 1e12 if flops else None
    fp64_pipe = None
    if inst:
        rate = inst * cells / flux_s / 1e12
        fp64_pipe = {"inst_per_interface": inst, "achieved_tinst_s": rate, "peak_tinst_s": peak64 / 2,
                     "frac": rate / (peak64 / 2),
                     "note": "FP64 instructions per second against the FP64 FMA instruction rate: "
                             "pipe utilisation (a DMUL or DADD occupies the pipe like a DFMA)"}
        # the probe runs below the power cap, the step at it: the same fraction
        # against the probe's rate scaled to the SM clock sampled in the timed
        # FP64 steps (pipe utilisation per cycle, as ncu counts it)
        probe_mhz = (peaks.get("probe_clocks") or {}).get("sm_mhz")
        step_mhz = (results["fp64"]["clocks"] or {}).get("sm_mhz")
        if probe_mhz and step_mhz:
            fp64_pipe.update({"sm_mhz_probe": probe_mhz, "sm_mhz_step": step_mhz,
                              "frac_clock_matched": rate / (peak64 / 2 * step_mhz / probe_mhz)})
    st64, st32 = results["fp64"]["stats"], results["mixed"]["stats"]
    rel = {k: abs(st32[k] - st64[k]) / abs(st64[k]) for k in ("tke", "diss", "skew_u", "skew_v", "skew_w")}

    cb = rg = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cb = cpu_baseline(nc, 1, 1, planes=8, procs=1)
    if rank == 0 and ws == 1 and not args.no_refgpu:
        rg = reference_gpu(nc, 3, 1)
    if prt and rank == 0 and ws == 1 and not args.no_cpu:
        prt["cpu_baseline"] = particle_cpu_baseline(W, case, prt["particles"])

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": results["fp64"]["ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": f"synthetic: seeded solenoidal DHIT field (k0 4, Mt {args.mach:g}, Re_lambda {args.re:g}), "
                    "one replica per GPU",
            "config": bench_config(nc, args.mach, args.re, ws),
            "roofline": {"bound": "fp64", "kernel": "flux sweep (k_flux, FP64)", "achieved": achieved,
                         "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64 if achieved else None,
                         "traffic": traffic,
                         "flops_per_interface": flops,
                         "flops_source": "FP64 flops the co-moving-frame flux executes per interface "
                                         "(2 x DFMA + DMUL + DADD, profiles/flux_fp64_ncu.txt)",
                         "peak_source": "FP64 FMA peak measured live by gks_peak_flops on this GPU, sustained"
                                        " (the probe repeated for 1.5 s; the kernel is timed inside the step loop)",
                         "peak_burst": peaks["fp64_burst"], "launch_ms": flux_ms,
                         "fp64_pipe": fp64_pipe,
                         "probe": {k: peaks.get(k) for k in ("sms", "probe_clocks", "fp64_nominal_at_probe_clock",
                                                             "fp64_nominal_at_max_clock",
                                                             "probe_frac_of_nominal_at_probe_clock",
                                                             "probe_frac_of_nominal_at_max_clock")},
                         "reference_ops_equivalent": {
                             "ops_per_interface": OPS_FLUX,
                             "tflops": OPS_FLUX * cells / flux_s / 1e12,
                             "step_tflops": OPS_CELL * cells / (results["fp64"]["ms"] * 1e-3) / 1e12,
                             "note": "the reference formulation's operation count (MCal contractions); "
                                     "not a roofline fraction"},
                         "fp32_peak": peaks["fp32"]},
            "hbm": {"achieved_gbs": BYTES_CELL * cells / (results["fp64"]["ms"] * 1e-3) / 1e9,
                    "peak_gbs": hbm_peak, "peak_source": hbm_src,
                    "note": "compulsory 80 B/cell-update; the path is FP64-pipe bound"},
            "stage_ms": stages["fp64"], "recon_ms": recon_ms, "stats_ms": stats_ms,
            "particles": prt,
            "ensemble": ens,
            "launch": {"fp64": results["fp64"]["launch"], "mixed": results["mixed"]["launch"],
                       "tuned": not args.no_tune},
            "e2e": {"value": whole_job_rate(ws, cells, e2e_ms), "unit": UNIT, "h2d_bytes_per_step": bytes_io,
                    "d2h_bytes_per_step": bytes_io, "ms_per_step": e2e_ms,
                    "call": "gks_evolve(W, 1) per step (the reference's evolve(W, dev, dt)), pinned host buffers",
                    "unpipelined_ms_per_step": e2e_plain_ms},
            "clocks": results["fp64"]["clocks"],
            "gpu_launches": 7 * args.steps,
        }
        if cb:
            line["cpu_baseline"] = cb
        if rg:
            line["reference_gpu"] = rg
        line["mixed"] = {"value": mixed_value, "ms_per_step": results["mixed"]["ms"],
                         "speedup_vs_fp64": mixed_value / value,
                         "rel_err_vs_fp64_after_steps": rel, "steps_compared": args.warmup + args.steps,
                         "dtype": "f32 weno/slopes/slope moments + f64 moments/erfc/update/reductions",
                         "stage_ms": stages["mixed"], "accuracy_t2": acc}
        # compact summary last, so that the end of the line carries it
        line["headline"] = {
            "fp64_cell_updates_per_s": value, "mixed_cell_updates_per_s": mixed_value,
            "mixed_over_fp64": mixed_value / value,
            "e2e_cell_updates_per_s": line["e2e"]["value"],
            "flux_fp64_pipe_frac": fp64_pipe["frac"] if fp64_pipe else None,
            "flux_fp64_pipe_frac_clock_matched": fp64_pipe.get("frac_clock_matched") if fp64_pipe else None,
            "mixed_rel_err_t2_final": {k: acc["rel_err_final"][k] for k in ("tke", "diss")} if acc else None,
            "mixed_rel_err_t2_max": {k: acc["rel_err_max_over_history"][k] for k in ("tke", "diss")} if acc else None,
            "stats_ms": stats_ms,
        }
        print(json.dumps(line))
    dist.close()
    return 0


def run_slabs(args):
    """One nc^3 field split over the ranks along y (gks_slabs: NCCL halo
    exchange after every step), or with --local-slabs P over P slabs in this
    process on one GPU (device-copy exchange): strong scaling of one field,
    the halo exchange inside the timed steps.  Not the headline line."""
    import socket

    import torch
    import torch.distributed as tdist

    import gks_b200 as gks
    import gks_ic
    import gks_slabs

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    gks.select_device(local)
    local_p = args.local_slabs
    if not local_p and not tdist.is_initialized():
        import datetime

        if ws == 1:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            if "MASTER_PORT" not in os.environ:
                with socket.socket() as sk:
                    sk.bind(("127.0.0.1", 0))
                    os.environ["MASTER_PORT"] = str(sk.getsockname()[1])
            os.environ.setdefault("RANK", "0")
            os.environ.setdefault("WORLD_SIZE", "1")
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
    nc = args.nc
    case = make_case(nc, 0, args.mach, args.re)
    W = gks_ic.to_conservative_padded(case)
    phys = gks.phys_from_case(case)
    tuned = None
    if not args.no_tune:
        with gks.Solver(phys, gks.FP64, device=local) as s:
            s.upload(W)
            s.timestep(CFL)
            s.autotune(2)
            tuned = s.launch_config()
    if local_p:
        f = gks_slabs.LocalSlabs(phys, local_p, gks.FP64)
        solvers, nslabs = f.solvers, local_p
        f.upload(W)
    else:
        f = gks_slabs.SlabField(phys, gks.FP64)
        solvers, nslabs = [f.solver], ws
        f.upload(gks_slabs.split_block(W, ws, rank))
    del W
    if tuned:
        for s in solvers:
            for kind in ("recon", "flux"):
                for d, a in enumerate("xyz"):
                    c = tuned[f"{kind}_{a}"]
                    s.set_launch(kind, d, c["variant"], c["grid"])
    dt = f.timestep(CFL)
    f.step(args.warmup)
    f.sync()
    if not local_p:
        tdist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(f.stream)
    f.step(args.steps)
    e1.record(f.stream)
    e1.synchronize()
    f.sync()
    ms = e0.elapsed_time(e1) / args.steps
    if not local_p and ws > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        ms = float(t.item())
    st = f.stats()
    f.close()
    if rank == 0:
        line = {"metric": METRIC, "value": nc ** 3 / (ms * 1e-3), "unit": UNIT, "n_gpus": 1 if local_p else ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": f"synthetic: seeded solenoidal DHIT field (k0 {K0}, Mt {args.mach:g}, Re_lambda {args.re:g})",
                "config": {"workload": f"DHIT {nc}^3 WENO-GKS step, FP64, one field in {nslabs} y-slabs",
                           "nc": nc, "slabs": nslabs, "slab_planes": nc // nslabs,
                           "exchange": "device copy, one process" if local_p else "NCCL send/recv, one rank per GPU",
                           "parallelism": f"y-slabs x{nslabs}", "tuned": bool(tuned)},
                "dt": dt, "stats": {k: float(v) for k, v in st.items()},
                "e2e": None, "e2e_note": "device-resident slabs; the host per-step call is the default line's"}
        print(json.dumps(line), flush=True)
    if not local_p:
        tdist.barrier()
        tdist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nc", type=int, default=NC)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-tune", action="store_true", help="keep the untuned launch configuration")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 96-field ensemble line")
    ap.add_argument("--no-refgpu", action="store_true", help="skip timing the reference's own GPU path")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the mixed-vs-FP64 run to t/t0 = 2")
    ap.add_argument("--no-particles", action="store_true", help="skip timing the Lagrangian particle tracker")
    ap.add_argument("--accuracy", action="store_true", help="mixed vs FP64 statistics to t/t0 = --t-end, then exit")
    ap.add_argument("--t-end", type=float, default=2.0, help="accuracy run length in eddy turnover times")
    ap.add_argument("--control", action="store_true",
                    help="with --accuracy: compare FP64 with FP64 started from the initial field rounded to FP32")
    ap.add_argument("--mach", type=float, default=MACH, help="turbulent Mach number of the field")
    ap.add_argument("--re", type=float, default=RE, help="Re_lambda of the field")
    ap.add_argument("--slabs", action="store_true",
                    help="one field split over the ranks along y (NCCL halo exchange); strong scaling")
    ap.add_argument("--local-slabs", type=int, default=0,
                    help="one field split into this many y-slabs in one process on one GPU")
    args = ap.parse_args()
    if args.accuracy:
        return run_accuracy(args)
    if args.warmup < 3 and args.impl == "ours":
        ap.error("at least 3 warm-up steps")
    if args.impl == "reference":
        return run_reference(args)
    if args.slabs or args.local_slabs:
        return run_slabs(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
