"""Python access to the CPU oracle (test infrastructure only).

Two checkers live under oracle/:

* ``build/liboracle.so``: the plain-C restatement of the reference hot path
  (gks_oracle.c), loaded through ctypes;
* ``_ref/ref_harness``: the reference's own CPU path compiled from its sources
  (see the Makefile), driven as a subprocess;
* ``_ref/ref_gpu_harness``: the same driver around the reference's own GPU
  path (GPUupdate.cu, GPUAlloc.cu) built for sm_100a; it needs a GPU.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use this
module, and only to check or time against; the product never imports it.
"""

from __future__ import annotations

import ctypes
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")
REF_HARNESS_FAST = os.path.join(HERE, "_ref", "ref_harness_fast")
REF_GPU_HARNESS = os.path.join(HERE, "_ref", "ref_gpu_harness")

VISC_SUTHERLAND = 0
VISC_POWER = 1
FIX_ZSWEEP = 1
DIRECT_ENERGY = 2
PR_FACTOR_CPU = 1.0 / 0.7  # GKMflux.cpp:289
PR_FACTOR_GPU = 1.0        # GPUupdate.cu:839


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("nc", ctypes.c_int), ("K", ctypes.c_int), ("visc_law", ctypes.c_int), ("flags", ctypes.c_int),
        ("gam", ctypes.c_double), ("R", ctypes.c_double), ("dx", ctypes.c_double),
        ("T0", ctypes.c_double), ("mu0", ctypes.c_double), ("visc_exp", ctypes.c_double),
        ("pr_factor", ctypes.c_double), ("p0", ctypes.c_double), ("den0", ctypes.c_double),
        ("Mt", ctypes.c_double), ("t0", ctypes.c_double),
    ]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_weno.argtypes = [dp, ctypes.c_double, ctypes.c_double, ctypes.c_int, dp, dp]
        L.orc_flux.argtypes = [dp, ctypes.c_double, ctypes.c_int, ctypes.c_double, dp]
        L.orc_halo.argtypes = [dp, ctypes.c_int]
        L.orc_step.argtypes = [dp, ctypes.POINTER(OrcParams), ctypes.c_double, dp]
        L.orc_maxval.argtypes = [dp, ctypes.POINTER(OrcParams)]
        L.orc_maxval.restype = ctypes.c_double
        L.orc_stats.argtypes = [dp, ctypes.POINTER(OrcParams), dp]
        L.orc_stats_ranks.argtypes = [dp, ctypes.POINTER(OrcParams), ctypes.c_int, dp]
        L.orc_bspline3.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_long, dp, dp]
        L.orc_spline_eval.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_long, dp, dp, dp, ctypes.c_long,
                                      dp, dp, dp]
        L.orc_particle_props.argtypes = [dp, ctypes.POINTER(OrcParams), ctypes.c_long, dp]
        L.orc_particle_track.argtypes = [ctypes.c_long, dp, ctypes.c_double]
        L.orc_particle_stats.argtypes = [ctypes.c_long, dp, dp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def params(nc, gam, mu0, p0, den0=1.0, Mt=0.3, t0=1.0, visc_law=VISC_SUTHERLAND, visc_exp=0.76,
           pr_factor=PR_FACTOR_CPU, flags=0, R=287.0) -> OrcParams:
    dx = 2.0 * (np.arctan(1.0) * 4.0) / nc
    K = int((5.0 - 3.0 * gam) / (gam - 1.0))
    T0 = p0 / (R * den0)
    return OrcParams(nc, K, visc_law, flags, gam, R, dx, T0, mu0, visc_exp, pr_factor, p0, den0, Mt, t0)


def weno(stencils: np.ndarray, gam=1.4, R=287.0, direct_energy=False):
    """stencils (n, 6, 5) -> (wl, wr) each (n, 5)."""
    s = np.ascontiguousarray(stencils, dtype=np.float64)
    n = s.shape[0]
    wl = np.empty((n, 5))
    wr = np.empty((n, 5))
    L = lib()
    for c in range(n):
        L.orc_weno(_p(s[c]), gam, R, int(direct_energy), _p(wl[c]), _p(wr[c]))
    return wl, wr


def flux(inputs: np.ndarray, gam=1.4, K=2, pr_factor=PR_FACTOR_CPU):
    """inputs (n, 53) -> F (n, 5)."""
    x = np.ascontiguousarray(inputs, dtype=np.float64)
    F = np.empty((x.shape[0], 5))
    L = lib()
    for c in range(x.shape[0]):
        L.orc_flux(_p(x[c]), gam, K, pr_factor, _p(F[c]))
    return F


def step(W: np.ndarray, prm: OrcParams, dt: float, nsteps: int = 1) -> np.ndarray:
    """Advance a padded (5, nt, nt, nt) block in place by nsteps steps."""
    assert W.shape[0] == 5 and W.flags["C_CONTIGUOUS"]
    scratch = np.zeros((15,) + W.shape[1:])
    L = lib()
    for _ in range(nsteps):
        L.orc_step(_p(W), ctypes.byref(prm), dt, _p(scratch))
    return W


def maxval(W: np.ndarray, prm: OrcParams) -> float:
    return lib().orc_maxval(_p(np.ascontiguousarray(W)), ctypes.byref(prm))


def stats(W: np.ndarray, prm: OrcParams) -> np.ndarray:
    out = np.empty(14)
    lib().orc_stats(_p(np.ascontiguousarray(W)), ctypes.byref(prm), _p(out))
    return out


def stats_ranks(W: np.ndarray, prm: OrcParams, nranks: int) -> np.ndarray:
    """Diagnostics of the field split over nranks ranks along y (orc_stats_ranks)."""
    out = np.empty(14)
    lib().orc_stats_ranks(_p(np.ascontiguousarray(W)), ctypes.byref(prm), nranks, _p(out))
    return out


def halo(W: np.ndarray, nc: int) -> np.ndarray:
    lib().orc_halo(_p(W), nc)
    return W


# --- Lagrangian particles (orc_bspline3 ... orc_particle_stats) -------------

PREC_FIELDS = 23  # ORC_PREC_FIELDS


def bspline3(data: np.ndarray) -> np.ndarray:
    """Natural cubic B-spline coefficients (N0+2, N1+2, N2+2) of data (N0, N1, N2)."""
    d = np.ascontiguousarray(data, dtype=np.float64)
    c = np.empty(tuple(n + 2 for n in d.shape))
    lib().orc_bspline3(d.shape[0], d.shape[1], d.shape[2], _p(d), _p(c))
    return c


def spline_eval(coef: np.ndarray, start, hinv, pos: np.ndarray):
    """Value (n,) and gradient (3, n) of the spline at pos (3, n)."""
    c = np.ascontiguousarray(coef, dtype=np.float64)
    x = np.ascontiguousarray(pos, dtype=np.float64)
    n = x.shape[1]
    val = np.empty(n)
    grad = np.empty((3, n))
    st = np.asarray(start, dtype=np.float64)
    hi = np.asarray(hinv, dtype=np.float64)
    N = [s - 2 for s in c.shape]
    lib().orc_spline_eval(N[0], N[1], N[2], _p(c), _p(st), _p(hi), n, _p(x), _p(val), _p(grad))
    return val, grad


def particle_props(W: np.ndarray, prm: OrcParams, rec: np.ndarray) -> np.ndarray:
    """Fill fields 3..22 of the particle records rec (23, n) from the padded block W (ghosts filled)."""
    assert rec.shape[0] == PREC_FIELDS and rec.flags["C_CONTIGUOUS"]
    lib().orc_particle_props(_p(np.ascontiguousarray(W)), ctypes.byref(prm), rec.shape[1], _p(rec))
    return rec


def particle_track(rec: np.ndarray, dt: float) -> np.ndarray:
    assert rec.shape[0] == PREC_FIELDS and rec.flags["C_CONTIGUOUS"]
    lib().orc_particle_track(rec.shape[1], _p(rec), dt)
    return rec


def particle_stats(rec: np.ndarray) -> np.ndarray:
    out = np.empty(9)
    lib().orc_particle_stats(rec.shape[1], _p(np.ascontiguousarray(rec)), _p(out))
    return out


# --- the reference build ---------------------------------------------------

def have_ref() -> bool:
    return os.path.exists(REF_HARNESS)


def have_ref_gpu() -> bool:
    return os.path.exists(REF_GPU_HARNESS)


def ref_run(casedir: str, nsteps: int, cfl: float, dumps, stats_on=True, outdir=None, gpu=False, field=False):
    """Run the reference binary (its CPU path, or with gpu=True its GPU path);
    returns dict(meta, stats, dumps, stdout, field).  With field=True the
    reference's writeField dumps the primitives once at the first step with
    t >= t0 into casedir/Results/Field; `field` is then (file name, bytes)."""
    outdir = outdir or tempfile.mkdtemp(prefix="gksref_")
    os.makedirs(outdir, exist_ok=True)
    dl = ",".join(str(d) for d in dumps) if dumps else ","
    cp = subprocess.run([REF_GPU_HARNESS if gpu else REF_HARNESS, "run", os.path.abspath(casedir), os.path.abspath(outdir), str(nsteps),
                         repr(cfl), "1" if stats_on else "0", dl, "1" if field else "0"],
                        check=True, capture_output=True, text=True)
    fld = None
    if field:
        fdir = os.path.join(casedir, "Results", "Field")
        names = sorted(os.listdir(fdir)) if os.path.isdir(fdir) else []
        if len(names) == 1:
            with open(os.path.join(fdir, names[0]), "rb") as f:
                fld = (names[0], f.read())
    meta = {}
    with open(os.path.join(outdir, "meta.txt")) as f:
        for line in f:
            k, v = line.split()
            meta[k] = float(v)
    st = np.fromfile(os.path.join(outdir, "stats.bin"), dtype=np.float64).reshape(-1, 9)
    nc = int(meta["nc"])
    nt = nc + 6
    out = {}
    for d in dumps:
        out[d] = np.fromfile(os.path.join(outdir, f"W_{d}.bin"), dtype=np.float64).reshape(5, nt, nt, nt)
    lines = [ln for ln in cp.stdout.splitlines() if ln.strip() and ln.strip()[0].isdigit()]
    return {"meta": meta, "stats": st, "dumps": out, "stdout": lines, "outdir": outdir, "field": fld}


def _blob(path, n, header: bytes, rows: np.ndarray):
    with open(path, "wb") as f:
        f.write(struct.pack("<i", n))
        f.write(header)
        f.write(np.ascontiguousarray(rows, dtype="<f8").tobytes())


def ref_weno(stencils: np.ndarray, gam=1.4):
    n = stencils.shape[0]
    d = tempfile.mkdtemp(prefix="gksweno_")
    _blob(os.path.join(d, "in"), n, struct.pack("<d", gam), stencils.reshape(n, 30))
    subprocess.run([REF_HARNESS, "weno", os.path.join(d, "in"), os.path.join(d, "out")], check=True)
    o = np.fromfile(os.path.join(d, "out"), dtype=np.float64).reshape(n, 10)
    return o[:, :5], o[:, 5:]


def ref_flux(inputs: np.ndarray, gam=1.4, K=2):
    n = inputs.shape[0]
    d = tempfile.mkdtemp(prefix="gksflux_")
    _blob(os.path.join(d, "in"), n, struct.pack("<dd", gam, float(K)), inputs.reshape(n, 53))
    subprocess.run([REF_HARNESS, "flux", os.path.join(d, "in"), os.path.join(d, "out")], check=True)
    return np.fromfile(os.path.join(d, "out"), dtype=np.float64).reshape(n, 5)


def ref_time_cmd(casedir: str, nsteps: int, slabs: int, cfl: float, warmup: int = 0, fast=True, gpu=False) -> list:
    exe = REF_GPU_HARNESS if gpu else (REF_HARNESS_FAST if fast else REF_HARNESS)
    return [exe, "time", os.path.abspath(casedir), str(nsteps), str(slabs), repr(cfl), str(warmup)]


def ref_time(casedir: str, nsteps: int, slabs: int, cfl: float, warmup: int = 0, fast=True, gpu=False,
             timeout=None) -> dict:
    import json
    cp = subprocess.run(ref_time_cmd(casedir, nsteps, slabs, cfl, warmup, fast, gpu), check=True,
                        capture_output=True, text=True, timeout=timeout)
    return json.loads(cp.stdout.strip().splitlines()[-1])
