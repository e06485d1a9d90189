"""Python binding of the gks_b200 C ABI (include/gks_b200.h) through ctypes.

The binding mirrors the reference's run loop objects: a ``Solver`` owns one
device context (one field, or an ensemble of fields of different sizes) and
exposes the calls the reference's driver makes each step -- upload of the
conservative fields in the reference's padded layout, the time step from the
CFL condition, the step itself, download, and the diagnostics PrintStats
prints.  There is no fallback: if ``lib/libgks_b200.so`` is missing or no GPU
is present, construction raises.
"""

from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgks_b200.so")

FP64 = 0
MIXED = 1
FIX_ZSWEEP = 1
DIRECT_ENERGY = 2
VISC_SUTHERLAND = 0
VISC_POWER = 1
PR_FACTOR_CPU = 1.0 / 0.7  # GKMflux.cpp:289
PR_FACTOR_GPU = 1.0        # GPUupdate.cu:839

ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "ESTATE", -5: "ENONFINITE", -6: "ETOOBIG"}

STATS_FIELDS = ["tke", "diss", "skew_u", "skew_v", "skew_w", "kurt_u", "kurt_v", "kurt_w",
                "prms", "trms", "vrms", "sijsij", "mach_t", "rho_mean"]


class GksError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gks error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Phys(ctypes.Structure):
    _fields_ = [
        ("nc", ctypes.c_int), ("K", ctypes.c_int), ("visc_law", ctypes.c_int), ("reserved", ctypes.c_int),
        ("gam", ctypes.c_double), ("gas_r", ctypes.c_double), ("T0", ctypes.c_double), ("mu0", ctypes.c_double),
        ("visc_exp", ctypes.c_double), ("pr_factor", ctypes.c_double),
        ("p0", ctypes.c_double), ("den0", ctypes.c_double), ("Mt", ctypes.c_double), ("t0", ctypes.c_double),
    ]


class StatsOut(ctypes.Structure):
    _fields_ = [
        ("tke", ctypes.c_double), ("diss", ctypes.c_double), ("skew", ctypes.c_double * 3),
        ("kurt", ctypes.c_double * 3), ("prms", ctypes.c_double), ("trms", ctypes.c_double),
        ("vrms", ctypes.c_double), ("sijsij", ctypes.c_double), ("mach_t", ctypes.c_double),
        ("rho_mean", ctypes.c_double),
    ]

    def as_array(self) -> np.ndarray:
        return np.array([self.tke, self.diss, *self.skew, *self.kurt, self.prms, self.trms, self.vrms,
                         self.sijsij, self.mach_t, self.rho_mean])


class ParticleStatsOut(ctypes.Structure):
    _fields_ = [
        ("tke", ctypes.c_double), ("sijsij", ctypes.c_double), ("dudx2", ctypes.c_double),
        ("dudx3", ctypes.c_double), ("dwdz2", ctypes.c_double), ("dwdz3", ctypes.c_double),
        ("skew_u", ctypes.c_double), ("skew_w", ctypes.c_double), ("count", ctypes.c_longlong),
    ]

    def as_array(self) -> np.ndarray:
        return np.array([self.tke, self.sijsij, self.dudx2, self.dudx3, self.dwdz2, self.dwdz3, self.skew_u,
                         self.skew_w, float(self.count)])


DP = ctypes.POINTER(ctypes.c_double)
DP5 = DP * 5
PREC_FIELDS = 23  # GKS_PREC_FIELDS: doubles of one particle record

# every symbol the header declares, with (restype, argtypes)
SIGNATURES = {
    "gks_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(Phys),
                                  ctypes.c_int, ctypes.c_int]),
    "gks_destroy": (None, [ctypes.c_void_p]),
    "gks_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "gks_upload": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, DP5]),
    "gks_download": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, DP5]),
    "gks_evolve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, DP5, ctypes.c_int]),
    "gks_host_register": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int)]),
    "gks_host_unregister": (ctypes.c_int, [ctypes.c_void_p]),
    "gks_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, DP]),
    "gks_set_dt": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]),
    "gks_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "gks_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(StatsOut)]),
    "gks_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "gks_check": (ctypes.c_int, [ctypes.c_void_p]),
    "gks_device_fields": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, DP5]),
    "gks_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "gks_get_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "gks_select_device": (ctypes.c_int, [ctypes.c_int]),
    "gks_time_stages": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, DP]),
    "gks_peak_flops": (ctypes.c_int, [ctypes.c_int, DP]),
    "gks_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "gks_get_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "gks_set_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gks_timestep_noalloc": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_void_p, DP]),
    "gks_create_slab": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(Phys), ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gks_stats_part": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, DP]),
    "gks_stats_reduce": (ctypes.c_int, [DP, ctypes.c_int, ctypes.POINTER(Phys), ctypes.POINTER(StatsOut)]),
    "gks_halo_buffers": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                        ctypes.POINTER(ctypes.c_size_t)]),
    "gks_halo_pack": (ctypes.c_int, [ctypes.c_void_p]),
    "gks_halo_unpack": (ctypes.c_int, [ctypes.c_void_p]),
    "gks_particles_locate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, DP, DP, DP]),
    "gks_particles_props": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "gks_particles_track": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]),
    "gks_particles_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ParticleStatsOut)]),
    "gks_particles_get": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, DP]),
}

STATS_PART = 28  # doubles of one gks_stats_part record

STAGES = ["recon_x", "flux_x", "recon_y", "flux_y", "recon_z", "flux_z", "update"]


def select_device(device: int) -> None:
    rc = load_library().gks_select_device(device)
    if rc != 0:
        raise GksError(rc, f"cannot select CUDA device {device}")


def peak_tflops(precision: int = FP64) -> float:
    """Measured FMA peak of the current device's FP64 (FP64) or FP32 (MIXED) pipe."""
    out = ctypes.c_double()
    rc = load_library().gks_peak_flops(precision, ctypes.byref(out))
    if rc != 0:
        raise GksError(rc, "peak measurement failed")
    return out.value

_lib = None


def load_library(path: str = LIB_PATH):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with __graft_entry__.build() (make -C gkm-dns_b200)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def phys_from_case(case, visc_law=VISC_SUTHERLAND, visc_exp=0.76, pr_factor=PR_FACTOR_CPU) -> Phys:
    """gks_phys from a gks_ic.DhitCase (or any object with its attributes)."""
    return Phys(nc=case.nc, K=case.K, visc_law=visc_law, reserved=0, gam=case.gam, gas_r=287.0, T0=case.T0,
                mu0=case.mu0, visc_exp=visc_exp, pr_factor=pr_factor, p0=case.p0, den0=case.rho0, Mt=case.Mt,
                t0=case.t0)


def _ptrs(W: np.ndarray) -> DP5:
    assert W.dtype == np.float64 and W.flags["C_CONTIGUOUS"] and W.shape[0] == 5
    return DP5(*[W[q].ctypes.data_as(DP) for q in range(5)])


@dataclasses.dataclass
class _Field:
    nc: int
    nty: int  # planes of the padded host block along y: nc + 6, or a slab's ny + 6


def stats_reduce(parts: np.ndarray, phys: Phys) -> dict:
    """Merge gks_stats_part records (one row of STATS_PART per part, e.g. per
    rank) into the diagnostics of the whole field (gks_stats_reduce)."""
    parts = np.ascontiguousarray(parts, dtype=np.float64).reshape(-1, STATS_PART)
    out = StatsOut()
    rc = load_library().gks_stats_reduce(parts.ctypes.data_as(DP), len(parts), ctypes.byref(phys), ctypes.byref(out))
    if rc != 0:
        raise GksError(rc, "gks_stats_reduce: bad parts")
    return dict(zip(STATS_FIELDS, out.as_array()))


class Solver:
    """One context on the current CUDA device holding one or more fields, or
    (slab=(ny, y0)) the y-slab of ny interior planes from global plane y0 of
    one field split over ranks (gks_create_slab)."""

    def __init__(self, phys, precision: int = FP64, flags: int = 0, device: int | None = None,
                 slab: tuple | None = None):
        lib = load_library()
        if device is not None:
            select_device(device)
        if isinstance(phys, Phys):
            phys = [phys]
        h = ctypes.c_void_p()
        if slab is None:
            arr = (Phys * len(phys))(*phys)
            rc = lib.gks_create(ctypes.byref(h), len(phys), arr, precision, flags)
        else:
            if len(phys) != 1:
                raise ValueError("a slab context holds one field")
            rc = lib.gks_create_slab(ctypes.byref(h), ctypes.byref(phys[0]), int(slab[0]), int(slab[1]),
                                     precision, flags)
        if rc != 0:
            raise GksError(rc, "context creation failed (no CUDA device, bad constants or out of memory)")
        self._lib = lib
        self._h = h
        self.phys = list(phys)
        self.slab = slab
        self.fields = [_Field(p.nc, (slab[0] if slab else p.nc) + 6) for p in phys]
        self.precision = precision
        self.flags = flags

    def _ck(self, rc):
        if rc != 0:
            msg = self._lib.gks_last_error(self._h)
            raise GksError(rc, msg.decode() if msg else "")

    def close(self):
        if self._h:
            self._lib.gks_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # state ---------------------------------------------------------------
    def host_shape(self, f: int = 0) -> tuple:
        """Shape of field f's padded host block: (5, nt, nt, nt), or (5, ny + 6, nt, nt) for a slab."""
        nt = self.fields[f].nc + 6
        return (5, self.fields[f].nty, nt, nt)

    def upload(self, W: np.ndarray, f: int = 0):
        """W: float64 padded block in the reference's layout (host_shape)."""
        if W.shape != self.host_shape(f):
            raise ValueError(f"expected shape {self.host_shape(f)}, got {W.shape}")
        W = np.ascontiguousarray(W, dtype=np.float64)
        self._ck(self._lib.gks_upload(self._h, f, _ptrs(W)))

    def download(self, f: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.host_shape(f))
        self._ck(self._lib.gks_download(self._h, f, _ptrs(out)))
        return out

    def evolve(self, W: np.ndarray, nsteps: int = 1, f: int = 0) -> np.ndarray:
        """The reference's per-step call on host memory: W (host_shape) is
        uploaded, advanced nsteps steps and overwritten with the result (ghosts
        as the periodic image).  One field and one step overlap the copies with
        the step; pass W in pinned memory for full overlap."""
        shape = self.host_shape(f)
        if W.shape != shape or W.dtype != np.float64 or not W.flags["C_CONTIGUOUS"]:
            raise ValueError(f"expected a C-contiguous float64 array of shape {shape}")
        self._ck(self._lib.gks_evolve(self._h, f, _ptrs(W), nsteps))
        return W

    def timestep(self, cfl: float, f: int = 0) -> float:
        dt = ctypes.c_double()
        self._ck(self._lib.gks_timestep(self._h, f, cfl, ctypes.byref(dt)))
        return dt.value

    def set_dt(self, dt: float, f: int = 0):
        self._ck(self._lib.gks_set_dt(self._h, f, dt))

    def step(self, nsteps: int = 1):
        self._ck(self._lib.gks_step(self._h, nsteps))

    def sync(self):
        self._ck(self._lib.gks_sync(self._h))

    def check(self):
        self._ck(self._lib.gks_check(self._h))

    def stats(self, f: int = 0) -> dict:
        out = StatsOut()
        self._ck(self._lib.gks_stats(self._h, f, ctypes.byref(out)))
        return dict(zip(STATS_FIELDS, out.as_array()))

    def stats_array(self, f: int = 0) -> np.ndarray:
        out = StatsOut()
        self._ck(self._lib.gks_stats(self._h, f, ctypes.byref(out)))
        return out.as_array()

    def stats_part(self, f: int = 0) -> np.ndarray:
        """Mergeable diagnostics record of field f (gks_stats_part): STATS_PART doubles."""
        out = np.empty(STATS_PART)
        self._ck(self._lib.gks_stats_part(self._h, f, out.ctypes.data_as(DP)))
        return out

    # Lagrangian particles -----------------------------------------------------
    def particles_locate(self, x0: np.ndarray, y0: np.ndarray, z0: np.ndarray, f: int = 0):
        """Place len(x0) particles at (x0, y0, z0) (locateParticles; the three
        arrays of InitialConditions/unirand), velocity and properties zero."""
        xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x0, y0, z0)]
        if not (xs[0].size == xs[1].size == xs[2].size):
            raise ValueError("x0, y0, z0 must have the same length")
        self._ck(self._lib.gks_particles_locate(self._h, f, xs[0].size, *[a.ctypes.data_as(DP) for a in xs]))
        self._np = getattr(self, "_np", {})
        self._np[f] = xs[0].size

    def particles_props(self, f: int = 0):
        """Splines of the current state and every particle's values and gradients (asynchronous)."""
        self._ck(self._lib.gks_particles_props(self._h, f))

    def particles_track(self, dt: float, f: int = 0):
        """Move every particle by dt with the velocity of the last props call (asynchronous)."""
        self._ck(self._lib.gks_particles_track(self._h, f, dt))

    def particles_stats(self, f: int = 0) -> np.ndarray:
        """GetParticleStats: TKE, SijSij, DUDX2, DUDX3, DWDZ2, DWDZ3, SKEWu, SKEWw, count."""
        out = ParticleStatsOut()
        self._ck(self._lib.gks_particles_stats(self._h, f, ctypes.byref(out)))
        return out.as_array()

    def particles_get(self, f: int = 0) -> np.ndarray:
        """The particle records, (PREC_FIELDS, n) doubles (field-major)."""
        rec = np.empty((PREC_FIELDS, self._np[f]))
        self._ck(self._lib.gks_particles_get(self._h, f, rec.ctypes.data_as(DP)))
        return rec

    # halo exchange of a slab ------------------------------------------------
    def halo_buffers(self) -> tuple:
        """Device addresses of the slab's halo buffers (send south, send north,
        receive south, receive north) and their length in doubles."""
        ptrs = (ctypes.c_void_p * 4)()
        n = ctypes.c_size_t()
        self._ck(self._lib.gks_halo_buffers(self._h, ptrs, ctypes.byref(n)))
        return [ptrs[i] for i in range(4)], n.value

    def halo_pack(self):
        self._ck(self._lib.gks_halo_pack(self._h))

    def halo_unpack(self):
        self._ck(self._lib.gks_halo_unpack(self._h))

    def device_fields(self, f: int = 0):
        arr = DP5()
        self._ck(self._lib.gks_device_fields(self._h, f, arr))
        return [ctypes.cast(arr[q], ctypes.c_void_p).value for q in range(5)]

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._ck(self._lib.gks_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def time_stages(self, reps: int = 3) -> dict:
        """Mean ms per stage over reps individually launched steps (advances the state)."""
        ms = (ctypes.c_double * 7)()
        self._ck(self._lib.gks_time_stages(self._h, reps, ms))
        return dict(zip(STAGES, list(ms)))

    def autotune(self, reps: int = 2):
        """Pick register-cap variant and grid of every reconstruction / flux kernel."""
        self._ck(self._lib.gks_autotune(self._h, reps))

    def launch_config(self) -> dict:
        out = {}
        for kind, kname in enumerate(("recon", "flux", "update")):
            for d, dname in enumerate("xyz"):
                b, g, v = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
                self._ck(self._lib.gks_get_launch(self._h, kind, d, ctypes.byref(b), ctypes.byref(g), ctypes.byref(v)))
                out[f"{kname}_{dname}"] = {"block": b.value, "grid": g.value, "variant": v.value}
        return out

    def set_launch(self, kind: str, d: int, variant: int, grid: int = 0):
        """Pin kernel `kind` ("recon", "flux", "update") of sweep d (0, 1, 2) to a
        register-cap variant and grid (0: one wave of resident blocks)."""
        k = ("recon", "flux", "update").index(kind)
        self._ck(self._lib.gks_set_launch(self._h, k, d, grid, variant))

    def set_stream(self, stream: int | None):
        self._ck(self._lib.gks_set_stream(self._h, ctypes.c_void_p(stream or 0)))
