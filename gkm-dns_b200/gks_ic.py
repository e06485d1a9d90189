"""Seeded initial conditions for decaying isotropic turbulence, in the
reference's own input layout.

The reference ships no inputs: its WENO solver reads
``InitialConditions/params`` and ``InitialConditions/Init<a><b><c>``
(weno/src/FlowField.cpp:15-50, 59-112), which a MATLAB tool wrote
(GKM/CUDA GKM/InitialConditions/init_BS.m).  This module restates that tool
with a seeded numpy generator:

* three uniform random fields, transformed and projected onto divergence-free
  modes (init_BS.m:24-37);
* each spherical shell |k| ~ n rescaled to E(n) = n^4 exp(-2 n^2 / k0^2)
  (init_BS.m:40-83; the shell energy of every mode with round(|k|) = n);
* back-transformed, real part kept (init_BS.m:89-91).

Differences from the MATLAB tool, all forced by the run configurations: the
wavenumber grid is numpy's FFT ordering (the MATLAB grid ``-kmax:kmax`` with
``kmax = (N-1)/2`` is only integral for odd N, and the configurations use even
N); density and pressure are uniform with the sound speed fixed to 1
(p0 = rho0 / gamma) and the velocity is scaled so that
sqrt(<u^2+v^2+w^2>) = Mt (instead of fixing the velocity and deriving the sound
speed, init_BS.m:149-151).  The derived constants follow init_BS.m:146-157:
urms = Mt c0 / sqrt(3), lambda = 2 / k0, mu0 = rho0 urms lambda / Re_lambda,
t0 = lambda / urms.

Array convention used throughout this package: a field is a numpy array
indexed [j, i, k] = (y, x, z), the reference's index order (param.h:37), and
the velocity components (u, v, w) point along (x, y, z) = (i, j, k).
"""

from __future__ import annotations

import dataclasses
import os
import struct

import numpy as np

GAS_R = 287.0  # param.h:18


@dataclasses.dataclass
class DhitCase:
    """One realisation: primitive fields on the nc^3 interior plus constants."""

    nc: int
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    rho: np.ndarray
    p: np.ndarray
    gam: float
    rho0: float
    Mt: float
    Re: float
    mu0: float
    p0: float
    t0: float
    k0: float
    seed: int

    @property
    def T0(self) -> float:
        """FlowField.cpp:46."""
        return self.p0 / (GAS_R * self.rho0)

    @property
    def dx(self) -> float:
        """FlowField.cpp:45 (pi is atan(1)*4, param.h:14)."""
        return 2.0 * (np.arctan(1.0) * 4.0) / self.nc

    @property
    def K(self) -> int:
        """FlowField.cpp:41."""
        return int((5.0 - 3.0 * self.gam) / (self.gam - 1.0))


def solenoidal_field(nc: int, k0: float, seed: int):
    """Random-phase divergence-free velocity with shell spectrum n^4 exp(-2n^2/k0^2)."""
    rng = np.random.default_rng(seed)
    uk = np.fft.fftn(rng.random((nc, nc, nc)))
    vk = np.fft.fftn(rng.random((nc, nc, nc)))
    wk = np.fft.fftn(rng.random((nc, nc, nc)))
    kf = np.fft.fftfreq(nc, d=1.0 / nc)
    # axis 0 = y (j), axis 1 = x (i), axis 2 = z (k); u is the x component
    ky, kx, kz = np.meshgrid(kf, kf, kf, indexing="ij")
    ksq = np.maximum(kx * kx + ky * ky + kz * kz, 1e-14)
    kdot = kx * uk + ky * vk + kz * wk
    uk = uk - kdot * kx / ksq
    vk = vk - kdot * ky / ksq
    wk = wk - kdot * kz / ksq
    shell = np.rint(np.sqrt(kx * kx + ky * ky + kz * kz)).astype(np.int64)
    nshell = int(shell.max()) + 1
    energy = np.abs(uk) ** 2 + np.abs(vk) ** 2 + np.abs(wk) ** 2
    espec = np.maximum(np.bincount(shell.ravel(), weights=energy.ravel(), minlength=nshell), 1e-14)
    n = np.arange(nshell, dtype=np.float64)
    target = n**4 * np.exp(-2.0 * n * n / (k0 * k0))
    fac = np.sqrt(target / espec)[shell]
    u = np.real(np.fft.ifftn(uk * fac))
    v = np.real(np.fft.ifftn(vk * fac))
    w = np.real(np.fft.ifftn(wk * fac))
    return u, v, w


def make_dhit(nc: int, k0: float = 4.0, Mt: float = 0.3, Re_lambda: float = 72.0,
              gam: float = 1.4, rho0: float = 1.0, seed: int = 0) -> DhitCase:
    u, v, w = solenoidal_field(nc, k0, seed)
    p0 = rho0 / gam  # sound speed 1
    c0 = np.sqrt(gam * p0 / rho0)
    q = np.sqrt(np.mean(u * u + v * v + w * w))
    s = Mt * c0 / q
    u, v, w = u * s, v * s, w * s
    urms = Mt * c0 / np.sqrt(3.0)
    lam = 2.0 / k0
    mu0 = rho0 * urms * lam / Re_lambda
    t0 = lam / urms
    rho = np.full((nc, nc, nc), rho0)
    p = np.full((nc, nc, nc), p0)
    return DhitCase(nc=nc, u=u, v=v, w=w, rho=rho, p=p, gam=gam, rho0=rho0, Mt=Mt, Re=Re_lambda,
                    mu0=float(mu0), p0=float(p0), t0=float(t0), k0=k0, seed=seed)


def to_conservative_padded(case: DhitCase) -> np.ndarray:
    """The five conservative fields on the padded block (5, nt, nt, nt), ghosts
    filled periodically; the arithmetic of Initialize_DHIT (FlowField.cpp:97-102)."""
    nc = case.nc
    d, u, v, w, p = case.rho, case.u, case.v, case.w, case.p
    vsq = u * u + v * v + w * w
    W = np.empty((5, nc, nc, nc))
    W[0] = d
    W[1] = u * d
    W[2] = v * d
    W[3] = w * d
    W[4] = d * (p / (d * (case.gam - 1.0)) + 0.5 * vsq)
    return pad_periodic(W)


def pad_periodic(W: np.ndarray) -> np.ndarray:
    """(5, nc, nc, nc) interior -> (5, nt, nt, nt) with 3 periodic ghost layers."""
    return np.pad(W, ((0, 0), (3, 3), (3, 3), (3, 3)), mode="wrap")


def write_params(path: str, case: DhitCase) -> None:
    """InitialConditions/params: int n, then doubles gamma, rho0, Mt, Re, mu0,
    p0, t0 (FlowField.cpp:15-39)."""
    with open(path, "wb") as f:
        f.write(struct.pack("<i", case.nc))
        f.write(struct.pack("<7d", case.gam, case.rho0, case.Mt, case.Re, case.mu0, case.p0, case.t0))


def read_params(path: str) -> dict:
    with open(path, "rb") as f:
        n = struct.unpack("<i", f.read(4))[0]
        vals = struct.unpack("<7d", f.read(56))
    keys = ["gam", "rho0", "Mt", "Re", "mu0", "p0", "t0"]
    out = dict(zip(keys, vals))
    out["nc"] = n
    return out


def file_order(a: np.ndarray) -> np.ndarray:
    """[j, i, k] array -> the Init file's MATLAB order J = k*ny*nx + i*ny + j
    (FlowField.cpp:95)."""
    return np.ascontiguousarray(a.transpose(2, 1, 0)).ravel()


def particle_positions(n: int, seed: int) -> np.ndarray:
    """n seeded positions uniform in [0, 2 pi)^3 as (x0, y0, z0), the content of
    InitialConditions/unirand (read by locateParticles, update.cpp:1278-1284)."""
    rng = np.random.default_rng(seed)
    return rng.random((3, n)) * (2.0 * (np.arctan(1.0) * 4.0))


def write_case(casedir: str, case: DhitCase, slab_planes: int | None = None, all_slabs: bool = False,
               particles: int = 0, particle_seed: int = 0) -> None:
    """Write params, particleCount and Init000 (and, with particles > 0, the
    particles' initial positions in unirand: x0, y0, z0 of `particles` doubles
    each).  With slab_planes, the y-slabs of slab_planes planes are the blocks
    of an (nc/slab_planes) x 1 x 1 process grid: Init000 holds the first
    slab_planes y-planes (process (0,0,0)) and, with all_slabs, Init<a>00 holds
    slab a for every process a, the file each rank's Initialize_DHIT reads
    (FlowField.cpp:73-75)."""
    ic = os.path.join(casedir, "InitialConditions")
    os.makedirs(ic, exist_ok=True)
    write_params(os.path.join(ic, "params"), case)
    with open(os.path.join(ic, "particleCount"), "wb") as f:
        f.write(struct.pack("<i", particles))
    if particles > 0:
        with open(os.path.join(ic, "unirand"), "wb") as f:
            f.write(particle_positions(particles, particle_seed).astype("<f8").tobytes())
    if slab_planes and case.nc % slab_planes:
        raise ValueError(f"{slab_planes} planes do not divide nc = {case.nc}")
    nslab = case.nc // slab_planes if (slab_planes and all_slabs) else 1
    for a in range(nslab):
        sl = slice(a * slab_planes, (a + 1) * slab_planes) if slab_planes else slice(None)
        with open(os.path.join(ic, f"Init{a}00"), "wb") as f:
            for arr in (case.u, case.v, case.w, case.rho, case.p):
                f.write(file_order(np.ascontiguousarray(arr[sl])).astype("<f8").tobytes())


def read_init(casedir: str) -> tuple[dict, np.ndarray]:
    """Read params + Init000 back into (params, padded conservative W)."""
    prm = read_params(os.path.join(casedir, "InitialConditions", "params"))
    nc = prm["nc"]
    raw = np.fromfile(os.path.join(casedir, "InitialConditions", "Init000"), dtype="<f8")
    if raw.size != 5 * nc**3:
        raise ValueError(f"Init000 holds {raw.size} values, expected {5 * nc**3}")
    fields = [raw[q * nc**3:(q + 1) * nc**3].reshape(nc, nc, nc).transpose(2, 1, 0) for q in range(5)]
    u, v, w, d, p = fields
    gam = prm["gam"]
    vsq = u * u + v * v + w * w
    W = np.empty((5, nc, nc, nc))
    W[0] = d
    W[1] = u * d
    W[2] = v * d
    W[3] = w * d
    W[4] = d * (p / (d * (gam - 1.0)) + 0.5 * vsq)
    return prm, pad_periodic(W)
