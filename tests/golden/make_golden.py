"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own CPU path (compiled from its sources into
oracle/_ref/ref_harness by oracle/Makefile) on seeded inputs and stores inputs
and outputs.  Needs the reference sources, so it runs only where they are
present; the fixtures it writes are committed and travel with the tests.

    python tests/golden/make_golden.py

Fixtures
  weno_ref.npz   ApplyWENO (update.cpp:502-625) on 400 stencils incl. edge cases
  flux_ref.npz   flux (GKMflux.cpp:11-215) on 400 interface states incl. edge cases
  dhit16.npz     16^3 DHIT (seed 1): IC, fields after 1 and 10 steps, stats history
  dhit32.npz     32^3 DHIT of the CPU configuration (k0 4, Mt 0.3, Re 72, seed 0,
                 CFL 0.5): 100-step stats history and printed lines, step-10 field
                 checksums and 4096 sampled cells
  dhit128.npz    128^3 (same physics, seed 0): 10-step field checksums, 8192 sampled
                 cells, stats history (python make_golden.py --c1; ~3 min of CPU)
  field8.npz     8^3 DHIT (seed 1, CFL 0.5): the reference's Results/Field text dump
                 (writeField, update.cpp:1305-1319), written once at the first step
                 with t >= t0 as Evolve does (python make_golden.py --field)
"""

import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gkm-dns_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import gks_ic  # noqa: E402
import pyoracle  # noqa: E402

GAM = 1.4


def cons(rho, u, v, w, p, gam=GAM):
    return np.stack([rho, rho * u, rho * v, rho * w, p / (gam - 1.0) + 0.5 * rho * (u * u + v * v + w * w)], -1)


def weno_stencils(rng, n=400):
    """(n, 6, 5) conservative stencils: random smooth, random rough, and edge cases."""
    out = []
    x = np.arange(6) - 2.5
    for c in range(n):
        kind = c % 8
        if kind == 0:    # constant state
            s = np.repeat(cons(*(rng.uniform(0.5, 1.5), *rng.normal(0, 0.3, 3), rng.uniform(0.4, 1.0)))[None], 6, 0)
        elif kind == 1:  # linear primitive profile
            g = rng.normal(0, 0.05, 5)
            rho = 1.0 + g[0] * x; u = 0.2 + g[1] * x; v = g[2] * x; w = -0.1 + g[3] * x; p = 0.7 + g[4] * x
            s = cons(rho, u, v, w, p)
        elif kind == 2:  # contact / shock-like jump between L and R
            a = cons(1.0, 0.1, 0.0, 0.0, 0.71)
            b = cons(0.4, -0.2, 0.1, 0.05, 0.3)
            s = np.where((x > 0)[:, None], b[None], a[None])
        elif kind == 3:  # tiny perturbations: smoothness indicators below eps
            base = cons(1.0, 0.3, -0.2, 0.1, 1 / GAM)
            s = base[None] * (1.0 + 1e-9 * rng.normal(size=(6, 5)))
        elif kind == 4:  # smooth sinusoid
            ph = rng.uniform(0, 6.3, 5)
            k = rng.uniform(0.2, 0.8)
            rho = 1 + 0.1 * np.sin(k * x + ph[0]); u = 0.3 * np.sin(k * x + ph[1]); v = 0.3 * np.sin(k * x + ph[2])
            w = 0.3 * np.sin(k * x + ph[3]); p = 1 / GAM + 0.05 * np.sin(k * x + ph[4])
            s = cons(rho, u, v, w, p)
        else:            # random turbulence-like cells
            rho = rng.uniform(0.8, 1.2, 6); u = rng.normal(0, 0.3, 6); v = rng.normal(0, 0.3, 6)
            w = rng.normal(0, 0.3, 6); p = rng.uniform(0.6, 0.8, 6)
            s = cons(rho, u, v, w, p)
        out.append(s)
    return np.array(out)


def flux_inputs(rng, n=400):
    """(n, 53) interface inputs: WL, WR, Wl, Wr, 6 slope vectors, tau, dt, dx."""
    rows = []
    for c in range(n):
        kind = c % 6
        dx = 2 * np.pi / rng.choice([32, 64, 128])
        dt = rng.uniform(0.2, 0.5) * dx / 1.5
        tau = rng.uniform(1e-4, 5e-3)
        if kind == 0:    # uniform state, zero slopes
            W = cons(1.0, rng.normal(0, 0.5), rng.normal(0, 0.3), rng.normal(0, 0.3), 1 / GAM)
            WL = WR = Wl = Wr = W
            D = np.zeros((6, 5))
        elif kind == 1:  # supersonic normal velocity (erfc tails)
            W = cons(1.0, rng.choice([-2.5, 2.5]), 0.1, -0.1, 1 / GAM)
            WL = WR = Wl = Wr = W
            D = rng.normal(0, 0.01, (6, 5))
        else:
            prim = lambda: (rng.uniform(0.8, 1.2), *rng.normal(0, 0.35, 3), rng.uniform(0.6, 0.8))  # noqa: E731
            WL = cons(*prim()); WR = cons(*prim())
            Wl = WL + (WR - WL) * rng.uniform(0.3, 0.7) + rng.normal(0, 0.01, 5) * np.array([1, .3, .3, .3, 1])
            Wr = WL + (WR - WL) * rng.uniform(0.3, 0.7) + rng.normal(0, 0.01, 5) * np.array([1, .3, .3, .3, 1])
            D = rng.normal(0, 0.5 if kind == 5 else 0.1, (6, 5))
        rows.append(np.concatenate([WL, WR, Wl, Wr, D.ravel(), [tau, dt, dx]]))
    return np.array(rows)


def dhit_run(nc, seed, nsteps, dumps, k0=4.0, Mt=0.3, Re=72.0):
    case = gks_ic.make_dhit(nc, k0=k0, Mt=Mt, Re_lambda=Re, seed=seed)
    d = tempfile.mkdtemp(prefix=f"golden{nc}_")
    gks_ic.write_case(d, case)
    r = pyoracle.ref_run(d, nsteps, 0.5, dumps)
    with open(os.path.join(d, "InitialConditions", "params"), "rb") as f:
        ph = f.read()
    with open(os.path.join(d, "InitialConditions", "Init000"), "rb") as f:
        ib = f.read()
    sha = hashlib.sha256(ph + ib).hexdigest()
    return case, r, sha


def interior(W):
    return np.ascontiguousarray(W[:, 3:-3, 3:-3, 3:-3])


def c1():
    """The 128^3 configuration, 10 steps through the reference."""
    case, r, sha = dhit_run(128, 0, 10, [10])
    w10 = interior(r["dumps"][10])
    srng = np.random.default_rng(11)
    sample = srng.integers(0, 128**3, 8192)
    flat = w10.reshape(5, -1)
    np.savez_compressed(
        os.path.join(HERE, "dhit128.npz"), stats=r["stats"], dt=r["meta"]["dt"], maxval=r["meta"]["maxVAL"],
        sample_idx=sample, sample_w10=flat[:, sample], sum_w10=flat.sum(1), sumsq_w10=(flat * flat).sum(1),
        mu0=case.mu0, p0=case.p0, t0=case.t0, Mt=case.Mt, seed=0, nc=128, ic_sha256=sha)


def field8():
    """The Results/Field dump of an 8^3 run that passes t = t0."""
    case = gks_ic.make_dhit(8, seed=1)
    d = tempfile.mkdtemp(prefix="golden8_")
    gks_ic.write_case(d, case)
    dt = pyoracle.ref_run(d, 1, 0.5, [], stats_on=False)["meta"]["dt"]
    nsteps = int(np.ceil(case.t0 / dt)) + 1
    r = pyoracle.ref_run(d, nsteps, 0.5, [], stats_on=False, field=True)
    name, text = r["field"]
    np.savez_compressed(os.path.join(HERE, "field8.npz"), name=name, text=np.frombuffer(text, dtype=np.uint8),
                        nsteps=nsteps, dt=dt, seed=1, nc=8)


def main():
    if not pyoracle.have_ref():
        pyoracle.build()
    if "--c1" in sys.argv:
        c1()
        return
    if "--field" in sys.argv:
        field8()
        return
    rng = np.random.default_rng(20240601)

    st = weno_stencils(rng)
    wl, wr = pyoracle.ref_weno(st, GAM)
    np.savez_compressed(os.path.join(HERE, "weno_ref.npz"), stencils=st, wl=wl, wr=wr, gam=GAM)

    fi = flux_inputs(rng)
    F = pyoracle.ref_flux(fi, GAM, 2)
    np.savez_compressed(os.path.join(HERE, "flux_ref.npz"), inputs=fi, F=F, gam=GAM, K=2)

    case, r, sha = dhit_run(16, 1, 10, [0, 1, 10])
    np.savez_compressed(
        os.path.join(HERE, "dhit16.npz"), ic=interior(r["dumps"][0]), w1=interior(r["dumps"][1]),
        w10=interior(r["dumps"][10]), stats=r["stats"], dt=r["meta"]["dt"], maxval=r["meta"]["maxVAL"],
        dt_ref_cfl=r["meta"]["dt_reference"], mu0=case.mu0, p0=case.p0, t0=case.t0, Mt=case.Mt, seed=1, nc=16,
        lines=np.array(r["stdout"]), ic_sha256=sha)

    case, r, sha = dhit_run(32, 0, 100, [10, 100])
    w10 = interior(r["dumps"][10])
    srng = np.random.default_rng(7)
    sample = srng.integers(0, 32**3, 4096)
    flat = w10.reshape(5, -1)
    np.savez_compressed(
        os.path.join(HERE, "dhit32.npz"), stats=r["stats"], lines=np.array(r["stdout"]), dt=r["meta"]["dt"],
        maxval=r["meta"]["maxVAL"], sample_idx=sample, sample_w10=flat[:, sample], sum_w10=flat.sum(1),
        sumsq_w10=(flat * flat).sum(1), sum_w100=interior(r["dumps"][100]).reshape(5, -1).sum(1),
        mu0=case.mu0, p0=case.p0, t0=case.t0, Mt=case.Mt, seed=0, nc=32, ic_sha256=sha)
    for fn in sorted(os.listdir(HERE)):
        if fn.endswith(".npz"):
            print(fn, os.path.getsize(os.path.join(HERE, fn)))


if __name__ == "__main__":
    main()
