"""GPU parity of the Lagrangian particles (gks_particles_*) against the oracle.

The reference's tracker (ParticleTrack.cpp, update.cpp:1082-1303) builds
einspline natural cubic B-splines of the primitives over the padded block,
evaluates value and gradient at each particle, moves the particles by
forward Euler and averages GetParticleStats' quantities.  The oracle restates
that (pinned to scipy's natural cubic spline in test_particles_oracle.py);
the device path computes every particle quantity in the oracle's operation
order, so records must agree bit for bit, and the statistics -- summed in a
different order -- to 1e-12 relative to the sum of magnitudes.
"""

import numpy as np
import pytest

import gks_ic

pytestmark = pytest.mark.gpu

TWO_PI = 2 * np.arctan(1.0) * 4.0


def setup(nc, seed, n, Mt=0.3):
    case = gks_ic.make_dhit(nc, k0=4.0, Mt=Mt, Re_lambda=72.0, seed=seed)
    W = gks_ic.to_conservative_padded(case)
    rng = np.random.default_rng(seed + 100)
    x0, y0, z0 = (rng.random(n) * TWO_PI for _ in range(3))
    return case, W, x0, y0, z0


def oracle_records(oracle, case, W, x0, y0, z0):
    prm = oracle.params(case.nc, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    rec = np.zeros((oracle.PREC_FIELDS, x0.size))
    rec[0], rec[1], rec[2] = y0, x0, z0
    return prm, oracle.particle_props(W, prm, rec)


def stats_close(got, rec, want):
    """GetParticleStats' means: the sums' order differs, so compare to the
    scale of the summed magnitudes."""
    U = rec[4:7]
    dudx, dwdz = rec[12], rec[19]
    scale = [np.mean((U**2).sum(0)), got[1], np.mean(dudx**2), np.mean(np.abs(dudx) ** 3), np.mean(dwdz**2),
             np.mean(np.abs(dwdz) ** 3)]
    for s in range(6):
        assert abs(got[s] - want[s]) <= 1e-12 * scale[s], (s, got[s], want[s])
    assert abs(got[6] - want[6]) <= 1e-10 * abs(want[6])
    assert abs(got[7] - want[7]) <= 1e-10 * abs(want[7])
    assert got[8] == want[8]


@pytest.mark.parametrize("nc,n", [(16, 3000), (24, 5000), (37, 4096)])
def test_particles_match_oracle(gks, oracle, nc, n):
    case, W, x0, y0, z0 = setup(nc, nc, n)
    prm, want = oracle_records(oracle, case, W, x0, y0, z0)
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(W)
        dt = s.timestep(0.5)
        s.particles_locate(x0, y0, z0)
        fresh = s.particles_get()
        assert np.array_equal(fresh[0:3], np.stack([y0, x0, z0])) and not fresh[3:].any()
        s.particles_props()
        got = s.particles_get()
        assert np.array_equal(got, want)
        stats_close(s.particles_stats(), want, oracle.particle_stats(want))
        # one particle step with the interpolated velocity, then the field's
        # step and the properties at the new positions
        s.particles_track(dt)
        oracle.particle_track(want, dt)
        assert np.array_equal(s.particles_get(), want)
        s.step(1)
        s.particles_props()
        W1 = W.copy()
        oracle.step(W1, prm, dt, 1)
        oracle.particle_props(W1, prm, want)
        got = s.particles_get()
        # the field after one device step differs from the oracle's by rounding
        # (step parity ~1e-15); properties follow to the same order
        scale = np.abs(want).max(1, keepdims=True)
        assert np.all(np.abs(got - want) <= 1e-12 * scale)


def test_particles_at_the_domain_edges(gks, oracle):
    """Positions exactly at 0 and 2 pi (the ends of the tracked range) and
    particles carried across the periodic boundary."""
    nc = 20
    case, W, _, _, _ = setup(nc, 4, 1)
    edge = np.array([0.0, TWO_PI, 0.0, TWO_PI, 1e-300, TWO_PI - 1e-15, np.pi])
    x0, y0, z0 = edge, edge[::-1].copy(), np.roll(edge, 2)
    prm, want = oracle_records(oracle, case, W, x0, y0, z0)
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(W)
        s.particles_locate(x0, y0, z0)
        s.particles_props()
        assert np.array_equal(s.particles_get(), want)
        for dt in (0.7, -1.3, 2.0):  # large steps cross the boundary either way
            s.particles_track(dt)
            oracle.particle_track(want, dt)
            got = s.particles_get()
            assert np.array_equal(got, want)
            assert np.all((got[0:3] >= 0) & (got[0:3] <= TWO_PI))


def test_particles_errors_and_state(gks):
    nc = 16
    case, W, x0, y0, z0 = setup(nc, 2, 10)
    with gks.Solver(gks.phys_from_case(case)) as s:
        for call in (lambda: s.particles_props(), lambda: s.particles_track(0.1), lambda: s.particles_stats()):
            with pytest.raises(gks.GksError) as ei:
                call()
            assert ei.value.code == -4  # GKS_ESTATE: before gks_particles_locate
        s.particles_locate(x0, y0, z0)
        with pytest.raises(gks.GksError) as ei:
            s.particles_props()
        assert ei.value.code == -4  # before upload
        bad = x0.copy()
        bad[3] = np.nan
        with pytest.raises(gks.GksError) as ei:
            s.particles_locate(bad, y0, z0)
        assert ei.value.code == -1
        with pytest.raises(gks.GksError) as ei:
            s.particles_track(np.inf)
        assert ei.value.code == -1
        # a new set replaces the old one, of another size
        s.upload(W)
        s.particles_locate(x0[:4], y0[:4], z0[:4])
        s.particles_props()
        assert s.particles_get().shape == (gks.PREC_FIELDS, 4)
    # a y-slab is not a whole periodic field
    with gks.Solver(gks.phys_from_case(case), slab=(8, 0)) as s:
        with pytest.raises(gks.GksError) as ei:
            s.particles_locate(x0, y0, z0)
        assert ei.value.code == -1


def test_particles_at_256_follow_a_uniform_stream(gks):
    """At the bench's 256^3 size with a million particles: in a uniform flow
    (constant density, velocity and pressure) the spline reproduces the
    constants and zero gradients, and a track moves every particle by U dt."""
    nc = 256
    n = 1 << 20
    case = gks_ic.make_dhit(16, k0=4.0, Mt=0.3, seed=0)
    phys = gks.phys_from_case(case)
    phys.nc = nc
    nt = nc + 6
    U = (0.3, -0.2, 0.1)
    p0 = 1.0 / 1.4
    W = np.empty((5, nt, nt, nt))
    W[0] = 1.0
    W[1], W[2], W[3] = U
    W[4] = p0 / 0.4 + 0.5 * sum(u * u for u in U)
    rng = np.random.default_rng(9)
    x0, y0, z0 = (rng.random(n) * TWO_PI for _ in range(3))
    with gks.Solver(phys) as s:
        s.upload(W)
        s.particles_locate(x0, y0, z0)
        s.particles_props()
        rec = s.particles_get()
        np.testing.assert_allclose(rec[3], 1.0, rtol=1e-13)
        for q in range(3):
            np.testing.assert_allclose(rec[4 + q], U[q], rtol=1e-12)
        np.testing.assert_allclose(rec[7], p0, rtol=1e-12)
        assert np.abs(rec[8:23]).max() < 1e-9
        dt = 0.01
        s.particles_track(dt)
        got = s.particles_get()
        want = np.stack([y0 + rec[5] * dt, x0 + rec[4] * dt, z0 + rec[6] * dt])
        want = np.where(want > TWO_PI, want - TWO_PI, want)
        want = np.where(want < 0, TWO_PI + want, want)
        assert np.array_equal(got[0:3], want)
        st = s.particles_stats()
        np.testing.assert_allclose(st[0], sum(u * u for u in U), rtol=1e-12)
        assert st[8] == n


def test_particles_on_an_ensemble_field_and_after_the_host_step(gks, oracle):
    """Particles belong to one field of a context: on the second field of an
    ensemble they see that field only; after gks_evolve (the pipelined host
    step, which swaps the field's state buffers) they see the new state."""
    cases = [setup(nc, nc + 50, 700) for nc in (18, 26)]
    with gks.Solver([gks.phys_from_case(c[0]) for c in cases]) as s:
        for f, (case, W, *_) in enumerate(cases):
            s.upload(W, f)
        case, W, x0, y0, z0 = cases[1]
        s.particles_locate(x0, y0, z0, f=1)
        s.particles_props(f=1)
        _, want = oracle_records(oracle, case, W, x0, y0, z0)
        assert np.array_equal(s.particles_get(f=1), want)
        with pytest.raises(gks.GksError) as ei:
            s.particles_props(f=0)  # field 0 has no particles
        assert ei.value.code == -4
    case, W, x0, y0, z0 = setup(32, 8, 900)
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(W)
        dt = s.timestep(0.5)
        host = W.copy()
        s.evolve(host)  # one field, one step: the slab-pipelined form
        s.particles_locate(x0, y0, z0)
        s.particles_props()
        _, want = oracle_records(oracle, case, host, x0, y0, z0)  # host: the new state, ghosts filled
        assert np.array_equal(s.particles_get(), want)


def test_driver_tracks_particles_like_the_oracle(tmp_path, oracle):
    """gks_dns --particles: every step the particles' properties from the
    current state, GetParticleStats' line, a move by dt, then the field's
    step -- the same sequence run by the oracle on the same case."""
    import os
    import subprocess

    from conftest import PKG

    nc, n, steps = 16, 400, 3
    case = gks_ic.make_dhit(nc, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=5)
    gks_ic.write_case(str(tmp_path), case, particles=n, particle_seed=9)
    r = subprocess.run([os.path.join(PKG, "driver", "gks_dns"), "--case", str(tmp_path), "--cfl", "0.5", "--steps",
                        str(steps), "--no-field", "--particles"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = [[float(x) for x in ln.split()[1:]] for ln in r.stdout.splitlines() if ln.startswith("particles ")]
    assert len(got) == steps + 1
    _, W = gks_ic.read_init(str(tmp_path))
    prm = oracle.params(nc, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    dt = 0.5 * prm.dx / oracle.maxval(W, prm)
    x0, y0, z0 = gks_ic.particle_positions(n, 9)
    rec = np.zeros((oracle.PREC_FIELDS, n))
    rec[0], rec[1], rec[2] = y0, x0, z0
    for s in range(steps + 1):
        oracle.particle_props(W, prm, rec)
        st = oracle.particle_stats(rec)
        want = [st[0], st[1], st[6], st[7], st[8]]
        np.testing.assert_allclose(got[s][1:], want, rtol=1e-9)
        if s < steps:
            oracle.particle_track(rec, dt)
            oracle.step(W, prm, dt, 1)
