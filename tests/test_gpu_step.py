"""GPU parity of the step, time step and diagnostics against the oracle.

Every call goes through the C ABI (include/gks_b200.h) via gks_b200.  The
reference (pinned bit for bit to the oracle, test_oracle_pin.py) defines the
answers: golden fixtures where they exist, the oracle run on the same input
otherwise.

Tolerances: the FP64 path must reproduce the reference to 1e-12 relative to
each conserved field's magnitude (max |W_gpu - W_ref| / max |W_ref| per
component) after 10 steps; diagnostics to 1e-10 relative.
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN

import gks_ic

pytestmark = pytest.mark.gpu

STEP_RTOL = 1e-12
STATS_RTOL = 1e-10


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def field_err(a, b):
    """Per-component max abs difference relative to the component's scale."""
    a = a.reshape(5, -1)
    b = b.reshape(5, -1)
    return np.abs(a - b).max(1) / np.abs(b).max(1)


def interior(W):
    return W[:, 3:-3, 3:-3, 3:-3]


def case16(g):
    class C:
        pass

    c = C()
    c.nc, c.gam, c.rho0, c.Mt, c.mu0, c.p0, c.t0 = 16, 1.4, 1.0, float(g["Mt"]), float(g["mu0"]), float(g["p0"]), float(g["t0"])
    c.K = 2
    c.T0 = c.p0 / (287.0 * c.rho0)
    return c


def test_timestep_is_bitwise_reference(gks):
    g = load("dhit16.npz")
    with gks.Solver(gks.phys_from_case(case16(g))) as s:
        s.upload(gks_ic.pad_periodic(g["ic"]))
        assert s.timestep(0.5) == float(g["dt"])
        assert s.timestep(0.02) == float(g["dt_ref_cfl"])


def test_fp64_step_matches_reference_16(gks):
    g = load("dhit16.npz")
    with gks.Solver(gks.phys_from_case(case16(g))) as s:
        s.upload(gks_ic.pad_periodic(g["ic"]))
        s.set_dt(float(g["dt"]))
        s.step(1)
        s.sync()
        e1 = field_err(interior(s.download()), g["w1"])
        s.step(9)
        s.sync()
        W = s.download()
    e10 = field_err(interior(W), g["w10"])
    assert np.all(e1 < STEP_RTOL), e1
    assert np.all(e10 < STEP_RTOL), e10
    # ghosts are the periodic image
    assert np.array_equal(W, gks_ic.pad_periodic(np.ascontiguousarray(interior(W))))


def test_fp64_step_matches_reference_32(gks, oracle):
    """The CPU configuration (32^3, k0 4, Mt 0.3, Re 72, seed 0): 10 steps."""
    g = load("dhit32.npz")
    case = gks_ic.make_dhit(32, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=0)
    W0 = gks_ic.to_conservative_padded(case)
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(W0)
        dt = s.timestep(0.5)
        assert dt == float(g["dt"])
        s.step(10)
        s.sync()
        W = interior(s.download()).reshape(5, -1)
    ref = g["sample_w10"]
    e = np.abs(W[:, g["sample_idx"]] - ref).max(1) / np.abs(ref).max(1)
    assert np.all(e < STEP_RTOL), e
    # and the whole field against the oracle
    prm = oracle.params(32, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    Wo = W0.copy()
    oracle.step(Wo, prm, dt, 10)
    assert np.all(field_err(W, interior(Wo)) < STEP_RTOL)


def test_fp64_stats_history_matches_reference_32(gks):
    """The CPU configuration (32^3, k0 4, Mt 0.3, Re_lambda 72, seed 0, CFL 0.5)
    for its full 100 steps: every step's statistics against the reference's
    PrintStats history (update.cpp:638-784; TKE, dissipation, skewness and
    kurtosis to 1e-10, the printed p / T / 1/rho rms columns to their 9 printed
    digits) and the step-100 field sums against the reference's."""
    g = load("dhit32.npz")
    case = gks_ic.make_dhit(32, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=0)
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(gks_ic.to_conservative_padded(case))
        dt = s.timestep(0.5)
        assert dt == float(g["dt"])
        hist = []
        for k in range(101):
            hist.append(s.stats_array())
            if k < 100:
                s.step(1)
        s.sync()
        W = interior(s.download()).reshape(5, -1)
    hist = np.array(hist)
    ref = g["stats"]
    assert ref.shape == (101, 9)
    np.testing.assert_allclose(np.arange(101) * dt / case.t0, ref[:, 0], rtol=1e-14, atol=0)
    np.testing.assert_allclose(hist[:, :8], ref[:, 1:9], rtol=STATS_RTOL, atol=1e-13)
    printed = np.array([[float(x) for x in str(line).split()] for line in g["lines"]])
    assert printed.shape == (101, 12)
    # at t = 0 pressure and density are uniform and their rms columns are round-off
    np.testing.assert_allclose(hist[1:, 8:11], printed[1:, 9:12], rtol=2e-8, atol=0)
    np.testing.assert_allclose(W.sum(1), g["sum_w100"], rtol=1e-12, atol=1e-9)


def test_fp64_step_matches_reference_128(gks):
    """128^3 (k0 4, Mt 0.3, Re 72, seed 0): 10 steps against the reference's
    own output (sampled cells, per-component sums and sums of squares)."""
    g = load("dhit128.npz")
    case = gks_ic.make_dhit(128, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=0)
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(gks_ic.to_conservative_padded(case))
        dt = s.timestep(0.5)
        assert dt == float(g["dt"])
        stats = [s.stats_array()]
        for _ in range(10):
            s.step(1)
            stats.append(s.stats_array())
        s.sync()
        W = interior(s.download()).reshape(5, -1)
    ref = g["sample_w10"]
    e = np.abs(W[:, g["sample_idx"]] - ref).max(1) / np.abs(ref).max(1)
    assert np.all(e < STEP_RTOL), e
    np.testing.assert_allclose(W.sum(1), g["sum_w10"], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose((W * W).sum(1), g["sumsq_w10"], rtol=1e-12)
    np.testing.assert_allclose(np.array(stats)[:, :8], g["stats"][:11, 1:9], rtol=STATS_RTOL, atol=1e-13)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_step_with_partial_segments_and_runs_matches_oracle(gks, oracle, prec):
    """40^3: two z segments per line (32 + 8 interfaces), window runs that the
    batch shortens to 8, both ends of every line wrapping; 3 steps against the
    oracle (FP64 to the parity tolerance, mixed to 1e-6)."""
    case = gks_ic.make_dhit(40, k0=4.0, Mt=0.4, Re_lambda=80.0, seed=5)
    W0 = gks_ic.to_conservative_padded(case)
    with gks.Solver(gks.phys_from_case(case), gks.FP64 if prec == "fp64" else gks.MIXED) as s:
        s.upload(W0)
        dt = s.timestep(0.5)
        s.step(3)
        s.sync()
        W = interior(s.download()).reshape(5, -1)
    prm = oracle.params(40, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    Wo = W0.copy()
    oracle.step(Wo, prm, dt, 3)
    assert np.all(field_err(W, interior(Wo)) < (STEP_RTOL if prec == "fp64" else 1e-6))


@pytest.mark.parametrize("nc", [16, 32])
def test_gpu_semantics_match_reference_gpu_path(gks, nc):
    """GKS_DIRECT_ENERGY with pr_factor 1 against the reference's own GPU path
    (GPUupdate.cu built for sm_100a and run on a B200, refgpu*.npz): 10 steps."""
    g = load(f"refgpu{nc}.npz")
    case = gks_ic.make_dhit(nc, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=int(g["seed"]))
    phys = gks.phys_from_case(case, pr_factor=gks.PR_FACTOR_GPU)
    with gks.Solver(phys, gks.FP64, gks.DIRECT_ENERGY) as s:
        s.upload(gks_ic.to_conservative_padded(case))
        dt = s.timestep(0.5)
        assert dt == float(g["dt"])
        stats = [s.stats_array()]
        for _ in range(10):
            s.step(1)
            stats.append(s.stats_array())
        s.sync()
        W = interior(s.download()).reshape(5, -1)
    if nc == 16:
        assert np.all(field_err(W, g["w10"]) < STEP_RTOL)
    else:
        ref = g["sample_w10"]
        assert np.all(np.abs(W[:, g["sample_idx"]] - ref).max(1) / np.abs(ref).max(1) < STEP_RTOL)
        np.testing.assert_allclose(W.sum(1), g["sum_w10"], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(np.array(stats)[:, :8], g["stats"][:11, 1:9], rtol=STATS_RTOL, atol=1e-13)


def test_stats_history_matches_reference_16(gks):
    g = load("dhit16.npz")
    with gks.Solver(gks.phys_from_case(case16(g))) as s:
        s.upload(gks_ic.pad_periodic(g["ic"]))
        s.set_dt(float(g["dt"]))
        for k in range(11):
            st = s.stats_array()
            ref = g["stats"][k][1:9]
            np.testing.assert_allclose(st[:8], ref, rtol=STATS_RTOL, atol=0)
            s.step(1)


def test_stats_match_oracle_all_columns(gks, oracle):
    case = gks_ic.make_dhit(20, k0=4.0, Mt=0.4, Re_lambda=80.0, seed=4)
    W = gks_ic.to_conservative_padded(case)
    prm = oracle.params(20, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(W)
        dt = s.timestep(0.5)
        s.step(4)
        got = s.stats_array()
    oracle.step(W, prm, dt, 4)
    ref = oracle.stats(W, prm)
    np.testing.assert_allclose(got, ref, rtol=STATS_RTOL, atol=1e-300)


def analytic_case(nc, seed):
    """A smooth periodic field with seeded noise, quick to build at any size:
    density, velocity and pressure from a few integer-wavenumber modes."""
    class C:
        pass

    c = C()
    c.nc, c.gam, c.rho0, c.Mt, c.mu0, c.p0, c.t0, c.K = nc, 1.4, 1.0, 0.4, 2e-3, 1 / 1.4, 1.0, 2
    c.T0 = c.p0 / (287.0 * c.rho0)
    x = (np.arange(nc) + 0.5) * (2 * np.pi / nc)
    Y, X, Z = x[:, None, None], x[None, :, None], x[None, None, :]  # index order (j, i, k)
    rng = np.random.default_rng(seed)
    noise = lambda: 1e-3 * rng.standard_normal((nc, nc, nc))  # noqa: E731
    rho = 1.0 + 0.05 * np.sin(X + 2 * Y) * np.cos(Z) + noise()
    # each velocity component has a skewed derivative along its own axis
    u = 0.3 * (np.sin(X) + 0.4 * np.sin(2 * X + 0.3)) + 0.1 * np.cos(Y + 1.0) * np.sin(2 * Z) + noise()
    v = 0.25 * (np.sin(Y) + 0.5 * np.sin(2 * Y + 1.0)) + 0.1 * np.cos(2 * X - Z) + noise()
    w = 0.2 * (np.sin(Z) + 0.6 * np.sin(2 * Z + 0.7)) - 0.1 * np.sin(X + Y) + noise()
    p = c.p0 * (1.0 + 0.1 * np.cos(X + Y + Z)) + noise()
    W = np.stack([rho, rho * u, rho * v, rho * w, p / (c.gam - 1) + 0.5 * rho * (u * u + v * v + w * w)])
    return c, gks_ic.pad_periodic(W)


@pytest.mark.parametrize("nc", [160, 283])
def test_stats_line_length_classes_match_oracle(gks, oracle, nc):
    """The statistics' spline kernel picks its nodes per lane from the line
    length nt = nc + 6 (5 up to nt = 160, 9 up to 288, 17 up to 544): 160^3
    and 283^3 take the 9- and 17-node forms that the smaller tests do not
    reach; every column against the oracle to 1e-10."""
    case, W = analytic_case(nc, seed=nc)
    prm = oracle.params(nc, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(W)
        got = s.stats_array()
    ref = oracle.stats(W, prm)
    np.testing.assert_allclose(got, ref, rtol=STATS_RTOL, atol=1e-300)


@pytest.mark.parametrize("variant", ["fix_zsweep", "direct_energy", "gpu_prandtl", "power_law"])
def test_variants_match_oracle(gks, oracle, variant):
    case = gks_ic.make_dhit(16, k0=4.0, Mt=0.5, Re_lambda=60.0, seed=9)
    W = gks_ic.to_conservative_padded(case)
    flags, oflags, law, prf = 0, 0, gks.VISC_SUTHERLAND, gks.PR_FACTOR_CPU
    if variant == "fix_zsweep":
        flags, oflags = gks.FIX_ZSWEEP, oracle.FIX_ZSWEEP
    elif variant == "direct_energy":
        flags, oflags = gks.DIRECT_ENERGY, oracle.DIRECT_ENERGY
    elif variant == "gpu_prandtl":
        prf = gks.PR_FACTOR_GPU
    else:
        law = gks.VISC_POWER
    phys = gks.phys_from_case(case, visc_law=law, visc_exp=0.76, pr_factor=prf)
    prm = oracle.params(16, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0, visc_law=law, visc_exp=0.76,
                        pr_factor=prf, flags=oflags)
    with gks.Solver(phys, gks.FP64, flags) as s:
        s.upload(W)
        dt = s.timestep(0.5)
        s.step(3)
        s.sync()
        got = interior(s.download())
    oracle.step(W, prm, dt, 3)
    assert np.all(field_err(got, interior(W)) < STEP_RTOL)


def test_zsweep_fix_changes_the_answer(gks):
    case = gks_ic.make_dhit(16, k0=4.0, Mt=0.5, seed=9)
    W = gks_ic.to_conservative_padded(case)
    out = []
    for flags in (0, gks.FIX_ZSWEEP):
        with gks.Solver(gks.phys_from_case(case), gks.FP64, flags) as s:
            s.upload(W)
            s.timestep(0.5)
            s.step(2)
            s.sync()
            out.append(s.download())
    assert field_err(out[0], out[1]).max() > 1e-8


def test_conservation_fp64_and_mixed(gks):
    case = gks_ic.make_dhit(24, k0=4.0, Mt=0.5, seed=2)
    W = gks_ic.to_conservative_padded(case)
    s0 = interior(W).reshape(5, -1).sum(1)
    scale = np.abs(interior(W)).reshape(5, -1).sum(1)
    for prec in (gks.FP64, gks.MIXED):
        with gks.Solver(gks.phys_from_case(case), prec) as s:
            s.upload(W)
            s.timestep(0.5)
            s.step(20)
            s.sync()
            s1 = interior(s.download()).reshape(5, -1).sum(1)
        assert np.all(np.abs(s1 - s0) <= 1e-12 * scale), (prec, np.abs(s1 - s0) / scale)


def test_rest_state_stays_at_rest(gks):
    case = gks_ic.make_dhit(8, seed=0)
    W = np.zeros((5, 14, 14, 14))
    W[0] = 1.0
    W[4] = (1 / 1.4) / 0.4
    for prec in (gks.FP64, gks.MIXED):
        with gks.Solver(gks.phys_from_case(case), prec) as s:
            s.upload(W)
            s.set_dt(0.05)
            s.step(3)
            s.sync()
            np.testing.assert_allclose(s.download(), W, rtol=0, atol=1e-15)


def test_ensemble_equals_individual_runs(gks):
    """Fields of different sizes in one context advance exactly as alone."""
    cases = [gks_ic.make_dhit(n, k0=4.0, Mt=m, seed=sd) for n, m, sd in ((12, 0.3, 1), (16, 0.4, 2), (20, 0.2, 3))]
    for prec in (gks.FP64, gks.MIXED):
        alone = []
        dts = []
        for c in cases:
            with gks.Solver(gks.phys_from_case(c), prec) as s:
                s.upload(gks_ic.to_conservative_padded(c))
                dts.append(s.timestep(0.5))
                s.step(4)
                s.sync()
                alone.append(s.download())
        with gks.Solver([gks.phys_from_case(c) for c in cases], prec) as s:
            for f, c in enumerate(cases):
                s.upload(gks_ic.to_conservative_padded(c), f)
                assert s.timestep(0.5, f) == dts[f]
            s.step(4)
            s.sync()
            for f in range(len(cases)):
                assert np.array_equal(s.download(f), alone[f])


def test_autotuned_launches_give_identical_results(gks):
    case = gks_ic.make_dhit(24, k0=4.0, Mt=0.5, seed=8)
    W = gks_ic.to_conservative_padded(case)
    for prec in (gks.FP64, gks.MIXED):
        out = []
        for tune in (False, True):
            with gks.Solver(gks.phys_from_case(case), prec) as s:
                s.upload(W)
                s.timestep(0.5)
                if tune:
                    s.autotune(1)
                    cfg = s.launch_config()
                    assert all(v["grid"] >= 1 for v in cfg.values())
                s.step(3)
                s.sync()
                out.append(s.download())
        assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_every_kernel_variant_gives_identical_results(gks, prec):
    """Each register-cap variant of the reconstruction and flux kernels, and a
    one-block grid-stride launch, reproduce the default launch bit for bit."""
    case = gks_ic.make_dhit(24, k0=4.0, Mt=0.5, seed=8)
    W = gks_ic.to_conservative_padded(case)
    p = gks.FP64 if prec == "fp64" else gks.MIXED

    def run(pin):
        with gks.Solver(gks.phys_from_case(case), p) as s:
            s.upload(W)
            s.timestep(0.5)
            for kind, variant, grid in pin:
                for d in range(3):
                    s.set_launch(kind, d, variant, grid)
            s.step(3)
            s.sync()
            return s.download()

    base = run([])
    for kind, nvar in (("recon", 6), ("flux", 3)):
        for v in range(nvar):
            for grid in (0, 1):
                got = run([(kind, v, grid)])
                diff = np.abs(got - base).max()
                assert diff == 0.0, (prec, kind, v, grid, diff)
    with pytest.raises(gks.GksError):
        run([("flux", 3, 0)])


def test_mixed_tracks_fp64(gks):
    case = gks_ic.make_dhit(32, k0=4.0, Mt=0.5, Re_lambda=100.0, seed=0)
    W = gks_ic.to_conservative_padded(case)
    res = {}
    for prec in (gks.FP64, gks.MIXED):
        with gks.Solver(gks.phys_from_case(case), prec) as s:
            s.upload(W)
            s.timestep(0.5)
            s.step(20)
            s.sync()
            res[prec] = (s.download(), s.stats())
    e = field_err(res[gks.MIXED][0], res[gks.FP64][0])
    assert np.all(e < 1e-6), e
    for key in ("tke", "diss"):
        a, b = res[gks.MIXED][1][key], res[gks.FP64][1][key]
        assert abs(a - b) < 1e-5 * abs(b), (key, a, b)


def test_nonfinite_state_is_reported(gks):
    case = gks_ic.make_dhit(8, seed=0)
    W = gks_ic.to_conservative_padded(case)
    W[0, 5, 5, 5] = np.nan
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(W)
        with pytest.raises(gks.GksError) as ei:
            s.check()
        assert ei.value.code == -5


def near_vacuum_double_rarefaction(case):
    """An 8^3 field with one near-vacuum cell (rho 1e-3, p 1e-6) whose x
    neighbours move away from it at 3x the sound speed: the first step takes
    more mass out of the cell than it holds, so its density turns negative
    (-0.068 in the oracle), a finite but unphysical state."""
    W = gks_ic.to_conservative_padded(case)
    V = np.ascontiguousarray(W[:, 3:-3, 3:-3, 3:-3])
    gam = case.gam

    def put(j, i, k, rho, u, p):
        V[:, j, i, k] = [rho, rho * u, 0.0, 0.0, p / (gam - 1) + 0.5 * rho * u * u]

    put(4, 4, 4, 1e-3, 0.0, 1e-6)
    put(4, 3, 4, 1.0, -3.0, 1 / gam)
    put(4, 5, 4, 1.0, 3.0, 1 / gam)
    return gks_ic.pad_periodic(V)


def test_step_that_breaks_the_state_is_reported(gks, oracle):
    """The update kernel's error word: a step that leaves a non-positive density
    or pressure makes gks_sync return GKS_ENONFINITE (no GPU fault: the state is
    finite but unphysical), gks_check then finds it too, and the context keeps
    working after a fresh upload."""
    case = gks_ic.make_dhit(8, seed=0)
    bad = near_vacuum_double_rarefaction(case)
    # the checker agrees that one step breaks this state
    prm = oracle.params(8, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    dt = 0.5 * (2 * np.pi / 8) / oracle.maxval(bad, prm)
    ref = bad.copy()
    oracle.step(ref, prm, dt, 1)
    assert interior(ref)[0].min() < -1e-2
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(bad)
        s.check()  # the uploaded state itself is physical
        assert s.timestep(0.5) == dt
        s.step(1)
        with pytest.raises(gks.GksError) as ei:
            s.sync()
        assert ei.value.code == -5
        with pytest.raises(gks.GksError) as ei:
            s.check()
        assert ei.value.code == -5
        # the error word was cleared by the sync that reported it; a good state runs on
        good = gks_ic.to_conservative_padded(case)
        s.upload(good)
        s.check()
        s.timestep(0.5)
        s.step(2)
        s.sync()
        s.check()


def test_call_order_is_enforced(gks):
    case = gks_ic.make_dhit(8, seed=0)
    with gks.Solver(gks.phys_from_case(case)) as s:
        with pytest.raises(gks.GksError) as ei:
            s.step(1)
        assert ei.value.code == -4
        s.upload(gks_ic.to_conservative_padded(case))
        with pytest.raises(gks.GksError):
            s.step(1)  # no dt yet
        with pytest.raises(gks.GksError):
            s.set_dt(-1.0)
        with pytest.raises(ValueError):
            s.upload(np.zeros((5, 10, 10, 10)))


def test_grid_size_limits_are_enforced(gks, oracle):
    """The stencil wraps the periodic box at most once (nc >= 4) and cell indices
    are 32-bit (nc <= 1024): sizes outside are refused with GKS_EINVAL."""
    case = gks_ic.make_dhit(8, seed=0)
    for nc in (3, 1025):
        p = gks.phys_from_case(case)
        p.nc = nc
        with pytest.raises(gks.GksError) as ei:
            gks.Solver(p)
        assert ei.value.code == -1
    # the smallest box: every stencil wraps the periodic box, checked against the oracle
    small = gks_ic.make_dhit(4, k0=2.0, Mt=0.2, seed=1)
    W = gks_ic.to_conservative_padded(small)
    with gks.Solver(gks.phys_from_case(small)) as s:
        s.upload(W)
        dt = s.timestep(0.5)
        s.step(2)
        s.sync()
        got = s.download()
    prm = oracle.params(4, small.gam, small.mu0, small.p0, 1.0, small.Mt, small.t0)
    ref = W.copy()
    oracle.step(ref, prm, dt, 2)
    err = np.abs(got - ref).reshape(5, -1).max(1) / np.abs(ref).reshape(5, -1).max(1)
    assert np.all(err < 1e-12), err


def test_mixed_accuracy_to_two_eddy_times(gks):
    """Mixed vs FP64 at t/t0 = 2 (64^3, Mt 0.5, Re_lambda 100): KE and dissipation
    within 1e-5 relative, the precision target of the mixed path."""
    case = gks_ic.make_dhit(64, k0=4.0, Mt=0.5, Re_lambda=100.0, seed=0)
    W = gks_ic.to_conservative_padded(case)
    out, tke0 = {}, None
    for prec in (gks.FP64, gks.MIXED):
        with gks.Solver(gks.phys_from_case(case), prec) as s:
            s.upload(W)
            tke0 = s.stats()["tke"]
            dt = s.timestep(0.5)
            n = int(np.ceil(2.0 * case.t0 / dt))
            s.step(n)
            s.sync()
            out[prec] = s.stats()
    for key in ("tke", "diss"):
        a, b = out[gks.MIXED][key], out[gks.FP64][key]
        assert abs(a - b) < 1e-5 * abs(b), (key, a, b)
    assert out[gks.FP64]["tke"] < 0.9 * tke0  # the turbulence decayed
