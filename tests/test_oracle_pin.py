"""Pin the CPU oracle (oracle/gks_oracle.c) to the reference's own outputs.

The golden fixtures were produced by the reference's CPU path compiled from
its sources (tests/golden/make_golden.py).  The oracle restates the same
formulas in the same operation order and is built without FMA contraction, so
agreement is required bit for bit.
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN

import gks_ic


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_weno_matches_reference_bitwise(oracle):
    g = load("weno_ref.npz")
    wl, wr = oracle.weno(g["stencils"], float(g["gam"]))
    assert np.array_equal(wl, g["wl"])
    assert np.array_equal(wr, g["wr"])


def test_flux_matches_reference_bitwise(oracle):
    g = load("flux_ref.npz")
    F = oracle.flux(g["inputs"], float(g["gam"]), int(g["K"]), oracle.PR_FACTOR_CPU)
    assert np.array_equal(F, g["F"])


def _params16(oracle, g):
    return oracle.params(int(g["nc"]), 1.4, float(g["mu0"]), float(g["p0"]), 1.0, float(g["Mt"]), float(g["t0"]))


def test_step_matches_reference_bitwise_16(oracle):
    g = load("dhit16.npz")
    prm = _params16(oracle, g)
    W = gks_ic.pad_periodic(g["ic"])
    assert oracle.maxval(W, prm) == float(g["maxval"])
    dt = 0.5 * prm.dx / oracle.maxval(W, prm)
    assert dt == float(g["dt"])
    oracle.step(W, prm, dt, 1)
    assert np.array_equal(W[:, 3:-3, 3:-3, 3:-3], g["w1"])
    oracle.step(W, prm, dt, 9)
    assert np.array_equal(W[:, 3:-3, 3:-3, 3:-3], g["w10"])


def test_stats_history_matches_reference_16(oracle):
    g = load("dhit16.npz")
    prm = _params16(oracle, g)
    W = gks_ic.pad_periodic(g["ic"])
    dt = float(g["dt"])
    for s in range(11):
        st = oracle.stats(W, prm)
        ref = g["stats"][s]
        assert ref[0] == pytest.approx(s * dt / float(g["t0"]), rel=1e-12)
        assert np.array_equal(st[:8], ref[1:9])
        oracle.step(W, prm, dt, 1)


def test_printed_rms_columns_16(oracle):
    """Prms, Trms, Vrms are printed only (8 digits, update.cpp:779-780)."""
    g = load("dhit16.npz")
    prm = _params16(oracle, g)
    W = gks_ic.pad_periodic(g["ic"])
    oracle.step(W, prm, float(g["dt"]), 3)
    st = oracle.stats(W, prm)
    cols = [float(x) for x in str(g["lines"][3]).split()]
    np.testing.assert_allclose(st[8:11], cols[9:12], rtol=5e-8, atol=1e-20)


@pytest.mark.parametrize("nc", [32, 128])
def test_dhit_ic_is_the_reference_input(nc):
    """The committed reference outputs at 32^3 and 128^3 were made from these exact input bytes."""
    g = load(f"dhit{nc}.npz")
    import hashlib
    import tempfile

    case = gks_ic.make_dhit(nc, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=0)
    d = tempfile.mkdtemp()
    gks_ic.write_case(d, case)
    with open(os.path.join(d, "InitialConditions", "params"), "rb") as f:
        b = f.read()
    with open(os.path.join(d, "InitialConditions", "Init000"), "rb") as f:
        b += f.read()
    assert hashlib.sha256(b).hexdigest() == str(g["ic_sha256"])


def test_dhit32_ten_steps_match_reference(oracle):
    g = load("dhit32.npz")
    case = gks_ic.make_dhit(32, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=0)
    prm = oracle.params(32, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    W = gks_ic.to_conservative_padded(case)
    dt = 0.5 * prm.dx / oracle.maxval(W, prm)
    assert dt == float(g["dt"])
    oracle.step(W, prm, dt, 10)
    flat = W[:, 3:-3, 3:-3, 3:-3].reshape(5, -1)
    assert np.array_equal(flat[:, g["sample_idx"]], g["sample_w10"])
    assert np.array_equal(flat.sum(1), g["sum_w10"])


def _err(a, b):
    a = a.reshape(5, -1)
    b = b.reshape(5, -1)
    return np.abs(a - b).max(1) / np.abs(b).max(1)


def test_gpu_semantics_match_reference_gpu_path(oracle):
    """The oracle's reference-GPU mode (direct-energy WENO, no 1/Pr) against the
    reference's own GPU path run on a B200 (refgpu*.npz, make_golden_refgpu.py):
    CUDA's FMA contraction and math library against the C restatement, so the
    bar is the 1e-12 relative parity tolerance, not bit equality."""
    g = load("refgpu16.npz")
    case = gks_ic.make_dhit(16, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=1)
    prm = oracle.params(16, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0, pr_factor=oracle.PR_FACTOR_GPU,
                        flags=oracle.DIRECT_ENERGY)
    W = gks_ic.to_conservative_padded(case)
    dt = 0.5 * prm.dx / oracle.maxval(W, prm)
    assert dt == float(g["dt"])
    stats = [oracle.stats(W, prm)]
    oracle.step(W, prm, dt, 1)
    assert np.all(_err(W[:, 3:-3, 3:-3, 3:-3], g["w1"]) < 1e-12)
    for _ in range(9):
        stats.append(oracle.stats(W, prm))
        oracle.step(W, prm, dt, 1)
    stats.append(oracle.stats(W, prm))
    assert np.all(_err(W[:, 3:-3, 3:-3, 3:-3], g["w10"]) < 1e-12)
    np.testing.assert_allclose(np.array(stats)[:, :8], g["stats"][:, 1:9], rtol=1e-10, atol=1e-13)

    g = load("refgpu32.npz")
    case = gks_ic.make_dhit(32, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=0)
    prm = oracle.params(32, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0, pr_factor=oracle.PR_FACTOR_GPU,
                        flags=oracle.DIRECT_ENERGY)
    W = gks_ic.to_conservative_padded(case)
    oracle.step(W, prm, float(g["dt"]), 10)
    flat = W[:, 3:-3, 3:-3, 3:-3].reshape(5, -1)
    ref = g["sample_w10"]
    assert np.all(np.abs(flat[:, g["sample_idx"]] - ref).max(1) / np.abs(ref).max(1) < 1e-12)
    np.testing.assert_allclose(flat.sum(1), g["sum_w10"], rtol=1e-12, atol=1e-9)


def test_gpu_and_cpu_semantics_differ(oracle):
    """The two reference paths are different schemes: the CPU-mode oracle is far
    from the reference GPU output (so the test above is not vacuous)."""
    g = load("refgpu16.npz")
    case = gks_ic.make_dhit(16, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=1)
    prm = oracle.params(16, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    W = gks_ic.to_conservative_padded(case)
    oracle.step(W, prm, float(g["dt"]), 1)
    assert np.all(_err(W[:, 3:-3, 3:-3, 3:-3], g["w1"]) > 1e-4)


def test_known_answer_weno_exact_on_constant_and_linear(oracle):
    g = load("weno_ref.npz")
    st = g["stencils"]
    wl, wr = oracle.weno(st, 1.4)
    const = np.arange(len(st)) % 8 == 0
    for c in np.where(const)[0]:
        np.testing.assert_allclose(wl[c, :4], st[c, 2, :4], rtol=1e-14)
        np.testing.assert_allclose(wr[c, :4], st[c, 2, :4], rtol=1e-14)
    # a linear profile is reproduced by every candidate: the interface value is the midpoint
    x = np.arange(6) - 2.5
    s = np.zeros((1, 6, 5))
    s[0, :, 0] = 1.0 + 0.01 * x
    s[0, :, 1] = 0.3 + 0.02 * x
    s[0, :, 2] = -0.1 + 0.01 * x
    s[0, :, 3] = 0.05 * x
    s[0, :, 4] = 2.0 + 0.03 * x
    wl, wr = oracle.weno(s, 1.4, direct_energy=True)
    np.testing.assert_allclose(wl[0], s[0, 2] + 0.5 * (s[0, 3] - s[0, 2]), rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(wr[0], wl[0], rtol=1e-13, atol=1e-15)


def test_known_answer_uniform_flux_is_euler_flux(oracle):
    """Uniform state, zero slopes: F = dt * Euler flux as tau -> 0."""
    gam = 1.4
    rho, u, v, w, p = 1.1, 0.4, -0.2, 0.1, 0.8
    E = p / (gam - 1) + 0.5 * rho * (u * u + v * v + w * w)
    W = np.array([rho, rho * u, rho * v, rho * w, E])
    dt = 1e-2
    inp = np.concatenate([W, W, W, W, np.zeros(30), [1e-9, dt, 0.1]])[None]
    F = oracle.flux(inp, gam, 2, oracle.PR_FACTOR_CPU)[0]
    euler = np.array([rho * u, rho * u * u + p, rho * u * v, rho * u * w, u * (E + p)])
    np.testing.assert_allclose(F, dt * euler, rtol=1e-6)


def test_oracle_conserves_and_keeps_rest(oracle):
    g = load("dhit16.npz")
    prm = _params16(oracle, g)
    W = gks_ic.pad_periodic(g["ic"])
    s0 = W[:, 3:-3, 3:-3, 3:-3].reshape(5, -1).sum(1)
    oracle.step(W, prm, float(g["dt"]), 5)
    s1 = W[:, 3:-3, 3:-3, 3:-3].reshape(5, -1).sum(1)
    scale = np.abs(W[:, 3:-3, 3:-3, 3:-3]).reshape(5, -1).sum(1)
    assert np.all(np.abs(s1 - s0) <= 1e-13 * scale)
    # rest state stays at rest
    R = np.zeros_like(W)
    R[0] = 1.0
    R[4] = (1 / 1.4) / 0.4
    R0 = R.copy()
    oracle.step(R, prm, 0.05, 2)
    np.testing.assert_allclose(R, R0, rtol=0, atol=1e-15)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "ref_harness")),
                    reason="reference build absent")
def test_live_reference_agrees_on_a_fresh_case(oracle, tmp_path):
    """A case not in the fixtures, run through the reference binary and the oracle."""
    case = gks_ic.make_dhit(12, k0=3.0, Mt=0.4, Re_lambda=50.0, seed=11)
    gks_ic.write_case(str(tmp_path), case)
    r = oracle.ref_run(str(tmp_path), 3, 0.5, [3], outdir=str(tmp_path / "out"))
    W = gks_ic.to_conservative_padded(case)
    prm = oracle.params(12, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    oracle.step(W, prm, r["meta"]["dt"], 3)
    assert np.array_equal(W, r["dumps"][3])
