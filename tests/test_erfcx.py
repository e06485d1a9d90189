"""The half-space seed 0.5 erfc(|x|) of the flux (gks_device.cuh half_erfc_abs):
the generated coefficient table matches its generator, and the device
evaluation order -- correctly rounded reciprocal, Horner with fused
multiply-adds -- emulated exactly on the CPU is accurate against erfc in
40-digit arithmetic over the whole range where exp(-a^2) does not underflow."""
import os
import re
import sys
from fractions import Fraction

import numpy as np
import pytest

mp = pytest.importorskip("mpmath")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gkm-dns_b200", "csrc")


def header_coefficients():
    text = open(os.path.join(CSRC, "gks_erfcx.cuh")).read()
    K = float(re.search(r"kErfcxK = ([0-9.]+);", text).group(1))
    deg = int(re.search(r"kErfcxDeg = (\d+);", text).group(1))
    body = text[text.index("kErfcxC"):]
    body = body[body.index("{") + 1:body.index("}")]
    coef = [float(v) for v in body.replace("\n", " ").split(",") if v.strip()]
    assert len(coef) == deg + 1
    return K, coef


def fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def device_half_erfc_abs(x, ex, K, coef):
    """Bit-exact CPU restatement of half_erfc_abs (every operation rounded once)."""
    a = abs(x)
    r = float(Fraction(1) / Fraction(a + K))  # __drcp_rn
    t = (a - K) * r
    p = coef[-1]
    for c in reversed(coef[:-1]):
        p = fma(p, t, c)
    return (0.5 * ex) * p


def test_table_matches_generator():
    sys.path.insert(0, CSRC)
    try:
        import gen_erfcx
    finally:
        sys.path.pop(0)
    K, coef = header_coefficients()
    assert K == gen_erfcx.K
    assert coef == gen_erfcx.coefficients()


@pytest.mark.parametrize("lo,hi,n,tol", [(0.0, 6.0, 1500, 1.5e-15), (6.0, 26.0, 400, 4e-15)])
def test_half_erfc_accuracy(lo, hi, n, tol):
    mp.mp.dps = 40
    K, coef = header_coefficients()
    worst = 0.0
    for a in np.linspace(lo, hi, n):
        a = float(a)
        ex = float(mp.exp(-mp.mpf(a) ** 2))  # a correctly rounded exp(-a^2)
        for x in (a, -a):
            got = device_half_erfc_abs(x, ex, K, coef)
            want = 0.5 * mp.erfc(mp.mpf(a))
            worst = max(worst, float(abs(got - want) / want))
    assert worst <= tol, worst


def test_seed_both_signs():
    """0.5 erfc(x) for x < 0 is 1 - 0.5 erfc(|x|): check the sum rule and a few values."""
    mp.mp.dps = 40
    K, coef = header_coefficients()
    for x in (-3.0, -1.0, -0.25, 0.0, 0.25, 1.0, 3.0):
        ex = float(mp.exp(-mp.mpf(x) ** 2))
        tail = device_half_erfc_abs(x, ex, K, coef)
        h0 = tail if x >= 0 else 1.0 - tail
        assert abs(h0 - float(0.5 * mp.erfc(x))) <= 2e-16


def header_small_coefficients():
    text = open(os.path.join(CSRC, "gks_erfcx.cuh")).read()
    deg = int(re.search(r"kErfSmallDeg = (\d+);", text).group(1))
    body = text[text.index("kErfSmallC"):]
    body = body[body.index("{") + 1:body.index("}")]
    coef = [float(v) for v in body.replace("\n", " ").split(",") if v.strip()]
    assert len(coef) == deg + 1
    return coef


def device_half_erfc_pm(x, ex, K, coef, small):
    """Bit-exact CPU restatement of half_erfc_pm: (0.5 erfc(x), 0.5 erfc(-x))."""
    if abs(x) <= 1.0:
        s = x * x
        p = small[-1]
        for c in reversed(small[:-1]):
            p = fma(p, s, c)
        hx = 0.5 * x
        return fma(-hx, p, 0.5), fma(hx, p, 0.5)
    tail = device_half_erfc_abs(x, ex, K, coef)
    return (tail, 1.0 - tail) if x >= 0 else (1.0 - tail, tail)


def test_small_table_matches_generator():
    sys.path.insert(0, CSRC)
    try:
        import gen_erfcx
    finally:
        sys.path.pop(0)
    assert header_small_coefficients() == gen_erfcx.small_coefficients()


def test_seed_pair_accuracy_across_the_branch():
    """Both seeds over |x| <= 1 (the polynomial) and beyond (the erfcx form),
    including the switch at |x| = 1: within 1e-15 relative of 0.5 erfc."""
    mp.mp.dps = 40
    K, coef = header_coefficients()
    small = header_small_coefficients()
    worst = 0.0
    xs = list(np.linspace(-3.0, 3.0, 1201)) + [np.nextafter(1.0, 0), 1.0, np.nextafter(1.0, 2),
                                                -np.nextafter(1.0, 0), -1.0, -np.nextafter(1.0, 2), 0.0]
    for x in xs:
        x = float(x)
        ex = float(mp.exp(-mp.mpf(x) ** 2))
        hp, hm = device_half_erfc_pm(x, ex, K, coef, small)
        for got, arg in ((hp, x), (hm, -x)):
            want = 0.5 * mp.erfc(mp.mpf(arg))
            worst = max(worst, float(abs(got - want) / want))
    assert worst <= 1e-15, worst
