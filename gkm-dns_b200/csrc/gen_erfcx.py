"""Generate gks_erfcx.cuh: the coefficients of the scaled complementary error
function erfcx(a) = exp(a^2) erfc(a), a >= 0, used for the half-space seeds of
the flux (0.5 erfc(-+ sqrt(lambda) U) next to exp(-lambda U^2), weno/src/GKMflux.cpp:48-66).

Method: the map t = (a - K) / (a + K) takes [0, inf) onto [-1, 1) (Shepherd and
Laframboise, "Chebyshev approximation of (1 + 2x) exp(x^2) erfc x in
0 <= x < inf", Math. Comp. 36 (1981) 249-253, use the same map).  erfcx is
analytic in t on [-1, 1] (near t = 1 it is (1 - t) times an analytic function of
1/a), so its Chebyshev interpolant in t converges geometrically.  The
interpolant of degree N at the N + 1 Chebyshev points of the first kind is
computed in 40-digit arithmetic (mpmath) and written out in monomial form for a
Horner evaluation in double.  K = 3 and N = 24 give a double-evaluation
relative error of 4.3e-16 for a <= 6, 7.3e-16 for a <= 12 and 1.6e-15 for
a <= 27 (beyond that exp(-a^2) underflows and the product is 0).

For |x| <= 1, where nearly every interface of a turbulent field lies, the
seeds come without a reciprocal from erf(x) = x P(x^2): P is the Chebyshev
interpolant of erf(a)/a in s = a^2 on [0, 1], degree NS = 11 in s (its next
Chebyshev coefficient is 4e-16 of the function), written in monomial form in s
(the coefficients alternate and decrease, so Horner in s is stable); its
double evaluation is accurate to 2.2e-16 relative in erf and 6.1e-16 in
0.5 erfc(x) = 0.5 - 0.5 x P(x^2).

Run:  python gen_erfcx.py  (writes gks_erfcx.cuh beside this file).
"""
import os

import mpmath as mp

K = 3
N = 24
NS = 11  # degree in s = a^2 of the small-argument erf polynomial (a <= 1)


def erfcx_of_t(t):
    if t >= 1:
        return mp.mpf(0)
    a = K * (1 + t) / (1 - t)
    return mp.erfc(a) * mp.exp(a * a)


def chebyshev_coefficients(fun, n):
    nodes = [mp.cos(mp.pi * (k + mp.mpf(1) / 2) / (n + 1)) for k in range(n + 1)]
    vals = [fun(x) for x in nodes]
    c = []
    for j in range(n + 1):
        s = sum(vals[k] * mp.cos(mp.pi * j * (k + mp.mpf(1) / 2) / (n + 1)) for k in range(n + 1))
        c.append(2 * s / (n + 1))
    c[0] /= 2
    return c


def to_monomial(c):
    n = len(c) - 1
    T = [[mp.mpf(1)], [mp.mpf(0), mp.mpf(1)]]
    for k in range(2, n + 1):
        a = [mp.mpf(0)] + [2 * x for x in T[k - 1]]
        b = T[k - 2] + [mp.mpf(0)] * (len(a) - len(T[k - 2]))
        T.append([x - y for x, y in zip(a, b)])
    m = [mp.mpf(0)] * (n + 1)
    for j in range(n + 1):
        for i, x in enumerate(T[j]):
            m[i] += c[j] * x
    return m


def coefficients():
    mp.mp.dps = 40
    return [float(x) for x in to_monomial(chebyshev_coefficients(erfcx_of_t, N))]


def erf_over_a(s):
    """erf(a) / a as a function of s = a^2 (2 / sqrt(pi) at s = 0)."""
    if s == 0:
        return 2 / mp.sqrt(mp.pi)
    a = mp.sqrt(s)
    return mp.erf(a) / a


def small_coefficients():
    """Monomial coefficients in s of the degree-NS Chebyshev interpolant of
    erf(a)/a on s in [0, 1] (Chebyshev variable t = 2 s - 1)."""
    mp.mp.dps = 40
    m_t = to_monomial(chebyshev_coefficients(lambda t: erf_over_a((t + 1) / 2), NS))
    m_s = [mp.mpf(0)] * (NS + 1)
    for i, x in enumerate(m_t):  # (2 s - 1)^i
        for k in range(i + 1):
            m_s[k] += x * mp.binomial(i, k) * mp.mpf(2) ** k * mp.mpf(-1) ** (i - k)
    return [float(x) for x in m_s]


def main():
    coef = coefficients()
    lines = [
        "// Generated by gen_erfcx.py (Chebyshev interpolant of erfcx(a) = exp(a^2) erfc(a)",
        "// in t = (a - %d) / (a + %d), degree %d, monomial form); do not edit." % (K, K, N),
        "#pragma once",
        "",
        "namespace gks {",
        "",
        "constexpr double kErfcxK = %d.0;" % K,
        "constexpr int kErfcxDeg = %d;" % N,
        "__device__ constexpr double kErfcxC[kErfcxDeg + 1] = {",
    ]
    for x in coef:
        lines.append("    %s," % repr(x))
    lines += ["};", "",
              "// erf(a) / a = P(a^2) on a <= 1: Chebyshev interpolant in s = a^2 of degree %d," % NS,
              "// monomial form in s.",
              "constexpr int kErfSmallDeg = %d;" % NS,
              "__device__ constexpr double kErfSmallC[kErfSmallDeg + 1] = {"]
    for x in small_coefficients():
        lines.append("    %s," % repr(x))
    lines += ["};", "", "} // namespace gks", ""]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gks_erfcx.cuh")
    with open(out, "w") as fh:
        fh.write("\n".join(lines))
    print("wrote", out)


if __name__ == "__main__":
    main()
