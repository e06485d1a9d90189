// Device math shared by the WENO-GKS kernels: WENO-SYMOO reconstruction
// (weno/src/update.cpp:502-625), the 1-D Maxwellian moment tables
// (weno/src/GKMflux.cpp:48-66), conservative -> primitive conversion
// (GKMflux.cpp:301-308) and the arithmetic helpers the flux (gks_flux.cuh)
// is written with.  The algebra is the reference's; the evaluation order is
// this file's own (one reciprocal per WENO side instead of eight divisions),
// so results agree with the reference to rounding, not bit for bit.  Every
// fused multiply-add is written out (the kernels are compiled without
// implicit contraction), so results do not depend on how the compiler
// schedules a particular register-cap variant.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include <type_traits>

#include "gks_erfcx.cuh"

namespace gks {

constexpr double kPi = 3.141592653589793;  // atan(1)*4, param.h:14
constexpr double kWenoEps = 1e-10;        // param.h:15

template <typename T> __device__ __forceinline__ T rcp(T x);
template <> __device__ __forceinline__ double rcp<double>(double x) { return __drcp_rn(x); }
template <> __device__ __forceinline__ float rcp<float>(float x) { return __frcp_rn(x); }

// Two FP32 lanes advanced by one paired instruction (f32x2 add/mul/fma of
// sm_100): the mixed flux runs two structurally identical moment evaluations
// (left and right Maxwellian, or two mirror-image equilibrium terms) as the
// .x and .y lanes of one instruction stream.
struct f2 {
    float2 v;
    f2() = default;
    __device__ __forceinline__ f2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ f2(float a, float b) : v(make_float2(a, b)) {}
};
__device__ __forceinline__ f2 operator+(f2 a, f2 b) { f2 r; r.v = __fadd2_rn(a.v, b.v); return r; }
__device__ __forceinline__ f2 operator*(f2 a, f2 b) { f2 r; r.v = __fmul2_rn(a.v, b.v); return r; }
__device__ __forceinline__ f2 operator-(f2 a, f2 b) { f2 r; r.v = __ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v); return r; }
__device__ __forceinline__ f2 operator-(f2 a) { f2 r; r.v = __fmul2_rn(a.v, make_float2(-1.f, -1.f)); return r; }
__device__ __forceinline__ f2 &operator+=(f2 &a, f2 b) { a = a + b; return a; }
__device__ __forceinline__ f2 &operator-=(f2 &a, f2 b) { a = a - b; return a; }
__device__ __forceinline__ f2 &operator*=(f2 &a, f2 b) { a = a * b; return a; }

// a*b + c with one rounding, for every arithmetic type used here.
__device__ __forceinline__ double fmaT(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fmaT(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ f2 fmaT(f2 a, f2 b, f2 c) { f2 r; r.v = __ffma2_rn(a.v, b.v, c.v); return r; }

template <> __device__ __forceinline__ f2 rcp<f2>(f2 x) { return f2(__frcp_rn(x.v.x), __frcp_rn(x.v.y)); }
__device__ __forceinline__ double fmaxT(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float fmaxT(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ f2 fmaxT(f2 a, f2 b) { return f2(fmaxf(a.v.x, b.v.x), fmaxf(a.v.y, b.v.y)); }

// A constant in type T (rounded once from its double value).
template <typename T> __device__ __forceinline__ constexpr T cst(double x) { return T(x); }
template <> __device__ __forceinline__ f2 cst<f2>(double x) { return f2(float(x)); }

// ---------------------------------------------------------------------------
// WENO-SYMOO on one scalar 6-point stencil (update.cpp:505-557): four cubic
// candidates per side, linear weights 1/20, 9/20, 9/20, 1/20, the fourth
// smoothness indicator replaced by the largest of the four, alpha = g/(eps+IS).
// The normalised weights are formed with one reciprocal per side (in double,
// one for both sides of an interface, see weno_pair):
// w_r = g_r prod_{s!=r} d_s / sum_t g_t prod_{s!=t} d_s, d = eps + IS.
// ---------------------------------------------------------------------------
// One side seen from (a, b, c | d, e, f): candidates on {a,b,c}, {b,c,d},
// {c,d,e}, {d,e,f}; q0..q3 are 13/12 of the squared second differences of
// those stencils, which both sides share.
template <typename T>
__device__ __forceinline__ void weno_side_nd(T a, T b, T c, T d, T e, T f, T q0, T q1, T q2, T q3, T eps, T &num,
                                             T &den)
{
    const T third = cst<T>(1.0 / 3.0), msixth = cst<T>(-1.0 / 6.0);
    const T ms7 = cst<T>(-7.0 / 6.0), s11 = cst<T>(11.0 / 6.0), s5 = cst<T>(5.0 / 6.0);
    const T p0 = fmaT(third, a, fmaT(ms7, b, s11 * c));
    const T p1 = fmaT(msixth, b, fmaT(s5, c, third * d));
    const T p2 = fmaT(third, c, fmaT(s5, d, msixth * e));
    const T p3 = fmaT(s11, d, fmaT(ms7, e, third * f));
    const T quarter = cst<T>(0.25);
    T t;
    t = fmaT(cst<T>(-4.0), b, fmaT(cst<T>(3.0), c, a));
    const T is0 = fmaT(quarter, t * t, q0);
    t = d - b;
    const T is1 = fmaT(quarter, t * t, q1);
    t = fmaT(cst<T>(3.0), d - c, d - e);
    const T is2 = fmaT(quarter, t * t, q2);
    t = fmaT(cst<T>(8.0), e, fmaT(cst<T>(-5.0), d, cst<T>(-3.0) * f));
    T is3 = fmaT(quarter, t * t, q3);
    is3 = fmaxT(fmaxT(fmaxT(is0, is1), is2), is3);
    const T d0 = eps + is0, d1 = eps + is1, d2 = eps + is2, d3 = eps + is3;
    const T d01 = d0 * d1, d23 = d2 * d3;
    const T n0 = cst<T>(0.05) * (d1 * d23);
    const T n1 = cst<T>(0.45) * (d0 * d23);
    const T n2 = cst<T>(0.45) * (d01 * d3);
    const T n3 = cst<T>(0.05) * (d01 * d2);
    den = n0 + n1 + n2 + n3;
    num = fmaT(n0, p0, fmaT(n1, p1, fmaT(n2, p2, n3 * p3)));
}

// Reciprocal of a WENO normaliser: correctly rounded in double; in FP32 the
// hardware approximation (rcp.approx, within one unit in the last place), as
// the weights only scale a difference from the centre cell and need FP32
// accuracy, not rounding to nearest.
template <typename T> __device__ __forceinline__ T rcp_weno(T x) { return rcp<T>(x); }
template <> __device__ __forceinline__ float rcp_weno<float>(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
template <> __device__ __forceinline__ f2 rcp_weno<f2>(f2 x) { return f2(rcp_weno<float>(x.v.x), rcp_weno<float>(x.v.y)); }

template <typename T>
__device__ __forceinline__ T weno_side(T a, T b, T c, T d, T e, T f, T q0, T q1, T q2, T q3, T eps)
{
    T num, den;
    weno_side_nd<T>(a, b, c, d, e, f, q0, q1, q2, q3, eps, num, den);
    return num * rcp_weno<T>(den);
}

// Both interface values of the stencil (LLL, LL, L, R, RR, RRR): wl seen from
// the left cell, wr from the right cell (update.cpp:508-557).
template <typename T>
__device__ __forceinline__ void weno_pair(T LLL, T LL, T L, T R, T RR, T RRR, T eps, T &wl, T &wr)
{
    const T k13 = cst<T>(13.0 / 12.0), m2 = cst<T>(-2.0);
    T s;
    s = fmaT(m2, LL, LLL + L);  const T q0 = k13 * s * s;
    s = fmaT(m2, L, LL + R);    const T q1 = k13 * s * s;
    s = fmaT(m2, R, L + RR);    const T q2 = k13 * s * s;
    s = fmaT(m2, RR, R + RRR);  const T q3 = k13 * s * s;
    if constexpr (std::is_same<T, double>::value) {
        // double: one reciprocal for both sides, 1/Dl = Dr / (Dl Dr) (the
        // normalisers lie between about 1e-30 and 1e9 with eps = 1e-10, so the
        // product stays far inside the double range)
        T nl, dl, nr, dr;
        weno_side_nd<T>(LLL, LL, L, R, RR, RRR, q0, q1, q2, q3, eps, nl, dl);
        weno_side_nd<T>(RRR, RR, R, L, LL, LLL, q3, q2, q1, q0, eps, nr, dr);
        const T r = rcp<T>(dl * dr);
        wl = nl * (dr * r);
        wr = nr * (dl * r);
    } else {
        wl = weno_side<T>(LLL, LL, L, R, RR, RRR, q0, q1, q2, q3, eps);
        wr = weno_side<T>(RRR, RR, R, L, LL, LLL, q3, q2, q1, q0, eps);
    }
}

// ---------------------------------------------------------------------------
// Half-space seed 0.5 erfc(|x|) from ex = exp(-x^2), which the half-space
// tables need anyway: erfc(a) = exp(-a^2) erfcx(a), erfcx evaluated as its
// Chebyshev interpolant in t = (a - K)/(a + K) (gen_erfcx.py; relative error
// below 5e-16 for a <= 6, 2e-15 up to the underflow of exp(-a^2)).  The other
// half is 1 - 0.5 erfc(|x|), without cancellation.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double half_erfc_abs(double x, double ex)
{
    const double a = fabs(x);
    const double t = (a - kErfcxK) * __drcp_rn(a + kErfcxK);
    double p = kErfcxC[kErfcxDeg];
#pragma unroll
    for (int i = kErfcxDeg - 1; i >= 0; --i) p = fma(p, t, kErfcxC[i]);
    return (0.5 * ex) * p;
}

// Both half-space seeds, hp = 0.5 erfc(x) and hm = 0.5 erfc(-x), from x and
// ex = exp(-x^2).  For |x| <= 1 (nearly every interface of a turbulent field)
// from erf(x) = x P(x^2), P the generated polynomial of degree kErfSmallDeg in
// x^2, with no reciprocal: hp = 0.5 - 0.5 x P, hm = 0.5 + 0.5 x P, each one
// fused multiply-add (relative error below 6.1e-16); beyond, from the erfcx
// form above, the far tail direct and the other value as 1 - tail.
__device__ __forceinline__ void half_erfc_pm(double x, double ex, double &hp, double &hm)
{
    if (fabs(x) <= 1.0) {
        const double s = x * x;
        double p = kErfSmallC[kErfSmallDeg];
#pragma unroll
        for (int i = kErfSmallDeg - 1; i >= 0; --i) p = fma(p, s, kErfSmallC[i]);
        const double hx = 0.5 * x;
        hp = fma(-hx, p, 0.5);
        hm = fma(hx, p, 0.5);
    } else {
        const double tail = half_erfc_abs(x, ex);
        hp = x >= 0.0 ? tail : 1.0 - tail;
        hm = x >= 0.0 ? 1.0 - tail : tail;
    }
}

// ---------------------------------------------------------------------------
// 1-D velocity moments of a Maxwellian (GKMflux.cpp:48-66).  s = 1/(2 lambda)
// is the variance; <u^n> = U <u^{n-1}> + (n-1) s <u^{n-2}>.
// ---------------------------------------------------------------------------
template <int N, typename T>
__device__ __forceinline__ void full_table(T U, T s, T *f)
{
    f[0] = T(1.0f);
    f[1] = U;
#pragma unroll
    for (int n = 2; n < N; ++n) f[n] = fmaT(U, f[n - 1], (T(float(n - 1)) * s) * f[n - 2]);
}

// Half-space moments over u > 0 (sign = +1) or u < 0 (sign = -1), seeded by
// 0.5 erfc(-+ sqrt(lambda) U) and -+ exp(-lambda U^2) / (2 sqrt(pi lambda)).
template <int N>
__device__ __forceinline__ void half_table(double U, double s, double h0, double g, double *h)
{
    // h0 = 0.5 erfc(...), g = +- 0.5 exp(-lambda U^2)/sqrt(pi lambda)
    h[0] = h0;
    h[1] = fma(U, h0, g);
#pragma unroll
    for (int n = 2; n < N; ++n) h[n] = fma(U, h[n - 1], (double(n - 1) * s) * h[n - 2]);
}

// ---------------------------------------------------------------------------
// Conservative -> primitive (GKMflux.cpp:301-308).
// ---------------------------------------------------------------------------
struct Prim {
    double den, rinv, U0, U1, U2, P, lam, s; // s = 1/(2 lambda) = P/den
};

// rho (rho E) - |m|^2 / 2 = rho^2 p / (gamma - 1): the pressure times rho^2 /
// (gamma - 1), without a division.
__device__ __forceinline__ double rho2p(const double W[5])
{
    return fma(-0.5, fma(W[1], W[1], fma(W[2], W[2], W[3] * W[3])), W[0] * W[4]);
}

// With A = rho2p(W) and one reciprocal r = 1 / (rho A): 1/rho = A r,
// p = (gamma - 1) A / rho, lambda = rho / (2 p) = rho^2 (rho r) / (2 (gamma - 1));
// hig = 1 / (2 (gamma - 1)).
__device__ __forceinline__ Prim prim(const double W[5], double gm1, double hig)
{
    Prim p;
    p.den = W[0];
    const double A = rho2p(W);
    const double r = rcp<double>(W[0] * A);
    p.rinv = A * r;
    p.U0 = W[1] * p.rinv;
    p.U1 = W[2] * p.rinv;
    p.U2 = W[3] * p.rinv;
    p.P = gm1 * (A * p.rinv);
    p.s = p.P * p.rinv;
    p.lam = hig * (W[0] * W[0]) * (W[0] * r);
    return p;
}

// The internal-degrees-of-freedom constants of a Maxwellian's moments in type
// T (K = internal degrees of freedom): r2 = K + 2, q4 = K + 4,
// r4 = (K + 2)(K + 4), nq = -(K + 3).  Precomputed per field, so that no
// integer-to-floating conversion runs per interface.
template <typename T> struct KConst {
    T r2, q4, r4, nq;
};

// Constants of one field that the flux needs (all precomputed per field).
struct FluxConst {
    double gm1;   // gamma - 1
    double hig;   // 1 / (2 (gamma - 1))
    double dt, dx;
    double ks[3]; // slope scales: 2/dx (normal), +-1/(2 dx) (transverse)
    double kA;    // pr_factor * 4 / (K + 3)
    double hK2;   // (K + 2) / 2
    KConst<double> kd; // in double and in float
    KConst<float> kf;
};

} // namespace gks
