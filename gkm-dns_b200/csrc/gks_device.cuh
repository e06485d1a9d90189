// Device math of the WENO-GKS hot path: WENO-SYMOO reconstruction, Maxwellian
// moment tables, moment vectors, the slope solve and the BGK-NS interface flux.
//
// The algebra is the reference's (weno/src/update.cpp:502-625 for WENO,
// weno/src/GKMflux.cpp:11-308 for the flux); the evaluation order is this
// file's own and is organised for the GPU:
//  * the flux is accumulated per Maxwellian (left, right, equilibrium) so that
//    only one side's moment tables are live at a time (the reference keeps
//    nine 3x7 tables live, GKMflux.cpp:18);
//  * only the normal-velocity half-space tables are built: the reference also
//    builds half-space tables of the transverse components (GKMflux.cpp:54-57
//    for j = 1, 2) but never reads them, which costs it 8 erfc and 8 exp per
//    interface;
//  * divisions become reciprocals shared across uses, and each MCal
//    (GKMflux.cpp:225-264) is evaluated by contracting the transverse
//    moments first (see mcal_a), which the compiler then shares between calls
//    with the same slope vector and transverse tables.
// Results therefore agree with the reference to rounding, not bit for bit.
//
// Precision: `S` is the type of the slope solves and slope-weighted moments
// (double in the FP64 path, float in the mixed path); moment tables, erfc /
// exp, the zeroth-order (slope-free) moments and the flux accumulation stay
// double in both.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

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

// a*b + c with one rounding, for every arithmetic type used here.
__device__ __forceinline__ double fmaT(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fmaT(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ f2 fmaT(f2 a, f2 b, f2 c) { f2 r; r.v = __ffma2_rn(a.v, b.v, c.v); return r; }

// ---------------------------------------------------------------------------
// WENO-SYMOO on one scalar 6-point stencil (update.cpp:505-557): four cubic
// candidates per side, linear weights 1/20, 9/20, 9/20, 1/20, the fourth
// smoothness indicator replaced by the largest of the four, alpha = g/(eps+IS).
// The normalised weights are formed with one reciprocal per side:
// w_r = g_r prod_{s!=r} d_s / sum_t g_t prod_{s!=t} d_s, d = eps + IS.
// ---------------------------------------------------------------------------
// One side seen from (a, b, c | d, e, f): candidates on {a,b,c}, {b,c,d},
// {c,d,e}, {d,e,f}; q0..q3 are 13/12 of the squared second differences of
// those stencils, which both sides share.
template <typename T>
__device__ __forceinline__ T weno_side(T a, T b, T c, T d, T e, T f, T q0, T q1, T q2, T q3, T eps)
{
    const T third = T(1) / T(3), sixth = T(1) / T(6);
    const T p0 = third * a - (T(7) * sixth) * b + (T(11) * sixth) * c;
    const T p1 = -sixth * b + (T(5) * sixth) * c + third * d;
    const T p2 = third * c + (T(5) * sixth) * d - sixth * e;
    const T p3 = (T(11) * sixth) * d - (T(7) * sixth) * e + third * f;
    T t;
    t = a - T(4) * b + T(3) * c;
    const T is0 = fmaT(T(0.25), t * t, q0);
    t = d - b;
    const T is1 = fmaT(T(0.25), t * t, q1);
    t = T(-3) * c + T(4) * d - e;
    const T is2 = fmaT(T(0.25), t * t, q2);
    t = T(-5) * d + T(8) * e - T(3) * f;
    T is3 = fmaT(T(0.25), t * t, q3);
    is3 = fmax(fmax(fmax(is0, is1), is2), is3);
    const T d0 = eps + is0, d1 = eps + is1, d2 = eps + is2, d3 = eps + is3;
    const T d01 = d0 * d1, d23 = d2 * d3;
    const T n0 = T(0.05) * (d1 * d23);
    const T n1 = T(0.45) * (d0 * d23);
    const T n2 = T(0.45) * (d01 * d3);
    const T n3 = T(0.05) * (d01 * d2);
    const T inv = rcp<T>(n0 + n1 + n2 + n3);
    return (n0 * p0 + n1 * p1 + n2 * p2 + n3 * p3) * inv;
}

// Both interface values of the stencil (LLL, LL, L, R, RR, RRR): wl seen from
// the left cell, wr from the right cell (update.cpp:508-557).
template <typename T>
__device__ __forceinline__ void weno_pair(T LLL, T LL, T L, T R, T RR, T RRR, T eps, T &wl, T &wr)
{
    const T k13 = T(13) / T(12);
    T s;
    s = LLL - T(2) * LL + L;  const T q0 = k13 * s * s;
    s = LL - T(2) * L + R;    const T q1 = k13 * s * s;
    s = L - T(2) * R + RR;    const T q2 = k13 * s * s;
    s = R - T(2) * RR + RRR;  const T q3 = k13 * s * s;
    wl = weno_side<T>(LLL, LL, L, R, RR, RRR, q0, q1, q2, q3, eps);
    wr = weno_side<T>(RRR, RR, R, L, LL, LLL, q3, q2, q1, q0, eps);
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
    h[1] = U * h0 + g;
#pragma unroll
    for (int n = 2; n < N; ++n) h[n] = U * h[n - 1] + double(n - 1) * s * h[n - 2];
}

// ---------------------------------------------------------------------------
// Moment vectors.  With psi = (1, u, v, w, (u^2+v^2+w^2+xi^2)/2), X the table
// of the normal velocity, Y and Z those of the transverse components and
// e2 = <xi^2>, e4 = <xi^4>:
//   mcal0<k,l,m>   M_q = <psi_q u^k v^l w^m>             (GKMflux.cpp:266-275)
//   mcal_a<k,l,m>  M_q = <psi_q u^k v^l w^m (a . psi)>   (GKMflux.cpp:225-264)
// mcal_a contracts the transverse moments first:
//   G(p,b,c) = <u^{k+p} v^{l+b} w^{m+c} (a.psi)>
//            = X[k+p] g0(b,c) + X[k+p+1] a1 YZ(b,c) + X[k+p+2] (a4/2) YZ(b,c)
//   g0(b,c)  = a0 YZ(b,c) + a2 YZ(b+1,c) + a3 YZ(b,c+1) + (a4/2)(YZ(b+2,c)+YZ(b,c+2)+e2 YZ(b,c))
//   M = (G000, G100, G010, G001, (G200+G020+G002 + e2 G000 + (a4/2)(e4-e2^2) X[k]YZ(0,0))/2)
// with YZ(b,c) = Y[l+b] Z[m+c]; this is the reference's sum regrouped.
// ---------------------------------------------------------------------------
template <typename T> struct V5 {
    T v[5];
};

template <int k, int l, int m, typename T>
__device__ __forceinline__ void mcal0(T M[5], const T *X, const T *Y, const T *Z, T e2)
{
    const T yz = Y[l] * Z[m];
    M[0] = X[k] * yz;
    M[1] = X[k + 1] * yz;
    M[2] = X[k] * (Y[l + 1] * Z[m]);
    M[3] = X[k] * (Y[l] * Z[m + 1]);
    M[4] = T(0.5f) * fmaT(X[k + 2], yz, X[k] * fmaT(e2, yz, Y[l + 2] * Z[m] + Y[l] * Z[m + 2]));
}

template <int k, int l, int m, typename T>
__device__ __forceinline__ void mcal_a(T M[5], const T *X, const T *Y, const T *Z, T e2, T e4, const T a[5])
{
#define YZ(b, c) (Y[l + (b)] * Z[m + (c)])
    const T h4 = T(0.5f) * a[4];
#define G0(b, c) fmaT(a[0], YZ(b, c), fmaT(a[2], YZ((b) + 1, c), fmaT(a[3], YZ(b, (c) + 1), \
                  h4 * fmaT(e2, YZ(b, c), YZ((b) + 2, c) + YZ(b, (c) + 2)))))
#define GG(p, b, c) fmaT(X[k + (p)], G0(b, c), fmaT(X[k + (p) + 1], a[1], X[k + (p) + 2] * h4) * YZ(b, c))
    const T m0 = GG(0, 0, 0);
    M[0] = m0;
    M[1] = GG(1, 0, 0);
    M[2] = GG(0, 1, 0);
    M[3] = GG(0, 0, 1);
    M[4] = T(0.5f) * (GG(2, 0, 0) + GG(0, 2, 0) + GG(0, 0, 2) +
                      fmaT(e2, m0, (h4 * (e4 - e2 * e2)) * (X[k] * YZ(0, 0))));
#undef GG
#undef G0
#undef YZ
}

template <typename T>
__device__ __forceinline__ void add5(T acc[5], const T x[5])
{
#pragma unroll
    for (int q = 0; q < 5; ++q) acc[q] += x[q];
}

// ---------------------------------------------------------------------------
// Slope solve (slopesolver, GKMflux.cpp:280-296): the Maxwellian-derivative
// coefficients a with <psi (a.psi)> g = b for a Maxwellian of velocity U and
// lambda.  q = |U|^2 + (K+3)/(2 lambda); kA = pr_factor * 4/(K+3).
// ---------------------------------------------------------------------------
template <typename T> struct SlopeFrame {
    T U0, U1, U2, nU0, nU1, nU2, tl, q, nq, kal2; // tl = 2 lambda, kal2 = kA lambda^2, nX = -X
};

template <typename T>
__device__ __forceinline__ SlopeFrame<T> slope_frame(T U0, T U1, T U2, T lam, T s, int K, T kA)
{
    SlopeFrame<T> f;
    f.U0 = U0;
    f.U1 = U1;
    f.U2 = U2;
    f.nU0 = -U0;
    f.nU1 = -U1;
    f.nU2 = -U2;
    f.tl = T(2.0f) * lam;
    f.q = fmaT(U0, U0, fmaT(U1, U1, fmaT(U2, U2, T(float(K + 3)) * s)));
    f.nq = -f.q;
    f.kal2 = (kA * lam) * lam;
    return f;
}

template <typename T>
__device__ __forceinline__ void slope_solve(const T b[5], const SlopeFrame<T> &f, T a[5])
{
    const T R2 = fmaT(f.nU0, b[0], b[1]);
    const T R3 = fmaT(f.nU1, b[0], b[2]);
    const T R4 = fmaT(f.nU2, b[0], b[3]);
    const T R5 = fmaT(f.nq, b[0], T(2.0f) * b[4]);
    const T d = fmaT(f.U0, R2, fmaT(f.U1, R3, f.U2 * R4));
    a[4] = f.kal2 * fmaT(T(-2.0f), d, R5);
    a[3] = fmaT(f.nU2, a[4], f.tl * R4);
    a[2] = fmaT(f.nU1, a[4], f.tl * R3);
    a[1] = fmaT(f.nU0, a[4], f.tl * R2);
    const T e = fmaT(a[1], f.U0, fmaT(a[2], f.U1, a[3] * f.U2));
    a[0] = fmaT(T(-0.5f) * f.q, a[4], b[0] - e);
}

// ---------------------------------------------------------------------------
// Conservative -> primitive (GKMflux.cpp:301-308).
// ---------------------------------------------------------------------------
struct Prim {
    double den, rinv, U0, U1, U2, P, lam, s; // s = 1/(2 lambda) = P/den
};

__device__ __forceinline__ Prim prim(const double W[5], double gm1)
{
    Prim p;
    p.den = W[0];
    p.rinv = rcp<double>(W[0]);
    p.U0 = W[1] * p.rinv;
    p.U1 = W[2] * p.rinv;
    p.U2 = W[3] * p.rinv;
    p.P = gm1 * (W[4] - 0.5 * (W[1] * p.U0 + W[2] * p.U1 + W[3] * p.U2));
    p.s = p.P * p.rinv;
    p.lam = 0.5 * p.den * rcp<double>(p.P);
    return p;
}

// Constants of one field that the flux needs.
struct FluxConst {
    double gm1;   // gamma - 1
    double dt, dx;
    double kA;    // pr_factor * 4 / (K + 3)
    int K;
};

template <typename S>
__device__ __forceinline__ void cast5(S out[5], const double in[5])
{
#pragma unroll
    for (int q = 0; q < 5; ++q) out[q] = S(in[q]);
}

// ---------------------------------------------------------------------------
// Time-integrated BGK-NS interface flux (GKMflux.cpp:11-215), in the frame of
// the interface normal.  The caller supplies the inputs through `src`, which
// is asked for them only when they are needed, so that one side's inputs are
// not live while the other side is processed:
//   src.state(side, W)      reconstructed state Wl (side 0) or Wr (side 1)
//   src.slopes(side, DW)    its slopes DW[d][q], d = normal, 1st, 2nd transverse
//   src.cells(WL, WR)       the cell averages either side of the interface
// tau0 = mu/p at the left cell.  Output F[5], the flux integrated over [0, dt].
// ---------------------------------------------------------------------------
template <typename S, int NEG, typename Src>
__device__ __forceinline__ void flux_side(const Src &src, const Prim &g, const FluxConst &c,
                                          double gmB2, double gmB3, double pF3, double pF4, double pF5,
                                          double We[5], double Fbase[5], S by_[5], S bz_[5], S Bs[5], S Fs[5])
{
    // tables of this Maxwellian (double): transverse Y, Z and the normal half space
    double Y[6], Z[6], X[7];
    full_table<6>(g.U1, g.s, Y);
    full_table<6>(g.U2, g.s, Z);
    const double e2 = double(c.K) * g.s;
    const double e4 = double(c.K * (c.K + 2)) * g.s * g.s;
    {
        const double sl = sqrt(g.lam);
        const double h0 = 0.5 * erfc(NEG ? sl * g.U0 : -sl * g.U0);
        const double ex = 0.5 * exp(-g.lam * g.U0 * g.U0) * rsqrt(kPi * g.lam);
        half_table<7>(g.U0, g.s, h0, NEG ? -ex : ex, X);
    }
    // zeroth-order moments (double): W0 (GKMflux.cpp:71-75) and the p3 term of F
    {
        double M0[5], M1[5];
        mcal0<0, 0, 0, double>(M0, X, Y, Z, e2);
        mcal0<1, 0, 0, double>(M1, X, Y, Z, e2);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            We[q] += g.den * M0[q];
            Fbase[q] += pF3 * g.den * M1[q];
        }
    }
    // slope coefficients of this side (phase I, GKMflux.cpp:102-117)
    const S den = S(g.den), rinv = S(g.rinv);
    const SlopeFrame<S> fr = slope_frame<S>(S(g.U0), S(g.U1), S(g.U2), S(g.lam), S(g.s), c.K, S(c.kA));
    S ax[5], ay[5], az[5];
    {
        S DW[3][5];
        src.slopes(NEG, DW);
        S b[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = DW[0][q] * rinv;
        slope_solve<S>(b, fr, ax);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = DW[1][q] * rinv;
        slope_solve<S>(b, fr, ay);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = DW[2][q] * rinv;
        slope_solve<S>(b, fr, az);
    }
    S Ys[6], Zs[6], Xs[7];
#pragma unroll
    for (int n = 0; n < 6; ++n) { Ys[n] = S(Y[n]); Zs[n] = S(Z[n]); }
#pragma unroll
    for (int n = 0; n < 7; ++n) Xs[n] = S(X[n]);
    const S e2s = S(e2), e4s = S(e4);
    // A of this side from the full-space time derivative (phase II, GKMflux.cpp:128-144)
    S A[5];
    {
        S Xf[6];
        full_table<6, S>(S(g.U0), S(g.s), Xf);
        S B[5], M[5];
        mcal_a<1, 0, 0, S>(B, Xf, Ys, Zs, e2s, e4s, ax);
        mcal_a<0, 1, 0, S>(M, Xf, Ys, Zs, e2s, e4s, ay);
        add5<S>(B, M);
        mcal_a<0, 0, 1, S>(M, Xf, Ys, Zs, e2s, e4s, az);
        add5<S>(B, M);
#pragma unroll
        for (int q = 0; q < 5; ++q) B[q] = -B[q];
        slope_solve<S>(B, fr, A);
    }
    // transverse slopes of the equilibrium state (by_, bz_, GKMflux.cpp:124-127, 136-137)
    {
        S M[5];
        mcal_a<0, 0, 0, S>(M, Xs, Ys, Zs, e2s, e4s, ay);
        add5<S>(by_, M);
        mcal_a<0, 0, 0, S>(M, Xs, Ys, Zs, e2s, e4s, az);
        add5<S>(bz_, M);
    }
    // B_ contributions (GKMflux.cpp:164-176)
    {
        S M[5], T1[5];
        mcal_a<1, 0, 0, S>(T1, Xs, Ys, Zs, e2s, e4s, ax);
        mcal_a<0, 1, 0, S>(M, Xs, Ys, Zs, e2s, e4s, ay);
        add5<S>(T1, M);
        mcal_a<0, 0, 1, S>(M, Xs, Ys, Zs, e2s, e4s, az);
        add5<S>(T1, M);
        mcal_a<0, 0, 0, S>(M, Xs, Ys, Zs, e2s, e4s, A);
        const S w1 = S(gmB2) * den, w2 = S(gmB3) * den;
#pragma unroll
        for (int q = 0; q < 5; ++q) Bs[q] += w1 * T1[q] + w2 * M[q];
    }
    // flux contributions (GKMflux.cpp:200-212)
    {
        S M[5], T1[5];
        mcal_a<2, 0, 0, S>(T1, Xs, Ys, Zs, e2s, e4s, ax);
        mcal_a<1, 1, 0, S>(M, Xs, Ys, Zs, e2s, e4s, ay);
        add5<S>(T1, M);
        mcal_a<1, 0, 1, S>(M, Xs, Ys, Zs, e2s, e4s, az);
        add5<S>(T1, M);
        mcal_a<1, 0, 0, S>(M, Xs, Ys, Zs, e2s, e4s, A);
        const S w1 = S(pF4) * den, w2 = S(pF5) * den;
#pragma unroll
        for (int q = 0; q < 5; ++q) Fs[q] += w1 * T1[q] + w2 * M[q];
    }
}

template <typename S, typename Src>
__device__ __forceinline__ void gks_flux(const Src &src, double tau0, const FluxConst &c, double F[5])
{
    Prim l, r;
    {
        double Ws[5];
        src.state(0, Ws);
        l = prim(Ws, c.gm1);
        src.state(1, Ws);
        r = prim(Ws, c.gm1);
    }
    // collision time with the pressure-jump term (GKMflux.cpp:149-150):
    // rho/lambda = 2p, so w = |p_l - p_r| / (p_l + p_r)
    const double dt = c.dt;
    const double tau = tau0 + dt * (fabs(l.P - r.P) * rcp<double>(l.P + r.P));
    const double ex = exp(-dt * rcp<double>(tau));
    const double om = 1.0 - ex;
    // gamma weights (GKMflux.cpp:155-157)
    const double igm0 = rcp<double>(dt - tau * om);
    const double gm1 = -om * igm0;
    const double gm2 = (-dt + 2.0 * tau * om - dt * ex) * igm0;
    const double gm3 = -gm1;
    const double gm4 = (dt * ex - tau * om) * igm0;
    const double gm5 = tau * gm3;
    // time integrals (GKMflux.cpp:186-190)
    const double Pt = tau * om;
    const double Qt = tau * (tau * om - dt * ex);
    const double p0 = dt - Pt;
    const double p1 = 0.5 * dt * dt - tau * p0;
    const double p2 = -tau * p0 + Qt;
    const double p3 = Pt;
    const double p4 = -Qt - tau * Pt;
    const double p5 = -tau * Pt;

    double We[5] = {0, 0, 0, 0, 0}, Fbase[5] = {0, 0, 0, 0, 0};
    S by_[5] = {0, 0, 0, 0, 0}, bz_[5] = {0, 0, 0, 0, 0}, Bs[5] = {0, 0, 0, 0, 0}, Fs[5] = {0, 0, 0, 0, 0};
    flux_side<S, 0>(src, l, c, gm4 + gm5, gm5, p3, p4, p5, We, Fbase, by_, bz_, Bs, Fs);
    flux_side<S, 1>(src, r, c, gm4 + gm5, gm5, p3, p4, p5, We, Fbase, by_, bz_, Bs, Fs);

    // equilibrium state at the interface (GKMflux.cpp:71-98)
    const Prim e = prim(We, c.gm1);
    double Y[6], Z[6], Xf[6], Xp[7], Xn[7];
    full_table<6>(e.U1, e.s, Y);
    full_table<6>(e.U2, e.s, Z);
    full_table<6>(e.U0, e.s, Xf);
    const double e2 = double(c.K) * e.s;
    const double e4 = double(c.K * (c.K + 2)) * e.s * e.s;
    {
        // 0.5 erfc(-+x) from one evaluation at |x|: the far tail is computed
        // directly, the other value as 1 - tail (no cancellation)
        const double sl = sqrt(e.lam);
        const double x = sl * e.U0;
        const double tail = 0.5 * erfc(fabs(x));
        const double hp = x >= 0.0 ? 1.0 - tail : tail; // 0.5 erfc(-x)
        const double hn = x >= 0.0 ? tail : 1.0 - tail; // 0.5 erfc(x)
        const double g = 0.5 * exp(-e.lam * e.U0 * e.U0) * rsqrt(kPi * e.lam);
        half_table<7>(e.U0, e.s, hp, g, Xp);
        half_table<7>(e.U0, e.s, hn, -g, Xn);
    }
    // B_ base terms: gm1 rho_e <psi>_e + gm3 W0 (GKMflux.cpp:174), nearly cancelling
    double Bbase[5];
    {
        double M0[5], M1[5];
        mcal0<0, 0, 0, double>(M0, Xf, Y, Z, e2);
        mcal0<1, 0, 0, double>(M1, Xf, Y, Z, e2);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            Bbase[q] = gm1 * e.den * M0[q] + gm3 * We[q];
            Fbase[q] += p0 * e.den * M1[q];
        }
    }
    const SlopeFrame<S> fr = slope_frame<S>(S(e.U0), S(e.U1), S(e.U2), S(e.lam), S(e.s), c.K, S(c.kA));
    S axl[5], axr[5], ay[5], az[5];
    {
        // normal slopes of the equilibrium state from the cell averages (GKMflux.cpp:109-110)
        double WL[5], WR[5];
        src.cells(WL, WR);
        const double k2 = 2.0 * e.rinv * (1.0 / c.dx);
        S b[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = S((We[q] - WL[q]) * k2);
        slope_solve<S>(b, fr, axl);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = S((WR[q] - We[q]) * k2);
        slope_solve<S>(b, fr, axr);
        slope_solve<S>(by_, fr, ay);
        slope_solve<S>(bz_, fr, az);
    }
    S Ys[6], Zs[6], Xfs[6], Xps[7], Xns[7];
#pragma unroll
    for (int n = 0; n < 6; ++n) { Ys[n] = S(Y[n]); Zs[n] = S(Z[n]); Xfs[n] = S(Xf[n]); }
#pragma unroll
    for (int n = 0; n < 7; ++n) { Xps[n] = S(Xp[n]); Xns[n] = S(Xn[n]); }
    const S e2s = S(e2), e4s = S(e4), dens = S(e.den);
    // A_ (phase III, GKMflux.cpp:159-180)
    S A[5];
    {
        S T1[5], M[5];
        mcal_a<1, 0, 0, S>(T1, Xps, Ys, Zs, e2s, e4s, axl);
        mcal_a<1, 0, 0, S>(M, Xns, Ys, Zs, e2s, e4s, axr);
        add5<S>(T1, M);
        mcal_a<0, 1, 0, S>(M, Xfs, Ys, Zs, e2s, e4s, ay);
        add5<S>(T1, M);
        mcal_a<0, 0, 1, S>(M, Xfs, Ys, Zs, e2s, e4s, az);
        add5<S>(T1, M);
        const S w = S(gm2) * dens;
        S B[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) B[q] = S((Bbase[q] + double(Bs[q] + w * T1[q])) * e.rinv);
        slope_solve<S>(B, fr, A);
    }
    // flux (GKMflux.cpp:192-213)
    {
        S T1[5], M[5];
        mcal_a<2, 0, 0, S>(T1, Xps, Ys, Zs, e2s, e4s, axl);
        mcal_a<2, 0, 0, S>(M, Xns, Ys, Zs, e2s, e4s, axr);
        add5<S>(T1, M);
        mcal_a<1, 1, 0, S>(M, Xfs, Ys, Zs, e2s, e4s, ay);
        add5<S>(T1, M);
        mcal_a<1, 0, 1, S>(M, Xfs, Ys, Zs, e2s, e4s, az);
        add5<S>(T1, M);
        mcal_a<1, 0, 0, S>(M, Xfs, Ys, Zs, e2s, e4s, A);
        const S w2 = S(p2) * dens, w1 = S(p1) * dens;
#pragma unroll
        for (int q = 0; q < 5; ++q) F[q] = Fbase[q] + double(Fs[q] + w2 * T1[q] + w1 * M[q]);
    }
}

} // namespace gks
