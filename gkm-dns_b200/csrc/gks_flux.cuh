// Time-integrated BGK-NS interface flux (weno/src/GKMflux.cpp:11-215) with the
// moments of every Maxwellian evaluated in the frame that moves with that
// Maxwellian's transverse velocity.
//
// The reference builds 1-D moment tables of all three velocity components for
// each of its three Maxwellians (left, right, equilibrium; GKMflux.cpp:48-66,
// 82-98) and contracts them in MCal (GKMflux.cpp:225-275): 41 calls per
// interface of about 80 operations each.  Here the transverse velocities are
// measured from the Maxwellian's own mean, c1 = v - U1 and c2 = w - U2.  In
// that frame the transverse moments are the central Gaussian ones --
// <c^2> = s, <c^4> = 3 s^2, every odd moment zero, s = 1/(2 lambda) -- so a
// moment vector <psi u^k v^l w^m (a.psi)> needs only the table X of the normal
// velocity (half or full space, as in the reference) and three constants:
//   rho^2 = c1^2 + c2^2 + xi^2,  r2 = <rho^2> = (K+2) s,
//   r4 = <rho^4> = (K+2)(K+4) s^2,  q4 = <c1^2 rho^2> = (K+4) s^2.
// The change of frame is the Galilean map of the collision invariants
// psi = (1, u, v, w, (u^2+v^2+w^2+xi^2)/2) = T psi' with
//   psi'_2 = c1, psi'_3 = c2, psi'_4 = (u^2 + rho^2)/2,
//   psi_4 = psi'_4 + U1 psi'_2 + U2 psi'_3 + (U1^2+U2^2)/2 psi'_0;
// moment vectors transform with T (to_lab), slope right-hand sides with T^-1
// (to_prime), and the slope solve (slopesolver, GKMflux.cpp:280-296) run in
// the primed frame, where the Maxwellian moves with (U0, 0, 0), returns the
// primed coefficients directly.  Sums of moment vectors of one Maxwellian are
// taken in its primed frame and transformed once.  The algebra is the
// reference's; only the order of evaluation differs, so results agree with it
// to rounding.
//
// Precision: `S` is the type of the slope solves and slope-weighted moment
// vectors -- the flux assembly -- (double in the FP64 path, float in the
// mixed path).  The primitive states, collision time and time weights, the
// moment-table recursions with their erfc / exp seeds, the zeroth-order
// (slope-free) moments -- the equilibrium state W0, the p0 and p3 terms of the
// flux and the gm1 / gm3 terms of B_ -- and the flux accumulation stay double
// in both paths.
#pragma once

#include "gks_device.cuh"

namespace gks {

// Constants of one Maxwellian in its transverse co-moving frame.
template <typename T> struct CoFrame {
    T U0, U1, U2, hu2; // velocity; hu2 = (U1^2 + U2^2)/2
    T s, tl, kal2, qn; // 1/(2 lambda), 2 lambda, kA lambda^2, U0^2 + (K+3) s
    T r2, r4, q4;      // <rho^2>, <rho^4>, <c1^2 rho^2>
};

template <typename T>
__device__ __forceinline__ CoFrame<T> co_frame(const Prim &g, int K, double kA)
{
    CoFrame<T> f;
    f.U0 = T(g.U0);
    f.U1 = T(g.U1);
    f.U2 = T(g.U2);
    f.s = T(g.s);
    const T lam = T(g.lam);
    f.hu2 = T(0.5f) * fmaT(f.U1, f.U1, f.U2 * f.U2);
    f.tl = T(2.0f) * lam;
    f.kal2 = (T(kA) * lam) * lam;
    f.qn = fmaT(f.U0, f.U0, T(float(K + 3)) * f.s);
    f.r2 = T(float(K + 2)) * f.s;
    const T s2 = f.s * f.s;
    f.q4 = T(float(K + 4)) * s2;
    f.r4 = T(float((K + 2) * (K + 4))) * s2;
    return f;
}

// Primed -> lab frame of a moment vector (m = T m').
template <typename T>
__device__ __forceinline__ void to_lab(T m[5], T U1, T U2, T hu2)
{
    m[4] = fmaT(U1, m[2], fmaT(U2, m[3], fmaT(hu2, m[0], m[4])));
    m[2] = fmaT(U1, m[0], m[2]);
    m[3] = fmaT(U2, m[0], m[3]);
}

// Lab -> primed frame of a slope right-hand side (b' = T^-1 b).
template <typename T>
__device__ __forceinline__ void to_prime(T b[5], T U1, T U2, T hu2)
{
    b[2] = fmaT(-U1, b[0], b[2]);
    b[3] = fmaT(-U2, b[0], b[3]);
    b[4] = fmaT(-U1, b[2], fmaT(-U2, b[3], fmaT(-hu2, b[0], b[4])));
}

// Slope solve (slopesolver, GKMflux.cpp:280-296) in the primed frame: the
// coefficients a' with <psi' psi'> a' = b' for the Maxwellian moving with
// (U0, 0, 0); kal2 carries the energy-coefficient factor (1/Pr at
// GKMflux.cpp:289, or 1).
template <typename T>
__device__ __forceinline__ void solve(const T b[5], const CoFrame<T> &f, T a[5])
{
    const T R2 = fmaT(-f.U0, b[0], b[1]);
    const T R5 = fmaT(-f.qn, b[0], T(2.0f) * b[4]);
    a[4] = f.kal2 * fmaT(T(-2.0f) * f.U0, R2, R5);
    a[3] = f.tl * b[3];
    a[2] = f.tl * b[2];
    a[1] = fmaT(-f.U0, a[4], f.tl * R2);
    a[0] = fmaT(-f.U0, a[1], fmaT(T(-0.5f) * f.qn, a[4], b[0]));
}

// M = <psi' u^k (a.psi')> over the normal table X (primed frame):
//   M0 = al X[k] + a1 X[k+1] + h X[k+2],   al = a0 + h r2, h = a4/2
//   M1 = al X[k+1] + a1 X[k+2] + h X[k+3]
//   M2 = a2 s X[k],  M3 = a3 s X[k]
//   M4 = ((al + h r2) X[k+2] + (a0 r2 + h r4) X[k] + a1 (X[k+3] + r2 X[k+1]) + h X[k+4]) / 2
template <int k, typename T>
__device__ __forceinline__ void mom_n(T M[5], const T *X, const CoFrame<T> &f, const T a[5])
{
    const T h = T(0.5f) * a[4];
    const T al = fmaT(h, f.r2, a[0]);
    M[0] = fmaT(al, X[k], fmaT(a[1], X[k + 1], h * X[k + 2]));
    M[1] = fmaT(al, X[k + 1], fmaT(a[1], X[k + 2], h * X[k + 3]));
    const T sx = f.s * X[k];
    M[2] = a[2] * sx;
    M[3] = a[3] * sx;
    const T c2 = fmaT(h, f.r2, al);
    const T c0 = fmaT(a[0], f.r2, h * f.r4);
    M[4] = T(0.5f) * fmaT(c2, X[k + 2], fmaT(c0, X[k], fmaT(a[1], fmaT(f.r2, X[k + 1], X[k + 3]), h * X[k + 4])));
}

// M = <psi' u^k c_D (a.psi')>, D = 2 (c1) or 3 (c2):
//   M0 = aD s X[k],  M1 = aD s X[k+1],  M_{5-D} = 0
//   M_D = s (a0 X[k] + a1 X[k+1] + h X[k+2]) + h q4 X[k]
//   M4 = aD (s X[k+2] + q4 X[k]) / 2
template <int k, int D, typename T>
__device__ __forceinline__ void mom_t(T M[5], const T *X, const CoFrame<T> &f, const T a[5])
{
    const T h = T(0.5f) * a[4];
    const T sa = f.s * a[D];
    M[0] = sa * X[k];
    M[1] = sa * X[k + 1];
    M[D] = fmaT(f.s, fmaT(a[0], X[k], fmaT(a[1], X[k + 1], h * X[k + 2])), (h * f.q4) * X[k]);
    M[5 - D] = T(0.0f);
    M[4] = (T(0.5f) * a[D]) * fmaT(f.s, X[k + 2], f.q4 * X[k]);
}

template <typename T>
__device__ __forceinline__ void add5(T acc[5], const T x[5])
{
#pragma unroll
    for (int q = 0; q < 5; ++q) acc[q] += x[q];
}

// Zeroth-order moment vectors of one Maxwellian in the lab frame, FP64:
// <psi u^k> = (X[k], X[k+1], U1 X[k], U2 X[k], X[k+2]/2 + c4 X[k]) with
// c4 = r2/2 + (U1^2 + U2^2)/2; the reference's MCal without slopes
// (GKMflux.cpp:266-275).
template <int k>
__device__ __forceinline__ void mom0_lab(double M[5], const double *X, const Prim &g, double c4)
{
    M[0] = X[k];
    M[1] = X[k + 1];
    M[2] = g.U1 * X[k];
    M[3] = g.U2 * X[k];
    M[4] = fma(0.5, X[k + 2], c4 * X[k]);
}

// One of the two initial Maxwellians (NEG = 0: left state, half space u > 0;
// NEG = 1: right state, u < 0).  Adds its share of W0 and of the p3 flux term
// (double), of the transverse right-hand sides by_, bz_ of the equilibrium
// slopes, of B_ and of the p4 / p5 flux terms (type S, lab frame).
template <typename S, int NEG, typename Src>
__device__ __forceinline__ void flux_side(const Src &src, const Prim &g, const FluxConst &c, double w45, double g5,
                                          double p3, double p4, double p5, double We[5], double Fb[5], S by[5],
                                          S bz[5], S Bs[5], S Fs[5])
{
    // normal-velocity tables (double): half space (GKMflux.cpp:52-60) and full space
    double Xh[7], Xf[6];
    {
        const double sl = sqrt(g.lam);
        const double h0 = 0.5 * erfc(NEG ? sl * g.U0 : -sl * g.U0);
        const double ex = 0.5 * exp(-g.lam * g.U0 * g.U0) * rsqrt(kPi * g.lam);
        half_table<7>(g.U0, g.s, h0, NEG ? -ex : ex, Xh);
    }
    full_table<6, double>(g.U0, g.s, Xf);
    // W0 (GKMflux.cpp:71-75) and the p3 term of F (GKMflux.cpp:209-212), double
    {
        const double c4 = fma(0.5, g.U1 * g.U1 + g.U2 * g.U2, double(c.K + 2) * 0.5 * g.s);
        double M[5];
        mom0_lab<0>(M, Xh, g, c4);
#pragma unroll
        for (int q = 0; q < 5; ++q) We[q] = fma(g.den, M[q], We[q]);
        mom0_lab<1>(M, Xh, g, c4);
        const double w = p3 * g.den;
#pragma unroll
        for (int q = 0; q < 5; ++q) Fb[q] = fma(w, M[q], Fb[q]);
    }
    const CoFrame<S> f = co_frame<S>(g, c.K, c.kA);
    S Xhs[7], Xfs[6];
#pragma unroll
    for (int n = 0; n < 7; ++n) Xhs[n] = S(Xh[n]);
#pragma unroll
    for (int n = 0; n < 6; ++n) Xfs[n] = S(Xf[n]);
    // slope coefficients (phase I, GKMflux.cpp:102-117) and the moment sums they
    // feed, in the primed frame: Bp -> A (phase II, GKMflux.cpp:128-144),
    // Bq -> B_ (GKMflux.cpp:172-173), Fq -> F (GKMflux.cpp:210-211);
    // ayz = U1 ay + U2 az collects the v / w weights' shift.
    S Bp[5], Bq[5], Fq[5], ayz[5];
    {
        S DW[3][5];
        src.slopes(NEG, DW);
        const S rinv = S(g.rinv);
        S a[5], b[5], M[5];
        // normal slope
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = DW[0][q] * rinv;
        to_prime<S>(b, f.U1, f.U2, f.hu2);
        solve<S>(b, f, a);
        mom_n<1, S>(M, Xfs, f, a);
#pragma unroll
        for (int q = 0; q < 5; ++q) Bp[q] = -M[q];
        mom_n<1, S>(Bq, Xhs, f, a);
        mom_n<2, S>(Fq, Xhs, f, a);
        // first transverse slope (weight v = c1 + U1)
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = DW[1][q] * rinv;
        to_prime<S>(b, f.U1, f.U2, f.hu2);
        solve<S>(b, f, a);
        mom_t<0, 2, S>(M, Xfs, f, a);
#pragma unroll
        for (int q = 0; q < 5; ++q) Bp[q] -= M[q];
        mom_n<0, S>(M, Xhs, f, a);
        to_lab<S>(M, f.U1, f.U2, f.hu2);
        add5<S>(by, M);
        mom_t<0, 2, S>(M, Xhs, f, a);
        add5<S>(Bq, M);
        mom_t<1, 2, S>(M, Xhs, f, a);
        add5<S>(Fq, M);
#pragma unroll
        for (int q = 0; q < 5; ++q) ayz[q] = f.U1 * a[q];
        // second transverse slope (weight w = c2 + U2)
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = DW[2][q] * rinv;
        to_prime<S>(b, f.U1, f.U2, f.hu2);
        solve<S>(b, f, a);
        mom_t<0, 3, S>(M, Xfs, f, a);
#pragma unroll
        for (int q = 0; q < 5; ++q) Bp[q] -= M[q];
        mom_n<0, S>(M, Xhs, f, a);
        to_lab<S>(M, f.U1, f.U2, f.hu2);
        add5<S>(bz, M);
        mom_t<0, 3, S>(M, Xhs, f, a);
        add5<S>(Bq, M);
        mom_t<1, 3, S>(M, Xhs, f, a);
        add5<S>(Fq, M);
#pragma unroll
        for (int q = 0; q < 5; ++q) ayz[q] = fmaT(f.U2, a[q], ayz[q]);
        mom_n<0, S>(M, Xfs, f, ayz);
#pragma unroll
        for (int q = 0; q < 5; ++q) Bp[q] -= M[q];
    }
    // time-derivative coefficients of this Maxwellian (GKMflux.cpp:142-144)
    S A[5];
    solve<S>(Bp, f, A);
    // its B_ and F contributions (GKMflux.cpp:172-176, 209-212), lab frame
    {
        const S sw45 = S(w45), sg5 = S(g5), sp4 = S(p4), sp5 = S(p5), den = S(g.den);
        S cc[5], M[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) cc[q] = fmaT(sw45, ayz[q], sg5 * A[q]);
        mom_n<0, S>(M, Xhs, f, cc);
#pragma unroll
        for (int q = 0; q < 5; ++q) M[q] = fmaT(sw45, Bq[q], M[q]);
        to_lab<S>(M, f.U1, f.U2, f.hu2);
#pragma unroll
        for (int q = 0; q < 5; ++q) Bs[q] = fmaT(den, M[q], Bs[q]);
#pragma unroll
        for (int q = 0; q < 5; ++q) cc[q] = fmaT(sp4, ayz[q], sp5 * A[q]);
        mom_n<1, S>(M, Xhs, f, cc);
#pragma unroll
        for (int q = 0; q < 5; ++q) M[q] = fmaT(sp4, Fq[q], M[q]);
        to_lab<S>(M, f.U1, f.U2, f.hu2);
#pragma unroll
        for (int q = 0; q < 5; ++q) Fs[q] = fmaT(den, M[q], Fs[q]);
    }
}

// Time-integrated BGK-NS flux through one interface, in the frame of the
// interface normal.  The caller supplies the inputs through `src`, which is
// asked for them only when they are needed, so that one side's inputs are not
// live while the other side is processed:
//   src.state(side, W)      reconstructed state Wl (side 0) or Wr (side 1)
//   src.slopes(side, DW)    its slopes DW[d][q], d = normal, 1st, 2nd transverse
//   src.cells(WL, WR)       the cell averages either side of the interface
// tau0 = mu/p at the left cell.  Output F[5], the flux integrated over [0, dt].
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

    double We[5] = {0, 0, 0, 0, 0}, Fb[5] = {0, 0, 0, 0, 0};
    S by[5] = {0, 0, 0, 0, 0}, bz[5] = {0, 0, 0, 0, 0}, Bs[5] = {0, 0, 0, 0, 0}, Fs[5] = {0, 0, 0, 0, 0};
    flux_side<S, 0>(src, l, c, gm4 + gm5, gm5, p3, p4, p5, We, Fb, by, bz, Bs, Fs);
    flux_side<S, 1>(src, r, c, gm4 + gm5, gm5, p3, p4, p5, We, Fb, by, bz, Bs, Fs);

    // equilibrium state at the interface and its tables (GKMflux.cpp:75-98)
    const Prim e = prim(We, c.gm1);
    double Xf[6], Xp[7], Xn[7];
    full_table<6, double>(e.U0, e.s, Xf);
    {
        // 0.5 erfc(-+x) from one evaluation at |x|: the far tail is computed
        // directly, the other value as 1 - tail (no cancellation)
        const double sl = sqrt(e.lam);
        const double x = sl * e.U0;
        const double tail = 0.5 * erfc(fabs(x));
        const double g = 0.5 * exp(-e.lam * e.U0 * e.U0) * rsqrt(kPi * e.lam);
        half_table<7>(e.U0, e.s, x >= 0.0 ? 1.0 - tail : tail, g, Xp);
        half_table<7>(e.U0, e.s, x >= 0.0 ? tail : 1.0 - tail, -g, Xn);
    }
    // B_ / rho_e in the primed frame of the equilibrium, with its nearly
    // cancelling zeroth-order part gm1 rho_e <psi>_e + gm3 W0 in double
    // (GKMflux.cpp:174-178); p0 term of F (GKMflux.cpp:209)
    double Bd[5];
    {
        const double c4 = fma(0.5, e.U1 * e.U1 + e.U2 * e.U2, double(c.K + 2) * 0.5 * e.s);
        double M[5];
        mom0_lab<0>(M, Xf, e, c4);
        const double w = gm1 * e.den;
#pragma unroll
        for (int q = 0; q < 5; ++q) Bd[q] = (fma(w, M[q], gm3 * We[q]) + double(Bs[q])) * e.rinv;
        to_prime<double>(Bd, e.U1, e.U2, 0.5 * fma(e.U1, e.U1, e.U2 * e.U2));
        mom0_lab<1>(M, Xf, e, c4);
        const double w0 = p0 * e.den;
#pragma unroll
        for (int q = 0; q < 5; ++q) Fb[q] = fma(w0, M[q], Fb[q]);
    }
    const CoFrame<S> f = co_frame<S>(e, c.K, c.kA);
    S Xfs[6], Xps[7], Xns[7];
#pragma unroll
    for (int n = 0; n < 6; ++n) Xfs[n] = S(Xf[n]);
#pragma unroll
    for (int n = 0; n < 7; ++n) {
        Xps[n] = S(Xp[n]);
        Xns[n] = S(Xn[n]);
    }
    // slopes of the equilibrium (GKMflux.cpp:109-117, 136-137)
    S axl[5], axr[5], ay[5], az[5], ayz[5];
    {
        double WL[5], WR[5];
        src.cells(WL, WR);
        const S k2 = S(2.0 * e.rinv / c.dx);
        S b[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = S(We[q] - WL[q]) * k2;
        to_prime<S>(b, f.U1, f.U2, f.hu2);
        solve<S>(b, f, axl);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = S(WR[q] - We[q]) * k2;
        to_prime<S>(b, f.U1, f.U2, f.hu2);
        solve<S>(b, f, axr);
        to_prime<S>(by, f.U1, f.U2, f.hu2);
        solve<S>(by, f, ay);
        to_prime<S>(bz, f.U1, f.U2, f.hu2);
        solve<S>(bz, f, az);
#pragma unroll
        for (int q = 0; q < 5; ++q) ayz[q] = fmaT(f.U1, ay[q], f.U2 * az[q]);
    }
    // A_ (phase III, GKMflux.cpp:159-180)
    S A[5];
    {
        S T1[5], M[5];
        mom_n<1, S>(T1, Xps, f, axl);
        mom_n<1, S>(M, Xns, f, axr);
        add5<S>(T1, M);
        mom_t<0, 2, S>(M, Xfs, f, ay);
        add5<S>(T1, M);
        mom_t<0, 3, S>(M, Xfs, f, az);
        add5<S>(T1, M);
        mom_n<0, S>(M, Xfs, f, ayz);
        add5<S>(T1, M);
        const S g2 = S(gm2);
        S B[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) B[q] = fmaT(g2, T1[q], S(Bd[q]));
        solve<S>(B, f, A);
    }
    // flux (GKMflux.cpp:192-213)
    {
        const S sp1 = S(p1), sp2 = S(p2);
        S T1[5], M[5], cc[5];
        mom_n<2, S>(T1, Xps, f, axl);
        mom_n<2, S>(M, Xns, f, axr);
        add5<S>(T1, M);
        mom_t<1, 2, S>(M, Xfs, f, ay);
        add5<S>(T1, M);
        mom_t<1, 3, S>(M, Xfs, f, az);
        add5<S>(T1, M);
#pragma unroll
        for (int q = 0; q < 5; ++q) cc[q] = fmaT(sp1, A[q], sp2 * ayz[q]);
        mom_n<1, S>(M, Xfs, f, cc);
#pragma unroll
        for (int q = 0; q < 5; ++q) T1[q] = fmaT(sp2, T1[q], M[q]);
        to_lab<S>(T1, f.U1, f.U2, f.hu2);
        const S dens = S(e.den);
#pragma unroll
        for (int q = 0; q < 5; ++q) F[q] = Fb[q] + double(fmaT(dens, T1[q], Fs[q]));
    }
}

} // namespace gks
