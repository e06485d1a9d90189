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

constexpr double kHalfRsqrtPi = 0.28209479177387814; // 1 / (2 sqrt(pi))

// Constants of one Maxwellian in its transverse co-moving frame.  The paired
// type f2 takes no operand negation, so for it the negatives are kept as
// well, making every use a plain fused multiply-add; in double a negated
// operand is free, and the negatives are formed at the use.
template <typename T> struct CoFrame {
    T U0, U1, U2, hu2;     // normal and transverse velocity, hu2 = (U1^2 + U2^2)/2 (to_lab)
    T nU0_, nU1_, nU2_, nhu2_; // their negatives (f2 only)
    T m2U0, nqn, nqh;      // -2 U0, -qn, -qn/2 with qn = U0^2 + (K+3) s (solve)
    T tl, kal2;            // 2 lambda, kA lambda^2 (solve)
    T s, r2, r4, q4;       // 1/(2 lambda), <rho^2>, <rho^4>, <c1^2 rho^2> (moments)
    static constexpr bool kDouble = std::is_same<T, double>::value;
    __device__ __forceinline__ T nU0() const { if constexpr (kDouble) return -U0; else return nU0_; }
    __device__ __forceinline__ T nU1() const { if constexpr (kDouble) return -U1; else return nU1_; }
    __device__ __forceinline__ T nU2() const { if constexpr (kDouble) return -U2; else return nU2_; }
    __device__ __forceinline__ T nhu2() const { if constexpr (kDouble) return -hu2; else return nhu2_; }
};

template <typename T, typename KT>
__device__ __forceinline__ CoFrame<T> co_frame(T U0, T U1, T U2, T s, T lam, const KConst<KT> &kc, T kA)
{
    CoFrame<T> f;
    f.U0 = U0;
    f.U1 = U1;
    f.U2 = U2;
    f.hu2 = T(0.5f) * fmaT(U1, U1, U2 * U2);
    const T m1 = T(-1.0f);
    if constexpr (!CoFrame<T>::kDouble) {
        f.nU0_ = m1 * U0;
        f.nU1_ = m1 * U1;
        f.nU2_ = m1 * U2;
        f.nhu2_ = m1 * f.hu2;
    }
    f.m2U0 = T(-2.0f) * U0;
    f.nqn = fmaT(f.nU0(), U0, T(kc.nq) * s);
    f.nqh = T(0.5f) * f.nqn;
    f.tl = T(2.0f) * lam;
    f.kal2 = (kA * lam) * lam;
    f.s = s;
    f.r2 = T(kc.r2) * s;
    const T s2 = s * s;
    f.q4 = T(kc.q4) * s2;
    f.r4 = T(kc.r4) * s2;
    return f;
}

// Primed -> lab frame of a moment vector (m = T m').
template <typename T>
__device__ __forceinline__ void to_lab(T m[5], const CoFrame<T> &f)
{
    m[4] = fmaT(f.U1, m[2], fmaT(f.U2, m[3], fmaT(f.hu2, m[0], m[4])));
    m[2] = fmaT(f.U1, m[0], m[2]);
    m[3] = fmaT(f.U2, m[0], m[3]);
}

// Lab -> primed frame of a slope right-hand side (b' = T^-1 b).
template <typename T>
__device__ __forceinline__ void to_prime(T b[5], T nU1, T nU2, T nhu2)
{
    b[2] = fmaT(nU1, b[0], b[2]);
    b[3] = fmaT(nU2, b[0], b[3]);
    b[4] = fmaT(nU1, b[2], fmaT(nU2, b[3], fmaT(nhu2, b[0], b[4])));
}

template <typename T>
__device__ __forceinline__ void to_prime(T b[5], const CoFrame<T> &f)
{
    to_prime<T>(b, f.nU1(), f.nU2(), f.nhu2());
}

// Slope solve (slopesolver, GKMflux.cpp:280-296) in the primed frame: the
// coefficients a' with <psi' psi'> a' = b' for the Maxwellian moving with
// (U0, 0, 0); kal2 carries the energy-coefficient factor (1/Pr at
// GKMflux.cpp:289, or 1).
template <typename T>
__device__ __forceinline__ void solve(const T b[5], const CoFrame<T> &f, T a[5])
{
    const T R2 = fmaT(f.nU0(), b[0], b[1]);
    const T R5 = fmaT(f.nqn, b[0], T(2.0f) * b[4]);
    a[4] = f.kal2 * fmaT(f.m2U0, R2, R5);
    a[3] = f.tl * b[3];
    a[2] = f.tl * b[2];
    a[1] = fmaT(f.nU0(), a[4], f.tl * R2);
    a[0] = fmaT(f.nU0(), a[1], fmaT(f.nqh, a[4], b[0]));
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

// acc += M with M = mom_n<k>(X, a), every product fused into the sum.
template <int k, typename T>
__device__ __forceinline__ void acc_mom_n(T acc[5], const T *X, const CoFrame<T> &f, const T a[5])
{
    const T h = T(0.5f) * a[4];
    const T al = fmaT(h, f.r2, a[0]);
    acc[0] = fmaT(al, X[k], fmaT(a[1], X[k + 1], fmaT(h, X[k + 2], acc[0])));
    acc[1] = fmaT(al, X[k + 1], fmaT(a[1], X[k + 2], fmaT(h, X[k + 3], acc[1])));
    const T sx = f.s * X[k];
    acc[2] = fmaT(a[2], sx, acc[2]);
    acc[3] = fmaT(a[3], sx, acc[3]);
    const T c2 = fmaT(h, f.r2, al);
    const T c0 = fmaT(a[0], f.r2, h * f.r4);
    acc[4] = fmaT(T(0.5f), fmaT(c2, X[k + 2], fmaT(c0, X[k], fmaT(a[1], fmaT(f.r2, X[k + 1], X[k + 3]), h * X[k + 4]))),
                  acc[4]);
}

// acc += <psi' u^k c_D (a.psi')>, D = 2 (c1) or 3 (c2); component 5 - D of
// the moment vanishes and is skipped:
//   M0 = aD s X[k],  M1 = aD s X[k+1]
//   M_D = s (a0 X[k] + a1 X[k+1] + h X[k+2]) + h q4 X[k]
//   M4 = aD (s X[k+2] + q4 X[k]) / 2
template <int k, int D, typename T>
__device__ __forceinline__ void acc_mom_t(T acc[5], const T *X, const CoFrame<T> &f, const T a[5])
{
    const T h = T(0.5f) * a[4];
    const T sa = f.s * a[D];
    acc[0] = fmaT(sa, X[k], acc[0]);
    acc[1] = fmaT(sa, X[k + 1], acc[1]);
    acc[D] = fmaT(f.s, fmaT(a[0], X[k], fmaT(a[1], X[k + 1], h * X[k + 2])), fmaT(h * f.q4, X[k], acc[D]));
    acc[4] = fmaT(T(0.5f) * a[D], fmaT(f.s, X[k + 2], f.q4 * X[k]), acc[4]);
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

// Weights of the time integration (GKMflux.cpp:155-157, 186-190) that the
// side passes use; the equilibrium pass forms its own from tau, ex, om, igm0.
struct SideWeights {
    double w45, g5, p3, p4, p5; // gm4 + gm5, gm5, p3, p4, p5
};

// Double part of the pass over one initial Maxwellian (NEG = 0: left state,
// half space u > 0; NEG = 1: right state, u < 0): its primitive state, its
// normal-velocity tables -- half space (GKMflux.cpp:52-60) and full space --
// and its share of W0 (GKMflux.cpp:71-75) and of the p3 flux term
// (GKMflux.cpp:209-212), added to the double sums of `src` (slots 0-4, 5-9).
template <int NEG, typename Src>
__device__ __forceinline__ Prim side_tables(const Src &src, const FluxConst &c, double p3, double Xh[7], double Xf[6])
{
    constexpr bool FIRST = NEG == 0;
    double W[5];
    src.state(NEG, W);
    const Prim g = prim(W, c.gm1, c.hig);
    {
        // one reciprocal square root: sqrt(lambda) = lambda / sqrt(lambda)
        const double rl = rsqrt(g.lam), sl = g.lam * rl;
        const double x = NEG ? sl * g.U0 : -sl * g.U0; // h0 = 0.5 erfc(x)
        const double e2 = exp(-g.lam * g.U0 * g.U0);
        double h0, hm;
        half_erfc_pm(x, e2, h0, hm);
        const double ex = e2 * (kHalfRsqrtPi * rl);
        half_table<7>(g.U0, g.s, h0, NEG ? -ex : ex, Xh);
    }
    full_table<6, double>(g.U0, g.s, Xf);
    const double c4 = fma(0.5, fma(g.U1, g.U1, g.U2 * g.U2), c.hK2 * g.s);
    double M[5];
    mom0_lab<0>(M, Xh, g, c4);
#pragma unroll
    for (int q = 0; q < 5; ++q) src.template put_d<FIRST>(q, g.den, M[q]);
    mom0_lab<1>(M, Xh, g, c4);
    const double w = p3 * g.den;
#pragma unroll
    for (int q = 0; q < 5; ++q) src.template put_d<FIRST>(5 + q, w, M[q]);
    return g;
}

// Slope part of the side pass, on the arithmetic type T of the flux assembly:
// double (one Maxwellian), or f2 (the left and right Maxwellians as the two
// lanes of paired FP32 instructions).  `io` supplies the state differences,
//   io.slope(d, b)        along d = normal, 1st, 2nd transverse, which
// sc[d] = ks[d] / rho turns into the right-hand sides b = DW / rho,
// and takes the lab-frame results,
//   io.emit(slot, den, M) adds den * M to S sum slot `slot` (lanes summed):
// the transverse right-hand sides by_, bz_ of the equilibrium slopes (slots
// 0-4, 5-9), B_ (10-14) and the p4 / p5 flux terms (15-19).
template <typename T, typename IO>
__device__ __forceinline__ void side_slopes(const IO &io, const CoFrame<T> &f, const T *Xh, const T *Xf,
                                            const T sc[3], T den, T w45, T g5, T p4, T p5)
{
    // slope coefficients (phase I, GKMflux.cpp:102-117) and the moment sums they
    // feed, in the primed frame: Bm = -B -> A (phase II, GKMflux.cpp:128-144),
    // Bq -> B_ (GKMflux.cpp:172-173), Fq -> F (GKMflux.cpp:210-211);
    // ayz = U1 ay + U2 az collects the v / w weights' shift.
    T Bm[5], Bq[5], Fq[5], ayz[5];
    {
        T a[5], b[5], M[5];
        const T one(1.0f);
        // normal slope
        io.slope(0, b);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] *= sc[0];
        to_prime<T>(b, f);
        solve<T>(b, f, a);
        mom_n<1, T>(Bm, Xf, f, a);
        mom_n<1, T>(Bq, Xh, f, a);
        mom_n<2, T>(Fq, Xh, f, a);
        // first transverse slope (weight v = c1 + U1)
        io.slope(1, b);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] *= sc[1];
        to_prime<T>(b, f);
        solve<T>(b, f, a);
        acc_mom_t<0, 2, T>(Bm, Xf, f, a);
        mom_n<0, T>(M, Xh, f, a);
        to_lab<T>(M, f);
#pragma unroll
        for (int q = 0; q < 5; ++q) io.emit(q, one, M[q]);
        acc_mom_t<0, 2, T>(Bq, Xh, f, a);
        acc_mom_t<1, 2, T>(Fq, Xh, f, a);
#pragma unroll
        for (int q = 0; q < 5; ++q) ayz[q] = f.U1 * a[q];
        // second transverse slope (weight w = c2 + U2)
        io.slope(2, b);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] *= sc[2];
        to_prime<T>(b, f);
        solve<T>(b, f, a);
        acc_mom_t<0, 3, T>(Bm, Xf, f, a);
        mom_n<0, T>(M, Xh, f, a);
        to_lab<T>(M, f);
#pragma unroll
        for (int q = 0; q < 5; ++q) io.emit(5 + q, one, M[q]);
        acc_mom_t<0, 3, T>(Bq, Xh, f, a);
        acc_mom_t<1, 3, T>(Fq, Xh, f, a);
#pragma unroll
        for (int q = 0; q < 5; ++q) ayz[q] = fmaT(f.U2, a[q], ayz[q]);
        acc_mom_n<0, T>(Bm, Xf, f, ayz);
    }
    // time-derivative coefficients of this Maxwellian (GKMflux.cpp:142-144):
    // An = -A from Bm = -B
    T An[5];
    solve<T>(Bm, f, An);
    // its B_ and F contributions (GKMflux.cpp:172-176, 209-212), lab frame
    {
        T cc[5], M[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) cc[q] = fmaT(w45, ayz[q], g5 * An[q]);
        mom_n<0, T>(M, Xh, f, cc);
#pragma unroll
        for (int q = 0; q < 5; ++q) M[q] = fmaT(w45, Bq[q], M[q]);
        to_lab<T>(M, f);
#pragma unroll
        for (int q = 0; q < 5; ++q) io.emit(10 + q, den, M[q]);
#pragma unroll
        for (int q = 0; q < 5; ++q) cc[q] = fmaT(p4, ayz[q], p5 * An[q]);
        mom_n<1, T>(M, Xh, f, cc);
#pragma unroll
        for (int q = 0; q < 5; ++q) M[q] = fmaT(p4, Fq[q], M[q]);
        to_lab<T>(M, f);
#pragma unroll
        for (int q = 0; q < 5; ++q) io.emit(15 + q, den, M[q]);
    }
}

// Slope inputs and results of one side pass in double.
template <int NEG, typename Src>
struct SideIO64 {
    const Src &src;
    __device__ __forceinline__ void slope(int d, double b[5]) const { src.slope(NEG, d, b); }
    __device__ __forceinline__ void emit(int slot, double a, double m) const
    {
        src.template put_s<NEG == 0>(slot, a, m);
    }
};

// Slope inputs and results of the paired side pass (left lane .x, right .y);
// the lane-summed results stay in the caller's registers (out[20]).
template <typename Src>
struct SideIO2 {
    const Src &src;
    float *out;
    __device__ __forceinline__ void slope(int d, f2 b[5]) const
    {
        float l[5], r[5];
        src.slope(0, d, l);
        src.slope(1, d, r);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = f2(l[q], r[q]);
    }
    __device__ __forceinline__ void emit(int slot, f2 a, f2 m) const
    {
        out[slot] = __fmaf_rn(a.v.y, m.v.y, __fmul_rn(a.v.x, m.v.x));
    }
};

// The two side passes of the FP64 path, one after the other; the equilibrium
// pass reads the parked sums behind a compiler memory barrier, so that the
// scheduler cannot start its long erfc / exp chains early and keep the side
// passes' state live at the same time.
template <typename Src>
__device__ __forceinline__ void flux_sides(const Src &src, const FluxConst &c, const SideWeights &tw, double, float *)
{
    {
        double Xh[7], Xf[6];
        const Prim g = side_tables<0>(src, c, tw.p3, Xh, Xf);
        const CoFrame<double> f = co_frame<double>(g.U0, g.U1, g.U2, g.s, g.lam, c.kd, c.kA);
        const double sc[3] = {c.ks[0] * g.rinv, c.ks[1] * g.rinv, c.ks[2] * g.rinv};
        side_slopes<double>(SideIO64<0, Src>{src}, f, Xh, Xf, sc, g.den, tw.w45, -tw.g5, tw.p4, -tw.p5);
    }
    {
        double Xh[7], Xf[6];
        const Prim g = side_tables<1>(src, c, tw.p3, Xh, Xf);
        const CoFrame<double> f = co_frame<double>(g.U0, g.U1, g.U2, g.s, g.lam, c.kd, c.kA);
        const double sc[3] = {c.ks[0] * g.rinv, c.ks[1] * g.rinv, c.ks[2] * g.rinv};
        side_slopes<double>(SideIO64<1, Src>{src}, f, Xh, Xf, sc, g.den, tw.w45, -tw.g5, tw.p4, -tw.p5);
    }
    asm volatile("" ::: "memory");
}

// The mixed path: the double parts of the two side passes (their erfc / exp
// chains overlap), then their FP32 slope parts together as the lanes of
// paired instructions.
template <typename Src>
__device__ __forceinline__ void flux_sides(const Src &src, const FluxConst &c, const SideWeights &tw, float, float *sout)
{
    f2 Xh[7], Xf[6];
    f2 U0, U1, U2, s, lam, rinv, den;
    {
        double XhL[7], XfL[6];
        const Prim g = side_tables<0>(src, c, tw.p3, XhL, XfL);
#pragma unroll
        for (int n = 0; n < 7; ++n) Xh[n].v.x = float(XhL[n]);
#pragma unroll
        for (int n = 0; n < 6; ++n) Xf[n].v.x = float(XfL[n]);
        U0.v.x = float(g.U0); U1.v.x = float(g.U1); U2.v.x = float(g.U2);
        s.v.x = float(g.s); lam.v.x = float(g.lam); rinv.v.x = float(g.rinv); den.v.x = float(g.den);
    }
    {
        double XhR[7], XfR[6];
        const Prim g = side_tables<1>(src, c, tw.p3, XhR, XfR);
#pragma unroll
        for (int n = 0; n < 7; ++n) Xh[n].v.y = float(XhR[n]);
#pragma unroll
        for (int n = 0; n < 6; ++n) Xf[n].v.y = float(XfR[n]);
        U0.v.y = float(g.U0); U1.v.y = float(g.U1); U2.v.y = float(g.U2);
        s.v.y = float(g.s); lam.v.y = float(g.lam); rinv.v.y = float(g.rinv); den.v.y = float(g.den);
    }
    const CoFrame<f2> f = co_frame<f2>(U0, U1, U2, s, lam, c.kf, f2(float(c.kA)));
    const f2 sc[3] = {f2(float(c.ks[0])) * rinv, f2(float(c.ks[1])) * rinv, f2(float(c.ks[2])) * rinv};
    side_slopes<f2>(SideIO2<Src>{src, sout}, f, Xh, Xf, sc, den, f2(float(tw.w45)), f2(float(-tw.g5)),
                    f2(float(tw.p4)), f2(float(-tw.p5)));
    asm volatile("" ::: "memory");
}

// The field's K constants in the type of the flux assembly.
template <typename S> __device__ __forceinline__ const KConst<S> &kconst(const FluxConst &c);
template <> __device__ __forceinline__ const KConst<double> &kconst<double>(const FluxConst &c) { return c.kd; }
template <> __device__ __forceinline__ const KConst<float> &kconst<float>(const FluxConst &c) { return c.kf; }

// Time-integrated BGK-NS flux through one interface, in the frame of the
// interface normal.  `src` supplies the inputs when they are needed, so that
// one side's inputs are not live while the other side is processed, and keeps
// the running sums of the two side passes:
//   src.state(side, W)        reconstructed state Wl (side 0) or Wr (side 1)
//   src.slope(side, d, DW)    its slopes along d = normal, 1st, 2nd transverse
//   src.cells(WL, WR)         the cell averages either side of the interface
//   src.put_d / put_s<FIRST>(slot, v), get_d / get_s(slot)   running sums
// (the mixed path keeps its type-S sums in registers: the paired side pass
// produces them all at once).
// mu/p at the left cell = tau_n / tau_d.  Output F[5], the flux integrated over [0, dt].
template <typename S, typename Src>
__device__ __forceinline__ void gks_flux(const Src &src, double tau_n, double tau_d, const FluxConst &c, double F[5])
{
    const double dt = c.dt;
    double tau, ex, om, igm0;
    SideWeights tw;
    {
        // collision time with the pressure-jump term (GKMflux.cpp:149-150):
        // rho/lambda = 2p, so w = |p_l - p_r| / (p_l + p_r); with
        // p = (gamma - 1) A / rho, A = rho2p(W), multiplied through by
        // rho_l rho_r / (gamma - 1): w = |A_l rho_r - A_r rho_l| / (A_l rho_r + A_r rho_l)
        double W[5];
        src.state(0, W);
        const double Al = rho2p(W), rl = W[0];
        src.state(1, W);
        const double a = Al * W[0], b = rho2p(W) * rl;
        // tau = tau_n / tau_d + dt w = N / D; one reciprocal r = 1 / (N D) gives
        // tau = N (N r) and 1 / tau = D (D r)
        const double D = tau_d * (a + b);
        const double N = fma(tau_n, a + b, dt * fabs(a - b) * tau_d);
        const double r = rcp<double>(N * D);
        tau = N * (N * r);
        ex = exp(-dt * (D * (D * r)));
        om = 1.0 - ex;
        // gamma weights (GKMflux.cpp:155-157) and time integrals (GKMflux.cpp:186-190)
        const double Pt = tau * om;
        igm0 = rcp<double>(dt - Pt);
        const double gm3 = om * igm0;
        const double gm4 = fma(dt, ex, -Pt) * igm0;
        tw.g5 = tau * gm3;
        tw.w45 = gm4 + tw.g5;
        const double Qt = tau * fma(-dt, ex, Pt);
        tw.p3 = Pt;
        tw.p4 = fma(-tau, Pt, -Qt);
        tw.p5 = -tau * Pt;
    }
    float sreg[20];
    flux_sides(src, c, tw, S(), sreg);
    auto gets = [&](int k) -> S {
        if constexpr (sizeof(S) == 4) return sreg[k];
        else return src.get_s(k);
    };
    const double gm1 = -om * igm0, gm3 = -gm1;
    const double Pt = tau * om, Qt = tau * fma(-dt, ex, Pt);
    const double gm2 = fma(-dt, ex, fma(2.0, Pt, -dt)) * igm0;
    const double p0 = dt - Pt;
    const double p1 = fma(0.5 * dt, dt, -tau * p0);
    const double p2 = fma(-tau, p0, Qt);

    // equilibrium state at the interface and its tables (GKMflux.cpp:75-98)
    double We[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) We[q] = src.get_d(q);
    const Prim e = prim(We, c.gm1, c.hig);
    double Xf[6], Xp[7], Xn[7];
    full_table<6, double>(e.U0, e.s, Xf);
    {
        // 0.5 erfc(-+x) from one evaluation (half_erfc_pm)
        const double rl = rsqrt(e.lam), sl = e.lam * rl;
        const double x = sl * e.U0;
        const double e2 = exp(-e.lam * e.U0 * e.U0);
        double hp, hm;
        half_erfc_pm(x, e2, hp, hm);
        const double g = e2 * (kHalfRsqrtPi * rl);
        half_table<7>(e.U0, e.s, hm, g, Xp);
        half_table<7>(e.U0, e.s, hp, -g, Xn);
    }
    const double c4 = fma(0.5, fma(e.U1, e.U1, e.U2 * e.U2), c.hK2 * e.s);
    // B_ / rho_e in the primed frame of the equilibrium, with its nearly
    // cancelling zeroth-order part gm1 rho_e <psi>_e + gm3 W0 in double
    // (GKMflux.cpp:174-178)
    double Bd[5];
    {
        double M[5];
        mom0_lab<0>(M, Xf, e, c4);
        const double w = gm1 * e.den;
#pragma unroll
        for (int q = 0; q < 5; ++q) Bd[q] = (fma(w, M[q], gm3 * We[q]) + double(gets(10 + q))) * e.rinv;
        to_prime<double>(Bd, -e.U1, -e.U2, -0.5 * fma(e.U1, e.U1, e.U2 * e.U2));
    }
    const CoFrame<S> f = co_frame<S>(S(e.U0), S(e.U1), S(e.U2), S(e.s), S(e.lam), kconst<S>(c), S(c.kA));
    S Xfs[6], Xps[7], Xns[7];
#pragma unroll
    for (int n = 0; n < 6; ++n) Xfs[n] = S(Xf[n]);
#pragma unroll
    for (int n = 0; n < 7; ++n) {
        Xps[n] = S(Xp[n]);
        Xns[n] = S(Xn[n]);
    }
    // slopes of the equilibrium (GKMflux.cpp:109-117, 136-137)
    asm volatile("" ::: "memory"); // parked cell averages and sums are read from here on
    S axl[5], axr[5], ay[5], az[5], ayz[5];
    {
        double WL[5], WR[5];
        src.cells(WL, WR);
        const S k2 = S(c.ks[0] * e.rinv); // 2 / (rho_e dx)
        S b[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = S(We[q] - WL[q]) * k2;
        to_prime<S>(b, f);
        solve<S>(b, f, axl);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = S(WR[q] - We[q]) * k2;
        to_prime<S>(b, f);
        solve<S>(b, f, axr);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = gets(q);
        to_prime<S>(b, f);
        solve<S>(b, f, ay);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = gets(5 + q);
        to_prime<S>(b, f);
        solve<S>(b, f, az);
#pragma unroll
        for (int q = 0; q < 5; ++q) ayz[q] = fmaT(f.U1, ay[q], f.U2 * az[q]);
    }
    // A_ (phase III, GKMflux.cpp:159-180)
    S A[5];
    {
        S T1[5];
        mom_n<1, S>(T1, Xps, f, axl);
        acc_mom_n<1, S>(T1, Xns, f, axr);
        acc_mom_t<0, 2, S>(T1, Xfs, f, ay);
        acc_mom_t<0, 3, S>(T1, Xfs, f, az);
        acc_mom_n<0, S>(T1, Xfs, f, ayz);
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
        acc_mom_n<2, S>(T1, Xns, f, axr);
        acc_mom_t<1, 2, S>(T1, Xfs, f, ay);
        acc_mom_t<1, 3, S>(T1, Xfs, f, az);
#pragma unroll
        for (int q = 0; q < 5; ++q) cc[q] = fmaT(sp1, A[q], sp2 * ayz[q]);
        mom_n<1, S>(M, Xfs, f, cc);
#pragma unroll
        for (int q = 0; q < 5; ++q) T1[q] = fmaT(sp2, T1[q], M[q]);
        to_lab<S>(T1, f);
        const S dens = S(e.den);
        asm volatile("" ::: "memory"); // the parked flux sums are read from here on
        double M0[5];
        mom0_lab<1>(M0, Xf, e, c4);
        const double w0 = p0 * e.den;
#pragma unroll
        for (int q = 0; q < 5; ++q)
            F[q] = fma(w0, M0[q], src.get_d(5 + q)) + double(fmaT(dens, T1[q], gets(15 + q)));
    }
}

} // namespace gks
