// Mixed FP32/FP64 BGK-NS interface flux (GKMflux.cpp:11-215), organised for
// paired FP32 instructions.
//
// FP64: primitive states, collision time and time weights, every moment table
// (full-space recursion, erfc / exp half-space seeds and their recursion),
// the zeroth-order moment vectors (equilibrium state W0, the p0 and p3 flux
// terms, the gm1 and gm3 terms of B_) and the flux accumulation.
// FP32: the slope and non-equilibrium coefficient solves and every
// slope-weighted moment vector (the rest of the flux assembly).
//
// The left and right Maxwellians are processed one after the other in
// scalar FP32 (flux_side); on the equilibrium side, where the side tables are
// dead, the FP32 work runs on pairs (type f2, one f32x2 instruction for two
// lanes):
//  * <u^k psi (ax_l.psi)>_{u>0} and
//    <u^k psi (ax_r.psi)>_{u<0} share one pass (Xp | Xn tables), and so do
//    the y- and z-slope terms, the z term written as a y term of the frame
//    with v and w exchanged: <psi w^m (az.psi)> = P <psi v^m (P az.psi)>
//    with P swapping components 2 and 3 and the Y and Z tables.
#pragma once

#include "gks_device.cuh"

namespace gks {

__device__ __forceinline__ f2 pk(double a, double b) { return f2(float(a), float(b)); }

// index of the component that holds component q after exchanging v and w
__device__ __forceinline__ constexpr int swap23(int q) { return q == 2 ? 3 : (q == 3 ? 2 : q); }

template <typename Src>
__device__ __forceinline__ void gks_flux_mixed(const Src &src, double tau0, const FluxConst &c, double F[5])
{
    Prim l, r;
    {
        double Ws[5];
        src.state(0, Ws);
        l = prim(Ws, c.gm1);
        src.state(1, Ws);
        r = prim(Ws, c.gm1);
    }
    // collision time and time weights in FP64 (GKMflux.cpp:149-157, 186-190)
    const double dt = c.dt;
    const double tau = tau0 + dt * (fabs(l.P - r.P) * rcp<double>(l.P + r.P));
    const double ex = exp(-dt * rcp<double>(tau));
    const double om = 1.0 - ex;
    const double igm0 = rcp<double>(dt - tau * om);
    const double gm1 = -om * igm0;
    const double gm2 = (-dt + 2.0 * tau * om - dt * ex) * igm0;
    const double gm3 = -gm1;
    const double gm4 = (dt * ex - tau * om) * igm0;
    const double gm5 = tau * gm3;
    const double Pt = tau * om;
    const double Qt = tau * (tau * om - dt * ex);
    const double p0 = dt - Pt;
    const double p1 = 0.5 * dt * dt - tau * p0;
    const double p2 = -tau * p0 + Qt;
    const double p3 = Pt;
    const double p4 = -Qt - tau * Pt;
    const double p5 = -tau * Pt;

    // left and right Maxwellians one after the other (the scalar FP32 side
    // pass of gks_flux; running them as pair lanes doubles the live state)
    double We[5] = {0, 0, 0, 0, 0}, Fbase[5] = {0, 0, 0, 0, 0};
    float by_[5] = {0, 0, 0, 0, 0}, bz_[5] = {0, 0, 0, 0, 0}, Bs[5] = {0, 0, 0, 0, 0}, Fs[5] = {0, 0, 0, 0, 0};
    flux_side<float, 0>(src, l, c, gm4 + gm5, gm5, p3, p4, p5, We, Fbase, by_, bz_, Bs, Fs);
    flux_side<float, 1>(src, r, c, gm4 + gm5, gm5, p3, p4, p5, We, Fbase, by_, bz_, Bs, Fs);

    // equilibrium state at the interface (GKMflux.cpp:71-98), tables in FP64
    const Prim e = prim(We, c.gm1);
    f2 Xpn[7], Xe[6], Yy[6], Zz[6], Yz[6], Zy[6];
    float ee2, ee4;
    double Bbase[5];
    {
        double Ye[6], Ze[6], Xfe[6], Xp[7], Xn[7];
        full_table<6>(e.U1, e.s, Ye);
        full_table<6>(e.U2, e.s, Ze);
        full_table<6>(e.U0, e.s, Xfe);
        const double e2d = double(c.K) * e.s;
        {
            // 0.5 erfc(-+x) from one evaluation at |x| (the far tail directly, the other as 1 - tail)
            const double sl = sqrt(e.lam);
            const double x = sl * e.U0;
            const double tail = 0.5 * erfc(fabs(x));
            const double g = 0.5 * exp(-e.lam * e.U0 * e.U0) * rsqrt(kPi * e.lam);
            half_table<7>(e.U0, e.s, x >= 0.0 ? 1.0 - tail : tail, g, Xp);
            half_table<7>(e.U0, e.s, x >= 0.0 ? tail : 1.0 - tail, -g, Xn);
        }
        double M0[5], M1[5];
        mcal0<0, 0, 0, double>(M0, Xfe, Ye, Ze, e2d);
        mcal0<1, 0, 0, double>(M1, Xfe, Ye, Ze, e2d);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            Bbase[q] = gm1 * e.den * M0[q] + gm3 * We[q];
            Fbase[q] += p0 * e.den * M1[q];
        }
#pragma unroll
        for (int n = 0; n < 7; ++n) Xpn[n] = pk(Xp[n], Xn[n]);
#pragma unroll
        for (int n = 0; n < 6; ++n) {
            const float xf = float(Xfe[n]), y = float(Ye[n]), z = float(Ze[n]);
            Xe[n] = f2(xf);
            Yy[n] = f2(y);
            Zz[n] = f2(z);
            Yz[n] = f2(y, z);
            Zy[n] = f2(z, y);
        }
        ee2 = float(e2d);
        ee4 = float(double(c.K * (c.K + 2)) * e.s * e.s);
    }
    const float U0 = float(e.U0), U1 = float(e.U1), U2 = float(e.U2), lam = float(e.lam), es = float(e.s);
    const float kA = float(c.kA);
    // ax_l | ax_r share the equilibrium frame; ay | az share it with v and w exchanged in lane .y
    const SlopeFrame<f2> fxx = slope_frame<f2>(f2(U0), f2(U1), f2(U2), f2(lam), f2(es), c.K, f2(kA));
    const SlopeFrame<f2> fyz = slope_frame<f2>(f2(U0), f2(U1, U2), f2(U2, U1), f2(lam), f2(es), c.K, f2(kA));
    f2 axlr[5], ayz[5];
    {
        double WL[5], WR[5];
        src.cells(WL, WR);
        const double k2 = 2.0 * e.rinv * (1.0 / c.dx); // GKMflux.cpp:109-110
        f2 b[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = pk((We[q] - WL[q]) * k2, (WR[q] - We[q]) * k2);
        slope_solve<f2>(b, fxx, axlr);
#pragma unroll
        for (int q = 0; q < 5; ++q) b[q] = f2(by_[q], bz_[swap23(q)]);
        slope_solve<f2>(b, fyz, ayz);
    }
    const f2 e2p(ee2), e4p(ee4);
    // A_ (phase III, GKMflux.cpp:159-180)
    float Ae[5];
    {
        f2 T1[5], M[5];
        mcal_a<1, 0, 0, f2>(T1, Xpn, Yy, Zz, e2p, e4p, axlr);
        mcal_a<0, 1, 0, f2>(M, Xe, Yz, Zy, e2p, e4p, ayz);
        const float w = float(gm2 * e.den);
        float B[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const float t = T1[q].v.x + T1[q].v.y + M[q].v.x + M[swap23(q)].v.y;
            B[q] = float((Bbase[q] + double(fmaf(w, t, Bs[q]))) * e.rinv);
        }
        const SlopeFrame<float> fe = slope_frame<float>(U0, U1, U2, lam, es, c.K, kA);
        slope_solve<float>(B, fe, Ae);
    }
    // flux (GKMflux.cpp:192-213)
    {
        f2 T1[5], M[5];
        mcal_a<2, 0, 0, f2>(T1, Xpn, Yy, Zz, e2p, e4p, axlr);
        mcal_a<1, 1, 0, f2>(M, Xe, Yz, Zy, e2p, e4p, ayz);
        float Xs[6], Ys[6], Zs[6], N[5];
#pragma unroll
        for (int n = 0; n < 6; ++n) {
            Xs[n] = Xe[n].v.x;
            Ys[n] = Yy[n].v.x;
            Zs[n] = Zz[n].v.x;
        }
        mcal_a<1, 0, 0, float>(N, Xs, Ys, Zs, ee2, ee4, Ae);
        const float w2 = float(p2 * e.den), w1 = float(p1 * e.den);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const float t = T1[q].v.x + T1[q].v.y + M[q].v.x + M[swap23(q)].v.y;
            F[q] = Fbase[q] + double(fmaf(w2, t, fmaf(w1, N[q], Fs[q])));
        }
    }
}

} // namespace gks
