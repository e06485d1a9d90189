/*
 * CPU oracle for the GKM-DNS WENO-GKS step (declarations and scope in
 * gks_oracle.h).  TEST INFRASTRUCTURE ONLY: never part of the product path.
 *
 * Every routine cites the reference lines it restates.  Formulas keep the
 * reference's operation order; the only intended deviations are skipping work
 * whose result the reference never reads (half-space tables of the transverse
 * velocity components, GKMflux.cpp:54-57 for j = 1, 2), which cannot change
 * any output.
 */
#include "gks_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NQ 5

/* ---------------------------------------------------------------------------
 * Conservative -> primitive (GKMflux.cpp:301-308).
 * ------------------------------------------------------------------------- */
static void prim(const double *W, double gam, double *den, double U[3], double *P)
{
    const double d = W[0];
    U[0] = W[1] / d;
    U[1] = W[2] / d;
    U[2] = W[3] / d;
    *den = d;
    *P = (d * (gam - 1)) * (W[4] / d - 0.5 * (U[0] * U[0] + U[1] * U[1] + U[2] * U[2]));
}

/* ---------------------------------------------------------------------------
 * One Maxwellian: its velocity moments (GKMflux.cpp:40-66, 77-98).
 *   full[j][n] = <u_j^n>              over all velocities
 *   pos[n]     = <u_0^n>              over u_0 > 0
 *   neg[n]     = <u_0^n>              over u_0 < 0
 *   e2, e4     = <xi^2>, <xi^4>       internal degrees of freedom
 * ------------------------------------------------------------------------- */
typedef struct {
    double den, P, lam;
    double U[3];
    double e2, e4;
    double full[3][7];
    double pos[7];
    double neg[7];
} maxwellian;

static void moments(maxwellian *g, int K, int want_pos, int want_neg)
{
    const double lam = g->lam;
    g->e2 = K / (2 * lam);
    g->e4 = 3 * K / (4 * lam * lam) + K * (K - 1) / (4 * lam * lam);
    for (int j = 0; j < 3; ++j) {
        const double u = g->U[j];
        double *f = g->full[j];
        f[0] = 1.0;
        f[1] = u;
        for (int n = 2; n < 7; ++n) f[n] = u * f[n - 1] + f[n - 2] * (n - 1) / (2 * lam);
    }
    const double u = g->U[0];
    if (want_pos) {
        double *h = g->pos;
        h[0] = 0.5 * (erfc(-sqrt(lam) * u));
        h[1] = u * h[0] + 0.5 * exp(-lam * u * u) / sqrt(lam * atan(1.0) * 4.0);
        for (int n = 2; n < 7; ++n) h[n] = u * h[n - 1] + h[n - 2] * (n - 1) / (2 * lam);
    }
    if (want_neg) {
        double *h = g->neg;
        h[0] = 0.5 * (erfc(sqrt(lam) * u));
        h[1] = u * h[0] - 0.5 * exp(-lam * u * u) / sqrt(lam * atan(1.0) * 4.0);
        for (int n = 2; n < 7; ++n) h[n] = u * h[n - 1] + h[n - 2] * (n - 1) / (2 * lam);
    }
}

/* ---------------------------------------------------------------------------
 * Moment vectors <psi u^k v^l w^m (a . psi)> with psi = (1,u,v,w,(u^2+v^2+w^2+xi^2)/2)
 * (MCal, GKMflux.cpp:225-275).  X is the normal-velocity table (full or half
 * space), Y and Z the full tables of the transverse components.
 * ------------------------------------------------------------------------- */
static inline double t3(const double *X, const double *Y, const double *Z, int a, int b, int c)
{
    return X[a] * Y[b] * Z[c];
}

static void mom0(double M[5], const double *X, const double *Y, const double *Z, double e2,
                 int k, int l, int m)
{
    const double v0 = 0.5 * (t3(X, Y, Z, 2 + k, l, m) + t3(X, Y, Z, k, 2 + l, m) +
                             t3(X, Y, Z, k, l, 2 + m) + t3(X, Y, Z, k, l, m) * e2);
    M[0] = t3(X, Y, Z, k, l, m);
    M[1] = t3(X, Y, Z, 1 + k, l, m);
    M[2] = t3(X, Y, Z, k, 1 + l, m);
    M[3] = t3(X, Y, Z, k, l, 1 + m);
    M[4] = v0;
}

static void mom(double M[5], const double *X, const double *Y, const double *Z, double e2,
                double e4, int k, int l, int m, const double a[5])
{
    const double v0 = 0.5 * (t3(X, Y, Z, 2 + k, l, m) + t3(X, Y, Z, k, 2 + l, m) +
                             t3(X, Y, Z, k, l, 2 + m) + t3(X, Y, Z, k, l, m) * e2);
    M[0] = a[0] * (t3(X, Y, Z, k, l, m)) + a[1] * (t3(X, Y, Z, 1 + k, l, m)) +
           a[2] * (t3(X, Y, Z, k, 1 + l, m)) + a[3] * (t3(X, Y, Z, k, l, 1 + m)) + a[4] * v0;

    const double v1 = 0.5 * (t3(X, Y, Z, 3 + k, l, m) + t3(X, Y, Z, 1 + k, 2 + l, m) +
                             t3(X, Y, Z, 1 + k, l, 2 + m) + t3(X, Y, Z, 1 + k, l, m) * e2);
    M[1] = a[0] * (t3(X, Y, Z, 1 + k, l, m)) + a[1] * (t3(X, Y, Z, 2 + k, l, m)) +
           a[2] * (t3(X, Y, Z, 1 + k, 1 + l, m)) + a[3] * (t3(X, Y, Z, 1 + k, l, 1 + m)) + a[4] * v1;

    const double v2 = 0.5 * (t3(X, Y, Z, 2 + k, 1 + l, m) + t3(X, Y, Z, k, 3 + l, m) +
                             t3(X, Y, Z, k, 1 + l, 2 + m) + t3(X, Y, Z, k, 1 + l, m) * e2);
    M[2] = a[0] * (t3(X, Y, Z, k, 1 + l, m)) + a[1] * (t3(X, Y, Z, 1 + k, 1 + l, m)) +
           a[2] * (t3(X, Y, Z, k, 2 + l, m)) + a[3] * (t3(X, Y, Z, k, 1 + l, 1 + m)) + a[4] * v2;

    const double v3 = 0.5 * (t3(X, Y, Z, 2 + k, l, 1 + m) + t3(X, Y, Z, k, 2 + l, 1 + m) +
                             t3(X, Y, Z, k, l, 3 + m) + t3(X, Y, Z, k, l, 1 + m) * e2);
    M[3] = a[0] * (t3(X, Y, Z, k, l, 1 + m)) + a[1] * (t3(X, Y, Z, 1 + k, l, 1 + m)) +
           a[2] * (t3(X, Y, Z, k, 1 + l, 1 + m)) + a[3] * (t3(X, Y, Z, k, l, 2 + m)) + a[4] * v3;

    M[4] = 0.25 * a[4] *
               (t3(X, Y, Z, 4 + k, l, m) + t3(X, Y, Z, k, 4 + l, m) + t3(X, Y, Z, k, l, 4 + m) +
                t3(X, Y, Z, k, l, m) * e4 + 2 * t3(X, Y, Z, 2 + k, 2 + l, m) +
                2 * t3(X, Y, Z, 2 + k, l, 2 + m) + 2 * t3(X, Y, Z, 2 + k, l, m) * e2 +
                2 * t3(X, Y, Z, k, 2 + l, 2 + m) + 2 * t3(X, Y, Z, k, 2 + l, m) * e2 +
                2 * t3(X, Y, Z, k, l, 2 + m) * e2) +
           a[0] * v0 + a[1] * v1 + a[2] * v2 + a[3] * v3;
}

/* Moments over a Maxwellian g with normal table X. */
#define MOM(M, g, X, k, l, m, a) mom(M, X, (g)->full[1], (g)->full[2], (g)->e2, (g)->e4, k, l, m, a)
#define MOM0(M, g, X, k, l, m) mom0(M, X, (g)->full[1], (g)->full[2], (g)->e2, k, l, m)

/* ---------------------------------------------------------------------------
 * Slope coefficients a from moment derivatives b (slopesolver,
 * GKMflux.cpp:280-296; pr_factor = 1/0.7 there, 1 in GPUupdate.cu:830-845).
 * ------------------------------------------------------------------------- */
static void slopes(const double b[5], const double U[3], double lam, int K, double prf, double a[5])
{
    const double R2 = b[1] - U[0] * b[0];
    const double R3 = b[2] - U[1] * b[0];
    const double R4 = b[3] - U[2] * b[0];
    const double R5 = 2 * b[4] - b[0] * (U[0] * U[0] + U[1] * U[1] + U[2] * U[2] + (K + 3) / (2 * lam));
    a[4] = prf * (R5 - 2 * U[0] * R2 - 2 * U[1] * R3 - 2 * U[2] * R4) * (4 * lam * lam) / (K + 3);
    a[3] = 2 * lam * R4 - U[2] * a[4];
    a[2] = 2 * lam * R3 - U[1] * a[4];
    a[1] = 2 * lam * R2 - U[0] * a[4];
    a[0] = b[0] - a[1] * U[0] - a[2] * U[1] - a[3] * U[2] -
           .5 * a[4] * (U[0] * U[0] + U[1] * U[1] + U[2] * U[2] + (K + 3) / (2 * lam));
}

/* ---------------------------------------------------------------------------
 * Interface flux (GKMflux.cpp:11-215).
 * ------------------------------------------------------------------------- */
void orc_flux(const double *in, double gam, int K, double prf, double *F)
{
    const double *WL = in, *WR = in + 5, *Wl = in + 10, *Wr = in + 15;
    const double *DWxl = in + 20, *DWxr = in + 25, *DWyl = in + 30, *DWyr = in + 35;
    const double *DWzl = in + 40, *DWzr = in + 45;
    double tau = in[50];
    const double dt = in[51], dx = in[52];

    maxwellian l, r, e;
    /* left / right states and their moments (GKMflux.cpp:40-66) */
    prim(Wl, gam, &l.den, l.U, &l.P);
    prim(Wr, gam, &r.den, r.U, &r.P);
    l.lam = 0.5 * l.den / l.P;
    r.lam = 0.5 * r.den / r.P;
    moments(&l, K, 1, 0);
    moments(&r, K, 0, 1);

    /* equilibrium state at the interface (GKMflux.cpp:71-77) */
    double Mpl000[5], Mnr000[5], We[5];
    MOM0(Mpl000, &l, l.pos, 0, 0, 0);
    MOM0(Mnr000, &r, r.neg, 0, 0, 0);
    for (int q = 0; q < NQ; ++q) We[q] = l.den * Mpl000[q] + r.den * Mnr000[q];
    prim(We, gam, &e.den, e.U, &e.P);
    e.lam = 0.5 * e.den / e.P;
    moments(&e, K, 1, 1); /* GKMflux.cpp:82-98 */

    /* slopes, phase I (GKMflux.cpp:102-119) */
    double bxl[5], bxr[5], byl[5], byr[5], bzl[5], bzr[5], bx_l[5], bx_r[5];
    for (int q = 0; q < NQ; ++q) {
        bxl[q] = DWxl[q] / l.den;
        bxr[q] = DWxr[q] / r.den;
        byl[q] = DWyl[q] / l.den;
        byr[q] = DWyr[q] / r.den;
        bzl[q] = DWzl[q] / l.den;
        bzr[q] = DWzr[q] / r.den;
        bx_l[q] = 2 * (We[q] - WL[q]) / (e.den * dx);
        bx_r[q] = 2 * (WR[q] - We[q]) / (e.den * dx);
    }
    double axl[5], axr[5], ayl[5], ayr[5], azl[5], azr[5], ax_l[5], ax_r[5];
    slopes(bxl, l.U, l.lam, K, prf, axl);
    slopes(bxr, r.U, r.lam, K, prf, axr);
    slopes(byl, l.U, l.lam, K, prf, ayl);
    slopes(byr, r.U, r.lam, K, prf, ayr);
    slopes(bzl, l.U, l.lam, K, prf, azl);
    slopes(bzr, r.U, r.lam, K, prf, azr);
    slopes(bx_l, e.U, e.lam, K, prf, ax_l);
    slopes(bx_r, e.U, e.lam, K, prf, ax_r);

    /* slopes, phase II (GKMflux.cpp:124-144) */
    double Mpl000_ay[5], Mnr000_ay[5], Mpl000_az[5], Mnr000_az[5];
    double Mfl100_ax[5], Mfr100_ax[5], Mfl010_ay[5], Mfr010_ay[5], Mfl001_az[5], Mfr001_az[5];
    MOM(Mpl000_ay, &l, l.pos, 0, 0, 0, ayl);
    MOM(Mnr000_ay, &r, r.neg, 0, 0, 0, ayr);
    MOM(Mpl000_az, &l, l.pos, 0, 0, 0, azl);
    MOM(Mnr000_az, &r, r.neg, 0, 0, 0, azr);
    MOM(Mfl100_ax, &l, l.full[0], 1, 0, 0, axl);
    MOM(Mfr100_ax, &r, r.full[0], 1, 0, 0, axr);
    MOM(Mfl010_ay, &l, l.full[0], 0, 1, 0, ayl);
    MOM(Mfr010_ay, &r, r.full[0], 0, 1, 0, ayr);
    MOM(Mfl001_az, &l, l.full[0], 0, 0, 1, azl);
    MOM(Mfr001_az, &r, r.full[0], 0, 0, 1, azr);
    double by_[5], bz_[5], Bl[5], Br[5];
    for (int q = 0; q < NQ; ++q) {
        by_[q] = Mpl000_ay[q] + Mnr000_ay[q];
        bz_[q] = Mpl000_az[q] + Mnr000_az[q];
        Bl[q] = -Mfl100_ax[q] - Mfl010_ay[q] - Mfl001_az[q];
        Br[q] = -Mfr100_ax[q] - Mfr010_ay[q] - Mfr001_az[q];
    }
    double ay_[5], az_[5], Al[5], Ar[5];
    slopes(by_, e.U, e.lam, K, prf, ay_);
    slopes(bz_, e.U, e.lam, K, prf, az_);
    slopes(Bl, l.U, l.lam, K, prf, Al);
    slopes(Br, r.U, r.lam, K, prf, Ar);

    /* collision time with numerical dissipation (GKMflux.cpp:149-150) */
    const double w = fabs(l.den / l.lam - r.den / r.lam) / (fabs(l.den / l.lam + r.den / r.lam));
    tau = tau + dt * w;

    /* slopes, phase III (GKMflux.cpp:155-180) */
    const double gm0 = dt - tau * (1 - exp(-dt / tau));
    const double gm1 = -(1 - exp(-dt / tau)) / gm0;
    const double gm2 = (-dt + 2 * tau * (1 - exp(-dt / tau)) - dt * exp(-dt / tau)) / gm0;
    const double gm3 = -gm1;
    const double gm4 = (dt * exp(-dt / tau) - tau * (1 - exp(-dt / tau))) / gm0;
    const double gm5 = tau * gm3;

    double Mfe000[5], Mpe100_ax[5], Mne100_ax[5], Mfe010_ay[5], Mfe001_az[5];
    double Mpl100_ax[5], Mnr100_ax[5], Mpl010_ay[5], Mnr010_ay[5], Mpl001_az[5], Mnr001_az[5];
    double Mpl000_A[5], Mnr000_A[5];
    MOM0(Mfe000, &e, e.full[0], 0, 0, 0);
    MOM(Mpe100_ax, &e, e.pos, 1, 0, 0, ax_l);
    MOM(Mne100_ax, &e, e.neg, 1, 0, 0, ax_r);
    MOM(Mfe010_ay, &e, e.full[0], 0, 1, 0, ay_);
    MOM(Mfe001_az, &e, e.full[0], 0, 0, 1, az_);
    MOM(Mpl100_ax, &l, l.pos, 1, 0, 0, axl);
    MOM(Mnr100_ax, &r, r.neg, 1, 0, 0, axr);
    MOM(Mpl010_ay, &l, l.pos, 0, 1, 0, ayl);
    MOM(Mnr010_ay, &r, r.neg, 0, 1, 0, ayr);
    MOM(Mpl001_az, &l, l.pos, 0, 0, 1, azl);
    MOM(Mnr001_az, &r, r.neg, 0, 0, 1, azr);
    MOM(Mpl000_A, &l, l.pos, 0, 0, 0, Al);
    MOM(Mnr000_A, &r, r.neg, 0, 0, 0, Ar);
    double B_[5];
    for (int q = 0; q < NQ; ++q) {
        B_[q] = gm1 * e.den * Mfe000[q] +
                gm2 * e.den * (Mpe100_ax[q] + Mne100_ax[q] + Mfe010_ay[q] + Mfe001_az[q]) +
                gm3 * (l.den * Mpl000[q] + r.den * Mnr000[q]) +
                (gm4 + gm5) * (l.den * (Mpl100_ax[q] + Mpl010_ay[q] + Mpl001_az[q]) +
                               r.den * (Mnr100_ax[q] + Mnr010_ay[q] + Mnr001_az[q])) +
                gm5 * (l.den * Mpl000_A[q] + r.den * Mnr000_A[q]);
        B_[q] = B_[q] / e.den;
    }
    double A_[5];
    slopes(B_, e.U, e.lam, K, prf, A_);

    /* time integrals and flux (GKMflux.cpp:186-213) */
    const double P = -tau * (exp(-dt / tau) - 1);
    const double Q = -tau * dt * exp(-dt / tau) - tau * tau * (exp(-dt / tau) - 1);
    const double p0 = (dt - P), p1 = 0.5 * dt * dt - tau * (p0);
    const double p2 = -tau * (p0) + Q, p3 = P;
    const double p4 = -Q - tau * P, p5 = -tau * P;

    double Mpl100[5], Mnr100[5], Mfe100[5], Mfe100_A[5], Mpe200_ax[5], Mne200_ax[5];
    double Mfe110_ay[5], Mfe101_az[5], Mpl200_ax[5], Mnr200_ax[5], Mpl110_ay[5], Mnr110_ay[5];
    double Mpl101_az[5], Mnr101_az[5], Mpl100_A[5], Mnr100_A[5];
    MOM0(Mpl100, &l, l.pos, 1, 0, 0);
    MOM0(Mnr100, &r, r.neg, 1, 0, 0);
    MOM0(Mfe100, &e, e.full[0], 1, 0, 0);
    MOM(Mfe100_A, &e, e.full[0], 1, 0, 0, A_);
    MOM(Mpe200_ax, &e, e.pos, 2, 0, 0, ax_l);
    MOM(Mne200_ax, &e, e.neg, 2, 0, 0, ax_r);
    MOM(Mfe110_ay, &e, e.full[0], 1, 1, 0, ay_);
    MOM(Mfe101_az, &e, e.full[0], 1, 0, 1, az_);
    MOM(Mpl200_ax, &l, l.pos, 2, 0, 0, axl);
    MOM(Mnr200_ax, &r, r.neg, 2, 0, 0, axr);
    MOM(Mpl110_ay, &l, l.pos, 1, 1, 0, ayl);
    MOM(Mnr110_ay, &r, r.neg, 1, 1, 0, ayr);
    MOM(Mpl101_az, &l, l.pos, 1, 0, 1, azl);
    MOM(Mnr101_az, &r, r.neg, 1, 0, 1, azr);
    MOM(Mpl100_A, &l, l.pos, 1, 0, 0, Al);
    MOM(Mnr100_A, &r, r.neg, 1, 0, 0, Ar);
    for (int q = 0; q < NQ; ++q) {
        F[q] = p0 * e.den * Mfe100[q] + p1 * e.den * Mfe100_A[q] +
               p2 * e.den * (Mpe200_ax[q] + Mne200_ax[q] + Mfe110_ay[q] + Mfe101_az[q]) +
               p3 * (l.den * Mpl100[q] + r.den * Mnr100[q]) +
               p4 * (l.den * (Mpl200_ax[q] + Mpl110_ay[q] + Mpl101_az[q]) +
                     r.den * (Mnr200_ax[q] + Mnr110_ay[q] + Mnr101_az[q])) +
               p5 * (l.den * Mpl100_A[q] + r.den * Mnr100_A[q]);
    }
}

/* ---------------------------------------------------------------------------
 * WENO-SYMOO (update.cpp:502-625): 4 candidate cubics on a 6-point stencil,
 * linear weights 1/20, 9/20, 9/20, 1/20, the last smoothness indicator replaced
 * by the largest of the four, alpha = gamma / (eps + IS).
 * ------------------------------------------------------------------------- */
static const double WENO_EPS = 1e-10; /* pow(10.0, -10.0), param.h:15 */

static void weno_scalar(double LLL, double LL, double L, double R, double RR, double RRR,
                        double *wl, double *wr)
{
    const double g0 = 1.0 / 20.0, g1 = 9.0 / 20.0, g2 = 9.0 / 20.0, g3 = 1.0 / 20.0;
    /* left-biased (value at the interface from the L side) */
    const double p0p = LLL / 3 - 7 * LL / 6 + 11 * L / 6;
    const double p1p = -LL / 6 + 5 * L / 6 + R / 3;
    const double p2p = L / 3 + 5 * R / 6 - RR / 6;
    const double p3p = 11 * R / 6 - 7 * RR / 6 + RRR / 3;
    /* right-biased */
    const double p0n = RRR / 3 - 7 * RR / 6 + 11 * R / 6;
    const double p1n = -RR / 6 + 5 * R / 6 + L / 3;
    const double p2n = R / 3 + 5 * L / 6 - LL / 6;
    const double p3n = 11 * L / 6 - 7 * LL / 6 + LLL / 3;

    double d, e;
    d = LLL - 2 * LL + L;  e = LLL - 4 * LL + 3 * L;   const double s0p = 13 * (d * d) / 12 + (e * e) / 4;
    d = RRR - 2 * RR + R;  e = RRR - 4 * RR + 3 * R;   const double s0n = 13 * (d * d) / 12 + (e * e) / 4;
    d = LL - 2 * L + R;    e = -LL + R;                const double s1p = 13 * (d * d) / 12 + (e * e) / 4;
    d = RR - 2 * R + L;    e = -RR + L;                const double s1n = 13 * (d * d) / 12 + (e * e) / 4;
    d = L - 2 * R + RR;    e = -3 * L + 4 * R - RR;    const double s2p = 13 * (d * d) / 12 + (e * e) / 4;
    d = R - 2 * L + LL;    e = -3 * R + 4 * L - LL;    const double s2n = 13 * (d * d) / 12 + (e * e) / 4;
    d = R - 2 * RR + RRR;  e = -5 * R + 8 * RR - 3 * RRR; const double s3p_ = 13 * (d * d) / 12 + (e * e) / 4;
    d = L - 2 * LL + LLL;  e = -5 * L + 8 * LL - 3 * LLL; const double s3n_ = 13 * (d * d) / 12 + (e * e) / 4;

    double mp = s0p < s1p ? s1p : s0p;
    mp = mp < s2p ? s2p : mp;
    mp = mp < s3p_ ? s3p_ : mp;
    double mn = s0n < s1n ? s1n : s0n;
    mn = mn < s2n ? s2n : mn;
    mn = mn < s3n_ ? s3n_ : mn;
    const double s3p = mp, s3n = mn;

    const double a0p = g0 * (1 / (WENO_EPS + s0p)), a0n = g0 * (1 / (WENO_EPS + s0n));
    const double a1p = g1 * (1 / (WENO_EPS + s1p)), a1n = g1 * (1 / (WENO_EPS + s1n));
    const double a2p = g2 * (1 / (WENO_EPS + s2p)), a2n = g2 * (1 / (WENO_EPS + s2n));
    const double a3p = g3 * (1 / (WENO_EPS + s3p)), a3n = g3 * (1 / (WENO_EPS + s3n));
    const double sp = a0p + a1p + a2p + a3p;
    const double sn = a0n + a1n + a2n + a3n;
    *wl = (a0p / (sp)) * p0p + (a1p / (sp)) * p1p + (a2p / (sp)) * p2p + (a3p / (sp)) * p3p;
    *wr = (a0n / (sn)) * p0n + (a1n / (sn)) * p1n + (a2n / (sn)) * p2n + (a3n / (sn)) * p3n;
}

/* Temperature of a conservative state (update.cpp:560-565). */
static double temp_of(const double *W, double gam, double R)
{
    return (gam - 1) * (W[4] / W[0] - 0.5 * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) / (W[0] * W[0])) / R;
}

void orc_weno(const double *s, double gam, double R, int direct_energy, double *wl, double *wr)
{
    const double *c[6] = {s, s + 5, s + 10, s + 15, s + 20, s + 25};
    const int nd = direct_energy ? 5 : 4;
    for (int q = 0; q < nd; ++q)
        weno_scalar(c[0][q], c[1][q], c[2][q], c[3][q], c[4][q], c[5][q], &wl[q], &wr[q]);
    if (direct_energy) return;
    double T[6];
    for (int a = 0; a < 6; ++a) T[a] = temp_of(c[a], gam, R);
    double Tl, Tr;
    weno_scalar(T[0], T[1], T[2], T[3], T[4], T[5], &Tl, &Tr);
    wl[4] = wl[0] * R * Tl / (gam - 1.0) + 0.5 * (wl[1] * wl[1] + wl[2] * wl[2] + wl[3] * wl[3]) / wl[0];
    wr[4] = wr[0] * R * Tr / (gam - 1.0) + 0.5 * (wr[1] * wr[1] + wr[2] * wr[2] + wr[3] * wr[3]) / wr[0];
}

/* ---------------------------------------------------------------------------
 * Periodic ghost fill: the effect of HaloTransfer on one periodic rank
 * (update.cpp:894-1054; equivalently PeriodicBC, FlowField.cpp:115-275).
 * ------------------------------------------------------------------------- */
static inline long wrap(long g, long nc) { return g < 3 ? g + nc : (g >= nc + 3 ? g - nc : g); }

void orc_halo(double *W, int nc)
{
    const long nt = nc + 6, N = nt * nt * nt;
    for (int q = 0; q < NQ; ++q) {
        double *w = W + q * N;
        for (long j = 0; j < nt; ++j)
            for (long i = 0; i < nt; ++i)
                for (long k = 0; k < nt; ++k) {
                    const long jj = wrap(j, nc), ii = wrap(i, nc), kk = wrap(k, nc);
                    if (jj != j || ii != i || kk != k) w[(j * nt + i) * nt + k] = w[(jj * nt + ii) * nt + kk];
                }
    }
}

/* ---------------------------------------------------------------------------
 * Sweeps (update.cpp:201-453) and update (update.cpp:455-469).
 * ------------------------------------------------------------------------- */
static double viscosity(const orc_params *p, double T)
{
    if (p->visc_law == ORC_VISC_POWER) return p->mu0 * pow((T / p->T0), p->visc_exp);
    return p->mu0 * pow((T / p->T0), 1.5) * (p->T0 + 110.4) / (T + 110.4);
}

typedef struct {
    int dir;           /* 0 x (along i), 1 y (along j), 2 z (along k) */
    long nrm;          /* stride along the sweep */
    long north, south; /* the transverse lines whose difference gives DWy */
    long front, back;  /* the transverse lines whose difference gives DWz */
    double ysign;      /* sign of the DWy difference (update.cpp:330) */
    int rot;           /* momentum component rotated into slot 1 (0: none) */
} sweep_geom;

static void gather_weno(const double *W, long N, long c, long stride, const orc_params *p,
                        double *wl, double *wr)
{
    double s[30];
    for (int a = 0; a < 6; ++a)
        for (int q = 0; q < NQ; ++q) s[a * 5 + q] = W[q * N + c + (a - 2) * stride];
    orc_weno(s, p->gam, p->R, p->flags & ORC_DIRECT_ENERGY, wl, wr);
}

static inline void swap5(double *v, int r)
{
    const double t = v[r];
    v[r] = v[1];
    v[1] = t;
}

static void sweep(const double *W, double *Fd, const orc_params *p, double dt, const sweep_geom *g)
{
    const long nc = p->nc, nt = nc + 6, N = nt * nt * nt;
    const double dx = p->dx;
    /* loop order j, i, k as in the reference, (j,i,k) = (y,x,z); the sweep
     * direction starts one cell lower (FoR, param.h:30) to include the
     * interface between the last ghost and the first interior cell */
    const long jlo = g->dir == 1 ? 2 : 3, ilo = g->dir == 0 ? 2 : 3, klo = g->dir == 2 ? 2 : 3;
    for (long j = jlo; j < nt - 3; ++j)
        for (long i = ilo; i < nt - 3; ++i)
            for (long k = klo; k < nt - 3; ++k) {
                const long c = (j * nt + i) * nt + k;
                double in[53];
                double *WL = in, *WR = in + 5, *Wl = in + 10, *Wr = in + 15;
                double *DWxl = in + 20, *DWxr = in + 25, *DWyl = in + 30, *DWyr = in + 35;
                double *DWzl = in + 40, *DWzr = in + 45;
                double WlN[5], WrN[5], WlS[5], WrS[5], WlF[5], WrF[5], WlB[5], WrB[5];
                for (int q = 0; q < NQ; ++q) {
                    WL[q] = W[q * N + c];
                    WR[q] = W[q * N + c + g->nrm];
                }
                gather_weno(W, N, c, g->nrm, p, Wl, Wr);
                gather_weno(W, N, c + g->north, g->nrm, p, WlN, WrN);
                gather_weno(W, N, c + g->south, g->nrm, p, WlS, WrS);
                gather_weno(W, N, c + g->front, g->nrm, p, WlF, WrF);
                gather_weno(W, N, c + g->back, g->nrm, p, WlB, WrB);
                for (int q = 0; q < NQ; ++q) {
                    DWxl[q] = 2 * (Wl[q] - WL[q]) / dx;
                    DWxr[q] = 2 * (WR[q] - Wr[q]) / dx;
                    DWyl[q] = g->ysign * 0.5 * (WlN[q] - WlS[q]) / dx;
                    DWyr[q] = g->ysign * 0.5 * (WrN[q] - WrS[q]) / dx;
                    DWzl[q] = 0.5 * (WlF[q] - WlB[q]) / dx;
                    DWzr[q] = 0.5 * (WrF[q] - WrB[q]) / dx;
                }
                /* collision time at the left cell (update.cpp:262-264, 882-891) */
                const double deni = WL[0];
                const double ui = WL[1] / deni, vi = WL[2] / deni, wi = WL[3] / deni;
                const double Vsqr = (ui * ui + vi * vi + wi * wi);
                const double Pi = (deni * (p->gam - 1)) * (WL[4] / deni - 0.5 * Vsqr);
                const double Ti = Pi / (p->R * deni);
                in[50] = viscosity(p, Ti) / Pi;
                in[51] = dt;
                in[52] = dx;
                if (g->rot) {
                    for (int v = 0; v < 10; ++v) swap5(in + 5 * v, g->rot);
                }
                double F[5];
                orc_flux(in, p->gam, p->K, p->pr_factor, F);
                if (g->rot) swap5(F, g->rot);
                for (int q = 0; q < NQ; ++q) Fd[q * N + c] = F[q];
            }
}

void orc_step(double *W, const orc_params *p, double dt, double *F)
{
    const long nc = p->nc, nt = nc + 6, N = nt * nt * nt;
    const long sj = nt * nt, si = nt, sk = 1;
    double *Fx = F, *Fy = F + 5 * N, *Fz = F + 10 * N;
    /* x: N/S = j+-1, F/B = k+-1 (update.cpp:218-244) */
    const sweep_geom gx = {0, si, +sj, -sj, +sk, -sk, 1.0, 0};
    /* y: N/S = i-+1 with DWy = -(N - S), F/B = k+-1, rotate rho v into slot 1 (update.cpp:291-350) */
    const sweep_geom gy = {1, sj, -si, +si, +sk, -sk, -1.0, 2};
    /* z: N/S = i+-1 (an x derivative), F/B = j+-1 (a y derivative), rho w into slot 1
     * (update.cpp:380-439); with ORC_FIX_ZSWEEP the rotated frame's own axes are used. */
    const sweep_geom gz_ref = {2, sk, +si, -si, +sj, -sj, 1.0, 3};
    const sweep_geom gz_fix = {2, sk, +sj, -sj, +si, -si, 1.0, 3};
    sweep(W, Fx, p, dt, &gx);
    sweep(W, Fy, p, dt, &gy);
    sweep(W, Fz, p, dt, (p->flags & ORC_FIX_ZSWEEP) ? &gz_fix : &gz_ref);
    const double dx = p->dx;
    for (int q = 0; q < NQ; ++q) {
        double *w = W + q * N;
        const double *fx = Fx + q * N, *fy = Fy + q * N, *fz = Fz + q * N;
        for (long j = 3; j < nt - 3; ++j)
            for (long i = 3; i < nt - 3; ++i)
                for (long k = 3; k < nt - 3; ++k) {
                    const long c = (j * nt + i) * nt + k;
                    w[c] -= (1 / dx) * (fx[c] - fx[c - si] + fy[c] - fy[c - sj] + fz[c] - fz[c - sk]);
                }
    }
    orc_halo(W, (int)nc);
}

/* ---------------------------------------------------------------------------
 * Time step bound (update.cpp:1057-1079).
 * ------------------------------------------------------------------------- */
double orc_maxval(const double *W, const orc_params *p)
{
    const long nc = p->nc, nt = nc + 6, N = nt * nt * nt;
    double mx = 0.0;
    for (long j = 3; j < nt - 3; ++j)
        for (long i = 3; i < nt - 3; ++i)
            for (long k = 3; k < nt - 3; ++k) {
                const long c = (j * nt + i) * nt + k;
                const double deni = W[c];
                const double ui = W[N + c] / deni, vi = W[2 * N + c] / deni, wi = W[3 * N + c] / deni;
                const double Vsqr = (ui * ui + vi * vi + wi * wi);
                const double Pi = (deni * (p->gam - 1)) * (W[4 * N + c] / deni - 0.5 * Vsqr);
                const double val = sqrt(Vsqr) + sqrt(p->gam * Pi / deni);
                if (mx < val) mx = val;
            }
    return mx;
}

/* ---------------------------------------------------------------------------
 * Statistics (update.cpp:638-784; spline gradients as in the nodal stand-in
 * for einspline: natural cubic spline slopes along each padded grid line).
 * ------------------------------------------------------------------------- */
static void line_slopes(long n, double h, const double *f, long stride, double *m, double *cp, double *dp)
{
    const double s = 3.0 / h;
    double b = 2.0, c = 1.0;
    double r = s * (f[stride] - f[0]);
    cp[0] = c / b;
    dp[0] = r / b;
    for (long i = 1; i < n; ++i) {
        const double a = 1.0;
        b = (i == n - 1) ? 2.0 : 4.0;
        c = (i == n - 1) ? 0.0 : 1.0;
        if (i == n - 1)
            r = s * (f[i * stride] - f[(i - 1) * stride]);
        else
            r = s * (f[(i + 1) * stride] - f[(i - 1) * stride]);
        const double den = b - a * cp[i - 1];
        cp[i] = c / den;
        dp[i] = (r - a * dp[i - 1]) / den;
    }
    m[(n - 1) * stride] = dp[n - 1];
    for (long i = n - 2; i >= 0; --i) m[i * stride] = dp[i] - cp[i] * m[(i + 1) * stride];
}

/* Slopes of field f (padded block of nty x nt x nt cells) along axis 0 (j), 1 (i) or 2 (k). */
static void axis_slopes(const double *f, double *g, long nty, long nt, double h, int axis, double *cp, double *dp)
{
    const long sj = nt * nt, si = nt;
    const long na = axis == 0 ? nt : nty, len = axis == 0 ? nty : nt;
    for (long a = 0; a < na; ++a)
        for (long b = 0; b < nt; ++b) {
            long base, stride;
            if (axis == 0) { base = a * si + b; stride = sj; }
            else if (axis == 1) { base = a * sj + b; stride = si; }
            else { base = a * sj + b * si; stride = 1; }
            line_slopes(len, h, f + base, stride, g + base, cp, dp);
        }
}

/* Spacing of a spline grid of num nodes from (sta - 3) dx + dx/2
 * (Interpolation.cpp:10-27), as einspline derives it from start and end. */
static double grid_h(long sta, long num, double dx)
{
    const double start = (sta - 3) * dx + 0.5 * dx;
    const double end = start + (num - 1) * dx;
    return (end - start) / (double)(num - 1);
}

static void prim_at(const double *W, long cs, long c, double gam, double R, double *deni, double *ui,
                    double *vi, double *wi, double *Vsqr, double *Pi, double *Ti)
{
    *deni = W[c];
    *ui = W[cs + c] / *deni;
    *vi = W[2 * cs + c] / *deni;
    *wi = W[3 * cs + c] / *deni;
    *Vsqr = (*ui * *ui + *vi * *vi + *wi * *wi);
    *Pi = (*deni * (gam - 1)) * (W[4 * cs + c] / *deni - 0.5 * *Vsqr);
    *Ti = *Pi / (R * *deni);
}

/* One rank's first pass of PrintStats (update.cpp:659-712) over its segment:
 * W is its padded block of nty x nt x nt cells (components cs apart), its
 * first plane the global plane sta0 - 3; the splines run over the segment's
 * own nodes (einspline per rank, Interpolation.cpp:3-31).  Adds the 18 local
 * sums to acc: TKE, Diss, SijSij, DUDX2-4, DVDY2-4, DWDZ2-4, P, T, 1/rho,
 * |u|^2, c, rho. */
static void seg_sums(const double *W, long cs, long nty, long nt, long sta0, const orc_params *p, double *acc)
{
    const long N = nty * nt * nt;
    const double gam = p->gam, R = p->R, dx = p->dx;
    double *u = malloc(sizeof(double) * N), *v = malloc(sizeof(double) * N), *w = malloc(sizeof(double) * N);
    double *gu[3], *gv[3], *gw[3];
    for (int d = 0; d < 3; ++d) {
        gu[d] = malloc(sizeof(double) * N);
        gv[d] = malloc(sizeof(double) * N);
        gw[d] = malloc(sizeof(double) * N);
    }
    const long nmax = nty > nt ? nty : nt;
    double *cp = malloc(sizeof(double) * nmax), *dp = malloc(sizeof(double) * nmax);
    for (long c = 0; c < N; ++c) { /* generateSplines, update.cpp:1215-1224 */
        const double d = W[c];
        u[c] = W[cs + c] / d;
        v[c] = W[2 * cs + c] / d;
        w[c] = W[3 * cs + c] / d;
    }
    for (int d = 0; d < 3; ++d) {
        const double h = d == 0 ? grid_h(sta0, nty, dx) : grid_h(0, nt, dx);
        axis_slopes(u, gu[d], nty, nt, h, d, cp, dp);
        axis_slopes(v, gv[d], nty, nt, h, d, cp, dp);
        axis_slopes(w, gw[d], nty, nt, h, d, cp, dp);
    }
    for (long j = 3; j < nty - 3; ++j)
        for (long i = 3; i < nt - 3; ++i)
            for (long k = 3; k < nt - 3; ++k) {
                const long c = (j * nt + i) * nt + k;
                double deni, ui, vi, wi, Vsqr, Pi, Ti;
                prim_at(W, cs, c, gam, R, &deni, &ui, &vi, &wi, &Vsqr, &Pi, &Ti);
                acc[12] += Pi;
                acc[13] += Ti;
                acc[14] += 1 / deni;
                const double dudx = gu[1][c], dudy = gu[0][c], dudz = gu[2][c];
                const double dvdx = gv[1][c], dvdy = gv[0][c], dvdz = gv[2][c];
                const double dwdx = gw[1][c], dwdy = gw[0][c], dwdz = gw[2][c];
                const double mu = viscosity(p, Ti);
                acc[1] += mu * (dudx * dudx + dudy * dudy + dudz * dudz + dvdx * dvdx + dvdy * dvdy +
                                dvdz * dvdz + dwdx * dwdx + dwdy * dwdy + dwdz * dwdz);
                acc[0] += deni * (u[c] * u[c] + v[c] * v[c] + w[c] * w[c]);
                acc[2] += (dudx * dudx + 0.5 * ((dudy + dvdx) * (dudy + dvdx)) +
                           0.5 * ((dudz + dwdx) * (dudz + dwdx)) + 0.5 * ((dwdy + dvdz) * (dwdy + dvdz)) +
                           dvdy * dvdy + dwdz * dwdz);
                acc[3] += dudx * dudx; acc[4] += dudx * dudx * dudx; acc[5] += dudx * dudx * dudx * dudx;
                acc[6] += dvdy * dvdy; acc[7] += dvdy * dvdy * dvdy; acc[8] += dvdy * dvdy * dvdy * dvdy;
                acc[9] += dwdz * dwdz; acc[10] += dwdz * dwdz * dwdz; acc[11] += dwdz * dwdz * dwdz * dwdz;
                acc[15] += Vsqr;
                acc[16] += sqrt(gam * Pi / deni);
                acc[17] += deni;
            }
    free(u); free(v); free(w);
    for (int d = 0; d < 3; ++d) { free(gu[d]); free(gv[d]); free(gw[d]); }
    free(cp); free(dp);
}

/* One rank's second pass (update.cpp:751-757): squared deviations from the
 * global means m[0..2] of p, T and 1/rho over its segment's interior. */
static void seg_devs(const double *W, long cs, long nty, long nt, const orc_params *p, const double *m, double *acc)
{
    for (long j = 3; j < nty - 3; ++j)
        for (long i = 3; i < nt - 3; ++i)
            for (long k = 3; k < nt - 3; ++k) {
                const long c = (j * nt + i) * nt + k;
                double deni, ui, vi, wi, Vsqr, Pi, Ti;
                prim_at(W, cs, c, p->gam, p->R, &deni, &ui, &vi, &wi, &Vsqr, &Pi, &Ti);
                acc[0] += (m[0] - Pi) * (m[0] - Pi);
                acc[1] += (m[1] - Ti) * (m[1] - Ti);
                acc[2] += (m[2] - 1 / deni) * (m[2] - 1 / deni);
            }
}

void orc_stats_ranks(const double *W, const orc_params *p, int nranks, double *out)
{
    const long nc = p->nc, nt = nc + 6, cs = nt * nt * nt, ny = nc / nranks, nty = ny + 6;
    const double gam = p->gam;
    /* every rank's segment is planes [r ny, r ny + ny + 6) of the padded block
     * (segment() / segmentFill, FlowField.cpp:278-303); its sums reduced in
     * rank order (MPI_Reduce, update.cpp:714-725) */
    double s[18] = {0};
    for (int r = 0; r < nranks; ++r) {
        double acc[18] = {0};
        seg_sums(W + r * ny * nt * nt, cs, nty, nt, r * ny, p, acc);
        for (int i = 0; i < 18; ++i) s[i] += acc[i];
    }
    const double Nc = (double)(nc * nc * nc);
    for (int i = 0; i < 18; ++i) s[i] /= Nc;
    double dv[3] = {0, 0, 0};
    for (int r = 0; r < nranks; ++r) {
        double acc[3] = {0, 0, 0};
        seg_devs(W + r * ny * nt * nt, cs, nty, nt, p, s + 12, acc);
        for (int i = 0; i < 3; ++i) dv[i] += acc[i];
    }
    const double Pr = sqrt(dv[0] / Nc), Tr = sqrt(dv[1] / Nc), Vr = sqrt(dv[2] / Nc);
    out[0] = s[0];
    out[1] = s[1];
    out[2] = s[4] / pow(s[3], 1.5);
    out[3] = s[7] / pow(s[6], 1.5);
    out[4] = s[10] / pow(s[9], 1.5);
    out[5] = s[5] / (s[3] * s[3]);
    out[6] = s[8] / (s[6] * s[6]);
    out[7] = s[11] / (s[9] * s[9]);
    out[8] = Pr / (gam * p->p0 * p->Mt * p->Mt);
    out[9] = Tr / ((gam - 1) * p->T0 * p->Mt * p->Mt);
    out[10] = Vr / (p->Mt * p->Mt / p->den0);
    out[11] = s[2];
    out[12] = sqrt(s[15]) / s[16];
    out[13] = s[17];
}

void orc_stats(const double *W, const orc_params *p, double *out) { orc_stats_ranks(W, p, 1, out); }

/* ---------------------------------------------------------------------------
 * Lagrangian particles (weno/src/ParticleTrack.cpp, update.cpp:1082-1303).
 *
 * The reference interpolates the primitives at a particle with einspline's
 * 3-D cubic B-spline under natural boundary conditions (get_bsplinep,
 * Interpolation.cpp:3-31; eval_UBspline_3d_d_vg in getParticleProp,
 * ParticleTrack.cpp:90-97).  einspline is an external library that is absent
 * here (no version pinned, weno/makefileGPU:4,7,13); its construction is
 * restated from the mathematics.  On a uniform grid of N nodes
 * x_n = start + n h the interpolant is
 *   s(x) = sum_{m=0}^{N+1} c_m beta(u - m + 1),   u = (x - start) / h,
 * with beta the centred cubic B-spline (beta(0) = 2/3, beta(+-1) = 1/6) and
 *   (c_n + 4 c_{n+1} + c_{n+2}) / 6 = f_n,          n = 0 .. N-1 (interpolation)
 *   c_0 - 2 c_1 + c_2 = 0 = c_{N-1} - 2 c_N + c_{N+1}   (s'' = 0 at both ends).
 * The end conditions with the first and last interpolation rows give
 * c_1 = f_0 and c_N = f_{N-1}; c_2 .. c_{N-1} solve the tridiagonal system of
 * rows (1, 4, 1) with right-hand sides 6 f_{m-1} (the first and last less the
 * known c_1, c_N), by forward elimination with the pivots w_2 = 1/4,
 * w_m = 1/(4 - w_{m-1}), and back substitution; then c_0 = 2 c_1 - c_2 and
 * c_{N+1} = 2 c_N - c_{N-1}.  In 3-D the coefficients are the tensor product:
 * the same solve along z, then x, then y.
 * ------------------------------------------------------------------------- */
void orc_bspline_pivots(long N, double *w)
{
    for (long m = 0; m < N + 2; ++m) w[m] = 0.0;
    w[2] = 0.25;
    for (long m = 3; m < N; ++m) w[m] = 1.0 / (4.0 - w[m - 1]);
}

/* One line: c[m * stride], m = 1 .. N, hold f_{m-1} on entry (N >= 4). */
static void bspline_line(long N, double *c, long stride, const double *w)
{
    const double f0 = c[stride], fl = c[N * stride];
    double d = (6.0 * c[2 * stride] - f0) * w[2];
    c[2 * stride] = d;
    for (long m = 3; m < N - 1; ++m) {
        d = (6.0 * c[m * stride] - d) * w[m];
        c[m * stride] = d;
    }
    d = ((6.0 * c[(N - 1) * stride] - fl) - d) * w[N - 1];
    c[(N - 1) * stride] = d;
    for (long m = N - 2; m >= 2; --m) c[m * stride] = c[m * stride] - w[m] * c[(m + 1) * stride];
    c[0] = 2.0 * f0 - c[2 * stride];
    c[(N + 1) * stride] = 2.0 * fl - c[(N - 1) * stride];
}

void orc_bspline3(long N0, long N1, long N2, const double *data, double *coef)
{
    const long M0 = N0 + 2, M1 = N1 + 2, M2 = N2 + 2;
    const long Nmax = N0 > N1 ? (N0 > N2 ? N0 : N2) : (N1 > N2 ? N1 : N2);
    double *w = (double *)malloc(sizeof(double) * (size_t)(Nmax + 2));
    for (long a = 0; a < M0 * M1 * M2; ++a) coef[a] = 0.0;
    for (long j = 0; j < N0; ++j)
        for (long i = 0; i < N1; ++i)
            for (long k = 0; k < N2; ++k) coef[((j + 1) * M1 + (i + 1)) * M2 + (k + 1)] = data[(j * N1 + i) * N2 + k];
    orc_bspline_pivots(N2, w);
    for (long j = 1; j <= N0; ++j)
        for (long i = 1; i <= N1; ++i) bspline_line(N2, coef + (j * M1 + i) * M2, 1, w);
    orc_bspline_pivots(N1, w);
    for (long j = 1; j <= N0; ++j)
        for (long k = 0; k < M2; ++k) bspline_line(N1, coef + j * M1 * M2 + k, M2, w);
    orc_bspline_pivots(N0, w);
    for (long i = 0; i < M1; ++i)
        for (long k = 0; k < M2; ++k) bspline_line(N0, coef + i * M2 + k, M1 * M2, w);
    free(w);
}

/* Cell index and basis weights (values b, derivatives db with respect to u)
 * of position x on a grid of num nodes; the index is clamped to the last
 * interval. */
static long bspline_weights(double x, double start, double hinv, long num, double b[4], double db[4])
{
    const double u = (x - start) * hinv;
    long i = (long)floor(u);
    if (i < 0) i = 0;
    if (i > num - 2) i = num - 2;
    const double t = u - (double)i;
    const double s = 1.0 - t, t2 = t * t, t3 = t2 * t;
    b[0] = (s * s * s) / 6.0;
    b[1] = (3.0 * t3 - 6.0 * t2 + 4.0) / 6.0;
    b[2] = (-3.0 * t3 + 3.0 * t2 + 3.0 * t + 1.0) / 6.0;
    b[3] = t3 / 6.0;
    db[0] = -0.5 * (s * s);
    db[1] = 1.5 * t2 - 2.0 * t;
    db[2] = (-1.5 * t2 + t) + 0.5;
    db[3] = 0.5 * t2;
    return i;
}

/* Value and gradient (axes 0, 1, 2) of the tensor-product spline with
 * coefficients C (dims M1, M2 of the two faster axes) at the cell i0[3] with
 * the weights of each axis. */
static void bspline_eval(const double *C, long M1, long M2, const long i0[3], const double by[4],
                         const double dby[4], const double bx[4], const double dbx[4], const double bz[4],
                         const double dbz[4], const double hinv[3], double *val, double g[3])
{
    double v = 0.0, gy = 0.0, gx = 0.0, gz = 0.0;
    for (int a = 0; a < 4; ++a) {
        double va = 0.0, gxa = 0.0, gza = 0.0;
        for (int b = 0; b < 4; ++b) {
            const double *r = C + ((i0[0] + a) * M1 + (i0[1] + b)) * M2 + i0[2];
            const double s = ((bz[0] * r[0] + bz[1] * r[1]) + bz[2] * r[2]) + bz[3] * r[3];
            const double sd = ((dbz[0] * r[0] + dbz[1] * r[1]) + dbz[2] * r[2]) + dbz[3] * r[3];
            va += bx[b] * s;
            gxa += dbx[b] * s;
            gza += bx[b] * sd;
        }
        v += by[a] * va;
        gy += dby[a] * va;
        gx += by[a] * gxa;
        gz += by[a] * gza;
    }
    *val = v;
    g[0] = gy * hinv[0];
    g[1] = gx * hinv[1];
    g[2] = gz * hinv[2];
}

void orc_spline_eval(long N0, long N1, long N2, const double *coef, const double start[3], const double hinv[3],
                     long n, const double *pos, double *val, double *grad)
{
    const long num[3] = {N0, N1, N2};
    for (long p = 0; p < n; ++p) {
        double b[3][4], db[3][4];
        long i0[3];
        for (int a = 0; a < 3; ++a) i0[a] = bspline_weights(pos[a * n + p], start[a], hinv[a], num[a], b[a], db[a]);
        double g[3];
        bspline_eval(coef, N1 + 2, N2 + 2, i0, b[0], db[0], b[1], db[1], b[2], db[2], hinv, &val[p], g);
        for (int a = 0; a < 3; ++a) grad[a * n + p] = g[a];
    }
}

/* The spline grid of one rank's padded block along an axis (get_bsplinep,
 * Interpolation.cpp:10-27): nt nodes from (sta - 3) dx + dx/2; einspline
 * derives the spacing from the end points, (end - start) / (num - 1). */
static void particle_grid(const orc_params *p, double *start, double *hinv)
{
    const long nt = p->nc + 6;
    const double st = (0 - 3) * p->dx + 0.5 * p->dx; /* sta = 0 on one rank */
    const double en = st + (nt - 1) * p->dx;
    *start = st;
    *hinv = 1.0 / ((en - st) / (double)(nt - 1));
}

/* generateSplines (update.cpp:1199-1213) over the padded block W (ghosts
 * filled), then getParticleProp (ParticleTrack.cpp:90-97) at every particle.
 * rec: ORC_PREC_FIELDS x n doubles, field-major; fields 0-2 (position
 * y, x, z = pos[0..2]) are read, 3-22 written: DEN, U[0..2], P and the
 * gradients (d/dy, d/dx, d/dz) of DEN, U[0], U[1], U[2], P. */
void orc_particle_props(const double *W, const orc_params *p, long n, double *rec)
{
    const long nt = p->nc + 6, Nt = nt * nt * nt, M = nt + 2;
    double *prim5 = (double *)malloc(sizeof(double) * (size_t)(5 * Nt));
    double *coef = (double *)malloc(sizeof(double) * (size_t)(M * M * M));
    for (long c = 0; c < Nt; ++c) {
        const double den = W[c];
        const double u = W[Nt + c] / den, v = W[2 * Nt + c] / den, w = W[3 * Nt + c] / den;
        const double Vsqr = u * u + v * v + w * w;
        prim5[c] = den;
        prim5[Nt + c] = u;
        prim5[2 * Nt + c] = v;
        prim5[3 * Nt + c] = w;
        prim5[4 * Nt + c] = (den * (p->gam - 1)) * (W[4 * Nt + c] / den - 0.5 * Vsqr);
    }
    double start, hinv;
    particle_grid(p, &start, &hinv);
    const double st3[3] = {start, start, start}, hi3[3] = {hinv, hinv, hinv};
    double *val = (double *)malloc(sizeof(double) * (size_t)n);
    double *grad = (double *)malloc(sizeof(double) * (size_t)(3 * n));
    for (int q = 0; q < 5; ++q) {
        orc_bspline3(nt, nt, nt, prim5 + q * Nt, coef);
        orc_spline_eval(nt, nt, nt, coef, st3, hi3, n, rec, val, grad);
        for (long a = 0; a < n; ++a) {
            rec[(3 + q) * n + a] = val[a];
            for (int d = 0; d < 3; ++d) rec[(8 + 3 * q + d) * n + a] = grad[d * n + a];
        }
    }
    free(grad);
    free(val);
    free(coef);
    free(prim5);
}

/* Particle::updatePosition (ParticleTrack.cpp:43-65): forward Euler with the
 * velocity of the last getParticleProp (pos[0] = y moves with U[1] = v,
 * pos[1] = x with U[0] = u), each coordinate wrapped once into [0, 2 pi]. */
void orc_particle_track(long n, double *rec, double dt)
{
    const double twopi = 2 * atan(1.0) * 4.0; /* 2*pi with param.h:14's pi */
    for (long a = 0; a < n; ++a) {
        double *py = rec + a, *px = rec + n + a, *pz = rec + 2 * n + a;
        *py += rec[5 * n + a] * dt;
        *px += rec[4 * n + a] * dt;
        *pz += rec[6 * n + a] * dt;
        double *pp[3] = {py, px, pz};
        for (int q = 0; q < 3; ++q) {
            if (*pp[q] > twopi) *pp[q] = *pp[q] - twopi;
            if (*pp[q] < 0) *pp[q] = twopi + *pp[q];
        }
    }
}

/* GetParticleStats (update.cpp:1134-1181) on one rank: out[9] = part_TKE,
 * part_SijSij, DUDX2, DUDX3, DWDZ2, DWDZ3, part_SKEWu, part_SKEWw, count. */
void orc_particle_stats(long n, const double *rec, double *out)
{
    double tke = 0.0, sij = 0.0, d2 = 0.0, d3 = 0.0, w2 = 0.0, w3 = 0.0;
    for (long a = 0; a < n; ++a) {
        const double U0 = rec[4 * n + a], U1 = rec[5 * n + a], U2 = rec[6 * n + a];
        tke += (U0 * U0 + U1 * U1 + U2 * U2);
        const double dudy = rec[11 * n + a], dudx = rec[12 * n + a], dudz = rec[13 * n + a];
        const double dvdy = rec[14 * n + a], dvdx = rec[15 * n + a], dvdz = rec[16 * n + a];
        const double dwdy = rec[17 * n + a], dwdx = rec[18 * n + a], dwdz = rec[19 * n + a];
        sij += (dudx * dudx + 0.5 * pow(dudy + dvdx, 2) + 0.5 * pow(dudz + dwdx, 2) + 0.5 * pow(dwdy + dvdz, 2) +
                dvdy * dvdy + dwdz * dwdz);
        d2 += dudx * dudx;
        d3 += dudx * dudx * dudx;
        w2 += dwdz * dwdz;
        w3 += dwdz * dwdz * dwdz;
    }
    tke /= n;
    sij /= n;
    d2 /= n;
    d3 /= n;
    w2 /= n;
    w3 /= n;
    out[0] = tke;
    out[1] = sij;
    out[2] = d2;
    out[3] = d3;
    out[4] = w2;
    out[5] = w3;
    out[6] = d3 / pow(d2, 1.5);
    out[7] = w3 / pow(w2, 1.5);
    out[8] = (double)n;
}
