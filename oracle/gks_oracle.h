/*
 * CPU oracle for the GKM-DNS WENO-GKS step: a plain-C restatement of the
 * reference's CPU hot path (weno/src/update.cpp built with -DUseCPU and
 * weno/src/GKMflux.cpp).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this library, and only as the checker.
 * The product library (gkm-dns_b200/csrc) never links or calls it.
 *
 * Each formula keeps the reference's operation order so that, built without
 * FMA contraction, results agree with the reference build bit for bit; the
 * pinning tests check that against oracle/_ref (the reference compiled from
 * its own sources).
 *
 * Field layout (the reference's, weno/src/param.h:37): a padded block of
 * nt = nc + 6 cells per edge (3 ghost layers), linear index
 * (j*nt + i)*nt + k with j = y slowest, i = x, k = z fastest, and the five
 * conserved components (rho, rho u, rho v, rho w, rho E) stored one after the
 * other (component q at offset q*nt^3).
 */
#ifndef GKS_ORACLE_H
#define GKS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_VISC_SUTHERLAND = 0, /* mu0 (T/T0)^1.5 (T0+110.4)/(T+110.4), update.cpp:263 */
    ORC_VISC_POWER = 1       /* mu0 (T/T0)^visc_exp, GKM/CUDA GKM/src/CPUupdate.cpp:65 */
};

enum {
    ORC_FIX_ZSWEEP = 1,      /* z sweep: transverse slopes along the rotated axes */
    ORC_DIRECT_ENERGY = 2    /* WENO on rho E directly (GPUupdate.cu:542-546) */
};

typedef struct {
    int nc;           /* interior cells per edge */
    int K;            /* internal degrees of freedom, FlowField.cpp:41 */
    int visc_law;     /* ORC_VISC_* */
    int flags;        /* ORC_FIX_ZSWEEP | ORC_DIRECT_ENERGY */
    double gam;       /* ratio of specific heats */
    double R;         /* gas constant, param.h:18 (287) */
    double dx;        /* 2 pi / nc, FlowField.cpp:45 */
    double T0;        /* p0 / (R rho0), FlowField.cpp:46 */
    double mu0;       /* reference viscosity */
    double visc_exp;  /* exponent of the power law */
    double pr_factor; /* factor on the energy slope coefficient: 1/0.7 (GKMflux.cpp:289) or 1 (GPUupdate.cu:839) */
    double p0, den0, Mt, t0; /* normalisation of the printed statistics, update.cpp:772-776 */
} orc_params;

/* WENO-SYMOO of one 6-cell stencil s[0..5] = (LLL, LL, L, R, RR, RRR), five
 * components each; energy through temperature unless direct_energy. */
void orc_weno(const double *s, double gam, double R, int direct_energy, double *wl, double *wr);

/* Time-integrated BGK-NS interface flux (GKMflux.cpp:11-215).
 * in[53] = WL, WR, Wl, Wr, DWxl, DWxr, DWyl, DWyr, DWzl, DWzr (5 each), tau, dt, dx. */
void orc_flux(const double *in, double gam, int K, double pr_factor, double *F);

/* Periodic fill of the 3 ghost layers of all five components. */
void orc_halo(double *W, int nc);

/* One time step in place: three sweeps + conservative update of the interior,
 * then the periodic ghost fill.  F is scratch of 15 * nt^3 doubles. */
void orc_step(double *W, const orc_params *p, double dt, double *F);

/* Largest |u| + c over the interior (update.cpp:1057-1079). */
double orc_maxval(const double *W, const orc_params *p);

/* Diagnostics of PrintStats (update.cpp:638-784) with node gradients of the
 * natural cubic spline over the padded block.  out[14] =
 * TKE, Diss, SKEWu, SKEWv, SKEWw, KURTu, KURTv, KURTw, Prms, Trms, Vrms,
 * SijSij, Mt (sqrt<|u|^2> / <c>), mean density. */
void orc_stats(const double *W, const orc_params *p, double *out);

/* The same for the field split over nranks ranks along y (procDim = {nranks,
 * 1, 1}; nc divisible by nranks): every rank's sums over its own segment,
 * with splines over the segment's padded nodes, reduced over the ranks as the
 * reference's PrintStats does with MPI (update.cpp:638-784). */
void orc_stats_ranks(const double *W, const orc_params *p, int nranks, double *out);


/* Lagrangian particles (ParticleTrack.cpp, update.cpp:1082-1303), restated
 * from the mathematics of einspline's natural cubic B-spline (see
 * gks_oracle.c).  A particle record holds ORC_PREC_FIELDS doubles, stored
 * field-major (field f of particle a at f*n + a): 0-2 position (y, x, z), 3 DEN,
 * 4-6 U (u, v, w), 7 P, then (d/dy, d/dx, d/dz) of DEN (8-10), u (11-13),
 * v (14-16), w (17-19), P (20-22). */
#define ORC_PREC_FIELDS 23

/* Pivots w[0 .. N+1] of the (1, 4, 1) elimination (w[2] .. w[N-1] used). */
void orc_bspline_pivots(long N, double *w);

/* Natural cubic B-spline coefficients of data[N0][N1][N2] into
 * coef[N0+2][N1+2][N2+2] (N0, N1, N2 >= 4). */
void orc_bspline3(long N0, long N1, long N2, const double *data, double *coef);

/* Value and gradient of that spline at n points pos[3][n] (axes 0, 1, 2) on
 * grids start[a] + m / hinv[a]: val[n], grad[3][n]. */
void orc_spline_eval(long N0, long N1, long N2, const double *coef, const double start[3], const double hinv[3],
                     long n, const double *pos, double *val, double *grad);

/* generateSplines + getParticleProp of every particle (positions in rec). */
void orc_particle_props(const double *W, const orc_params *p, long n, double *rec);

/* Particle::updatePosition of every particle. */
void orc_particle_track(long n, double *rec, double dt);

/* GetParticleStats: out[9] = TKE, SijSij, DUDX2, DUDX3, DWDZ2, DWDZ3, SKEWu,
 * SKEWw, particle count. */
void orc_particle_stats(long n, const double *rec, double *out);

#ifdef __cplusplus
}
#endif

#endif
