/*
 * gks_b200: B200 (sm_100a) implementation of the GKM-DNS per-step hot path --
 * WENO-SYMOO interface reconstruction in the x/y/z sweeps, the BGK gas-kinetic
 * interface flux and the conservative update -- behind a plain C ABI.
 *
 * Replaces, in the reference (nishantp9/GKM-DNS, WENO tree):
 *   void evolve(ptype *W[5], DevAlloc *dev, ptype dt)        weno/src/GPUupdate.h:33
 *   void evolveEulerian(ptype *W[5], ptype *Fx[5], ...)       weno/src/update.h:16 (CPU path)
 *   class DevAlloc (50 device buffers)                        weno/src/GPUAlloc.h:6-22
 *   void timestep(ptype *W[5])                                weno/src/update.cpp:1057-1079
 *   void PrintStats(ptype *W[5], UBspline_3d_d *splinep[5])   weno/src/update.cpp:638-784
 *   void HaloTransfer(...) on one periodic rank               weno/src/update.cpp:894-1054
 *   HaloTransfer's y exchange between ranks (send_HaloS/N)    weno/src/update.cpp:899-954
 *   segment() / procDim y-decomposition                       weno/src/FlowField.cpp:278-288, Main.cpp:21-30
 * The compatibility shim with the reference's own evolve()/DevAlloc
 * signatures is gkm-dns_b200/driver/gks_compat.h.
 *
 * Conventions
 * - A field is the reference's padded block: nt = nc + 6 cells per edge
 *   (3 ghost layers), linear index (j*nt + i)*nt + k with j = y slowest,
 *   i = x, k = z fastest (weno/src/param.h:37), five separate double arrays
 *   rho, rho u, rho v, rho w, rho E.  The domain is the periodic cube
 *   [0, 2 pi)^3, dx = 2 pi / nc.
 * - The state stays resident on the device between calls; upload/download
 *   convert between the host's padded layout and the device layout
 *   (interior only; the periodic halo is applied inside the kernels).
 * - One context holds one field or a batch of independent fields of
 *   different sizes (an ensemble); every stage of a step advances all fields
 *   of the context in one launch.
 * - Every call returns 0 on success or a negative GKS_E* code; the message of
 *   the last failure is gks_last_error(ctx).  A context is not thread-safe.
 */
#ifndef GKS_B200_H
#define GKS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GKS_ABI_VERSION 1

/* precision */
#define GKS_FP64 0  /* every operation in FP64 (parity path) */
#define GKS_MIXED 1 /* WENO weights, slope solves, slope moments in FP32; moments, erfc, update, reductions FP64 */

/* flags: the reference's behaviour is the default (0) */
#define GKS_FIX_ZSWEEP 1    /* z sweep: transverse slopes along the rotated frame's axes
                               (the reference uses d/dx and d/dy in swapped slots, update.cpp:380-421) */
#define GKS_DIRECT_ENERGY 2 /* WENO on rho E directly, as the reference GPU kernel does
                               (GPUupdate.cu:542-546); default is WENO of T (update.cpp:560-619) */

/* viscosity law */
#define GKS_VISC_SUTHERLAND 0 /* mu0 (T/T0)^1.5 (T0+110.4)/(T+110.4), update.cpp:263 */
#define GKS_VISC_POWER 1      /* mu0 (T/T0)^visc_exp, GKM/CUDA GKM/src/CPUupdate.cpp:65 */

/* error codes */
#define GKS_OK 0
#define GKS_EINVAL (-1)   /* bad argument */
#define GKS_ECUDA (-2)    /* CUDA runtime failure */
#define GKS_ENOMEM (-3)   /* device allocation failed */
#define GKS_ESTATE (-4)   /* call out of order (e.g. step before upload / dt) */
#define GKS_ENONFINITE (-5) /* non-finite or non-positive density/pressure found */
#define GKS_ETOOBIG (-6)  /* size beyond a fixed capacity */

typedef struct gks_ctx gks_ctx;

/* Physical constants of one field; the reference reads them from
 * InitialConditions/params and param.h (FlowField.cpp:15-50). */
typedef struct {
    int nc;           /* interior cells per edge (>= 4) */
    int K;            /* internal degrees of freedom, int((5-3 gam)/(gam-1)) (FlowField.cpp:41) */
    int visc_law;     /* GKS_VISC_* */
    int reserved;
    double gam;       /* ratio of specific heats */
    double gas_r;     /* gas constant R (287, param.h:18); not named R, which param.h defines as a macro */
    double T0;        /* p0 / (R rho0) (FlowField.cpp:46) */
    double mu0;       /* viscosity at T0 */
    double visc_exp;  /* exponent of GKS_VISC_POWER */
    double pr_factor; /* factor on the energy slope coefficient: 1/0.7 as the CPU reference
                         (GKMflux.cpp:289), 1.0 as the GPU reference (GPUupdate.cu:839) */
    double p0, den0, Mt, t0; /* normalisation of the statistics (update.cpp:772-776) */
} gks_phys;

/* Diagnostics of one field (PrintStats, update.cpp:638-784). */
typedef struct {
    double tke;      /* <rho |u|^2> */
    double diss;     /* <mu du_i/dx_j du_i/dx_j> */
    double skew[3];  /* <(du/dx)^3>/<(du/dx)^2>^1.5, same for dv/dy, dw/dz */
    double kurt[3];  /* <(du/dx)^4>/<(du/dx)^2>^2, ... */
    double prms;     /* rms pressure / (gam p0 Mt^2) */
    double trms;     /* rms temperature / ((gam-1) T0 Mt^2) */
    double vrms;     /* rms specific volume / (Mt^2 / den0) */
    double sijsij;   /* <S_ij S_ij> (computed, not printed, by the reference) */
    double mach_t;   /* sqrt(<|u|^2>) / <c> (not in the reference's printout) */
    double rho_mean; /* <rho> */
} gks_stats_out;

/* Create a context for nfields fields with the given constants (one gks_phys
 * per field).  precision is GKS_FP64 or GKS_MIXED; flags a GKS_FIX_* mask. */
int gks_create(gks_ctx **out, int nfields, const gks_phys *phys, int precision, int flags);
void gks_destroy(gks_ctx *ctx);
const char *gks_last_error(const gks_ctx *ctx);

/* Host <-> device state of field f, reference padded layout (ghosts are
 * ignored on upload and written as the periodic image on download, i.e. the
 * state after the reference's HaloTransfer). */
int gks_upload(gks_ctx *ctx, int f, double *const W[5]);
int gks_download(gks_ctx *ctx, int f, double *const W[5]);

/* The reference's per-step call, evolve(W, dev, dt) (GPUupdate.h:33,
 * GPUupdate.cu:65-196): upload W (padded layout), advance nsteps steps with
 * the field's dt (gks_set_dt / gks_timestep), download W with its ghosts as
 * the periodic image.  Synchronous; the state stays resident afterwards.  For
 * one field and one step the copies overlap the step: W goes up in y-slabs on
 * one copy stream, each slab's stages run as soon as the planes they read
 * have arrived, and updated planes come back on another copy stream -- with W
 * in pinned (page-locked) host memory both PCIe directions and the kernels
 * run concurrently; pageable W works but overlaps less.  When the five arrays
 * lie one after another in one block (W[q] = W[0] + q (nc+6)^3), each slab
 * moves in one pitched copy per direction instead of five; page-lock such a
 * block as one range (gks_host_register) to keep that.  The first such call
 * allocates 25 nc^3 + 5 (nc+6)^3 doubles of pipeline buffers for the context
 * (4.1 GB at 256^3).  Otherwise (an ensemble, nsteps > 1, nc < 16) it is
 * gks_upload + gks_step + gks_download.  Results are bit-identical either way.
 * After a failure the field's device state is undefined: upload it again. */
int gks_evolve(gks_ctx *ctx, int f, double *const W[5], int nsteps);

/* Page-lock `bytes` of caller memory at p (cudaHostRegister) so that copies
 * from and to it run asynchronously at full PCIe rate -- what gks_evolve
 * needs to overlap them.  *registered (may be NULL) is set to 1 if this call
 * registered the range, 0 if it was page-locked already (nothing done).
 * Release with gks_host_unregister before freeing the memory.  No counterpart
 * in the reference, which copies from pageable memory (GPUupdate.cu:74-78). */
int gks_host_register(void *p, size_t bytes, int *registered);
int gks_host_unregister(void *p);

/* Time step: dt = cfl*dx/max(|u|+c) over the interior (timestep,
 * update.cpp:1057-1079); the result is also made the step's dt. */
int gks_timestep(gks_ctx *ctx, int f, double cfl, double *dt_out);
int gks_set_dt(gks_ctx *ctx, int f, double dt);

/* Advance every field of the context by nsteps single-stage steps
 * (evolveEulerian, update.cpp:194-199): three fused reconstruction + flux
 * sweeps and the conservative update per step, captured once as a CUDA
 * graph.  Asynchronous on the context's stream. */
int gks_step(gks_ctx *ctx, int nsteps);

/* Diagnostics of field f on the current state (synchronises). */
int gks_stats(gks_ctx *ctx, int f, gks_stats_out *out);

/* The diagnostics as a mergeable part, for a field split over ranks: part[28]
 * receives the means over field f's interior cells of the 18 quantities
 * PrintStats sums (update.cpp:659-712), the means of x - K and (x - K)^2 for
 * x = p, T, 1/rho, the shifts K (x at the first interior cell) and the number
 * of interior cells.  gks_stats_reduce merges the parts of all ranks (the
 * reference's MPI_Reduce / MPI_Allreduce of the sums, update.cpp:714-762) into
 * the normalised output; gks_stats(ctx, f, out) equals gks_stats_part followed
 * by gks_stats_reduce of that one part. */
int gks_stats_part(gks_ctx *ctx, int f, double *part);
int gks_stats_reduce(const double *parts, int nparts, const gks_phys *phys, gks_stats_out *out);

/* One y-slab of a periodic nc^3 field split over ranks along y -- the
 * reference's decomposition with procDim = {P, 1, 1} (Main.cpp:21-30,
 * segment(), FlowField.cpp:278-288): ny interior planes (nc_segy, >= 3)
 * starting at global plane y0 (sta[0]).  Host arrays are the rank's padded
 * block, (ny + 6) x (nc + 6) x (nc + 6); the device stores the ny interior
 * planes with the three ghost planes either side, and x / z stay periodic
 * inside the slab.  gks_upload takes the ghost planes from the host block;
 * gks_download writes the interior planes with their x / z ghosts and leaves
 * the y ghost planes as they were uploaded, as the reference's evolve leaves
 * ghosts until the next HaloTransfer.  After the upload and after every step
 * the caller exchanges the y halo (gks_halo_*), as the reference's Evolve
 * calls HaloTransfer (update.cpp:106-108, 140-142): a step, and the
 * diagnostics, read ghost planes that must hold the neighbours' current
 * state.  gks_timestep gives the slab's own dt (the field's is the minimum
 * over ranks); gks_stats_part its part of the diagnostics, with y-derivatives
 * from splines over the slab's padded block as the reference's multi-rank
 * PrintStats takes them (Interpolation.cpp:10-27).
 * gks_step and gks_evolve advance a slab one step per call (more return
 * GKS_EINVAL: its ghosts would go stale).  The stage timer and the tuner run
 * whole-field launches and refuse a slab; gks_set_launch pins a
 * configuration tuned on a periodic field. */
int gks_create_slab(gks_ctx **out, const gks_phys *phys, int ny, int y0, int precision, int flags);

/* The slab's four halo buffers in device memory, each 15 nc^2 doubles laid out
 * [component][plane 0..2][nc^2] (send_HaloS / recv_HaloS of update.cpp:899-954
 * without the x / z ghost columns): bufs[0] send south (interior planes 0-2),
 * bufs[1] send north (the last three interior planes), bufs[2] receive from
 * the south neighbour (its last three), bufs[3] receive from the north
 * neighbour (its first three).  *elems (may be NULL) = 15 nc^2. */
int gks_halo_buffers(gks_ctx *ctx, double **bufs, size_t *elems);

/* Copy the boundary planes into the send buffers / the receive buffers into
 * the ghost planes; asynchronous on the context's stream, like gks_step.
 * One exchange step of the halo is pack, send south and north / receive from
 * north and south (NCCL, MPI or a device copy), unpack. */
int gks_halo_pack(gks_ctx *ctx);
int gks_halo_unpack(gks_ctx *ctx);

/* Wait for all work of the context. */
int gks_sync(gks_ctx *ctx);

/* Check every field for non-finite or non-positive density / pressure; returns
 * GKS_ENONFINITE and names the first offending field in gks_last_error. */
int gks_check(gks_ctx *ctx);

/* Device-resident arrays of field f (nc^3 doubles each, index
 * (j*nc + i)*nc + k; for a slab (ny + 6) nc^2, its ghost planes included),
 * for callers that keep the state on the GPU. */
int gks_device_fields(gks_ctx *ctx, int f, double *dW[5]);

/* Run subsequent work on a caller-provided cudaStream_t (NULL: the context's
 * own stream).  Invalidates the captured step graph. */
int gks_set_stream(gks_ctx *ctx, void *stream);

/* The cudaStream_t the context launches on (for event timing by callers). */
int gks_get_stream(gks_ctx *ctx, void **stream);

/* Make `device` the calling thread's CUDA device for this library (contexts
 * are created on the device current at gks_create). */
int gks_select_device(int device);

/* Advance reps steps launching the seven stages one by one with CUDA events
 * between them; ms[0..6] receives the mean time of recon x, flux x, recon y,
 * flux y, recon z, flux z, update.  For profiling: the state advances. */
int gks_time_stages(gks_ctx *ctx, int reps, double *ms);

/* Tune the launch configuration of the reconstruction and flux kernels of
 * every sweep on the context's current fields: register-cap variant (resident
 * blocks per SM) and persistent grid size, each candidate timed with CUDA
 * events over `reps` launches.  Results are cached per process by device,
 * precision, flags and field sizes; the state is not modified. */
int gks_autotune(gks_ctx *ctx, int reps);

/* The launch configuration in use: kind 0 reconstruction, 1 flux, 2 update;
 * dir 0..2 = x, y, z. */
int gks_get_launch(gks_ctx *ctx, int kind, int dir, int *block, int *grid, int *variant);

/* Pin the launch configuration of one kernel kind and sweep (for example to
 * restore a tuning saved by a previous run): `variant` indexes the kind's
 * register-cap variants (gks_get_launch reports the one in use), `grid` is the
 * number of blocks of the persistent grid-stride launch, 0 for one wave of
 * resident blocks.  Results do not depend on the configuration. */
int gks_set_launch(gks_ctx *ctx, int kind, int dir, int grid, int variant);

/* Peak FMA throughput of the FP64 (GKS_FP64) or FP32 (GKS_MIXED) pipe of
 * the current device in TFLOP/s, 2 flops per FMA (a short microbenchmark). */
int gks_peak_flops(int precision, double *tflops);

/* Lagrangian particles of field f (a whole periodic field, not a y-slab),
 * replacing the reference's particle tracker on one rank:
 *   locateParticles (reads InitialConditions/unirand)  weno/src/update.cpp:1269-1292
 *   generateSplines + Particle::getParticleProp        weno/src/update.cpp:1199-1213,
 *                                                      ParticleTrack.cpp:90-97
 *   evolveParticles / Particle::track (one rank)        weno/src/update.cpp:1082-1131,
 *                                                      ParticleTrack.cpp:38-65
 *   GetParticleStats                                    weno/src/update.cpp:1134-1181
 * (the reference defines these but its Evolve loop never calls them).
 * A particle record holds GKS_PREC_FIELDS doubles; gks_particles_get returns
 * them field-major (field q of particle a at rec[q*n + a]):
 *   0-2   position pos[0..2] = (y, x, z), in [0, 2 pi]
 *   3     DEN           4-6  U[0..2] = (u, v, w)      7  P
 *   8-10  gradD (d/dy, d/dx, d/dz)   11-13 gradU   14-16 gradV
 *   17-19 gradW         20-22 gradP
 * Values and gradients come from the natural cubic B-spline interpolant of
 * the primitives over the padded block (einspline's UBspline_3d_d with
 * NATURAL ends, as get_bsplinep builds it, Interpolation.cpp:3-31), in FP64
 * whatever the context's precision.
 *
 * gks_particles_locate: n particles at (x0[a], y0[a], z0[a]) -- the three
 * arrays of InitialConditions/unirand in the order the reference reads them
 * -- with zero velocity and properties; replaces the field's particles.
 * gks_particles_props: the splines of the field's current state and every
 * particle's values and gradients (asynchronous on the context's stream; the
 * first call allocates 5 (nc+8)^3 doubles of spline coefficients).
 * gks_particles_track: every particle moves by dt with the velocity of the
 * last props call (forward Euler, each coordinate wrapped into [0, 2 pi], as
 * Particle::updatePosition); asynchronous.
 * gks_particles_stats: GetParticleStats' means over the particles
 * (synchronises).  gks_particles_get: the records into host memory
 * (GKS_PREC_FIELDS x n doubles; synchronises). */
#define GKS_PREC_FIELDS 23

typedef struct {
    double tke;            /* <|U|^2> over the particles (part_TKE; no factor 1/2, update.cpp:1144) */
    double sijsij;         /* <S_ij S_ij> (part_SijSij) */
    double dudx2, dudx3;   /* <(du/dx)^2>, <(du/dx)^3> */
    double dwdz2, dwdz3;   /* <(dw/dz)^2>, <(dw/dz)^3> */
    double skew_u, skew_w; /* part_SKEWu, part_SKEWw */
    long long count;       /* particles (totalCount) */
} gks_particle_stats_out;

int gks_particles_locate(gks_ctx *ctx, int f, int n, const double *x0, const double *y0, const double *z0);
int gks_particles_props(gks_ctx *ctx, int f);
int gks_particles_track(gks_ctx *ctx, int f, double dt);
int gks_particles_stats(gks_ctx *ctx, int f, gks_particle_stats_out *out);
int gks_particles_get(gks_ctx *ctx, int f, double *rec);

/* The time step without allocating anything -- for callers that may not
 * allocate device memory: host codes that own and pool every byte of device
 * memory themselves, and loops that cannot afford cudaMalloc's implicit
 * device synchronisation (gks_create, which gks_timestep needs, allocates).
 * No counterpart in the reference: its timestep() (update.cpp:1057-1079) runs
 * on the host.
 * dW: the caller's five device arrays in this library's interior layout
 * (nc^3 doubles each, index (j*nc + i)*nc + k), e.g. from gks_device_fields.
 * Returns dt = cfl * (2 pi/nc) / max(|u| + c) in *dt_out (host memory), the
 * same value gks_timestep gives; it synchronises `stream` (NULL: the legacy
 * default stream) to hand dt back.  Limit: nc <= 1024, else GKS_ETOOBIG.
 * It cannot be called while `stream` is being captured into a graph: it
 * synchronises the stream and copies dt into host memory, neither of which a
 * capture allows.  Scratch is a fixed file-scope device array of 1026 64-bit
 * words that every GPU loading the library holds until exit; the first call
 * on a device (and the first after its CUDA context is replaced, e.g. by
 * cudaDeviceReset) looks up the array's address.  Calls share the scratch:
 * calls that overlap on the GPU race and must be serialised. */
int gks_timestep_noalloc(const double *const dW[5], int nc, double gam, double cfl, void *stream,
                         double *dt_out);

#ifdef __cplusplus
}
#endif

#endif
