// Field descriptors and kernel launchers shared by the kernels (gks_kernels.cu)
// and the C ABI (gks_capi.cu).
//
// Device layout of a field: five arrays of nc^3 doubles (interior cells only,
// index (j*nc + i)*nc + k, j = y, i = x, k = z), the periodic halo being
// applied by index wrapping inside the kernels.  One y-slab of a field split
// over ranks along y stores its ny interior planes with the three ghost
// planes either side (ny + 6 planes; x and z still wrap), which the halo
// exchange between steps fills.  Per field the context also
// holds a reconstruction buffer (the left and right WENO states of the
// interface at the high side of every cell, for the sweep in progress: ten
// values per cell as five arrays of 16-byte pairs; the slab-pipelined host
// step gives each sweep its own buffer) and a flux buffer (15 arrays: the x,
// y and z interface fluxes of the step).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gks_limits.h"

namespace gks {

struct FieldDev {
    double *W[5];     // state, interior layout
    double *Wout[5];  // where the update writes the new state: W itself, except in the slab-pipelined host step
    double *rec[3];   // per sweep x, y, z: five arrays of nc^3 16-byte pairs, Wl[0..4] then Wr[0..4]
                      // (one shared buffer except in the pipelined step)
    double *F[15];    // Fx[0..4], Fy[0..4], Fz[0..4]
    double *tau[2];   // mu/p of each cell as numerator / denominator, set by the x-sweep reconstruction
    const double *spl_cp;   // natural-spline Thomas coefficients of the x / z lines, nc + 6 entries
    const double *spl_inv;  // reciprocal pivots, nc + 6 entries
    const double *spl_cpy;  // the same for the y lines: ny + 2 yhost entries (== spl_cp but for a slab)
    const double *spl_invy;
    long long base;   // first work item of this field in the batch (a multiple of kItemAlign)
    long long ncell;  // ny * nc^2 (< 2^31)
    long long wbase;  // first window item of this field (x / y reconstruction; a multiple of kItemAlign)
    long long nwin;   // window items: nc^2 * nrun
    int run;          // interfaces per window item (the same for every field of a batch)
    int nrun;         // runs per line: ceil(nc / run)
    long long zbase;  // first z-segment item of this field (z reconstruction; one warp per item)
    long long nzseg;  // z segments: nc^2 * ceil(nc / 32)
    int nc;           // cells per edge along x and z (and of the whole field along y)
    int ny;           // planes stored along y: nc, or a slab's interior planes + 6
    int nyw;          // modulus of the y-index wrap: nc, or kNoWrap for a slab (its ghosts are stored)
    int yhost;        // device plane j is plane j + yhost of the padded host layout: 3, or 0 for a slab
    int ylo, yhi;     // interior planes [ylo, yhi): [0, nc), or [3, ny - 3) for a slab
    unsigned nc_magic; // x / nc == (umulhi(x, nc_magic) + x) >> nc_shift for 32-bit x
    int nc_shift;
    int K;
    int visc_law;     // 0 Sutherland, 1 power law
    int flags;        // GKS_FIX_ZSWEEP | GKS_DIRECT_ENERGY
    double dx, inv_dx, dt;
    double gam, gm1, R, iR, cT, icT; // iR = 1/R, cT = (gam-1)/R, icT = R/(gam-1)
    double T0, iT0, mu0, visc_exp;
    double kA;        // pr_factor * 4/(K+3)
    double spl_s;     // 3/h of the spline grid along x and z
    double spl_sy;    // along y (a slab's grid starts at its own first plane)
    // flux constants computed once on the host (no per-interface conversions
    // or products): 1/(2 (gam-1)), slope scales 2/dx and 1/(2 dx), (K+2)/2,
    // and K + 2, K + 4, (K+2)(K+4), -(K+3) in double and in float
    double hig, ksn, kst, hK2;
    double kd[4];
    float kf[4];
};

// y-wrap modulus of a slab: larger than any plane index, so nothing wraps.
constexpr int kNoWrap = 1 << 30;

// Field item ranges start at multiples of this, so that a block of up to
// kItemAlign consecutive items never spans two fields.
constexpr int kItemAlign = 256;

// Longest run of interfaces per work item of the windowed x / y
// reconstruction, for either precision (0 FP64, 1 mixed; 64 measured fastest
// on B200 at 256^3 for both).  A batch halves it, down to kWinRunMin, while it has fewer than
// kWinItemsPerSm items per SM, so that small fields still fill the GPU.
__host__ __device__ constexpr int win_run(int) { return 64; }
constexpr int kWinRunMin = 8;
constexpr int kWinItemsPerSm = 768;

struct Batch {
    FieldDev *fields; // device array
    int nfields;
    long long total;  // end of the last field's item range
    long long wtotal; // end of the last field's window item range
    long long ztotal; // end of the last field's z-segment item range
    int *err;         // device error word (bit 0: non-finite / non-positive state after update)
    // work items a launch processes: [lo, hi) of the launched kernel's item
    // space; hi < 0 means all of them (the launchers fill the range in)
    long long lo = 0, hi = -1;
    // the descriptor of a one-field batch (nfields == 1), equal to fields[0]:
    // kernels read it from their launch parameters
    FieldDev one;
};

// Launch configuration chosen by the tuner per kernel kind and sweep: block
// size, persistent grid, and the register-cap variant of the kernel.
struct LaunchCfg {
    int block;
    int grid;
    int variant;
};

enum KernelKind { K_RECON = 0, K_FLUX = 1, K_UPDATE = 2, K_KINDS = 3 };
constexpr int kReconVariants = 6;
constexpr int kFluxVariants = 3;

// Threads per block of each kernel kind.
constexpr int kReconBlock = 128;
constexpr int kFluxBlock = 64;
constexpr int kUpdateBlock = 256;

// Work items of a kernel kind / sweep / variant over the whole batch: window
// runs (x / y reconstruction variants 0-2), z segments of one warp each (z
// reconstruction variants 0-2), else cells.
inline long long batch_items(const Batch &b, int kind, int dir, int variant)
{
    if (kind == K_RECON && variant < 3) return dir < 2 ? b.wtotal : b.ztotal;
    return b.total;
}

// Stage launchers (asynchronous on `st`).  prec: 0 FP64, 1 mixed.  Each
// processes the items [b.lo, b.hi) (all items when b.hi < 0) with at most
// cfg.grid blocks.
cudaError_t launch_recon(const Batch &b, int dir, int prec, LaunchCfg cfg, cudaStream_t st);
cudaError_t launch_flux(const Batch &b, int dir, int prec, LaunchCfg cfg, cudaStream_t st);
cudaError_t launch_update(const Batch &b, LaunchCfg cfg, cudaStream_t st);

// Resident blocks per SM of a kernel kind / variant (for persistent grids).
cudaError_t max_resident_blocks(int kind, int dir, int prec, int variant, int block, int *blocks_per_sm);

// Layout conversion of one field: padded host layout (5 x nty x nt^2, contiguous,
// nt = nc + 6, nty = ny + 2 yhost) <-> device layout.  gather fills the device
// cells [lo, hi) of f.W (hi < 0: all); scatter fills the padded cells [lo, hi)
// of `stage` (hi < 0: all) from f.W, x / z ghosts (and y ghosts of a periodic
// field) as the periodic image, a slab's y ghost planes from its stored ones.
cudaError_t launch_gather(const FieldDev &f, const double *stage, int nsm, cudaStream_t st, long long lo = 0,
                          long long hi = -1);
cudaError_t launch_scatter(const FieldDev &f, double *stage, int nsm, cudaStream_t st, long long lo = 0,
                           long long hi = -1);

// max(|u| + c) over the interior planes of one field into *out_bits (uint64 image of a positive double;
// *out_bits must be zero on entry).
cudaError_t launch_maxwave(const FieldDev &f, unsigned long long *out_bits, int nsm, cudaStream_t st);

// Statistics of one field over its interior planes.  scratch: 12 * ncell doubles
// (the first 3 unused); partial: stats_partial_elems(nsm) doubles.
// Writes 24 means into sums[0..23]: the 18 PrintStats means and, for p, T and
// 1/rho, the means of x - K and (x - K)^2, and K itself into sums[24..26]
// (K = the values at the first interior cell).
cudaError_t launch_stats(const FieldDev &f, double *scratch, double *partial, double *sums, int nsm, cudaStream_t st);

// Lagrangian particles of one periodic field (gks_particles.cu).  coef:
// 5 (nc + 8)^3 doubles, the natural cubic B-spline coefficients of den, u, v,
// w, p over the padded block, the five fields interleaved per node, w: the nc + 8 pivots of the line
// solves; rec: GKS_PREC_FIELDS x n doubles, field-major.  The statistics write
// the six means TKE, SijSij, DUDX2, DUDX3, DWDZ2, DWDZ3 into sums[0..5]
// (partial: particle_partial_elems(nsm) doubles).
cudaError_t launch_particle_splines(const FieldDev &f, double *coef, const double *w, int nsm, cudaStream_t st);
cudaError_t launch_particle_props(const FieldDev &f, const double *coef, double start, double hinv, double *rec,
                                  long long n, int nsm, cudaStream_t st);
cudaError_t launch_particle_track(double *rec, long long n, double dt, double twopi, int nsm, cudaStream_t st);
cudaError_t launch_particle_stats(const double *rec, long long n, double *partial, double *sums, int nsm,
                                  cudaStream_t st);
int particle_partial_elems(int nsm);

// Scan a field's interior planes for non-finite values or non-positive density / pressure; sets bit 1 of *err.
cudaError_t launch_check(const FieldDev &f, int *err, int nsm, cudaStream_t st);

} // namespace gks
