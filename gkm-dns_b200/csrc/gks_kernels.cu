// Kernels of the WENO-GKS step and its diagnostics (sm_100a).
//
// A step is seven launches over every field of the batch: for each sweep
// direction a reconstruction launch (WENO once per cell line and interface)
// and a flux launch (transverse slopes from the neighbouring lines' WENO
// states, BGK-NS flux), then the conservative update.  All launches are
// persistent grid-stride loops over the cells of all fields, so one launch
// covers an ensemble of fields of different sizes.  The periodic halo of the
// reference (HaloTransfer on one rank, update.cpp:894-1054) is the index wrap
// in `along` and in the windowed reconstruction's cell map.
#include "gks_device.cuh"
#include "gks_flux.cuh"
#include "gks_kernels.cuh"
#include "../../include/gks_b200.h"

#include <cuda_runtime.h>
#include <algorithm>
#include <type_traits>

namespace gks {

namespace {

__device__ __forceinline__ int field_of(const FieldDev *f, int n, long long it)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (f[mid].base <= it) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

struct Cell {
    int j, i, k, nc;
    int nyw;    // y-wrap modulus (FieldDev::nyw)
    unsigned c; // (j*nc + i)*nc + k
};

// x / nc by multiply-high with the field's precomputed magic number.
__device__ __forceinline__ unsigned div_nc(unsigned x, const FieldDev &f)
{
    return (unsigned)(((unsigned long long)__umulhi(x, f.nc_magic) + x) >> f.nc_shift);
}

__device__ __forceinline__ Cell decode(unsigned c, const FieldDev &f)
{
    Cell x;
    x.nc = f.nc;
    x.nyw = f.nyw;
    x.c = c;
    const unsigned r = div_nc(c, f);
    x.k = int(c - r * f.nc);
    const unsigned jj = div_nc(r, f);
    x.i = int(r - jj * f.nc);
    x.j = int(jj);
    return x;
}

__device__ __forceinline__ int wrap(int x, int n) { return x < 0 ? x + n : (x >= n ? x - n : x); }

// Displacement along the sweep axis: DIR 0 = x (i), 1 = y (j), 2 = z (k);
// only the swept coordinate wraps (y not at all in a slab, whose ghost planes
// are stored).
template <int DIR>
__device__ __forceinline__ unsigned along(const Cell &x, int d)
{
    const int n = x.nc;
    if (DIR == 0) return x.c + (unsigned)((wrap(x.i + d, n) - x.i) * n);
    if (DIR == 1) return x.c + (unsigned)((wrap(x.j + d, x.nyw) - x.j) * n * n);
    return x.c + (unsigned)(wrap(x.k + d, n) - x.k);
}

__device__ __forceinline__ double viscosity(const FieldDev &f, double T)
{
    const double x = T * f.iT0;
    if (f.visc_law == GKS_VISC_POWER) return f.mu0 * pow(x, f.visc_exp);
    // mu0 (T/T0)^1.5 (T0 + 110.4)/(T + 110.4), update.cpp:263
    return f.mu0 * (x * sqrt(x)) * (f.T0 + 110.4) * __drcp_rn(T + 110.4);
}

// Collision time mu / p of the state W (update.cpp:262-264) as a fraction
// num / den, which the flux divides out together with its other terms.
// Sutherland, with A = rho2p(W), T = cT A / rho^2 and p = (gamma - 1) A / rho:
//   mu / p = mu0 y^1.5 (T0 + 110.4) / ((gamma - 1) A (cT A + 110.4 rho^2)),  y = cT A / T0,
// in which the powers of rho cancel (no reciprocal at all).
__device__ __forceinline__ void visc_over_p(const FieldDev &f, const double W[5], double &num, double &den)
{
    const double A = rho2p(W);
    if (f.visc_law == GKS_VISC_POWER) {
        const double ri = __drcp_rn(W[0]);
        den = f.gm1 * (A * ri);
        num = viscosity(f, den * ri * f.iR);
        return;
    }
    const double y = (f.cT * A) * f.iT0;
    den = (f.gm1 * A) * fma(110.4 * W[0], W[0], f.cT * A);
    num = (f.mu0 * (y * sqrt(y))) * (f.T0 + 110.4);
}

// mu/p of cell c, stored once per step by the x-sweep reconstruction for the
// flux kernels of all three sweeps (the left cell of interface c is c in each).
__device__ __forceinline__ void store_tau(const FieldDev &f, unsigned c, const double W[5])
{
    double n, d;
    visc_over_p(f, W, n, d);
    f.tau[0][c] = n;
    f.tau[1][c] = d;
}

__device__ __forceinline__ double temperature(const double W[5], double cT)
{
    // (gam-1)(E/rho - |m|^2/(2 rho^2))/R, update.cpp:560
    const double ri = __drcp_rn(W[0]);
    const double ke = fma(W[1], W[1], fma(W[2], W[2], W[3] * W[3]));
    return cT * fma(-0.5 * ke, ri * ri, W[4] * ri);
}

// rho E from the reconstructed density, momentum and temperature
// (update.cpp:618-619): rho T R/(gam-1) + |m|^2 / (2 rho), ri = 1/rho.
__device__ __forceinline__ double energy(const double w[5], double T, double ri, double icT)
{
    const double ke = fma(w[1], w[1], fma(w[2], w[2], w[3] * w[3]));
    return fma(w[0] * T, icT, (0.5 * ke) * ri);
}

// The reconstruction record of cell c: Wl[0..4] then Wr[0..4] as five
// 16-byte pairs, pair k of every cell in its own array of n = nc^3 pairs
// (rec + 2 k n doubles, 16-byte aligned): a warp's load or store of one pair
// for 32 consecutive cells is 512 contiguous bytes, and a record takes five
// 16-byte accesses instead of ten 8-byte ones.
__device__ __forceinline__ void put_record(double *rec, unsigned c, const double wl[5], const double wr[5], long long n)
{
    double2 *p = reinterpret_cast<double2 *>(rec) + c;
    p[0] = make_double2(wl[0], wl[1]);
    p[n] = make_double2(wl[2], wl[3]);
    p[2 * n] = make_double2(wl[4], wr[0]);
    p[3 * n] = make_double2(wr[1], wr[2]);
    p[4 * n] = make_double2(wr[3], wr[4]);
}

__device__ __forceinline__ void get_record(const double *rec, unsigned c, double v[10], long long n)
{
    const double2 *p = reinterpret_cast<const double2 *>(rec) + c;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const double2 t = __ldg(p + k * n);
        v[2 * k] = t.x;
        v[2 * k + 1] = t.y;
    }
}

// ---------------------------------------------------------------------------
// WENO of one interface from its 6-cell stencil s[0..5] (LLL .. RRR) and the
// stencil's temperatures T[0..5] (used unless GKS_DIRECT_ENERGY)
// (update.cpp:247, 502-625 / GPUupdate.cu:917-977).
// ---------------------------------------------------------------------------
template <int PREC, typename SG>
__device__ __forceinline__ void recon_point(const SG &s, const double (&T)[6], bool direct, double icT, double wl[5],
                                            double wr[5])
{
    if (PREC == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
            weno_pair<double>(s(0, q), s(1, q), s(2, q), s(3, q), s(4, q), s(5, q), kWenoEps, wl[q], wr[q]);
        if (direct) {
            weno_pair<double>(s(0, 4), s(1, 4), s(2, 4), s(3, 4), s(4, 4), s(5, 4), kWenoEps, wl[4], wr[4]);
        } else {
            double tl, tr;
            weno_pair<double>(T[0], T[1], T[2], T[3], T[4], T[5], kWenoEps, tl, tr);
            // E from the reconstructed temperature (update.cpp:618-619)
            const double r = __drcp_rn(wl[0] * wr[0]); // one reciprocal for both densities
            wl[4] = energy(wl, tl, wr[0] * r, icT);
            wr[4] = energy(wr, tr, wl[0] * r, icT);
        }
    } else {
        // mixed: WENO in FP32 on differences from the left cell, added back
        // in FP64; components (0, 1) and (2, 3) as the two lanes of paired
        // FP32 instructions, the fifth (energy or temperature) alone
        const float epsf = float(kWenoEps);
#pragma unroll
        for (int q = 0; q < 4; q += 2) {
            const double c0 = s(2, q), c1 = s(2, q + 1);
            f2 v[6];
#pragma unroll
            for (int a = 0; a < 6; ++a) v[a] = f2(float(s(a, q) - c0), float(s(a, q + 1) - c1));
            f2 dl, dr;
            weno_pair<f2>(v[0], v[1], f2(0.0f), v[3], v[4], v[5], f2(epsf), dl, dr);
            wl[q] = c0 + double(dl.v.x);
            wr[q] = c0 + double(dr.v.x);
            wl[q + 1] = c1 + double(dl.v.y);
            wr[q + 1] = c1 + double(dr.v.y);
        }
        if (direct) {
            const double c0 = s(2, 4);
            float dl, dr;
            weno_pair<float>(float(s(0, 4) - c0), float(s(1, 4) - c0), 0.0f, float(s(3, 4) - c0),
                             float(s(4, 4) - c0), float(s(5, 4) - c0), epsf, dl, dr);
            wl[4] = c0 + double(dl);
            wr[4] = c0 + double(dr);
        } else {
            float dl, dr;
            weno_pair<float>(float(T[0] - T[2]), float(T[1] - T[2]), 0.0f, float(T[3] - T[2]),
                             float(T[4] - T[2]), float(T[5] - T[2]), epsf, dl, dr);
            const double tl = T[2] + double(dl), tr = T[2] + double(dr);
            const double r = __drcp_rn(wl[0] * wr[0]); // one reciprocal for both densities
            wl[4] = energy(wl, tl, wr[0] * r, icT);
            wr[4] = energy(wr, tr, wl[0] * r, icT);
        }
    }
}

// The stencil as a 6 x 5 array in registers.
struct StencilRegs {
    const double (&v)[6][5];
    __device__ double operator()(int a, int q) const { return v[a][q]; }
};

template <int PREC>
__device__ __forceinline__ void recon_point(const double (&s)[6][5], const double (&T)[6], bool direct, double icT,
                                            double wl[5], double wr[5])
{
    recon_point<PREC>(StencilRegs{s}, T, direct, icT, wl, wr);
}

// ---------------------------------------------------------------------------
// Reconstruction: Wl, Wr at the interface between cell c and its +1
// neighbour along DIR, one interface per work item, the stencil read
// straight from the state (used for the z sweep, where the lanes of a warp
// are consecutive along the sweep and L1 serves the overlapping stencils).
// ---------------------------------------------------------------------------
template <int DIR, int PREC, int MINB>
__global__ void __launch_bounds__(kReconBlock, MINB) k_recon(Batch b)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long it = b.lo + (long long)blockIdx.x * blockDim.x + threadIdx.x; it < b.hi; it += stride) {
        const FieldDev &f = b.fields[field_of(b.fields, b.nfields, it)];
        if (it - f.base >= f.ncell) continue; // alignment padding after the field
        const Cell x = decode(unsigned(it - f.base), f);
        unsigned idx[6];
#pragma unroll
        for (int a = 0; a < 6; ++a) idx[a] = along<DIR>(x, a - 2);
        double s[6][5];
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
            for (int q = 0; q < 5; ++q) s[a][q] = __ldg(f.W[q] + idx[a]);
        if (DIR == 0) store_tau(f, x.c, s[2]);
        const bool direct = (f.flags & GKS_DIRECT_ENERGY) != 0;
        double T[6];
        if (!direct) {
#pragma unroll
            for (int a = 0; a < 6; ++a) T[a] = temperature(s[a], f.cT);
        }
        double wl[5], wr[5];
        recon_point<PREC>(s, T, direct, f.icT, wl, wr);
        put_record(f.rec[DIR], x.c, wl, wr, f.ncell);
    }
}

// Field of z-segment item `it` (the last field whose segment range starts at or before it).
__device__ __forceinline__ int field_of_zseg(const FieldDev *f, int n, long long it)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (f[mid].zbase <= it) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// Reconstruction for the z sweep with a warp-staged segment: a work item is
// one warp's 32 consecutive interfaces along z of one (j, i) line.  The lanes
// load the 37 cells the segment's stencils span (one coalesced load per lane
// and component, five lanes load the upper halo), compute each cell's
// temperature once and stage cells and temperatures in the warp's own
// shared-memory tile; each lane then reads its six-cell stencil from there.
// ---------------------------------------------------------------------------
// Asynchronous 8-byte copy global -> shared (cp.async), its groups and waits.
__device__ __forceinline__ void cp_async8(double *smem, const double *gmem)
{
    const unsigned a = unsigned(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

constexpr int kZSegWarps = kReconBlock / 32, kZSegCells = 32 + 5;

template <int PREC, int MINB>
__global__ void __launch_bounds__(kReconBlock, MINB) k_recon_zseg(Batch b)
{
    __shared__ double tiles[kZSegWarps][6][kZSegCells];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double (*tile)[kZSegCells] = tiles[wid];
    const long long stride = (long long)gridDim.x * kZSegWarps;
    for (long long it = b.lo + (long long)blockIdx.x * kZSegWarps + wid; it < b.hi; it += stride) {
        const FieldDev &f = b.fields[field_of_zseg(b.fields, b.nfields, it)];
        const long long loc = it - f.zbase; // < nzseg: segment ranges are contiguous
        const int nc = f.nc, nseg = (nc + 31) >> 5;
        const long long line = loc / nseg;
        const int k0 = int(loc - line * nseg) << 5;
        const unsigned lbase = unsigned(line) * unsigned(nc); // cell (j, i, 0)
        const bool direct = (f.flags & GKS_DIRECT_ENERGY) != 0;
        // stage cells k0-2 .. k0+34 (those the active lanes' stencils reach:
        // k0-2 .. min(k0+34, nc+2), so each index wraps at most once) and their
        // temperatures; lane l takes cells l and l + 32, all ten loads issued at once
        const int nh = min(kZSegCells, nc - k0 + 5);
        const int h1 = lane + 32;
        const bool one = lane < nh, two = h1 < nh;
        double w[5], v[5];
        {
            const unsigned c0 = lbase + unsigned(wrap(k0 - 2 + (one ? lane : 0), nc));
            const unsigned c1 = lbase + unsigned(wrap(k0 - 2 + (two ? h1 : 0), nc));
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                w[q] = one ? __ldg(f.W[q] + c0) : 0.0;
                v[q] = two ? __ldg(f.W[q] + c1) : 0.0;
            }
        }
        if (one) {
#pragma unroll
            for (int q = 0; q < 5; ++q) tile[q][lane] = w[q];
            tile[5][lane] = direct ? 0.0 : temperature(w, f.cT);
        }
        if (two) {
#pragma unroll
            for (int q = 0; q < 5; ++q) tile[q][h1] = v[q];
            tile[5][h1] = direct ? 0.0 : temperature(v, f.cT);
        }
        __syncwarp();
        const int k = k0 + lane;
        if (k < nc) {
            double s[6][5], T[6];
#pragma unroll
            for (int a = 0; a < 6; ++a) {
#pragma unroll
                for (int q = 0; q < 5; ++q) s[a][q] = tile[q][lane + a];
                T[a] = tile[5][lane + a];
            }
            double wl[5], wr[5];
            recon_point<PREC>(s, T, direct, f.icT, wl, wr);
            put_record(f.rec[2], lbase + unsigned(k), wl, wr, f.ncell);
        }
        __syncwarp();
    }
}

// Field of window item `it` (the last field whose window range starts at or before it).
__device__ __forceinline__ int field_of_win(const FieldDev *f, int n, long long it)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (f[mid].wbase <= it) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// Reconstruction for the x (DIR 0) and y (DIR 1) sweeps with a sliding
// window: a work item is a run of f.run consecutive interfaces along the
// sweep at one (transverse line, k); the lanes of a warp take consecutive
// k, so every load is coalesced.  The window moves by one cell per
// interface: one new cell (five loads) and one temperature per interface
// instead of thirty loads and six temperatures.  The cells live in a ring of
// kWinRing slots in the thread's own part of shared memory
// ([slot][component][thread], no bank conflicts) -- the six stencil cells and
// the kWinPrefetch cells beyond them, which arrive by asynchronous copies so
// that their latency overlaps the WENO of the interfaces before them -- and
// only the six temperatures stay in registers (about 40 fewer registers than
// with the window in registers).  Item order: k
// fastest, then run, then the transverse line.  The loop is kept rolled
// (FP64) or unrolled twice (mixed).
// ---------------------------------------------------------------------------
constexpr int kWinPrefetch = 2; // 2, 4 and 8 measured within 1 %
constexpr int kWinRing = 8;     // ring slots per thread: 6 stencil cells + the cells in flight


template <int DIR, int PREC, int MINB>
__global__ void __launch_bounds__(kReconBlock, MINB) k_recon_win(Batch b)
{
    constexpr int PF = kWinPrefetch, NR = kWinRing;
    static_assert(NR >= 5 + PF && (NR & (NR - 1)) == 0, "the ring holds the window and the cells in flight");
    __shared__ double ring[NR][5][kReconBlock];
    const int tid = threadIdx.x;
    static_assert(DIR == 0 || DIR == 1, "windowed reconstruction is for the x and y sweeps");
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long it = b.lo + (long long)blockIdx.x * blockDim.x + threadIdx.x; it < b.hi; it += stride) {
        const FieldDev &f = b.fields[field_of_win(b.fields, b.nfields, it)];
        const long long loc = it - f.wbase;
        if (loc >= f.nwin) continue; // alignment padding after the field
        const int nc = f.nc;
        const unsigned u = unsigned(loc);
        const unsigned rest = div_nc(u, f);
        const int k = int(u - rest * unsigned(nc));
        const int line = int(rest / unsigned(f.nrun));
        const int RUN = f.run;
        const int s0 = int(rest - unsigned(line) * unsigned(f.nrun)) * RUN;
        // cell (line, sweep position p, k): x sweep (j, i, k), y sweep (j = p, i = line)
        const unsigned step = DIR == 0 ? unsigned(nc) : unsigned(nc) * unsigned(nc);
        const unsigned lbase = DIR == 0 ? unsigned(line) * unsigned(nc) * unsigned(nc) + unsigned(k)
                                        : unsigned(line) * unsigned(nc) + unsigned(k);
        auto cell = [&](int p) -> unsigned { return lbase + unsigned(wrap(p, DIR == 0 ? nc : f.nyw)) * step; };
        const bool direct = (f.flags & GKS_DIRECT_ENERGY) != 0;
        // cells of the run's stencils: s0 - 2 .. last (unwrapped, at most nc + 2),
        // cell pc in ring slot pc mod NR, one copy group per cell (empty past the run)
        const int last = min(s0 + RUN, nc) + 2;
        auto fetch = [&](int pc) {
            if (pc <= last) {
                const unsigned c = cell(pc);
#pragma unroll
                for (int q = 0; q < 5; ++q) cp_async8(&ring[pc & (NR - 1)][q][tid], f.W[q] + c);
            }
            cp_async_commit();
        };
        auto temp_of = [&](int pc) -> double {
            double w[5];
#pragma unroll
            for (int q = 0; q < 5; ++q) w[q] = ring[pc & (NR - 1)][q][tid];
            return temperature(w, f.cT);
        };
#pragma unroll
        for (int d = 0; d < 5 + PF; ++d) fetch(s0 - 2 + d);
        cp_async_wait<PF>(); // the five first window cells have landed
        double T[6];
#pragma unroll
        for (int a = 0; a < 5; ++a) T[a + 1] = direct ? 0.0 : temp_of(s0 - 2 + a);
        constexpr int UNROLL = PREC == 0 ? 1 : 2;
#pragma unroll UNROLL
        for (int r = 0; r < RUN; ++r) {
            const int p = s0 + r;
            if (p >= nc) break;
#pragma unroll
            for (int a = 0; a < 5; ++a) T[a] = T[a + 1];
            cp_async_wait<PF - 1>(); // cell p + 3 (issued PF groups ago) has landed
            T[5] = direct ? 0.0 : temp_of(p + 3);
            const auto sg = [&](int a, int q) -> double { return ring[(p - 2 + a) & (NR - 1)][q][tid]; };
            double wl[5], wr[5];
            recon_point<PREC>(sg, T, direct, f.icT, wl, wr);
            const unsigned c = cell(p);
            if (DIR == 0) {
                double w[5];
#pragma unroll
                for (int q = 0; q < 5; ++q) w[q] = sg(2, q);
                store_tau(f, c, w);
            }
            put_record(f.rec[DIR], c, wl, wr, f.ncell);
            // cell p + 3 + PF takes the slot of cell p + 3 + PF - NR, which no
            // stencil from here on reads (it lies below p - 2 for NR >= 5 + PF)
            fetch(p + 3 + PF);
        }
        cp_async_wait<0>(); // nothing in flight into the ring before the next item
    }
}

// ---------------------------------------------------------------------------
// Flux at the interface between cell c and its +1 neighbour along DIR
// (derivsX/Y/Z, update.cpp:201-453, and flux, GKMflux.cpp:11-215).
// Transverse lines: x sweep N,S = y+-1, F,B = z+-1; y sweep N,S = x-+1 with
// DWy = -(N-S)/2dx, F,B = z+-1; z sweep N,S = x+-1, F,B = y+-1 (the
// reference's assignment) or, with GKS_FIX_ZSWEEP, N,S = y+-1, F,B = x+-1.
// Momentum is rotated into slot 1 for y (rho v) and z (rho w).
// ---------------------------------------------------------------------------
template <int DIR>
__device__ __forceinline__ void transverse(const Cell &x, int flags, unsigned &n, unsigned &s, unsigned &fr,
                                           unsigned &bk)
{
    if (DIR == 0) {
        n = along<1>(x, 1); s = along<1>(x, -1);
        fr = along<2>(x, 1); bk = along<2>(x, -1);
    } else if (DIR == 1) {
        n = along<0>(x, -1); s = along<0>(x, 1);
        fr = along<2>(x, 1); bk = along<2>(x, -1);
    } else {
        if (flags & GKS_FIX_ZSWEEP) {
            n = along<1>(x, 1); s = along<1>(x, -1);
            fr = along<0>(x, 1); bk = along<0>(x, -1);
        } else {
            n = along<0>(x, 1); s = along<0>(x, -1);
            fr = along<1>(x, 1); bk = along<1>(x, -1);
        }
    }
}

// Inputs and running sums of one interface (see gks_flux).  All global loads
// are issued at once when the interface starts, so that their latency
// overlaps; what is not needed until later -- the right state and its slopes,
// the two cell averages -- is parked in this thread's own shared-memory slots
// ([slot][thread], no bank conflicts) instead of registers, and so are the
// sums the two side passes of the flux accumulate for the equilibrium pass.
// Slot q of the rotated frame holds original component perm(q): rho v (y
// sweep) or rho w (z sweep) moves into slot 1 (update.cpp:340-350, 429-439).
template <int DIR, typename S>
struct SweepSrc {
    double Wl[5];
    S DWl[3][5];
    S (*park_dw)[kFluxBlock];      // [15][block]: right-side slopes
    double (*park_w)[kFluxBlock];  // [15][block]: WL, WR, Wr
    double (*sum_d)[kFluxBlock];   // [10][block]: double sums of the side passes
    S (*sum_s)[kFluxBlock];        // [20][block]: S sums of the side passes (FP64 path)

    __device__ static constexpr int perm(int q)
    {
        return DIR == 0 ? q : (q == 1 ? (DIR == 1 ? 2 : 3) : (q == (DIR == 1 ? 2 : 3) ? 1 : q));
    }

    // DWxl = 2(Wl - WL)/dx, DWxr = 2(WR - Wr)/dx; transverse central differences of
    // the neighbouring lines' states (update.cpp:253-260, 327-334, 416-423), here
    // the differences, which the flux scales by FluxConst::ks
    __device__ __forceinline__ void load(const FieldDev &f, unsigned c, unsigned c1, unsigned cn, unsigned cs,
                                         unsigned cf, unsigned cb)
    {
        // differences in double (they cancel); the flux scales them (FluxConst::ks)
        const int t = threadIdx.x;
        const double *rec = f.rec[DIR];
        double r0[10], rn[10], rs[10], rf[10], rb[10];
        get_record(rec, c, r0, f.ncell);
        get_record(rec, cn, rn, f.ncell);
        get_record(rec, cs, rs, f.ncell);
        get_record(rec, cf, rf, f.ncell);
        get_record(rec, cb, rb, f.ncell);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const int o = perm(q);
            const double wL = __ldg(f.W[o] + c), wR = __ldg(f.W[o] + c1);
            const double wr = r0[5 + o];
            Wl[q] = r0[o];
            DWl[0][q] = S(Wl[q] - wL);
            DWl[1][q] = S(rn[o] - rs[o]);
            DWl[2][q] = S(rf[o] - rb[o]);
            park_dw[q][t] = S(wR - wr);
            park_dw[5 + q][t] = S(rn[5 + o] - rs[5 + o]);
            park_dw[10 + q][t] = S(rf[5 + o] - rb[5 + o]);
            park_w[q][t] = wL;
            park_w[5 + q][t] = wR;
            park_w[10 + q][t] = wr;
        }
    }

    __device__ __forceinline__ void state(int side, double W[5]) const
    {
#pragma unroll
        for (int q = 0; q < 5; ++q) W[q] = side == 0 ? Wl[q] : park_w[10 + q][threadIdx.x];
    }

    // slopes of one side along one direction (0 normal, 1 and 2 transverse)
    __device__ __forceinline__ void slope(int side, int d, S DW[5]) const
    {
#pragma unroll
        for (int q = 0; q < 5; ++q) DW[q] = side == 0 ? DWl[d][q] : park_dw[5 * d + q][threadIdx.x];
    }

    __device__ __forceinline__ void cells(double WL[5], double WR[5]) const
    {
        const int t = threadIdx.x;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            WL[q] = park_w[q][t];
            WR[q] = park_w[5 + q][t];
        }
    }

    // running sums of a * b: the first side pass stores, the second adds (one
    // explicit rounding each, so that no compiler contraction choice -- which
    // may differ between register-cap variants -- changes the result)
    template <bool FIRST> __device__ __forceinline__ void put_d(int i, double a, double b) const
    {
        double &x = sum_d[i][threadIdx.x];
        x = FIRST ? __dmul_rn(a, b) : __fma_rn(a, b, x);
    }
    template <bool FIRST> __device__ __forceinline__ void put_s(int i, S a, S b) const
    {
        S &x = sum_s[i][threadIdx.x];
        if constexpr (sizeof(S) == 8) x = FIRST ? __dmul_rn(a, b) : __fma_rn(a, b, x);
        else x = FIRST ? __fmul_rn(a, b) : __fmaf_rn(a, b, x);
    }
    __device__ __forceinline__ double get_d(int i) const { return sum_d[i][threadIdx.x]; }
    __device__ __forceinline__ S get_s(int i) const { return sum_s[i][threadIdx.x]; }
};

// The flux of work item `it` of field f.
template <int DIR, typename S>
__device__ __forceinline__ void flux_item(const FieldDev &f, long long it, S (*park_dw)[kFluxBlock],
                                          double (*park_w)[kFluxBlock], double (*sum_d)[kFluxBlock],
                                          S (*sum_s)[kFluxBlock])
{
    const Cell x = decode(unsigned(it - f.base), f);
    unsigned cn, cs, cf, cb;
    transverse<DIR>(x, f.flags, cn, cs, cf, cb);
    SweepSrc<DIR, S> src;
    src.park_dw = park_dw;
    src.park_w = park_w;
    src.sum_d = sum_d;
    src.sum_s = sum_s;
    src.load(f, x.c, along<DIR>(x, 1), cn, cs, cf, cb);
    // collision time mu / p at the left cell (update.cpp:262-264), stored by
    // this step's x-sweep reconstruction
    const double tau_n = __ldg(f.tau[0] + x.c), tau_d = __ldg(f.tau[1] + x.c);
    FluxConst fc;
    fc.gm1 = f.gm1;
    fc.hig = f.hig;
    fc.dt = f.dt;
    fc.dx = f.dx;
    fc.ks[0] = f.ksn;
    fc.ks[1] = DIR == 1 ? -f.kst : f.kst; // y sweep: DWy = -(N - S)/(2 dx)
    fc.ks[2] = f.kst;
    fc.kA = f.kA;
    fc.hK2 = f.hK2;
    fc.kd = {f.kd[0], f.kd[1], f.kd[2], f.kd[3]};
    fc.kf = {f.kf[0], f.kf[1], f.kf[2], f.kf[3]};
    double F[5];
    gks_flux<S>(src, tau_n, tau_d, fc, F);
    constexpr int ROT = DIR == 0 ? 0 : (DIR == 1 ? 2 : 3);
    if (ROT) {
        const double t = F[1];
        F[1] = F[ROT];
        F[ROT] = t;
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) f.F[DIR * 5 + q][x.c] = F[q];
}

// A batch of one field reads the field's descriptor from the launch
// parameters (b.one: constant-bank operands, nothing loaded per interface);
// an ensemble looks each interface's field up in the device array.
template <int DIR, int PREC, int REGS>
__global__ void __launch_bounds__(kFluxBlock) __maxnreg__(REGS) k_flux(Batch b)
{
    using S = typename std::conditional<PREC == 0, double, float>::type;
    __shared__ S park_dw[15][kFluxBlock];
    __shared__ double park_w[15][kFluxBlock];
    __shared__ double sum_d[10][kFluxBlock];
    __shared__ S sum_s[20][kFluxBlock];
    const long long stride = (long long)gridDim.x * blockDim.x;
    if (b.nfields == 1) {
        const long long end = b.hi < b.one.ncell ? b.hi : b.one.ncell; // alignment padding after the field
        for (long long it = b.lo + (long long)blockIdx.x * blockDim.x + threadIdx.x; it < end; it += stride)
            flux_item<DIR, S>(b.one, it, park_dw, park_w, sum_d, sum_s);
        return;
    }
    for (long long it = b.lo + (long long)blockIdx.x * blockDim.x + threadIdx.x; it < b.hi; it += stride) {
        const FieldDev &f = b.fields[field_of(b.fields, b.nfields, it)];
        if (it - f.base >= f.ncell) continue; // alignment padding after the field
        flux_item<DIR, S>(f, it, park_dw, park_w, sum_d, sum_s);
    }
}

// ---------------------------------------------------------------------------
// Conservative update of the interior (update.cpp:455-469), evaluated in the
// reference's order: W - (1/dx)*(Fx - Fx[i-1] + Fy - Fy[j-1] + Fz - Fz[k-1]),
// written to Wout (W itself, except in the slab-pipelined host step).  Also
// flags non-finite or non-positive density / pressure.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kUpdateBlock) k_update(Batch b)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long it = b.lo + (long long)blockIdx.x * blockDim.x + threadIdx.x; it < b.hi; it += stride) {
        const FieldDev &f = b.fields[field_of(b.fields, b.nfields, it)];
        if (it - f.base >= f.ncell) continue; // alignment padding after the field
        const Cell x = decode(unsigned(it - f.base), f);
        const unsigned c = x.c;
        const unsigned cx = along<0>(x, -1), cy = along<1>(x, -1), cz = along<2>(x, -1);
        double w[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            double d = __dsub_rn(f.F[q][c], f.F[q][cx]);
            d = __dadd_rn(d, f.F[5 + q][c]);
            d = __dsub_rn(d, f.F[5 + q][cy]);
            d = __dadd_rn(d, f.F[10 + q][c]);
            d = __dsub_rn(d, f.F[10 + q][cz]);
            w[q] = __dsub_rn(f.W[q][c], __dmul_rn(f.inv_dx, d));
            f.Wout[q][c] = w[q];
        }
        const double p = f.gm1 * (w[4] - 0.5 * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]) / w[0]);
        if (!(w[0] > 0.0) || !(p > 0.0) || !isfinite(w[0] + w[1] + w[2] + w[3] + w[4]))
            atomicOr(b.err, 1);
    }
}

// ---------------------------------------------------------------------------
// Layout conversion: padded staging (5 x nt^3) <-> interior.
// ---------------------------------------------------------------------------
__global__ void k_gather(FieldDev f, const double *__restrict__ stage, long long lo, long long hi)
{
    const int nc = f.nc, nt = nc + 6;
    const long long Nt = (long long)(f.ny + 2 * f.yhost) * nt * nt;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long c = lo + (long long)blockIdx.x * blockDim.x + threadIdx.x; c < hi; c += stride) {
        const Cell x = decode(unsigned(c), f);
        const long long p = ((long long)(x.j + f.yhost) * nt + (x.i + 3)) * nt + (x.k + 3);
#pragma unroll
        for (int q = 0; q < 5; ++q) f.W[q][c] = stage[q * Nt + p];
    }
}

__global__ void k_scatter(FieldDev f, double *__restrict__ stage, long long lo, long long hi)
{
    const int nc = f.nc, nt = nc + 6;
    const long long Nt = (long long)(f.ny + 2 * f.yhost) * nt * nt;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long p = lo + (long long)blockIdx.x * blockDim.x + threadIdx.x; p < hi; p += stride) {
        const int kk = int(p % nt);
        const int ii = int((p / nt) % nt);
        const int jj = int(p / ((long long)nt * nt));
        const long long c = ((long long)wrap(jj - f.yhost, f.nyw) * nc + wrap(ii - 3, nc)) * nc + wrap(kk - 3, nc);
#pragma unroll
        for (int q = 0; q < 5; ++q) stage[q * Nt + p] = f.W[q][c];
    }
}

// ---------------------------------------------------------------------------
// Largest |u| + c (timestep, update.cpp:1057-1079), each operation rounded as
// the reference writes it so that dt matches bit for bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__global__ void k_maxwave(FieldDev f, unsigned long long *out)
{
    double m = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long plane = (long long)f.nc * f.nc, c1 = f.yhi * plane;
    for (long long c = f.ylo * plane + (long long)blockIdx.x * blockDim.x + threadIdx.x; c < c1; c += stride) {
        const double den = f.W[0][c];
        const double u = __ddiv_rn(f.W[1][c], den), v = __ddiv_rn(f.W[2][c], den), w = __ddiv_rn(f.W[3][c], den);
        const double vsq = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w));
        const double P = __dmul_rn(__dmul_rn(den, f.gm1), __dsub_rn(__ddiv_rn(f.W[4][c], den), __dmul_rn(0.5, vsq)));
        const double val = __dadd_rn(__dsqrt_rn(vsq), __dsqrt_rn(__ddiv_rn(__dmul_rn(f.gam, P), den)));
        m = val > m ? val : m;
    }
    m = warp_max(m);
    __shared__ double sm[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sm[wid] = m;
    __syncthreads();
    if (wid == 0) {
        m = lane < (blockDim.x >> 5) ? sm[lane] : 0.0;
        m = warp_max(m);
        if (lane == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
}

// ---------------------------------------------------------------------------
// Statistics (PrintStats, update.cpp:638-784).  Velocity gradients are the
// node slopes of the natural cubic spline through each padded grid line
// (nt = nc + 6 points, periodic ghosts), the interpolant the reference builds
// with einspline (Interpolation.cpp:3-31); at nodes a tensor-product natural
// spline reduces to these 1-D slopes.  Scratch layout: [3 + 3*comp + axis]
// d(comp)/d(axis), axis 0 = y, 1 = x, 2 = z (slots 0-2 unused).
// ---------------------------------------------------------------------------

// Slopes of the natural cubic spline through the nt = nc + 6 nodes of a
// padded periodic grid line (the reference's einspline over its padded
// block):
//   2 m0 + m1 = s (f1 - f0);  m_{p-1} + 4 m_p + m_{p+1} = s (f_{p+1} - f_{p-1});
//   m_{n-2} + 2 m_{n-1} = s (f_{n-1} - f_{n-2}),  s = 3/h,
// solved by the Thomas recurrences with precomputed pivots,
//   forward  d_p = (r_p - d_{p-1}) inv_p,   backward  m_p = d_p - cp_p m_{p+1},
// each step an affine map of the previous value.  One warp solves one line:
// lane L owns the B consecutive nodes [L B, L B + B) (B odd, 32 B >= nt),
// composes the affine maps of its nodes, an inclusive warp scan of the
// composed maps (five shuffle steps) hands every lane the value entering its
// nodes, and the lane runs its nodes again from there -- forward, then the
// same backward.  The associativity of the scan changes only the rounding.
//
// A block takes LW lines: it copies rho, rho u, rho v, rho w of all their
// nodes into shared memory with asynchronous copies (all in flight at once,
// no registers), turns the momenta into velocities in place, each warp solves
// its line for the components (NCI of them interleaved, for latency), and the
// slopes leave through the same tiles:
//   y, x lines: LW consecutive k of one (i) / (j): tiles [node][line], every
//               group of LW threads one contiguous run of LW doubles;
//   z lines:    LW consecutive (j, i) lines:      tiles [line][node], each
//               line one contiguous run of nc doubles.
// Odd B keeps the solve's shared-memory accesses free of bank conflicts.
template <int AXIS, int B, int LW> struct SplineTiles {
    static constexpr int NCI = B <= 9 ? 3 : 1; // components solved together
    __host__ __device__ static int tile(int nt) { return AXIS == 2 ? LW * nt : nt * (LW + 1); }
    __host__ __device__ static size_t bytes(int nt) { return (4 * (size_t)tile(nt) + 2 * (size_t)nt) * sizeof(double); }
};

template <int AXIS, int B, int LW>
__global__ void __launch_bounds__(32 * LW, B <= 9 ? 2 : 1) k_spline_scan(FieldDev f, double *scr)
{
    using ST = SplineTiles<AXIS, B, LW>;
    constexpr int NCI = ST::NCI;
    extern __shared__ double smem[];
    // nodes of a line: nc + 6 along x / z; along y ny + 2 yhost (the same for a
    // periodic field; a slab's ny stored planes, its ghosts included)
    const int nc = f.nc, nt = AXIS == 0 ? f.ny + 2 * f.yhost : nc + 6;
    const long long n = f.ncell;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int tsz = ST::tile(nt);
    double *cpv = smem + 4 * tsz, *invv = cpv + nt;
    // tile a (0 rho, 1-3 the velocity components), node, line
    auto T = [&](int a, int node, int line) -> double & {
        return AXIS == 2 ? smem[a * tsz + line * nt + node] : smem[a * tsz + node * (LW + 1) + line];
    };
    for (int p = threadIdx.x; p < nt; p += blockDim.x) {
        cpv[p] = AXIS == 0 ? f.spl_cpy[p] : f.spl_cp[p];
        invv[p] = AXIS == 0 ? f.spl_invy[p] : f.spl_inv[p];
    }
    // the block's lines: y / x lines are (outer, k) with k in [k0, k0 + LW),
    // outer = i (y lines) or j (x lines, interior planes); z lines are l in
    // [l0, l0 + LW), l = j nc + i (interior planes)
    const int nkb = (nc + LW - 1) / LW;
    const long long set = blockIdx.x;
    const int outer = AXIS == 2 ? 0 : (AXIS == 1 ? f.ylo : 0) + int(set / nkb);
    const int k0 = AXIS == 2 ? 0 : int(set - (long long)(outer - (AXIS == 1 ? f.ylo : 0)) * nkb) * LW;
    const long long l0 = AXIS == 2 ? (long long)f.ylo * nc + set * LW : 0;
    // cell of line `line` at position q (0 .. nc-1) along the axis
    auto cell = [&](int line, int q) -> long long {
        if (AXIS == 0) return ((long long)q * nc + outer) * nc + k0 + line;
        if (AXIS == 1) return ((long long)outer * nc + q) * nc + k0 + line;
        return (l0 + line) * nc + q;
    };
    auto active = [&](int line) -> bool {
        return AXIS == 2 ? l0 + line < (long long)f.yhi * nc : k0 + line < nc;
    };
    // visit every (node, line) of the set: y / x, LW consecutive threads on
    // the LW lines of one node; z, warp w along the nodes of line w
    auto each = [&](auto fn) {
        if (AXIS == 2) {
            if (active(w))
                for (int p = lane; p < nt; p += 32) fn(p, w);
        } else {
            for (int e = threadIdx.x; e < nt * LW; e += 32 * LW) {
                const int line = e % LW;
                if (active(line)) fn(e / LW, line);
            }
        }
    };
    // stage rho and the momenta (node p holds cell wrap(p - 3); along y plane
    // wrap(p - yhost, nyw), a slab's plane p), then velocities
    each([&](int p, int line) {
        const long long c = cell(line, AXIS == 0 ? wrap(p - f.yhost, f.nyw) : wrap(p - 3, nc));
#pragma unroll
        for (int a = 0; a < 4; ++a) cp_async8(&T(a, p, line), f.W[a] + c);
    });
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    each([&](int p, int line) {
        const double ri = __drcp_rn(T(0, p, line));
#pragma unroll
        for (int a = 1; a < 4; ++a) T(a, p, line) *= ri;
    });
    __syncthreads();
    if (active(w)) {
        const double s = AXIS == 0 ? f.spl_sy : f.spl_s;
        const int p0 = lane * B;
#pragma unroll 1
        for (int c0 = 0; c0 < 3; c0 += NCI) {
            // right-hand sides and the composed forward maps d -> A d + C of the lane's nodes
            double r[NCI][B], A[NCI], C[NCI];
#pragma unroll
            for (int q = 0; q < NCI; ++q) {
                A[q] = 1.0;
                C[q] = 0.0;
            }
#pragma unroll
            for (int j = 0; j < B; ++j) {
                const int p = p0 + j;
                if (p < nt) {
                    const double iv = invv[p];
                    // rows 0 and nt-1 are the one-sided natural-end rows
                    const int pa = p == 0 ? 0 : p - 1, pb = p == nt - 1 ? p : p + 1;
#pragma unroll
                    for (int q = 0; q < NCI; ++q) {
                        r[q][j] = s * (T(1 + c0 + q, pb, w) - T(1 + c0 + q, pa, w));
                        A[q] = -iv * A[q];
                        C[q] = (r[q][j] - C[q]) * iv;
                    }
                }
            }
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
                for (int q = 0; q < NCI; ++q) {
                    const double Ap = __shfl_up_sync(0xffffffffu, A[q], off);
                    const double Cp = __shfl_up_sync(0xffffffffu, C[q], off);
                    if (lane >= off) {
                        C[q] = A[q] * Cp + C[q];
                        A[q] = A[q] * Ap;
                    }
                }
            }
            double d[NCI];
#pragma unroll
            for (int q = 0; q < NCI; ++q) {
                d[q] = __shfl_up_sync(0xffffffffu, C[q], 1);
                if (lane == 0) d[q] = 0.0;
            }
#pragma unroll
            for (int j = 0; j < B; ++j) {
                const int p = p0 + j;
                if (p < nt) {
                    const double iv = invv[p];
#pragma unroll
                    for (int q = 0; q < NCI; ++q) {
                        d[q] = (r[q][j] - d[q]) * iv;
                        r[q][j] = d[q];
                    }
                }
            }
            // backward: the composed maps m_next -> G m_next + H of the lane's nodes
            double G[NCI], H[NCI];
#pragma unroll
            for (int q = 0; q < NCI; ++q) {
                G[q] = 1.0;
                H[q] = 0.0;
            }
#pragma unroll
            for (int j = B - 1; j >= 0; --j) {
                const int p = p0 + j;
                if (p < nt) {
                    const double cc = cpv[p];
#pragma unroll
                    for (int q = 0; q < NCI; ++q) {
                        H[q] = r[q][j] - cc * H[q];
                        G[q] = -cc * G[q];
                    }
                }
            }
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
                for (int q = 0; q < NCI; ++q) {
                    const double Gn = __shfl_down_sync(0xffffffffu, G[q], off);
                    const double Hn = __shfl_down_sync(0xffffffffu, H[q], off);
                    if (lane + off < 32) {
                        H[q] = G[q] * Hn + H[q];
                        G[q] = G[q] * Gn;
                    }
                }
            }
            double m[NCI];
#pragma unroll
            for (int q = 0; q < NCI; ++q) {
                m[q] = __shfl_down_sync(0xffffffffu, H[q], 1);
                if (lane == 31) m[q] = 0.0;
            }
#pragma unroll
            for (int j = B - 1; j >= 0; --j) {
                const int p = p0 + j;
                if (p < nt) {
                    const double cc = cpv[p];
#pragma unroll
                    for (int q = 0; q < NCI; ++q) {
                        m[q] = r[q][j] - cc * m[q];
                        r[q][j] = m[q];
                    }
                }
            }
            __syncwarp(); // every lane has read its neighbours' velocities
#pragma unroll
            for (int j = 0; j < B; ++j) {
                const int p = p0 + j;
                if (p < nt) {
#pragma unroll
                    for (int q = 0; q < NCI; ++q) T(1 + c0 + q, p, w) = r[q][j];
                }
            }
            __syncwarp();
        }
    }
    __syncthreads();
    // slopes of nodes 3 .. nt-4 (the interior cells)
    each([&](int p, int line) {
        if (p >= 3 && p <= nt - 4) {
            const long long c = cell(line, AXIS == 0 ? p - f.yhost : p - 3);
#pragma unroll
            for (int a = 1; a < 4; ++a) scr[(3 + 3 * (a - 1) + AXIS) * n + c] = T(a, p, line);
        }
    });
}

constexpr int NSUM1 = kStatsSums;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int N>
__device__ __forceinline__ void block_sums(double (&v)[N], double *out)
{
    __shared__ double sm[N][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const double x = warp_sum(v[i]);
        if (lane == 0) sm[i][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < N) {
        double t = 0.0;
        for (int w = 0; w < nw; ++w) t += sm[threadIdx.x][w];
        out[threadIdx.x] = t;
    }
}

// Primitive state of a cell (c2p, update.cpp:882-891) with one reciprocal of
// the density; ri = 1/rho.
__device__ __forceinline__ void cell_prim(const FieldDev &f, long long c, double &den, double &ri, double &u,
                                          double &v, double &w, double &P, double &T)
{
    den = f.W[0][c];
    ri = __drcp_rn(den);
    u = f.W[1][c] * ri;
    v = f.W[2][c] * ri;
    w = f.W[3][c] * ri;
    const double vsq = fma(u, u, fma(v, v, w * w));
    P = (den * f.gm1) * fma(-0.5, vsq, f.W[4][c] * ri);
    T = P * ri * f.iR;
}

// One pass over the interior cells: the means PrintStats forms
// (update.cpp:659-712) and, for the rms of p, T and 1/rho (update.cpp:751-762),
// the first two moments of x - K with K the value at the first interior cell
// (shifted one-pass variance, well conditioned because K lies inside the
// field's range); K goes to kout[0..2].
__global__ void __launch_bounds__(256, 2) k_sums1(FieldDev f, const double *scr, double *partial, double *kout)
{
    const long long n = f.ncell;
    const long long plane = (long long)f.nc * f.nc, c0 = f.ylo * plane, c1 = f.yhi * plane;
    double acc[NSUM1];
#pragma unroll
    for (int i = 0; i < NSUM1; ++i) acc[i] = 0.0;
    double Kp, Kt, Kv;
    {
        double den, u, v, w;
        cell_prim(f, c0, den, Kv, u, v, w, Kp, Kt);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        kout[0] = Kp;
        kout[1] = Kt;
        kout[2] = Kv;
    }
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long c = c0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; c < c1; c += stride) {
        double den, ri, u, v, w, P, T;
        cell_prim(f, c, den, ri, u, v, w, P, T);
        const double *g = scr + 3 * n;
        const double dudy = g[c], dudx = g[n + c], dudz = g[2 * n + c];
        const double dvdy = g[3 * n + c], dvdx = g[4 * n + c], dvdz = g[5 * n + c];
        const double dwdy = g[6 * n + c], dwdx = g[7 * n + c], dwdz = g[8 * n + c];
        const double mu = viscosity(f, T);
        acc[0] += den * (u * u + v * v + w * w);
        acc[1] += mu * (dudx * dudx + dudy * dudy + dudz * dudz + dvdx * dvdx + dvdy * dvdy + dvdz * dvdz +
                        dwdx * dwdx + dwdy * dwdy + dwdz * dwdz);
        acc[2] += dudx * dudx + 0.5 * (dudy + dvdx) * (dudy + dvdx) + 0.5 * (dudz + dwdx) * (dudz + dwdx) +
                  0.5 * (dwdy + dvdz) * (dwdy + dvdz) + dvdy * dvdy + dwdz * dwdz;
        const double a2 = dudx * dudx, b2 = dvdy * dvdy, c2 = dwdz * dwdz;
        acc[3] += a2; acc[4] += a2 * dudx; acc[5] += a2 * a2;
        acc[6] += b2; acc[7] += b2 * dvdy; acc[8] += b2 * b2;
        acc[9] += c2; acc[10] += c2 * dwdz; acc[11] += c2 * c2;
        acc[12] += P;
        acc[13] += T;
        acc[14] += ri;
        acc[15] += u * u + v * v + w * w;
        acc[16] += sqrt(f.gam * P * ri);
        acc[17] += den;
        const double dP = P - Kp, dT = T - Kt, dV = ri - Kv;
        acc[18] += dP;
        acc[19] += dP * dP;
        acc[20] += dT;
        acc[21] += dT * dT;
        acc[22] += dV;
        acc[23] += dV * dV;
    }
    block_sums<NSUM1>(acc, partial + (long long)blockIdx.x * NSUM1);
}

// Sum the per-block partials, one warp per quantity, in a fixed order (so the
// result does not depend on timing); optionally scaled by 1/ncell.
__global__ void k_finalize(const double *partial, int nblocks, int nsum, double scale, double *out)
{
    const int i = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (i >= nsum) return;
    double t = 0.0;
    for (int bidx = lane; bidx < nblocks; bidx += 32) t += partial[(long long)bidx * nsum + i];
    t = warp_sum(t);
    if (lane == 0) out[i] = t * scale;
}

__global__ void k_check(FieldDev f, int *err)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long plane = (long long)f.nc * f.nc, c1 = f.yhi * plane;
    for (long long c = f.ylo * plane + (long long)blockIdx.x * blockDim.x + threadIdx.x; c < c1; c += stride) {
        double w[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) w[q] = f.W[q][c];
        const double p = f.gm1 * (w[4] - 0.5 * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]) / w[0]);
        if (!(w[0] > 0.0) || !(p > 0.0) || !isfinite(w[0] + w[1] + w[2] + w[3] + w[4])) atomicOr(err, 2);
    }
}

template <typename KernelT>
cudaError_t occ(KernelT k, int block, int *n)
{
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, k, block, 0);
}

// Register-cap variants: reconstruction blocks of 128 threads at 3 / 4 / 5
// resident blocks per SM (launch bounds; 168 / 128 / 96 registers), each in
// the windowed and the one-interface form; flux blocks of 64 threads at
// explicit caps of 200 / 168 / 128 registers (5 / 6 / 8 resident blocks).  A
// launch bound of 5 blocks of 64 threads would not give the 200: the compiler
// rounds the resident warps up to a multiple of four and caps at 168, as for
// 6 blocks.  The tuner picks one variant per kernel, precision and sweep.
// Every variant gives bit-identical results.
constexpr int kReconMinb[3] = {3, 4, 5};
constexpr int kFluxRegs[kFluxVariants] = {200, 168, 128};

// The item range of a launch (all items of its kind when b.hi < 0) and the
// blocks it needs: at most cfg.grid, no more than the range fills.
Batch resolve_range(Batch b, int kind, int dir, int variant)
{
    if (b.hi < 0) {
        b.lo = 0;
        b.hi = batch_items(b, kind, dir, variant);
    }
    return b;
}

int range_grid(int grid, long long items, int items_per_block)
{
    const long long need = (items + items_per_block - 1) / items_per_block;
    return int(std::max(1LL, std::min((long long)grid, need)));
}

// Reconstruction variants: 0-2 the windowed kernel (x, y sweeps) or the
// warp-staged segment kernel (z sweep) at the three register caps, 3-5 the
// one-interface-per-thread kernel at the same caps.
template <int DIR, int PREC>
cudaError_t recon_go(Batch b, LaunchCfg cfg, cudaStream_t st)
{
    b = resolve_range(b, K_RECON, DIR, cfg.variant);
    if (b.hi <= b.lo) return cudaSuccess;
    const long long items = b.hi - b.lo;
    if (DIR < 2 && cfg.variant < 3) {
        const int g = range_grid(cfg.grid, items, cfg.block);
        switch (cfg.variant) {
        case 1: k_recon_win<DIR < 2 ? DIR : 0, PREC, kReconMinb[1]><<<g, cfg.block, 0, st>>>(b); break;
        case 2: k_recon_win<DIR < 2 ? DIR : 0, PREC, kReconMinb[2]><<<g, cfg.block, 0, st>>>(b); break;
        default: k_recon_win<DIR < 2 ? DIR : 0, PREC, kReconMinb[0]><<<g, cfg.block, 0, st>>>(b); break;
        }
    } else if (DIR == 2 && cfg.variant < 3) {
        const int g = range_grid(cfg.grid, items, kZSegWarps);
        switch (cfg.variant) {
        case 1: k_recon_zseg<PREC, kReconMinb[1]><<<g, cfg.block, 0, st>>>(b); break;
        case 2: k_recon_zseg<PREC, kReconMinb[2]><<<g, cfg.block, 0, st>>>(b); break;
        default: k_recon_zseg<PREC, kReconMinb[0]><<<g, cfg.block, 0, st>>>(b); break;
        }
    } else {
        const int g = range_grid(cfg.grid, items, cfg.block);
        switch (cfg.variant % 3) {
        case 1: k_recon<DIR, PREC, kReconMinb[1]><<<g, cfg.block, 0, st>>>(b); break;
        case 2: k_recon<DIR, PREC, kReconMinb[2]><<<g, cfg.block, 0, st>>>(b); break;
        default: k_recon<DIR, PREC, kReconMinb[0]><<<g, cfg.block, 0, st>>>(b); break;
        }
    }
    return cudaGetLastError();
}

template <int DIR, int PREC>
cudaError_t flux_go(Batch b, LaunchCfg cfg, cudaStream_t st)
{
    b = resolve_range(b, K_FLUX, DIR, cfg.variant);
    if (b.hi <= b.lo) return cudaSuccess;
    const int g = range_grid(cfg.grid, b.hi - b.lo, cfg.block);
    switch (cfg.variant) {
    case 1: k_flux<DIR, PREC, kFluxRegs[1]><<<g, cfg.block, 0, st>>>(b); break;
    case 2: k_flux<DIR, PREC, kFluxRegs[2]><<<g, cfg.block, 0, st>>>(b); break;
    default: k_flux<DIR, PREC, kFluxRegs[0]><<<g, cfg.block, 0, st>>>(b); break;
    }
    return cudaGetLastError();
}

template <int DIR, int PREC>
cudaError_t occ_kind(int kind, int variant, int block, int *n)
{
    if (kind == K_RECON && DIR < 2 && variant < 3) {
        constexpr int D = DIR < 2 ? DIR : 0;
        if (variant == 1) return occ(k_recon_win<D, PREC, kReconMinb[1]>, block, n);
        if (variant == 2) return occ(k_recon_win<D, PREC, kReconMinb[2]>, block, n);
        return occ(k_recon_win<D, PREC, kReconMinb[0]>, block, n);
    }
    if (kind == K_RECON && DIR == 2 && variant < 3) {
        if (variant == 1) return occ(k_recon_zseg<PREC, kReconMinb[1]>, block, n);
        if (variant == 2) return occ(k_recon_zseg<PREC, kReconMinb[2]>, block, n);
        return occ(k_recon_zseg<PREC, kReconMinb[0]>, block, n);
    }
    if (kind == K_RECON) {
        if (variant % 3 == 1) return occ(k_recon<DIR, PREC, kReconMinb[1]>, block, n);
        if (variant % 3 == 2) return occ(k_recon<DIR, PREC, kReconMinb[2]>, block, n);
        return occ(k_recon<DIR, PREC, kReconMinb[0]>, block, n);
    }
    if (variant == 1) return occ(k_flux<DIR, PREC, kFluxRegs[1]>, block, n);
    if (variant == 2) return occ(k_flux<DIR, PREC, kFluxRegs[2]>, block, n);
    return occ(k_flux<DIR, PREC, kFluxRegs[0]>, block, n);
}

template <int PREC>
cudaError_t occ_dir(int kind, int dir, int variant, int block, int *n)
{
    return dir == 0 ? occ_kind<0, PREC>(kind, variant, block, n)
                    : dir == 1 ? occ_kind<1, PREC>(kind, variant, block, n) : occ_kind<2, PREC>(kind, variant, block, n);
}

} // namespace

cudaError_t launch_recon(const Batch &b, int dir, int prec, LaunchCfg cfg, cudaStream_t st)
{
    if (prec == 0) return dir == 0 ? recon_go<0, 0>(b, cfg, st) : dir == 1 ? recon_go<1, 0>(b, cfg, st) : recon_go<2, 0>(b, cfg, st);
    return dir == 0 ? recon_go<0, 1>(b, cfg, st) : dir == 1 ? recon_go<1, 1>(b, cfg, st) : recon_go<2, 1>(b, cfg, st);
}

cudaError_t launch_flux(const Batch &b, int dir, int prec, LaunchCfg cfg, cudaStream_t st)
{
    if (prec == 0) return dir == 0 ? flux_go<0, 0>(b, cfg, st) : dir == 1 ? flux_go<1, 0>(b, cfg, st) : flux_go<2, 0>(b, cfg, st);
    return dir == 0 ? flux_go<0, 1>(b, cfg, st) : dir == 1 ? flux_go<1, 1>(b, cfg, st) : flux_go<2, 1>(b, cfg, st);
}

cudaError_t launch_update(const Batch &batch, LaunchCfg cfg, cudaStream_t st)
{
    const Batch b = resolve_range(batch, K_UPDATE, 0, 0);
    if (b.hi <= b.lo) return cudaSuccess;
    k_update<<<range_grid(cfg.grid, b.hi - b.lo, cfg.block), cfg.block, 0, st>>>(b);
    return cudaGetLastError();
}

cudaError_t max_resident_blocks(int kind, int dir, int prec, int variant, int block, int *n)
{
    if (kind == K_UPDATE) return occ(k_update, block, n);
    return prec == 0 ? occ_dir<0>(kind, dir, variant, block, n) : occ_dir<1>(kind, dir, variant, block, n);
}

cudaError_t launch_gather(const FieldDev &f, const double *stage, int nsm, cudaStream_t st, long long lo, long long hi)
{
    if (hi < 0) hi = f.ncell;
    if (hi <= lo) return cudaSuccess;
    k_gather<<<helper_grid(hi - lo, 256, nsm), 256, 0, st>>>(f, stage, lo, hi);
    return cudaGetLastError();
}

cudaError_t launch_scatter(const FieldDev &f, double *stage, int nsm, cudaStream_t st, long long lo, long long hi)
{
    const long long nt = f.nc + 6;
    if (hi < 0) hi = (f.ny + 2 * f.yhost) * nt * nt;
    if (hi <= lo) return cudaSuccess;
    k_scatter<<<helper_grid(hi - lo, 256, nsm), 256, 0, st>>>(f, stage, lo, hi);
    return cudaGetLastError();
}

cudaError_t launch_maxwave(const FieldDev &f, unsigned long long *out_bits, int nsm, cudaStream_t st)
{
    k_maxwave<<<helper_grid(f.ncell, 256, nsm), 256, 0, st>>>(f, out_bits);
    return cudaGetLastError();
}

template <int AXIS, int B, int LW>
cudaError_t spline_go(const FieldDev &f, double *scratch, cudaStream_t st)
{
    const size_t bytes = SplineTiles<AXIS, B, LW>::bytes(f.nc + 6);
    cudaError_t e = cudaFuncSetAttribute(k_spline_scan<AXIS, B, LW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)bytes);
    if (e != cudaSuccess) return e;
    // lines: y lines (i, k) of the whole slab, x and z lines of the interior planes
    const long long ny = f.yhi - f.ylo;
    const long long sets = AXIS == 2 ? (ny * f.nc + LW - 1) / LW
                                     : (AXIS == 0 ? f.nc : ny) * ((f.nc + LW - 1) / LW);
    k_spline_scan<AXIS, B, LW><<<(unsigned)sets, 32 * LW, bytes, st>>>(f, scratch);
    return cudaGetLastError();
}

// Nodes per lane B (odd, 32 B >= nt) and lines per block LW: 8 lines (64
// contiguous bytes per row of a y / x tile) up to nt = 288, 4 beyond, so that
// the four tiles stay within 170 KB of shared memory.
template <int AXIS>
cudaError_t spline_axis(const FieldDev &f, double *scratch, cudaStream_t st)
{
    const int nt = f.nc + 6;
    if (nt <= 160) return spline_go<AXIS, 5, 8>(f, scratch, st);
    if (nt <= 288) return spline_go<AXIS, 9, 8>(f, scratch, st);
    if (nt <= 544) return spline_go<AXIS, 17, 4>(f, scratch, st);
    return spline_go<AXIS, 33, 4>(f, scratch, st);
}

cudaError_t launch_stats(const FieldDev &f, double *scratch, double *partial, double *sums, int nsm, cudaStream_t st)
{
    const int block = 256;
    const int grid = stats_grid(f.ncell, block, nsm); // partial holds stats_partial_elems(nsm) >= kStatsSums * grid
    cudaError_t e = spline_axis<0>(f, scratch, st);
    if (e == cudaSuccess) e = spline_axis<1>(f, scratch, st);
    if (e == cudaSuccess) e = spline_axis<2>(f, scratch, st);
    if (e != cudaSuccess) return e;
    k_sums1<<<grid, block, 0, st>>>(f, scratch, partial, sums + NSUM1);
    const double cells = double(f.yhi - f.ylo) * f.nc * f.nc;
    k_finalize<<<1, 32 * NSUM1, 0, st>>>(partial, grid, NSUM1, 1.0 / cells, sums);
    return cudaGetLastError();
}

cudaError_t launch_check(const FieldDev &f, int *err, int nsm, cudaStream_t st)
{
    k_check<<<helper_grid(f.ncell, 256, nsm), 256, 0, st>>>(f, err);
    return cudaGetLastError();
}

} // namespace gks
