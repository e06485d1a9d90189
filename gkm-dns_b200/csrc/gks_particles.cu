// Lagrangian particles of one periodic field (weno/src/ParticleTrack.cpp,
// update.cpp:1082-1303): spline interpolation of the primitives at every
// particle, the particle step and the particle statistics.
//
// The reference interpolates with einspline's 3-D cubic B-spline under natural
// boundary conditions over the rank's padded block (generateSplines,
// update.cpp:1199-1213; get_bsplinep, Interpolation.cpp:3-31) and evaluates
// value and gradient at each particle (getParticleProp,
// ParticleTrack.cpp:90-97).  Here the same interpolant is built on the device
// from the resident state:
//   * k_node_prims: the five primitives (den, u, v, w, p) at the (nc+6)^3
//     nodes of the padded block -- the ghost nodes as the periodic image --
//     written into the interior of one coefficient array of (nc+8)^3 nodes
//     with the five fields interleaved per node (node-major, so that the 4 x 4
//     x 4 block a particle reads is 16 runs of 20 contiguous doubles);
//   * k_bspline_zlines, k_bspline_lines<AXIS>: the natural cubic B-spline
//     coefficients, one tridiagonal (1, 4, 1) solve per grid line, along z,
//     then x, then y (the tensor product).  With c_1 = f_0 and c_N = f_{N-1} fixed by the natural
//     end conditions, c_2 .. c_{N-1} come from forward elimination with the
//     host-computed pivots w_2 = 1/4, w_m = 1/(4 - w_{m-1}) and back
//     substitution, then c_0 = 2 c_1 - c_2 and c_{N+1} = 2 c_N - c_{N-1};
//   * k_particle_props: per particle the cell and cubic B-spline weights
//     along each axis, then value and gradient of the five splines from
//     their 4 x 4 x 4 coefficient blocks.
// Every operation is written in the oracle's order and this file is compiled
// without implicit contraction, so results agree with the oracle bit for bit
// except the statistics sums, whose order differs (a deterministic tree).
//
// Particle records: GKS_PREC_FIELDS doubles per particle, field-major (field
// q of particle a at q * n + a, so that a warp's accesses are coalesced):
// position (y, x, z) = the reference's pos[0..2], DEN, U[0..2] = (u, v, w),
// P, and the gradients (d/dy, d/dx, d/dz) of DEN, u, v, w and P.
#include "gks_kernels.cuh"
#include "../../include/gks_b200.h"

#include <cuda_runtime.h>
#include <algorithm>

namespace gks {

namespace {

constexpr int kPrtBlock = 128;
constexpr int kLineBlock = 128;
constexpr int kSumBlock = 256;
constexpr int kNSum = 6; // TKE, SijSij, DUDX2, DUDX3, DWDZ2, DWDZ3
constexpr int kNF = 5;   // fields interleaved per node: den, u, v, w, p

__device__ __forceinline__ int wrap_nc(int x, int n) { return x < 0 ? x + n : (x >= n ? x - n : x); }

// generateSplines' primitives at every node of the padded block
// (update.cpp:1201-1208): den, u, v, w, p, into the coefficient array at
// node offset (1, 1, 1).
__global__ void __launch_bounds__(kLineBlock) k_node_prims(FieldDev f, double *coef)
{
    const int nc = f.nc;
    const long long nt = nc + 6, M = nt + 2, N3 = nt * nt * nt;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const double gm1 = f.gam - 1;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < N3; c += stride) {
        const int k = int(c % nt);
        const long long r = c / nt;
        const int i = int(r % nt), j = int(r / nt);
        const long long cell = ((long long)wrap_nc(j - 3, nc) * nc + wrap_nc(i - 3, nc)) * nc + wrap_nc(k - 3, nc);
        const double den = f.W[0][cell];
        const double u = f.W[1][cell] / den, v = f.W[2][cell] / den, w = f.W[3][cell] / den;
        const double Vsqr = u * u + v * v + w * w;
        const double p = (den * gm1) * (f.W[4][cell] / den - 0.5 * Vsqr);
        double *o = coef + kNF * (((long long)(j + 1) * M + (i + 1)) * M + (k + 1));
        o[0] = den;
        o[1] = u;
        o[2] = v;
        o[3] = w;
        o[4] = p;
    }
}

// Natural cubic B-spline coefficients of one grid line in place:
// c[m * s], m = 1 .. N, hold the data f_{m-1} on entry (N >= 4).
// Both recurrences move through the line in groups of kLineGroup positions,
// every load of a group issued before its first use, so that a thread keeps
// kLineGroup loads in flight instead of one (the recurrences themselves are
// sequential).
constexpr int kLineGroup = 8;

__device__ __forceinline__ void bspline_line(long long N, double *c, long long s, const double *__restrict__ w)
{
    const double f0 = c[s], fl = c[N * s];
    double d = (6.0 * c[2 * s] - f0) * __ldg(w + 2);
    c[2 * s] = d;
    // forward elimination over m = 3 .. N-2, then the last row m = N-1
    long long m = 3;
    for (; m + kLineGroup <= N - 1; m += kLineGroup) {
        double v[kLineGroup];
#pragma unroll
        for (int g = 0; g < kLineGroup; ++g) v[g] = c[(m + g) * s];
#pragma unroll
        for (int g = 0; g < kLineGroup; ++g) {
            d = (6.0 * v[g] - d) * __ldg(w + m + g);
            c[(m + g) * s] = d;
        }
    }
    for (; m < N - 1; ++m) {
        d = (6.0 * c[m * s] - d) * __ldg(w + m);
        c[m * s] = d;
    }
    d = ((6.0 * c[(N - 1) * s] - fl) - d) * __ldg(w + N - 1);
    c[(N - 1) * s] = d;
    const double cl = d; // c_{N-1}
    double cn = d;
    // back substitution over m = N-2 .. 2
    m = N - 2;
    for (; m - kLineGroup + 1 >= 2; m -= kLineGroup) {
        double v[kLineGroup];
#pragma unroll
        for (int g = 0; g < kLineGroup; ++g) v[g] = c[(m - g) * s];
#pragma unroll
        for (int g = 0; g < kLineGroup; ++g) {
            cn = v[g] - __ldg(w + m - g) * cn;
            c[(m - g) * s] = cn;
        }
    }
    for (; m >= 2; --m) {
        cn = c[m * s] - __ldg(w + m) * cn;
        c[m * s] = cn;
    }
    c[0] = 2.0 * f0 - cn;
    c[(N + 1) * s] = 2.0 * fl - cl;
}

// One pass of line solves over all five fields along AXIS (0 y, 1 x): a
// thread per line and field, consecutive threads on consecutive (k, field),
// so that every access of a warp is one contiguous run; the lines include the
// end coefficients of the passes before (x pass N M lines per field, y pass
// M^2).
template <int AXIS>
__global__ void __launch_bounds__(kLineBlock) k_bspline_lines(double *coef, long long N, const double *w)
{
    static_assert(AXIS == 0 || AXIS == 1, "the z pass is k_bspline_zlines");
    const long long M = N + 2;
    const long long L = kNF * (AXIS == 1 ? N * M : M * M);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < L; t += stride) {
        if (AXIS == 1) {
            // t = ((j - 1) M + k) kNF + q: element m of the line at ((j M + m) M + k) kNF + q
            const long long l = t / kNF, q = t - l * kNF, j = 1 + l / M, k = l % M;
            bspline_line(N, coef + (j * M * M + k) * kNF + q, M * kNF, w);
        } else {
            // t = (i M + k) kNF + q: element m at ((m M + i) M + k) kNF + q
            bspline_line(N, coef + t, M * M * kNF, w);
        }
    }
}

// The z pass, whose lines are contiguous: a block takes kZRows grid rows
// (j, i) with their kNF interleaved fields and moves them through shared
// memory in tiles of kZChunk positions -- a row's chunk is one contiguous run
// of kNF kZChunk doubles -- each thread running the recurrences of one row
// and field: the arithmetic of bspline_line, chunk by chunk, forward
// elimination over increasing positions, back substitution and the two end
// coefficients over decreasing ones.  The tile's row pitch (kZPitch = 5 mod
// 16 doubles) keeps a half-warp's accesses, thread t at row t / 5 and field
// t % 5, on distinct banks.
constexpr int kZRows = 32;
constexpr int kZThreads = kNF * kZRows;
constexpr int kZChunk = 32;
constexpr int kZRun = kNF * kZChunk;     // doubles of one row's chunk
constexpr int kZPitch = kZRun + 5;       // 165 = 5 mod 16
constexpr int kZBatch = 16;              // reads of a thread in flight at once

__global__ void __launch_bounds__(kZThreads) k_bspline_zlines(double *coef, long long N, const double *__restrict__ w)
{
    __shared__ double tile[kZRows][kZPitch];
    __shared__ double *rbase[kZRows];
    const long long M = N + 2, R = N * N;
    const int t = threadIdx.x, r = t / kNF, q = t - r * kNF;
    const long long nchunk = (M + kZChunk - 1) / kZChunk;
    for (long long r0 = (long long)blockIdx.x * kZRows; r0 < R; r0 += (long long)gridDim.x * kZRows) {
        if (t < kZRows) {
            const long long rr = r0 + t; // row (1 + rr / N, 1 + rr % N)
            rbase[t] = rr < R ? coef + ((1 + rr / N) * M + (1 + rr % N)) * M * kNF : nullptr;
        }
        __syncthreads();
        const bool mine = rbase[r] != nullptr;
        const double *line = mine ? rbase[r] + q : nullptr; // element m at line[m * kNF]
        double f0 = 0.0, fl = 0.0, d = 0.0;
        if (mine) {
            f0 = line[kNF];
            fl = line[N * kNF];
        }
        // tile <-> global: each row's chunk [p0, p0 + kZChunk) x fields is one run
        auto move = [&](long long p0, bool load) {
            const long long lim = (M - p0) * kNF; // doubles of the row left from p0
            if (load) {
#pragma unroll
                for (int h = 0; h < kZRows * kZRun / kZThreads; h += kZBatch) {
                    double v[kZBatch];
#pragma unroll
                    for (int b = 0; b < kZBatch; ++b) {
                        const int idx = t + (h + b) * kZThreads, rw = idx / kZRun, e = idx - rw * kZRun;
                        const double *bp = rbase[rw];
                        v[b] = (bp && e < lim) ? bp[p0 * kNF + e] : 0.0;
                    }
#pragma unroll
                    for (int b = 0; b < kZBatch; ++b) {
                        const int idx = t + (h + b) * kZThreads, rw = idx / kZRun, e = idx - rw * kZRun;
                        tile[rw][e] = v[b];
                    }
                }
            } else {
#pragma unroll
                for (int h = 0; h < kZRows * kZRun / kZThreads; ++h) {
                    const int idx = t + h * kZThreads, rw = idx / kZRun, e = idx - rw * kZRun;
                    double *bp = rbase[rw];
                    if (bp && e < lim) bp[p0 * kNF + e] = tile[rw][e];
                }
            }
        };
        for (long long c = 0; c < nchunk; ++c) {
            const long long p0 = c * kZChunk;
            move(p0, true);
            __syncthreads();
            if (mine) {
#pragma unroll
                for (int e = 0; e < kZChunk; ++e) {
                    const long long m = p0 + e;
                    const double x = tile[r][e * kNF + q], wm = __ldg(w + (m < M ? m : M - 1));
                    if (m >= 2 && m <= N - 1) {
                        if (m == 2) d = (6.0 * x - f0) * wm;
                        else if (m < N - 1) d = (6.0 * x - d) * wm;
                        else d = ((6.0 * x - fl) - d) * wm;
                        tile[r][e * kNF + q] = d;
                    }
                }
            }
            __syncthreads();
            move(p0, false);
            __syncthreads();
        }
        const double cl = d; // c_{N-1}
        double cn = d;
        for (long long c = nchunk - 1; c >= 0; --c) {
            const long long p0 = c * kZChunk;
            move(p0, true);
            __syncthreads();
            if (mine) {
#pragma unroll
                for (int e = kZChunk - 1; e >= 0; --e) {
                    const long long m = p0 + e;
                    const double x = tile[r][e * kNF + q], wm = __ldg(w + (m < M ? m : M - 1));
                    if (m == N + 1) {
                        tile[r][e * kNF + q] = 2.0 * fl - cl;
                    } else if (m >= 2 && m <= N - 2) {
                        cn = x - wm * cn;
                        tile[r][e * kNF + q] = cn;
                    } else if (m == 0) {
                        tile[r][e * kNF + q] = 2.0 * f0 - cn; // cn = c_2 here
                    }
                }
            }
            __syncthreads();
            move(p0, false);
            __syncthreads();
        }
    }
}

// Cell and cubic B-spline weights of position x along one axis of num nodes;
// the cell is clamped to the last interval (as the oracle's).
__device__ __forceinline__ int bspline_weights(double x, double start, double hinv, int num, double b[4],
                                               double db[4])
{
    const double u = (x - start) * hinv;
    double fl = floor(u);
    fl = fmin(fmax(fl, 0.0), double(num - 2)); // NaN -> 0: stays inside the arrays
    const int i = int(fl);
    const double t = u - fl;
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

// getParticleProp (ParticleTrack.cpp:90-97) of every particle: value and
// gradient of the five splines at its position.  A row of the 4 x 4 x 4
// coefficient block -- four nodes along z with their five fields -- is one
// contiguous run of 20 doubles, read once for all fields; each field's sums
// keep the order of a field-by-field evaluation (rows along y, then x, nodes
// along z innermost).  Measured alternatives: the five fields in separate
// arrays read 8.4 GB of DRAM per 2^20 particles at 256^3 (1.43 ms) against
// 4.1 GB here (1.65 ms, latency-bound at 8 warps per SM: the 35 sums and the
// row take 254 registers; capped at 168 they spill and take 1.74 ms); field
// by field over the interleaved rows, each field's pass fetching the rows
// again, 17 GB and 5.7 ms (L2 does not hold a resident wave's rows between
// passes).
__global__ void __launch_bounds__(kPrtBlock) k_particle_props(const double *__restrict__ coef, int nt, double start,
                                                              double hinv, double *rec, long long n)
{
    const long long M = nt + 2;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x; a < n; a += stride) {
        double by[4], dby[4], bx[4], dbx[4], bz[4], dbz[4];
        const int iy = bspline_weights(rec[a], start, hinv, nt, by, dby);
        const int ix = bspline_weights(rec[n + a], start, hinv, nt, bx, dbx);
        const int iz = bspline_weights(rec[2 * n + a], start, hinv, nt, bz, dbz);
        double v[kNF], gy[kNF], gx[kNF], gz[kNF];
#pragma unroll
        for (int q = 0; q < kNF; ++q) v[q] = gy[q] = gx[q] = gz[q] = 0.0;
#pragma unroll
        for (int ia = 0; ia < 4; ++ia) {
            double va[kNF], gxa[kNF], gza[kNF];
#pragma unroll
            for (int q = 0; q < kNF; ++q) va[q] = gxa[q] = gza[q] = 0.0;
#pragma unroll
            for (int ib = 0; ib < 4; ++ib) {
                const double *r = coef + (((long long)(iy + ia) * M + (ix + ib)) * M + iz) * kNF;
                double x[4 * kNF];
#pragma unroll
                for (int c = 0; c < 4 * kNF; ++c) x[c] = __ldg(r + c);
#pragma unroll
                for (int q = 0; q < kNF; ++q) {
                    const double r0 = x[q], r1 = x[kNF + q], r2 = x[2 * kNF + q], r3 = x[3 * kNF + q];
                    const double sv = ((bz[0] * r0 + bz[1] * r1) + bz[2] * r2) + bz[3] * r3;
                    const double sd = ((dbz[0] * r0 + dbz[1] * r1) + dbz[2] * r2) + dbz[3] * r3;
                    va[q] += bx[ib] * sv;
                    gxa[q] += dbx[ib] * sv;
                    gza[q] += bx[ib] * sd;
                }
            }
#pragma unroll
            for (int q = 0; q < kNF; ++q) {
                v[q] += by[ia] * va[q];
                gy[q] += dby[ia] * va[q];
                gx[q] += by[ia] * gxa[q];
                gz[q] += by[ia] * gza[q];
            }
        }
#pragma unroll
        for (int q = 0; q < kNF; ++q) {
            rec[(3 + q) * n + a] = v[q];
            rec[(8 + 3 * q) * n + a] = gy[q] * hinv;
            rec[(9 + 3 * q) * n + a] = gx[q] * hinv;
            rec[(10 + 3 * q) * n + a] = gz[q] * hinv;
        }
    }
}

// Particle::updatePosition (ParticleTrack.cpp:43-65): pos[0] (y) moves with
// U[1] = v, pos[1] (x) with U[0] = u, pos[2] (z) with U[2] = w; each
// coordinate is wrapped once into [0, 2 pi].
__global__ void __launch_bounds__(kPrtBlock) k_particle_track(double *rec, long long n, double dt, double twopi)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x; a < n; a += stride) {
        const int vel[3] = {5, 4, 6};
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            double x = rec[q * n + a];
            x += rec[vel[q] * n + a] * dt;
            if (x > twopi) x = x - twopi;
            if (x < 0) x = twopi + x;
            rec[q * n + a] = x;
        }
    }
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// GetParticleStats' sums (update.cpp:1141-1162): per block, in a fixed order
// (grid-stride per thread, warp tree, warps in order).
__global__ void __launch_bounds__(kSumBlock) k_particle_sums(const double *__restrict__ rec, long long n,
                                                             double *partial)
{
    double acc[kNSum] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x; a < n; a += stride) {
        const double U0 = rec[4 * n + a], U1 = rec[5 * n + a], U2 = rec[6 * n + a];
        acc[0] += (U0 * U0 + U1 * U1 + U2 * U2);
        const double dudy = rec[11 * n + a], dudx = rec[12 * n + a], dudz = rec[13 * n + a];
        const double dvdy = rec[14 * n + a], dvdx = rec[15 * n + a], dvdz = rec[16 * n + a];
        const double dwdy = rec[17 * n + a], dwdx = rec[18 * n + a], dwdz = rec[19 * n + a];
        const double s1 = dudy + dvdx, s2 = dudz + dwdx, s3 = dwdy + dvdz;
        acc[1] += (dudx * dudx + 0.5 * (s1 * s1) + 0.5 * (s2 * s2) + 0.5 * (s3 * s3) + dvdy * dvdy + dwdz * dwdz);
        acc[2] += dudx * dudx;
        acc[3] += dudx * dudx * dudx;
        acc[4] += dwdz * dwdz;
        acc[5] += dwdz * dwdz * dwdz;
    }
    __shared__ double sm[kSumBlock / 32][kNSum];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < kNSum; ++s) {
        const double v = warp_sum(acc[s]);
        if (lane == 0) sm[wid][s] = v;
    }
    __syncthreads();
    if (threadIdx.x < kNSum) {
        double v = 0.0;
        for (int w = 0; w < kSumBlock / 32; ++w) v += sm[w][threadIdx.x];
        partial[(long long)blockIdx.x * kNSum + threadIdx.x] = v;
    }
}

// The block sums in a fixed order (one warp per quantity), divided by n.
__global__ void k_particle_final(const double *partial, int nblocks, double nd, double *out)
{
    const int s = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (s >= kNSum) return;
    double v = 0.0;
    for (int b = lane; b < nblocks; b += 32) v += partial[(long long)b * kNSum + s];
    v = warp_sum(v);
    if (lane == 0) out[s] = v / nd;
}

int grid_for(long long items, int block, int nsm, int per_sm)
{
    const long long need = (items + block - 1) / block;
    return int(std::max(1LL, std::min(need, (long long)nsm * per_sm)));
}

} // namespace

int particle_partial_elems(int nsm) { return nsm * 4 * kNSum; }

cudaError_t launch_particle_splines(const FieldDev &f, double *coef, const double *w, int nsm, cudaStream_t st)
{
    const long long nt = f.nc + 6, M = nt + 2;
    k_node_prims<<<grid_for(nt * nt * nt, kLineBlock, nsm, 16), kLineBlock, 0, st>>>(f, coef);
    k_bspline_zlines<<<grid_for(kNF * nt * nt, kZThreads, nsm, 4), kZThreads, 0, st>>>(coef, nt, w);
    k_bspline_lines<1><<<grid_for(kNF * nt * M, kLineBlock, nsm, 16), kLineBlock, 0, st>>>(coef, nt, w);
    k_bspline_lines<0><<<grid_for(kNF * M * M, kLineBlock, nsm, 16), kLineBlock, 0, st>>>(coef, nt, w);
    return cudaGetLastError();
}

cudaError_t launch_particle_props(const FieldDev &f, const double *coef, double start, double hinv, double *rec,
                                  long long n, int nsm, cudaStream_t st)
{
    k_particle_props<<<grid_for(n, kPrtBlock, nsm, 16), kPrtBlock, 0, st>>>(coef, f.nc + 6, start, hinv, rec, n);
    return cudaGetLastError();
}

cudaError_t launch_particle_track(double *rec, long long n, double dt, double twopi, int nsm, cudaStream_t st)
{
    k_particle_track<<<grid_for(n, kPrtBlock, nsm, 16), kPrtBlock, 0, st>>>(rec, n, dt, twopi);
    return cudaGetLastError();
}

cudaError_t launch_particle_stats(const double *rec, long long n, double *partial, double *sums, int nsm,
                                  cudaStream_t st)
{
    const int g = grid_for(n, kSumBlock, nsm, 4);
    k_particle_sums<<<g, kSumBlock, 0, st>>>(rec, n, partial);
    k_particle_final<<<1, 32 * kNSum, 0, st>>>(partial, g, double(n), sums);
    return cudaGetLastError();
}

} // namespace gks
