// C ABI of the WENO-GKS step (declarations in include/gks_b200.h).
//
// A context owns, per field, one device allocation of 32 * nc^3 doubles
// (state 5, reconstruction records 10, fluxes 15, mu/p 2; the statistics reuse
// the flux arrays as scratch), the field's descriptor in a device array, and one
// CUDA graph holding a whole step for all fields (seven persistent launches).
// The reference instead allocates 50 padded arrays per rank and copies the
// whole field host<->device every step (GPUAlloc.cu:3-17, GPUupdate.cu:74-190).
#include "../../include/gks_b200.h"
#include "gks_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

using gks::FieldDev;

namespace {

struct FieldHost {
    gks_phys phys;
    FieldDev dev;
    double *mem = nullptr;
    double *spl = nullptr;
    // one y-slab of a field split over ranks (gks_create_slab): its interior
    // planes, and the four halo buffers of 15 nc^2 doubles each (send south,
    // send north, receive south, receive north)
    int slab = 0;
    double *halo = nullptr;
    // slab-pipelined host step (gks_evolve): one allocation of 25 nc^3 doubles
    // -- the spare state the step writes (5) and the y and z sweeps' own
    // reconstruction buffers (10 + 10) -- made on first use
    double *pipe = nullptr;
    double *spare[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    // Lagrangian particles (gks_particles_*): one allocation of the nprt
    // particle records (GKS_PREC_FIELDS doubles each, field-major) followed by
    // the statistics scratch; and, made by the first gks_particles_props, the
    // spline coefficients of the five primitives over the padded block
    // (5 (nc+8)^3 doubles, interleaved per node) followed by the nc + 8 pivots
    // of their line solves
    double *prt = nullptr;
    long long nprt = 0;
    double *coef = nullptr;
    bool uploaded = false;
    bool have_dt = false;
};

} // namespace

struct gks_ctx {
    int nfields = 0;
    int precision = 0;
    int flags = 0;
    int device = 0;
    int nsm = 0; // SMs of the device, set by gks_create
    std::vector<FieldHost> fh;
    FieldDev *d_fields = nullptr;
    gks::Batch batch{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaGraphExec_t graph = nullptr;
    double *d_stage = nullptr;
    size_t stage_elems = 0;
    // gks_evolve: the padded staging of the downloaded state, the copy streams
    // and one event per slab and direction
    double *d_stage_out = nullptr;
    size_t stage_out_elems = 0;
    cudaStream_t h2d = nullptr, d2h = nullptr;
    std::vector<cudaEvent_t> ev_in, ev_out;
    double *d_partial = nullptr;
    double *d_sums = nullptr;
    unsigned long long *d_bits = nullptr;
    int *d_err = nullptr;
    gks::LaunchCfg cfg[gks::K_KINDS][3];
    std::string err;
};

namespace {

int fail(gks_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

int cuda_fail(gks_ctx *c, cudaError_t e, const char *what)
{
    return fail(c, GKS_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                 \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

void drop_graph(gks_ctx *ctx)
{
    if (ctx->graph) {
        cudaGraphExecDestroy(ctx->graph);
        ctx->graph = nullptr;
    }
}

int check_field(gks_ctx *ctx, int f)
{
    if (!ctx) return GKS_EINVAL;
    if (f < 0 || f >= ctx->nfields) return fail(ctx, GKS_EINVAL, "field index out of range");
    return GKS_OK;
}

// Coefficients of the natural-spline slope system on nt points:
// Thomas pivots for rows (2,1), (1,4,1)..., (1,2).
void spline_coeffs(int nt, std::vector<double> &cp, std::vector<double> &inv)
{
    cp.assign(nt, 0.0);
    inv.assign(nt, 0.0);
    cp[0] = 0.5;
    inv[0] = 0.5;
    for (int p = 1; p < nt; ++p) {
        const double b = (p == nt - 1) ? 2.0 : 4.0;
        const double c = (p == nt - 1) ? 0.0 : 1.0;
        const double den = b - cp[p - 1];
        cp[p] = c / den;
        inv[p] = 1.0 / den;
    }
}

// Doubles of the padded host layout of field f: 5 x nty x nt^2 (nty = nt, or
// the slab's planes with their ghosts).
size_t host_elems(const gks_ctx *ctx, int f)
{
    const FieldDev &d = ctx->fh[f].dev;
    const size_t nt = (size_t)d.nc + 6;
    return 5 * (size_t)(d.ny + 2 * d.yhost) * nt * nt;
}

int ensure_stage(gks_ctx *ctx, int f)
{
    const size_t need = host_elems(ctx, f);
    if (ctx->stage_elems >= need) return GKS_OK;
    if (ctx->d_stage) cudaFree(ctx->d_stage);
    ctx->d_stage = nullptr;
    ctx->stage_elems = 0;
    if (cudaMalloc(&ctx->d_stage, need * sizeof(double)) != cudaSuccess)
        return fail(ctx, GKS_ENOMEM, "staging buffer allocation failed");
    ctx->stage_elems = need;
    return GKS_OK;
}

// Publish field f's descriptor: to the device array every kernel of an
// ensemble reads, and for a one-field context also into the launch
// parameters (Batch::one), which a captured step graph holds by value, so
// the graph is captured again on the next step.
int push_field(gks_ctx *ctx, int f)
{
    CK(cudaMemcpyAsync(ctx->d_fields + f, &ctx->fh[f].dev, sizeof(FieldDev), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->nfields == 1) {
        ctx->batch.one = ctx->fh[0].dev;
        drop_graph(ctx);
    }
    return GKS_OK;
}

int read_err(gks_ctx *ctx, int *word, bool clear)
{
    CK(cudaMemcpyAsync(word, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    if (clear) CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return GKS_OK;
}

// Persistent grid: `mult` times the resident blocks of the kernel, no more
// blocks than the work needs.
gks::LaunchCfg persistent(gks_ctx *ctx, int kind, int dir, int variant, int mult)
{
    gks::LaunchCfg c;
    c.block = kind == gks::K_UPDATE ? gks::kUpdateBlock : (kind == gks::K_FLUX ? gks::kFluxBlock : gks::kReconBlock);
    c.variant = variant;
    int per_sm = 1;
    if (gks::max_resident_blocks(kind, dir, ctx->precision, variant, c.block, &per_sm) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    long long g = (long long)ctx->nsm * per_sm * mult;
    // work items: window runs (x / y reconstruction variants 0-2), warp-sized
    // z segments of 32 threads each (z reconstruction variants 0-2), else cells
    const long long items = (kind == gks::K_RECON && variant < 3)
                                ? (dir < 2 ? ctx->batch.wtotal : ctx->batch.ztotal * 32)
                                : ctx->batch.total;
    const long long need = (items + c.block - 1) / c.block;
    if (g > need) g = need;
    if (g < 1) g = 1;
    c.grid = (int)g;
    return c;
}

// Untuned defaults: the flux at the 168-register cap (6 blocks of 64
// threads per SM), the reconstruction at its natural register count.
void choose_launch(gks_ctx *ctx)
{
    for (int kind = 0; kind < gks::K_KINDS; ++kind)
        for (int dir = 0; dir < 3; ++dir) {
            const int variant = kind == gks::K_FLUX ? 1 : 0;
            ctx->cfg[kind][dir] = persistent(ctx, kind, dir, variant, 1);
        }
}

// Tuned configurations of this process, per device / precision / flags / sizes.
std::mutex g_tune_mu;
std::map<std::string, std::array<gks::LaunchCfg, gks::K_KINDS * 3>> g_tune_cache;

std::string tune_key(const gks_ctx *ctx)
{
    std::vector<int> ns;
    for (const FieldHost &h : ctx->fh) ns.push_back(h.phys.nc);
    std::sort(ns.begin(), ns.end());
    std::string k = "d" + std::to_string(ctx->device) + "p" + std::to_string(ctx->precision) + "f" +
                    std::to_string(ctx->flags) + ":";
    for (int n : ns) k += std::to_string(n) + ",";
    return k;
}

int record_slab_step(gks_ctx *ctx);

int record_step(gks_ctx *ctx)
{
    if (ctx->fh[0].slab) return record_slab_step(ctx);
    for (int dir = 0; dir < 3; ++dir) {
        CK(gks::launch_recon(ctx->batch, dir, ctx->precision, ctx->cfg[gks::K_RECON][dir], ctx->stream));
        CK(gks::launch_flux(ctx->batch, dir, ctx->precision, ctx->cfg[gks::K_FLUX][dir], ctx->stream));
    }
    CK(gks::launch_update(ctx->batch, ctx->cfg[gks::K_UPDATE][0], ctx->stream));
    return GKS_OK;
}

int build_graph(gks_ctx *ctx)
{
    drop_graph(ctx);
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = record_step(ctx);
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc != GKS_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
    const cudaError_t ei = cudaGraphInstantiate(&ctx->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return cuda_fail(ctx, ei, "cudaGraphInstantiate");
    return GKS_OK;
}

// ---------------------------------------------------------------------------
// Slab-pipelined host step (gks_evolve, one field, one step): the padded host
// state goes up in y-slabs on one copy stream, each slab's reconstruction,
// flux and update stages run on the context's stream as soon as the planes
// they read are on the device, and the updated planes come back on a second
// copy stream, so that the two PCIe directions and the step overlap.
//
// Planes are counted in an unwrapped y coordinate u in [-3, nc - 3) (plane
// u mod nc), uploaded in increasing u: first the three planes below 0 (nc-3
// .. nc-1), then thin slabs (4, 4, 8 planes), so that the first updated
// planes start down early, slabs of about nc / kPipeSlabs planes, and thin
// slabs again (8, 4, 4), so that little work is left after the last upload.
// The y ghost planes go down with the planes they copy: the top ones
// (images of planes 0-2) early, the bottom ones (nc-3 .. nc-1) last.  With F the uploaded
// frontier, the stages advance as far as the planes they read allow (each
// stage covers every plane once):
//   x, z reconstruction  u in [-3, nc-3)   needs W(u)                    u < F
//   x, z flux            u in [-2, nc-2)   needs rec(u-1 .. u+1)         u < rec - 1
//   y reconstruction     u in [-1, nc-1)   needs W(u-2 .. u+3)           u < F - 3
//   y flux               u in [-1, nc-1)   needs rec_y(u), W(u+1), mu/p  u < rec_y, rec
//   update               u in [0, nc)      needs Fx, Fz (u), Fy(u-1, u)
// and every stage completes after the last slab.  Ranges that wrap past a
// stage's end are deferred to completion, so no stage reads a plane before it
// exists.  The update writes the new state into a spare buffer (the old state
// is still read by later slabs' stencils); afterwards the two swap.  The
// sweeps keep separate reconstruction buffers, as their slabs interleave.
// ---------------------------------------------------------------------------
constexpr int kPipeSlabs = 24;
constexpr int kPipeMinNc = 16;
constexpr int kPipeEvents = kPipeSlabs + 16; // events per direction: at least the slabs + 1

// The upload slabs of a field of nc planes, in unwrapped planes (see above).
std::vector<std::pair<long long, long long>> pipe_slabs(long long nc)
{
    std::vector<std::pair<long long, long long>> s{{-3, 0}};
    const long long n = nc - 3, S = (n + kPipeSlabs - 1) / kPipeSlabs;
    const long long head[3] = {4, 4, 8}, tail[3] = {8, 4, 4};
    long long a = 0;
    if (n >= 32 + 2 * S) {
        for (long long w : head) {
            s.push_back({a, a + w});
            a += w;
        }
        for (; a < n - 16; a += S) s.push_back({a, std::min(a + S, n - 16)});
        a = n - 16;
        for (long long w : tail) {
            s.push_back({a, a + w});
            a += w;
        }
        return s;
    }
    for (; a < n; a += S) s.push_back({a, std::min(a + S, n)});
    return s;
}

int ensure_pipe(gks_ctx *ctx, FieldHost &h)
{
    const size_t n = (size_t)h.phys.nc * h.phys.nc * h.phys.nc;
    if (!h.pipe) {
        if (cudaMalloc(&h.pipe, (25 * n + 2) * sizeof(double)) != cudaSuccess) {
            h.pipe = nullptr;
            return fail(ctx, GKS_ENOMEM, "pipelined-step buffers allocation failed");
        }
        for (int q = 0; q < 5; ++q) h.spare[q] = h.pipe + q * n;
    }
    const size_t nt = (size_t)h.phys.nc + 6, need = 5 * nt * nt * nt;
    if (ctx->stage_out_elems < need) {
        if (ctx->d_stage_out) cudaFree(ctx->d_stage_out);
        ctx->d_stage_out = nullptr;
        ctx->stage_out_elems = 0;
        if (cudaMalloc(&ctx->d_stage_out, need * sizeof(double)) != cudaSuccess)
            return fail(ctx, GKS_ENOMEM, "download staging allocation failed");
        ctx->stage_out_elems = need;
    }
    if (!ctx->h2d) CK(cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking));
    if (!ctx->d2h) CK(cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking));
    while ((int)ctx->ev_in.size() < kPipeEvents) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->ev_in.push_back(e);
    }
    while ((int)ctx->ev_out.size() < kPipeEvents) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->ev_out.push_back(e);
    }
    return GKS_OK;
}

// One stage over the physical planes [p0, p1) of the single field.
int pipe_stage(gks_ctx *ctx, const FieldDev &d, int kind, int dir, long long p0, long long p1)
{
    if (p1 <= p0) return GKS_OK;
    const long long nc = d.nc;
    gks::Batch b = ctx->batch;
    b.one = d; // this step's descriptor (spare state, per-sweep reconstruction buffers)
    gks::LaunchCfg c = ctx->cfg[kind][dir];
    long long per_plane = nc * nc; // cells
    if (kind == gks::K_RECON && c.variant < 3) {
        if (dir == 0) per_plane = (long long)d.nrun * nc; // window items (j, run, k)
        else if (dir == 2) per_plane = nc * ((nc + 31) / 32); // z segments ((j, i), segment)
        else c = persistent(ctx, kind, dir, c.variant + 3, 1); // y windows run along y: one interface per thread
    }
    b.lo = p0 * per_plane;
    b.hi = p1 * per_plane;
    if (kind == gks::K_RECON) CK(gks::launch_recon(b, dir, ctx->precision, c, ctx->stream));
    else if (kind == gks::K_FLUX) CK(gks::launch_flux(b, dir, ctx->precision, c, ctx->stream));
    else CK(gks::launch_update(b, c, ctx->stream));
    return GKS_OK;
}

// One step of a y-slab (gks_create_slab): ranged launches over its stored
// planes j = 0 .. ny+5 (the ny interior planes 3 .. ny+2 and three ghost
// planes either side, which the halo exchange filled):
//   x, z reconstruction  planes [2, ny+4)  (the x / z fluxes' transverse
//                                           neighbours; mu/p of plane 2)
//   x, z flux            planes [3, ny+3)
//   y reconstruction     planes [2, ny+3)  (interface j + 1/2: cells j-2 .. j+3)
//   y flux               planes [2, ny+3)
//   update               planes [3, ny+3)  (Fy of planes j-1 and j)
// Every stage reads planes inside [0, ny+6) only: the y index never wraps.
int record_slab_step(gks_ctx *ctx)
{
    const FieldDev &d = ctx->fh[0].dev;
    const long long S = ctx->fh[0].slab;
    int rc;
    if ((rc = pipe_stage(ctx, d, gks::K_RECON, 0, 2, S + 4))) return rc;
    if ((rc = pipe_stage(ctx, d, gks::K_FLUX, 0, 3, S + 3))) return rc;
    if ((rc = pipe_stage(ctx, d, gks::K_RECON, 1, 2, S + 3))) return rc;
    if ((rc = pipe_stage(ctx, d, gks::K_FLUX, 1, 2, S + 3))) return rc;
    if ((rc = pipe_stage(ctx, d, gks::K_RECON, 2, 2, S + 4))) return rc;
    if ((rc = pipe_stage(ctx, d, gks::K_FLUX, 2, 3, S + 3))) return rc;
    return pipe_stage(ctx, d, gks::K_UPDATE, 0, 3, S + 3);
}

int evolve_slabs(gks_ctx *ctx, double *const W[5]);

int evolve_pipelined(gks_ctx *ctx, double *const W[5])
{
    FieldHost &h = ctx->fh[0];
    int rc = ensure_stage(ctx, 0);
    if (!rc) rc = ensure_pipe(ctx, h);
    if (rc) return rc;
    rc = evolve_slabs(ctx, W);
    if (rc != GKS_OK) {
        // drain what was enqueued and put the field's own descriptor back, so
        // that later work reads and writes the field's state buffers; their
        // contents are undefined until the next upload
        cudaStreamSynchronize(ctx->h2d);
        cudaStreamSynchronize(ctx->d2h);
        cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();
        cudaMemcpy(ctx->d_fields, &h.dev, sizeof(FieldDev), cudaMemcpyHostToDevice);
        ctx->batch.one = h.dev;
        drop_graph(ctx);
        h.uploaded = false;
    }
    return rc;
}

// The pipelined step proper (see above); the caller restores the field's
// descriptor if it fails.
int evolve_slabs(gks_ctx *ctx, double *const W[5])
{
    FieldHost &h = ctx->fh[0];
    const long long nc = h.phys.nc, nt = nc + 6, P = nt * nt, Nt = P * nt, plane = nc * nc;
    // descriptor of this step: reads the uploaded state, writes the spare,
    // the y and z sweeps into their own reconstruction buffers
    FieldDev d = h.dev;
    const size_t n = (size_t)nc * nc * nc;
    for (int q = 0; q < 5; ++q) d.Wout[q] = h.spare[q];
    const size_t r0 = (5 * n + 1) & ~(size_t)1; // 16-byte aligned pair arrays
    d.rec[1] = h.pipe + r0;
    d.rec[2] = h.pipe + r0 + 10 * n;
    CK(cudaMemcpyAsync(ctx->d_fields, &d, sizeof(FieldDev), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream)); // the h2d stream writes the stage the last call may still read

    // the caller's five arrays one after another (a (5, nt, nt, nt) block) and a
    // pitch the copy engine accepts: one pitched copy per slab and direction
    int max_pitch = 0;
    CK(cudaDeviceGetAttribute(&max_pitch, cudaDevAttrMaxPitch, ctx->device));
    const size_t pitch = (size_t)Nt * sizeof(double);
    bool contiguous = pitch <= (size_t)max_pitch;
    for (int q = 1; q < 5 && contiguous; ++q) contiguous = W[q] == W[0] + q * Nt;
    const std::vector<std::pair<long long, long long>> slabs = pipe_slabs(nc);
    if (slabs.size() + 1 > ctx->ev_in.size() || slabs.size() > ctx->ev_out.size())
        return fail(ctx, GKS_ETOOBIG, "pipelined step: more slabs than events");
    struct Cur {
        long long done, end;
    };
    Cur rec{-3, nc - 3}, flx{-2, nc - 2}, recy{-1, nc - 1}, fly{-1, nc - 1}, upd{0, nc};
    // run fn over the physical planes of unwrapped [a, b)
    auto phys = [&](long long a, long long b, auto fn) -> int {
        int r = GKS_OK;
        if (a < b && a < 0 && !r) r = fn(a + nc, std::min(b, 0LL) + nc);
        if (a < b && b > 0 && !r) r = fn(std::max(a, 0LL), b);
        return r;
    };
    auto advance = [&](Cur &c, long long ready, auto fn) -> int {
        ready = std::min(ready, c.end);
        if (ready <= c.done) return GKS_OK;
        const int r = phys(c.done, ready, fn);
        c.done = ready;
        return r;
    };
    // padded host planes downloaded after slab k
    std::vector<std::vector<std::pair<long long, long long>>> out_planes;
    bool top_ghosts = false;
    for (size_t k = 0; k < slabs.size(); ++k) {
        const long long a = slabs[k].first, b = slabs[k].second;
        const bool all = k + 1 == slabs.size();
        // upload: padded planes of unwrapped [a, b) (physical planes + 3): one
        // pitched copy of five rows when the caller's components lie one after
        // another in one block, else one copy per component
        int r = phys(a, b, [&](long long p0, long long p1) -> int {
            const size_t off = (size_t)(p0 + 3) * P, bytes = (size_t)(p1 - p0) * P * sizeof(double);
            if (contiguous) {
                // refused when the block is page-locked in several pieces (one
                // registration per component): copy per component from here on
                if (cudaMemcpy2DAsync(ctx->d_stage + off, pitch, W[0] + off, pitch, bytes, 5, cudaMemcpyHostToDevice,
                                      ctx->h2d) == cudaSuccess)
                    return GKS_OK;
                cudaGetLastError();
                contiguous = false;
            }
            for (int q = 0; q < 5; ++q)
                CK(cudaMemcpyAsync(ctx->d_stage + q * Nt + off, W[q] + off, bytes, cudaMemcpyHostToDevice, ctx->h2d));
            return GKS_OK;
        });
        if (r) return r;
        CK(cudaEventRecord(ctx->ev_in[k], ctx->h2d));
        CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_in[k], 0));
        r = phys(a, b, [&](long long p0, long long p1) -> int {
            CK(gks::launch_gather(d, ctx->d_stage, ctx->nsm, ctx->stream, p0 * plane, p1 * plane));
            return GKS_OK;
        });
        if (r) return r;
        const long long F = b;
        auto st = [&](int kind, int dir) {
            return [&, kind, dir](long long p0, long long p1) { return pipe_stage(ctx, d, kind, dir, p0, p1); };
        };
        auto two = [&](int kind, int d0, int d1) {
            return [&, kind, d0, d1](long long p0, long long p1) {
                int e = pipe_stage(ctx, d, kind, d0, p0, p1);
                return e ? e : pipe_stage(ctx, d, kind, d1, p0, p1);
            };
        };
        if ((r = advance(rec, all ? rec.end : F, two(gks::K_RECON, 0, 2)))) return r;
        if ((r = advance(flx, rec.done == rec.end ? flx.end : rec.done - 1, two(gks::K_FLUX, 0, 2)))) return r;
        if ((r = advance(recy, all ? recy.end : F - 3, st(gks::K_RECON, 1)))) return r;
        if ((r = advance(fly, std::min(recy.done, rec.done == rec.end ? fly.end : rec.done), st(gks::K_FLUX, 1))))
            return r;
        const long long u0 = upd.done;
        const long long rx = flx.done == flx.end ? upd.end : flx.done;
        const long long ry = fly.done == fly.end ? upd.end : fly.done;
        if ((r = advance(upd, std::min(rx, ry), st(gks::K_UPDATE, 0)))) return r;
        // the updated planes, with their i / k ghosts, into the download staging
        FieldDev dn = d;
        for (int q = 0; q < 5; ++q) dn.W[q] = d.Wout[q];
        const long long u1 = upd.done;
        std::vector<std::pair<long long, long long>> rng;
        if (u1 > u0) {
            CK(gks::launch_scatter(dn, ctx->d_stage_out, ctx->nsm, ctx->stream, (u0 + 3) * P, (u1 + 3) * P));
            rng.push_back({u0 + 3, u1 + 3});
        }
        if (!top_ghosts && u1 >= 3) { // the top y ghost planes: the periodic images of planes 0 .. 2
            CK(gks::launch_scatter(dn, ctx->d_stage_out, ctx->nsm, ctx->stream, (nt - 3) * P, Nt));
            rng.push_back({nt - 3, nt});
            top_ghosts = true;
        }
        if (all) { // the bottom ones: the images of planes nc-3 .. nc-1
            CK(gks::launch_scatter(dn, ctx->d_stage_out, ctx->nsm, ctx->stream, 0, 3 * P));
            rng.push_back({0, 3});
        }
        CK(cudaEventRecord(ctx->ev_out[k], ctx->stream));
        out_planes.push_back(rng);
    }
    // downloads, each after its slab's update (enqueued after all uploads and
    // stages, so that a blocking copy into pageable memory holds up nothing)
    for (size_t k = 0; k < out_planes.size(); ++k) {
        CK(cudaStreamWaitEvent(ctx->d2h, ctx->ev_out[k], 0));
        for (auto pr : out_planes[k]) {
            if (pr.second <= pr.first) continue;
            const size_t off = (size_t)pr.first * P, bytes = (size_t)(pr.second - pr.first) * P * sizeof(double);
            if (contiguous) {
                if (cudaMemcpy2DAsync(W[0] + off, pitch, ctx->d_stage_out + off, pitch, bytes, 5,
                                      cudaMemcpyDeviceToHost, ctx->d2h) == cudaSuccess)
                    continue;
                cudaGetLastError();
                contiguous = false;
            }
            for (int q = 0; q < 5; ++q)
                CK(cudaMemcpyAsync(W[q] + off, ctx->d_stage_out + q * Nt + off, bytes, cudaMemcpyDeviceToHost,
                                   ctx->d2h));
        }
    }
    CK(cudaEventRecord(ctx->ev_in[slabs.size()], ctx->d2h));
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_in[slabs.size()], 0));
    // the new state is the spare: swap, so that the field's descriptor names it
    for (int q = 0; q < 5; ++q) {
        double *old = h.dev.W[q];
        h.dev.W[q] = h.dev.Wout[q] = h.spare[q];
        h.spare[q] = old;
    }
    CK(cudaMemcpyAsync(ctx->d_fields, &h.dev, sizeof(FieldDev), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->batch.one = h.dev;
    drop_graph(ctx);
    h.uploaded = true;
    return GKS_OK;
}

} // namespace

extern "C" {

const char *gks_last_error(const gks_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

} // extern "C"

namespace {

// A context of `nfields` periodic fields, or (slab > 0, one field) of the
// y-slab of `slab` interior planes starting at global plane y0.
int create_ctx(gks_ctx **out, int nfields, const gks_phys *phys, int precision, int flags, int slab, int y0)
{
    if (!out || nfields < 1 || !phys) return GKS_EINVAL;
    *out = nullptr;
    if (precision != GKS_FP64 && precision != GKS_MIXED) return GKS_EINVAL;
    if (flags & ~(GKS_FIX_ZSWEEP | GKS_DIRECT_ENERGY)) return GKS_EINVAL;
    for (int f = 0; f < nfields; ++f) {
        const gks_phys &p = phys[f];
        if (p.nc < 4 || p.nc > 1024 || !(p.gam > 1.0) || !(p.gas_r > 0) || !(p.T0 > 0) || !(p.mu0 >= 0) ||
            p.K < 0 || (p.visc_law != GKS_VISC_SUTHERLAND && p.visc_law != GKS_VISC_POWER) || !(p.pr_factor > 0))
            return GKS_EINVAL;
    }
    gks_ctx *ctx = new gks_ctx();
    ctx->nfields = nfields;
    ctx->precision = precision;
    ctx->flags = flags;
    auto bail = [&](int rc) {
        gks_destroy(ctx);
        return rc;
    };
    if (cudaGetDevice(&ctx->device) != cudaSuccess) return bail(GKS_ECUDA);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) return bail(GKS_ECUDA);
    ctx->nsm = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(GKS_ECUDA);
    ctx->own_stream = true;

    ctx->fh.resize(nfields);
    // run length of the windowed reconstruction: the longest that leaves the
    // batch at least kWinItemsPerSm window items per SM
    int run = gks::win_run(precision == GKS_MIXED ? 1 : 0);
    for (; run > gks::kWinRunMin; run /= 2) {
        long long items = 0;
        for (int f = 0; f < nfields; ++f)
            items += (long long)(slab ? slab + 6 : phys[f].nc) * phys[f].nc * ((phys[f].nc + run - 1) / run);
        if (items >= (long long)gks::kWinItemsPerSm * ctx->nsm) break;
    }
    long long base = 0, wbase = 0, zbase = 0;
    const double pi = std::atan(1.0) * 4.0; // param.h:14
    for (int f = 0; f < nfields; ++f) {
        FieldHost &h = ctx->fh[f];
        h.phys = phys[f];
        h.slab = slab;
        const gks_phys &p = phys[f];
        const int ny = slab ? slab + 6 : p.nc; // stored planes
        const long long n = (long long)ny * p.nc * p.nc;
        // state 5 n, reconstruction pairs 10 n (from an even offset: 16-byte
        // aligned), fluxes 15 n, mu/p 2 n
        const long long r0 = (5 * n + 1) & ~1LL;
        const size_t elems = (size_t)(r0 + 27 * n);
        if (cudaMalloc(&h.mem, elems * sizeof(double)) != cudaSuccess) return bail(GKS_ENOMEM);
        if (cudaMemset(h.mem, 0, elems * sizeof(double)) != cudaSuccess) return bail(GKS_ECUDA);
        FieldDev &d = h.dev;
        memset(&d, 0, sizeof(d));
        for (int q = 0; q < 5; ++q) d.W[q] = d.Wout[q] = h.mem + q * n;
        for (int sw = 0; sw < 3; ++sw) d.rec[sw] = h.mem + r0;
        for (int q = 0; q < 15; ++q) d.F[q] = h.mem + r0 + (10 + q) * n;
        for (int q = 0; q < 2; ++q) d.tau[q] = h.mem + r0 + (25 + q) * n;
        // spline coefficients: x / z lines of nt nodes, y lines of nty (a
        // slab's own when it is a slab)
        const int nt = p.nc + 6, nty = slab ? ny : nt;
        const size_t nspl = 2 * (size_t)nt + (slab ? 2 * (size_t)nty : 0);
        if (cudaMalloc(&h.spl, nspl * sizeof(double)) != cudaSuccess) return bail(GKS_ENOMEM);
        for (int a = 0; a < (slab ? 2 : 1); ++a) {
            const int m = a ? nty : nt;
            double *dst = h.spl + (a ? 2 * (size_t)nt : 0);
            std::vector<double> cp, inv;
            spline_coeffs(m, cp, inv);
            if (cudaMemcpy(dst, cp.data(), m * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(dst + m, inv.data(), m * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
                return bail(GKS_ECUDA);
        }
        d.spl_cp = h.spl;
        d.spl_inv = h.spl + nt;
        d.spl_cpy = slab ? h.spl + 2 * nt : d.spl_cp;
        d.spl_invy = slab ? h.spl + 2 * nt + nty : d.spl_inv;
        d.ny = ny;
        d.nyw = slab ? gks::kNoWrap : p.nc;
        d.yhost = slab ? 0 : 3;
        d.ylo = slab ? 3 : 0;
        d.yhi = slab ? slab + 3 : p.nc;
        if (slab && cudaMalloc(&h.halo, 4 * 15 * (size_t)p.nc * p.nc * sizeof(double)) != cudaSuccess)
            return bail(GKS_ENOMEM);
        d.base = base;
        d.ncell = n;
        base += (n + gks::kItemAlign - 1) / gks::kItemAlign * gks::kItemAlign;
        d.run = run;
        d.nrun = (p.nc + run - 1) / run;
        d.nwin = (long long)ny * p.nc * d.nrun;
        d.wbase = wbase;
        wbase += (d.nwin + gks::kItemAlign - 1) / gks::kItemAlign * gks::kItemAlign;
        d.nzseg = (long long)ny * p.nc * ((p.nc + 31) / 32);
        d.zbase = zbase;
        zbase += d.nzseg;
        d.nc = p.nc;
        // magic number for x / nc (round-up method): l = ceil(log2 nc),
        // m = floor(2^32 (2^l - nc) / nc) + 1, x / nc = (umulhi(x, m) + x) >> l
        {
            int l = 0;
            while ((1u << l) < (unsigned)p.nc) ++l;
            d.nc_shift = l;
            d.nc_magic = (unsigned)(((1ull << 32) * ((1ull << l) - (unsigned)p.nc)) / (unsigned)p.nc + 1);
        }
        d.K = p.K;
        d.visc_law = p.visc_law;
        d.flags = flags;
        d.dx = 2.0 * pi / p.nc; // FlowField.cpp:45
        d.inv_dx = 1 / d.dx;
        d.dt = 0.0;
        d.gam = p.gam;
        d.gm1 = p.gam - 1;
        d.R = p.gas_r;
        d.iR = 1.0 / p.gas_r;
        d.cT = (p.gam - 1) / p.gas_r;
        d.icT = p.gas_r / (p.gam - 1.0);
        d.T0 = p.T0;
        d.iT0 = 1.0 / p.T0;
        d.mu0 = p.mu0;
        d.visc_exp = p.visc_exp;
        d.kA = p.pr_factor * 4.0 / (p.K + 3);
        d.hig = 0.5 * (d.icT * d.iR); // R / (gamma - 1) * 1 / R
        d.ksn = 2.0 * d.inv_dx;
        d.kst = 0.5 * d.inv_dx;
        d.hK2 = (p.K + 2) * 0.5;
        const int kint[4] = {p.K + 2, p.K + 4, (p.K + 2) * (p.K + 4), -(p.K + 3)};
        for (int i = 0; i < 4; ++i) {
            d.kd[i] = (double)kint[i];
            d.kf[i] = (float)kint[i];
        }
        // spline grids of the reference's einspline call (Interpolation.cpp:10-27):
        // a segment's grid starts at its first plane sta, here 0 along x and z
        // and y0 along y
        auto scale = [&](int sta, int num) {
            const double start = (sta - 3) * d.dx + 0.5 * d.dx;
            const double end = start + (num - 1) * d.dx;
            return 3.0 / ((end - start) / (double)(num - 1));
        };
        d.spl_s = scale(0, nt);
        d.spl_sy = scale(slab ? y0 : 0, nty);
    }
    if (cudaMalloc(&ctx->d_fields, nfields * sizeof(FieldDev)) != cudaSuccess) return bail(GKS_ENOMEM);
    for (int f = 0; f < nfields; ++f)
        if (cudaMemcpy(ctx->d_fields + f, &ctx->fh[f].dev, sizeof(FieldDev), cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(GKS_ECUDA);
    if (cudaMalloc(&ctx->d_partial, gks::stats_partial_elems(ctx->nsm) * sizeof(double)) != cudaSuccess)
        return bail(GKS_ENOMEM);
    if (cudaMalloc(&ctx->d_sums, 32 * sizeof(double)) != cudaSuccess) return bail(GKS_ENOMEM);
    if (cudaMalloc(&ctx->d_bits, sizeof(unsigned long long)) != cudaSuccess) return bail(GKS_ENOMEM);
    if (cudaMalloc(&ctx->d_err, sizeof(int)) != cudaSuccess) return bail(GKS_ENOMEM);
    if (cudaMemset(ctx->d_err, 0, sizeof(int)) != cudaSuccess) return bail(GKS_ECUDA);
    ctx->batch.fields = ctx->d_fields;
    ctx->batch.nfields = nfields;
    ctx->batch.total = base;
    ctx->batch.wtotal = wbase;
    ctx->batch.ztotal = zbase;
    ctx->batch.err = ctx->d_err;
    ctx->batch.one = ctx->fh[0].dev;
    choose_launch(ctx);
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(GKS_ECUDA);
    *out = ctx;
    return GKS_OK;
}

} // namespace

extern "C" {

int gks_create(gks_ctx **out, int nfields, const gks_phys *phys, int precision, int flags)
{
    return create_ctx(out, nfields, phys, precision, flags, 0, 0);
}

int gks_create_slab(gks_ctx **out, const gks_phys *phys, int ny, int y0, int precision, int flags)
{
    if (!out || !phys) return GKS_EINVAL;
    *out = nullptr;
    if (ny < 3 || ny > phys->nc || y0 < 0 || y0 + ny > phys->nc) return GKS_EINVAL;
    return create_ctx(out, 1, phys, precision, flags, ny, y0);
}

void gks_destroy(gks_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drop_graph(ctx);
    for (FieldHost &h : ctx->fh) {
        if (h.mem) cudaFree(h.mem);
        if (h.spl) cudaFree(h.spl);
        if (h.pipe) cudaFree(h.pipe);
        if (h.halo) cudaFree(h.halo);
        if (h.prt) cudaFree(h.prt);
        if (h.coef) cudaFree(h.coef);
    }
    if (ctx->d_fields) cudaFree(ctx->d_fields);
    if (ctx->d_stage) cudaFree(ctx->d_stage);
    if (ctx->d_stage_out) cudaFree(ctx->d_stage_out);
    for (cudaEvent_t e : ctx->ev_in) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->ev_out) cudaEventDestroy(e);
    if (ctx->h2d) cudaStreamDestroy(ctx->h2d);
    if (ctx->d2h) cudaStreamDestroy(ctx->d2h);
    if (ctx->d_partial) cudaFree(ctx->d_partial);
    if (ctx->d_sums) cudaFree(ctx->d_sums);
    if (ctx->d_bits) cudaFree(ctx->d_bits);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int gks_upload(gks_ctx *ctx, int f, double *const W[5])
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    if (!W) return fail(ctx, GKS_EINVAL, "null field pointer");
    for (int q = 0; q < 5; ++q)
        if (!W[q]) return fail(ctx, GKS_EINVAL, "null component pointer");
    CK(cudaSetDevice(ctx->device));
    if ((rc = ensure_stage(ctx, f))) return rc;
    const size_t Nt = host_elems(ctx, f) / 5;
    for (int q = 0; q < 5; ++q)
        CK(cudaMemcpyAsync(ctx->d_stage + q * Nt, W[q], Nt * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(gks::launch_gather(ctx->fh[f].dev, ctx->d_stage, ctx->nsm, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->fh[f].uploaded = true;
    return GKS_OK;
}

int gks_download(gks_ctx *ctx, int f, double *const W[5])
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    if (!W) return fail(ctx, GKS_EINVAL, "null field pointer");
    for (int q = 0; q < 5; ++q)
        if (!W[q]) return fail(ctx, GKS_EINVAL, "null component pointer");
    CK(cudaSetDevice(ctx->device));
    if ((rc = ensure_stage(ctx, f))) return rc;
    const size_t Nt = host_elems(ctx, f) / 5;
    CK(gks::launch_scatter(ctx->fh[f].dev, ctx->d_stage, ctx->nsm, ctx->stream));
    for (int q = 0; q < 5; ++q)
        CK(cudaMemcpyAsync(W[q], ctx->d_stage + q * Nt, Nt * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return GKS_OK;
}

int gks_evolve(gks_ctx *ctx, int f, double *const W[5], int nsteps)
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    if (!W) return fail(ctx, GKS_EINVAL, "null field pointer");
    for (int q = 0; q < 5; ++q)
        if (!W[q]) return fail(ctx, GKS_EINVAL, "null component pointer");
    if (nsteps < 1) return fail(ctx, GKS_EINVAL, "nsteps must be at least 1");
    if (ctx->fh[f].slab && nsteps > 1)
        return fail(ctx, GKS_EINVAL, "a slab advances one step per call: its ghosts come from the caller's halo exchange");
    if (!ctx->fh[f].have_dt) return fail(ctx, GKS_ESTATE, "evolve before dt of field " + std::to_string(f));
    CK(cudaSetDevice(ctx->device));
    if (ctx->nfields == 1 && nsteps == 1 && ctx->fh[f].phys.nc >= kPipeMinNc && !ctx->fh[f].slab)
        return evolve_pipelined(ctx, W);
    // several fields or steps: upload, the captured steps, download
    if ((rc = gks_upload(ctx, f, W))) return rc;
    for (int g = 0; g < ctx->nfields; ++g)
        if (!ctx->fh[g].uploaded) return fail(ctx, GKS_ESTATE, "evolve with field " + std::to_string(g) + " not uploaded");
    if ((rc = gks_step(ctx, nsteps))) return rc;
    return gks_download(ctx, f, W);
}

int gks_host_register(void *p, size_t bytes, int *registered)
{
    if (registered) *registered = 0;
    if (!p || bytes == 0) return GKS_EINVAL;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) == cudaSuccess && a.type == cudaMemoryTypeHost) return GKS_OK;
    cudaGetLastError(); // an unregistered pointer may leave an error behind on older runtimes
    if (cudaHostRegister(p, bytes, cudaHostRegisterDefault) != cudaSuccess) {
        cudaGetLastError();
        return GKS_ECUDA;
    }
    if (registered) *registered = 1;
    return GKS_OK;
}

int gks_host_unregister(void *p)
{
    if (!p) return GKS_EINVAL;
    if (cudaHostUnregister(p) != cudaSuccess) {
        cudaGetLastError();
        return GKS_ECUDA;
    }
    return GKS_OK;
}

int gks_set_dt(gks_ctx *ctx, int f, double dt)
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(ctx, GKS_EINVAL, "dt must be positive and finite");
    CK(cudaSetDevice(ctx->device));
    ctx->fh[f].dev.dt = dt;
    ctx->fh[f].have_dt = true;
    return push_field(ctx, f);
}

int gks_timestep(gks_ctx *ctx, int f, double cfl, double *dt_out)
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    if (!(cfl > 0.0)) return fail(ctx, GKS_EINVAL, "cfl must be positive");
    if (!ctx->fh[f].uploaded) return fail(ctx, GKS_ESTATE, "timestep before upload");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemsetAsync(ctx->d_bits, 0, sizeof(unsigned long long), ctx->stream));
    CK(gks::launch_maxwave(ctx->fh[f].dev, ctx->d_bits, ctx->nsm, ctx->stream));
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, ctx->d_bits, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    double maxval;
    memcpy(&maxval, &bits, sizeof(double));
    if (!(maxval > 0.0) || !std::isfinite(maxval)) return fail(ctx, GKS_ENONFINITE, "max wave speed is not finite");
    const double dt = cfl * ctx->fh[f].dev.dx / maxval; // update.cpp:1078
    if (dt_out) *dt_out = dt;
    return gks_set_dt(ctx, f, dt);
}

int gks_step(gks_ctx *ctx, int nsteps)
{
    if (!ctx) return GKS_EINVAL;
    if (nsteps < 0) return fail(ctx, GKS_EINVAL, "negative step count");
    if (ctx->fh[0].slab && nsteps > 1)
        return fail(ctx, GKS_EINVAL, "a slab advances one step between halo exchanges");
    for (int f = 0; f < ctx->nfields; ++f) {
        if (!ctx->fh[f].uploaded) return fail(ctx, GKS_ESTATE, "step before upload of field " + std::to_string(f));
        if (!ctx->fh[f].have_dt) return fail(ctx, GKS_ESTATE, "step before dt of field " + std::to_string(f));
    }
    CK(cudaSetDevice(ctx->device));
    if (!ctx->graph) {
        int rc = build_graph(ctx);
        if (rc) return rc;
    }
    for (int s = 0; s < nsteps; ++s) CK(cudaGraphLaunch(ctx->graph, ctx->stream));
    return GKS_OK;
}

int gks_sync(gks_ctx *ctx)
{
    if (!ctx) return GKS_EINVAL;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    int word = 0;
    int rc = read_err(ctx, &word, true);
    if (rc) return rc;
    if (word) return fail(ctx, GKS_ENONFINITE, "a step produced non-finite or non-positive density/pressure");
    return GKS_OK;
}

int gks_check(gks_ctx *ctx)
{
    if (!ctx) return GKS_EINVAL;
    CK(cudaSetDevice(ctx->device));
    for (int f = 0; f < ctx->nfields; ++f) {
        CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
        CK(gks::launch_check(ctx->fh[f].dev, ctx->d_err, ctx->nsm, ctx->stream));
        int word = 0;
        int rc = read_err(ctx, &word, true);
        if (rc) return rc;
        if (word) return fail(ctx, GKS_ENONFINITE, "field " + std::to_string(f) + " holds non-finite or non-positive density/pressure");
    }
    return GKS_OK;
}

int gks_stats_part(gks_ctx *ctx, int f, double *part)
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    if (!part) return fail(ctx, GKS_EINVAL, "null output");
    if (!ctx->fh[f].uploaded) return fail(ctx, GKS_ESTATE, "stats before upload");
    CK(cudaSetDevice(ctx->device));
    const FieldDev &d = ctx->fh[f].dev;
    CK(gks::launch_stats(d, d.F[0], ctx->d_partial, ctx->d_sums, ctx->nsm, ctx->stream));
    CK(cudaMemcpyAsync(part, ctx->d_sums, 27 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    part[27] = double(d.yhi - d.ylo) * d.nc * d.nc;
    return GKS_OK;
}

int gks_stats_reduce(const double *parts, int nparts, const gks_phys *phys, gks_stats_out *out)
{
    if (!parts || nparts < 1 || !phys || !out) return GKS_EINVAL;
    // cell-weighted means of the parts (MPI_Reduce / MPI_Allreduce of the
    // sums, update.cpp:714-741); the shifted moments of p, T and 1/rho move
    // to the first part's shift K: with e = K_r - K,
    //   E[x - K] = E[x - K_r] + e,  E[(x - K)^2] = E[(x - K_r)^2] + 2 e E[x - K_r] + e^2
    double N = 0.0;
    for (int r = 0; r < nparts; ++r) {
        if (!(parts[28 * r + 27] > 0.0)) return GKS_EINVAL;
        N += parts[28 * r + 27];
    }
    double s[24] = {};
    for (int r = 0; r < nparts; ++r) {
        const double *m = parts + 28 * r, w = m[27] / N;
        for (int i = 0; i < 18; ++i) s[i] += w * m[i];
        for (int x = 0; x < 3; ++x) {
            const double e = m[24 + x] - parts[24 + x], m1 = m[18 + 2 * x], m2 = m[19 + 2 * x];
            s[18 + 2 * x] += w * (m1 + e);
            s[19 + 2 * x] += w * (m2 + (2.0 * e * m1 + e * e));
        }
    }
    const gks_phys &p = *phys;
    // PrintStats normalisation (update.cpp:727-776)
    out->tke = s[0];
    out->diss = s[1];
    out->sijsij = s[2];
    out->skew[0] = s[4] / std::pow(s[3], 1.5);
    out->skew[1] = s[7] / std::pow(s[6], 1.5);
    out->skew[2] = s[10] / std::pow(s[9], 1.5);
    out->kurt[0] = s[5] / (s[3] * s[3]);
    out->kurt[1] = s[8] / (s[6] * s[6]);
    out->kurt[2] = s[11] / (s[9] * s[9]);
    // population variances from the shifted moments: E[(x-K)^2] - E[x-K]^2
    auto var = [&](int i) { return std::max(0.0, s[i + 1] - s[i] * s[i]); };
    out->prms = std::sqrt(var(18)) / (p.gam * p.p0 * p.Mt * p.Mt);
    out->trms = std::sqrt(var(20)) / ((p.gam - 1) * p.T0 * p.Mt * p.Mt);
    out->vrms = std::sqrt(var(22)) / (p.Mt * p.Mt / p.den0);
    out->mach_t = std::sqrt(s[15]) / s[16];
    out->rho_mean = s[17];
    return GKS_OK;
}

int gks_stats(gks_ctx *ctx, int f, gks_stats_out *out)
{
    double part[28];
    int rc = gks_stats_part(ctx, f, part);
    if (rc) return rc;
    if (!out) return fail(ctx, GKS_EINVAL, "null output");
    return gks_stats_reduce(part, 1, &ctx->fh[f].phys, out);
}

// ---------------------------------------------------------------------------
// Lagrangian particles of one periodic field (kernels in gks_particles.cu).
// ---------------------------------------------------------------------------
int gks_particles_locate(gks_ctx *ctx, int f, int n, const double *x0, const double *y0, const double *z0)
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    FieldHost &h = ctx->fh[f];
    if (h.slab) return fail(ctx, GKS_EINVAL, "particles: a y-slab is not a whole periodic field");
    if (n < 1 || !x0 || !y0 || !z0) return fail(ctx, GKS_EINVAL, "particles: need n >= 1 and three position arrays");
    for (int a = 0; a < n; ++a)
        if (!std::isfinite(x0[a]) || !std::isfinite(y0[a]) || !std::isfinite(z0[a]))
            return fail(ctx, GKS_EINVAL, "particles: non-finite initial position");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream)); // earlier work may still read the old records
    const size_t rec = (size_t)GKS_PREC_FIELDS * n;
    if (h.nprt != n) {
        if (h.prt) cudaFree(h.prt);
        h.prt = nullptr;
        h.nprt = 0;
        if (cudaMalloc(&h.prt, (rec + gks::particle_partial_elems(ctx->nsm) + 8) * sizeof(double)) != cudaSuccess) {
            h.prt = nullptr;
            return fail(ctx, GKS_ENOMEM, "particle records allocation failed");
        }
        h.nprt = n;
    }
    // a new Particle holds zeros (Particle::Particle, ParticleTrack.cpp:6-10),
    // its position pos[0..2] = (y0, x0, z0) (initializeParticle, :12-18)
    CK(cudaMemsetAsync(h.prt, 0, rec * sizeof(double), ctx->stream));
    const double *src[3] = {y0, x0, z0};
    for (int q = 0; q < 3; ++q)
        CK(cudaMemcpyAsync(h.prt + (size_t)q * n, src[q], n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return GKS_OK;
}

int gks_particles_props(gks_ctx *ctx, int f)
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    FieldHost &h = ctx->fh[f];
    if (!h.nprt) return fail(ctx, GKS_ESTATE, "particles: props before gks_particles_locate");
    if (!h.uploaded) return fail(ctx, GKS_ESTATE, "particles: props before upload");
    CK(cudaSetDevice(ctx->device));
    const long long nt = h.phys.nc + 6, M = nt + 2, M3 = M * M * M;
    if (!h.coef) {
        if (cudaMalloc(&h.coef, (5 * M3 + M) * sizeof(double)) != cudaSuccess) {
            h.coef = nullptr;
            return fail(ctx, GKS_ENOMEM, "particle spline coefficients allocation failed");
        }
        // pivots of the (1, 4, 1) eliminations along lines of nt nodes
        std::vector<double> w(M, 0.0);
        w[2] = 0.25;
        for (long long m = 3; m < nt; ++m) w[m] = 1.0 / (4.0 - w[m - 1]);
        CK(cudaMemcpy(h.coef + 5 * M3, w.data(), M * sizeof(double), cudaMemcpyHostToDevice));
    }
    // the spline grid of the padded block (get_bsplinep, Interpolation.cpp:10-27,
    // sta = 0): nt nodes from -3 dx + dx/2, spacing (end - start) / (nt - 1)
    const double dx = h.dev.dx;
    const double start = (0 - 3) * dx + 0.5 * dx, end = start + (nt - 1) * dx;
    const double hinv = 1.0 / ((end - start) / (double)(nt - 1));
    CK(gks::launch_particle_splines(h.dev, h.coef, h.coef + 5 * M3, ctx->nsm, ctx->stream));
    CK(gks::launch_particle_props(h.dev, h.coef, start, hinv, h.prt, h.nprt, ctx->nsm, ctx->stream));
    return GKS_OK;
}

int gks_particles_track(gks_ctx *ctx, int f, double dt)
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    FieldHost &h = ctx->fh[f];
    if (!h.nprt) return fail(ctx, GKS_ESTATE, "particles: track before gks_particles_locate");
    if (!std::isfinite(dt)) return fail(ctx, GKS_EINVAL, "particles: dt must be finite");
    CK(cudaSetDevice(ctx->device));
    const double twopi = 2 * std::atan(1.0) * 4.0; // 2*pi as param.h:14 defines pi
    CK(gks::launch_particle_track(h.prt, h.nprt, dt, twopi, ctx->nsm, ctx->stream));
    return GKS_OK;
}

int gks_particles_stats(gks_ctx *ctx, int f, gks_particle_stats_out *out)
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    FieldHost &h = ctx->fh[f];
    if (!out) return fail(ctx, GKS_EINVAL, "null output");
    if (!h.nprt) return fail(ctx, GKS_ESTATE, "particles: stats before gks_particles_locate");
    CK(cudaSetDevice(ctx->device));
    double *partial = h.prt + (size_t)GKS_PREC_FIELDS * h.nprt;
    double *sums = partial + gks::particle_partial_elems(ctx->nsm);
    CK(gks::launch_particle_stats(h.prt, h.nprt, partial, sums, ctx->nsm, ctx->stream));
    double m[6];
    CK(cudaMemcpyAsync(m, sums, sizeof(m), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    // normalisation of GetParticleStats (update.cpp:1168-1175)
    out->tke = m[0];
    out->sijsij = m[1];
    out->dudx2 = m[2];
    out->dudx3 = m[3];
    out->dwdz2 = m[4];
    out->dwdz3 = m[5];
    out->skew_u = m[3] / std::pow(m[2], 1.5);
    out->skew_w = m[5] / std::pow(m[4], 1.5);
    out->count = h.nprt;
    return GKS_OK;
}

int gks_particles_get(gks_ctx *ctx, int f, double *rec)
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    FieldHost &h = ctx->fh[f];
    if (!rec) return fail(ctx, GKS_EINVAL, "null output");
    if (!h.nprt) return fail(ctx, GKS_ESTATE, "particles: get before gks_particles_locate");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(rec, h.prt, (size_t)GKS_PREC_FIELDS * h.nprt * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return GKS_OK;
}

int gks_halo_buffers(gks_ctx *ctx, double **bufs, size_t *elems)
{
    if (!ctx || !bufs) return GKS_EINVAL;
    const FieldHost &h = ctx->fh[0];
    if (!h.slab) return fail(ctx, GKS_EINVAL, "halo buffers belong to a slab context");
    const size_t m = 15 * (size_t)h.phys.nc * h.phys.nc;
    for (int i = 0; i < 4; ++i) bufs[i] = h.halo + i * m;
    if (elems) *elems = m;
    return GKS_OK;
}

} // extern "C"

namespace {

// Three planes [j0, j0 + 3) of the five components <-> a halo buffer laid out
// [component][plane][nc^2]: one pitched copy when the components lie evenly
// spaced in one allocation (as gks_create_slab lays them out), else one copy
// per component.
int halo_copy(gks_ctx *ctx, long long j0, double *buf, bool to_buf)
{
    const FieldHost &h = ctx->fh[0];
    const size_t P = (size_t)h.phys.nc * h.phys.nc, n = (size_t)h.dev.ncell, width = 3 * P * sizeof(double);
    bool even = true;
    for (int q = 1; q < 5; ++q) even = even && h.dev.W[q] == h.dev.W[0] + q * n;
    int max_pitch = 0;
    CK(cudaDeviceGetAttribute(&max_pitch, cudaDevAttrMaxPitch, ctx->device));
    if (even && n * sizeof(double) <= (size_t)max_pitch) {
        double *st = h.dev.W[0] + j0 * P;
        if (to_buf)
            CK(cudaMemcpy2DAsync(buf, width, st, n * sizeof(double), width, 5, cudaMemcpyDeviceToDevice, ctx->stream));
        else
            CK(cudaMemcpy2DAsync(st, n * sizeof(double), buf, width, width, 5, cudaMemcpyDeviceToDevice, ctx->stream));
        return GKS_OK;
    }
    for (int q = 0; q < 5; ++q) {
        double *st = h.dev.W[q] + j0 * P, *b = buf + q * 3 * P;
        CK(cudaMemcpyAsync(to_buf ? b : st, to_buf ? st : b, width, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return GKS_OK;
}

int halo_ready(gks_ctx *ctx)
{
    if (!ctx) return GKS_EINVAL;
    if (!ctx->fh[0].slab) return fail(ctx, GKS_EINVAL, "halo exchange belongs to a slab context");
    if (!ctx->fh[0].uploaded) return fail(ctx, GKS_ESTATE, "halo exchange before upload");
    CK(cudaSetDevice(ctx->device));
    return GKS_OK;
}

} // namespace

extern "C" {

int gks_halo_pack(gks_ctx *ctx)
{
    int rc = halo_ready(ctx);
    if (rc) return rc;
    double *b[4];
    gks_halo_buffers(ctx, b, nullptr);
    const long long S = ctx->fh[0].slab;
    if ((rc = halo_copy(ctx, 3, b[0], true))) return rc; // south: the first three interior planes
    return halo_copy(ctx, S, b[1], true);                // north: the last three
}

int gks_halo_unpack(gks_ctx *ctx)
{
    int rc = halo_ready(ctx);
    if (rc) return rc;
    double *b[4];
    gks_halo_buffers(ctx, b, nullptr);
    const long long S = ctx->fh[0].slab;
    if ((rc = halo_copy(ctx, 0, b[2], false))) return rc; // from the south neighbour's north planes
    return halo_copy(ctx, S + 3, b[3], false);             // from the north neighbour's south planes
}

int gks_device_fields(gks_ctx *ctx, int f, double *dW[5])
{
    int rc = check_field(ctx, f);
    if (rc) return rc;
    if (!dW) return fail(ctx, GKS_EINVAL, "null output");
    for (int q = 0; q < 5; ++q) dW[q] = ctx->fh[f].dev.W[q];
    ctx->fh[f].uploaded = true; // the caller may fill the arrays in place
    return GKS_OK;
}

int gks_set_stream(gks_ctx *ctx, void *stream)
{
    if (!ctx) return GKS_EINVAL;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    drop_graph(ctx);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    if (stream) {
        ctx->stream = (cudaStream_t)stream;
        ctx->own_stream = false;
    } else {
        CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->own_stream = true;
    }
    return GKS_OK;
}

int gks_select_device(int device)
{
    return cudaSetDevice(device) == cudaSuccess ? GKS_OK : GKS_ECUDA;
}

int gks_time_stages(gks_ctx *ctx, int reps, double *ms)
{
    if (!ctx || !ms || reps < 1) return GKS_EINVAL;
    if (ctx->fh[0].slab) return fail(ctx, GKS_EINVAL, "stage timing runs whole-field launches: not for a slab");
    for (int f = 0; f < ctx->nfields; ++f)
        if (!ctx->fh[f].uploaded || !ctx->fh[f].have_dt) return fail(ctx, GKS_ESTATE, "time_stages before upload/dt");
    CK(cudaSetDevice(ctx->device));
    cudaEvent_t ev[8];
    for (int i = 0; i < 8; ++i) CK(cudaEventCreate(&ev[i]));
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    int rc = GKS_OK;
    for (int r = 0; r < reps && rc == GKS_OK; ++r) {
        cudaError_t e = cudaEventRecord(ev[0], ctx->stream);
        for (int dir = 0; dir < 3 && e == cudaSuccess; ++dir) {
            e = gks::launch_recon(ctx->batch, dir, ctx->precision, ctx->cfg[gks::K_RECON][dir], ctx->stream);
            if (e == cudaSuccess) e = cudaEventRecord(ev[2 * dir + 1], ctx->stream);
            if (e == cudaSuccess)
                e = gks::launch_flux(ctx->batch, dir, ctx->precision, ctx->cfg[gks::K_FLUX][dir], ctx->stream);
            if (e == cudaSuccess) e = cudaEventRecord(ev[2 * dir + 2], ctx->stream);
        }
        if (e == cudaSuccess) e = gks::launch_update(ctx->batch, ctx->cfg[gks::K_UPDATE][0], ctx->stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev[7], ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[7]);
        for (int i = 0; i < 7 && e == cudaSuccess; ++i) {
            float t = 0;
            e = cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
            acc[i] += t;
        }
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "stage timing");
    }
    for (int i = 0; i < 8; ++i) cudaEventDestroy(ev[i]);
    if (rc) return rc;
    for (int i = 0; i < 7; ++i) ms[i] = acc[i] / reps;
    return GKS_OK;
}

int gks_autotune(gks_ctx *ctx, int reps)
{
    if (!ctx || reps < 1) return GKS_EINVAL;
    if (ctx->fh[0].slab)
        return fail(ctx, GKS_EINVAL, "the tuner times whole-field launches: tune a periodic field of the same edge "
                                     "and pin its choice on the slab (gks_set_launch)");
    for (int f = 0; f < ctx->nfields; ++f)
        if (!ctx->fh[f].uploaded || !ctx->fh[f].have_dt) return fail(ctx, GKS_ESTATE, "autotune before upload/dt");
    CK(cudaSetDevice(ctx->device));
    const std::string key = tune_key(ctx);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            for (int i = 0; i < gks::K_KINDS * 3; ++i) ctx->cfg[i / 3][i % 3] = it->second[i];
            drop_graph(ctx);
            return GKS_OK;
        }
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int rc = GKS_OK;
    // time `reps` launches of one candidate after one untimed launch; the
    // reconstruction and flux kernels only write scratch, so repeating them
    // leaves the state unchanged (the update is not tuned for that reason)
    auto time_it = [&](int kind, int dir, gks::LaunchCfg c, float *ms) -> cudaError_t {
        auto go = [&]() {
            return kind == gks::K_RECON ? gks::launch_recon(ctx->batch, dir, ctx->precision, c, ctx->stream)
                                        : gks::launch_flux(ctx->batch, dir, ctx->precision, c, ctx->stream);
        };
        cudaError_t e = go();
        if (e == cudaSuccess) e = cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < reps && e == cudaSuccess; ++r) e = go();
        if (e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
        return e;
    };
    const int mults[2] = {1, 2};
    for (int dir = 0; dir < 3 && rc == GKS_OK; ++dir) {
        for (int kind : {int(gks::K_RECON), int(gks::K_FLUX)}) {
            const int nvar = kind == gks::K_RECON ? gks::kReconVariants : gks::kFluxVariants;
            // every candidate is timed in two interleaved rounds and keeps its
            // faster one, so that one disturbed measurement does not decide
            std::vector<gks::LaunchCfg> cand;
            for (int v = 0; v < nvar; ++v)
                for (int m : mults) cand.push_back(persistent(ctx, kind, dir, v, m));
            std::vector<float> t(cand.size(), 1e30f);
            for (int round = 0; round < 2 && rc == GKS_OK; ++round)
                for (size_t i = 0; i < cand.size() && rc == GKS_OK; ++i) {
                    float ms = 0;
                    const cudaError_t e = time_it(kind, dir, cand[i], &ms);
                    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "autotune");
                    else if (ms < t[i]) t[i] = ms;
                }
            gks::LaunchCfg bestc = ctx->cfg[kind][dir];
            float best = 1e30f;
            for (size_t i = 0; i < cand.size(); ++i)
                if (t[i] < best) {
                    best = t[i];
                    bestc = cand[i];
                }
            ctx->cfg[kind][dir] = bestc;
            // leave this sweep's reconstruction in place for timing its flux
            if (rc == GKS_OK && kind == gks::K_RECON) {
                const cudaError_t e = gks::launch_recon(ctx->batch, dir, ctx->precision, bestc, ctx->stream);
                if (e != cudaSuccess) rc = cuda_fail(ctx, e, "autotune");
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    std::array<gks::LaunchCfg, gks::K_KINDS * 3> a;
    for (int i = 0; i < gks::K_KINDS * 3; ++i) a[i] = ctx->cfg[i / 3][i % 3];
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = a;
    }
    drop_graph(ctx);
    return GKS_OK;
}

int gks_get_launch(gks_ctx *ctx, int kind, int dir, int *block, int *grid, int *variant)
{
    if (!ctx || kind < 0 || kind >= gks::K_KINDS || dir < 0 || dir > 2) return GKS_EINVAL;
    const gks::LaunchCfg &c = ctx->cfg[kind][dir];
    if (block) *block = c.block;
    if (grid) *grid = c.grid;
    if (variant) *variant = c.variant;
    return GKS_OK;
}

int gks_set_launch(gks_ctx *ctx, int kind, int dir, int grid, int variant)
{
    if (!ctx || kind < 0 || kind >= gks::K_KINDS || dir < 0 || dir > 2) return GKS_EINVAL;
    const int nvar = kind == gks::K_RECON ? gks::kReconVariants : (kind == gks::K_FLUX ? gks::kFluxVariants : 1);
    if (variant < 0 || variant >= nvar) return fail(ctx, GKS_EINVAL, "no such kernel variant");
    if (grid < 0) return fail(ctx, GKS_EINVAL, "negative grid");
    CK(cudaSetDevice(ctx->device));
    gks::LaunchCfg c = persistent(ctx, kind, dir, variant, 1);
    if (grid > 0) c.grid = grid;
    ctx->cfg[kind][dir] = c;
    drop_graph(ctx);
    return GKS_OK;
}

int gks_get_stream(gks_ctx *ctx, void **stream)
{
    if (!ctx || !stream) return GKS_EINVAL;
    *stream = (void *)ctx->stream;
    return GKS_OK;
}

} // extern "C"
