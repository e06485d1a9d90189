// gks_timestep_noalloc: the time step (largest |u| + c over a field, then
// dt = cfl dx / max) for callers that may not allocate device memory.
//
// Who needs it: host codes that own every byte of device memory themselves
// (a solver that reserves its whole HBM budget up front, or pools it behind
// its own allocator) and loops that cannot afford cudaMalloc's implicit device
// synchronisation.  gks_timestep works on a context, and gks_create
// allocates; this entry point takes the caller's own device arrays and
// allocates nothing: its only scratch is the file-scope array below, which
// every GPU that loads the library holds until the process exits.
//
// Scratch layout (g_noalloc_scratch, 64-bit words):
//   [0, kBlocks)      per-block maxima (bit images of non-negative doubles)
//   [kBlocks]         arrival counter of the blocks of one call
//   [kBlocks + 1]     the field's maximum, written by the last block
// A call launches `grid` <= kBlocks blocks; block b writes slot b, and the
// last block to arrive reads slots [0, grid) only, so slots left over from an
// earlier call with a larger grid are never read.  The counter and the result
// are cleared before every launch.  Calls share the array: two calls whose
// kernels overlap on the GPU (different streams, or threads) race on it and
// must be serialised by the caller.
//
// The array's device address is looked up (cudaGetSymbolAddress) once per
// device and CUDA context, with that device current, on the first call there:
// a host-side mention of g_noalloc_scratch names a host stand-in, not device
// memory.  If the context is replaced (cudaDeviceReset, then new work), the
// next call sees a new context id and looks the address up again.
#include "../../include/gks_b200.h"

#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "gks_limits.h"

namespace {

constexpr int kBlocks = 1024;  // partial maxima held in the scratch
constexpr int kThreads = 256;
constexpr int kMaxNc = 1024;   // largest field edge accepted (nc^3 cells, 32-bit safe)
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kBlocks + 2];

struct Fields {
    const double *W[5];
};

__device__ __forceinline__ double warp_max_na(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// |u| + c of every cell, each operation rounded as the reference writes it
// (timestep, update.cpp:1064-1073), so that dt matches gks_timestep bit for bit.
__global__ void __launch_bounds__(kThreads) k_maxwave_noalloc(Fields f, long long ncell, double gam,
                                                              unsigned long long *scratch)
{
    const double gm1 = gam - 1;
    double m = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += stride) {
        const double den = f.W[0][c];
        const double u = __ddiv_rn(f.W[1][c], den), v = __ddiv_rn(f.W[2][c], den), w = __ddiv_rn(f.W[3][c], den);
        const double vsq = __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), __dmul_rn(w, w));
        const double P = __dmul_rn(__dmul_rn(den, gm1), __dsub_rn(__ddiv_rn(f.W[4][c], den), __dmul_rn(0.5, vsq)));
        const double val = __dadd_rn(__dsqrt_rn(vsq), __dsqrt_rn(__ddiv_rn(__dmul_rn(gam, P), den)));
        m = val > m ? val : m;
    }
    m = warp_max_na(m);
    __shared__ double sm[kThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sm[wid] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int i = 0; i < kThreads / 32; ++i) b = fmax(b, sm[i]);
        scratch[blockIdx.x] = (unsigned long long)__double_as_longlong(b);
        __threadfence();
        const unsigned long long ticket = atomicAdd(&scratch[kBlocks], 1ull);
        last = ticket == (unsigned long long)gridDim.x - 1;
    }
    __syncthreads();
    if (last) { // the last block to arrive reduces the partials of this call
        double b = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
            b = fmax(b, __longlong_as_double((long long)__ldcg(&scratch[i])));
        b = warp_max_na(b);
        if (lane == 0) sm[wid] = b;
        __syncthreads();
        if (threadIdx.x == 0) {
            double r = 0.0;
            for (int i = 0; i < kThreads / 32; ++i) r = fmax(r, sm[i]);
            scratch[kBlocks + 1] = (unsigned long long)__double_as_longlong(r);
        }
    }
}

std::mutex g_setup_mu;
gks::ContextAddressCache<kMaxDevices> g_scratch_cache;

// Unique id of the calling thread's current CUDA context (cuCtxGetId, reached
// through the runtime's driver entry point so the library needs no link to the
// driver library); 0 where the driver does not provide it.
unsigned long long current_context_id()
{
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetId fn = []() -> GetId {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return (GetId)p;
    }();
    unsigned long long id = 0;
    if (fn && fn(nullptr, &id) != CUDA_SUCCESS) id = 0;
    return id;
}

// Device address of the scratch on `dev` in its current context.
int scratch_for(int dev, unsigned long long **out)
{
    if (dev < 0 || dev >= kMaxDevices) return GKS_EINVAL;
    // make the device's primary context current (it exists from here on), so
    // that its id and the symbol lookup below refer to the same context
    if (cudaSetDevice(dev) != cudaSuccess) return GKS_ECUDA;
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lk(g_setup_mu);
    void *p = nullptr;
    const int rc = g_scratch_cache.get(dev, ctx, [](void **a) {
        return cudaGetSymbolAddress(a, g_noalloc_scratch) == cudaSuccess ? 0 : 1;
    }, &p);
    if (rc != 0) return GKS_ECUDA;
    *out = (unsigned long long *)p;
    return GKS_OK;
}

} // namespace

extern "C" int gks_timestep_noalloc(const double *const dW[5], int nc, double gam, double cfl, void *stream,
                                    double *dt_out)
{
    if (!dW || !dt_out || !(cfl > 0.0) || !(gam > 1.0) || nc < 4) return GKS_EINVAL;
    for (int q = 0; q < 5; ++q)
        if (!dW[q]) return GKS_EINVAL;
    if (nc > kMaxNc) return GKS_ETOOBIG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GKS_ECUDA;
    unsigned long long *scr = nullptr;
    int rc = scratch_for(dev, &scr);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // the arrival counter and the result must start at zero
    if (cudaMemsetAsync(scr + kBlocks, 0, 2 * sizeof(unsigned long long), st) != cudaSuccess) return GKS_ECUDA;
    Fields f;
    for (int q = 0; q < 5; ++q) f.W[q] = dW[q];
    const long long ncell = (long long)nc * nc * nc;
    long long g = (ncell + kThreads - 1) / kThreads;
    const int grid = (int)(g < kBlocks ? g : kBlocks);
    k_maxwave_noalloc<<<grid, kThreads, 0, st>>>(f, ncell, gam, scr);
    if (cudaGetLastError() != cudaSuccess) return GKS_ECUDA;
    unsigned long long bits = 0;
    if (cudaMemcpyAsync(&bits, scr + kBlocks + 1, sizeof(bits), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return GKS_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return GKS_ECUDA;
    double maxval = 0;
    static_assert(sizeof(maxval) == sizeof(bits), "64-bit double");
    memcpy(&maxval, &bits, sizeof(maxval));
    if (!(maxval > 0.0) || !std::isfinite(maxval)) return GKS_ENONFINITE;
    const double dx = 2.0 * (std::atan(1.0) * 4.0) / nc; // FlowField.cpp:45, as gks_create
    *dt_out = cfl * dx / maxval;                          // update.cpp:1078
    return GKS_OK;
}
