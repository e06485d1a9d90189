// Peak FMA throughput of the FP64 and FP32 pipes, the denominators of the
// step's roofline (the hot path is bound by the FP64 / FP32 CUDA-core pipes:
// no dense contraction, ~350 flop per byte of compulsory traffic).
// Every thread runs 8 independent FMA chains; 2 flops per FMA.
#include "../../include/gks_b200.h"

#include <cuda_runtime.h>

namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_chains(T *sink, int iters, T b, T c)
{
    T a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = T(threadIdx.x + j) * T(1e-3);
#pragma unroll 4
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = fma(a[j], b, c);
    }
    T s = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += a[j];
    if (s == T(-12345.0)) sink[blockIdx.x] = s; // never true; keeps the chains live
}

template <typename T>
int measure(double *tflops)
{
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GKS_ECUDA;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return GKS_ECUDA;
    const int block = 256, grid = nsm * 8, iters = sizeof(T) == 8 ? 40000 : 80000;
    T *sink = nullptr;
    if (cudaMalloc(&sink, grid * sizeof(T)) != cudaSuccess) return GKS_ENOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const T b = T(0.999999), c = T(1e-6);
    k_fma_chains<T><<<grid, block>>>(sink, iters / 8, b, c); // warm-up
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(e0);
        k_fma_chains<T><<<grid, block>>>(sink, iters, b, c);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess) return GKS_ECUDA;
    const double flops = 2.0 * 8.0 * (double)iters * (double)grid * block;
    *tflops = flops / (best * 1e-3) / 1e12;
    return GKS_OK;
}

} // namespace

extern "C" int gks_peak_flops(int precision, double *tflops)
{
    if (!tflops) return GKS_EINVAL;
    return precision == GKS_FP64 ? measure<double>(tflops) : measure<float>(tflops);
}
