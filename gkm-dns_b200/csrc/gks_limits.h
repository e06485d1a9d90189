// Launch-size arithmetic shared by the kernels' launchers and the C ABI, and
// the per-context address cache of the zero-allocation entry point.  Plain
// host C++ (no CUDA types), so that the CPU tests compile it on its own and
// check the limits for any SM count.
#pragma once

#include <cstddef>

namespace gks {

// Sums the statistics reduction keeps per block (k_sums1).
constexpr int kStatsSums = 24;
// Blocks per SM of the grid-stride helper kernels (gather, scatter, maxwave,
// check) and of the statistics reduction.
constexpr int kHelperBlocksPerSm = 32;
constexpr int kStatsBlocksPerSm = 8;

// Grid of a grid-stride helper kernel over `items` work items: enough blocks
// for the items, at most kHelperBlocksPerSm per SM, at least one.
inline int helper_grid(long long items, int block, int nsm)
{
    long long g = (items + block - 1) / block;
    const long long cap = (long long)(nsm > 0 ? nsm : 1) * kHelperBlocksPerSm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// Grid of the statistics reduction (one partial-sum record per block).
inline int stats_grid(long long ncell, int block, int nsm)
{
    const int g = helper_grid(ncell, block, nsm);
    const int cap = (nsm > 0 ? nsm : 1) * kStatsBlocksPerSm;
    return g < cap ? g : cap;
}

// Doubles of the per-block partial sums the statistics of any field need on
// a device with nsm SMs.
inline size_t stats_partial_elems(int nsm)
{
    return (size_t)(nsm > 0 ? nsm : 1) * kStatsBlocksPerSm * kStatsSums;
}

// Device address of a file-scope __device__ array, cached per device and
// re-resolved whenever the device's current context is not the one the cached
// address was resolved in (after cudaDeviceReset the primary context -- and
// with it the module and the array -- is created anew).  ctx_id is the
// context's unique id; resolve(&addr) looks the address up in the current
// context and returns 0 on success.
template <int NDEV> struct ContextAddressCache {
    unsigned long long ctx[NDEV] = {};
    void *addr[NDEV] = {};

    template <typename Resolve> int get(int dev, unsigned long long ctx_id, Resolve &&resolve, void **out)
    {
        if (dev < 0 || dev >= NDEV || !out) return -1;
        if (!addr[dev] || ctx[dev] != ctx_id) {
            void *p = nullptr;
            const int rc = resolve(&p);
            if (rc != 0 || !p) {
                addr[dev] = nullptr;
                return rc != 0 ? rc : -1;
            }
            addr[dev] = p;
            ctx[dev] = ctx_id;
        }
        *out = addr[dev];
        return 0;
    }
};

} // namespace gks
