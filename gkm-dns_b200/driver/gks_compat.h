// Drop-in for the reference's GPU call site.
//
// The reference's WENO driver calls, once per step,
//     void evolve(ptype *W[5], DevAlloc *dev, ptype dt);      weno/src/GPUupdate.h:33
// with a DevAlloc created once at the start of Evolve (update.cpp:58) and the
// grid / physics constants read from the globals of param.h.  This header
// provides the same two names on top of the gks_b200 C ABI: include it in
// place of "GPUupdate.h" and "GPUAlloc.h" (update.h:32-33), compile with
// -DUseGPU and link -lgks_b200.  The call site in update.cpp stays unchanged.
//
// Semantics: one periodic block per process (procDim 1x1x1; the kernels wrap
// the halo themselves), or one y-slab per rank of a field split along y
// (procDim = {P, 1, 1}: a gks_create_slab context of nc_segy planes from
// sta[0], whose y ghosts come from the caller's HaloTransfer as in the
// reference); decompositions along x or z are refused.  FP64 by default.
// Compile-time options:
//   GKS_COMPAT_MIXED          use the mixed FP32/FP64 path
//   GKS_COMPAT_GPU_SEMANTICS  reproduce the reference GPU kernel's choices
//                             (WENO on rho E, no 1/Pr factor) instead of the
//                             CPU path's (the parity default)
//   GKS_COMPAT_NO_PIN         leave the caller's W arrays pageable (by default
//                             the first evolve() page-locks them with
//                             cudaHostRegister, as the overlapped copies need,
//                             and ~DevAlloc releases them; the reference
//                             allocates W once per run, Main.cpp:36)
// As in the reference, evolve() uploads W, advances one step and downloads W
// (gks_evolve: for a whole periodic block the copies overlap the step slab by
// slab; with W in pinned host memory both PCIe directions and the step run
// concurrently); the downloaded x / z ghosts, and a whole block's y ghosts,
// already hold the periodic image, and the caller's HaloTransfer that follows
// refreshes a slab's y ghosts from its neighbours.
#pragma once

#include <cstdio>
#include <cstdlib>

#include "gks_b200.h"

static_assert(sizeof(ptype) == sizeof(double), "gks_b200 advances double-precision fields");

class DevAlloc
{
public:
    DevAlloc();
    ~DevAlloc()
    {
        unpin();
        gks_destroy(ctx);
    }
    DevAlloc(const DevAlloc &) = delete;
    DevAlloc &operator=(const DevAlloc &) = delete;
    gks_ctx *ctx = nullptr;
    // the host arrays page-locked by pin() (null: none)
    void *pinned[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    size_t pinned_bytes = 0;

    // Page-lock the five arrays of W (nt^3 doubles each) unless they already
    // are; a different W than last time replaces the earlier registration.
    void pin(ptype *W[5])
    {
#ifndef GKS_COMPAT_NO_PIN
        const size_t bytes = (size_t)Nt_seg * sizeof(ptype);
        bool same = bytes == pinned_bytes;
        for (int q = 0; q < 5 && same; ++q) same = pinned[q] == (void *)W[q];
        if (same) return;
        unpin();
        // one range when the five arrays lie one after another (then each slab
        // moves in one pitched copy per direction), else one per array; a
        // failure leaves W pageable: the copies still work, overlapping less
        bool block = true;
        for (int q = 1; q < 5 && block; ++q) block = W[q] == W[0] + (size_t)q * Nt_seg;
        int made = 0;
        if (block) {
            if (gks_host_register(W[0], 5 * bytes, &made) == GKS_OK && made) pinned[0] = W[0];
        } else {
            for (int q = 0; q < 5; ++q)
                if (gks_host_register(W[q], bytes, &made) == GKS_OK && made) pinned[q] = W[q];
        }
        pinned_bytes = bytes;
#else
        (void)W;
#endif
    }
    void unpin()
    {
        for (int q = 0; q < 5; ++q)
            if (pinned[q]) gks_host_unregister(pinned[q]);
        for (int q = 0; q < 5; ++q) pinned[q] = nullptr;
        pinned_bytes = 0;
    }
};

inline void gks_compat_check(gks_ctx *ctx, int rc, const char *what)
{
    if (rc == GKS_OK) return;
    fprintf(stderr, "gks_b200: %s failed (%d): %s\n", what, rc, gks_last_error(ctx));
    abort(); // the reference signature has no error return
}

inline DevAlloc::DevAlloc()
{
    // procDim[0] splits y (FlowField.cpp:22, segment() :282)
    const bool whole = procDim[0] == 1 && nc_segy == nc_segx;
    if (procDim[1] != 1 || procDim[2] != 1 || nc_segx != nc_segz || nc_segy * procDim[0] != nc_segx) {
        fprintf(stderr, "gks_b200: one periodic cube per process or a split along y only (procDim {P,1,1}) "
                        "is required\n");
        abort();
    }
    gks_phys p{};
    p.nc = nc_segx;
    p.K = K;
    p.visc_law = GKS_VISC_SUTHERLAND; // update.cpp:263
    p.gam = gam;
    p.gas_r = R;
    p.T0 = T0;
    p.mu0 = mu0;
    p.visc_exp = 0.76;
#ifdef GKS_COMPAT_GPU_SEMANTICS
    p.pr_factor = 1.0; // GPUupdate.cu:839
    const int flags = GKS_DIRECT_ENERGY;
#else
    p.pr_factor = 1 / 0.7; // GKMflux.cpp:289
    const int flags = 0;
#endif
    p.p0 = p0;
    p.den0 = den0;
    p.Mt = Mt;
    p.t0 = t0;
#ifdef GKS_COMPAT_MIXED
    const int precision = GKS_MIXED;
#else
    const int precision = GKS_FP64;
#endif
    if (whole) gks_compat_check(nullptr, gks_create(&ctx, 1, &p, precision, flags), "gks_create");
    else gks_compat_check(nullptr, gks_create_slab(&ctx, &p, nc_segy, sta[0], precision, flags), "gks_create_slab");
}

inline void evolve(ptype *W[5], DevAlloc *dev, ptype dt)
{
    dev->pin(W);
    gks_compat_check(dev->ctx, gks_set_dt(dev->ctx, 0, dt), "gks_set_dt");
    gks_compat_check(dev->ctx, gks_evolve(dev->ctx, 0, W, 1), "gks_evolve");
    gks_compat_check(dev->ctx, gks_sync(dev->ctx), "gks_sync");
}
