"""gks_evolve, the reference's per-step call on host memory (evolve(W, dev,
dt), GPUupdate.h:33): the slab-pipelined form (one field, one step: copies in
y-slabs overlapping the step) must give exactly what gks_upload + gks_step(1)
+ gks_download give, for any field size (slabs that do not divide the
field, the smallest pipelined size, odd sizes), both precisions, pageable and
pinned host memory; the state it leaves resident must continue exactly; the
other forms (ensembles, several steps) fall back to the plain sequence."""

import numpy as np
import pytest

import gks_ic

pytestmark = pytest.mark.gpu


def plain(gks, case, W, prec, dt, nsteps=1, flags=0):
    with gks.Solver(gks.phys_from_case(case), prec, flags) as s:
        s.upload(W)
        s.set_dt(dt)
        s.step(nsteps)
        s.sync()
        return s.download()


@pytest.mark.parametrize("nc", [16, 19, 40, 64, 100, 130])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_pipelined_evolve_equals_upload_step_download(gks, nc, prec):
    case = gks_ic.make_dhit(nc, k0=4.0, Mt=0.4, Re_lambda=80.0, seed=nc)
    W0 = gks_ic.to_conservative_padded(case)
    p = gks.FP64 if prec == "fp64" else gks.MIXED
    with gks.Solver(gks.phys_from_case(case), p) as s:
        s.upload(W0)
        dt = s.timestep(0.5)
        ref1 = plain(gks, case, W0, p, dt)
        ref2 = plain(gks, case, ref1, p, dt)
        W = W0.copy()
        s.evolve(W)
        assert np.array_equal(W, ref1)
        s.evolve(W)  # a second call: the buffers swapped by the first are reused
        assert np.array_equal(W, ref2)
        s.sync()
        # the resident state continues exactly (graph steps after the pipelined ones)
        s.step(1)
        s.sync()
        ref3 = plain(gks, case, ref2, p, dt)
        assert np.array_equal(s.download(), ref3)
        # and a pipelined call after graph steps
        W3 = ref3.copy()
        s.evolve(W3)
        assert np.array_equal(W3, plain(gks, case, ref3, p, dt))


def test_pipelined_evolve_from_pinned_memory_and_variants(gks):
    import torch

    nc = 48
    case = gks_ic.make_dhit(nc, k0=3.0, Mt=0.5, seed=3)
    W0 = gks_ic.to_conservative_padded(case)
    for flags in (0, gks.FIX_ZSWEEP | gks.DIRECT_ENERGY):
        with gks.Solver(gks.phys_from_case(case), gks.FP64, flags) as s:
            s.upload(W0)
            dt = s.timestep(0.5)
            host = torch.empty(W0.shape, dtype=torch.float64, pin_memory=True).numpy()
            host[...] = W0
            s.evolve(host)
            assert np.array_equal(host, plain(gks, case, W0, gks.FP64, dt, flags=flags))


def test_evolve_fallbacks_and_errors(gks):
    cases = [gks_ic.make_dhit(n, k0=4.0, Mt=0.3, seed=n) for n in (12, 20)]
    Ws = [gks_ic.to_conservative_padded(c) for c in cases]
    # several steps in one call
    with gks.Solver(gks.phys_from_case(cases[1])) as s:
        s.upload(Ws[1])
        dt = s.timestep(0.5)
        W = Ws[1].copy()
        s.evolve(W, nsteps=3)
        assert np.array_equal(W, plain(gks, cases[1], Ws[1], gks.FP64, dt, 3))
        with pytest.raises(gks.GksError) as ei:
            s.evolve(W, nsteps=0)
        assert ei.value.code == -1
    # an ensemble: one field's call advances every field of the context
    with gks.Solver([gks.phys_from_case(c) for c in cases]) as s:
        dts = []
        for f, (c, w) in enumerate(zip(cases, Ws)):
            s.upload(w, f)
            dts.append(s.timestep(0.5, f))
        W = Ws[0].copy()
        s.evolve(W, f=0)
        assert np.array_equal(W, plain(gks, cases[0], Ws[0], gks.FP64, dts[0]))
        assert np.array_equal(s.download(1), plain(gks, cases[1], Ws[1], gks.FP64, dts[1]))
    # dt must be set first
    with gks.Solver(gks.phys_from_case(cases[1])) as s:
        with pytest.raises(gks.GksError) as ei:
            s.evolve(Ws[1].copy())
        assert ei.value.code == -4


def test_host_register_pins_a_pageable_field(gks):
    """gks_host_register page-locks caller memory (reporting whether it did),
    leaves already pinned memory alone, and evolve gives the same answer on
    the registered array."""
    import ctypes

    lib = gks.load_library()
    nc = 24
    case = gks_ic.make_dhit(nc, k0=4.0, Mt=0.4, seed=7)
    W0 = gks_ic.to_conservative_padded(case)
    W = W0.copy()
    made = ctypes.c_int(-1)
    ptrs = [W[q].ctypes.data for q in range(5)]
    for p in ptrs:
        assert lib.gks_host_register(ctypes.c_void_p(p), W[0].nbytes, ctypes.byref(made)) == 0
        assert made.value == 1
    assert lib.gks_host_register(ctypes.c_void_p(ptrs[0]), W[0].nbytes, ctypes.byref(made)) == 0
    assert made.value == 0  # already page-locked: nothing done
    try:
        with gks.Solver(gks.phys_from_case(case)) as s:
            s.upload(W0)
            dt = s.timestep(0.5)
            s.evolve(W)
        assert np.array_equal(W, plain(gks, case, W0, gks.FP64, dt))
    finally:
        for p in ptrs:
            assert lib.gks_host_unregister(ctypes.c_void_p(p)) == 0
    assert lib.gks_host_register(None, 8, None) == -1


def test_evolve_with_separate_component_arrays(gks):
    """The five host arrays need not be one block: separately allocated
    components take one copy per component and slab instead of one pitched
    copy, with the same result."""
    import ctypes

    nc = 40
    case = gks_ic.make_dhit(nc, k0=4.0, Mt=0.4, seed=11)
    W0 = gks_ic.to_conservative_padded(case)
    comps = [np.ascontiguousarray(W0[q]).copy() for q in range(5)]  # five separate allocations
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(W0)
        dt = s.timestep(0.5)
        ptrs = gks.DP5(*[c.ctypes.data_as(gks.DP) for c in comps])
        rc = gks.load_library().gks_evolve(s._h, 0, ptrs, 1)
        assert rc == 0
    assert np.array_equal(np.stack(comps), plain(gks, case, W0, gks.FP64, dt))
