"""The zero-allocation time step, gks_timestep_noalloc.

It exists for callers that may not allocate device memory -- codes that own
and pool all device memory themselves, or loops that cannot afford
cudaMalloc's implicit synchronisation -- so here the five state arrays are the
caller's own (allocated by torch, not by this library).  Its answer must equal
the context entry point's (gks_timestep) exactly, the tolerance every dt test
here uses, on consecutive calls: the shared scratch must not carry anything
from one call into the next.  This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

import gks_ic

pytestmark = pytest.mark.gpu


def noalloc_dt(gks, arrays, nc, gam, cfl, stream=None):
    lib = gks.load_library()
    ptrs = (ctypes.c_void_p * 5)(*[a.data_ptr() for a in arrays])
    dt = ctypes.c_double(-1.0)
    rc = lib.gks_timestep_noalloc(ptrs, nc, gam, cfl, ctypes.c_void_p(stream) if stream else None,
                                  ctypes.byref(dt))
    return rc, dt.value


def test_noalloc_timestep_equals_context_timestep(gks):
    import torch

    torch.cuda.set_device(0)
    gks.select_device(0)
    # 24^3 and 40^3 launch 54 and 250 blocks; 64^3 exactly the 1024 the
    # scratch holds; 96^3 is capped at 1024 blocks with the grid-stride loop active
    cases = [gks_ic.make_dhit(24, k0=4.0, Mt=0.3, seed=21), gks_ic.make_dhit(40, k0=3.0, Mt=0.5, seed=22),
             gks_ic.make_dhit(64, k0=4.0, Mt=0.4, seed=23), gks_ic.make_dhit(96, k0=5.0, Mt=0.2, seed=24)]
    expected, arrays = [], []
    for case in cases:
        W = gks_ic.to_conservative_padded(case)
        with gks.Solver(gks.phys_from_case(case)) as s:
            s.upload(W)
            expected.append((s.timestep(0.5), s.timestep(0.02)))
        interior = np.ascontiguousarray(W[:, 3:-3, 3:-3, 3:-3])
        arrays.append([torch.from_numpy(interior[q].copy()).cuda() for q in range(5)])
    torch.cuda.synchronize()
    # two calls in a row on different fields, in both orders, and twice on the same field
    for order in ([0, 1], [1, 0], [1, 1], [3, 2, 0, 3], [2, 3, 1]):
        for i in order:
            for k, cfl in enumerate((0.5, 0.02)):
                rc, dt = noalloc_dt(gks, arrays[i], cases[i].nc, cases[i].gam, cfl)
                assert rc == 0
                assert dt == expected[i][k]
    # on a caller's own (non-default) stream
    side = torch.cuda.Stream()
    for i in (3, 0, 2):
        rc, dt = noalloc_dt(gks, arrays[i], cases[i].nc, cases[i].gam, 0.5, stream=side.cuda_stream)
        assert rc == 0
        assert dt == expected[i][0]


def test_noalloc_rejects_oversize_and_bad_arguments(gks):
    import torch

    a = [torch.zeros(8, dtype=torch.float64, device="cuda") for _ in range(5)]
    rc, _ = noalloc_dt(gks, a, 1025, 1.4, 0.5)
    assert rc == -6  # GKS_ETOOBIG: nc above the stated maximum of 1024
    rc, _ = noalloc_dt(gks, a, 16, 1.4, -1.0)
    assert rc == -1  # GKS_EINVAL
