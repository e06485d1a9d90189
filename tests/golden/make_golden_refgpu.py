"""Golden fixtures from the reference's own GPU path (needs a GPU).

Runs oracle/_ref/ref_gpu_harness -- the reference's GPUupdate.cu and
GPUAlloc.cu with update.cpp -DUseGPU, built for sm_100a by oracle/Makefile,
driven by the same harness as the CPU fixtures -- on the seeded inputs of
make_golden.py.  The reference's GPU path reconstructs the five conservative
components directly (GPUupdate.cu:917-977) and has no 1/Pr factor in its
slope solver (GPUupdate.cu:836-851); everything else is the CPU path's
algorithm.  The harness binary is built where the reference sources are; this
script only runs it, so it can run on any machine that has the built binary
and a GPU.

    python tests/golden/make_golden_refgpu.py [outdir]      (default: tests/golden)

Fixtures
  refgpu16.npz   16^3 DHIT (seed 1, as dhit16.npz): fields after 1 and 10
                 steps, stats history
  refgpu32.npz   32^3 DHIT (k0 4, Mt 0.3, Re 72, seed 0, CFL 0.5, as dhit32.npz):
                 step-10 field checksums and 4096 sampled cells, stats history
"""

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gkm-dns_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import gks_ic  # noqa: E402
import pyoracle  # noqa: E402


def run(nc, seed, nsteps, dumps):
    case = gks_ic.make_dhit(nc, k0=4.0, Mt=0.3, Re_lambda=72.0, seed=seed)
    d = tempfile.mkdtemp(prefix=f"refgpu{nc}_")
    gks_ic.write_case(d, case)
    return case, pyoracle.ref_run(d, nsteps, 0.5, dumps, gpu=True)


def interior(W):
    return np.ascontiguousarray(W[:, 3:-3, 3:-3, 3:-3])


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(out, exist_ok=True)
    if not pyoracle.have_ref_gpu():
        sys.exit("oracle/_ref/ref_gpu_harness is missing: run make in oracle/ where the reference sources are")

    case, r = run(16, 1, 10, [1, 10])
    np.savez_compressed(
        os.path.join(out, "refgpu16.npz"), w1=interior(r["dumps"][1]), w10=interior(r["dumps"][10]),
        stats=r["stats"], dt=r["meta"]["dt"], lines=np.array(r["stdout"]), seed=1, nc=16)

    case, r = run(32, 0, 10, [10])
    w10 = interior(r["dumps"][10])
    srng = np.random.default_rng(7)
    sample = srng.integers(0, 32**3, 4096)
    flat = w10.reshape(5, -1)
    np.savez_compressed(
        os.path.join(out, "refgpu32.npz"), stats=r["stats"], dt=r["meta"]["dt"], sample_idx=sample,
        sample_w10=flat[:, sample], sum_w10=flat.sum(1), sumsq_w10=(flat * flat).sum(1), seed=0, nc=32)
    for fn in ("refgpu16.npz", "refgpu32.npz"):
        print(fn, os.path.getsize(os.path.join(out, fn)))


if __name__ == "__main__":
    main()
