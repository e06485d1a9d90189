"""CPU tests of the input generator (restating init_BS.m), the reference
file layouts, and the C ABI library's exported symbols (no GPU calls)."""

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

import gks_ic


def test_ic_is_solenoidal_and_scaled():
    case = gks_ic.make_dhit(24, k0=4.0, Mt=0.3, seed=3)
    q = np.sqrt(np.mean(case.u**2 + case.v**2 + case.w**2))
    assert q == pytest.approx(0.3, rel=1e-12)  # sound speed 1
    kf = np.fft.fftfreq(24, d=1.0 / 24)
    ky, kx, kz = np.meshgrid(kf, kf, kf, indexing="ij")
    div = kx * np.fft.fftn(case.u) + ky * np.fft.fftn(case.v) + kz * np.fft.fftn(case.w)
    # the Nyquist planes of an even grid are not representable exactly after taking the real part
    interior = (np.abs(kx) < 12) & (np.abs(ky) < 12) & (np.abs(kz) < 12)
    assert np.abs(div[interior]).max() < 1e-10 * np.abs(np.fft.fftn(case.u)).max()
    assert abs(np.mean(case.u)) < 1e-14


def test_ic_constants_follow_init_bs():
    case = gks_ic.make_dhit(16, k0=4.0, Mt=0.5, Re_lambda=100.0, seed=0)
    urms = 0.5 / np.sqrt(3.0)
    assert case.p0 == pytest.approx(1 / 1.4)
    assert case.mu0 == pytest.approx(urms * 0.5 / 100.0)
    assert case.t0 == pytest.approx(0.5 / urms)
    assert case.K == 2
    assert case.T0 == pytest.approx((1 / 1.4) / 287.0)


def test_ic_is_seeded():
    a = gks_ic.make_dhit(12, seed=5)
    b = gks_ic.make_dhit(12, seed=5)
    c = gks_ic.make_dhit(12, seed=6)
    assert np.array_equal(a.u, b.u) and not np.array_equal(a.u, c.u)


def test_ic_spectrum_shape():
    case = gks_ic.make_dhit(32, k0=4.0, seed=2)
    kf = np.fft.fftfreq(32, d=1.0 / 32)
    ky, kx, kz = np.meshgrid(kf, kf, kf, indexing="ij")
    shell = np.rint(np.sqrt(kx**2 + ky**2 + kz**2)).astype(int)
    e = sum(np.abs(np.fft.fftn(a)) ** 2 for a in (case.u, case.v, case.w))
    E = np.bincount(shell.ravel(), e.ravel())
    n = np.arange(len(E))
    target = n**4 * np.exp(-2 * n * n / 16.0)
    ratio = E[1:12] / target[1:12]
    assert np.allclose(ratio, ratio[0], rtol=1e-6)


def test_case_files_round_trip(tmp_path):
    case = gks_ic.make_dhit(8, seed=1)
    gks_ic.write_case(str(tmp_path), case)
    prm, W = gks_ic.read_init(str(tmp_path))
    assert prm["nc"] == 8 and prm["gam"] == 1.4 and prm["mu0"] == case.mu0
    ref = gks_ic.to_conservative_padded(case)
    assert np.array_equal(W, ref)
    raw = np.fromfile(str(tmp_path / "InitialConditions" / "Init000"), dtype="<f8")
    # MATLAB order J = k*ny*nx + i*ny + j (FlowField.cpp:95): the second value is u[j=1, i=0, k=0]
    assert raw[1] == case.u[1, 0, 0] and raw[8] == case.u[0, 1, 0] and raw[64] == case.u[0, 0, 1]


def test_slab_case_holds_first_planes(tmp_path):
    case = gks_ic.make_dhit(8, seed=1)
    gks_ic.write_case(str(tmp_path), case, slab_planes=2)
    raw = np.fromfile(str(tmp_path / "InitialConditions" / "Init000"), dtype="<f8")
    assert raw.size == 5 * 2 * 64


def test_all_slabs_tile_the_field(tmp_path):
    """Init<a>00 holds y-planes [2a, 2a+2): the slabs together are the whole field."""
    case = gks_ic.make_dhit(8, seed=1)
    gks_ic.write_case(str(tmp_path), case, slab_planes=2, all_slabs=True)
    for a in range(4):
        raw = np.fromfile(str(tmp_path / "InitialConditions" / f"Init{a}00"), dtype="<f8").reshape(5, 8, 8, 2)
        # file order: k slowest, then i, then j (FlowField.cpp:95)
        u = raw[0].transpose(2, 1, 0)
        assert np.array_equal(u, case.u[2 * a:2 * a + 2])
        assert np.array_equal(raw[3].transpose(2, 1, 0), case.rho[2 * a:2 * a + 2])


def _header_symbols():
    with open(os.path.join(ROOT, "include", "gks_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gks_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    path = os.path.join(ROOT, "gkm-dns_b200", "lib", "libgks_b200.so")
    assert os.path.exists(path), "build the library first (__graft_entry__.build())"
    lib = ctypes.CDLL(path)
    syms = _header_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s


def test_binding_declares_every_symbol():
    import gks_b200

    assert sorted(gks_b200.SIGNATURES) == _header_symbols()


def test_create_without_gpu_fails_cleanly(gks):
    """No device here: the product path must refuse, not fall back."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    case = gks_ic.make_dhit(8, seed=0)
    with pytest.raises(gks.GksError):
        gks.Solver(gks.phys_from_case(case))


def test_missing_library_raises(tmp_path):
    import gks_b200

    saved = gks_b200._lib
    gks_b200._lib = None
    try:
        with pytest.raises(ImportError):
            gks_b200.load_library(str(tmp_path / "nope.so"))
    finally:
        gks_b200._lib = saved
