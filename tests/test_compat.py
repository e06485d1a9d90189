"""The reference call-site shim (gkm-dns_b200/driver/gks_compat.h) and the
drop-in driver (gks_dns) against the reference's file formats."""

import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT

import gks_ic

COMPAT_SRC = os.path.join(ROOT, "tests", "compat", "compat_main.cpp")


def build_compat(out):
    cmd = ["g++", "-O2", "-std=c++17", f"-I{ROOT}/include", f"-I{PKG}/driver", COMPAT_SRC, "-o", out,
           f"-L{PKG}/lib", "-lgks_b200", f"-Wl,-rpath,{PKG}/lib"]
    subprocess.run(cmd, check=True)


def test_compat_header_compiles(tmp_path):
    build_compat(str(tmp_path / "compat_main"))


def test_driver_rejects_missing_case(tmp_path):
    exe = os.path.join(PKG, "driver", "gks_dns")
    assert os.path.exists(exe)
    r = subprocess.run([exe, "--case", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 2 and "cannot open" in r.stderr


def test_driver_rejects_short_init(tmp_path):
    case = gks_ic.make_dhit(8, seed=0)
    gks_ic.write_case(str(tmp_path), case)
    p = tmp_path / "InitialConditions" / "Init000"
    p.write_bytes(p.read_bytes()[:1000])
    r = subprocess.run([os.path.join(PKG, "driver", "gks_dns"), "--case", str(tmp_path)], capture_output=True,
                       text=True)
    assert r.returncode == 2 and "shorter" in r.stderr


@pytest.mark.gpu
def test_compat_evolve_matches_solver(tmp_path, gks):
    case = gks_ic.make_dhit(16, k0=4.0, Mt=0.3, seed=5)
    W = gks_ic.to_conservative_padded(case)
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(W)
        dt = s.timestep(0.5)
        s.step(3)
        s.sync()
        ref = s.download()
    exe = str(tmp_path / "compat_main")
    build_compat(exe)
    W.tofile(str(tmp_path / "in.bin"))
    subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), "16", repr(dt), "3", repr(case.gam),
                    repr(case.mu0), repr(case.p0), "1.0", repr(case.Mt), repr(case.t0)], check=True)
    got = np.fromfile(str(tmp_path / "out.bin")).reshape(W.shape)
    assert np.array_equal(got, ref)


@pytest.mark.gpu
def test_compat_evolve_on_y_split_ranks(tmp_path, gks):
    """The shim under the reference's y decomposition (procDim = {2, 1, 1}):
    each rank's evolve(W, dev, dt) advances its slab block, whose y ghosts the
    caller's HaloTransfer refreshes between steps (here: merged and split
    again on the host); two steps equal the whole field's."""
    import gks_slabs

    case = gks_ic.make_dhit(16, k0=4.0, Mt=0.3, seed=6)
    W = gks_ic.to_conservative_padded(case)
    with gks.Solver(gks.phys_from_case(case)) as s:
        s.upload(W)
        dt = s.timestep(0.5)
        s.step(2)
        s.sync()
        ref = s.download()
    exe = str(tmp_path / "compat_main")
    build_compat(exe)
    cur = W
    for step in range(2):
        blocks = []
        for r in range(2):
            b = gks_slabs.split_block(cur, 2, r)
            b.tofile(str(tmp_path / "in.bin"))
            subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), "16", repr(dt), "1",
                            repr(case.gam), repr(case.mu0), repr(case.p0), "1.0", repr(case.Mt), repr(case.t0),
                            "2", str(r)], check=True)
            blocks.append(np.fromfile(str(tmp_path / "out.bin")).reshape(b.shape))
        cur = gks_slabs.merge_blocks(blocks)  # HaloTransfer
    assert np.array_equal(cur, ref)


@pytest.mark.gpu
def test_driver_prints_reference_lines(tmp_path, oracle):
    """gks_dns on the 16^3 golden case prints the reference's statistics lines."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "dhit16.npz"))
    case = gks_ic.make_dhit(16, seed=1)
    gks_ic.write_case(str(tmp_path), case)
    r = subprocess.run([os.path.join(PKG, "driver", "gks_dns"), "--case", str(tmp_path), "--cfl", "0.5",
                        "--steps", "10", "--reinit", str(tmp_path / "final")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip() and ln.strip()[0].isdigit()]
    ref = [str(x) for x in g["lines"]]
    assert len(lines) == 11 and len(ref) == 11
    for a, b in zip(lines, ref):
        va = [float(x) for x in a.split()]
        vb = [float(x) for x in b.split()]
        # columns 9-11 (p, T, 1/rho rms, O(0.1) once the flow develops) are pure
        # round-off at t = 0, where pressure and density are uniform
        np.testing.assert_allclose(va, vb, rtol=2e-8, atol=1e-10)
        assert a.count("  ") == b.count("  ")
    # the reinit file holds the final state in the Init layout
    raw = np.fromfile(str(tmp_path / "final"))
    assert raw.size == 5 * 16**3
    u = raw[:16**3].reshape(16, 16, 16).transpose(2, 1, 0)
    w10 = g["w10"]
    np.testing.assert_allclose(u, w10[1] / w10[0], rtol=0, atol=1e-12)


FIELD_LINE = r"^-?\d+ -?\d+ -?\d+( -?\d\.\d{15}e[+-]\d{2}){5}$"


def parse_field(text: str):
    rows = [ln.split() for ln in text.splitlines()]
    ijk = np.array([[int(x) for x in r[:3]] for r in rows])
    vals = np.array([[float(x) for x in r[3:]] for r in rows])
    return ijk, vals


def test_field_golden_is_the_oracle_dump(oracle):
    """The Results/Field golden (the reference's writeField after 13 steps of
    the 8^3 case) equals, byte for byte, the same dump formatted from the
    oracle's state: it pins the fixture on the CPU."""
    import re

    g = np.load(os.path.join(ROOT, "tests", "golden", "field8.npz"))
    text = g["text"].tobytes().decode()
    case = gks_ic.make_dhit(8, seed=1)
    W = gks_ic.to_conservative_padded(case)
    prm = oracle.params(8, case.gam, case.mu0, case.p0, 1.0, case.Mt, case.t0)
    dt = 0.5 * (2 * np.pi / 8) / oracle.maxval(W, prm)
    assert dt == float(g["dt"])
    # writeField runs at the first step with t >= t0 (update.cpp:126-129), before that step
    t, n = 0.0, 0
    while not t >= case.t0:
        t += dt
        n += 1
    assert str(g["name"]) == f"Field_0_{n + 1}" and int(g["nsteps"]) == n + 1
    oracle.step(W, prm, dt, n)
    lines = []
    gam = case.gam
    for j in range(8):
        for i in range(8):
            for k in range(8):
                w = W[:, j + 3, i + 3, k + 3]
                d = w[0]
                u, v, ww = w[1] / d, w[2] / d, w[3] / d
                vsq = u * u + v * v + ww * ww
                p = (d * (gam - 1)) * (w[4] / d - 0.5 * vsq)
                lines.append("%d %d %d %.15e %.15e %.15e %.15e %.15e" % (i, j, k, d, u, v, ww, p))
    assert "\n".join(lines) + "\n" == text
    assert all(re.match(FIELD_LINE, ln) for ln in lines)


@pytest.mark.gpu
def test_driver_writes_reference_field(tmp_path):
    """gks_dns writes the reference's Results/Field dump (writeField,
    update.cpp:1305-1319): same file name (rank, iteration), same line layout
    and number format, the same cells in the same order, and primitives equal
    to the reference's to 1e-12 relative to each column's scale."""
    import re

    g = np.load(os.path.join(ROOT, "tests", "golden", "field8.npz"))
    ref_text = g["text"].tobytes().decode()
    case = gks_ic.make_dhit(8, seed=1)
    gks_ic.write_case(str(tmp_path), case)
    r = subprocess.run([os.path.join(PKG, "driver", "gks_dns"), "--case", str(tmp_path), "--cfl", "0.5",
                        "--steps", str(int(g["nsteps"]))], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    fdir = tmp_path / "Results" / "Field"
    assert sorted(os.listdir(fdir)) == [str(g["name"])]
    text = (fdir / str(g["name"])).read_text()
    lines = text.splitlines()
    assert len(lines) == 8**3 and text.endswith("\n")
    assert all(re.match(FIELD_LINE, ln) for ln in lines)
    ijk, vals = parse_field(text)
    rijk, rvals = parse_field(ref_text)
    assert np.array_equal(ijk, rijk)
    scale = np.abs(rvals).max(0)
    assert np.all(np.abs(vals - rvals).max(0) <= 1e-12 * scale), np.abs(vals - rvals).max(0) / scale


def test_driver_particles_need_their_inputs(tmp_path):
    """--particles reads numparticles from particleCount and the positions from
    unirand; a case without them is refused before any device work."""
    exe = os.path.join(PKG, "driver", "gks_dns")
    case = gks_ic.make_dhit(8, seed=2)
    gks_ic.write_case(str(tmp_path), case)  # particleCount 0, no unirand
    r = subprocess.run([exe, "--case", str(tmp_path), "--particles"], capture_output=True, text=True)
    assert r.returncode == 2 and "no particles" in r.stderr
    gks_ic.write_case(str(tmp_path), case, particles=10)
    with open(tmp_path / "InitialConditions" / "unirand", "r+b") as f:
        f.truncate(8 * 25)  # fewer than 3 x 10 doubles
    r = subprocess.run([exe, "--case", str(tmp_path), "--particles"], capture_output=True, text=True)
    assert r.returncode == 2 and "shorter" in r.stderr
    pos = np.fromfile(str(tmp_path / "InitialConditions" / "unirand"))
    assert pos.size == 25 and np.all((pos >= 0) & (pos < 2 * np.pi))
