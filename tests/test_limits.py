"""Launch-size limits derived from the device's SM count, and the per-context
scratch-address cache of the zero-allocation entry point, checked on the CPU
by compiling gkm-dns_b200/csrc/gks_limits.h into a small C++ program
(tests/native/limits_check.cpp)."""

import os
import subprocess

from conftest import PKG, ROOT


def test_limits_hold_for_any_sm_count(tmp_path):
    exe = str(tmp_path / "limits_check")
    subprocess.run(["g++", "-O1", "-std=c++17", f"-I{PKG}/csrc", os.path.join(ROOT, "tests", "native", "limits_check.cpp"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"
