"""Shared fixtures and paths for the gks_b200 tests.

Markers: ``gpu`` tests need a CUDA device (run on a B200); everything else
runs on the CPU.  The oracle (oracle/) is imported here only as the checker.
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gkm-dns_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle

    pyoracle.lib()
    return pyoracle


@pytest.fixture(scope="session")
def gks():
    import gks_b200

    gks_b200.load_library()
    return gks_b200
