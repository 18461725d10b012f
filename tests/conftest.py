"""Shared fixtures: library loading and run set-ups for the parity tests."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "rast-3dmhd_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_built():
    if not os.path.exists(os.path.join(PKG, "libmhd3d_host.so")):
        subprocess.run(["make", "-s", "-C", PKG, "host"], check=True)
    if not os.path.exists(os.path.join(ORACLE, "liboracle3dmhd.so")):
        subprocess.run(["make", "-s", "-C", ORACLE], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def mhd3d():
    import mhd3d as m
    return m


@pytest.fixture(scope="session")
def oracle():
    import oracle_py
    return oracle_py
