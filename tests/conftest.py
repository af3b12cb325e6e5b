"""Shared pytest configuration for the dense plane-sweep tests.

Tests marked ``gpu`` need a CUDA device and the built CUDA library; every
other test runs on the CPU (the oracle, host logic, ABI checks).
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "video-to-3d_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "_build", "liboracle_v3d.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                       stdout=subprocess.DEVNULL)
    return lib


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (test infrastructure), loaded through ctypes."""
    _ensure_oracle()
    from tests import oracle_ffi
    return oracle_ffi.Oracle()
