"""Shared pytest setup: the ``gpu`` marker, import paths and library loading helpers."""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "photon-v2_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libphoton_gpu.so")


@pytest.fixture(scope="session")
def gpu_lib():
    """The loaded library on a machine with a GPU; GPU tests fail (not skip) without one."""
    import photon_gpu

    lib = photon_gpu.load()
    assert photon_gpu.device_count() > 0, "no CUDA device visible to libphoton_gpu.so"
    return lib
