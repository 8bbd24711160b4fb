"""Shared pytest set-up: the `gpu` marker, import paths, and the two builds of the library.

`cuda_library` is the product: libgbght.so compiled by nvcc for sm_100a. `hostcheck_library` is a
test-only build of the same kernel bodies and C ABI with the host C++ compiler, in which every
launch runs block by block on one CPU thread. The CPU suite uses it to check the kernels' index
arithmetic against the oracle; no product path loads it.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gbghomogeneousturbulence.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def cuda_library():
    import gbght_build
    return gbght_build.build()


@pytest.fixture(scope="session")
def hostcheck_library():
    import gbght_build
    return gbght_build.build_hostcheck()
