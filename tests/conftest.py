"""Shared fixtures.  `-m gpu` tests need a CUDA device and call the CUDA
path through the C ABI (libffb200.so); the rest run on the CPU."""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fflame-rust_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def native():
    from ffb200 import _native
    return _native


@pytest.fixture(scope="session")
def renderer(native):
    r = native.Renderer(0)
    yield r
    r.close()
