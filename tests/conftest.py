"""Test configuration: the `gpu` marker and shared fixtures.

Tests marked `gpu` need a CUDA device (a B200) and call the library through
its C ABI; everything else runs on the CPU: the oracle against the
reference's own CPU code and golden vectors, the C-ABI library's exports and
its host-side argument checks.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls the library through its C ABI")


def _ensure_library():
    lib = os.path.join(ROOT, "clgpu_b200", "libiclblas_b200.so")
    if not os.path.exists(lib):
        from clgpu_b200 import build as b
        b.build_library()
    return lib


@pytest.fixture(scope="session")
def libpath():
    return _ensure_library()


@pytest.fixture(scope="session")
def cuda():
    """The GPU tests fail (not skip) without a device: a silent skip would
    hide a broken GPU run."""
    import torch
    assert torch.cuda.is_available(), "gpu-marked test needs a CUDA device"
    _ensure_library()
    return torch.device("cuda:0")


@pytest.fixture()
def handle(cuda):
    from clgpu_b200 import iclblas as B
    h = B.Handle()
    yield h
    h.destroy()
