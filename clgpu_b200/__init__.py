"""iclBLAS hot path for NVIDIA B200 (sm_100a).

The product is the shared library ``libiclblas_b200.so`` with the C ABI of
``include/iclBLAS.h``; ``clgpu_b200.iclblas`` is its Python binding.
"""
from . import iclblas  # noqa: F401
from .iclblas import Handle, IclblasError, lib  # noqa: F401

__all__ = ["iclblas", "Handle", "IclblasError", "lib"]
