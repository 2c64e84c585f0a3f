"""The precision studies measure errors against FP64 products and solves
computed by torch on the GPU (cuBLAS / cuSOLVER in float64).  These tests tie
that FP64 reference to the reference's own arithmetic on fixed samples at the
configs' depth: a 64 x 64 block of an 8192-deep GEMM against the reference's
cpu_gemm in double (tests/blas_funcs/test_gemm.hpp, compiled in oracle/_ref)
and the oracle's double GEMM; 64 right-hand sides of the 8192 x 8192 STRSM
config against the oracle's double TRSM (the restatement of Strsm_naive.cl).
Agreement is required to 1e-12 relative (max-norm)."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle_lib as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_gemm_sample_k8192(cuda):
    K = 8192
    rng = np.random.default_rng(2)
    # op(A) rows 0..63 and B columns 0..63 of the 8192^3 config, FP32 values
    A = rng.uniform(-1, 1, (64, K)).astype(np.float32).astype(np.float64)
    Bm = rng.uniform(-1, 1, (K, 64)).astype(np.float32).astype(np.float64)
    A[:, ::7] *= 10.0 ** rng.uniform(-4, 4, A[:, ::7].shape)   # a spread of magnitudes
    got = (torch.from_numpy(A).to(cuda) @ torch.from_numpy(Bm).to(cuda)).cpu().numpy()
    Acm = np.asfortranarray(A).reshape(-1, order="F")
    Bcm = np.asfortranarray(Bm).reshape(-1, order="F")
    Cd = np.zeros(64 * 64)
    O.dgemm(0, 0, 64, 64, K, 1.0, Acm, 64, Bcm, K, 0.0, Cd, 64)
    assert _rel(got, Cd.reshape(64, 64, order="F")) <= 1e-12
    R = O.ref()
    if R is not None:
        Cr = np.zeros(64 * 64)
        R.ref_cpu_dgemm(0, 0, 64, 64, K, 1.0, Acm.ctypes.data, 64, Bcm.ctypes.data, K, 0.0, Cr.ctypes.data, 64)
        assert _rel(got, Cr.reshape(64, 64, order="F")) <= 1e-12


def test_trsm_sample_m8192(cuda):
    M = 8192
    g = torch.Generator(device=cuda).manual_seed(3)
    L = torch.tril(torch.randn(M, M, generator=g, device=cuda) / M ** 0.5, -1)
    L = L + torch.diag(torch.rand(M, generator=g, device=cuda) + 1.0)
    Bm = torch.rand(64, M, generator=g, device=cuda) * 2 - 1     # 64 right-hand sides (FP32)
    X = torch.linalg.solve_triangular(L.double(), Bm.t().double(), upper=False).cpu().numpy()
    Lcm = L.t().contiguous().cpu().numpy().astype(np.float64).reshape(-1)   # column-major
    Xo = Bm.cpu().numpy().astype(np.float64).reshape(-1)                    # column-major M x 64
    O.dtrsm(0, 1, 0, 0, M, 64, 1.0, Lcm, M, Xo, M)
    assert _rel(X, Xo.reshape(64, M).T) <= 1e-12
