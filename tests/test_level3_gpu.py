"""Level-3 parity on the GPU (GEMM, TRSM; float and complex) against the oracle.

SGEMM in the plain FP32 mode is bit-exact with the oracle, which restates the
reference's FP32 FMA order (each output sums k in order with fused
multiply-adds).  CGEMM / TRSM: relative Frobenius error <= 1e-5 against the
oracle (FP64 arithmetic).
"""
import numpy as np
import pytest

import oracle_lib as O
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _shape(op, rows, cols):
    """(stored rows, stored cols) of an operand whose op(X) is rows x cols."""
    return (rows, cols) if op == 0 else (cols, rows)


@pytest.mark.parametrize("ta", [0, 1, 2])
@pytest.mark.parametrize("tb", [0, 1, 2])
@pytest.mark.parametrize("mnk", [(1, 1, 1), (5, 7, 3), (64, 64, 64), (129, 65, 33), (300, 257, 190)])
@pytest.mark.parametrize("beta", [0.0, 0.5])
def test_sgemm_bit_exact(handle, ta, tb, mnk, beta):
    m, n, k = mnk
    rng = np.random.default_rng(m + 3 * n + 7 * k + 11 * ta + 13 * tb)
    ar, ac = _shape(ta, m, k)
    br, bc = _shape(tb, k, n)
    lda, ldb, ldc = ar + 1, br + 2, m + 3
    A = O.colmajor(ar, ac, lda, rng)
    Bm = O.colmajor(br, bc, ldb, rng)
    Cm = O.colmajor(m, n, ldc, rng)
    if beta == 0.0:
        Cm.reshape(n, ldc)[:, :m] = np.nan  # C must not be read
    C_ref = Cm.copy()
    O.sgemm(ta, tb, m, n, k, 1.5, A, lda, Bm, ldb, beta, C_ref, ldc)
    assert B.iclblasSgemm(handle, ta, tb, m, n, k, 1.5, A, lda, Bm, ldb, beta, Cm, ldc) == B.SUCCESS
    assert np.array_equal(Cm, C_ref, equal_nan=True)


def test_sgemm_config_512(handle):
    """Plain SGEMM config: NN, 512^3, lda=ldb=ldc=512, alpha=1.5, beta=0.5,
    U(-1,1) from seed 0; <= 1e-5 relative Frobenius error against the
    reference's double-accumulating cpu_gemm, and bit-exact with the oracle."""
    n = 512
    rng = np.random.default_rng(0)
    A = rng.uniform(-1, 1, n * n).astype(np.float32)
    Bm = rng.uniform(-1, 1, n * n).astype(np.float32)
    Cm = rng.uniform(-1, 1, n * n).astype(np.float32)
    C_ref = Cm.copy()
    O.sgemm(0, 0, n, n, n, 1.5, A, n, Bm, n, 0.5, C_ref, n)
    C_dbl = Cm.astype(np.float64)
    O.dgemm(0, 0, n, n, n, 1.5, A.astype(np.float64), n, Bm.astype(np.float64), n, 0.5, C_dbl, n)
    assert B.iclblasSgemm(handle, 0, 0, n, n, n, 1.5, A, n, Bm, n, 0.5, Cm, n) == B.SUCCESS
    assert np.array_equal(Cm, C_ref)
    assert O.rel_fro(Cm, C_dbl) <= TOL


def test_sgemm_quarter_integers_exact(handle):
    """The reference's blas_funcs GEMM test values (0.25*UniformInt[-4,4]) at
    256^3 are exact in FP32: the result equals the double computation."""
    n = 256
    rng = np.random.default_rng(2)
    A = O.quarter_ints(n * n, rng)
    Bm = O.quarter_ints(n * n, rng)
    Cm = O.quarter_ints(n * n, rng)
    C_dbl = Cm.astype(np.float64)
    O.dgemm(0, 1, n, n, n, 0.5, A.astype(np.float64), n, Bm.astype(np.float64), n, -1.0, C_dbl, n)
    assert B.iclblasSgemm(handle, 0, 1, n, n, n, 0.5, A, n, Bm, n, -1.0, Cm, n) == B.SUCCESS
    assert np.array_equal(Cm.astype(np.float64), C_dbl)


def test_sgemm_k0_and_alpha0(handle):
    m, n = 33, 17
    rng = np.random.default_rng(4)
    Cm = rng.uniform(-1, 1, m * n).astype(np.float32)
    A = np.ones(m, np.float32)
    C_ref = Cm.copy()
    O.sgemm(0, 0, m, n, 0, 2.0, A, m, A, 1, 0.25, C_ref, m)
    assert B.iclblasSgemm(handle, 0, 0, m, n, 0, 2.0, A, m, A, 1, 0.25, Cm, m) == B.SUCCESS
    assert np.array_equal(Cm, C_ref)


@pytest.mark.parametrize("ta", [0, 1, 2])
@pytest.mark.parametrize("tb", [0, 2])
@pytest.mark.parametrize("mnk", [(1, 1, 1), (17, 9, 5), (100, 70, 129)])
def test_cgemm(handle, ta, tb, mnk):
    m, n, k = mnk
    rng = np.random.default_rng(m + n + k + ta * 5 + tb)
    ar, ac = _shape(ta, m, k)
    br, bc = _shape(tb, k, n)
    A = O.colmajor(ar, ac, ar + 1, rng, np.complex64)
    Bm = O.colmajor(br, bc, br, rng, np.complex64)
    for beta in (0.0, 0.5 + 0.5j):
        Cm = O.colmajor(m, n, m, rng, np.complex64)
        C_ref = Cm.copy()
        O.cgemm(ta, tb, m, n, k, 1 - 2j, A, ar + 1, Bm, br, beta, C_ref, m)
        assert B.iclblasCgemm(handle, ta, tb, m, n, k, 1 - 2j, A, ar + 1, Bm, br, beta, Cm, m) == B.SUCCESS
        assert O.rel_fro(Cm, C_ref) <= TOL


def tri(n, lda, lower, rng, dtype=np.float32):
    A = O.colmajor(n, n, lda, rng, dtype)
    M = A.reshape(n, lda).T[:n]  # view: M[i, j] = A[j*lda + i]
    d = rng.uniform(1, 2, n)
    if np.dtype(dtype) == np.complex64:
        d = d * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    off = (rng.standard_normal((n, n)) / np.sqrt(n)).astype(np.float32)
    mask = np.tril(np.ones((n, n), bool), -1) if lower else np.triu(np.ones((n, n), bool), 1)
    M[mask] = off[mask]
    M[np.arange(n), np.arange(n)] = d
    return A


@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("diag", [0, 1])
@pytest.mark.parametrize("mn", [(1, 1), (40, 13), (150, 97)])
def test_strsm(handle, side, uplo, trans, diag, mn):
    m, n = mn
    rng = np.random.default_rng(m + n + 2 * side + 4 * uplo + 8 * trans + 16 * diag)
    na = m if side == 0 else n
    A = tri(na, na + 1, uplo == 1, rng)
    Bm = O.colmajor(m, n, m + 2, rng)
    B_ref = Bm.copy()
    O.strsm(side, uplo, trans, diag, m, n, -1.25, A, na + 1, B_ref, m + 2)
    assert B.iclblasStrsm(handle, side, uplo, trans, diag, m, n, -1.25, A, na + 1, Bm, m + 2) == B.SUCCESS
    assert O.rel_fro(Bm, B_ref) <= TOL


@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_ctrsm(handle, side, uplo, trans):
    m, n = 70, 45
    rng = np.random.default_rng(side + 2 * uplo + 4 * trans)
    na = m if side == 0 else n
    A = tri(na, na, uplo == 1, rng, np.complex64)
    for diag in (0, 1):
        Bm = O.colmajor(m, n, m, rng, np.complex64)
        B_ref = Bm.copy()
        O.ctrsm(side, uplo, trans, diag, m, n, 0.5 + 1j, A, na, B_ref, m)
        assert B.iclblasCtrsm(handle, side, uplo, trans, diag, m, n, 0.5 + 1j, A, na, Bm, m) == B.SUCCESS
        assert O.rel_fro(Bm, B_ref) <= TOL


def test_strsm_large_left_lower(handle):
    """STRSM config shape at reduced RHS (the oracle solve is O(M^2 N)):
    M = 2048, NRHS = 256, L with diagonal U(1,2) and N(0,1)/sqrt(M) below."""
    m, n = 2048, 256
    rng = np.random.default_rng(3)
    A = tri(m, m, True, rng)
    Bm = rng.uniform(-1, 1, m * n).astype(np.float32)
    B_ref = Bm.copy()
    O.strsm(0, 1, 0, 0, m, n, 1.0, A, m, B_ref, m)
    assert B.iclblasStrsm(handle, 0, 1, 0, 0, m, n, 1.0, A, m, Bm, m) == B.SUCCESS
    assert O.rel_fro(Bm, B_ref) <= TOL
