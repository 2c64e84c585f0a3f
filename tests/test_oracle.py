"""Pins the oracle restatement (oracle/oracle.c) to the reference's own CPU code.

oracle/_ref/libiclref.so is built from the reference's sources where they lie
(tests/blas_funcs/*.hpp CPU templates, tests/blas_reference/blas_reference.cpp,
and the serial OpenCL kernels compiled as C++).  Where the oracle restates the
same double-precision arithmetic the results must be bit-identical; against
the serial FP32 kernels (GEMV/TRSV/TRSM), which round differently, the bar is
a relative Frobenius error far below the 1e-5 parity tolerance.
"""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built (reference tree absent at build time)")

rng0 = np.random.default_rng


def _p(a):
    return a.ctypes.data


@pytest.mark.parametrize("n,inc", [(1, 1), (17, 1), (1000, 1), (513, 3)])
def test_level1_real_bit_exact(n, inc):
    rng = rng0(10 + n + inc)
    R = O.ref()
    x = rng.uniform(-1, 1, n * inc).astype(np.float32)
    y = rng.uniform(-1, 1, n * inc).astype(np.float32)
    assert O.sdot(n, x, inc, y, inc) == R.ref_cpu_sdot(n, _p(x), inc, _p(y), inc)
    assert O.snrm2(n, x, inc) == R.ref_cpu_snrm2(n, _p(x), inc)
    assert O.sasum(n, x, inc) == R.ref_cpu_sasum(n, _p(x), inc)
    assert O.isamax(n, x, inc) == R.ref_cpu_isamax(n, _p(x), inc)
    y1, y2 = y.copy(), y.copy()
    O.saxpy(n, 0.75, x, inc, y1, inc)
    R.ref_cpu_saxpy(n, 0.75, _p(x), inc, _p(y2), inc)
    assert np.array_equal(y1, y2)
    x1, x2 = x.copy(), x.copy()
    O.sscal(n, -1.5, x1, inc)
    R.ref_cpu_sscal(n, -1.5, _p(x2), inc)
    assert np.array_equal(x1, x2)


def test_isamax_ties_and_nan():
    R = O.ref()
    x = np.array([1, -5, 3, 5, -5, 2], np.float32)
    assert O.isamax(6, x, 1) == R.ref_cpu_isamax(6, _p(x), 1) == 1   # first of the ties
    x = np.array([np.nan, 1, 7, 2], np.float32)
    assert O.isamax(4, x, 1) == R.ref_cpu_isamax(4, _p(x), 1) == 0   # NaN first pins 0
    x = np.array([1, np.nan, 7, 2], np.float32)
    assert O.isamax(4, x, 1) == R.ref_cpu_isamax(4, _p(x), 1) == 2   # later NaN skipped


@pytest.mark.parametrize("n,inc", [(1, 1), (31, 1), (777, 2)])
def test_level1_complex(n, inc):
    rng = rng0(20 + n)
    R = O.ref()
    x = O.colmajor(n * inc, 1, n * inc, rng, np.complex64)
    y = O.colmajor(n * inc, 1, n * inc, rng, np.complex64)
    for conj in (0, 1):
        out = np.zeros(2, np.float32)
        R.ref_cpu_cdot(n, _p(x), inc, _p(y), inc, conj, _p(out))
        assert O.cdot(n, x, inc, y, inc, conj) == complex(out[0], out[1])
    assert O.scnrm2(n, x, inc) == R.ref_cpu_scnrm2(n, _p(x), inc)
    assert O.scasum(n, x, inc) == R.ref_cpu_scasum(n, _p(x), inc)
    assert O.icamax(n, x, inc) == R.ref_cpu_icamax(n, _p(x), inc)
    a = 0.5 - 0.25j
    abox = O.cbox(a)
    x1, x2 = x.copy(), x.copy()
    O.cscal(n, a, x1, inc)
    R.ref_cpu_cscal(n, _p(abox), _p(x2), inc)
    assert np.array_equal(x1, x2)
    # Caxpy_reference accumulates in complex<float>: within float rounding
    y1, y2 = y.copy(), y.copy()
    O.caxpy(n, a, x, inc, y1, inc)
    xc = x.copy()
    R.ref_caxpy_reference(n, _p(abox), _p(xc), inc, _p(y2), inc)
    assert np.max(np.abs(y1 - y2)) <= 4e-7 * (1 + np.max(np.abs(y2)))


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1), (2, 2)])
@pytest.mark.parametrize("beta", [0.0, 0.5])
def test_sgemm_vs_cpu_gemm(ta, tb, beta):
    """Quarter-integer inputs (the reference's own test values) make every
    product and partial sum exact, so the FP32-order oracle and the double
    accumulating cpu_gemm agree bit for bit."""
    rng = rng0(30 + 3 * ta + tb)
    m, n, k = 37, 29, 45
    lda = (m if ta == 0 else k) + 3
    ldb = (k if tb == 0 else n) + 2
    ldc = m + 1
    A = O.quarter_ints(lda * (k if ta == 0 else m), rng)
    Bm = O.quarter_ints(ldb * (n if tb == 0 else k), rng)
    Cm = O.quarter_ints(ldc * n, rng)
    C1, C2 = Cm.copy(), Cm.copy()
    O.sgemm(ta, tb, m, n, k, 1.5, A, lda, Bm, ldb, beta, C1, ldc)
    O.ref().ref_cpu_sgemm(ta, tb, m, n, k, 1.5, _p(A), lda, _p(Bm), ldb, beta, _p(C2), ldc)
    assert np.array_equal(C1, C2)


def test_sgemm_random_vs_cpu_gemm_and_naive():
    rng = rng0(33)
    m = n = k = 64
    A = O.colmajor(m, k, m, rng)
    Bm = O.colmajor(k, n, k, rng)
    Cm = O.colmajor(m, n, m, rng)
    C1, C2, C3 = Cm.copy(), Cm.copy(), Cm.copy()
    O.sgemm(0, 0, m, n, k, 1.5, A, m, Bm, k, 0.5, C1, m)
    O.ref().ref_cpu_sgemm(0, 0, m, n, k, 1.5, _p(A), m, _p(Bm), k, 0.5, _p(C2), m)
    O.ref().ref_naive_sgemm(0, 0, m, n, k, 1.5, _p(A), m, _p(Bm), k, 0.5, _p(C3), m)
    assert O.rel_fro(C1, C2) < 1e-6
    assert O.rel_fro(C1, C3) < 1e-6


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 2), (2, 0)])
def test_cgemm_vs_cpu_gemm(ta, tb):
    rng = rng0(40 + ta + tb)
    m, n, k = 19, 23, 17
    A = O.colmajor(m if ta == 0 else k, k if ta == 0 else m, m if ta == 0 else k, rng, np.complex64)
    Bm = O.colmajor(k if tb == 0 else n, n if tb == 0 else k, k if tb == 0 else n, rng, np.complex64)
    Cm = O.colmajor(m, n, m, rng, np.complex64)
    al, be = 1.5 - 0.5j, 0.25 + 1j
    alb, beb = O.cbox(al), O.cbox(be)
    C1, C2 = Cm.copy(), Cm.copy()
    O.cgemm(ta, tb, m, n, k, al, A, m if ta == 0 else k, Bm, k if tb == 0 else n, be, C1, m)
    O.ref().ref_cpu_cgemm(ta, tb, m, n, k, _p(alb), _p(A), m if ta == 0 else k, _p(Bm),
                          k if tb == 0 else n, _p(beb), _p(C2), m)
    assert O.rel_fro(C1, C2) < 1e-7
    C3 = Cm.copy()
    O.ref().ref_naive_cgemm(ta, tb, m, n, k, _p(alb), _p(A), m if ta == 0 else k, _p(Bm),
                            k if tb == 0 else n, _p(beb), _p(C3), m)
    assert O.rel_fro(C1, C3) < 1e-6


@pytest.mark.parametrize("trans", [0, 1, 2])
def test_gemv_vs_naive_kernels(trans):
    rng = rng0(50 + trans)
    m, n, lda = 70, 45, 73
    A = O.colmajor(m, n, lda, rng)
    xl, yl = (n, m) if trans == 0 else (m, n)
    x = rng.uniform(-1, 1, xl * 2).astype(np.float32)
    y = rng.uniform(-1, 1, yl * 3).astype(np.float32)
    y1, y2 = y.copy(), y.copy()
    O.sgemv(trans, m, n, 0.75, A, lda, x, 2, -0.5, y1, 3)
    O.ref().ref_naive_sgemv(trans, m, n, 0.75, _p(A), lda, _p(x), 2, -0.5, _p(y2), 3)
    assert O.rel_fro(y1, y2) < 1e-6
    Ac = O.colmajor(m, n, lda, rng, np.complex64)
    xc = O.colmajor(xl, 1, xl, rng, np.complex64)
    yc = O.colmajor(yl, 1, yl, rng, np.complex64)
    y1, y2 = yc.copy(), yc.copy()
    alb, beb = O.cbox(0.5 + 1j), O.cbox(1 - 0.5j)
    O.cgemv(trans, m, n, 0.5 + 1j, Ac, lda, xc, 1, 1 - 0.5j, y1, 1)
    O.ref().ref_naive_cgemv(trans, m, n, _p(alb), _p(Ac), lda, _p(xc), 1, _p(beb), _p(y2), 1)
    assert O.rel_fro(y1, y2) < 1e-6


def _tri(n, lda, lower, rng, dtype=np.float32):
    """Well-conditioned triangle: |diag| in [1, 2], off-diagonal N(0,1)/sqrt(n)."""
    A = O.colmajor(n, n, lda, rng, dtype)
    M = A.reshape(n, lda).T  # M[i, j] = A[j*lda + i]
    for j in range(n):
        M[j, j] = rng.uniform(1, 2) * (1 if dtype == np.float32 else np.exp(1j * rng.uniform(0, 6.28)))
        off = rng.standard_normal(n) / np.sqrt(n)
        if lower:
            M[j + 1:n, j] = off[j + 1:n]
        else:
            M[:j, j] = off[:j]
    return A


@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("diag", [0, 1])
def test_trsv_vs_naive_kernels(uplo, trans, diag):
    rng = rng0(60 + 6 * uplo + 2 * trans + diag)
    n, lda = 57, 61
    A = _tri(n, lda, uplo == 1, rng)
    x = rng.uniform(-1, 1, n * 2).astype(np.float32)
    x1, x2 = x.copy(), x.copy()
    O.strsv(uplo, trans, diag, n, A, lda, x1, 2)
    O.ref().ref_naive_strsv(uplo, trans, diag, n, _p(A), lda, _p(x2), 2)
    assert O.rel_fro(x1, x2) < 1e-5
    Ac = _tri(n, lda, uplo == 1, rng, np.complex64)
    xc = O.colmajor(n, 1, n, rng, np.complex64)
    x1, x2 = xc.copy(), xc.copy()
    O.ctrsv(uplo, trans, diag, n, Ac, lda, x1, 1)
    O.ref().ref_naive_ctrsv(uplo, trans, diag, n, _p(Ac), lda, _p(x2), 1)
    assert O.rel_fro(x1, x2) < 1e-5


@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("diag", [0, 1])
def test_trsm_vs_naive_kernels(side, uplo, trans, diag):
    rng = rng0(70 + 12 * side + 6 * uplo + 2 * trans + diag)
    m, n = 33, 21
    na = m if side == 0 else n
    lda, ldb = na + 2, m + 3
    A = _tri(na, lda, uplo == 1, rng)
    Bm = O.colmajor(m, n, ldb, rng)
    B1, B2 = Bm.copy(), Bm.copy()
    O.strsm(side, uplo, trans, diag, m, n, -0.75, A, lda, B1, ldb)
    O.ref().ref_naive_strsm(side, uplo, trans, diag, m, n, -0.75, _p(A), lda, _p(B2), ldb)
    assert O.rel_fro(B1, B2) < 1e-5
    Ac = _tri(na, lda, uplo == 1, rng, np.complex64)
    Bc = O.colmajor(m, n, ldb, rng, np.complex64)
    B1, B2 = Bc.copy(), Bc.copy()
    O.ctrsm(side, uplo, trans, diag, m, n, 0.5 - 1j, Ac, lda, B1, ldb)
    alb = O.cbox(0.5 - 1j)
    O.ref().ref_naive_ctrsm(side, uplo, trans, diag, m, n, _p(alb), _p(Ac), lda, _p(B2), ldb)
    assert O.rel_fro(B1, B2) < 1e-5


def test_dgemm_dtrsm_consistency():
    """FP64 oracle pieces used by the precision study: solve then multiply back."""
    rng = rng0(80)
    m, n = 48, 16
    L = _tri(m, m, True, rng).astype(np.float64)
    Bm = rng.uniform(-1, 1, m * n)
    X = Bm.copy()
    O.dtrsm(0, 1, 0, 0, m, n, 2.0, L, m, X, m)
    # multiply back with the stored triangle only (the other one is junk)
    Lt = np.ascontiguousarray(np.tril(L.reshape(m, m).T).T).reshape(-1)
    R = np.zeros(m * n)
    O.dgemm(0, 0, m, n, m, 1.0, Lt, m, X, m, 0.0, R, m)
    assert np.max(np.abs(R - 2.0 * Bm)) < 1e-12
