"""Pins the oracle's rank-1 updates, Ssymv / Chemv and the GEMM-shaped level-3
restatements (oracle/oracle.c) to the reference's own code compiled in
oracle/_ref: the serial kernels Sger_naive.cl, Cgeru_naive.cl,
Cgerc_naive.cl, Ssymv_naive_{lower,upper}.cl, Chemv_naive.cl,
Ssyrk_naive.cl, Ssyr2k_naive.cl, Ssymm_naive.cl and the CPU template
cpu_symv (tests/blas_funcs/test_symv.hpp).

Bars: the rank-1 updates evaluate the same FP32 expressions as the kernels:
bit-identical.  The others sum in FP32 in the kernels and in double in the
oracle: relative Frobenius error <= 1e-5 (5e-7 against the double
template), and elements outside the referenced triangle untouched.
Strmm_naive.cl does not compute the product the reference header documents;
test_strmm_kernel_is_not_the_documented_product records what it does.
"""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built (reference tree absent at build time)")


def _p(a):
    return a.ctypes.data


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def cvec(rng, n):
    return rng.uniform(-1, 1, (n, 2)).astype(np.float32).view(np.complex64).reshape(-1)


@pytest.mark.parametrize("m,n,incx,incy,lda", [(3, 5, 1, 1, 3), (17, 17, 2, 1, 20), (68, 33, 1, 3, 70)])
def test_ger_bit_exact(m, n, incx, incy, lda):
    rng = np.random.default_rng(m * 7 + n)
    R = O.ref()
    x = rng.uniform(-2, 2, m * incx).astype(np.float32)
    y = rng.uniform(-2, 2, n * incy).astype(np.float32)
    A = rng.uniform(-2, 2, lda * n).astype(np.float32)
    A1, A2 = A.copy(), A.copy()
    O.sger(m, n, 0.75, x, incx, y, incy, A1, lda)
    R.ref_naive_sger(m, n, 0.75, _p(x), incx, _p(y), incy, _p(A2), lda)
    assert np.array_equal(bits(A1), bits(A2))
    xc, yc, Ac = cvec(rng, m * incx), cvec(rng, n * incy), cvec(rng, lda * n)
    for conj in (0, 1):
        A1, A2 = Ac.copy(), Ac.copy()
        O.cger(conj, m, n, 0.5 - 0.25j, xc, incx, yc, incy, A1, lda)
        alb = O.cbox(0.5 - 0.25j)   # kept alive across the call
        R.ref_naive_cger(conj, m, n, _p(alb), _p(xc), incx, _p(yc), incy, _p(A2), lda)
        assert np.array_equal(bits(A1), bits(A2)), conj


@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("n,lda,inc", [(1, 1, 1), (33, 35, 1), (252, 252, 2)])
def test_symv_hemv(uplo, n, lda, inc):
    rng = np.random.default_rng(n + 10 * uplo)
    R = O.ref()
    A = rng.uniform(-1, 1, lda * n).astype(np.float32)
    x = rng.uniform(-1, 1, n * inc).astype(np.float32)
    y = rng.uniform(-1, 1, n * inc).astype(np.float32)
    for beta in (0.5, 0.0):
        y1, y2, y3 = y.copy(), y.copy(), y.copy()
        O.ssymv(uplo, n, 1.25, A, lda, x, inc, beta, y1, inc)
        R.ref_naive_ssymv(uplo, n, 1.25, _p(A), lda, _p(x), inc, beta, _p(y2), inc)
        R.ref_cpu_ssymv(uplo, n, 1.25, _p(A), lda, _p(x), inc, beta, _p(y3), inc)
        assert O.rel_fro(y1, y2) <= 1e-5
        assert O.rel_fro(y1, y3) <= 5e-7
    Ac, xc, yc = cvec(rng, lda * n), cvec(rng, n * inc), cvec(rng, n * inc)
    # Chemv_naive.cl writes its diagonal term as an OpenCL vector literal
    # (:31,41), which the C++ build of the kernel reads as 0; the kernel is
    # compared on a matrix with a zero diagonal, the double template on the
    # full one.
    A0 = Ac.copy()
    A0[np.arange(n) * (lda + 1)] = 0
    al, be = 0.5 - 1j, 0.25 + 0.5j
    alb = O.cbox(al)
    for b in (be, 0j):
        bb = O.cbox(b)
        y1, y3 = yc.copy(), yc.copy()
        O.chemv(uplo, n, al, Ac, lda, xc, inc, b, y1, inc)
        R.ref_cpu_chemv(uplo, n, _p(alb), _p(Ac), lda, _p(xc), inc, _p(bb), _p(y3), inc)
        assert O.rel_fro(y1, y3) <= 5e-7
        y1, y2 = yc.copy(), yc.copy()
        O.chemv(uplo, n, al, A0, lda, xc, inc, b, y1, inc)
        R.ref_naive_chemv(uplo, n, _p(alb), _p(A0), lda, _p(xc), inc, _p(bb), _p(y2), inc)
        assert O.rel_fro(y1, y2) <= 1e-5


def _tri_mask(n, ldc, uplo):
    M = np.zeros((n, ldc), bool)  # [col, row] of column-major storage
    for j in range(n):
        for i in range(n):
            if (i >= j) if uplo == 1 else (i <= j):
                M[j, i] = True
    return M.reshape(-1)


@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1])
def test_syrk_syr2k(uplo, trans):
    rng = np.random.default_rng(3 + uplo + 2 * trans)
    R = O.ref()
    n, k = 37, 19
    lda = (n if trans == 0 else k) + 2
    cols = k if trans == 0 else n
    A = rng.uniform(-1, 1, lda * cols).astype(np.float32)
    Bm = rng.uniform(-1, 1, lda * cols).astype(np.float32)
    ldc = n + 3
    Cm = rng.uniform(-1, 1, ldc * n).astype(np.float32)
    mask = _tri_mask(n, ldc, uplo)
    C1, C2 = Cm.copy(), Cm.copy()
    O.ssyrk(uplo, trans, n, k, 0.75, A, lda, -0.5, C1, ldc)
    R.ref_naive_ssyr2k(uplo, trans, n, k, 0.75, _p(A), lda, None, lda, -0.5, _p(C2), ldc)
    assert O.rel_fro(C1[mask], C2[mask]) <= 1e-5
    assert np.array_equal(C1[~mask], Cm[~mask]) and np.array_equal(C2[~mask], Cm[~mask])
    C1, C2 = Cm.copy(), Cm.copy()
    O.ssyr2k(uplo, trans, n, k, 0.75, A, lda, Bm, lda, -0.5, C1, ldc)
    R.ref_naive_ssyr2k(uplo, trans, n, k, 0.75, _p(A), lda, _p(Bm), lda, -0.5, _p(C2), ldc)
    assert O.rel_fro(C1[mask], C2[mask]) <= 1e-5
    assert np.array_equal(C1[~mask], Cm[~mask])


@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
def test_symm(side, uplo):
    rng = np.random.default_rng(5 + side + 2 * uplo)
    R = O.ref()
    m, n = 29, 23
    na = m if side == 0 else n
    lda, ldb, ldc = na + 1, m + 2, m + 3
    A = rng.uniform(-1, 1, lda * na).astype(np.float32)
    Bm = rng.uniform(-1, 1, ldb * n).astype(np.float32)
    Cm = rng.uniform(-1, 1, ldc * n).astype(np.float32)
    C1, C2 = Cm.copy(), Cm.copy()
    O.ssymm(side, uplo, m, n, 1.5, A, lda, Bm, ldb, 0.25, C1, ldc)
    R.ref_naive_ssymm(side, uplo, m, n, 1.5, _p(A), lda, _p(Bm), ldb, 0.25, _p(C2), ldc)
    assert O.rel_fro(C1, C2) <= 1e-5


def test_strmm_oracle_is_the_documented_product():
    """orc_strmm = alpha * op(T) @ B (or B @ op(T)) with T the triangle of A."""
    rng = np.random.default_rng(8)
    m, n = 13, 9
    for side in (0, 1):
        na = m if side == 0 else n
        for uplo in (0, 1):
            for transa in (0, 1):
                for diag in (0, 1):
                    A = rng.uniform(-1, 1, (na, na)).astype(np.float32)
                    Bm = rng.uniform(-1, 1, (n, m)).astype(np.float32)   # [col, row]
                    Cm = np.zeros((n, m), np.float32)
                    O.strmm(side, uplo, transa, diag, m, n, 0.5, A.reshape(-1), na, Bm.reshape(-1), m,
                            Cm.reshape(-1), m)
                    Ad = A.T.astype(np.float64)          # row-major view of A
                    T = np.tril(Ad) if uplo == 1 else np.triu(Ad)
                    if diag == 1:
                        np.fill_diagonal(T, 1.0)
                    opT = T.T if transa else T
                    Bd = Bm.T.astype(np.float64)
                    want = 0.5 * (opT @ Bd if side == 0 else Bd @ opT)
                    assert np.allclose(Cm.T, want, rtol=1e-6, atol=1e-6)


def test_strmm_kernel_is_not_the_documented_product():
    """The reference's Strmm_naive.cl (left, upper, N) writes only C(i, j)
    with j >= i, and there computes alpha * sum_k A(i,k) B(k,j) over all k,
    i.e. a GEMM row of the full A: the values the reference's own
    test_Strmm.cpp expects.  The library and the oracle compute the
    documented triangular product instead."""
    rng = np.random.default_rng(9)
    m = n = 6
    A = rng.uniform(-1, 1, m * m).astype(np.float32)
    Bm = rng.uniform(-1, 1, m * n).astype(np.float32)
    Cm = np.full(m * n, 7.0, np.float32)
    O.ref().ref_naive_strmm(0, 0, 0, 0, m, n, 2.0, _p(A), m, _p(Bm), m, _p(Cm), m)
    full = 2.0 * (A.reshape(m, m).T.astype(np.float64) @ Bm.reshape(n, m).T.astype(np.float64))
    got = Cm.reshape(n, m).T
    for i in range(m):
        for j in range(n):
            if j >= i:
                assert abs(got[i, j] - full[i, j]) <= 1e-5 * (1 + abs(full[i, j]))
            else:
                assert got[i, j] == 7.0
    doc = np.zeros(m * n, np.float32)
    O.strmm(0, 0, 0, 0, m, n, 2.0, A, m, Bm, m, doc, m)
    assert not np.allclose(doc.reshape(n, m).T, got)
