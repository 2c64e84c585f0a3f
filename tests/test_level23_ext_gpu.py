"""Rank-1 updates, Ssymv / Chemv and the GEMM-shaped level-3 routines
(Ssyrk, Ssyr2k, Ssymm, Strmm) on the GPU, through the C ABI, against the
oracle.

Bars: Sger / Cgeru / Cgerc bit-exact (the same FP32 expressions as the
reference kernels, restated by the oracle); Ssymv / Chemv and the level-3
routines in PLAIN_FP32 mode relative Frobenius <= 1e-5 against the oracle
(FP64 sums); in the tensor-core modes the mode's GEMM bar (TF32 2e-3,
3xBF16 3e-5, 6xBF16 2e-6).  Triangles a routine must not touch are checked
bit for bit.
"""
import numpy as np
import pytest

import oracle_lib as O
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu

TOL = 1e-5
MODE_TOL = {B.MATH_PLAIN_FP32: 1e-5, B.MATH_TF32: 2e-3, B.MATH_BF16X3: 3e-5, B.MATH_BF16X6: 2e-6}


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def same(a, b):
    fa = np.ascontiguousarray(a).view(np.float32)
    fb = np.ascontiguousarray(b).view(np.float32)
    return fa.shape == fb.shape and bool(np.all((bits(fa) == bits(fb)) | (np.isnan(fa) & np.isnan(fb))))


def cvec(rng, n, scale=1.0):
    return (scale * rng.uniform(-1, 1, (n, 2))).astype(np.float32).view(np.complex64).reshape(-1)


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


# ------------------------------------------------------------------ ger
@pytest.mark.parametrize("m,n,incx,incy,lda", [(1, 1, 1, 1, 1), (3, 5, 1, 1, 3), (1000, 37, 1, 1, 1000),
                                                (1001, 37, 1, 1, 1004), (517, 300, 2, 3, 520),
                                                (4099, 129, 1, 2, 4100)])
def test_ger_bit_exact(handle, m, n, incx, incy, lda):
    rng = np.random.default_rng(m + 3 * n)
    x = rng.uniform(-2, 2, m * incx).astype(np.float32)
    y = rng.uniform(-2, 2, n * incy).astype(np.float32)
    A = rng.uniform(-2, 2, lda * n).astype(np.float32)
    Ar, A1 = A.copy(), A.copy()
    O.sger(m, n, 0.75, x, incx, y, incy, Ar, lda)
    assert B.iclblasSger(handle, m, n, 0.75, x, incx, y, incy, A1, lda) == B.SUCCESS
    assert same(A1, Ar)
    xc, yc, Ac = cvec(rng, m * incx), cvec(rng, n * incy), cvec(rng, lda * n)
    for conj, fn in ((False, B.iclblasCgeru), (True, B.iclblasCgerc)):
        Ar, A1 = Ac.copy(), Ac.copy()
        O.cger(conj, m, n, 0.5 - 0.25j, xc, incx, yc, incy, Ar, lda)
        assert fn(handle, m, n, 0.5 - 0.25j, xc, incx, yc, incy, A1, lda) == B.SUCCESS
        assert same(A1, Ar), conj


def test_ger_device_operands_misaligned(handle):
    rng = np.random.default_rng(2)
    m, n, lda = 2053, 70, 2056
    x = rng.uniform(-1, 1, m + 1).astype(np.float32)
    y = rng.uniform(-1, 1, n).astype(np.float32)
    A = rng.uniform(-1, 1, lda * n + 1).astype(np.float32)
    for off in (0, 1):  # off = 1: x and A not 16-byte aligned -> element path
        Ar = A.copy()
        O.sger(m, n, -1.5, x[off:], 1, y, 1, Ar[off:], lda)
        dA = dev(A)
        assert B.iclblasSger(handle, m, n, -1.5, dev(x)[off:], 1, dev(y), 1, dA[off:], lda) == B.SUCCESS
        assert same(host(dA), Ar)


# ------------------------------------------------------------------ symv / hemv
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("n,lda,incx,incy", [(1, 1, 1, 1), (2, 2, 1, 1), (127, 127, 1, 1), (128, 130, 1, 1),
                                             (129, 132, 2, 3), (1000, 1001, 1, 1), (2053, 2056, 1, 2)])
def test_symv_hemv(handle, uplo, n, lda, incx, incy):
    rng = np.random.default_rng(n + 100 * uplo)
    A = rng.uniform(-1, 1, lda * n).astype(np.float32)
    x = rng.uniform(-1, 1, n * incx).astype(np.float32)
    y = rng.uniform(-1, 1, n * incy).astype(np.float32)
    for beta in (0.5, 0.0):
        yr, y1 = y.copy(), y.copy()
        O.ssymv(uplo, n, 1.25, A, lda, x, incx, beta, yr, incy)
        assert B.iclblasSsymv(handle, uplo, n, 1.25, A, lda, x, incx, beta, y1, incy) == B.SUCCESS
        assert O.rel_fro(y1, yr) <= TOL
        assert np.array_equal(y1.reshape(-1)[np.setdiff1d(np.arange(len(y)), np.arange(n) * incy)],
                              y.reshape(-1)[np.setdiff1d(np.arange(len(y)), np.arange(n) * incy)])
    Ac, xc, yc = cvec(rng, lda * n), cvec(rng, n * incx), cvec(rng, n * incy)
    for beta in (0.25 + 0.5j, 0j):
        yr, y1 = yc.copy(), yc.copy()
        O.chemv(uplo, n, 0.5 - 1j, Ac, lda, xc, incx, beta, yr, incy)
        assert B.iclblasChemv(handle, uplo, n, 0.5 - 1j, Ac, lda, xc, incx, beta, y1, incy) == B.SUCCESS
        assert O.rel_fro(y1, yr) <= TOL


def test_symv_reads_only_its_triangle(handle):
    """NaN in the triangle a routine does not reference must not reach y."""
    rng = np.random.default_rng(5)
    n, lda = 300, 304
    for uplo in (0, 1):
        A = rng.uniform(-1, 1, (n, lda)).astype(np.float32)   # [col, row]
        Ac = cvec(rng, lda * n).reshape(n, lda)
        for j in range(n):
            if uplo == 1:
                A[j, :j] = np.nan
                Ac[j, :j] = np.nan
            else:
                A[j, j + 1:n] = np.nan
                Ac[j, j + 1:n] = np.nan
            Ac[j, j] = complex(Ac[j, j].real, np.nan)            # Hermitian diagonal: imaginary part unused
        x = rng.uniform(-1, 1, n).astype(np.float32)
        y = np.full(n, np.nan, np.float32)                        # beta = 0: y not read
        yr = np.zeros(n, np.float32)
        O.ssymv(uplo, n, 1.0, np.nan_to_num(A).reshape(-1), lda, x, 1, 0.0, yr, 1)
        assert B.iclblasSsymv(handle, uplo, n, 1.0, A.reshape(-1), lda, x, 1, 0.0, y, 1) == B.SUCCESS
        assert not np.isnan(y).any() and O.rel_fro(y, yr) <= TOL
        xc = cvec(rng, n)
        yc = np.full(n, np.nan, np.complex64)
        yr = np.zeros(n, np.complex64)
        Ar = Ac.copy()
        Ar[np.isnan(Ar.real) | np.isnan(Ar.imag)] = 0
        for j in range(n):
            Ar[j, j] = Ac[j, j].real
        O.chemv(uplo, n, 1.0, Ar.reshape(-1), lda, xc, 1, 0j, yr, 1)
        assert B.iclblasChemv(handle, uplo, n, 1.0, Ac.reshape(-1), lda, xc, 1, 0j, yc, 1) == B.SUCCESS
        assert not np.isnan(yc).any() and O.rel_fro(yc, yr) <= TOL


def test_symv_large_device(handle):
    rng = np.random.default_rng(6)
    n = 8192 + 37
    A = rng.uniform(-1, 1, n * n).astype(np.float32)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    y = rng.uniform(-1, 1, n).astype(np.float32)
    for uplo in (0, 1):
        yr = y.copy()
        O.ssymv(uplo, n, 0.5, A, n, x, 1, 2.0, yr, 1)
        dy = dev(y)
        assert B.iclblasSsymv(handle, uplo, n, 0.5, dev(A), n, dev(x), 1, 2.0, dy, 1) == B.SUCCESS
        assert O.rel_fro(host(dy), yr) <= TOL


# ------------------------------------------------------------------ level 3
def _tri_mask(n, ldc, uplo):
    M = np.zeros((n, ldc), bool)
    for j in range(n):
        if uplo == 1:
            M[j, j:n] = True
        else:
            M[j, :j + 1] = True
    return M.reshape(-1)


@pytest.mark.parametrize("mode", [B.MATH_PLAIN_FP32, B.MATH_TF32, B.MATH_BF16X3, B.MATH_BF16X6])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("n,k", [(1, 1), (37, 19), (300, 64), (777, 300)])
def test_syrk_syr2k(handle, mode, uplo, trans, n, k):
    handle.set_math_mode(mode)
    rng = np.random.default_rng(n + k + uplo + 2 * trans)
    lda = (n if trans == 0 else k) + 2
    cols = k if trans == 0 else n
    A = rng.uniform(-1, 1, lda * cols).astype(np.float32)
    Bm = rng.uniform(-1, 1, lda * cols).astype(np.float32)
    ldc = n + 3
    Cm = rng.uniform(-1, 1, ldc * n).astype(np.float32)
    mask = _tri_mask(n, ldc, uplo)
    for beta in (-0.5, 0.0):
        Cr, C1 = Cm.copy(), Cm.copy()
        O.ssyrk(uplo, trans, n, k, 0.75, A, lda, beta, Cr, ldc)
        assert B.iclblasSsyrk(handle, uplo, trans, n, k, 0.75, A, lda, beta, C1, ldc) == B.SUCCESS
        assert O.rel_fro(C1[mask], Cr[mask]) <= MODE_TOL[mode]
        assert np.array_equal(C1[~mask], Cm[~mask])
        Cr, C1 = Cm.copy(), Cm.copy()
        O.ssyr2k(uplo, trans, n, k, 0.75, A, lda, Bm, lda, beta, Cr, ldc)
        assert B.iclblasSsyr2k(handle, uplo, trans, n, k, 0.75, A, lda, Bm, lda, beta, C1, ldc) == B.SUCCESS
        assert O.rel_fro(C1[mask], Cr[mask]) <= MODE_TOL[mode]
        assert np.array_equal(C1[~mask], Cm[~mask])


@pytest.mark.parametrize("mode", [B.MATH_PLAIN_FP32, B.MATH_BF16X6])
@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("m,n", [(1, 1), (29, 23), (300, 517)])
def test_symm(handle, mode, side, uplo, m, n):
    handle.set_math_mode(mode)
    rng = np.random.default_rng(m + n + side + 2 * uplo)
    na = m if side == 0 else n
    lda, ldb, ldc = na + 1, m + 2, m + 3
    A = rng.uniform(-1, 1, lda * na).astype(np.float32)
    Bm = rng.uniform(-1, 1, ldb * n).astype(np.float32)
    Cm = rng.uniform(-1, 1, ldc * n).astype(np.float32)
    for beta in (0.25, 0.0):
        Cr, C1 = Cm.copy(), Cm.copy()
        O.ssymm(side, uplo, m, n, 1.5, A, lda, Bm, ldb, beta, Cr, ldc)
        assert B.iclblasSsymm(handle, side, uplo, m, n, 1.5, A, lda, Bm, ldb, beta, C1, ldc) == B.SUCCESS
        assert O.rel_fro(C1, Cr) <= MODE_TOL[mode]


@pytest.mark.parametrize("mode", [B.MATH_PLAIN_FP32, B.MATH_BF16X6])
@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("transa", [0, 1, 2])
@pytest.mark.parametrize("diag", [0, 1])
def test_trmm_all_variants(handle, mode, side, uplo, transa, diag):
    handle.set_math_mode(mode)
    rng = np.random.default_rng(side + 2 * uplo + 4 * transa + 12 * diag)
    for m, n in ((1, 1), (37, 23), (600, 300)):
        na = m if side == 0 else n
        lda, ldb, ldc = na + 1, m + 2, m + 3
        A = rng.uniform(-1, 1, lda * na).astype(np.float32)
        Bm = rng.uniform(-1, 1, ldb * n).astype(np.float32)
        Cm = rng.uniform(-1, 1, ldc * n).astype(np.float32)
        Cr, C1 = Cm.copy(), Cm.copy()
        O.strmm(side, uplo, transa, diag, m, n, 0.5, A, lda, Bm, ldb, Cr, ldc)
        assert B.iclblasStrmm(handle, side, uplo, transa, diag, m, n, 0.5, A, lda, Bm, ldb, C1, ldc) == B.SUCCESS
        assert O.rel_fro(C1, Cr) <= MODE_TOL[mode], (m, n)
        gaps = np.ones(ldc * n, bool).reshape(n, ldc)
        gaps[:, :m] = False
        assert np.array_equal(C1[gaps.reshape(-1)], Cm[gaps.reshape(-1)])


@pytest.mark.parametrize("side", [0, 1])
def test_trmm_in_place(handle, side):
    """C == B (the reference's own test calls it this way), host and device."""
    rng = np.random.default_rng(11 + side)
    m, n = 700, 333
    na = m if side == 0 else n
    A = rng.uniform(-1, 1, na * na).astype(np.float32)
    Bm = rng.uniform(-1, 1, m * n).astype(np.float32)
    Cr = np.zeros(m * n, np.float32)
    O.strmm(side, 1, 0, 0, m, n, 2.0, A, na, Bm, m, Cr, m)
    B1 = Bm.copy()
    assert B.iclblasStrmm(handle, side, 1, 0, 0, m, n, 2.0, A, na, B1, m, B1, m) == B.SUCCESS
    assert O.rel_fro(B1, Cr) <= TOL
    dB = dev(Bm)
    assert B.iclblasStrmm(handle, side, 1, 0, 0, m, n, 2.0, dev(A), na, dB, m, dB, m) == B.SUCCESS
    assert O.rel_fro(host(dB), Cr) <= TOL


def test_level3_large_device_modes(handle):
    """2048-sized problems on device operands in every mode (recursion with
    several levels of splits)."""
    rng = np.random.default_rng(12)
    n, k = 2048 + 65, 1024
    A = rng.uniform(-1, 1, n * k).astype(np.float32)
    Cm = rng.uniform(-1, 1, n * n).astype(np.float32)
    mask = _tri_mask(n, n, 1)
    Cr = Cm.copy()
    O.ssyrk(1, 0, n, k, 1.0, A, n, 0.5, Cr, n)
    for mode in (B.MATH_PLAIN_FP32, B.MATH_TF32, B.MATH_BF16X3, B.MATH_BF16X6):
        handle.set_math_mode(mode)
        dC = dev(Cm)
        assert B.iclblasSsyrk(handle, 1, 0, n, k, 1.0, dev(A), n, 0.5, dC, n) == B.SUCCESS
        C1 = host(dC)
        assert O.rel_fro(C1[mask], Cr[mask]) <= MODE_TOL[mode], mode
        assert np.array_equal(C1[~mask], Cm[~mask])


# ------------------------------------------------------------------ argument rules
def test_argument_rules(handle):
    a = np.ones(64, np.float32)
    ac = np.ones(64, np.complex64)
    assert B.iclblasSger(handle, 0, 3, 1.0, None, 1, None, 1, None, 1) == B.SUCCESS     # m == 0 first
    assert B.iclblasSger(handle, 3, 3, 0.0, None, 1, None, 1, None, 1) == B.SUCCESS     # alpha == 0 first
    assert B.iclblasSger(handle, -1, 3, 1.0, a, 1, a, 1, a, 3) == B.INVALID_VALUE
    assert B.iclblasSger(handle, 3, 3, 1.0, a, 0, a, 1, a, 3) == B.INVALID_VALUE
    assert B.iclblasSger(handle, 3, 3, 1.0, a, 1, a, -1, a, 3) == B.NOT_SUPPORTED
    assert B.iclblasSger(handle, 3, 3, 1.0, a, 1, a, 1, a, 0) == B.INVALID_VALUE
    assert B.iclblasCgeru(handle, 3, 3, 1.0, ac, 1, ac, 0, ac, 3) == B.INVALID_VALUE
    assert B.iclblasSsymv(handle, 0, 0, 1.0, None, 1, None, 1, 0.0, None, 1) == B.SUCCESS
    assert B.iclblasSsymv(handle, 0, 3, 0.0, None, 1, None, 1, 1.0, None, 1) == B.SUCCESS  # alpha 0, beta 1
    assert B.iclblasSsymv(handle, 0, -3, 1.0, a, 3, a, 1, 0.0, a, 1) == B.INVALID_VALUE
    assert B.iclblasChemv(handle, 1, 3, 1.0, ac, 3, ac, 1, 0j, None, 1) == B.INVALID_VALUE
    assert B.iclblasSsyrk(handle, 0, 0, 3, 0, 1.0, None, 1, 2.0, None, 1) == B.SUCCESS      # k == 0 returns first
    assert B.iclblasSsyrk(handle, 0, 0, 3, -1, 1.0, a, 3, 2.0, a, 3) == B.INVALID_VALUE
    assert B.iclblasSsyr2k(handle, 0, 0, 3, 2, 1.0, a, 3, None, 3, 2.0, a, 3) == B.INVALID_VALUE
    assert B.iclblasSsymm(handle, 0, 0, 0, 3, 1.0, None, 1, None, 1, 1.0, None, 1) == B.SUCCESS
    assert B.iclblasStrmm(handle, 0, 0, 0, 0, 0, 3, 1.0, None, 1, None, 1, None, 1) == B.SUCCESS
    assert B.iclblasStrmm(handle, 0, 0, 0, 0, 3, 3, 1.0, a, 3, a, 3, None, 3) == B.INVALID_VALUE
    # alpha == 0: C = 0 without reading A or B
    Cm = np.full(9, 5.0, np.float32)
    nanm = np.full(9, np.nan, np.float32)
    assert B.iclblasStrmm(handle, 0, 0, 0, 0, 3, 3, 0.0, nanm, 3, nanm, 3, Cm, 3) == B.SUCCESS
    assert np.array_equal(Cm, np.zeros(9, np.float32))
