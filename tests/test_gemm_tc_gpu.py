"""Tensor-core GEMM modes (TF32, 3xBF16, 6xBF16) on the GPU against the FP64 oracle.

These modes have no reference counterpart; they are pinned to the FP64
oracle (orc_dgemm, the same arithmetic as the FP32 oracle in double).  Error
bars (relative Frobenius, U(-1,1) data, K <= 513): TF32 <= 2e-3 (10-bit
mantissa operands), 3xBF16 <= 3e-5 (three leading split products; the
dropped terms are ~2^-16 relative), 6xBF16 <= 2e-6 (FP32 level; measured
2.2e-7 at 8192^3 where the plain FP32 path gives 1.6e-6).
"""
import numpy as np
import pytest

import oracle_lib as O
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu

BARS = {B.MATH_TF32: 2e-3, B.MATH_BF16X3: 3e-5, B.MATH_BF16X6: 2e-6}


def _shape(op, rows, cols):
    return (rows, cols) if op == 0 else (cols, rows)


def _dref(ta, tb, m, n, k, alpha, A, lda, Bm, ldb, beta, Cm, ldc):
    Cd = Cm.astype(np.float64)
    O.dgemm(ta, tb, m, n, k, alpha, A.astype(np.float64), lda, Bm.astype(np.float64), ldb, beta, Cd, ldc)
    return Cd


@pytest.mark.parametrize("mode", [B.MATH_TF32, B.MATH_BF16X3, B.MATH_BF16X6])
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("mnk", [(1, 1, 1), (100, 7, 33), (129, 257, 64), (300, 300, 513), (256, 512, 256)])
def test_sgemm_tensor_core_modes(handle, mode, ta, tb, mnk):
    m, n, k = mnk
    rng = np.random.default_rng(m * 7 + n * 3 + k + 100 * ta + 10 * tb + mode)
    ar, ac = _shape(ta, m, k)
    br, bc = _shape(tb, k, n)
    lda, ldb, ldc = ar + 3, br + 1, m + 2
    A = O.colmajor(ar, ac, lda, rng)
    Bm = O.colmajor(br, bc, ldb, rng)
    Cm = O.colmajor(m, n, ldc, rng)
    ref = _dref(ta, tb, m, n, k, 1.25, A, lda, Bm, ldb, -0.5, Cm, ldc)
    handle.set_math_mode(mode)
    assert B.iclblasSgemm(handle, ta, tb, m, n, k, 1.25, A, lda, Bm, ldb, -0.5, Cm, ldc) == B.SUCCESS
    err = O.rel_fro(Cm.reshape(n, ldc)[:, :m], ref.reshape(n, ldc)[:, :m])
    assert err <= BARS[mode], err
    # padding rows of C untouched
    assert np.array_equal(Cm.reshape(n, ldc)[:, m:], ref.reshape(n, ldc)[:, m:].astype(np.float32))


@pytest.mark.parametrize("mode", [B.MATH_TF32, B.MATH_BF16X3, B.MATH_BF16X6])
def test_sgemm_tensor_core_beta0_ignores_c(handle, mode):
    m, n, k = 200, 300, 96
    rng = np.random.default_rng(5)
    A = O.colmajor(m, k, m, rng)
    Bm = O.colmajor(k, n, k, rng)
    Cm = np.full(m * n, np.nan, np.float32)
    ref = _dref(0, 0, m, n, k, 2.0, A, m, Bm, k, 0.0, np.zeros(m * n, np.float32), m)
    handle.set_math_mode(mode)
    assert B.iclblasSgemm(handle, 0, 0, m, n, k, 2.0, A, m, Bm, k, 0.0, Cm, m) == B.SUCCESS
    assert np.all(np.isfinite(Cm))
    assert O.rel_fro(Cm, ref) <= BARS[mode]


@pytest.mark.parametrize("mode", [B.MATH_TF32, B.MATH_BF16X3, B.MATH_BF16X6])
@pytest.mark.parametrize("ta,tb", [(0, 0), (2, 0), (1, 2)])
def test_cgemm_tensor_core_modes(handle, mode, ta, tb):
    m, n, k = 150, 130, 77
    rng = np.random.default_rng(ta * 3 + tb + mode)
    ar, ac = _shape(ta, m, k)
    br, bc = _shape(tb, k, n)
    A = O.colmajor(ar, ac, ar, rng, np.complex64)
    Bm = O.colmajor(br, bc, br, rng, np.complex64)
    Cm = O.colmajor(m, n, m + 1, rng, np.complex64)
    al, be = 0.75 - 0.5j, 0.25 + 0.5j
    # FP64 reference with numpy (complex128) on the same op semantics
    Ad = A.astype(np.complex128).reshape(ac, ar).T
    Bd = Bm.astype(np.complex128).reshape(bc, br).T
    opA = Ad if ta == 0 else (Ad.T if ta == 1 else Ad.conj().T)
    opB = Bd if tb == 0 else (Bd.T if tb == 1 else Bd.conj().T)
    Cd = Cm.astype(np.complex128).reshape(n, m + 1).T[:m]
    ref = al * (opA @ opB) + be * Cd
    handle.set_math_mode(mode)
    assert B.iclblasCgemm(handle, ta, tb, m, n, k, al, A, ar, Bm, br, be, Cm, m + 1) == B.SUCCESS
    got = Cm.reshape(n, m + 1).T[:m]
    assert O.rel_fro(got, ref) <= BARS[mode]


def test_plain_mode_unchanged_after_tc(handle):
    """Switching back to PLAIN_FP32 restores the bit-exact CUDA-core path."""
    m, n, k = 64, 48, 40
    rng = np.random.default_rng(8)
    A = O.colmajor(m, k, m, rng)
    Bm = O.colmajor(k, n, k, rng)
    Cm = O.colmajor(m, n, m, rng)
    C_ref = Cm.copy()
    O.sgemm(0, 0, m, n, k, 1.0, A, m, Bm, k, 1.0, C_ref, m)
    handle.set_math_mode(B.MATH_BF16X3)
    handle.set_math_mode(B.MATH_PLAIN_FP32)
    assert B.iclblasSgemm(handle, 0, 0, m, n, k, 1.0, A, m, Bm, k, 1.0, Cm, m) == B.SUCCESS
    assert np.array_equal(Cm, C_ref)


@pytest.mark.parametrize("mode", [B.MATH_TF32, B.MATH_BF16X3, B.MATH_BF16X6])
def test_sgemm_tensor_core_256_wide_tiles(handle, mode):
    """Large enough for 256-column tiles (the sizes above run 128-column ones)."""
    m, n, k = 1536, 2560, 100
    rng = np.random.default_rng(500 + mode)
    A = O.colmajor(k, m, k + 4, rng)          # op T
    Bm = O.colmajor(k, n, k, rng)
    Cm = O.colmajor(m, n, m, rng)
    ref = _dref(1, 0, m, n, k, 0.75, A, k + 4, Bm, k, -1.25, Cm, m)
    handle.set_math_mode(mode)
    assert B.iclblasSgemm(handle, 1, 0, m, n, k, 0.75, A, k + 4, Bm, k, -1.25, Cm, m) == B.SUCCESS
    assert O.rel_fro(Cm, ref) <= BARS[mode]


def test_cgemm_tensor_core_256_wide_tiles(handle):
    m, n, k = 1280, 1600, 40
    rng = np.random.default_rng(77)
    A = O.colmajor(m, k, m, rng, np.complex64)
    Bm = O.colmajor(n, k, n, rng, np.complex64)   # op C
    Cm = O.colmajor(m, n, m, rng, np.complex64)
    al, be = 0.5 + 0.25j, -0.75j
    Ad = A.astype(np.complex128).reshape(k, m).T
    Bd = Bm.astype(np.complex128).reshape(k, n).T
    ref = al * (Ad @ Bd.conj().T) + be * Cm.astype(np.complex128).reshape(n, m).T
    handle.set_math_mode(B.MATH_BF16X6)
    assert B.iclblasCgemm(handle, 0, 2, m, n, k, al, A, m, Bm, n, be, Cm, m) == B.SUCCESS
    assert O.rel_fro(Cm.reshape(n, m).T, ref) <= BARS[B.MATH_BF16X6]


@pytest.mark.parametrize("mode", [B.MATH_TF32, B.MATH_BF16X3, B.MATH_BF16X6])
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 1)])
def test_sgemm_tensor_core_cta_pairs(handle, mode, ta, tb):
    """Enough 256 x 256 tiles for the CTA-pair (2-SM) kernel; ragged edges."""
    m, n, k = 2560 + 37, 2048 + 5, 200
    rng = np.random.default_rng(900 + mode + 10 * ta)
    ar, ac = _shape(ta, m, k)
    br, bc = _shape(tb, k, n)
    A = O.colmajor(ar, ac, ar + 1, rng)
    Bm = O.colmajor(br, bc, br, rng)
    Cm = O.colmajor(m, n, m, rng)
    ref = _dref(ta, tb, m, n, k, 1.5, A, ar + 1, Bm, br, 0.5, Cm, m)
    handle.set_math_mode(mode)
    assert B.iclblasSgemm(handle, ta, tb, m, n, k, 1.5, A, ar + 1, Bm, br, 0.5, Cm, m) == B.SUCCESS
    assert O.rel_fro(Cm, ref) <= BARS[mode]


def test_cgemm_tensor_core_cta_pairs(handle):
    m, n, k = 2560, 1100, 60
    rng = np.random.default_rng(78)
    A = O.colmajor(m, k, m, rng, np.complex64)
    Bm = O.colmajor(k, n, k, rng, np.complex64)
    Cm = O.colmajor(m, n, m, rng, np.complex64)
    al, be = 1.0 - 0.5j, 0.25 + 0.25j
    Ad = A.astype(np.complex128).reshape(k, m).T
    Bd = Bm.astype(np.complex128).reshape(n, k).T
    ref = al * (Ad @ Bd) + be * Cm.astype(np.complex128).reshape(n, m).T
    handle.set_math_mode(B.MATH_BF16X3)
    assert B.iclblasCgemm(handle, 0, 0, m, n, k, al, A, m, Bm, k, be, Cm, m) == B.SUCCESS
    assert O.rel_fro(Cm.reshape(n, m).T, ref) <= BARS[B.MATH_BF16X3]


@pytest.mark.parametrize("mode", [B.MATH_TF32, B.MATH_BF16X3, B.MATH_BF16X6])
@pytest.mark.parametrize("m,n,k", [(300, 217, 70), (2560 + 37, 2048 + 5, 96)])
def test_sgemm_tensor_core_staged_c_edges(handle, mode, m, n, k):
    """ldc a multiple of 4 floats: C is read and written through TMA boxes
    (single CTAs and CTA pairs), which must clip at row m and column n and
    leave the rows between m and ldc untouched."""
    rng = np.random.default_rng(1300 + mode + m)
    ldc = (m + 3) // 4 * 4 + 4
    A = O.colmajor(m, k, m, rng)
    Bm = O.colmajor(k, n, k + 1, rng)
    Cm = O.colmajor(m, n, ldc, rng)
    ref = _dref(0, 0, m, n, k, 1.5, A, m, Bm, k + 1, -0.75, Cm, ldc)
    handle.set_math_mode(mode)
    assert B.iclblasSgemm(handle, 0, 0, m, n, k, 1.5, A, m, Bm, k + 1, -0.75, Cm, ldc) == B.SUCCESS
    got, want = Cm.reshape(n, ldc), ref.reshape(n, ldc)
    assert O.rel_fro(got[:, :m], want[:, :m]) <= BARS[mode]
    assert np.array_equal(got[:, m:], want[:, m:].astype(np.float32))


@pytest.mark.parametrize("m,n", [(150, 131), (2560 + 3, 1030)])
def test_cgemm_tensor_core_staged_c_edges(handle, m, n):
    """Complex C through TMA boxes of (re, im) pairs: ragged edges, ldc even."""
    k = 45
    rng = np.random.default_rng(1400 + m)
    ldc = m + (m % 2) + 2
    A = O.colmajor(m, k, m, rng, np.complex64)
    Bm = O.colmajor(k, n, k, rng, np.complex64)
    Cm = O.colmajor(m, n, ldc, rng, np.complex64)
    C0 = Cm.copy()
    al, be = 0.5 - 1.0j, -0.25 + 0.75j
    Ad = A.astype(np.complex128).reshape(k, m).T
    Bd = Bm.astype(np.complex128).reshape(n, k).T
    ref = al * (Ad @ Bd) + be * Cm.astype(np.complex128).reshape(n, ldc).T[:m]
    handle.set_math_mode(B.MATH_BF16X6)
    assert B.iclblasCgemm(handle, 0, 0, m, n, k, al, A, m, Bm, k, be, Cm, ldc) == B.SUCCESS
    assert O.rel_fro(Cm.reshape(n, ldc).T[:m], ref) <= BARS[B.MATH_BF16X6]
    assert np.array_equal(Cm.reshape(n, ldc)[:, m:], C0.reshape(n, ldc)[:, m:])
