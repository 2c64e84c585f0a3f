"""TRSM residual refinement (iclblasSetTrsmRefinement; no reference
counterpart) against FP64 solves of the same FP32 inputs.

Without refinement the 3xBF16 solve is at the 2^-16 level of its split
products (a few 1e-6 on these sizes); one step with an FP32-accurate residual
brings it to the FP32 level (bar 1e-6), TF32 needs two steps for the same bar,
and PLAIN_FP32 stays within the library's 1e-5 bar.  Matrices: diagonal of
modulus U(1,2), off-diagonal N(0,1)/sqrt(n) (the STRSM config's
construction), junk in the unused triangle.
"""
import numpy as np
import pytest
import scipy.linalg as sla

from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu


def tri(n, lower, rng, cplx):
    off = rng.standard_normal((n, n)) / np.sqrt(n)
    d = rng.uniform(1, 2, n)
    if cplx:
        off = off + 1j * rng.standard_normal((n, n)) / np.sqrt(n)
        d = d * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    L = (np.tril(off, -1) if lower else np.triu(off, 1)) + np.diag(d)
    junk = rng.standard_normal((n, n))
    full = L + (np.triu(junk, 1) if lower else np.tril(junk, -1))
    return L, full


def ref_solve(L, Bm, side, trans, alpha):
    op = L if trans == 0 else (L.T if trans == 1 else L.conj().T)
    low = np.allclose(np.triu(op, 1), 0)
    if side == 0:
        return alpha * sla.solve_triangular(op, Bm, lower=low)
    # X op = B  <=>  op^T X^T = B^T
    return alpha * sla.solve_triangular(op.T, Bm.T, lower=not low).T


def run(handle, mode, steps, side, uplo, trans, m, n, cplx, seed, alpha):
    rng = np.random.default_rng(seed)
    na = m if side == 0 else n
    L, full = tri(na, uplo == 1, rng, cplx)
    dt = np.complex64 if cplx else np.float32
    Bm = rng.uniform(-1, 1, (m, n))
    if cplx:
        Bm = Bm + 1j * rng.uniform(-1, 1, (m, n))
    A32 = np.asfortranarray(full.astype(dt))
    B32 = np.asfortranarray(Bm.astype(dt))
    # reference on the FP32-rounded inputs
    Lr = A32.astype(np.complex128 if cplx else np.float64)
    Lr = np.tril(Lr) if uplo == 1 else np.triu(Lr)
    X64 = ref_solve(Lr, B32.astype(Lr.dtype), side, trans, alpha)
    a = A32.reshape(-1, order="F").copy()
    b = B32.reshape(-1, order="F").copy()
    handle.set_math_mode(mode)
    handle.set_trsm_refinement(steps)
    call = B.iclblasCtrsm if cplx else B.iclblasStrsm
    assert call(handle, side, uplo, trans, 0, m, n, alpha, a, na, b, m) == B.SUCCESS
    handle.set_trsm_refinement(0)
    X = b.reshape(m, n, order="F")
    return np.linalg.norm(X - X64) / np.linalg.norm(X64)


CASES = [(0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 2)]


@pytest.mark.parametrize("side,uplo,trans", CASES)
def test_strsm_3xbf16_one_step(handle, side, uplo, trans):
    m, n = (1100, 96) if side == 0 else (96, 1100)
    e0 = run(handle, B.MATH_BF16X3, 0, side, uplo, trans, m, n, False, 5 + trans, 1.0)
    e1 = run(handle, B.MATH_BF16X3, 1, side, uplo, trans, m, n, False, 5 + trans, 1.0)
    assert e1 <= 1e-6, (e0, e1)
    assert e1 < e0 / 3, (e0, e1)


def test_strsm_tf32_two_steps_alpha(handle):
    e2 = run(handle, B.MATH_TF32, 2, 0, 1, 0, 700, 50, False, 11, -0.75)
    assert e2 <= 1e-6, e2


def test_strsm_plain_one_step(handle):
    e1 = run(handle, B.MATH_PLAIN_FP32, 1, 0, 0, 1, 520, 33, False, 12, 2.0)
    assert e1 <= 1e-5, e1


@pytest.mark.parametrize("side,uplo,trans", [(0, 0, 2), (1, 1, 0)])
def test_ctrsm_3xbf16_one_step(handle, side, uplo, trans):
    m, n = (600, 40) if side == 0 else (40, 600)
    e1 = run(handle, B.MATH_BF16X3, 1, side, uplo, trans, m, n, True, 21, 0.5 - 0.25j)
    assert e1 <= 1e-6, e1


def test_refinement_setting_validated(handle):
    assert B.lib().iclblasSetTrsmRefinement(handle.value, 3) == B.INVALID_VALUE
    assert B.lib().iclblasSetTrsmRefinement(handle.value, -1) == B.INVALID_VALUE
