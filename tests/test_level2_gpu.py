"""Level-2 parity on the GPU (GEMV, TRSV; float and complex) against the oracle.

Tolerance: relative Frobenius error <= 1e-5 against the oracle (FP64
accumulation), the parity bar for floating-point routines; the kernels
accumulate in FP32 in a different order, so exact equality is not expected.
"""
import numpy as np
import pytest

import oracle_lib as O
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu
TOL = 1e-5

GEMV_SHAPES = [(1, 1), (7, 5), (64, 64), (1000, 37), (37, 1000), (4097, 513), (513, 4099)]


def _vec(n, inc, rng, dtype):
    return O.colmajor(n * inc, 1, n * inc, rng, dtype)


@pytest.mark.parametrize("m,n", GEMV_SHAPES)
@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("beta", [0.0, -0.5])
def test_sgemv(handle, m, n, trans, beta):
    rng = np.random.default_rng(m * 31 + n + trans)
    for lda, inc in ((m, 1), (m + 3, 2)):
        A = O.colmajor(m, n, lda, rng)
        xl, yl = (n, m) if trans == 0 else (m, n)
        x = _vec(xl, inc, rng, np.float32)
        y = _vec(yl, inc, rng, np.float32)
        if beta == 0.0:
            y[::inc] = np.nan  # y must not be read
        y_ref = y.copy()
        O.sgemv(trans, m, n, 1.25, A, lda, x, inc, beta, y_ref, inc)
        assert B.iclblasSgemv(handle, trans, m, n, 1.25, A, lda, x, inc, beta, y, inc) == B.SUCCESS
        assert np.all(np.isfinite(y[::inc][:yl]))
        assert O.rel_fro(y, y_ref) <= TOL


@pytest.mark.parametrize("m,n", GEMV_SHAPES)
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_cgemv(handle, m, n, trans):
    rng = np.random.default_rng(m * 17 + n + trans)
    for lda, inc, beta in ((m, 1, 0.5 - 0.25j), (m + 1, 2, 0.0)):
        A = O.colmajor(m, n, lda, rng, np.complex64)
        xl, yl = (n, m) if trans == 0 else (m, n)
        x = _vec(xl, inc, rng, np.complex64)
        y = _vec(yl, inc, rng, np.complex64)
        y_ref = y.copy()
        O.cgemv(trans, m, n, 1 + 0.5j, A, lda, x, inc, beta, y_ref, inc)
        assert B.iclblasCgemv(handle, trans, m, n, 1 + 0.5j, A, lda, x, inc, beta, y, inc) == B.SUCCESS
        assert O.rel_fro(y, y_ref) <= TOL


def test_sgemv_16384_both_ops(handle):
    """The bandwidth config's SGEMV (16384^2, N and T) at full size."""
    n = 16384
    rng = np.random.default_rng(1)
    A = rng.uniform(-1, 1, n * n).astype(np.float32)
    for trans in (0, 1):
        x = rng.uniform(-1, 1, n).astype(np.float32)
        y = rng.uniform(-1, 1, n).astype(np.float32)
        y_ref = y.copy()
        O.sgemv(trans, n, n, 1.0, A, n, x, 1, 1.0, y_ref, 1)
        assert B.iclblasSgemv(handle, trans, n, n, 1.0, A, n, x, 1, 1.0, y, 1) == B.SUCCESS
        assert O.rel_fro(y, y_ref) <= TOL


def tri(n, lda, lower, rng, dtype=np.float32):
    """Triangle with |diag| in [1, 2] and off-diagonal N(0,1)/sqrt(n) (the
    STRSM/STRSV config's construction); the other triangle holds junk."""
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


TRSV_SIZES = [1, 5, 64, 65, 200, 1000, 4100]


@pytest.mark.parametrize("n", TRSV_SIZES)
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("diag", [0, 1])
def test_strsv(handle, n, uplo, trans, diag):
    rng = np.random.default_rng(n * 13 + 6 * uplo + 2 * trans + diag)
    for lda, inc in ((n, 1), (n + 2, 3)):
        A = tri(n, lda, uplo == 1, rng)
        x = rng.uniform(-1, 1, n * inc).astype(np.float32)
        x_ref = x.copy()
        O.strsv(uplo, trans, diag, n, A, lda, x_ref, inc)
        assert B.iclblasStrsv(handle, uplo, trans, diag, n, A, lda, x, inc) == B.SUCCESS
        assert O.rel_fro(x, x_ref) <= TOL


@pytest.mark.parametrize("n", [1, 33, 64, 300, 2050])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_ctrsv(handle, n, uplo, trans):
    rng = np.random.default_rng(n * 5 + uplo + 2 * trans)
    A = tri(n, n + 1, uplo == 1, rng, np.complex64)
    x = O.colmajor(n, 1, n, rng, np.complex64)
    for diag in (0, 1):
        x1 = x.copy()
        x_ref = x.copy()
        O.ctrsv(uplo, trans, diag, n, A, n + 1, x_ref, 1)
        assert B.iclblasCtrsv(handle, uplo, trans, diag, n, A, n + 1, x1, 1) == B.SUCCESS
        assert O.rel_fro(x1, x_ref) <= TOL


def test_strsv_16384_lower(handle):
    """The STRSV config: n = 16384, lower, no-trans, non-unit."""
    n = 16384
    rng = np.random.default_rng(3)
    A = tri(n, n, True, rng)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    x_ref = x.copy()
    O.strsv(1, 0, 0, n, A, n, x_ref, 1)
    assert B.iclblasStrsv(handle, 1, 0, 0, n, A, n, x, 1) == B.SUCCESS
    assert O.rel_fro(x, x_ref) <= TOL


def test_trsv_device_pointers(handle, cuda):
    import torch
    handle.set_stream(torch.cuda.current_stream())
    n = 3000
    rng = np.random.default_rng(9)
    A = tri(n, n, False, rng)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    x_ref = x.copy()
    O.strsv(0, 1, 0, n, A, n, x_ref, 1)
    Ad = torch.from_numpy(A).to(cuda)
    xd = torch.from_numpy(x).to(cuda)
    assert B.iclblasStrsv(handle, 0, 1, 0, n, Ad, n, xd, 1) == B.SUCCESS
    assert handle.synchronize() == B.SUCCESS
    assert O.rel_fro(xd.cpu().numpy(), x_ref) <= TOL


@pytest.mark.parametrize("n", [64, 130, 2048, 3001])
@pytest.mark.parametrize("uplo,trans", [(0, 0), (1, 0), (0, 1), (1, 2)])
def test_strsv_tma_path_padded_lda(handle, n, uplo, trans):
    """lda a multiple of 4 above n (the TMA-staged path), stride 2, three
    calls in a row on one handle (each call a new epoch)."""
    rng = np.random.default_rng(n + 7 * uplo + trans)
    lda = (n + 4 + 3) // 4 * 4
    for diag in (0, 1, 0):
        A = tri(n, lda, uplo == 1, rng)
        x = rng.uniform(-1, 1, 2 * n).astype(np.float32)
        x_ref = x.copy()
        O.strsv(uplo, trans, diag, n, A, lda, x_ref, 2)
        assert B.iclblasStrsv(handle, uplo, trans, diag, n, A, lda, x, 2) == B.SUCCESS
        assert O.rel_fro(x, x_ref) <= TOL
        assert np.array_equal(x[1::2], x_ref[1::2])   # entries between the strided ones untouched


def test_strsv_replayed_in_cuda_graph(handle, cuda):
    """A captured STRSV replayed several times gives the eager result each time
    (the publication epoch advances on the device, not at capture)."""
    import torch
    n = 5000
    rng = np.random.default_rng(21)
    A = tri(n, n, True, rng)
    x0 = rng.uniform(-1, 1, n).astype(np.float32)
    x_ref = x0.copy()
    O.strsv(1, 0, 0, n, A, n, x_ref, 1)
    Ad = torch.from_numpy(A).to(cuda)
    x0d = torch.from_numpy(x0).to(cuda)
    xw = x0d.clone()
    # first call outside capture (sizes the handle's buffers)
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasStrsv(handle, 1, 0, 0, n, Ad, n, xw, 1) == B.SUCCESS
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    handle.set_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        xw.copy_(x0d)
        st = B.iclblasStrsv(handle, 1, 0, 0, n, Ad, n, xw, 1)
    assert st == B.SUCCESS
    for _ in range(3):
        xw.fill_(7.0)
        g.replay()
        torch.cuda.synchronize()
        assert O.rel_fro(xw.cpu().numpy(), x_ref) <= TOL
    handle.set_stream(torch.cuda.current_stream())
    del g
