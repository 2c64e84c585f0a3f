"""Host operands, in both kinds of host memory a caller can pass.

Pinned (page-locked) memory: large elementwise calls run as a chunked
pipeline (each chunk's output copied back while the next chunk's inputs are
copied in).  Ordinary (pageable) memory, what a caller of the reference's API
passes: operands of 4 MiB and more move through the handle's two pinned
bounce buffers, host-side copies of one chunk overlapping the DMA of the
other.  Either way the results must equal the all-device call's bit for bit
(the same kernels), including strided operands, whose gap elements stay
untouched, and outputs larger than a bounce buffer.  GEMM and GEMV with
beta == 0 do not copy a contiguous C / y in (NaN there must not leak into
the result)."""
import numpy as np
import pytest
import torch

from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu

N = (1 << 25) + 5   # above the pipelining threshold, not a multiple of the chunk


def host(a: np.ndarray, mem: str):
    """a in pinned (a page-locked torch tensor) or pageable (numpy) memory."""
    return torch.from_numpy(a).pin_memory() if mem == "pinned" else a


def back(h) -> np.ndarray:
    return h.numpy() if isinstance(h, torch.Tensor) else h


@pytest.mark.parametrize("mem", ["pinned", "pageable"])
@pytest.mark.parametrize("incx,incy", [(1, 1), (2, 3)])
def test_saxpy_host_equals_device(handle, cuda, mem, incx, incy):
    rng = np.random.default_rng(incx + 10 * incy)
    x = rng.uniform(-1, 1, (N - 1) * incx + 1).astype(np.float32)
    y = rng.uniform(-1, 1, (N - 1) * incy + 1).astype(np.float32)
    yd = torch.from_numpy(y).to(cuda)
    xd = torch.from_numpy(x).to(cuda)
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasSaxpy(handle, N, 0.75, xd, incx, yd, incy) == B.SUCCESS
    torch.cuda.synchronize()
    yh = host(y.copy(), mem)
    assert B.iclblasSaxpy(handle, N, 0.75, host(x, mem), incx, yh, incy) == B.SUCCESS
    yh = back(yh)
    assert np.array_equal(yh, yd.cpu().numpy())
    if incy > 1:   # gap elements untouched
        gaps = np.ones(yh.size, bool)
        gaps[::incy] = False
        assert np.array_equal(yh[gaps], y[gaps])


@pytest.mark.parametrize("mem", ["pinned", "pageable"])
def test_sscal_host_equals_device(handle, cuda, mem):
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, N).astype(np.float32)
    xd = torch.from_numpy(x).to(cuda)
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasSscal(handle, N, -1.5, xd, 1) == B.SUCCESS
    xh = host(x.copy(), mem)
    assert B.iclblasSscal(handle, N, -1.5, xh, 1) == B.SUCCESS
    assert np.array_equal(back(xh), xd.cpu().numpy())


@pytest.mark.parametrize("mem", ["pinned", "pageable"])
def test_caxpy_and_cscal_host_equal_device(handle, cuda, mem):
    rng = np.random.default_rng(4)
    x = (rng.uniform(-1, 1, N) + 1j * rng.uniform(-1, 1, N)).astype(np.complex64)
    y = (rng.uniform(-1, 1, N) + 1j * rng.uniform(-1, 1, N)).astype(np.complex64)
    xd = torch.from_numpy(x.view(np.float32)).to(cuda)
    yd = torch.from_numpy(y.view(np.float32)).to(cuda)
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasCaxpy(handle, N, 0.5 - 0.25j, xd, 1, yd, 1) == B.SUCCESS
    assert B.iclblasCscal(handle, N, 1.25 + 0.5j, yd, 1) == B.SUCCESS
    xh = host(x.view(np.float32).copy(), mem)
    yh = host(y.view(np.float32).copy(), mem)
    assert B.iclblasCaxpy(handle, N, 0.5 - 0.25j, xh, 1, yh, 1) == B.SUCCESS
    assert B.iclblasCscal(handle, N, 1.25 + 0.5j, yh, 1) == B.SUCCESS
    assert np.array_equal(back(yh), yd.cpu().numpy())


def test_mixed_device_x_host_y(handle, cuda):
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, N).astype(np.float32)
    y = rng.uniform(-1, 1, N).astype(np.float32)
    xd = torch.from_numpy(x).to(cuda)
    yd = torch.from_numpy(y).to(cuda)
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasSaxpy(handle, N, 2.0, xd, 1, yd, 1) == B.SUCCESS
    yh = y.copy()
    assert B.iclblasSaxpy(handle, N, 2.0, xd, 1, yh, 1) == B.SUCCESS   # only y staged
    assert np.array_equal(yh, yd.cpu().numpy())


def test_pageable_reductions_equal_device(handle, cuda):
    rng = np.random.default_rng(6)
    x = rng.uniform(-1, 1, N).astype(np.float32)
    y = rng.uniform(-1, 1, N).astype(np.float32)
    xd, yd = torch.from_numpy(x).to(cuda), torch.from_numpy(y).to(cuda)
    handle.set_stream(torch.cuda.current_stream())
    rd = torch.zeros(3, device=cuda)
    rid = torch.zeros(1, dtype=torch.int32, device=cuda)
    assert B.iclblasSdot(handle, N, xd, 1, yd, 1, rd[0:1]) == B.SUCCESS
    assert B.iclblasSnrm2(handle, N, xd, 1, rd[1:2]) == B.SUCCESS
    assert B.iclblasSasum(handle, N, xd, 1, rd[2:3]) == B.SUCCESS
    assert B.iclblasIsamax(handle, N, xd, 1, rid) == B.SUCCESS
    torch.cuda.synchronize()
    r = np.zeros(3, np.float32)
    ri = np.zeros(1, np.int32)
    assert B.iclblasSdot(handle, N, x, 1, y, 1, r[0:1]) == B.SUCCESS
    assert B.iclblasSnrm2(handle, N, x, 1, r[1:2]) == B.SUCCESS
    assert B.iclblasSasum(handle, N, x, 1, r[2:3]) == B.SUCCESS
    assert B.iclblasIsamax(handle, N, x, 1, ri) == B.SUCCESS
    assert np.array_equal(r, rd.cpu().numpy())
    assert ri[0] == rid.item()


@pytest.mark.parametrize("trans", [0, 1])
def test_pageable_sgemv_equals_device_beta0_nan_y(handle, cuda, trans):
    m, n = 6000, 3000                        # A: 72 MB, two bounce buffers' worth
    rng = np.random.default_rng(7 + trans)
    A = rng.uniform(-1, 1, m * n).astype(np.float32)
    xl, yl = (n, m) if trans == 0 else (m, n)
    x = rng.uniform(-1, 1, xl).astype(np.float32)
    yd = torch.zeros(yl, device=cuda)
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasSgemv(handle, trans, m, n, 1.25, torch.from_numpy(A).to(cuda), m, torch.from_numpy(x).to(cuda),
                          1, 0.0, yd, 1) == B.SUCCESS
    torch.cuda.synchronize()
    y = np.full(yl, np.nan, np.float32)      # beta == 0: not copied in, not read
    assert B.iclblasSgemv(handle, trans, m, n, 1.25, A, m, x, 1, 0.0, y, 1) == B.SUCCESS
    assert np.array_equal(y, yd.cpu().numpy())


@pytest.mark.parametrize("ldc_pad", [0, 3])
def test_pageable_sgemm_beta0_large_c(handle, cuda, ldc_pad):
    """C of 2304 x 2304 (21 MB): copied out through both bounce buffers; beta
    == 0 with NaN in C: with ldc == m C is not copied in at all, with padded
    rows it is (the gap rows must come back untouched)."""
    m, k = 2304, 64
    ldc = m + ldc_pad
    rng = np.random.default_rng(8 + ldc_pad)
    A = rng.uniform(-1, 1, m * k).astype(np.float32)
    Bm = rng.uniform(-1, 1, k * m).astype(np.float32)
    Cd = torch.zeros(ldc * m, device=cuda)
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasSgemm(handle, 0, 0, m, m, k, 1.0, torch.from_numpy(A).to(cuda), m, torch.from_numpy(Bm).to(cuda),
                          k, 0.0, Cd, ldc) == B.SUCCESS
    torch.cuda.synchronize()
    C = np.full(ldc * m, np.nan, np.float32)
    assert B.iclblasSgemm(handle, 0, 0, m, m, k, 1.0, A, m, Bm, k, 0.0, C, ldc) == B.SUCCESS
    Cm, Cdm = C.reshape(m, ldc), Cd.cpu().numpy().reshape(m, ldc)
    assert np.array_equal(Cm[:, :m], Cdm[:, :m])
    assert np.all(np.isnan(Cm[:, m:]))       # the gap rows: untouched


def test_pageable_strsm_equals_device(handle, cuda):
    m, n = 1500, 1200                        # B: 7.2 MB in and out through the bounce buffers
    rng = np.random.default_rng(9)
    L = np.tril(rng.standard_normal((m, m)) / np.sqrt(m), -1) + np.diag(rng.uniform(1, 2, m))
    A = np.ascontiguousarray(L.T, dtype=np.float32).reshape(-1)
    Bm = rng.uniform(-1, 1, m * n).astype(np.float32)
    Bd = torch.from_numpy(Bm).to(cuda)
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasStrsm(handle, 0, 1, 0, 0, m, n, 0.5, torch.from_numpy(A).to(cuda), m, Bd, m) == B.SUCCESS
    torch.cuda.synchronize()
    Bh = Bm.copy()
    assert B.iclblasStrsm(handle, 0, 1, 0, 0, m, n, 0.5, A, m, Bh, m) == B.SUCCESS
    assert np.array_equal(Bh, Bd.cpu().numpy())
