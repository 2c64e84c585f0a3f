"""Large elementwise calls with host operands run as a chunked pipeline
(each chunk's output copied back while the next chunk's inputs are copied
in).  Their results must equal the all-device call's bit for bit (the same
elementwise kernels), including strided operands, whose gap elements stay
untouched."""
import numpy as np
import pytest
import torch

from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu

N = (1 << 25) + 5   # above the pipelining threshold, not a multiple of the chunk


@pytest.mark.parametrize("incx,incy", [(1, 1), (2, 3)])
def test_saxpy_host_pipelined_equals_device(handle, cuda, incx, incy):
    rng = np.random.default_rng(incx + 10 * incy)
    x = rng.uniform(-1, 1, (N - 1) * incx + 1).astype(np.float32)
    y = rng.uniform(-1, 1, (N - 1) * incy + 1).astype(np.float32)
    yd = torch.from_numpy(y).to(cuda)
    xd = torch.from_numpy(x).to(cuda)
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasSaxpy(handle, N, 0.75, xd, incx, yd, incy) == B.SUCCESS
    torch.cuda.synchronize()
    yh = y.copy()
    assert B.iclblasSaxpy(handle, N, 0.75, x, incx, yh, incy) == B.SUCCESS   # host operands: pipelined
    assert np.array_equal(yh, yd.cpu().numpy())
    if incy > 1:   # gap elements untouched
        gaps = np.ones(yh.size, bool)
        gaps[::incy] = False
        assert np.array_equal(yh[gaps], y[gaps])


def test_sscal_host_pipelined_equals_device(handle, cuda):
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, N).astype(np.float32)
    xd = torch.from_numpy(x).to(cuda)
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasSscal(handle, N, -1.5, xd, 1) == B.SUCCESS
    xh = x.copy()
    assert B.iclblasSscal(handle, N, -1.5, xh, 1) == B.SUCCESS
    assert np.array_equal(xh, xd.cpu().numpy())


def test_caxpy_and_cscal_host_pipelined_equal_device(handle, cuda):
    rng = np.random.default_rng(4)
    x = (rng.uniform(-1, 1, N) + 1j * rng.uniform(-1, 1, N)).astype(np.complex64)
    y = (rng.uniform(-1, 1, N) + 1j * rng.uniform(-1, 1, N)).astype(np.complex64)
    xd = torch.from_numpy(x.view(np.float32)).to(cuda)
    yd = torch.from_numpy(y.view(np.float32)).to(cuda)
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasCaxpy(handle, N, 0.5 - 0.25j, xd, 1, yd, 1) == B.SUCCESS
    assert B.iclblasCscal(handle, N, 1.25 + 0.5j, yd, 1) == B.SUCCESS
    yh = y.copy()
    assert B.iclblasCaxpy(handle, N, 0.5 - 0.25j, x, 1, yh, 1) == B.SUCCESS
    assert B.iclblasCscal(handle, N, 1.25 + 0.5j, yh, 1) == B.SUCCESS
    assert np.array_equal(yh.view(np.float32), yd.cpu().numpy())


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
