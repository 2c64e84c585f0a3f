"""Largest sizes the int-typed API admits: vectors of n = 2^31 - 1 elements
and a GEMV whose matrix has more than 2^31 elements, in device memory (about
26 GB at most at a time).  Inputs are chosen so the exact results are known:
the tests catch 32-bit index arithmetic anywhere on these paths."""
import numpy as np
import pytest
import torch

from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu

NMAX = 2**31 - 1


@pytest.fixture
def big_ones(cuda):
    x = torch.ones(NMAX, dtype=torch.float32, device=cuda)
    yield x
    del x
    torch.cuda.empty_cache()


def test_sasum_snrm2_sdot_at_int_max(handle, cuda, big_ones):
    handle.set_stream(torch.cuda.current_stream())
    r = torch.zeros(1, device=cuda)
    assert B.iclblasSasum(handle, NMAX, big_ones, 1, r) == B.SUCCESS
    assert r.item() == np.float32(float(NMAX))          # exact FP64 sum, one rounding
    assert B.iclblasSnrm2(handle, NMAX, big_ones, 1, r) == B.SUCCESS
    assert r.item() == np.float32(np.sqrt(float(NMAX)))
    assert B.iclblasSdot(handle, NMAX, big_ones, 1, big_ones, 1, r) == B.SUCCESS
    assert r.item() == np.float32(float(NMAX))


def test_isamax_at_int_max(handle, cuda, big_ones):
    handle.set_stream(torch.cuda.current_stream())
    ri = torch.zeros(1, dtype=torch.int32, device=cuda)
    big_ones[NMAX - 1] = -3.0
    assert B.iclblasIsamax(handle, NMAX, big_ones, 1, ri) == B.SUCCESS
    assert ri.item() == NMAX - 1                          # 0-based, last element
    big_ones[NMAX - 7] = 3.0                              # tie: the first index wins
    assert B.iclblasIsamax(handle, NMAX, big_ones, 1, ri) == B.SUCCESS
    assert ri.item() == NMAX - 7


def test_saxpy_sscal_at_int_max(handle, cuda, big_ones):
    handle.set_stream(torch.cuda.current_stream())
    y = torch.full((NMAX,), 2.0, dtype=torch.float32, device=cuda)
    assert B.iclblasSaxpy(handle, NMAX, 0.5, big_ones, 1, y, 1) == B.SUCCESS
    assert B.iclblasSscal(handle, NMAX, 4.0, y, 1) == B.SUCCESS
    torch.cuda.synchronize()
    assert y[0].item() == 10.0 and y[NMAX - 1].item() == 10.0 and y[NMAX // 2 + 3].item() == 10.0
    assert torch.count_nonzero(y != 10.0).item() == 0
    del y


def test_sgemv_matrix_above_2_pow_31_elements(handle, cuda):
    handle.set_stream(torch.cuda.current_stream())
    m, n = 65536, 32769                                    # m*n > 2^31
    A = torch.ones(m * n, dtype=torch.float32, device=cuda)
    A[(n - 1) * m:] = 2.0                                  # last column twice as large
    x = torch.ones(n, device=cuda)
    y = torch.zeros(m, device=cuda)
    assert B.iclblasSgemv(handle, 0, m, n, 1.0, A, m, x, 1, 0.0, y, 1) == B.SUCCESS
    torch.cuda.synchronize()
    assert torch.all(y == float(n + 1)).item()
    xt = torch.ones(m, device=cuda)
    yt = torch.zeros(n, device=cuda)
    assert B.iclblasSgemv(handle, 1, m, n, 1.0, A, m, xt, 1, 0.0, yt, 1) == B.SUCCESS
    torch.cuda.synchronize()
    assert torch.all(yt[: n - 1] == float(m)).item() and yt[n - 1].item() == 2.0 * m
    del A
    torch.cuda.empty_cache()
