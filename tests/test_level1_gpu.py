"""Level-1 parity on the GPU: the library (through its C ABI) against the oracle.

Bars: iamax bit-exact (index work); scal and complex axpy/scal bit-exact
(same double arithmetic as the oracle, one rounding); real axpy within 1 ulp
(fma vs the oracle's double-then-float rounding); dot/nrm2/asum (and complex
variants) within 1 ulp of the double-accumulated oracle (different summation
order of the same double sums).
"""
import numpy as np
import pytest

import oracle_lib as O
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 5, 64, 1000, 4097, 65537, (1 << 20) + 3]


def _ulp_ok(got, want, ulps=1):
    return int(O.ulp_diff(np.float32(got), np.float32(want)).max()) <= ulps


def _cnear(got, want, scale):
    # each component within 1 ulp of its value or of the terms' magnitude
    tol = 2.0 ** -23 * max(abs(want.real), abs(want.imag), 1e-30) + 1e-12 * scale
    return abs(got.real - want.real) <= tol and abs(got.imag - want.imag) <= tol


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [1, 3])
def test_real_reductions_host(handle, n, inc):
    rng = np.random.default_rng(n * 7 + inc)
    x = rng.uniform(-1, 1, n * inc).astype(np.float32)
    y = rng.uniform(-1, 1, n * inc).astype(np.float32)
    r = np.zeros(1, np.float32)
    assert B.iclblasSdot(handle, n, x, inc, y, inc, r) == B.SUCCESS
    assert _ulp_ok(r[0], O.sdot(n, x, inc, y, inc))
    assert B.iclblasSnrm2(handle, n, x, inc, r) == B.SUCCESS
    assert _ulp_ok(r[0], O.snrm2(n, x, inc))
    assert B.iclblasSasum(handle, n, x, inc, r) == B.SUCCESS
    assert _ulp_ok(r[0], O.sasum(n, x, inc))
    ri = np.zeros(1, np.int32)
    assert B.iclblasIsamax(handle, n, x, inc, ri) == B.SUCCESS
    assert ri[0] == O.isamax(n, x, inc)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [1, 2])
def test_axpy_scal_host(handle, n, inc):
    rng = np.random.default_rng(n + 100 * inc)
    x = rng.uniform(-1, 1, n * inc).astype(np.float32)
    y = rng.uniform(-1, 1, n * inc).astype(np.float32)
    y_ref = y.copy()
    O.saxpy(n, 0.37, x, inc, y_ref, inc)
    assert B.iclblasSaxpy(handle, n, 0.37, x, inc, y, inc) == B.SUCCESS
    assert O.ulp_diff(y, y_ref).max() <= 1
    x_ref = x.copy()
    O.sscal(n, -1.75, x_ref, inc)
    assert B.iclblasSscal(handle, n, -1.75, x, inc) == B.SUCCESS
    assert np.array_equal(x, x_ref)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [1, 2])
def test_complex_level1_host(handle, n, inc):
    rng = np.random.default_rng(n * 3 + inc)
    x = O.colmajor(n * inc, 1, n * inc, rng, np.complex64)
    y = O.colmajor(n * inc, 1, n * inc, rng, np.complex64)
    r = np.zeros(1, np.complex64)
    scale = float(np.sum(np.abs(x[::inc][:n]) * np.abs(y[::inc][:n])))
    assert B.iclblasCdotu(handle, n, x, inc, y, inc, r) == B.SUCCESS
    assert _cnear(complex(r[0]), O.cdot(n, x, inc, y, inc, False), scale)
    assert B.iclblasCdotc(handle, n, x, inc, y, inc, r) == B.SUCCESS
    assert _cnear(complex(r[0]), O.cdot(n, x, inc, y, inc, True), scale)
    rf = np.zeros(1, np.float32)
    assert B.iclblasScnrm2(handle, n, x, inc, rf) == B.SUCCESS
    assert _ulp_ok(rf[0], O.scnrm2(n, x, inc))
    assert B.iclblasScasum(handle, n, x, inc, rf) == B.SUCCESS
    assert _ulp_ok(rf[0], O.scasum(n, x, inc))
    ri = np.zeros(1, np.int32)
    assert B.iclblasIcamax(handle, n, x, inc, ri) == B.SUCCESS
    assert ri[0] == O.icamax(n, x, inc)
    a = 0.3 - 0.8j
    y_ref = y.copy()
    O.caxpy(n, a, x, inc, y_ref, inc)
    assert B.iclblasCaxpy(handle, n, a, x, inc, y, inc) == B.SUCCESS
    assert np.array_equal(y, y_ref)
    x_ref = x.copy()
    O.cscal(n, a, x_ref, inc)
    assert B.iclblasCscal(handle, n, a, x, inc) == B.SUCCESS
    assert np.array_equal(x, x_ref)
    x_ref = x.copy()
    O.cscal(n, 2.5, x_ref, inc)
    assert B.iclblasCsscal(handle, n, 2.5, x, inc) == B.SUCCESS
    assert np.array_equal(x, x_ref)


def test_device_pointers_and_misaligned(handle, cuda):
    """Device (torch) operands run asynchronously on the handle's stream;
    an operand offset by one element takes the scalar (unaligned) path."""
    import torch
    handle.set_stream(torch.cuda.current_stream())
    n = 300001
    rng = np.random.default_rng(5)
    xh = rng.uniform(-1, 1, n + 1).astype(np.float32)
    yh = rng.uniform(-1, 1, n + 1).astype(np.float32)
    x = torch.from_numpy(xh).to(cuda)
    y = torch.from_numpy(yh).to(cuda)
    r = torch.zeros(1, dtype=torch.float32, device=cuda)
    ri = torch.zeros(1, dtype=torch.int32, device=cuda)
    for off in (0, 1):
        xv, yv = x[off:off + n], y[off:off + n]
        assert B.iclblasSdot(handle, n, xv, 1, yv, 1, r) == B.SUCCESS
        torch.cuda.synchronize()
        assert _ulp_ok(r.item(), O.sdot(n, xh[off:off + n], 1, yh[off:off + n], 1))
        assert B.iclblasIsamax(handle, n, xv, 1, ri) == B.SUCCESS
        torch.cuda.synchronize()
        assert ri.item() == O.isamax(n, xh[off:off + n], 1)
    yd = y.clone()
    assert B.iclblasSaxpy(handle, n, 1.25, x[1:], 1, yd[1:], 1) == B.SUCCESS
    torch.cuda.synchronize()
    y_ref = yh.copy()
    O.saxpy(n, 1.25, xh[1:], 1, y_ref[1:], 1)
    assert O.ulp_diff(yd.cpu().numpy(), y_ref).max() <= 1


def test_isamax_ties_nan_edges(handle):
    r = np.zeros(1, np.int32)
    x = np.array([1, -5, 3, 5, -5, 2], np.float32)
    assert B.iclblasIsamax(handle, 6, x, 1, r) == B.SUCCESS and r[0] == 1
    x = np.array([np.nan, 1, 7, 2, 9], np.float32)
    assert B.iclblasIsamax(handle, 5, x, 1, r) == B.SUCCESS and r[0] == 0
    x = np.array([1, np.nan, 7, 2, 7], np.float32)
    assert B.iclblasIsamax(handle, 5, x, 1, r) == B.SUCCESS and r[0] == 2
    x = np.zeros(1000, np.float32)
    assert B.iclblasIsamax(handle, 1000, x, 1, r) == B.SUCCESS and r[0] == 0
    x = np.full(77, -0.0, np.float32)
    x[40] = 0.0
    assert B.iclblasIsamax(handle, 77, x, 1, r) == B.SUCCESS and r[0] == 0
    # reference C-API case: 0-based index of the planted max (test_Isamax.cpp:18-47)
    x = np.arange(256, dtype=np.float32)
    x[47] = 666.0
    assert B.iclblasIsamax(handle, 256, x, 1, r) == B.SUCCESS and r[0] == 47


def test_full_size_isamax_ties_2_28(handle):
    """n = 2^28 (the bandwidth config): a planted maximum and a later tie must
    give the first index exactly; the reference's float-encoded index is inexact
    above 2^24, this path is not."""
    n = 1 << 28
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    i1, i2 = (1 << 24) + 12345, n - 7
    x[i1] = -3.5
    x[i2] = 3.5
    r = np.zeros(1, np.int32)
    assert B.iclblasIsamax(handle, n, x, 1, r) == B.SUCCESS
    assert r[0] == i1 == O.isamax(n, x, 1)
    rf = np.zeros(1, np.float32)
    y = rng.uniform(-1, 1, n).astype(np.float32)
    assert B.iclblasSdot(handle, n, x, 1, y, 1, rf) == B.SUCCESS
    assert _ulp_ok(rf[0], O.sdot(n, x, 1, y, 1))
