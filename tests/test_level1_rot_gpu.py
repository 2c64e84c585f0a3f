"""Copy, swap, plane rotations, iamin and the rotation generators on the GPU:
the library (through its C ABI) against the oracle, bit-exact.

The oracle restates the reference kernels' FP32 expressions with their fused
multiply-adds (pinned to those kernels in tests/test_oracle_rot.py), and the
CUDA kernels evaluate the same expressions, so every output must match to the
bit; iamin is index work and must match exactly.
"""
import numpy as np
import pytest

import oracle_lib as O
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 5, 64, 1000, 4097, 65537, (1 << 20) + 3]


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def same(a, b):
    """Bit-identical, except that any two NaNs match (the GPU writes a
    canonical NaN where the CPU propagates its operand's payload)."""
    fa = np.ascontiguousarray(a).view(np.float32)
    fb = np.ascontiguousarray(b).view(np.float32)
    return fa.shape == fb.shape and bool(np.all((bits(fa) == bits(fb)) | (np.isnan(fa) & np.isnan(fb))))


def vec(rng, n, dtype, scale=4.0):
    if np.dtype(dtype) == np.complex64:
        return rng.uniform(-scale, scale, (n, 2)).astype(np.float32).view(np.complex64).reshape(-1)
    return rng.uniform(-scale, scale, n).astype(np.float32)


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


# ------------------------------------------------------------------ copy / swap
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dtype", [np.float32, np.complex64])
@pytest.mark.parametrize("incx,incy", [(1, 1), (2, 3)])
def test_copy_swap_host(handle, n, dtype, incx, incy):
    rng = np.random.default_rng(n + incx)
    x = vec(rng, n * incx, dtype)
    y = vec(rng, n * incy, dtype)
    cp = B.iclblasScopy if dtype == np.float32 else B.iclblasCcopy
    sw = B.iclblasSswap if dtype == np.float32 else B.iclblasCswap
    y1, yr = y.copy(), y.copy()
    O.copy(n, x, incx, yr, incy)
    assert cp(handle, n, x, incx, y1, incy) == B.SUCCESS
    assert same(y1, yr)
    x1, y1, xr, yr = x.copy(), y.copy(), x.copy(), y.copy()
    O.swap(n, xr, incx, yr, incy)
    assert sw(handle, n, x1, incx, y1, incy) == B.SUCCESS
    assert same(x1, xr) and same(y1, yr)


@pytest.mark.parametrize("offset", [0, 1, 2, 3])
def test_copy_swap_device_misaligned(handle, offset):
    """Device operands at every 4-byte offset: the 16-byte vector path only
    when both bases are aligned, the scalar path otherwise; same bits."""
    rng = np.random.default_rng(50 + offset)
    n = 100003
    x = vec(rng, n + 4, np.float32)
    y = vec(rng, n + 4, np.float32)
    dx, dy = dev(x), dev(y)
    yr = y.copy()
    O.copy(n, x[offset:], 1, yr[1:], 1)
    assert B.iclblasScopy(handle, n, dx[offset:], 1, dy[1:], 1) == B.SUCCESS
    assert same(host(dy), yr)
    xr, yr = x.copy(), host(dy).copy()
    dx, dy = dev(x), dev(yr)
    O.swap(n, xr[offset:], 1, yr[offset:], 1)
    assert B.iclblasSswap(handle, n, dx[offset:], 1, dy[offset:], 1) == B.SUCCESS
    assert same(host(dx), xr) and same(host(dy), yr)


def test_copy_swap_large_host_pipelined(handle):
    """Host vectors past the chunking threshold (2 x 2^24 elements): the
    pipelined staging path gives the same result as the whole call."""
    n = (1 << 25) + 12345
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n).astype(np.float32)
    y = rng.standard_normal(n).astype(np.float32)
    y1 = y.copy()
    assert B.iclblasScopy(handle, n, x, 1, y1, 1) == B.SUCCESS
    assert np.array_equal(y1, x)
    x1, y1 = x.copy(), y.copy()
    assert B.iclblasSswap(handle, n, x1, 1, y1, 1) == B.SUCCESS
    assert np.array_equal(x1, y) and np.array_equal(y1, x)
    x1, y1 = x.copy(), y.copy()
    xr, yr = x.copy(), y.copy()
    O.srot(n, xr, 1, yr, 1, 0.6, 0.8)
    assert B.iclblasSrot(handle, n, x1, 1, y1, 1, 0.6, 0.8) == B.SUCCESS
    assert same(x1, xr) and same(y1, yr)


# ------------------------------------------------------------------ rotations
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("incx,incy", [(1, 1), (1, 2), (3, 1)])
def test_rot_family_host(handle, n, incx, incy):
    rng = np.random.default_rng(7 * n + incx + 10 * incy)
    c, s = 0.6, -0.8
    x, y = vec(rng, n * incx, np.float32), vec(rng, n * incy, np.float32)
    x1, y1, xr, yr = x.copy(), y.copy(), x.copy(), y.copy()
    O.srot(n, xr, incx, yr, incy, c, s)
    assert B.iclblasSrot(handle, n, x1, incx, y1, incy, c, s) == B.SUCCESS
    assert same(x1, xr) and same(y1, yr)
    xc, yc = vec(rng, n * incx, np.complex64), vec(rng, n * incy, np.complex64)
    x1, y1, xr, yr = xc.copy(), yc.copy(), xc.copy(), yc.copy()
    O.csrot(n, xr, incx, yr, incy, c, s)
    assert B.iclblasCsrot(handle, n, x1, incx, y1, incy, c, s) == B.SUCCESS
    assert same(x1, xr) and same(y1, yr)
    sc = 0.25 - 0.5j
    x1, y1, xr, yr = xc.copy(), yc.copy(), xc.copy(), yc.copy()
    O.crot(n, xr, incx, yr, incy, 1.5, sc)
    assert B.iclblasCrot(handle, n, x1, incx, y1, incy, 1.5, sc) == B.SUCCESS
    assert same(x1, xr) and same(y1, yr)


@pytest.mark.parametrize("flag", [-1.0, 0.0, 1.0])
@pytest.mark.parametrize("n,inc", [(1, 1), (4097, 1), ((1 << 20) + 3, 1), (1000, 3)])
def test_rotm_host_and_device_param(handle, flag, n, inc):
    rng = np.random.default_rng(int(flag) + 5 + n)
    param = np.array([flag, 0.75, -1.5, 2.25, 0.125], np.float32)
    x, y = vec(rng, n * inc, np.float32), vec(rng, n * inc, np.float32)
    xr, yr = x.copy(), y.copy()
    O.srotm(n, xr, inc, yr, inc, param)
    x1, y1 = x.copy(), y.copy()
    assert B.iclblasSrotm(handle, n, x1, inc, y1, inc, param) == B.SUCCESS
    assert same(x1, xr) and same(y1, yr)
    dx, dy, dp = dev(x), dev(y), dev(param)
    assert B.iclblasSrotm(handle, n, dx, inc, dy, inc, dp) == B.SUCCESS
    assert same(host(dx), xr) and same(host(dy), yr)


@pytest.mark.parametrize("flag", [-2.0, 5.0, np.nan])
def test_rotm_identity_and_unknown_flags(handle, flag):
    rng = np.random.default_rng(1)
    n = 4099
    param = np.array([flag, 3, 3, 3, 3], np.float32)
    x, y = vec(rng, n, np.float32), vec(rng, n, np.float32)
    x1, y1 = x.copy(), y.copy()
    assert B.iclblasSrotm(handle, n, x1, 1, y1, 1, param) == B.SUCCESS
    assert same(x1, x) and same(y1, y)
    dx, dy, dp = dev(x), dev(y), dev(param)
    assert B.iclblasSrotm(handle, n, dx, 1, dy, 1, dp) == B.SUCCESS
    assert same(host(dx), x) and same(host(dy), y)


def test_rot_device_operands_and_stream_order(handle):
    """Device vectors: calls are asynchronous and run in stream order."""
    rng = np.random.default_rng(2)
    n = 1 << 20
    x, y = vec(rng, n, np.float32), vec(rng, n, np.float32)
    dx, dy = dev(x), dev(y)
    xr, yr = x.copy(), y.copy()
    for c, s in ((0.6, 0.8), (0.8, -0.6), (1.0, 0.25)):
        O.srot(n, xr, 1, yr, 1, c, s)
        assert B.iclblasSrot(handle, n, dx, 1, dy, 1, c, s) == B.SUCCESS
    handle.synchronize()
    assert same(host(dx), xr) and same(host(dy), yr)


# ------------------------------------------------------------------ iamin
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [1, 3])
def test_iamin_host(handle, n, inc):
    rng = np.random.default_rng(n + 31 * inc)
    x = vec(rng, n * inc, np.float32)
    xc = vec(rng, n * inc, np.complex64)
    ri = np.full(1, -7, np.int32)
    assert B.iclblasIsamin(handle, n, x, inc, ri) == B.SUCCESS and ri[0] == O.isamin(n, x, inc)
    assert B.iclblasIcamin(handle, n, xc, inc, ri) == B.SUCCESS and ri[0] == O.icamin(n, xc, inc)


def test_iamin_ties_nan_inf(handle):
    n = 300001
    base = np.full(n, 3.0, np.float32)
    cases = []
    a = base.copy(); a[[70000, 5, 299999]] = -0.5; cases.append(a)         # first of the ties
    a = base.copy(); a[0] = np.nan; a[9] = 0.0; cases.append(a)             # NaN first pins 0
    a = base.copy(); a[1] = np.nan; a[200000] = 0.25; cases.append(a)       # later NaN skipped
    a = np.full(n, np.inf, np.float32); cases.append(a)                    # nothing below x[0]
    a = np.full(n, np.inf, np.float32); a[123457] = 1e38; cases.append(a)
    a = base.copy(); a[299999] = -0.0; a[299998] = 0.0; cases.append(a)
    a = base.copy(); a[-3:] = 0.125; cases.append(a)                        # in the scalar tail
    ri = np.zeros(1, np.int32)
    for a in cases:
        assert B.iclblasIsamin(handle, n, a, 1, ri) == B.SUCCESS and ri[0] == O.isamin(n, a, 1)
        ac = a.astype(np.complex64)
        assert B.iclblasIcamin(handle, n, ac, 1, ri) == B.SUCCESS and ri[0] == O.icamin(n, ac, 1)
    # complex key is |re| + |im| (scabs1), not the modulus
    xc = np.array([3 + 0j, 2 + 2j, 0 + 2.5j], np.complex64)
    assert B.iclblasIcamin(handle, 3, xc, 1, ri) == B.SUCCESS and ri[0] == 2


def test_iamin_device_result(handle):
    rng = np.random.default_rng(4)
    n = 1 << 22
    x = vec(rng, n, np.float32)
    import torch
    r = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    assert B.iclblasIsamin(handle, n, dev(x), 1, r) == B.SUCCESS
    assert int(host(r)[0]) == O.isamin(n, x, 1)


# ------------------------------------------------------------------ generators
def test_rotg_random_host_and_device(handle):
    rng = np.random.default_rng(12)
    ab = np.concatenate([rng.uniform(-10, 10, (200, 2)),
                         [[0, 3], [3, 0], [0, 0], [-2, 2], [1e-20, 3e-20], [1e20, -7e19], [np.nan, 1]]])
    for a, b in ab.astype(np.float32):
        want = np.array(O.srotg(a, b), np.float32)
        v = np.array([a, b, 0, 0], np.float32)
        assert B.iclblasSrotg(handle, v[0:], v[1:], v[2:], v[3:]) == B.SUCCESS
        assert same(v, want), (a, b)
    v = np.array([1.0, 1.5, 0.5, 1.0], np.float32)
    dv = dev(v)
    assert B.iclblasSrotg(handle, dv[0:], dv[1:], dv[2:], dv[3:]) == B.SUCCESS
    assert same(host(dv), np.array(O.srotg(1.0, 1.5), np.float32))


def test_crotg_random(handle):
    rng = np.random.default_rng(13)
    for _ in range(200):
        a = complex(*rng.uniform(-10, 10, 2)) if rng.random() > 0.05 else 0j
        b = complex(*rng.uniform(-10, 10, 2))
        ar, c, s = O.crotg(a, b)
        v = np.array([a, b, 0], np.complex64)
        cc = np.zeros(1, np.float32)
        assert B.iclblasCrotg(handle, v[0:], v[1:], cc, v[2:]) == B.SUCCESS
        assert same(np.array([v[0], v[2]], np.complex64), np.array([ar, s], np.complex64)) and same(cc, np.array([c], np.float32))
        assert v[1] == np.complex64(b)   # b is read only


def test_rotmg_all_branches(handle):
    rng = np.random.default_rng(14)
    rows = [tuple(r) for r in rng.uniform(-2, 10, (300, 4))]
    rows += [(1.1, -1.0, 3.3, 3.2), (0.0, 1.2, 3.3, 3.2), (1 / 4096 / 4096, 1 / 4096 / 4096, 3.3, 3.2),
             (1e-12, 2e-12, 1.0, 0.5), (1e9, 3e9, 2.0, 1.0), (5e8, 1e-10, 1.0, 4.0), (-1.0, 2.0, 1.0, 1.0),
             (1.0, 0.0, 1.0, 1.0), (1.0, 1.0, 1.0, 0.0), (np.inf, 1.0, 1.0, 2.0), (1.0, np.inf, 1.0, 2.0)]
    rows += [(d1 * 10.0 ** rng.integers(-12, 12), d2 * 10.0 ** rng.integers(-12, 12), x1, y1)
             for d1, d2, x1, y1 in rng.uniform(0.1, 5, (200, 4))]
    for d1, d2, x1, y1 in rows:
        pw = np.full(5, 7, np.float32)
        want = np.array(O.srotmg(d1, d2, x1, y1, pw), np.float32)
        v = np.array([d1, d2, x1], np.float32)
        y = np.array([y1], np.float32)
        p = np.full(5, 7, np.float32)
        assert B.iclblasSrotmg(handle, v[0:], v[1:], v[2:], y, p) == B.SUCCESS
        assert same(v, want) and same(p, pw), (d1, d2, x1, y1, v, want, p, pw)
    # device operands
    v = dev(np.array([1.1, -1.0, 3.3], np.float32))
    y = dev(np.array([3.2], np.float32))
    p = dev(np.full(5, 7, np.float32))
    pw = np.full(5, 7, np.float32)
    want = np.array(O.srotmg(1.1, -1.0, 3.3, 3.2, pw), np.float32)
    assert B.iclblasSrotmg(handle, v[0:], v[1:], v[2:], y, p) == B.SUCCESS
    assert same(host(v), want) and same(host(p), pw)


# ------------------------------------------------------------------ argument rules
def test_argument_rules(handle):
    x = np.ones(8, np.float32)
    y = np.ones(8, np.float32)
    for fn in (B.iclblasScopy, B.iclblasSswap):
        assert fn(handle, 0, None, 1, None, 1) == B.SUCCESS          # n <= 0: no work, no checks
        assert fn(handle, -3, None, 1, None, 1) == B.SUCCESS
        assert fn(handle, 4, x, 0, y, 1) == B.INVALID_VALUE
        assert fn(handle, 4, x, 1, y, 0) == B.INVALID_VALUE
        assert fn(handle, 4, x, -1, y, 1) == B.NOT_SUPPORTED
        assert fn(handle, 4, None, 1, y, 1) == B.INVALID_VALUE
        assert fn(handle, 4, x, 1, None, 1) == B.INVALID_VALUE
        assert fn(None, 4, x, 1, y, 1) == B.INVALID_VALUE
    assert B.iclblasSrot(handle, 4, None, 1, None, 1, 1.0, 0.0) == B.SUCCESS   # identity rotation returns first
    assert B.iclblasSrot(handle, 4, x, 0, y, 1, 0.6, 0.8) == B.INVALID_VALUE
    assert B.iclblasCsrot(handle, 4, None, 1, None, 1, 1.0, 0.0) == B.SUCCESS
    assert B.iclblasCrot(handle, 4, None, 1, None, 1, 1.0, 0j) == B.SUCCESS
    assert B.iclblasSrotm(handle, 4, None, 1, None, 1, np.array([-2, 0, 0, 0, 0], np.float32)) == B.SUCCESS
    ri = np.full(1, 9, np.int32)
    assert B.iclblasIsamin(handle, 0, x, 1, ri) == B.SUCCESS and ri[0] == 0
    ri[0] = 9
    assert B.iclblasIsamin(handle, 4, x, -1, ri) == B.SUCCESS and ri[0] == 0
    assert B.iclblasSrotg(handle, None, x[1:], x[2:], x[3:]) == B.INVALID_VALUE
    assert B.iclblasSrotmg(handle, x[0:], x[1:], x[2:], None, y) == B.INVALID_VALUE
