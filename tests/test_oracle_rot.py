"""Pins the oracle's iamin / copy / swap / rotation restatements
(oracle/oracle.c) to the reference's own serial OpenCL kernels compiled as
C++ (oracle/_ref/libiclref.so: Isamin_naive.cl, Icamin_naive.cl,
Srot_naive.cl, Csrot_naive.cl, Crot_naive.cl, Srotm_naive.cl, Srotg_naive.cl,
Crotg_naive.cl, Srotmg_naive.cl).  Both evaluate the same FP32 expressions
with the same fused multiply-adds, so every result must be bit-identical.
"""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built (reference tree absent at build time)")


def _p(a):
    return a.ctypes.data


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _vec(rng, n, dtype, scale=4.0):
    if np.dtype(dtype) == np.complex64:
        return (rng.uniform(-scale, scale, (n, 2)).astype(np.float32)).view(np.complex64).reshape(-1)
    return rng.uniform(-scale, scale, n).astype(np.float32)


@pytest.mark.parametrize("n,inc", [(1, 1), (2, 1), (33, 1), (1000, 1), (257, 3)])
def test_iamin_matches_naive_kernels(n, inc):
    rng = np.random.default_rng(100 + n + inc)
    R = O.ref()
    x = _vec(rng, n * inc, np.float32)
    assert O.isamin(n, x, inc) == R.ref_naive_isamin(n, _p(x), inc)
    xc = _vec(rng, n * inc, np.complex64)
    assert O.icamin(n, xc, inc) == R.ref_naive_icamin(n, _p(xc), inc)


def test_iamin_ties_nan_inf():
    R = O.ref()
    cases = [
        [3, -1, 2, 1, -1],          # first of the ties
        [np.nan, 1, 0.5, 2],        # NaN first pins 0
        [4, np.nan, 0.5, 2],        # later NaN skipped
        [np.inf, np.inf, -np.inf],  # nothing smaller than x[0]
        [np.inf, 7, -np.inf, 3],
        [-0.0, 0.0, 1.0],
    ]
    for c in cases:
        x = np.array(c, np.float32)
        assert O.isamin(len(c), x, 1) == R.ref_naive_isamin(len(c), _p(x), 1), c
        xc = np.array(c, np.complex64)
        assert O.icamin(len(c), xc, 1) == R.ref_naive_icamin(len(c), _p(xc), 1), c


@pytest.mark.parametrize("n,incx,incy", [(1, 1, 1), (37, 1, 1), (500, 2, 3), (129, 3, 1)])
def test_rotations_match_naive_kernels(n, incx, incy):
    rng = np.random.default_rng(200 + n)
    R = O.ref()
    for c, s in [(0.6, 0.8), (2.0, 1.0), (-0.25, 1.75), (1.0, -3.0)]:
        x = _vec(rng, n * incx, np.float32)
        y = _vec(rng, n * incy, np.float32)
        x1, y1, x2, y2 = x.copy(), y.copy(), x.copy(), y.copy()
        O.srot(n, x1, incx, y1, incy, c, s)
        R.ref_naive_srot(n, _p(x2), incx, _p(y2), incy, c, s)
        assert np.array_equal(bits(x1), bits(x2)) and np.array_equal(bits(y1), bits(y2))

        xc = _vec(rng, n * incx, np.complex64)
        yc = _vec(rng, n * incy, np.complex64)
        x1, y1, x2, y2 = xc.copy(), yc.copy(), xc.copy(), yc.copy()
        O.csrot(n, x1, incx, y1, incy, c, s)
        R.ref_naive_csrot(n, _p(x2), incx, _p(y2), incy, c, s)
        assert np.array_equal(bits(x1), bits(x2)) and np.array_equal(bits(y1), bits(y2))

        sc = complex(s, 0.5 * c - 0.3)
        x1, y1, x2, y2 = xc.copy(), yc.copy(), xc.copy(), yc.copy()
        O.crot(n, x1, incx, y1, incy, c, sc)
        scb = O.cbox(sc)   # kept alive across the call
        R.ref_naive_crot(n, _p(x2), incx, _p(y2), incy, c, _p(scb))
        assert np.array_equal(bits(x1), bits(x2)) and np.array_equal(bits(y1), bits(y2))


@pytest.mark.parametrize("flag", [-1.0, 0.0, 1.0, 5.0])
@pytest.mark.parametrize("incx,incy", [(1, 1), (2, 3)])
def test_srotm_matches_naive_kernel(flag, incx, incy):
    rng = np.random.default_rng(300 + int(flag) + incx)
    R = O.ref()
    n = 301
    param = np.array([flag, 0.75, -1.5, 2.25, 0.125], np.float32)
    x = _vec(rng, n * incx, np.float32)
    y = _vec(rng, n * incy, np.float32)
    x1, y1, x2, y2 = x.copy(), y.copy(), x.copy(), y.copy()
    O.srotm(n, x1, incx, y1, incy, param)
    R.ref_naive_srotm(n, _p(x2), incx, _p(y2), incy, _p(param))
    assert np.array_equal(bits(x1), bits(x2)) and np.array_equal(bits(y1), bits(y2))
    if flag == 5.0:
        assert np.array_equal(x1, x) and np.array_equal(y1, y)


def _generator_inputs(rng, k=400):
    vals = list(rng.uniform(-10, 10, (k, 2)))
    vals += [(0.0, 3.0), (3.0, 0.0), (0.0, 0.0), (-2.0, 2.0), (2.0, -2.0), (1.0, 1.5), (-0.0, 5.0),
             (1e-20, 3e-20), (1e20, -7e19), (1e-30, 1e30)]
    return vals


def test_srotg_matches_naive_kernel():
    R = O.ref()
    for a, b in _generator_inputs(np.random.default_rng(7)):
        mine = np.array(O.srotg(a, b), np.float32)
        v = np.array([a, b, -9, -9], np.float32)
        R.ref_naive_srotg(_p(v[0:]), _p(v[1:]), _p(v[2:]), _p(v[3:]))
        ref = v[[0, 1, 2, 3]]
        assert np.array_equal(bits(mine), bits(ref)), (a, b, mine, ref)


def test_crotg_matches_naive_kernel():
    R = O.ref()
    rng = np.random.default_rng(8)
    for _ in range(400):
        a = complex(*rng.uniform(-10, 10, 2))
        b = complex(*rng.uniform(-10, 10, 2)) if rng.random() > 0.1 else 0j
        ar, c, s = O.crotg(a, b)
        v = np.array([a, b, 0], np.complex64)
        cc = np.zeros(1, np.float32)
        R.ref_naive_crotg(_p(v[0:]), _p(v[1:]), _p(cc), _p(v[2:]))
        assert np.array_equal(bits(np.array([ar, s], np.complex64)), bits(np.array([v[0], v[2]], np.complex64)))
        assert bits(np.float32(c)) == bits(cc[0])
    # a == 0: c = 0, s = 1, a = b (Crotg_naive.cl:23-28)
    ar, c, s = O.crotg(0j, 2 - 3j)
    assert ar == np.complex64(2 - 3j) and c == 0 and s == np.complex64(1)


def _rotmg_early(d1, d2, x1, y1):
    """The reference's host-side checks (iclBLAS_S.cpp:101-128)."""
    f = np.float32
    if f(d1) < 0:
        return [-1, 0, 0, 0, 0]
    if f(d2) == 0 or f(y1) == 0:
        return [-2]
    if f(f(f(-f(d2)) * f(y1)) * f(y1)) >= f(f(f(d1) * f(x1)) * f(x1)):
        return [-1, 0, 0, 0, 0]
    return None


def test_srotmg_matches_naive_kernel():
    R = O.ref()
    rng = np.random.default_rng(9)
    cases = [tuple(r) for r in rng.uniform(-2, 10, (300, 4))]
    cases += [(1.1, -1.0, 3.3, 3.2), (0.0, 1.2, 3.3, 3.2), (2.0, 1.0, 1.0, 3.0),
              (1 / 4096 / 4096, 1 / 4096 / 4096, 3.3, 3.2), (1e-12, 2e-12, 1.0, 0.5), (1e9, 3e9, 2.0, 1.0),
              (5e8, 1e-10, 1.0, 4.0), (-1.0, 2.0, 1.0, 1.0), (1.0, 0.0, 1.0, 1.0), (1.0, 1.0, 1.0, 0.0)]
    cases += [(d1 * 10.0 ** rng.integers(-12, 12), d2 * 10.0 ** rng.integers(-12, 12), x1, y1)
              for d1, d2, x1, y1 in rng.uniform(0.1, 5, (200, 4))]
    for d1, d2, x1, y1 in cases:
        p1 = np.array([7, 7, 7, 7, 7], np.float32)
        mine = np.array(O.srotmg(d1, d2, x1, y1, p1), np.float32)
        early = _rotmg_early(d1, d2, x1, y1)
        if early is not None:
            assert list(p1[:len(early)]) == early and np.all(p1[len(early):] == 7)
            assert np.array_equal(mine, np.array([d1, d2, x1], np.float32))
            continue
        p2 = np.array([7, 7, 7, 7, 7], np.float32)
        v = np.array([d1, d2, x1], np.float32)
        R.ref_naive_srotmg(_p(v[0:]), _p(v[1:]), _p(v[2:]), float(np.float32(y1)), _p(p2))
        assert np.array_equal(bits(p1), bits(p2)), (d1, d2, x1, y1, p1, p2)
        assert np.array_equal(bits(mine), bits(v)), (d1, d2, x1, y1)


def test_copy_swap_strided():
    rng = np.random.default_rng(11)
    for dtype in (np.float32, np.complex64):
        n, incx, incy = 77, 3, 2
        x = _vec(rng, n * incx, dtype)
        y = _vec(rng, n * incy, dtype)
        y1 = y.copy()
        O.copy(n, x, incx, y1, incy)
        ref = y.copy()
        ref[::incy][:n] = x[::incx][:n]
        assert np.array_equal(y1, ref)
        x1, y1 = x.copy(), y.copy()
        O.swap(n, x1, incx, y1, incy)
        rx, ry = x.copy(), y.copy()
        rx[::incx][:n], ry[::incy][:n] = y[::incy][:n], x[::incx][:n]
        assert np.array_equal(x1, rx) and np.array_equal(y1, ry)
