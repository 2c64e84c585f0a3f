"""iclblasHgemm (half-precision GEMM extension) on the GPU against the
oracle (orc_hgemm: exact products summed in double, one rounding to half).

Bar, per element: |gpu - oracle| <= one half-precision ulp of the result
plus the FP32 summation bound (k + 2) 2^-24 (|alpha| sum_l |a_il b_lj| +
|beta c_ij|) -- the GPU sums the K products in FP32, so a result made small
by cancellation may differ by more than one of its own ulps -- and at least
99 % of the elements bit-identical.
"""
import numpy as np
import pytest

import oracle_lib as O
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu


def half_ulps(a, b):
    a = np.ascontiguousarray(a, np.float16).view(np.int16).astype(np.int64)
    b = np.ascontiguousarray(b, np.float16).view(np.int16).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFF), a)
    b = np.where(b < 0, -(b & 0x7FFF), b)
    return np.abs(a - b)


def within_bound(got, want, k, alpha, beta, absprod, cabs):
    got = got.astype(np.float64)
    want64 = want.astype(np.float64)
    ulp = np.spacing(np.abs(want).astype(np.float16)).astype(np.float64)
    bound = ulp + (k + 2) * 2.0 ** -24 * (abs(alpha) * absprod + abs(beta) * cabs)
    return np.all(np.abs(got - want64) <= bound)


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _ld(rows, aligned, extra):
    """Leading dimension: a multiple of 8 halves (16 bytes: operands read in
    place, C stored through TMA) or rows + extra (packed operands, direct
    stores)."""
    return (rows + 7) // 8 * 8 + 8 if aligned else rows + extra


_SIZES = [(1, 1, 1), (128, 128, 64), (300, 517, 129), (1000, 999, 2049), (33, 2000, 5)]
# every size with packed operands; the in-place layouts on the sizes the
# oracle finishes quickly
_CASES = [s + (False,) for s in _SIZES] + [s + (True,) for s in _SIZES if s[2] < 1000]


@pytest.mark.parametrize("m,n,k,aligned", _CASES)
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_hgemm_vs_oracle(handle, m, n, k, ta, tb, aligned):
    rng = np.random.default_rng(m + n + k + 2 * ta + tb)
    lda = _ld(k if ta else m, aligned, 1)
    ldb = _ld(n if tb else k, aligned, 2)
    ldc = _ld(m, aligned, 3)
    A = rng.uniform(-1, 1, lda * (m if ta else k)).astype(np.float16)
    Bm = rng.uniform(-1, 1, ldb * (k if tb else n)).astype(np.float16)
    Cm = rng.uniform(-1, 1, ldc * n).astype(np.float16)
    # |op(A)| |op(B)| in float64, laid out like C (column-major, ldc)
    Am = (A.reshape(m, lda)[:, :k] if ta else A.reshape(k, lda)[:, :m].T).astype(np.float64)
    Bmat = (Bm.reshape(k, ldb)[:, :n] if tb else Bm.reshape(n, ldb)[:, :k].T).astype(np.float64)
    absprod = np.zeros((n, ldc))
    absprod[:, :m] = (np.abs(Am) @ np.abs(Bmat)).T
    absprod = absprod.reshape(-1)
    for beta in (0.5, 0.0):
        Cr, C1 = Cm.copy(), Cm.copy()
        O.hgemm(ta, tb, m, n, k, 1.25, A, lda, Bm, ldb, beta, Cr, ldc)
        assert B.iclblasHgemm(handle, ta, tb, m, n, k, 1.25, A, lda, Bm, ldb, beta, C1, ldc) == B.SUCCESS
        assert within_bound(C1, Cr, k, 1.25, beta, absprod, np.abs(Cm.astype(np.float64)))
        assert (half_ulps(C1, Cr) == 0).mean() >= 0.99
        gaps = np.ones((n, ldc), bool)
        gaps[:, :m] = False
        assert np.array_equal(C1.reshape(-1)[gaps.reshape(-1)], Cm[gaps.reshape(-1)])


def test_hgemm_beta_zero_nan_c_and_k_zero(handle):
    rng = np.random.default_rng(7)
    m, n, k = 200, 130, 70
    A = rng.uniform(-1, 1, m * k).astype(np.float16)
    Bm = rng.uniform(-1, 1, k * n).astype(np.float16)
    Cn = np.full(m * n, np.nan, np.float16)
    Cr = np.zeros(m * n, np.float16)
    O.hgemm(0, 0, m, n, k, 1.0, A, m, Bm, k, 0.0, Cr, m)
    assert B.iclblasHgemm(handle, 0, 0, m, n, k, 1.0, A, m, Bm, k, 0.0, Cn, m) == B.SUCCESS
    absprod = (np.abs(A.reshape(k, m).T.astype(np.float64)) @ np.abs(Bm.reshape(n, k).T.astype(np.float64))).T
    assert not np.isnan(Cn).any()
    assert within_bound(Cn, Cr, k, 1.0, 0.0, absprod.reshape(-1), 0.0)
    # k == 0: C = beta C
    Cm = rng.uniform(-1, 1, m * n).astype(np.float16)
    C1 = Cm.copy()
    assert B.iclblasHgemm(handle, 0, 0, m, n, 0, 1.0, A, m, Bm, 1, 2.0, C1, m) == B.SUCCESS
    assert np.array_equal(C1, (2.0 * Cm.astype(np.float32)).astype(np.float16))


def test_hgemm_device_large_vs_fp32(handle):
    import torch
    m = n = k = 4096
    g = torch.Generator(device="cuda").manual_seed(3)
    A = (torch.rand(k, m, generator=g, device="cuda") * 2 - 1).half()   # column-major m x k
    Bt = (torch.rand(n, k, generator=g, device="cuda") * 2 - 1).half()  # column-major k x n
    Cm = torch.empty(n, m, device="cuda", dtype=torch.half)
    assert B.iclblasHgemm(handle, 0, 0, m, n, k, 1.0, A, m, Bt, k, 0.0, Cm, m) == B.SUCCESS
    ref = (Bt.double() @ A.double())   # (C^T) = B^T A^T in row-major terms
    err = float(torch.linalg.norm(Cm.double() - ref) / torch.linalg.norm(ref))
    assert err <= 5e-4, err


def test_hgemm_argument_rules(handle):
    a = np.ones(16, np.float16)
    assert B.iclblasHgemm(handle, 0, 0, -1, 2, 2, 1.0, a, 2, a, 2, 0.0, a, 2) == B.INVALID_VALUE
    assert B.iclblasHgemm(handle, 0, 0, 0, 2, 2, 1.0, None, 1, None, 1, 0.0, None, 1) == B.SUCCESS
    assert B.iclblasHgemm(handle, 0, 0, 2, 2, 2, 1.0, a, 0, a, 2, 0.0, a, 2) == B.INVALID_VALUE
    assert B.iclblasHgemm(handle, 5, 0, 2, 2, 2, 1.0, a, 2, a, 2, 0.0, a, 2) == B.INVALID_VALUE


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 1)])
def test_hgemm_device_pairs_beta_vs_fp64(handle, ta, tb):
    """CTA-pair tiles (enough 256 x 256 tiles), operands read in place, C read
    and written through TMA boxes (beta != 0), ragged m and n."""
    import torch
    m, n, k = 2560 + 40, 2048 + 24, 200
    g = torch.Generator(device="cuda").manual_seed(11 + ta)
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (n, k) if tb else (k, n)
    A = (torch.rand(ac, ar, generator=g, device="cuda") * 2 - 1).half()   # column-major ar x ac
    Bt = (torch.rand(bc, br, generator=g, device="cuda") * 2 - 1).half()  # column-major br x bc
    C0 = (torch.rand(n, m, generator=g, device="cuda") * 2 - 1).half()   # column-major m x n
    Cm = C0.clone()
    assert B.iclblasHgemm(handle, ta, tb, m, n, k, 1.5, A, ar, Bt, br, 0.5, Cm, m) == B.SUCCESS
    opA = A.double().t() if ta == 0 else A.double()      # m x k
    opB = Bt.double().t() if tb == 0 else Bt.double()    # k x n
    ref = 1.5 * (opA @ opB) + 0.5 * C0.double().t()      # m x n
    err = float(torch.linalg.norm(Cm.double().t() - ref) / torch.linalg.norm(ref))
    assert err <= 5e-4, err
