"""The benchmark configurations at their full sizes, on a B200, through the C ABI.

Each test builds its config's seeded synthetic operands on the GPU, runs the
library's routine in every math mode, and compares with an FP64 computation
of the same FP32 inputs (torch float64 on the GPU: products, triangular
solves and their autograd gradients).  That FP64 reference is tied to the
reference's own arithmetic on samples: tests/test_fp64_reference_tie_gpu.py
(the reference's double cpu_gemm and the oracle's double TRSM at config
depth) and, here, the reference's serial FP32 kernels Strsm_naive.cl /
Ctrsm_naive.cl (compiled in oracle/_ref) on 64 right-hand sides of the
solves.

Bars (relative Frobenius error against FP64, unless stated):
  plain FP32 (the drop-in default)   1e-5   the north_star's bar for every call
  6xBF16                             1e-6   the north_star's bar for the split GEMM
  3xBF16 + 1 refinement step (TRSM)  1e-6   likewise for the refined solve
  TF32 + 2 refinement steps (TRSM)   1e-6
  3xBF16 (three products)            1e-5 GEMM, 3e-5 TRSM   (measured 3.8e-6 / 5.3e-6)
  TF32                               1e-3 GEMM, 2e-3 TRSM   (measured 2.6e-4 / 3.5e-4)
Level-1 reductions and SAXPY at n = 2^28: within 1 ulp of the FP64 value
rounded to FP32.  The batched config: worst instance 1e-5 for X, dB and dA,
and central differences (eps = 1e-3) on sampled entries within 1e-3.
"""
import numpy as np
import pytest
import torch

import oracle_lib as O
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu

PLAIN, TF32, X3, X6 = B.MATH_PLAIN_FP32, B.MATH_TF32, B.MATH_BF16X3, B.MATH_BF16X6
GEMM_BARS = {PLAIN: 1e-5, TF32: 1e-3, X3: 1e-5, X6: 1e-6}
# (mode, refinement steps) -> bar
TRSM_BARS = {(PLAIN, 0): 1e-5, (TF32, 0): 2e-3, (X3, 0): 3e-5, (X6, 0): 1e-6, (X3, 1): 1e-6, (TF32, 2): 1e-6}


def rel(a, b) -> float:
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


def ulps32(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """|a - b| in float32 ulps (both float32 tensors), by integer ordering."""
    ia = a.contiguous().view(torch.int32).to(torch.int64)
    ib = b.contiguous().view(torch.int32).to(torch.int64)
    ia = torch.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
    ib = torch.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
    return (ia - ib).abs()


# ---------------------------------------------------------------- level 1/2 sweep (n = 2^28, CGEMV 8192^2)
N1 = 1 << 28


@pytest.fixture(scope="module")
def level1_vectors(cuda):
    g = torch.Generator(device=cuda).manual_seed(1)
    x = torch.rand(N1, generator=g, device=cuda) * 2 - 1
    y = torch.rand(N1, generator=g, device=cuda) * 2 - 1
    yield x, y
    del x, y
    torch.cuda.empty_cache()


def test_saxpy_2e28(handle, level1_vectors):
    x, y = level1_vectors
    handle.set_stream(torch.cuda.current_stream())
    yw = y.clone()
    assert B.iclblasSaxpy(handle, N1, 0.5, x, 1, yw, 1) == B.SUCCESS
    want = (0.5 * x.double() + y.double()).float()
    torch.cuda.synchronize()
    assert ulps32(yw, want).max().item() <= 1


@pytest.mark.parametrize("routine", ["snrm2", "sasum", "sdot", "isamax"])
def test_level1_reductions_2e28(handle, level1_vectors, routine):
    x, y = level1_vectors
    handle.set_stream(torch.cuda.current_stream())
    r = torch.zeros(1, device=x.device)
    ri = torch.zeros(1, dtype=torch.int32, device=x.device)
    if routine == "snrm2":
        assert B.iclblasSnrm2(handle, N1, x, 1, r) == B.SUCCESS
        want = torch.linalg.vector_norm(x.double())
    elif routine == "sasum":
        assert B.iclblasSasum(handle, N1, x, 1, r) == B.SUCCESS
        want = x.double().abs().sum()
    elif routine == "sdot":
        assert B.iclblasSdot(handle, N1, x, 1, y, 1, r) == B.SUCCESS
        want = (x.double() * y.double()).sum()
    else:
        assert B.iclblasIsamax(handle, N1, x, 1, ri) == B.SUCCESS
        ax = x.abs()
        m = ax.max()
        want_i = int(torch.nonzero(ax == m)[0].item())      # first index of the largest |x|
        torch.cuda.synchronize()
        assert ri.item() == want_i
        return
    torch.cuda.synchronize()
    assert ulps32(r, want.float().view(1)).max().item() <= 1, (r.item(), want.item())


@pytest.mark.parametrize("trans", [0, 2])
def test_cgemv_8192(handle, cuda, trans):
    """CGEMV 8192 x 8192 complex64, op N and C, alpha = 1+1i, beta = 0.5."""
    handle.set_stream(torch.cuda.current_stream())
    n = 8192
    g = torch.Generator(device=cuda).manual_seed(1)

    def crand(k):
        return torch.complex(torch.rand(k, generator=g, device=cuda) * 2 - 1,
                             torch.rand(k, generator=g, device=cuda) * 2 - 1)

    A = crand(n * n)
    x = crand(n)
    y = crand(n)
    yw = y.clone()
    assert B.iclblasCgemv(handle, trans, n, n, 1 + 1j, A, n, x, 1, 0.5, yw, 1) == B.SUCCESS
    Am = A.view(n, n).t().to(torch.complex128)          # Am[i, j] = A[j*n + i]
    op = Am if trans == 0 else Am.conj().t()
    want = (1 + 1j) * (op @ x.to(torch.complex128)) + 0.5 * y.to(torch.complex128)
    torch.cuda.synchronize()
    assert rel(yw.to(torch.complex128), want) <= 1e-5


# ---------------------------------------------------------------- precision: S/C GEMM 8192^3
GN = 8192


def _gemm_operands(cuda, cplx, scaled):
    g = torch.Generator(device=cuda).manual_seed(2)

    def rnd(k):
        t = torch.rand(k, generator=g, device=cuda) * 2 - 1
        return torch.complex(t, torch.rand(k, generator=g, device=cuda) * 2 - 1) if cplx else t

    A = rnd(GN * GN)
    Bm = rnd(GN * GN)
    if scaled:
        # row i of A (element (i, j) at j*GN + i) times 10^U(-4, 4)
        sc = 10.0 ** (torch.rand(GN, generator=g, device=cuda) * 8 - 4)
        A = (A.view(GN, GN) * sc.view(1, GN)).reshape(-1)
    return A, Bm


@pytest.mark.parametrize("ta,scaled", [(0, False), (1, False), (0, True), (1, True)])
def test_sgemm_8192_every_mode(handle, cuda, ta, scaled):
    """SGEMM 8192^3, op(A) = A or A^T, B no-trans, U(-1,1) (seed 2), and the
    variant whose rows of A are scaled by 10^U(-4,4).  For the scaled NN
    product the largest per-row relative error is checked as well."""
    handle.set_stream(torch.cuda.current_stream())
    A, Bm = _gemm_operands(cuda, False, scaled)
    Am = A.view(GN, GN).t()
    opA = Am if ta == 0 else Am.t()
    ref = opA.double() @ Bm.view(GN, GN).t().double()
    C = torch.empty(GN * GN, device=cuda)
    errs = {}
    for mode in (PLAIN, TF32, X3, X6):
        handle.set_math_mode(mode)
        assert B.iclblasSgemm(handle, ta, 0, GN, GN, GN, 1.0, A, GN, Bm, GN, 0.0, C, GN) == B.SUCCESS
        Cm = C.view(GN, GN).t().double()
        errs[mode] = rel(Cm, ref)
        if scaled and ta == 0:
            row = (torch.linalg.norm(Cm - ref, dim=1) / torch.linalg.norm(ref, dim=1)).max().item()
            errs[(mode, "row")] = row
            assert row <= GEMM_BARS[mode], (mode, row)
    handle.set_math_mode(PLAIN)
    for mode in (PLAIN, TF32, X3, X6):
        assert errs[mode] <= GEMM_BARS[mode], (mode, errs)
    # the precision claim: 6xBF16 at least as accurate as the plain FP32 path
    assert errs[X6] <= errs[PLAIN]


@pytest.mark.parametrize("ta", [0, 1])
def test_cgemm_8192_every_mode(handle, cuda, ta):
    handle.set_stream(torch.cuda.current_stream())
    A, Bm = _gemm_operands(cuda, True, False)
    Am = A.view(GN, GN).t()
    opA = Am if ta == 0 else Am.t()
    ref = opA.to(torch.complex128) @ Bm.view(GN, GN).t().to(torch.complex128)
    C = torch.empty(GN * GN, dtype=torch.complex64, device=cuda)
    for mode in (PLAIN, TF32, X3, X6):
        handle.set_math_mode(mode)
        assert B.iclblasCgemm(handle, ta, 0, GN, GN, GN, 1.0 + 0j, A, GN, Bm, GN, 0.0, C, GN) == B.SUCCESS
        err = rel(C.view(GN, GN).t().to(torch.complex128), ref)
        assert err <= GEMM_BARS[mode], (mode, err)
    handle.set_math_mode(PLAIN)


# ---------------------------------------------------------------- triangular solves: STRSM 8192 x 4096, CTRSM 4096 x 2048
def _tri(n, lower, cplx, g, cuda):
    """Diagonal U(1,2) (complex: that modulus, random phase), strictly
    triangular part N(0,1)/sqrt(n).  Row-major [i, j] = L(i, j)."""
    L = torch.randn(n, n, generator=g, device=cuda) / n ** 0.5
    L = torch.tril(L, -1) if lower else torch.triu(L, 1)
    d = torch.rand(n, generator=g, device=cuda) + 1.0
    if cplx:
        Li = torch.randn(n, n, generator=g, device=cuda) / n ** 0.5
        Li = torch.tril(Li, -1) if lower else torch.triu(Li, 1)
        ph = torch.rand(n, generator=g, device=cuda) * 6.283185307
        return torch.complex(L, Li) + torch.diag(torch.polar(d, ph))
    return L + torch.diag(d)


def _trsm_case(handle, cuda, cplx):
    g = torch.Generator(device=cuda).manual_seed(3)
    if cplx:
        m, nrhs, lower, trans = 4096, 2048, False, 2     # upper, conj-trans
    else:
        m, nrhs, lower, trans = 8192, 4096, True, 0      # lower, no-trans
    L = _tri(m, lower, cplx, g, cuda)
    Acm = L.t().contiguous().reshape(-1)                 # column-major storage
    B0 = torch.rand(nrhs, m, generator=g, device=cuda) * 2 - 1
    if cplx:
        B0 = torch.complex(B0, torch.rand(nrhs, m, generator=g, device=cuda) * 2 - 1)
    B0 = B0.reshape(-1)                                  # column-major m x nrhs
    wide = torch.complex128 if cplx else torch.float64
    op = L if trans == 0 else L.conj().t()
    X64 = torch.linalg.solve_triangular(op.to(wide), B0.view(nrhs, m).t().to(wide),
                                        upper=(not lower) if trans == 0 else lower)
    return m, nrhs, lower, trans, Acm, B0, X64


@pytest.mark.parametrize("cplx", [False, True], ids=["strsm_8192x4096", "ctrsm_4096x2048_upper_conj"])
def test_trsm_config_every_mode(handle, cuda, cplx):
    handle.set_stream(torch.cuda.current_stream())
    m, nrhs, lower, trans, Acm, B0, X64 = _trsm_case(handle, cuda, cplx)
    call = B.iclblasCtrsm if cplx else B.iclblasStrsm
    one = (1.0 + 0j) if cplx else 1.0
    X = B0.clone()
    errs = {}
    for (mode, steps), bar in TRSM_BARS.items():
        handle.set_math_mode(mode)
        handle.set_trsm_refinement(steps)
        X.copy_(B0)
        assert call(handle, 0, 1 if lower else 0, trans, 0, m, nrhs, one, Acm, m, X, m) == B.SUCCESS
        errs[(mode, steps)] = rel(X.view(nrhs, m).t().to(X64.dtype), X64)
    handle.set_math_mode(PLAIN)
    handle.set_trsm_refinement(0)
    assert handle.synchronize() == B.SUCCESS
    for key, bar in TRSM_BARS.items():
        assert errs[key] <= bar, (key, errs)


@pytest.mark.parametrize("cplx", [False, True], ids=["strsm_8192x4096", "ctrsm_4096x2048_upper_conj"])
def test_trsm_config_tied_to_reference_kernel(handle, cuda, cplx):
    """64 right-hand sides of the config solved by the reference's serial
    kernel (Strsm_naive.cl / Ctrsm_naive.cl in FP32, compiled in
    oracle/_ref; the oracle's restatement when the reference was not built):
    it agrees with the FP64 solve at FP32 level, and so does the library's
    plain FP32 solve of the full config."""
    handle.set_stream(torch.cuda.current_stream())
    m, nrhs, lower, trans, Acm, B0, X64 = _trsm_case(handle, cuda, cplx)
    X = B0.clone()
    call = B.iclblasCtrsm if cplx else B.iclblasStrsm
    one = (1.0 + 0j) if cplx else 1.0
    assert call(handle, 0, 1 if lower else 0, trans, 0, m, nrhs, one, Acm, m, X, m) == B.SUCCESS
    torch.cuda.synchronize()
    k = 64
    A_h = Acm.cpu().numpy()
    Bk = B0[:m * k].cpu().numpy().copy()                 # the first 64 columns
    R = O.ref()
    if R is not None:
        P = lambda a: a.ctypes.data  # noqa: E731
        if cplx:
            R.ref_naive_ctrsm(0, 1 if lower else 0, trans, 0, m, k, P(O.cbox(1.0)), P(A_h), m, P(Bk), m)
        else:
            R.ref_naive_strsm(0, 1 if lower else 0, trans, 0, m, k, 1.0, P(A_h), m, P(Bk), m)
    else:
        (O.ctrsm if cplx else O.strsm)(0, 1 if lower else 0, trans, 0, m, k, one, A_h, m, Bk, m)
    Xk64 = X64[:, :k].cpu().numpy()
    naive = Bk.reshape(k, m).T
    assert O.rel_fro(naive, Xk64) <= 1e-5
    ours = X[:m * k].cpu().numpy().reshape(k, m).T
    assert O.rel_fro(ours, naive) <= 2e-5


# ---------------------------------------------------------------- batched uneven TRSM forward + adjoint, 512 instances
def _batched_case(cuda, batch=512):
    rng = np.random.default_rng(4)
    g = torch.Generator(device=cuda).manual_seed(4)
    ns = rng.integers(32, 1025, batch)
    rs = rng.integers(1, 257, batch)
    Ls, As, B0, G0 = [], [], [], []
    for n, r in zip(ns, rs):
        n, r = int(n), int(r)
        L = torch.tril(torch.randn(n, n, generator=g, device=cuda) / n ** 0.5, -1)
        L = L + torch.diag(torch.rand(n, generator=g, device=cuda) + 1.0)
        Ls.append(L)
        As.append(L.t().contiguous().reshape(-1))
        B0.append(torch.randn(r, n, generator=g, device=cuda).reshape(-1))
        G0.append(torch.randn(r, n, generator=g, device=cuda).reshape(-1))
    return ns, rs, Ls, As, B0, G0


def test_batched_config_forward_and_adjoint(handle, cuda):
    """512 instances, n ~ UniformInt[32,1024], nrhs ~ UniformInt[1,256],
    seed 4: X = L^-1 B and the adjoint (dB, dA) in one persistent launch per
    stage, every instance against FP64 autograd of solve_triangular, and
    central differences of the FP64 loss on sampled entries."""
    handle.set_stream(torch.cuda.current_stream())
    ns, rs, Ls, As, B0, G0 = _batched_case(cuda)
    batch = len(ns)
    X = [b.clone() for b in B0]
    Gw = [gg.clone() for gg in G0]
    dA = [torch.empty(int(n) * int(n), device=cuda) for n in ns]
    P = lambda ts: torch.tensor([t.data_ptr() for t in ts], dtype=torch.int64, device=cuda)  # noqa: E731
    pA, pX, pG, pdA = P(As), P(X), P(Gw), P(dA)
    plan = B.BatchPlan(handle, "trsm", side=0, uplo=1, trans=0, diag=0, m=[int(v) for v in ns],
                       n=[int(v) for v in rs], lda=[int(v) for v in ns], ldb=[int(v) for v in ns])
    try:
        assert B.iclblasStrsmBatchedUneven(handle, plan, 1.0, pA, pX) == B.SUCCESS
        assert B.iclblasStrsmBatchedUnevenBackward(handle, plan, 1.0, pA, pX, pG, pdA) == B.SUCCESS
        torch.cuda.synchronize()
        worst = [0.0, 0.0, 0.0]
        for i in range(batch):
            n, r = int(ns[i]), int(rs[i])
            L64 = Ls[i].double().requires_grad_()
            B64 = B0[i].view(r, n).t().double().requires_grad_()
            G64 = G0[i].view(r, n).t().double()
            X64 = torch.linalg.solve_triangular(L64, B64, upper=False)
            (X64 * G64).sum().backward()
            got = (X[i].view(r, n).t().double(), Gw[i].view(r, n).t().double(), dA[i].view(n, n).t().double())
            want = (X64.detach(), B64.grad, torch.tril(L64.grad))
            for j in range(3):
                worst[j] = max(worst[j], rel(got[j], want[j]))
        assert max(worst) <= 1e-5, worst

        # central differences (eps = 1e-3) of sum(G * X) in FP64 on sampled
        # entries of three instances (smallest, median and largest order)
        eps = 1e-3
        srng = np.random.default_rng(40)
        order = np.argsort(ns)
        for i in (int(order[0]), int(order[batch // 2]), int(order[-1])):
            n, r = int(ns[i]), int(rs[i])
            L64 = Ls[i].double()
            B64 = B0[i].view(r, n).t().double()
            G64 = G0[i].view(r, n).t().double()
            dAm = dA[i].view(n, n).t().double()
            dBm = Gw[i].view(r, n).t().double()

            def loss(Lx, Bx):
                return (torch.linalg.solve_triangular(Lx, Bx, upper=False) * G64).sum().item()

            for _ in range(6):
                a = int(srng.integers(0, n))
                b = int(srng.integers(0, a + 1))
                Lp, Lm = L64.clone(), L64.clone()
                Lp[a, b] += eps
                Lm[a, b] -= eps
                fd = (loss(Lp, B64) - loss(Lm, B64)) / (2 * eps)
                assert abs(dAm[a, b].item() - fd) <= 1e-3 * max(1.0, abs(fd)), (i, a, b, dAm[a, b].item(), fd)
            for _ in range(6):
                a, b = int(srng.integers(0, n)), int(srng.integers(0, r))
                Bp, Bq = B64.clone(), B64.clone()
                Bp[a, b] += eps
                Bq[a, b] -= eps
                fd = (loss(L64, Bp) - loss(L64, Bq)) / (2 * eps)
                assert abs(dBm[a, b].item() - fd) <= 1e-3 * max(1.0, abs(fd)), (i, a, b, dBm[a, b].item(), fd)
    finally:
        plan.destroy()
