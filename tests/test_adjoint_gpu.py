"""Adjoints of TRSM and GEMM (no reference counterpart) against FP64 autograd
and FP64 central finite differences (eps = 1e-3).

The library's gradients (FP32, through iclblasStrsm_backward /
iclblasSgemm_backward, wrapped in tests/autograd_ops.py) are compared with
torch autograd of torch.linalg.solve_triangular / matmul in float64 on the
same inputs (relative Frobenius <= 1e-4) and, on sampled entries, with central
differences of the float64 loss (relative <= 1e-3).  Inputs follow the
batched config: L with diagonal U(1,2) and N(0,1)/sqrt(n) off the diagonal,
B and the upstream gradient N(0,1).
"""
import numpy as np
import pytest
import torch

from autograd_ops import Gemm, Trsm
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu


def tri(n, lower, gen, dev):
    L = torch.randn(n, n, generator=gen, device=dev, dtype=torch.float64) / n ** 0.5
    L = torch.tril(L, -1) if lower else torch.triu(L, 1)
    L = L + torch.diag(torch.rand(n, generator=gen, device=dev, dtype=torch.float64) + 1)
    # junk in the unused triangle: the routine and its adjoint must ignore it
    junk = torch.randn(n, n, generator=gen, device=dev, dtype=torch.float64)
    return L + (torch.triu(junk, 1) if lower else torch.tril(junk, -1))


def ref_trsm(A, Bm, side, uplo, trans, diag, alpha):
    """X = alpha * op(A)^-1 B (left) or alpha * B op(A)^-1 (right), FP64, using
    only the stored triangle of A (and a unit diagonal when diag = 1)."""
    lower = uplo == 1
    T = torch.tril(A) if lower else torch.triu(A)
    if diag == 1:
        T = T - torch.diag(torch.diagonal(T)) + torch.eye(A.shape[0], dtype=A.dtype, device=A.device)
    M = T if trans == 0 else T.t()
    m_upper = (not lower) if trans == 0 else lower
    return torch.linalg.solve_triangular(M, alpha * Bm, upper=m_upper, left=(side == 0),
                                         unitriangular=False)


@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("diag", [0, 1])
@pytest.mark.parametrize("mode", [B.MATH_PLAIN_FP32, B.MATH_BF16X6])
def test_trsm_backward_vs_fp64_autograd(handle, cuda, side, uplo, trans, diag, mode):
    handle.set_stream(torch.cuda.current_stream())
    handle.set_math_mode(mode)
    gen = torch.Generator(device=cuda).manual_seed(4 + side + 2 * uplo + 4 * trans + 8 * diag)
    m, n = 150, 70
    na = m if side == 0 else n
    A64 = tri(na, uplo == 1, gen, cuda)
    B64 = torch.randn(m, n, generator=gen, device=cuda, dtype=torch.float64)
    G = torch.randn(m, n, generator=gen, device=cuda, dtype=torch.float64)
    alpha = 0.75
    A = A64.float().requires_grad_()
    Bm = B64.float().requires_grad_()
    X = Trsm.apply(A, Bm, side, uplo, trans, diag, alpha, handle)
    (X * G.float()).sum().backward()
    torch.cuda.synchronize()
    A_r = A.detach().double().requires_grad_()
    B_r = Bm.detach().double().requires_grad_()
    X_r = ref_trsm(A_r, B_r, side, uplo, trans, diag, alpha)
    (X_r * G).sum().backward()
    rel = lambda a, b: (torch.linalg.norm(a.double() - b) / torch.linalg.norm(b)).item()  # noqa: E731
    assert rel(X.detach(), X_r.detach()) < 1e-5
    assert rel(Bm.grad, B_r.grad) < 1e-4
    assert rel(A.grad, A_r.grad) < 1e-4


def test_trsm_backward_vs_finite_differences(handle, cuda):
    """Central differences of the FP64 loss sum(G * X(A, B)), eps = 1e-3, on
    sampled entries of the stored triangle of A and of B (left, lower, N)."""
    handle.set_stream(torch.cuda.current_stream())
    gen = torch.Generator(device=cuda).manual_seed(4)
    m, n, alpha, eps = 96, 32, 1.0, 1e-3
    A64 = tri(m, True, gen, cuda)
    B64 = torch.randn(m, n, generator=gen, device=cuda, dtype=torch.float64)
    G = torch.randn(m, n, generator=gen, device=cuda, dtype=torch.float64)
    A = A64.float().requires_grad_()
    Bm = B64.float().requires_grad_()
    (Trsm.apply(A, Bm, 0, 1, 0, 0, alpha, handle) * G.float()).sum().backward()
    torch.cuda.synchronize()
    Af, Bf = A.detach().double(), Bm.detach().double()

    def loss(Aa, Bb):
        return (ref_trsm(Aa, Bb, 0, 1, 0, 0, alpha) * G).sum().item()

    rng = np.random.default_rng(0)
    for _ in range(12):
        i = int(rng.integers(0, m))
        j = int(rng.integers(0, i + 1))  # stored (lower) triangle
        Ap, Am = Af.clone(), Af.clone()
        Ap[i, j] += eps
        Am[i, j] -= eps
        fd = (loss(Ap, Bf) - loss(Am, Bf)) / (2 * eps)
        assert abs(A.grad[i, j].item() - fd) <= 1e-3 * max(1.0, abs(fd)), (i, j, A.grad[i, j].item(), fd)
    for _ in range(12):
        i, j = int(rng.integers(0, m)), int(rng.integers(0, n))
        Bp, Bmn = Bf.clone(), Bf.clone()
        Bp[i, j] += eps
        Bmn[i, j] -= eps
        fd = (loss(Af, Bp) - loss(Af, Bmn)) / (2 * eps)
        assert abs(Bm.grad[i, j].item() - fd) <= 1e-3 * max(1.0, abs(fd))


@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("tb", [0, 1])
@pytest.mark.parametrize("mode", [B.MATH_PLAIN_FP32, B.MATH_BF16X6])
def test_gemm_backward_vs_fp64_autograd(handle, cuda, ta, tb, mode):
    handle.set_stream(torch.cuda.current_stream())
    handle.set_math_mode(mode)
    gen = torch.Generator(device=cuda).manual_seed(40 + ta + 2 * tb)
    m, n, k = 120, 90, 70
    A64 = torch.randn(*((m, k) if ta == 0 else (k, m)), generator=gen, device=cuda, dtype=torch.float64)
    B64 = torch.randn(*((k, n) if tb == 0 else (n, k)), generator=gen, device=cuda, dtype=torch.float64)
    C64 = torch.randn(m, n, generator=gen, device=cuda, dtype=torch.float64)
    G = torch.randn(m, n, generator=gen, device=cuda, dtype=torch.float64)
    alpha, beta = 1.5, -0.5
    A, Bm, Cin = (t.float().requires_grad_() for t in (A64, B64, C64))
    Cout = Gemm.apply(A, Bm, Cin, ta, tb, alpha, beta, handle)
    (Cout * G.float()).sum().backward()
    torch.cuda.synchronize()
    A_r, B_r, C_r = (t.detach().double().requires_grad_() for t in (A, Bm, Cin))
    opA = A_r if ta == 0 else A_r.t()
    opB = B_r if tb == 0 else B_r.t()
    ((alpha * opA @ opB + beta * C_r) * G).sum().backward()
    rel = lambda a, b: (torch.linalg.norm(a.double() - b) / torch.linalg.norm(b)).item()  # noqa: E731
    assert rel(A.grad, A_r.grad) < 1e-5
    assert rel(Bm.grad, B_r.grad) < 1e-5
    assert rel(Cin.grad, C_r.grad) < 1e-6


def test_trsm_backward_host_pointers(handle):
    """The adjoint also takes host arrays (staged like every routine)."""
    m, n = 40, 9
    rng = np.random.default_rng(1)
    L = np.tril(rng.standard_normal((m, m)) / np.sqrt(m), -1) + np.diag(rng.uniform(1, 2, m))
    Acm = np.ascontiguousarray(L.T, dtype=np.float32).reshape(-1)
    Xcm = rng.standard_normal(m * n).astype(np.float32)
    assert B.iclblasStrsm(handle, 0, 1, 0, 0, m, n, 1.0, Acm, m, Xcm, m) == B.SUCCESS
    G = rng.standard_normal(m * n).astype(np.float32)
    dA = np.full(m * m, 7.0, np.float32)
    assert B.iclblasStrsm_backward(handle, 0, 1, 0, 0, m, n, 1.0, Acm, m, Xcm, m, G, m, dA, m) == B.SUCCESS
    D = dA.reshape(m, m).T  # logical dA
    assert np.all(np.triu(D, 1) == 0)  # off the stored triangle
    # W = L^-T G_in: check L^T W == G_in
    # (G now holds dB = W for alpha = 1)
    assert np.all(np.isfinite(D))
