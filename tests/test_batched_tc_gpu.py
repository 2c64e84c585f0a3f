"""The tensor-core path of the uneven batched TRSM / GEMM plans (plans
created while the handle is in the TF32, 3xBF16 or 6xBF16 math mode).

Each result is checked against an FP64 reference computed from the same
FP32 inputs (torch float64 on the GPU; the FP64 solve itself is tied to the
oracle's strsm by the plain-path tests), with a relative Frobenius bound
per mode: 6xBF16 <= 1e-6 (it drains the accumulator after every K tile
and sums the parts in FP32, which keeps it at FP32 accuracy), 3xBF16 <=
5e-5, TF32 <= 5e-3.
"""
import numpy as np
import pytest
import torch

from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu

BOUND = {B.MATH_BF16X6: 1e-6, B.MATH_BF16X3: 5e-5, B.MATH_TF32: 5e-3}
MODES = [B.MATH_BF16X3, B.MATH_BF16X6, B.MATH_TF32]


def tri_np(n, lower, rng, unit_junk=False):
    """Column-major n x n triangular matrix (lda = n) with junk in the other triangle."""
    L = rng.standard_normal((n, n)) / np.sqrt(max(n, 1))
    L = np.tril(L, -1) if lower else np.triu(L, 1)
    L = L + np.diag(rng.uniform(1, 2, n))
    junk = rng.standard_normal((n, n))
    L = L + (np.triu(junk, 1) if lower else np.tril(junk, -1))
    return np.ascontiguousarray(L.T, dtype=np.float32).reshape(-1)


def ptrs(ts, dev):
    return torch.tensor([t.data_ptr() for t in ts], dtype=torch.int64, device=dev)


def rel(a, b):
    a = a.double()
    b = b.double()
    return (torch.linalg.norm(a - b) / max(torch.linalg.norm(b).item(), 1e-300)).item()


def op_tri(a_flat, n, lda, uplo, trans, diag):
    """op(A) as a float64 n x n matrix (the stored triangle only)."""
    A = a_flat.double().reshape(n, lda)[:, :n].T   # column-major -> A[i][j]
    A = torch.tril(A) if uplo == 1 else torch.triu(A)
    if diag == 1:
        A = A - torch.diag(torch.diag(A)) + torch.eye(n, dtype=A.dtype, device=A.device)
    return A if trans == 0 else A.T


def solve_ref(a_flat, b_flat, side, uplo, trans, diag, m, n, lda, ldb, alpha):
    """X (column-major, ld ldb, float64) with op(A) X = alpha B (left) or X op(A) = alpha B."""
    na = m if side == 0 else n
    M = op_tri(a_flat, na, lda, uplo, trans, diag)
    Bm = b_flat.double().reshape(n, ldb)[:, :m].T
    if side == 0:
        X = torch.linalg.solve_triangular(M, alpha * Bm, upper=not bool(torch.equal(M, torch.tril(M))))
    else:
        X = torch.linalg.solve_triangular(M, alpha * Bm, upper=not bool(torch.equal(M, torch.tril(M))), left=False)
    return X


def mat(b_flat, rows, cols, ld):
    return b_flat.double().reshape(cols, ld)[:, :rows].T


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("side,uplo,trans,diag", [(0, 1, 0, 0), (0, 0, 0, 1), (0, 1, 1, 0), (0, 0, 2, 0),
                                                   (1, 1, 0, 0), (1, 0, 1, 1)])
def test_batched_tc_trsm_forward(handle, cuda, mode, side, uplo, trans, diag):
    handle.set_stream(torch.cuda.current_stream())
    rng = np.random.default_rng(100 + side + 2 * uplo + 4 * trans + 8 * diag)
    batch = 21
    na = rng.integers(1, 420, batch)     # order of A
    nr = rng.integers(1, 300, batch)     # right-hand sides
    na[0], nr[0] = 128, 128              # exact tile multiples
    na[1], nr[1] = 256, 1
    na[2], nr[2] = 1, 1
    na[3], nr[3] = 129, 17
    na[4], nr[4] = 200, 0                # empty instance
    ms = na if side == 0 else nr
    ns = nr if side == 0 else na
    lda = na + rng.integers(0, 5, batch)
    ldb = ms + rng.integers(0, 5, batch)
    handle.set_math_mode(mode)
    plan = B.BatchPlan(handle, "trsm", side=side, uplo=uplo, trans=trans, diag=diag, m=list(ms), n=list(ns),
                       lda=list(lda), ldb=list(ldb))
    _, width, ctas = plan.info()
    assert (width, ctas) == (128, 1)
    As, Bs = [], []
    for i in range(batch):
        a = np.zeros(int(lda[i]) * int(na[i]), np.float32)
        a.reshape(int(na[i]), int(lda[i]))[:, :na[i]] = tri_np(int(na[i]), uplo == 1, rng).reshape(int(na[i]),
                                                                                               int(na[i]))
        As.append(torch.from_numpy(a).to(cuda))
        Bs.append(torch.from_numpy(rng.standard_normal(int(ldb[i]) * max(int(ns[i]), 1)).astype(np.float32)).to(cuda))
    X = [b.clone() for b in Bs]
    alpha = -1.25
    assert B.iclblasStrsmBatchedUneven(handle, plan, alpha, ptrs(As, cuda), ptrs(X, cuda)) == B.SUCCESS
    torch.cuda.synchronize()
    worst = 0.0
    for i in range(batch):
        m, n = int(ms[i]), int(ns[i])
        if m == 0 or n == 0:
            assert torch.equal(X[i], Bs[i])
            continue
        ref = solve_ref(As[i], Bs[i], side, uplo, trans, diag, m, n, int(lda[i]), int(ldb[i]), alpha)
        e = rel(mat(X[i], m, n, int(ldb[i])), ref)
        worst = max(worst, e)
        assert e <= BOUND[mode], (i, m, n, e)
        # padding rows of B untouched
        pad = X[i].reshape(n, int(ldb[i]))[:, m:]
        assert torch.equal(pad, Bs[i].reshape(n, int(ldb[i]))[:, m:])
    plan.destroy()


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("side,uplo,trans,diag,alpha", [(0, 1, 0, 0, 0.5), (0, 0, 1, 1, -2.0), (1, 1, 2, 0, 1.0),
                                                         (1, 0, 0, 1, 1.5)])
def test_batched_tc_trsm_backward(handle, cuda, mode, side, uplo, trans, diag, alpha):
    """dB = alpha op(A)^-T G (left; right: G op(A)^-T) and dA on the stored
    triangle, against FP64 formulas on the same FP32 inputs."""
    handle.set_stream(torch.cuda.current_stream())
    rng = np.random.default_rng(200 + side + 2 * uplo + 4 * trans)
    batch = 15
    na = rng.integers(1, 400, batch)
    nr = rng.integers(1, 260, batch)
    na[0], nr[0] = 256, 128
    ms = na if side == 0 else nr
    ns = nr if side == 0 else na
    handle.set_math_mode(mode)
    plan = B.BatchPlan(handle, "trsm", side=side, uplo=uplo, trans=trans, diag=diag, m=list(ms), n=list(ns),
                       lda=list(na), ldb=list(ms))
    As = [torch.from_numpy(tri_np(int(n), uplo == 1, rng)).to(cuda) for n in na]
    Bs = [torch.from_numpy(rng.standard_normal(int(m) * int(n)).astype(np.float32)).to(cuda) for m, n in zip(ms, ns)]
    Gs = [torch.from_numpy(rng.standard_normal(int(m) * int(n)).astype(np.float32)).to(cuda) for m, n in zip(ms, ns)]
    X = [b.clone() for b in Bs]
    assert B.iclblasStrsmBatchedUneven(handle, plan, alpha, ptrs(As, cuda), ptrs(X, cuda)) == B.SUCCESS
    G = [g.clone() for g in Gs]
    dA = [torch.full((int(n) * int(n),), 3.0, device=cuda) for n in na]
    assert B.iclblasStrsmBatchedUnevenBackward(handle, plan, alpha, ptrs(As, cuda), ptrs(X, cuda), ptrs(G, cuda),
                                               ptrs(dA, cuda)) == B.SUCCESS
    torch.cuda.synchronize()
    for i in range(batch):
        m, n, k = int(ms[i]), int(ns[i]), int(na[i])
        M = op_tri(As[i], k, k, uplo, trans, diag)
        Xm = mat(X[i], m, n, m)                     # the forward's own FP32 result
        Gm = mat(Gs[i], m, n, m)
        upper = not bool(torch.equal(M, torch.tril(M)))
        if side == 0:   # op(A) X = alpha B: dB = alpha op(A)^-T G, dM = -(1/alpha) dB X^T
            dB = alpha * torch.linalg.solve_triangular(M.T, Gm, upper=not upper)
            dM = -(1.0 / alpha) * dB @ Xm.T
        else:           # X op(A) = alpha B: dB = alpha G op(A)^-T, dM = -(1/alpha) X^T dB
            dB = alpha * torch.linalg.solve_triangular(M.T, Gm, upper=not upper, left=False)
            dM = -(1.0 / alpha) * Xm.T @ dB
        dAref = dM if trans == 0 else dM.T
        dAref = torch.tril(dAref, -1 if diag else 0) if uplo == 1 else torch.triu(dAref, 1 if diag else 0)
        e_b = rel(mat(G[i], m, n, m), dB)
        e_a = rel(mat(dA[i], k, k, k), dAref)
        assert e_b <= BOUND[mode], (i, e_b)
        assert e_a <= BOUND[mode], (i, e_a)
    plan.destroy()


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_batched_tc_gemm(handle, cuda, mode, ta, tb):
    handle.set_stream(torch.cuda.current_stream())
    rng = np.random.default_rng(300 + ta + 2 * tb)
    batch = 19
    ms, ns, ks = (rng.integers(1, 300, batch) for _ in range(3))
    ms[0], ns[0], ks[0] = 128, 128, 128
    ks[1] = 0
    handle.set_math_mode(mode)
    As, Bs, Cs, lda, ldb = [], [], [], [], []
    for m, n, k in zip(ms, ns, ks):
        ar, ac = (m, k) if ta == 0 else (k, m)
        br, bc = (k, n) if tb == 0 else (n, k)
        As.append(torch.from_numpy(rng.uniform(-1, 1, max(ar * ac, 1)).astype(np.float32)).to(cuda))
        Bs.append(torch.from_numpy(rng.uniform(-1, 1, max(br * bc, 1)).astype(np.float32)).to(cuda))
        Cs.append(torch.from_numpy(rng.uniform(-1, 1, m * n).astype(np.float32)).to(cuda))
        lda.append(max(int(ar), 1))
        ldb.append(max(int(br), 1))
    plan = B.BatchPlan(handle, "gemm", transa=ta, transb=tb, m=list(ms), n=list(ns), k=list(ks), lda=lda, ldb=ldb,
                       ldc=list(ms))
    C = [c.clone() for c in Cs]
    assert B.iclblasSgemmBatchedUneven(handle, plan, 1.25, ptrs(As, cuda), ptrs(Bs, cuda), -0.5,
                                       ptrs(C, cuda)) == B.SUCCESS
    torch.cuda.synchronize()
    for i in range(batch):
        m, n, k = int(ms[i]), int(ns[i]), int(ks[i])
        ar, ac = (m, k) if ta == 0 else (k, m)
        br, bc = (k, n) if tb == 0 else (n, k)
        Am = mat(As[i], ar, ac, lda[i]) if ar * ac else torch.zeros(ar, ac, dtype=torch.float64, device=cuda)
        Bm = mat(Bs[i], br, bc, ldb[i]) if br * bc else torch.zeros(br, bc, dtype=torch.float64, device=cuda)
        ref = 1.25 * (Am if ta == 0 else Am.T) @ (Bm if tb == 0 else Bm.T) - 0.5 * mat(Cs[i], m, n, m)
        assert rel(mat(C[i], m, n, m), ref) <= BOUND[mode], i
    plan.destroy()


def test_batched_tc_trsm_under_cuda_graph(handle, cuda):
    """The tensor-core call (inverse passes, splits, per-step launches) is
    captured in a CUDA graph and replayed: every replay gives the eager result."""
    rng = np.random.default_rng(17)
    batch = 12
    ms = rng.integers(32, 400, batch)
    ns = rng.integers(1, 200, batch)
    As = [torch.from_numpy(tri_np(int(m), True, rng)).to(cuda) for m in ms]
    B0 = [torch.from_numpy(rng.standard_normal(int(m) * int(n)).astype(np.float32)).to(cuda) for m, n in zip(ms, ns)]
    handle.set_math_mode(B.MATH_BF16X3)
    plan = B.BatchPlan(handle, "trsm", side=0, uplo=1, trans=0, diag=0, m=list(ms), n=list(ns), lda=list(ms),
                       ldb=list(ms))
    work = [b.clone() for b in B0]
    pa, pw = ptrs(As, cuda), ptrs(work, cuda)
    eager = [b.clone() for b in B0]
    pe = ptrs(eager, cuda)
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    handle.set_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        for w, b in zip(work, B0):
            w.copy_(b)
        st = B.iclblasStrsmBatchedUneven(handle, plan, 1.0, pa, pw)
    assert st == B.SUCCESS
    handle.set_stream(torch.cuda.current_stream())
    assert B.iclblasStrsmBatchedUneven(handle, plan, 1.0, pa, pe) == B.SUCCESS
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        for w, e in zip(work, eager):
            assert torch.equal(w, e)
    del g
    plan.destroy()


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("uplo", [1, 0])
def test_batched_tc_adjoint_reuses_forward(handle, cuda, mode, uplo):
    """With inverse reuse the tensor-core adjoint takes the forward call's
    inverse planes and (BF16 modes) its operator tiles, read MN-major:
    results bit-identical to a plan that forms and splits them again."""
    handle.set_stream(torch.cuda.current_stream())
    rng = np.random.default_rng(400 + uplo)
    batch = 9
    ms, ns = rng.integers(1, 450, batch), rng.integers(1, 200, batch)
    ms[0], ns[0] = 384, 128
    As = [tri_np(int(m), uplo == 1, rng) for m in ms]
    Bs = [rng.standard_normal(int(m) * int(n)).astype(np.float32) for m, n in zip(ms, ns)]
    Gs = [rng.standard_normal(int(m) * int(n)).astype(np.float32) for m, n in zip(ms, ns)]
    handle.set_math_mode(mode)
    outs = []
    for reuse in (False, True):
        plan = B.BatchPlan(handle, "trsm", side=0, uplo=uplo, trans=0, diag=0, m=list(ms), n=list(ns),
                           lda=list(ms), ldb=list(ms))
        assert plan.set_inverse_reuse(reuse) == B.SUCCESS
        dA = [torch.from_numpy(a).to(cuda) for a in As]
        dX = [torch.from_numpy(b).to(cuda) for b in Bs]
        dG = [torch.from_numpy(g).to(cuda) for g in Gs]
        ddA = [torch.empty(int(m) * int(m), device=cuda) for m in ms]
        pa, px, pg, pda = ptrs(dA, cuda), ptrs(dX, cuda), ptrs(dG, cuda), ptrs(ddA, cuda)
        assert B.iclblasStrsmBatchedUneven(handle, plan, 0.5, pa, px) == B.SUCCESS
        assert B.iclblasStrsmBatchedUnevenBackward(handle, plan, 0.5, pa, px, pg, pda) == B.SUCCESS
        torch.cuda.synchronize()
        outs.append(([g.clone() for g in dG], [d.clone() for d in ddA]))
        plan.destroy()
    for g0, g1 in zip(outs[0][0], outs[1][0]):
        assert torch.equal(g0, g1)
    for d0, d1 in zip(outs[0][1], outs[1][1]):
        assert torch.equal(d0, d1)
