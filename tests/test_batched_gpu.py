"""Uneven batched TRSM / GEMM (one persistent launch each), the batched TRSM
adjoint, CUDA-graph capture and the tuner's cache.

Batched TRSM instances are checked against the oracle (relative Frobenius
<= 1e-5 per instance); batched GEMM is bit-exact with the oracle's FP32 FMA
order; the batched adjoint against the single-instance adjoint (relative
Frobenius <= 1e-5).
"""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import oracle_lib as O
from clgpu_b200 import iclblas as B

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def tri_np(n, lower, rng):
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
    return (torch.linalg.norm(a - b) / max(torch.linalg.norm(b).item(), 1e-30)).item()


@pytest.mark.parametrize("uplo,trans,diag", [(1, 0, 0), (0, 0, 0), (1, 1, 0), (0, 1, 1), (1, 2, 1)])
def test_batched_trsm_matches_oracle(handle, cuda, uplo, trans, diag):
    handle.set_stream(torch.cuda.current_stream())
    rng = np.random.default_rng(10 + uplo + 2 * trans + 4 * diag)
    batch = 37
    ms = rng.integers(1, 300, batch)
    ns = rng.integers(1, 100, batch)
    ms[0], ns[0] = 64, 64      # exact block multiples
    ms[1], ns[1] = 1, 1
    ms[2], ns[2] = 128, 0      # empty instance
    As = [tri_np(int(m), uplo == 1, rng) for m in ms]
    Bs = [rng.standard_normal(int(m) * max(int(n), 1)).astype(np.float32) for m, n in zip(ms, ns)]
    plan = B.BatchPlan(handle, "trsm", side=0, uplo=uplo, trans=trans, diag=diag, m=list(ms), n=list(ns),
                       lda=list(ms), ldb=list(ms))
    flops, width, ctas = plan.info()
    assert width in (32, 64) and ctas in (1, 2, 4)
    assert abs(flops - float(np.sum(ms.astype(float) ** 2 * ns))) < 1
    dA = [torch.from_numpy(a).to(cuda) for a in As]
    dB = [torch.from_numpy(b).to(cuda) for b in Bs]
    pa, pb = ptrs(dA, cuda), ptrs(dB, cuda)
    assert B.iclblasStrsmBatchedUneven(handle, plan, -1.5, pa, pb) == B.SUCCESS
    torch.cuda.synchronize()
    for i in range(batch):
        m, n = int(ms[i]), int(ns[i])
        ref = Bs[i].copy()
        if n:
            O.strsm(0, uplo, trans, diag, m, n, -1.5, As[i], m, ref, m)
        assert O.rel_fro(dB[i].cpu().numpy(), ref) <= 1e-5, i
    plan.destroy()


def test_batched_trsm_padded_leading_dims(handle, cuda):
    handle.set_stream(torch.cuda.current_stream())
    rng = np.random.default_rng(5)
    batch = 9
    ms = rng.integers(1, 150, batch)
    ns = rng.integers(1, 70, batch)
    ldas = ms + rng.integers(0, 9, batch)
    ldbs = ms + rng.integers(0, 9, batch)
    As, Bs = [], []
    for m, n, la, lb in zip(ms, ns, ldas, ldbs):
        a = np.zeros(int(la) * int(m), np.float32)
        a.reshape(int(m), int(la))[:, :m] = tri_np(int(m), True, rng).reshape(int(m), int(m))
        As.append(a)
        Bs.append(rng.standard_normal(int(lb) * int(n)).astype(np.float32))
    plan = B.BatchPlan(handle, "trsm", side=0, uplo=1, trans=0, diag=0, m=list(ms), n=list(ns), lda=list(ldas),
                       ldb=list(ldbs))
    dA = [torch.from_numpy(a).to(cuda) for a in As]
    dB = [torch.from_numpy(b).to(cuda) for b in Bs]
    assert B.iclblasStrsmBatchedUneven(handle, plan, 1.0, ptrs(dA, cuda), ptrs(dB, cuda)) == B.SUCCESS
    torch.cuda.synchronize()
    for i in range(batch):
        ref = Bs[i].copy()
        O.strsm(0, 1, 0, 0, int(ms[i]), int(ns[i]), 1.0, As[i], int(ldas[i]), ref, int(ldbs[i]))
        got = dB[i].cpu().numpy()
        assert O.rel_fro(got, ref) <= 1e-5, i
        # padding rows untouched
        pad = ref.reshape(int(ns[i]), int(ldbs[i]))[:, ms[i]:]
        assert np.array_equal(got.reshape(int(ns[i]), int(ldbs[i]))[:, ms[i]:], pad)
    plan.destroy()


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_batched_gemm_bit_exact(handle, cuda, ta, tb):
    handle.set_stream(torch.cuda.current_stream())
    rng = np.random.default_rng(20 + ta + 2 * tb)
    batch = 29
    ms, ns, ks = (rng.integers(1, 200, batch) for _ in range(3))
    ms[0], ns[0], ks[0] = 64, 64, 64
    ks[1] = 0
    As, Bs, Cs, ldas, ldbs = [], [], [], [], []
    for m, n, k in zip(ms, ns, ks):
        ar, ac = (m, k) if ta == 0 else (k, m)
        br, bc = (k, n) if tb == 0 else (n, k)
        As.append(rng.uniform(-1, 1, max(ar * ac, 1)).astype(np.float32))
        Bs.append(rng.uniform(-1, 1, max(br * bc, 1)).astype(np.float32))
        Cs.append(rng.uniform(-1, 1, m * n).astype(np.float32))
        ldas.append(max(int(ar), 1))
        ldbs.append(max(int(br), 1))
    plan = B.BatchPlan(handle, "gemm", transa=ta, transb=tb, m=list(ms), n=list(ns), k=list(ks), lda=ldas, ldb=ldbs,
                       ldc=list(ms))
    dA = [torch.from_numpy(a).to(cuda) for a in As]
    dB = [torch.from_numpy(b).to(cuda) for b in Bs]
    dC = [torch.from_numpy(c).to(cuda) for c in Cs]
    assert B.iclblasSgemmBatchedUneven(handle, plan, 1.25, ptrs(dA, cuda), ptrs(dB, cuda), -0.5,
                                       ptrs(dC, cuda)) == B.SUCCESS
    torch.cuda.synchronize()
    for i in range(batch):
        ref = Cs[i].copy()
        O.sgemm(ta, tb, int(ms[i]), int(ns[i]), int(ks[i]), 1.25, As[i], ldas[i], Bs[i], ldbs[i], -0.5, ref,
                int(ms[i]))
        assert np.array_equal(dC[i].cpu().numpy(), ref), i
    plan.destroy()


@pytest.mark.parametrize("uplo,trans,diag,alpha", [(1, 0, 0, 0.5), (0, 1, 0, 1.0), (1, 1, 1, -2.0), (0, 0, 1, 1.0)])
def test_batched_trsm_backward_matches_single(handle, cuda, uplo, trans, diag, alpha):
    handle.set_stream(torch.cuda.current_stream())
    rng = np.random.default_rng(30 + uplo + trans)
    batch = 17
    ms = rng.integers(1, 200, batch)
    ns = rng.integers(1, 80, batch)
    As = [torch.from_numpy(tri_np(int(m), uplo == 1, rng)).to(cuda) for m in ms]
    Bs = [torch.from_numpy(rng.standard_normal(int(m) * int(n)).astype(np.float32)).to(cuda) for m, n in zip(ms, ns)]
    Gs = [torch.from_numpy(rng.standard_normal(int(m) * int(n)).astype(np.float32)).to(cuda) for m, n in zip(ms, ns)]
    plan = B.BatchPlan(handle, "trsm", side=0, uplo=uplo, trans=trans, diag=diag, m=list(ms), n=list(ns),
                       lda=list(ms), ldb=list(ms))
    Xs = [b.clone() for b in Bs]
    assert B.iclblasStrsmBatchedUneven(handle, plan, alpha, ptrs(As, cuda), ptrs(Xs, cuda)) == B.SUCCESS
    Gb = [g.clone() for g in Gs]
    dAb = [torch.full((int(m) * int(m),), 3.0, device=cuda) for m in ms]
    assert B.iclblasStrsmBatchedUnevenBackward(handle, plan, alpha, ptrs(As, cuda), ptrs(Xs, cuda), ptrs(Gb, cuda),
                                               ptrs(dAb, cuda)) == B.SUCCESS
    for i in range(batch):
        m, n = int(ms[i]), int(ns[i])
        x1 = Bs[i].clone()
        assert B.iclblasStrsm(handle, 0, uplo, trans, diag, m, n, alpha, As[i], m, x1, m) == B.SUCCESS
        g1 = Gs[i].clone()
        dA1 = torch.zeros(m * m, device=cuda)
        assert B.iclblasStrsm_backward(handle, 0, uplo, trans, diag, m, n, alpha, As[i], m, x1, m, g1, m, dA1,
                                       m) == B.SUCCESS
        torch.cuda.synchronize()
        assert rel(Xs[i], x1) <= 1e-5, i
        assert rel(Gb[i], g1) <= 1e-5, i
        assert rel(dAb[i], dA1) <= 1e-5, i
    plan.destroy()


def test_batched_trsm_under_cuda_graph(handle, cuda):
    """Plan built first; the call (memset + persistent launch) is captured in a
    CUDA graph together with the copies that restore B, and replayed; every
    replay gives the eager result."""
    rng = np.random.default_rng(7)
    batch = 24
    ms = rng.integers(32, 257, batch)
    ns = rng.integers(1, 65, batch)
    As = [torch.from_numpy(tri_np(int(m), True, rng)).to(cuda) for m in ms]
    B0 = [torch.from_numpy(rng.standard_normal(int(m) * int(n)).astype(np.float32)).to(cuda) for m, n in zip(ms, ns)]
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


@pytest.mark.parametrize("uplo,trans,diag", [(1, 0, 0), (0, 0, 1), (1, 1, 0), (0, 2, 0)])
def test_batched_trsm_right_side_matches_oracle(handle, cuda, uplo, trans, diag):
    """X op(A) = alpha B, run on B's rows."""
    handle.set_stream(torch.cuda.current_stream())
    rng = np.random.default_rng(40 + uplo + 2 * trans + 4 * diag)
    batch = 23
    ms = rng.integers(1, 120, batch)      # rows of B (right-hand sides)
    ns = rng.integers(1, 260, batch)      # order of A
    ms[0], ns[0] = 64, 128
    ldbs = ms + rng.integers(0, 5, batch)
    As = [tri_np(int(n), uplo == 1, rng) for n in ns]
    Bs = [rng.standard_normal(int(lb) * int(n)).astype(np.float32) for lb, n in zip(ldbs, ns)]
    plan = B.BatchPlan(handle, "trsm", side=1, uplo=uplo, trans=trans, diag=diag, m=list(ms), n=list(ns),
                       lda=list(ns), ldb=list(ldbs))
    flops, _, _ = plan.info()
    assert abs(flops - float(np.sum(ns.astype(float) ** 2 * ms))) < 1
    dA = [torch.from_numpy(a).to(cuda) for a in As]
    dB = [torch.from_numpy(b).to(cuda) for b in Bs]
    assert B.iclblasStrsmBatchedUneven(handle, plan, 0.75, ptrs(dA, cuda), ptrs(dB, cuda)) == B.SUCCESS
    torch.cuda.synchronize()
    for i in range(batch):
        ref = Bs[i].copy()
        O.strsm(1, uplo, trans, diag, int(ms[i]), int(ns[i]), 0.75, As[i], int(ns[i]), ref, int(ldbs[i]))
        got = dB[i].cpu().numpy()
        assert O.rel_fro(got, ref) <= 1e-5, i
        assert np.array_equal(got.reshape(int(ns[i]), int(ldbs[i]))[:, ms[i]:],
                              ref.reshape(int(ns[i]), int(ldbs[i]))[:, ms[i]:])   # padding rows untouched
    plan.destroy()


@pytest.mark.parametrize("uplo,trans,diag,alpha", [(1, 0, 0, 1.0), (0, 1, 0, -0.5), (1, 2, 1, 2.0)])
def test_batched_trsm_right_backward_matches_single(handle, cuda, uplo, trans, diag, alpha):
    handle.set_stream(torch.cuda.current_stream())
    rng = np.random.default_rng(60 + uplo + trans)
    batch = 13
    ms = rng.integers(1, 90, batch)
    ns = rng.integers(1, 200, batch)
    As = [torch.from_numpy(tri_np(int(n), uplo == 1, rng)).to(cuda) for n in ns]
    Bs = [torch.from_numpy(rng.standard_normal(int(m) * int(n)).astype(np.float32)).to(cuda) for m, n in zip(ms, ns)]
    Gs = [torch.from_numpy(rng.standard_normal(int(m) * int(n)).astype(np.float32)).to(cuda) for m, n in zip(ms, ns)]
    plan = B.BatchPlan(handle, "trsm", side=1, uplo=uplo, trans=trans, diag=diag, m=list(ms), n=list(ns),
                       lda=list(ns), ldb=list(ms))
    Xs = [b.clone() for b in Bs]
    assert B.iclblasStrsmBatchedUneven(handle, plan, alpha, ptrs(As, cuda), ptrs(Xs, cuda)) == B.SUCCESS
    Gb = [g.clone() for g in Gs]
    dAb = [torch.full((int(n) * int(n),), 3.0, device=cuda) for n in ns]
    assert B.iclblasStrsmBatchedUnevenBackward(handle, plan, alpha, ptrs(As, cuda), ptrs(Xs, cuda), ptrs(Gb, cuda),
                                               ptrs(dAb, cuda)) == B.SUCCESS
    for i in range(batch):
        m, n = int(ms[i]), int(ns[i])
        x1 = Bs[i].clone()
        assert B.iclblasStrsm(handle, 1, uplo, trans, diag, m, n, alpha, As[i], n, x1, m) == B.SUCCESS
        g1 = Gs[i].clone()
        dA1 = torch.zeros(n * n, device=cuda)
        assert B.iclblasStrsm_backward(handle, 1, uplo, trans, diag, m, n, alpha, As[i], n, x1, m, g1, m, dA1,
                                       n) == B.SUCCESS
        torch.cuda.synchronize()
        assert rel(Xs[i], x1) <= 1e-5, i
        assert rel(Gb[i], g1) <= 1e-5, i
        assert rel(dAb[i], dA1) <= 1e-5, i
    plan.destroy()


def test_batched_rejects_bad_arguments(handle, cuda):
    with pytest.raises(B.IclblasError) as ei:   # right side: lda below the order of A (n)
        B.BatchPlan(handle, "trsm", side=1, uplo=1, trans=0, diag=0, m=[4], n=[9], lda=[8], ldb=[4])
    assert ei.value.status == B.INVALID_VALUE
    with pytest.raises(B.IclblasError) as ei:
        B.BatchPlan(handle, "trsm", side=0, uplo=1, trans=0, diag=0, m=[8], n=[4], lda=[7], ldb=[8])
    assert ei.value.status == B.INVALID_VALUE
    plan = B.BatchPlan(handle, "trsm", side=0, uplo=1, trans=0, diag=0, m=[8], n=[4], lda=[8], ldb=[8])
    host_ptrs = np.zeros(1, np.int64)   # pointer arrays must be device memory
    assert B.iclblasStrsmBatchedUneven(handle, plan, 1.0, host_ptrs, host_ptrs) == B.INVALID_VALUE
    gplan = B.BatchPlan(handle, "gemm", transa=0, transb=0, m=[8], n=[8], k=[8], lda=[8], ldb=[8], ldc=[8])
    d = torch.zeros(1, dtype=torch.int64, device=cuda)
    assert B.iclblasStrsmBatchedUneven(handle, gplan, 1.0, d, d) == B.INVALID_VALUE   # wrong plan kind
    plan.destroy()
    gplan.destroy()


def test_tune_cache_file(tmp_path):
    """ICLBLAS_TUNE_CACHE persists the tuner's choice; a second process with
    the same shapes reads it back (same choice)."""
    cache = tmp_path / "tune.txt"
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "from clgpu_b200 import iclblas as B\n"
        "h = B.Handle()\n"
        "p = B.BatchPlan(h, 'gemm', transa=0, transb=0, m=[100, 200], n=[50, 60], k=[70, 80], lda=[100, 200],"
        " ldb=[70, 80], ldc=[100, 200])\n"
        "print(p.info()[1], p.info()[2])\n"
    ) % ROOT
    env = dict(os.environ, ICLBLAS_TUNE_CACHE=str(cache))
    r1 = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r1.returncode == 0, r1.stderr
    text = cache.read_text()
    assert text.startswith("gemm") and len(text.splitlines()) == 1
    r2 = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r2.returncode == 0, r2.stderr
    assert r1.stdout.split() == r2.stdout.split()
    assert len(cache.read_text().splitlines()) == 1   # read back, not re-tuned


def test_batched_adjoint_reuses_forward_inverses(handle, cuda):
    """With inverse reuse the adjoint skips forming the diagonal-block
    inverses and uses the forward call's: results bit-identical to a plan
    that forms them again.  GEMM plans have no inverses to reuse."""
    handle.set_stream(torch.cuda.current_stream())
    rng = np.random.default_rng(31)
    batch = 17
    ms, ns = rng.integers(1, 400, batch), rng.integers(1, 90, batch)
    As = [tri_np(int(m), True, rng) for m in ms]
    Bs = [rng.standard_normal(int(m) * int(n)).astype(np.float32) for m, n in zip(ms, ns)]
    Gs = [rng.standard_normal(int(m) * int(n)).astype(np.float32) for m, n in zip(ms, ns)]
    kw = dict(side=0, uplo=1, trans=0, diag=0, m=list(ms), n=list(ns), lda=list(ms), ldb=list(ms))
    outs = []
    for reuse in (False, True):
        plan = B.BatchPlan(handle, "trsm", **kw)
        assert plan.set_inverse_reuse(reuse) == B.SUCCESS
        dA = [torch.from_numpy(a).to(cuda) for a in As]
        dX = [torch.from_numpy(b).to(cuda) for b in Bs]
        dG = [torch.from_numpy(g).to(cuda) for g in Gs]
        ddA = [torch.empty(int(m) * int(m), device=cuda) for m in ms]
        pa, px, pg, pda = ptrs(dA, cuda), ptrs(dX, cuda), ptrs(dG, cuda), ptrs(ddA, cuda)
        assert B.iclblasStrsmBatchedUneven(handle, plan, 0.5, pa, px) == B.SUCCESS
        assert B.iclblasStrsmBatchedUnevenBackward(handle, plan, 0.5, pa, px, pg, pda) == B.SUCCESS
        torch.cuda.synchronize()
        outs.append([t.cpu().numpy() for t in dX + dG + ddA])
        plan.destroy()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
    gplan = B.BatchPlan(handle, "gemm", transa=0, transb=0, m=[4], n=[4], k=[4], lda=[4], ldb=[4], ldc=[4])
    assert gplan.set_inverse_reuse(True) == B.INVALID_VALUE
    gplan.destroy()
