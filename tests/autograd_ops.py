"""Test-only torch.autograd.Function wrappers over the library's C ABI.

The forward calls iclblasStrsm / iclblasSgemm and the backward calls the
hand-written adjoints iclblasStrsm_backward / iclblasSgemm_backward, on the
tensors' device memory.  Logical matrices are ordinary (row-major) torch
tensors; they are handed to the column-major library as transposed
contiguous copies.
"""
import torch

from clgpu_b200 import iclblas as B


def _cm(t):
    """Column-major storage of a logical 2-D matrix (a contiguous t^T)."""
    return t.t().contiguous()


class Trsm(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A, Bm, side, uplo, trans, diag, alpha, handle):
        m, n = Bm.shape
        na = A.shape[0]
        Acm = _cm(A)
        Xcm = _cm(Bm)
        B.check(B.iclblasStrsm(handle, side, uplo, trans, diag, m, n, alpha, Acm, na, Xcm, m), "iclblasStrsm")
        ctx.save_for_backward(Acm, Xcm)
        ctx.cfg = (side, uplo, trans, diag, alpha, handle, m, n, na)
        return Xcm.t()

    @staticmethod
    def backward(ctx, G):
        Acm, Xcm = ctx.saved_tensors
        side, uplo, trans, diag, alpha, handle, m, n, na = ctx.cfg
        Gcm = _cm(G)
        dAcm = torch.zeros_like(Acm)
        B.check(B.iclblasStrsm_backward(handle, side, uplo, trans, diag, m, n, alpha, Acm, na, Xcm, m, Gcm, m, dAcm,
                                        na), "iclblasStrsm_backward")
        return dAcm.t(), Gcm.t(), None, None, None, None, None, None


class Gemm(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A, Bm, Cin, transa, transb, alpha, beta, handle):
        m, n = Cin.shape
        k = A.shape[1] if transa == 0 else A.shape[0]
        Acm, Bcm, Ccm = _cm(A), _cm(Bm), _cm(Cin)
        lda, ldb = A.shape[0], Bm.shape[0]
        B.check(B.iclblasSgemm(handle, transa, transb, m, n, k, alpha, Acm, lda, Bcm, ldb, beta, Ccm, m),
                "iclblasSgemm")
        ctx.save_for_backward(Acm, Bcm)
        ctx.cfg = (transa, transb, alpha, beta, handle, m, n, k, lda, ldb, A.shape, Bm.shape)
        return Ccm.t()

    @staticmethod
    def backward(ctx, G):
        Acm, Bcm = ctx.saved_tensors
        transa, transb, alpha, beta, handle, m, n, k, lda, ldb, ashape, bshape = ctx.cfg
        Gcm = _cm(G)
        dA = torch.empty_like(Acm)
        dB = torch.empty_like(Bcm)
        dC = torch.empty_like(Gcm)
        B.check(B.iclblasSgemm_backward(handle, transa, transb, m, n, k, alpha, Acm, lda, Bcm, ldb, beta, Gcm, m, dA,
                                        lda, dB, ldb, dC, m), "iclblasSgemm_backward")
        return dA.t(), dB.t(), dC.t(), None, None, None, None, None
