// Adjoints (reverse-mode derivatives) of TRSM and GEMM.  No reference
// counterpart.
//
// TRSM, left side, X = alpha * M^-1 * B with M = op(A):
//     W = M^-T G                      (TRSM with the transposed operator)
//     dB = alpha * W
//     dM = -W X^T,   dA = dM (op N) or dM^T (op T/C), kept on the stored
//                    triangle (and off the diagonal for a unit diagonal).
// Right side, X = alpha * B * M^-1:
//     W = G M^-T,  dB = alpha * W,  dM = -X^T W.
// GEMM, C = alpha*op(A)*op(B) + beta*C:
//     d op(A) = alpha * G op(B)^T,  d op(B) = alpha * op(A)^T G,  dC = beta * G.
// The products run through the library's GEMM and TRSM (and so follow the
// handle's math mode).  dA is formed by the triangular-output GEMM, which
// computes only the tiles meeting the stored triangle; one small kernel then
// zeroes the other triangle (and a unit diagonal).
#include "common.cuh"

namespace iclb {

namespace {

// Zero the entries of the n x n block that are not on the stored triangle
// (the triangular-output GEMM leaves them untouched); with a unit diagonal
// the diagonal is not an input either.
__global__ void mask_triangle_kernel(int n, int lower, int unit, float* __restrict__ D, long ldd)
{
    const long total = (long)n * n;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const int j = (int)(e / n), i = (int)(e % n);
        const bool keep = lower ? (i > j || (i == j && !unit)) : (i < j || (i == j && !unit));
        if (!keep) D[(long)j * ldd + i] = 0.f;
    }
}

// D = s * S (m x n blocks, column-major)
__global__ void scale_copy_kernel(int m, int n, float s, const float* __restrict__ S, long lds, float* __restrict__ D,
                                  long ldd)
{
    const long total = (long)m * n;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long j = e / m, i = e % m;
        D[j * ldd + i] = s * S[j * lds + i];
    }
}

int grid_for(iclblasHandle_t h, long total)
{
    long g = (total + 255) / 256;
    long cap = (long)h->sm_count * 8;
    return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace

cudaError_t strsm_backward(iclblasHandle_t h, int side, int uplo, int trans, int diag, int m, int n, float alpha,
                           const float* A, int lda, const float* X, int ldx, float* G, int ldg, float* dA, int ldda)
{
    const bool left = side == ICLBLAS_SIDE_LEFT;
    const bool t = trans != ICLBLAS_OP_N;
    const int flipped = t ? ICLBLAS_OP_N : ICLBLAS_OP_T;
    // W in place of G
    cudaError_t e = strsm(h, side, uplo, flipped, diag, m, n, 1.f, A, lda, G, ldg);
    if (e != cudaSuccess) return e;
    if (dA) {
        const int na = left ? m : n;
        // only the stored triangle of dA is formed (1: row >= col, 2: row <= col)
        const int tri = uplo == ICLBLAS_FILL_MODE_LOWER ? 1 : 2;
        if (left) {
            // dM = -W X^T (m x m, inner n); dA = dM or dM^T = -X W^T
            e = t ? sgemm_tri(h, tri, ICLBLAS_OP_N, ICLBLAS_OP_T, m, m, n, -1.f, X, ldx, G, ldg, 0.f, dA, ldda)
                  : sgemm_tri(h, tri, ICLBLAS_OP_N, ICLBLAS_OP_T, m, m, n, -1.f, G, ldg, X, ldx, 0.f, dA, ldda);
        } else {
            // dM = -X^T W (n x n, inner m); dA = dM or dM^T = -W^T X
            e = t ? sgemm_tri(h, tri, ICLBLAS_OP_T, ICLBLAS_OP_N, n, n, m, -1.f, G, ldg, X, ldx, 0.f, dA, ldda)
                  : sgemm_tri(h, tri, ICLBLAS_OP_T, ICLBLAS_OP_N, n, n, m, -1.f, X, ldx, G, ldg, 0.f, dA, ldda);
        }
        if (e != cudaSuccess) return e;
        mask_triangle_kernel<<<grid_for(h, (long)na * na), 256, 0, h->stream>>>(
            na, uplo == ICLBLAS_FILL_MODE_LOWER, diag == ICLBLAS_DIAG_UNIT, dA, ldda);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (alpha != 1.f) {
        scale_copy_kernel<<<grid_for(h, (long)m * n), 256, 0, h->stream>>>(m, n, alpha, G, ldg, G, ldg);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t sgemm_backward(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const float* A, int lda,
                           const float* B, int ldb, float beta, const float* G, int ldg, float* dA, int ldda,
                           float* dB, int lddb, float* dC, int lddc)
{
    const bool at = ta != ICLBLAS_OP_N, bt = tb != ICLBLAS_OP_N;
    cudaError_t e = cudaSuccess;
    if (dA) {
        // d op(A) = alpha G op(B)^T (m x k); stored A is op(A) or its transpose
        if (!at)
            e = bt ? sgemm(h, ICLBLAS_OP_N, ICLBLAS_OP_N, m, k, n, alpha, G, ldg, B, ldb, 0.f, dA, ldda)
                   : sgemm(h, ICLBLAS_OP_N, ICLBLAS_OP_T, m, k, n, alpha, G, ldg, B, ldb, 0.f, dA, ldda);
        else
            e = bt ? sgemm(h, ICLBLAS_OP_T, ICLBLAS_OP_T, k, m, n, alpha, B, ldb, G, ldg, 0.f, dA, ldda)
                   : sgemm(h, ICLBLAS_OP_N, ICLBLAS_OP_T, k, m, n, alpha, B, ldb, G, ldg, 0.f, dA, ldda);
        if (e != cudaSuccess) return e;
    }
    if (dB) {
        // d op(B) = alpha op(A)^T G (k x n)
        if (!bt)
            e = at ? sgemm(h, ICLBLAS_OP_N, ICLBLAS_OP_N, k, n, m, alpha, A, lda, G, ldg, 0.f, dB, lddb)
                   : sgemm(h, ICLBLAS_OP_T, ICLBLAS_OP_N, k, n, m, alpha, A, lda, G, ldg, 0.f, dB, lddb);
        else
            e = at ? sgemm(h, ICLBLAS_OP_T, ICLBLAS_OP_T, n, k, m, alpha, G, ldg, A, lda, 0.f, dB, lddb)
                   : sgemm(h, ICLBLAS_OP_T, ICLBLAS_OP_N, n, k, m, alpha, G, ldg, A, lda, 0.f, dB, lddb);
        if (e != cudaSuccess) return e;
    }
    if (dC) {
        scale_copy_kernel<<<grid_for(h, (long)m * n), 256, 0, h->stream>>>(m, n, beta, G, ldg, dC, lddc);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace iclb
