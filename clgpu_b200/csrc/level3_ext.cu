// Level-3 routines built on the GEMM engine: Ssyrk, Ssyr2k, Ssymm, Strmm.
//
// All four are GEMM-shaped, so they run as S GEMM calls in the handle's math
// mode (plain FP32 on the CUDA cores, or TF32 / 3xBF16 / 6xBF16 on the
// tensor cores) plus small bandwidth-bound helper kernels.  Each GEMM is
// kept large so that it fills the GPU: deep-K GEMMs with small outputs,
// which a recursive halving down to small leaves produces, ran these
// routines at a fifth of the GEMM rate.
//   - Ssyrk / Ssyr2k: one GEMM (two for Ssyr2k) in the engines'
//     triangular-output mode, which computes only the tiles meeting C's
//     triangle and writes (and, for beta, reads) only the triangle.
//   - Ssymm: the symmetric operand is expanded to a full matrix in solver
//     scratch (its stored triangle read once) and multiplied by one GEMM.
//   - Strmm: the triangle of A is expanded (zeros outside it, ones on a
//     unit diagonal); C is formed in panels, each one GEMM over the non-zero
//     part of the expanded factor.  C is a separate output as in the
//     reference's interface (iclBLAS.h:1753); when C overlaps B, B is first
//     copied to solver scratch so the in-place call the reference's own test
//     makes (C == B) gives the product of the original B.
// Solver scratch holds the expanded operands and the B copy; the GEMMs may
// grow the general scratch without disturbing it.
#include <algorithm>

#include "common.cuh"

namespace iclb {
namespace {

constexpr int kThreads = 256;

// ------------------------------------------------------------------ helpers
// Full n x n symmetric matrix F from the stored triangle of A.
__global__ void __launch_bounds__(kThreads) symmetrize_kernel(int n, bool lower, const float* __restrict__ A, long lda,
                                                              float* __restrict__ F)
{
    const long total = (long)n * n;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const int i = (int)(e % n), j = (int)(e / n);
        const bool stored = lower ? (i >= j) : (i <= j);
        F[e] = stored ? A[(long)j * lda + i] : A[(long)i * lda + j];
    }
}

// Dense n x n copy of a triangular block of A: the stored triangle, zeros
// elsewhere, ones on a unit diagonal.
__global__ void __launch_bounds__(kThreads) expand_tri_kernel(int n, bool lower, bool unit, const float* __restrict__ A,
                                                              long lda, float* __restrict__ D)
{
    const long total = (long)n * n;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const int i = (int)(e % n), j = (int)(e / n);
        float v;
        if (i == j) v = unit ? 1.f : A[(long)j * lda + i];
        else v = (lower ? (i > j) : (i < j)) ? A[(long)j * lda + i] : 0.f;
        D[e] = v;
    }
}

__global__ void __launch_bounds__(kThreads) copy_matrix_kernel(int m, int n, const float* __restrict__ S, long lds,
                                                               float* __restrict__ D, long ldd)
{
    const long total = (long)m * n;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long i = e % m, j = e / m;
        D[j * ldd + i] = S[j * lds + i];
    }
}

int grid_for(iclblasHandle_t h, long units)
{
    long g = (units + kThreads - 1) / kThreads;
    g = std::min<long>(g, (long)h->sm_count * 8);
    return (int)std::max<long>(g, 1);
}

// ------------------------------------------------------------------ panels
// Panel width for a triangular dimension of t: about t/8, a multiple of 128,
// within [256, 2048]; t itself when that is smaller.
int panel_of(int t)
{
    int p = ((t + 7) / 8 + 127) / 128 * 128;
    p = std::max(256, std::min(2048, p));
    return std::min(p, t);
}

// ------------------------------------------------------------------ syrk / syr2k
// One triangular-output GEMM (two for Ssyr2k): the GEMM engines skip the
// tiles wholly outside C's triangle and mask the diagonal tiles, so the
// flops are n^2 k plus the diagonal tiles' other halves.
struct Rk {
    iclblasHandle_t h;
    bool lower, trans;  // trans: C = alpha op(A)^T op(B) with A, B k x n
    int n, k;
    float alpha, beta;
    const float *A, *B;  // B == nullptr: syrk
    int lda, ldb;
    float* C;
    int ldc;

    cudaError_t run() const
    {
        const int tri = lower ? 1 : 2;
        // trans == false: op(X) = X (n x k), product X Y^T = gemm(N, T); else X^T Y = gemm(T, N)
        const int ta = trans ? 1 : 0, tb = trans ? 0 : 1;
        cudaError_t e = sgemm_tri(h, tri, ta, tb, n, n, k, alpha, A, lda, B ? B : A, B ? ldb : lda, beta, C, ldc);
        if (e == cudaSuccess && B) e = sgemm_tri(h, tri, ta, tb, n, n, k, alpha, B, ldb, A, lda, 1.f, C, ldc);
        return e;
    }
};

// ------------------------------------------------------------------ trmm
// The triangle of A is expanded once into a dense matrix D (zeros outside
// it, ones on a unit diagonal).  C is then formed in panels along the
// triangular dimension, each one GEMM over the part of D's rows or columns
// that is not zero for it: a fraction panel / dim of extra flops.
struct Tm {
    iclblasHandle_t h;
    bool left, ta, oplower;  // ta: op(A) = A^T; oplower: op(A) is lower triangular
    float alpha;
    const float* D;  // dense na x na expansion of A's triangle, ld = na
    int na;
    const float* B;
    int ldb;
    float* C;
    int ldc;
    int m, n;

    // op(D) block starting at (r, c), as a GEMM operand
    const float* opblk(int r, int c) const { return ta ? D + (long)r * na + c : D + (long)c * na + r; }

    cudaError_t run() const
    {
        const int pw = panel_of(na);
        for (int p0 = 0; p0 < na; p0 += pw) {
            const int w = std::min(pw, na - p0);
            cudaError_t e;
            if (left) {
                // C rows [p0, p0+w) = alpha op(D)[p0.., k0..k1) B[k0..k1, :]
                const int k0 = oplower ? 0 : p0, k1 = oplower ? p0 + w : na;
                e = sgemm(h, ta ? 1 : 0, 0, w, n, k1 - k0, alpha, opblk(p0, k0), na, B + k0, ldb, 0.f, C + p0, ldc);
            } else {
                // C cols [p0, p0+w) = alpha B[:, k0..k1) op(D)[k0..k1, p0..)
                const int k0 = oplower ? p0 : 0, k1 = oplower ? na : p0 + w;
                e = sgemm(h, 0, ta ? 1 : 0, m, w, k1 - k0, alpha, B + (long)k0 * ldb, ldb, opblk(k0, p0), na, 0.f,
                          C + (long)p0 * ldc, ldc);
            }
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
};

bool overlaps(const void* a, size_t abytes, const void* b, size_t bbytes)
{
    const char *pa = (const char*)a, *pb = (const char*)b;
    return pa < pb + bbytes && pb < pa + abytes;
}

size_t extent_bytes(int rows, int cols, int ld)
{
    return (rows > 0 && cols > 0) ? ((size_t)(cols - 1) * (size_t)ld + (size_t)rows) * sizeof(float) : 0;
}

}  // namespace

cudaError_t ssyrk(iclblasHandle_t h, int uplo, int trans, int n, int k, float alpha, const float* A, int lda,
                  float beta, float* C, int ldc)
{
    Rk r{h, uplo == ICLBLAS_FILL_MODE_LOWER, trans != ICLBLAS_OP_N, n, k, alpha, beta, A, nullptr, lda, 0, C, ldc};
    return r.run();
}

cudaError_t ssyr2k(iclblasHandle_t h, int uplo, int trans, int n, int k, float alpha, const float* A, int lda,
                   const float* B, int ldb, float beta, float* C, int ldc)
{
    Rk r{h, uplo == ICLBLAS_FILL_MODE_LOWER, trans != ICLBLAS_OP_N, n, k, alpha, beta, A, B, lda, ldb, C, ldc};
    return r.run();
}

cudaError_t ssymm(iclblasHandle_t h, int side, int uplo, int m, int n, float alpha, const float* A, int lda,
                  const float* B, int ldb, float beta, float* C, int ldc)
{
    const bool left = side == ICLBLAS_SIDE_LEFT;
    const int na = left ? m : n;
    float* F = (float*)solver_scratch(h, sizeof(float) * (size_t)na * (size_t)na);
    if (!F) return cudaErrorMemoryAllocation;
    symmetrize_kernel<<<grid_for(h, (long)na * na), kThreads, 0, h->stream>>>(na, uplo == ICLBLAS_FILL_MODE_LOWER, A,
                                                                             lda, F);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (left) return sgemm(h, 0, 0, m, n, m, alpha, F, na, B, ldb, beta, C, ldc);
    return sgemm(h, 0, 0, m, n, n, alpha, B, ldb, F, na, beta, C, ldc);
}

cudaError_t strmm(iclblasHandle_t h, int side, int uplo, int transa, int diag, int m, int n, float alpha,
                  const float* A, int lda, const float* B, int ldb, float* C, int ldc)
{
    if (alpha == 0.f)  // C = 0; A and B are not read
        return sgemm(h, 0, 0, m, n, 0, 0.f, nullptr, 1, nullptr, 1, 0.f, C, ldc);
    const bool left = side == ICLBLAS_SIDE_LEFT;
    const int na = left ? m : n;
    const bool copy_b = overlaps(B, extent_bytes(m, n, ldb), C, extent_bytes(m, n, ldc));
    const size_t d_bytes = ((sizeof(float) * (size_t)na * (size_t)na) + 255) & ~(size_t)255;
    const size_t bcopy_bytes = copy_b ? sizeof(float) * (size_t)m * (size_t)n : 0;
    char* ws = (char*)solver_scratch(h, d_bytes + bcopy_bytes);
    if (!ws) return cudaErrorMemoryAllocation;
    float* D = (float*)ws;
    const bool lower = uplo == ICLBLAS_FILL_MODE_LOWER, ta = transa != ICLBLAS_OP_N;
    expand_tri_kernel<<<grid_for(h, (long)na * na), kThreads, 0, h->stream>>>(na, lower, diag == ICLBLAS_DIAG_UNIT, A,
                                                                             lda, D);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const float* Bsrc = B;
    int ldbs = ldb;
    if (copy_b) {
        float* Bc = (float*)(ws + d_bytes);
        copy_matrix_kernel<<<grid_for(h, (long)m * n), kThreads, 0, h->stream>>>(m, n, B, ldb, Bc, m);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        Bsrc = Bc;
        ldbs = m;
    }
    Tm t{h, left, ta, lower != ta, alpha, D, na, Bsrc, ldbs, C, ldc, m, n};
    return t.run();
}

}  // namespace iclb
