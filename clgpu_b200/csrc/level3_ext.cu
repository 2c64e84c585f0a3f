// Level-3 routines built on the GEMM engine: Ssyrk, Ssyr2k, Ssymm, Strmm.
//
// All four are GEMM-shaped, so they run as S GEMM calls in the handle's math
// mode (plain FP32 on the CUDA cores, or TF32 / 3xBF16 / 6xBF16 on the
// tensor cores) plus small bandwidth-bound helper kernels:
//   - Ssyrk / Ssyr2k: the output triangle is split recursively in halves;
//     the off-diagonal block of each split is one GEMM (two for Ssyr2k)
//     applying beta, and each diagonal leaf (at most kLeaf rows) is a full
//     leaf x leaf product into solver scratch followed by a masked update of
//     the stored triangle.  Flops: n^2 k (n^2 k x2 for Ssyr2k) plus the
//     leaves' other halves, n kLeaf k.
//   - Ssymm: the symmetric operand is expanded to a full matrix in solver
//     scratch (its stored triangle read once) and multiplied by one GEMM.
//   - Strmm: the triangular factor op(A) is split recursively; the
//     off-diagonal block of each split is one GEMM accumulating into C, and
//     each diagonal leaf is expanded (zeros outside the triangle, ones on a
//     unit diagonal) and multiplied by one GEMM.  C is a separate output as
//     in the reference's interface (iclBLAS.h:1753); when C overlaps B, B is
//     first copied to solver scratch so the in-place call the reference's
//     own test makes (C == B) gives the product of the original B.
// Solver scratch holds the leaves, the expanded operands and the B copy; the
// GEMMs may grow the general scratch without disturbing it.
#include <algorithm>

#include "common.cuh"

namespace iclb {
namespace {

constexpr int kThreads = 256;
constexpr int kLeaf = 256;

// ------------------------------------------------------------------ helpers
// C(i,j) over the stored triangle of an n x n block = W(i,j) (+ W(j,i) when
// SYM2) + beta C(i,j); beta == 0 writes C without reading it.
template <bool SYM2>
__global__ void __launch_bounds__(kThreads) tri_update_kernel(int n, bool lower, const float* __restrict__ W, int ldw,
                                                              float beta, float* C, long ldc)
{
    const long total = (long)n * n;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const int i = (int)(e % n), j = (int)(e / n);
        if (lower ? (i < j) : (i > j)) continue;
        float v = W[(long)j * ldw + i];
        if (SYM2) v = __fadd_rn(v, W[(long)i * ldw + j]);
        float* c = C + (long)j * ldc + i;
        *c = (beta != 0.f) ? fmaf(beta, *c, v) : v;
    }
}

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

// Split point: half of n rounded to a multiple of 64 (at least 64).
int split_of(int n) { return std::max(64, ((n / 2) + 63) / 64 * 64); }

// ------------------------------------------------------------------ syrk / syr2k
struct Rk {
    iclblasHandle_t h;
    bool lower, trans;  // trans: C = alpha op(A)^T op(B) with A, B k x n
    int k;
    float alpha, beta;
    const float *A, *B;  // B == nullptr: syrk
    int lda, ldb;
    float* C;
    int ldc;
    float* W;  // kLeaf x kLeaf leaf buffer

    // pointer to rows [r, ...) of op(X) (X = A or B)
    const float* rows(const float* X, int ld, int r) const { return trans ? X + (long)r * ld : X + r; }

    // P = alpha * opX(rows r..) * opY(rows c..)^T (+ beta0 P), P an mr x nc block of C or W
    cudaError_t prod(const float* X, int ldx, const float* Y, int ldy, int r, int c, int mr, int nc, float beta0,
                     float* P, int ldp) const
    {
        // trans == false: X is n x k, product X_r Y_c^T = gemm(N, T);
        // trans == true:  X is k x n, product X_r^T Y_c = gemm(T, N).
        return sgemm(h, trans ? 1 : 0, trans ? 0 : 1, mr, nc, k, alpha, rows(X, ldx, r), ldx, rows(Y, ldy, c), ldy,
                     beta0, P, ldp);
    }

    cudaError_t run(int off, int n) const
    {
        if (n <= kLeaf) {
            cudaError_t e = prod(A, lda, B ? B : A, B ? ldb : lda, off, off, n, n, 0.f, W, kLeaf);
            if (e != cudaSuccess) return e;
            float* Cb = C + (long)off * ldc + off;
            if (B)
                tri_update_kernel<true><<<grid_for(h, (long)n * n), kThreads, 0, h->stream>>>(n, lower, W, kLeaf, beta,
                                                                                              Cb, ldc);
            else
                tri_update_kernel<false><<<grid_for(h, (long)n * n), kThreads, 0, h->stream>>>(n, lower, W, kLeaf,
                                                                                               beta, Cb, ldc);
            return cudaGetLastError();
        }
        const int n1 = split_of(n), n2 = n - n1;
        cudaError_t e = run(off, n1);
        if (e != cudaSuccess) return e;
        e = run(off + n1, n2);
        if (e != cudaSuccess) return e;
        // off-diagonal block: lower C21 (rows off+n1.., cols off..), upper C12
        const int r = lower ? off + n1 : off, c = lower ? off : off + n1;
        const int mr = lower ? n2 : n1, nc = lower ? n1 : n2;
        float* P = C + (long)c * ldc + r;
        if (!B) return prod(A, lda, A, lda, r, c, mr, nc, beta, P, ldc);
        e = prod(A, lda, B, ldb, r, c, mr, nc, beta, P, ldc);
        if (e != cudaSuccess) return e;
        return prod(B, ldb, A, lda, r, c, mr, nc, 1.f, P, ldc);
    }
};

// ------------------------------------------------------------------ trmm
struct Tm {
    iclblasHandle_t h;
    bool left, lower, ta, unit;  // lower: A's stored triangle; ta: op(A) = A^T
    float alpha;
    const float* A;
    int lda;
    const float* B;
    int ldb;
    float* C;
    int ldc;
    int m, n;  // C is m x n
    float* D;  // kLeaf x kLeaf leaf buffer

    // op(A) block rows [r, r+nr) x cols [c, c+nc) as a GEMM operand: pointer and transpose flag
    const float* opblk(int r, int c) const { return ta ? A + (long)r * lda + c : A + (long)c * lda + r; }

    // effective triangle of op(A)
    bool op_lower() const { return lower != ta; }

    // C rows/cols [off, off+t) <- alpha * op(A)[off.., off..] applied to B (left: rows, right: cols)
    cudaError_t run(int off, int t, float beta0) const
    {
        if (t <= kLeaf) {
            expand_tri_kernel<<<grid_for(h, (long)t * t), kThreads, 0, h->stream>>>(
                t, lower, unit, A + (long)off * lda + off, lda, D);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
            if (left)
                return sgemm(h, ta ? 1 : 0, 0, t, n, t, alpha, D, t, B + off, ldb, beta0, C + off, ldc);
            return sgemm(h, 0, ta ? 1 : 0, m, t, t, alpha, B + (long)off * ldb, ldb, D, t, beta0,
                         C + (long)off * ldc, ldc);
        }
        const int t1 = split_of(t), t2 = t - t1;
        const int o1 = off, o2 = off + t1;
        const bool L = op_lower();
        if (left) {
            // C1 = a T11 B1 (+ a T12 B2 if upper); C2 = a T22 B2 (+ a T21 B1 if lower)
            cudaError_t e = run(o1, t1, beta0);
            if (e == cudaSuccess) e = run(o2, t2, beta0);
            if (e != cudaSuccess) return e;
            if (L)
                return sgemm(h, ta ? 1 : 0, 0, t2, n, t1, alpha, opblk(o2, o1), lda, B + o1, ldb, 1.f, C + o2, ldc);
            return sgemm(h, ta ? 1 : 0, 0, t1, n, t2, alpha, opblk(o1, o2), lda, B + o2, ldb, 1.f, C + o1, ldc);
        }
        // right: C1 = a B1 T11 (+ a B2 T21 if lower); C2 = a B2 T22 (+ a B1 T12 if upper)
        cudaError_t e = run(o1, t1, beta0);
        if (e == cudaSuccess) e = run(o2, t2, beta0);
        if (e != cudaSuccess) return e;
        if (L)
            return sgemm(h, 0, ta ? 1 : 0, m, t1, t2, alpha, B + (long)o2 * ldb, ldb, opblk(o2, o1), lda, 1.f,
                         C + (long)o1 * ldc, ldc);
        return sgemm(h, 0, ta ? 1 : 0, m, t2, t1, alpha, B + (long)o1 * ldb, ldb, opblk(o1, o2), lda, 1.f,
                     C + (long)o2 * ldc, ldc);
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
    float* W = (float*)solver_scratch(h, sizeof(float) * kLeaf * kLeaf);
    if (!W) return cudaErrorMemoryAllocation;
    Rk r{h, uplo == ICLBLAS_FILL_MODE_LOWER, trans != ICLBLAS_OP_N, k, alpha, beta, A, nullptr, lda, 0, C, ldc, W};
    return r.run(0, n);
}

cudaError_t ssyr2k(iclblasHandle_t h, int uplo, int trans, int n, int k, float alpha, const float* A, int lda,
                   const float* B, int ldb, float beta, float* C, int ldc)
{
    float* W = (float*)solver_scratch(h, sizeof(float) * kLeaf * kLeaf);
    if (!W) return cudaErrorMemoryAllocation;
    Rk r{h, uplo == ICLBLAS_FILL_MODE_LOWER, trans != ICLBLAS_OP_N, k, alpha, beta, A, B, lda, ldb, C, ldc, W};
    return r.run(0, n);
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
    const bool copy_b = overlaps(B, extent_bytes(m, n, ldb), C, extent_bytes(m, n, ldc));
    const size_t leaf_bytes = sizeof(float) * kLeaf * kLeaf;
    const size_t bcopy_bytes = copy_b ? sizeof(float) * (size_t)m * (size_t)n : 0;
    char* ws = (char*)solver_scratch(h, leaf_bytes + bcopy_bytes);
    if (!ws) return cudaErrorMemoryAllocation;
    const float* Bsrc = B;
    int ldbs = ldb;
    if (copy_b) {
        float* Bc = (float*)(ws + leaf_bytes);
        copy_matrix_kernel<<<grid_for(h, (long)m * n), kThreads, 0, h->stream>>>(m, n, B, ldb, Bc, m);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        Bsrc = Bc;
        ldbs = m;
    }
    const bool left = side == ICLBLAS_SIDE_LEFT;
    Tm t{h, left, uplo == ICLBLAS_FILL_MODE_LOWER, transa != ICLBLAS_OP_N, diag == ICLBLAS_DIAG_UNIT,
         alpha, A, lda, Bsrc, ldbs, C, ldc, m, n, (float*)ws};
    return t.run(0, left ? m : n, 0.f);
}

}  // namespace iclb
