// TRSM: op(A) X = alpha*B (left) or X op(A) = alpha*B (right), X overwrites B;
// float and complex, every side/uplo/op/diag combination.
//
// Replaces the reference's single-work-item Strsm_naive / Ctrsm_naive
// (libs/blas/funcs/Strsm/Strsm_naive.cl:18-126, Ctrsm/Ctrsm_naive.cl:18-183),
// which run the whole O(m^2 n) solve on one work item.  Here the solve is
// recursive on the triangular operand M = op(A):
//     left, M lower:   X1 = M11 \ (s*B1);  B2 = s*B2 - M21*X1;  X2 = M22 \ B2
// (and the mirrored orders for upper / right side), so almost all flops run in
// large GEMMs with k = half the remaining size.  As in the reference
// (Strsm_naive.cl:35, Ctrsm_naive.cl:43) the solve runs on the unscaled B and
// alpha multiplies the solution afterwards (one pass over B when alpha != 1);
// scaling B first rounds differently and misses the reference's 4-ulp
// known-answer checks after cancellation.  Leaves of <= 64 rows are solved in
// shared memory, one RHS per thread.  GEMMs use the handle's math mode (the
// plain FP32 default is the CUDA-core kernel).
#include <algorithm>

#include "common.cuh"

namespace iclb {

cudaError_t sgemm_simt(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const float* A, int lda,
                       const float* B, int ldb, float beta, float* C, int ldc);
cudaError_t cgemm_simt(iclblasHandle_t h, int ta, int tb, int m, int n, int k, cfloat alpha, const cfloat* A, int lda,
                       const cfloat* B, int ldb, cfloat beta, cfloat* C, int ldc);

namespace {

// Leaf size: 64 for float, 32 for complex (two 33x32 complex tiles fit the
// static shared-memory limit; 65x64 would not).
template <class T>
struct Leaf {
    static constexpr int value = 64;
};
template <>
struct Leaf<cfloat> {
    static constexpr int value = 32;
};

__device__ __forceinline__ float zero_v(float) { return 0.f; }
__device__ __forceinline__ cfloat zero_v(cfloat) { return cfloat{0.f, 0.f}; }
__device__ __forceinline__ float conj_v(float v) { return v; }
__device__ __forceinline__ cfloat conj_v(cfloat v) { return cfloat{v.re, -v.im}; }
__device__ __forceinline__ float mulv(float a, float b) { return a * b; }
__device__ __forceinline__ cfloat mulv(cfloat a, cfloat b)
{
    return cfloat{fmaf(a.re, b.re, -a.im * b.im), fmaf(a.re, b.im, a.im * b.re)};
}
__device__ __forceinline__ void msub(float& acc, float a, float x) { acc = fmaf(-a, x, acc); }
__device__ __forceinline__ void msub(cfloat& acc, cfloat a, cfloat x)
{
    acc.re = fmaf(-a.re, x.re, acc.re);
    acc.re = fmaf(a.im, x.im, acc.re);
    acc.im = fmaf(-a.re, x.im, acc.im);
    acc.im = fmaf(-a.im, x.re, acc.im);
}
__device__ __forceinline__ float divv(float a, float d) { return a / d; }
__device__ __forceinline__ cfloat divv(cfloat a, cfloat d)
{
    float q = fmaf(d.re, d.re, d.im * d.im);
    return cfloat{fmaf(a.re, d.re, a.im * d.im) / q, fmaf(a.im, d.re, -a.re * d.im) / q};
}

// Leaf solve of an nm x nm triangle.  `op` is how M's elements are read from
// A: M(i,j) = A[a0 + i + j*lda] (op 0), A[a0 + j + i*lda] (op 1),
// conj of the latter (op 2).  Left side: RHS j is column j of B (rows
// 0..nm-1), solved with M.  Right side: RHS i is row i of B, solved with M^T
// (x^T M = b^T).  One thread per RHS; M and the RHS block live in shared memory.
template <class T, int LEAF = Leaf<T>::value>
__global__ void __launch_bounds__(LEAF) trsm_leaf_kernel(int left, int m_lower, int op, int unit, int nm, int nrhs,
                                                         T scale, const T* __restrict__ A, long lda,
                                                         T* __restrict__ B, long ldb)
{
    __shared__ T Ms[LEAF][LEAF + 1];
    __shared__ T Xs[LEAF][LEAF + 1];  // Xs[e][t]: element e of RHS t
    const int t = threadIdx.x;
    const int rhs0 = blockIdx.x * LEAF;
    // M into shared memory, coalesced along A's columns
    for (int idx = t; idx < LEAF * LEAF; idx += LEAF) {
        const int r = idx % LEAF, c = idx / LEAF;  // A-local (r, c)
        T v = zero_v(T());
        if (r < nm && c < nm) v = A[(long)c * lda + r];
        // M(i,j) from A-local (r,c): op 0 -> (r,c); op 1/2 -> (c,r)
        if (op == 0) Ms[r][c] = v;
        else Ms[c][r] = (op == 2) ? conj_v(v) : v;
    }
    // RHS block, scaled
    for (int idx = t; idx < LEAF * LEAF; idx += LEAF) {
        const int a = idx % LEAF, b = idx / LEAF;  // contiguous index first
        T v = zero_v(T());
        if (left) {  // element a of RHS column rhs0+b
            if (a < nm && rhs0 + b < nrhs) v = mulv(B[(long)(rhs0 + b) * ldb + a], scale);
            Xs[a][b] = v;
        } else {  // element b of RHS row rhs0+a
            if (b < nm && rhs0 + a < nrhs) v = mulv(B[(long)b * ldb + rhs0 + a], scale);
            Xs[b][a] = v;
        }
    }
    __syncthreads();
    // Effective triangle: left uses M, right uses M^T (lower <-> upper).
    const bool lower = left ? m_lower : !m_lower;
    if (rhs0 + t < nrhs) {
        if (lower) {
            for (int k = 0; k < nm; ++k) {
                T xk = Xs[k][t];
                if (!unit) xk = divv(xk, left ? Ms[k][k] : Ms[k][k]);
                Xs[k][t] = xk;
                for (int r = k + 1; r < nm; ++r) msub(Xs[r][t], left ? Ms[r][k] : Ms[k][r], xk);
            }
        } else {
            for (int k = nm - 1; k >= 0; --k) {
                T xk = Xs[k][t];
                if (!unit) xk = divv(xk, Ms[k][k]);
                Xs[k][t] = xk;
                for (int r = 0; r < k; ++r) msub(Xs[r][t], left ? Ms[r][k] : Ms[k][r], xk);
            }
        }
    }
    __syncthreads();
    for (int idx = t; idx < LEAF * LEAF; idx += LEAF) {
        const int a = idx % LEAF, b = idx / LEAF;
        if (left) {
            if (a < nm && rhs0 + b < nrhs) B[(long)(rhs0 + b) * ldb + a] = Xs[a][b];
        } else {
            if (b < nm && rhs0 + a < nrhs) B[(long)b * ldb + rhs0 + a] = Xs[b][a];
        }
    }
}

template <class T>
struct Gemm;
template <>
struct Gemm<float> {
    static cudaError_t run(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const float* A, int lda,
                           const float* B, int ldb, float beta, float* C, int ldc)
    {
        return sgemm(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    }
    static float one() { return 1.f; }
    static float minus_one() { return -1.f; }
};
template <>
struct Gemm<cfloat> {
    static cudaError_t run(iclblasHandle_t h, int ta, int tb, int m, int n, int k, cfloat alpha, const cfloat* A,
                           int lda, const cfloat* B, int ldb, cfloat beta, cfloat* C, int ldc)
    {
        return cgemm(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    }
    static cfloat one() { return cfloat{1.f, 0.f}; }
    static cfloat minus_one() { return cfloat{-1.f, 0.f}; }
};

template <class T>
struct Solver {
    static constexpr int LEAF = Leaf<T>::value;
    iclblasHandle_t h;
    int left, op, unit, m_lower;
    const T* A;
    long lda;
    T* B;
    long ldb;
    int nrhs;  // RHS count (n for left, m for right)

    // Pointer and GEMM op of block M[r0.., c0..] of M = op(A).
    const T* mblk(int r0, int c0) const { return op == 0 ? A + r0 + (long)c0 * lda : A + c0 + (long)r0 * lda; }

    // Solve the diagonal range [o, o+sz) of M against the matching part of B.
    cudaError_t solve(int o, int sz, T scale)
    {
        if (sz <= LEAF) {
            const T* a0 = A + o + (long)o * lda;
            T* b0 = left ? B + o : B + (long)o * ldb;
            trsm_leaf_kernel<T><<<ceil_div(nrhs, LEAF), LEAF, 0, h->stream>>>(left, m_lower, op, unit, sz, nrhs,
                                                                                scale, a0, lda, b0, ldb);
            return cudaGetLastError();
        }
        int h1 = (sz / 2 + LEAF - 1) / LEAF * LEAF;  // first half, a multiple of the leaf
        const int o1 = o, s1 = h1, o2 = o + h1, s2 = sz - h1;
        // Forward (first half first) when: left & M lower, or right & M upper.
        const bool forward = left ? m_lower : !m_lower;
        const int fo = forward ? o1 : o2, fs = forward ? s1 : s2;  // solved first
        const int so = forward ? o2 : o1, ss = forward ? s2 : s1;  // updated, solved second
        cudaError_t e = solve(fo, fs, scale);
        if (e != cudaSuccess) return e;
        if (left) {
            // B[so] = scale*B[so] - M[so, fo] * X[fo]
            e = Gemm<T>::run(h, op, ICLBLAS_OP_N, ss, nrhs, fs, Gemm<T>::minus_one(), mblk(so, fo), lda, B + fo, ldb,
                             scale, B + so, ldb);
        } else {
            // B[:, so] = scale*B[:, so] - X[:, fo] * M[fo, so]
            e = Gemm<T>::run(h, ICLBLAS_OP_N, op, nrhs, ss, fs, Gemm<T>::minus_one(), B + (long)fo * ldb, ldb,
                             mblk(fo, so), lda, scale, B + (long)so * ldb, ldb);
        }
        if (e != cudaSuccess) return e;
        return solve(so, ss, Gemm<T>::one());
    }
};

// B[:, :] *= alpha for an m x n column-major block.
template <class T>
__global__ void scale_kernel(int m, int n, T alpha, T* __restrict__ B, long ldb)
{
    const long total = (long)m * n;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long j = e / m, i = e % m;
        T* p = B + j * ldb + i;
        *p = mulv(*p, alpha);
    }
}

__host__ bool is_one(float a) { return a == 1.f; }
__host__ bool is_one(cfloat a) { return a.re == 1.f && a.im == 0.f; }

template <class T>
cudaError_t trsm_impl(iclblasHandle_t h, int side, int uplo, int trans, int diag, int m, int n, T alpha, const T* A,
                      int lda, T* B, int ldb)
{
    Solver<T> s;
    s.h = h;
    s.left = side == ICLBLAS_SIDE_LEFT;
    s.op = trans;
    s.unit = diag == ICLBLAS_DIAG_UNIT;
    const bool lower = uplo == ICLBLAS_FILL_MODE_LOWER;
    s.m_lower = (trans == ICLBLAS_OP_N) ? lower : !lower;
    s.A = A;
    s.lda = lda;
    s.B = B;
    s.ldb = ldb;
    s.nrhs = s.left ? n : m;
    cudaError_t e = s.solve(0, s.left ? m : n, Gemm<T>::one());
    if (e != cudaSuccess || is_one(alpha)) return e;
    const long total = (long)m * n;
    const int grid = (int)std::min<long>((total + 255) / 256, (long)h->sm_count * 8);
    scale_kernel<T><<<grid, 256, 0, h->stream>>>(m, n, alpha, B, ldb);
    return cudaGetLastError();
}

}  // namespace

cudaError_t strsm(iclblasHandle_t h, int side, int uplo, int trans, int diag, int m, int n, float alpha,
                  const float* A, int lda, float* B, int ldb)
{
    return trsm_impl<float>(h, side, uplo, trans == ICLBLAS_OP_C ? ICLBLAS_OP_T : trans, diag, m, n, alpha, A, lda, B,
                            ldb);
}

cudaError_t ctrsm(iclblasHandle_t h, int side, int uplo, int trans, int diag, int m, int n, cfloat alpha,
                  const cfloat* A, int lda, cfloat* B, int ldb)
{
    return trsm_impl<cfloat>(h, side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb);
}

}  // namespace iclb
