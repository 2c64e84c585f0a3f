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

// ------------------------------------------------------------------ FP64 leaves
template <class T>
struct Wide;
template <>
struct Wide<float> {
    using type = double;
};
template <>
struct Wide<cfloat> {
    using type = double2;
};

__device__ __forceinline__ double wz(double) { return 0.0; }
__device__ __forceinline__ double2 wz(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double widen(float a) { return (double)a; }
__device__ __forceinline__ double2 widen(cfloat a) { return make_double2(a.re, a.im); }
__device__ __forceinline__ float narrow(double a, float) { return (float)a; }
__device__ __forceinline__ cfloat narrow(double2 a, cfloat) { return cfloat{(float)a.x, (float)a.y}; }
__device__ __forceinline__ double wone(double) { return 1.0; }
__device__ __forceinline__ double2 wone(double2) { return make_double2(1.0, 0.0); }
__device__ __forceinline__ void wfma(double& acc, double a, double b) { acc = fma(a, b, acc); }
__device__ __forceinline__ void wfma(double2& acc, double2 a, double2 b)
{
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}
__device__ __forceinline__ void wfms(double& acc, double a, double b) { acc = fma(-a, b, acc); }
__device__ __forceinline__ void wfms(double2& acc, double2 a, double2 b)
{
    acc.x = fma(-a.x, b.x, fma(a.y, b.y, acc.x));
    acc.y = fma(-a.x, b.y, fma(-a.y, b.x, acc.y));
}
__device__ __forceinline__ double wdiv(double a, double d) { return a / d; }
__device__ __forceinline__ double2 wdiv(double2 a, double2 d)
{
    const double q = d.x * d.x + d.y * d.y;
    return make_double2((a.x * d.x + a.y * d.y) / q, (a.y * d.x - a.x * d.y) / q);
}

// Inverse in FP64 of every NB x NB diagonal block of M = op(A) (the last
// block may be partial).  M(i,j) = A[i + j*lda] (op 0) or A[j + i*lda]
// (op 1; op 2 conjugates).  Block b is written column-major to
// inv[b*NB*NB ...], zero outside the block.  Thread j forms column j of the
// inverse by substitution on e_j.
template <class T, int NB>
__global__ void __launch_bounds__(NB) trsm_inv_diag_kernel(int n, int op, int m_lower, int unit,
                                                           const T* __restrict__ A, long lda,
                                                           typename Wide<T>::type* __restrict__ inv)
{
    using W = typename Wide<T>::type;
    extern __shared__ uint8_t smem_raw[];
    W(*M)[NB + 1] = (W(*)[NB + 1])smem_raw;
    W(*Y)[NB + 1] = M + NB;
    const int b = blockIdx.x, o = b * NB, nb = min(NB, n - o);
    for (int idx = threadIdx.x; idx < NB * NB; idx += NB) {
        const int r = idx % NB, c = idx / NB;  // A-local (r, c): coalesced down A's columns
        W v = wz(W());
        if (r < nb && c < nb) {
            T a = A[(long)(o + c) * lda + (o + r)];
            if (op == 2) a = conj_v(a);
            v = widen(a);
        }
        if (op == 0) M[r][c] = v;
        else M[c][r] = v;
    }
    __syncthreads();
    const int j = threadIdx.x;
    if (m_lower) {
        for (int i = 0; i < NB; ++i) {
            W y = wz(W());
            if (i >= j && i < nb && j < nb) {
                y = (i == j) ? wone(W()) : wz(W());
                for (int k = j; k < i; ++k) wfms(y, M[i][k], Y[k][j]);
                if (!unit) y = wdiv(y, M[i][i]);
            }
            Y[i][j] = y;
        }
    } else {
        for (int i = NB - 1; i >= 0; --i) {
            W y = wz(W());
            if (i <= j && i < nb && j < nb) {
                y = (i == j) ? wone(W()) : wz(W());
                for (int k = i + 1; k <= j; ++k) wfms(y, M[i][k], Y[k][j]);
                if (!unit) y = wdiv(y, M[i][i]);
            }
            Y[i][j] = y;
        }
    }
    __syncthreads();
    W* out = inv + (long)b * NB * NB;
    for (int idx = threadIdx.x; idx < NB * NB; idx += NB) out[idx] = Y[idx % NB][idx / NB];
}

// Leaf of a left solve: B[0:nb, r] = inv * B[0:nb, r] for the RHS columns of
// this block (64 per CTA), in FP64.  Thread t owns row t % NB of the block
// and RHS columns t / NB + G*q (G = 256 / NB groups).
template <class T, int NB>
__global__ void __launch_bounds__(256) trsm_apply_left_kernel(int nb, int nrhs, const typename Wide<T>::type* inv,
                                                              T* __restrict__ B, long ldb)
{
    using W = typename Wide<T>::type;
    constexpr int R = 64;        // RHS per CTA
    constexpr int G = 256 / NB;  // RHS groups
    constexpr int Q = R / G;     // RHS per thread
    extern __shared__ uint8_t smem_raw[];
    W(*Iv)[NB + 1] = (W(*)[NB + 1])smem_raw;
    W(*Bv)[R + 1] = (W(*)[R + 1])(smem_raw + sizeof(W) * NB * (NB + 1));
    const int r0 = blockIdx.x * R;
    for (int idx = threadIdx.x; idx < NB * NB; idx += 256) Iv[idx % NB][idx / NB] = inv[idx];
    for (int idx = threadIdx.x; idx < NB * R; idx += 256) {
        const int k = idx % NB, r = idx / NB;
        W v = wz(W());
        if (k < nb && r0 + r < nrhs) v = widen(B[(long)(r0 + r) * ldb + k]);
        Bv[k][r] = v;
    }
    __syncthreads();
    const int i = threadIdx.x % NB, g = threadIdx.x / NB;
    W acc[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) acc[q] = wz(W());
    for (int k = 0; k < nb; ++k) {
        const W a = Iv[i][k];
#pragma unroll
        for (int q = 0; q < Q; ++q) wfma(acc[q], a, Bv[k][g + G * q]);
    }
    if (i < nb) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int r = r0 + g + G * q;
            if (r < nrhs) B[(long)r * ldb + i] = narrow(acc[q], T());
        }
    }
}

// Leaf of a right solve: B[r, 0:nb] = B[r, 0:nb] * inv for the rows of this
// block (64 per CTA), in FP64.  Thread t owns row t % 64 and columns
// t / 64 + 4*q.
template <class T, int NB>
__global__ void __launch_bounds__(256) trsm_apply_right_kernel(int nb, int nrows, const typename Wide<T>::type* inv,
                                                               T* __restrict__ B, long ldb)
{
    using W = typename Wide<T>::type;
    constexpr int R = 64;  // rows per CTA
    constexpr int Q = NB / 4;
    extern __shared__ uint8_t smem_raw[];
    W(*Iv)[NB + 1] = (W(*)[NB + 1])smem_raw;
    W(*Bv)[NB + 1] = (W(*)[NB + 1])(smem_raw + sizeof(W) * NB * (NB + 1));
    const int r0 = blockIdx.x * R;
    for (int idx = threadIdx.x; idx < NB * NB; idx += 256) Iv[idx % NB][idx / NB] = inv[idx];
    for (int idx = threadIdx.x; idx < R * NB; idx += 256) {
        const int r = idx % R, k = idx / R;
        W v = wz(W());
        if (k < nb && r0 + r < nrows) v = widen(B[(long)k * ldb + r0 + r]);
        Bv[r][k] = v;
    }
    __syncthreads();
    const int r = threadIdx.x % R, g = threadIdx.x / R;
    W acc[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) acc[q] = wz(W());
    for (int k = 0; k < nb; ++k) {
        const W bv = Bv[r][k];
#pragma unroll
        for (int q = 0; q < Q; ++q) wfma(acc[q], bv, Iv[k][g + 4 * q]);
    }
    if (r0 + r < nrows) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int c = g + 4 * q;
            if (c < nb) B[(long)c * ldb + r0 + r] = narrow(acc[q], T());
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

    const typename Wide<T>::type* inv = nullptr;  // FP64 inverses of M's diagonal blocks

    // Solve the diagonal range [o, o+sz) of M against the matching part of B.
    cudaError_t solve(int o, int sz, T scale)
    {
        if (sz <= LEAF) {
            using W = typename Wide<T>::type;
            const W* ib = inv + (long)(o / LEAF) * LEAF * LEAF;
            if (left) {
                const size_t sm = sizeof(W) * (LEAF * (LEAF + 1) + LEAF * 65);
                trsm_apply_left_kernel<T, LEAF><<<ceil_div(nrhs, 64), 256, sm, h->stream>>>(sz, nrhs, ib, B + o, ldb);
            } else {
                const size_t sm = sizeof(W) * (LEAF * (LEAF + 1) + 64 * (LEAF + 1));
                trsm_apply_right_kernel<T, LEAF><<<ceil_div(nrhs, 64), 256, sm, h->stream>>>(
                    sz, nrhs, ib, B + (long)o * ldb, ldb);
            }
            (void)scale;
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
    // FP64 inverses of all diagonal blocks of op(A), one launch
    using W = typename Wide<T>::type;
    constexpr int NB = Solver<T>::LEAF;
    const int na = s.left ? m : n;
    const int nblk = ceil_div(na, NB);
    W* inv = (W*)solver_scratch(h, sizeof(W) * (size_t)nblk * NB * NB);
    if (!inv) return cudaErrorMemoryAllocation;
    const size_t sm_inv = sizeof(W) * 2 * NB * (NB + 1);
    cudaError_t e = cudaFuncSetAttribute(trsm_inv_diag_kernel<T, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sm_inv);
    if (e != cudaSuccess) return e;
    const size_t sm_app = sizeof(W) * (NB * (NB + 1) + NB * 65);
    const size_t sm_app_r = sizeof(W) * (NB * (NB + 1) + 64 * (NB + 1));
    if ((e = cudaFuncSetAttribute(trsm_apply_left_kernel<T, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm_app)) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(trsm_apply_right_kernel<T, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm_app_r)) != cudaSuccess)
        return e;
    trsm_inv_diag_kernel<T, NB><<<nblk, NB, sm_inv, h->stream>>>(na, s.op, s.m_lower, s.unit, A, lda, inv);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    s.inv = inv;
    e = s.solve(0, na, Gemm<T>::one());
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
