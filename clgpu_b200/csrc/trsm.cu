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
// known-answer checks after cancellation.  Leaves are 512 rows (256 complex):
// their inverses are formed on the GPU in FP64 (64 x 64 diagonal blocks by
// substitution, then doubling steps up to the leaf size), rounded to the
// working type, and applied as GEMMs.  Every GEMM uses the handle's math mode
// (the plain FP32 default is the CUDA-core kernel).
#include <algorithm>
#include <type_traits>

#include "common.cuh"

namespace iclb {

cudaError_t sgemm_simt(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const float* A, int lda,
                       const float* B, int ldb, float beta, float* C, int ldc, int tri);
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
__device__ __forceinline__ float one_v(float) { return 1.f; }
__device__ __forceinline__ cfloat one_v(cfloat) { return cfloat{1.f, 0.f}; }
__device__ __forceinline__ float addv(float a, float b) { return a + b; }
__device__ __forceinline__ cfloat addv(cfloat a, cfloat b) { return cfloat{a.re + b.re, a.im + b.im}; }
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
__device__ __forceinline__ void wneg(double& a) { a = -a; }
__device__ __forceinline__ void wneg(double2& a) { a.x = -a.x; a.y = -a.y; }
__device__ __forceinline__ double wdiv(double a, double d) { return a / d; }
__device__ __forceinline__ double2 wdiv(double2 a, double2 d)
{
    const double q = d.x * d.x + d.y * d.y;
    return make_double2((a.x * d.x + a.y * d.y) / q, (a.y * d.x - a.x * d.y) / q);
}

// Inverse in FP64 of every NB x NB diagonal block of M = op(A) over the
// padded range [0, nbig*BIG): M(i,j) = A[i + j*lda] (op 0) or A[j + i*lda]
// (op 1; op 2 conjugates); rows and columns at or beyond n are the identity.
// Block b is written into its big block's column-major BIG x BIG inverse
// (inv + (b*NB / BIG) * BIG*BIG, at local offset (b*NB) % BIG).  Thread j
// forms column j of the inverse by substitution on e_j.
template <class T, int NB>
__global__ void __launch_bounds__(NB) trsm_inv_diag_kernel(int n, int op, int m_lower, int unit, int big,
                                                           const T* __restrict__ A, long lda,
                                                           typename Wide<T>::type* __restrict__ inv)
{
    using W = typename Wide<T>::type;
    extern __shared__ uint8_t smem_raw[];
    W(*M)[NB + 1] = (W(*)[NB + 1])smem_raw;
    W(*Y)[NB + 1] = M + NB;
    const int b = blockIdx.x, o = b * NB, nb = max(0, min(NB, n - o));
    for (int idx = threadIdx.x; idx < NB * NB; idx += NB) {
        const int r = idx % NB, c = idx / NB;  // A-local (r, c): coalesced down A's columns
        W v = (r == c && r >= nb) ? wone(W()) : wz(W());
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
    const bool unit_j = unit || j >= nb;  // padding rows have a unit diagonal
    if (m_lower) {
        for (int i = 0; i < NB; ++i) {
            W y = wz(W());
            if (i >= j) {
                y = (i == j) ? wone(W()) : wz(W());
                for (int k = j; k < i; ++k) wfms(y, M[i][k], Y[k][j]);
                if (!(unit || i >= nb)) y = wdiv(y, M[i][i]);
            }
            Y[i][j] = y;
        }
    } else {
        for (int i = NB - 1; i >= 0; --i) {
            W y = wz(W());
            if (i <= j) {
                y = (i == j) ? wone(W()) : wz(W());
                for (int k = i + 1; k <= j; ++k) wfms(y, M[i][k], Y[k][j]);
                if (!(unit || i >= nb)) y = wdiv(y, M[i][i]);
            }
            Y[i][j] = y;
        }
    }
    (void)unit_j;
    __syncthreads();
    const int bb = o / big, lo = o % big;
    W* out = inv + (long)bb * big * big + (long)lo * big + lo;
    for (int idx = threadIdx.x; idx < NB * NB; idx += NB) out[(long)(idx / NB) * big + idx % NB] = Y[idx % NB][idx / NB];
}

// The same inverses for real 64 x 64 blocks on 256 threads: the four 16 x 16
// diagonal blocks by substitution (one column per thread, the column in
// registers), then two doubling steps (16 -> 32 -> 64) forming each
// off-diagonal block from products of known inverses.  Padding rows and
// columns (at or beyond n) are an identity, as above.  One column per
// thread over all 64 rows (trsm_inv_diag_kernel) is a 64-step dependent
// chain per thread.
__global__ void __launch_bounds__(256) trsm_inv_diag64_kernel(int n, int op, int m_lower, int unit, int big,
                                                               const float* __restrict__ A, long lda,
                                                               double* __restrict__ inv)
{
    constexpr int NB = 64;
    extern __shared__ uint8_t smem_raw[];
    double(*M)[NB + 1] = (double(*)[NB + 1])smem_raw;       // the block of op(A), padded
    double(*R)[NB + 1] = M + NB;                              // its inverse
    double(*Tm)[NB / 2 + 1] = (double(*)[NB / 2 + 1])(R + NB);  // doubling temporary
    double* rd = &Tm[0][0] + (NB / 2) * (NB / 2 + 1);          // 1 / diagonal
    const int t = threadIdx.x, o = blockIdx.x * NB, nb = max(0, min(NB, n - o));
    for (int idx = t; idx < NB * NB; idx += 256) {
        const int r = idx % NB, c = idx / NB;  // A-local (r, c): coalesced down A's columns
        double v = (r == c && r >= nb) ? 1.0 : 0.0;
        if (r < nb && c < nb) v = (double)A[(long)(o + c) * lda + (o + r)];
        if (op == 0) M[r][c] = v;
        else M[c][r] = v;
        R[r][c] = 0.0;
    }
    __syncthreads();
    if (t < NB) rd[t] = unit ? 1.0 : 1.0 / M[t][t];
    __syncthreads();
    if (t < NB) {
        const int b = (t / 16) * 16, j = t % 16;
        double y[16];
        if (m_lower) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                double acc = (i == j) ? 1.0 : 0.0;
#pragma unroll
                for (int k = 0; k < i; ++k) acc = fma(-M[b + i][b + k], y[k], acc);
                y[i] = (i >= j) ? acc * rd[b + i] : 0.0;
            }
        } else {
#pragma unroll
            for (int i = 15; i >= 0; --i) {
                double acc = (i == j) ? 1.0 : 0.0;
#pragma unroll
                for (int k = i + 1; k < 16; ++k) acc = fma(-M[b + i][b + k], y[k], acc);
                y[i] = (i <= j) ? acc * rd[b + i] : 0.0;
            }
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) R[b + i][b + j] = y[i];
    }
    __syncthreads();
    // lower M = [[P, 0], [C, Q]]: off-diagonal inverse block -Q^-1 C P^-1;
    // upper M = [[P, C], [0, Q]]: -P^-1 C Q^-1
    auto doubling = [&](auto hc) {
        constexpr int h = decltype(hc)::value;
        constexpr int nout = (NB / (2 * h)) * h * h;
        for (int idx = t; idx < nout; idx += 256) {
            const int pr = idx / (h * h), e = idx % (h * h), r = e % h, c = e / h, q = pr * 2 * h;
            double a0 = 0.0, a1 = 0.0;
#pragma unroll
            for (int k = 0; k < h; k += 2) {
                if (m_lower) {
                    a0 = fma(M[q + h + r][q + k], R[q + k][q + c], a0);
                    a1 = fma(M[q + h + r][q + k + 1], R[q + k + 1][q + c], a1);
                } else {
                    a0 = fma(M[q + r][q + h + k], R[q + h + k][q + h + c], a0);
                    a1 = fma(M[q + r][q + h + k + 1], R[q + h + k + 1][q + h + c], a1);
                }
            }
            Tm[pr * h + r][c] = a0 + a1;
        }
        __syncthreads();
        for (int idx = t; idx < nout; idx += 256) {
            const int pr = idx / (h * h), e = idx % (h * h), r = e % h, c = e / h, q = pr * 2 * h;
            double a0 = 0.0, a1 = 0.0;
#pragma unroll
            for (int k = 0; k < h; k += 2) {
                if (m_lower) {
                    a0 = fma(R[q + h + r][q + h + k], Tm[pr * h + k][c], a0);
                    a1 = fma(R[q + h + r][q + h + k + 1], Tm[pr * h + k + 1][c], a1);
                } else {
                    a0 = fma(R[q + r][q + k], Tm[pr * h + k][c], a0);
                    a1 = fma(R[q + r][q + k + 1], Tm[pr * h + k + 1][c], a1);
                }
            }
            if (m_lower) R[q + h + r][q + c] = -(a0 + a1);
            else R[q + r][q + h + c] = -(a0 + a1);
        }
        __syncthreads();
    };
    doubling(std::integral_constant<int, 16>{});
    doubling(std::integral_constant<int, 32>{});
    const int bb = o / big, lo = o % big;
    double* out = inv + (long)bb * big * big + (long)lo * big + lo;
    for (int idx = t; idx < NB * NB; idx += 256) out[(long)(idx / NB) * big + idx % NB] = R[idx % NB][idx / NB];
}
constexpr size_t kInvDiag64Smem = sizeof(double) * (2 * 64 * 65 + 32 * 33 + 64);

// One doubling step of the block inverses: for every 2s x 2s diagonal block
// (offset o in big block bb) whose two s x s diagonal inverses are known,
//   lower M = [[P, 0], [C, Q]]:  inv = [[P^-1, 0], [-Q^-1 C P^-1, Q^-1]]
//   upper M = [[P, C], [0, Q]]:  inv = [[P^-1, -P^-1 C Q^-1], [0, Q^-1]]
// STEP 0 forms T = C * P^-1 (lower) or T = C * Q^-1 (upper) with C read from
// A through op; STEP 1 forms the off-diagonal block -Q^-1 T (lower) or
// -P^-1 T (upper) into the inverse.  FP64, TS x TS tiles, 256 threads, each
// thread (TS/16) x (TS/16) outputs; blockIdx.z enumerates the 2s blocks.
template <class T, int TS, int STEP>
__global__ void __launch_bounds__(256) trsm_inv_double_kernel(int n, int op, int m_lower, int s, int big,
                                                              const T* __restrict__ A, long lda,
                                                              typename Wide<T>::type* __restrict__ inv,
                                                              typename Wide<T>::type* __restrict__ tmp)
{
    using W = typename Wide<T>::type;
    constexpr int KC = 16;
    constexpr int PT = TS / 16;  // outputs per thread per dimension
    __shared__ W Xs[TS][KC + 1];
    __shared__ W Ys[KC][TS + 1];
    const int pairs = big / (2 * s);
    const int z = blockIdx.z, bb = z / pairs, o = (z % pairs) * 2 * s;
    const int gbase = bb * big;  // global row/col of the big block
    W* invb = inv + (long)bb * big * big;
    W* tz = tmp + (long)z * s * s;
    const int i0 = blockIdx.y * TS, j0 = blockIdx.x * TS;  // output tile (rows, cols) in s x s
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    // X (s x s) and Y (s x s) sources; output location
    //  STEP 0 lower: X = C = M[o+s.., o..],  Y = P^-1 = inv[o.., o..],     out = tmp
    //  STEP 0 upper: X = C = M[o.., o+s..],  Y = Q^-1 = inv[o+s.., o+s..], out = tmp
    //  STEP 1 lower: X = Q^-1 = inv[o+s.., o+s..], Y = tmp, out = inv[o+s.., o..] (negated)
    //  STEP 1 upper: X = P^-1 = inv[o.., o..],     Y = tmp, out = inv[o.., o+s..] (negated)
    const int xr = (STEP == 0) ? (m_lower ? o + s : o) : (m_lower ? o + s : o);
    const int xc = (STEP == 0) ? (m_lower ? o : o + s) : (m_lower ? o + s : o);
    const int yo = m_lower ? o : o + s;  // STEP 0 diagonal inverse offset
    W acc[PT][PT];
#pragma unroll
    for (int a = 0; a < PT; ++a)
#pragma unroll
        for (int c = 0; c < PT; ++c) acc[a][c] = wz(W());
    // K slices of KC, the next slice's operands prefetched into registers
    constexpr int XPT = TS * KC / 256, YPT = KC * TS / 256;
    W rx[XPT], ry[YPT];
    auto load = [&](int k0) {
#pragma unroll
        for (int u = 0; u < XPT; ++u) {
            const int idx = threadIdx.x + 256 * u, r = idx % TS, k = idx / TS;
            W v;
            if (STEP == 0) {
                const int gi = gbase + xr + i0 + r, gj = gbase + xc + k0 + k;  // M(gi, gj)
                v = wz(W());
                if (gi < n && gj < n) {
                    T a = (op == 0) ? A[(long)gj * lda + gi] : A[(long)gi * lda + gj];
                    if (op == 2) a = conj_v(a);
                    v = widen(a);
                }
            } else {
                v = invb[(long)(xc + k0 + k) * big + xr + i0 + r];
            }
            rx[u] = v;
        }
#pragma unroll
        for (int u = 0; u < YPT; ++u) {
            const int idx = threadIdx.x + 256 * u, k = idx % KC, c = idx / KC;
            ry[u] = (STEP == 0) ? invb[(long)(yo + j0 + c) * big + yo + k0 + k] : tz[(long)(j0 + c) * s + k0 + k];
        }
    };
    auto store = [&]() {
#pragma unroll
        for (int u = 0; u < XPT; ++u) {
            const int idx = threadIdx.x + 256 * u;
            Xs[idx % TS][idx / TS] = rx[u];
        }
#pragma unroll
        for (int u = 0; u < YPT; ++u) {
            const int idx = threadIdx.x + 256 * u;
            Ys[idx % KC][idx / KC] = ry[u];
        }
    };
    load(0);
    for (int k0 = 0; k0 < s; k0 += KC) {
        __syncthreads();
        store();
        __syncthreads();
        if (k0 + KC < s) load(k0 + KC);
#pragma unroll
        for (int k = 0; k < KC; ++k) {
            W xv[PT], yv[PT];
#pragma unroll
            for (int a = 0; a < PT; ++a) xv[a] = Xs[ty + 16 * a][k];
#pragma unroll
            for (int c = 0; c < PT; ++c) yv[c] = Ys[k][tx + 16 * c];
#pragma unroll
            for (int a = 0; a < PT; ++a)
#pragma unroll
                for (int c = 0; c < PT; ++c) wfma(acc[a][c], xv[a], yv[c]);
        }
    }
#pragma unroll
    for (int a = 0; a < PT; ++a)
#pragma unroll
        for (int c = 0; c < PT; ++c) {
            const int i = i0 + ty + 16 * a, j = j0 + tx + 16 * c;
            if (STEP == 0) {
                tz[(long)j * s + i] = acc[a][c];
            } else {
                W v = acc[a][c];
                wneg(v);
                const int orow = m_lower ? o + s : o, ocol = m_lower ? o : o + s;
                invb[(long)(ocol + j) * big + orow + i] = v;
            }
        }
}

// FP64 inverse blocks rounded to the working precision (for the GEMM apply).
template <class T>
__global__ void narrow_kernel(long count, const typename Wide<T>::type* __restrict__ src, T* __restrict__ dst)
{
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < count; e += (long)gridDim.x * blockDim.x)
        dst[e] = narrow(src[e], T());
}

// Copy of every leaf's diagonal block of M = op(A) (op 2 conjugates) with
// the other triangle zeroed (and the diagonal 1 for a unit diagonal), leaf
// bb at out + bb*big*big, column-major with leading dimension big; rows and
// columns at or beyond n are zero.  Used for the refinement residual.
template <class T>
__global__ void leaf_tri_kernel(int n, int op, int m_lower, int unit, int big, int nbig, const T* __restrict__ A,
                                long lda, T* __restrict__ out)
{
    const long per = (long)big * big, total = per * nbig;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long bb = e / per, rem = e % per;
        const int c = (int)(rem / big), r = (int)(rem % big);
        const long i = bb * big + r, j = bb * big + c;
        T v = zero_v(T());
        if (i < n && j < n && (r == c || (m_lower ? r > c : r < c))) {
            if (r == c && unit) v = one_v(T());
            else if (op == 0) v = A[i + j * lda];
            else {
                v = A[j + i * lda];
                if (op == 2) v = conj_v(v);
            }
        }
        out[e] = v;
    }
}

// X = alpha * (X + D) for m x n column-major blocks.
template <class T>
__global__ void add_scale_kernel(int m, int n, T alpha, T* __restrict__ X, long ldx, const T* __restrict__ D,
                                 long ldd)
{
    const long total = (long)m * n;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long j = e / m, i = e % m;
        T* p = X + j * ldx + i;
        *p = mulv(addv(*p, D[j * ldd + i]), alpha);
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
    static float zero() { return 0.f; }
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
    static cfloat zero() { return cfloat{0.f, 0.f}; }
    static cfloat minus_one() { return cfloat{-1.f, 0.f}; }
};

template <class T>
struct Solver {
    static constexpr int NB = Leaf<T>::value;  // base inverse block
    iclblasHandle_t h;
    int left, op, unit, m_lower;
    const T* A;
    long lda;
    T* B;
    long ldb;
    int nrhs;  // RHS count (n for left, m for right)
    int big;   // leaf size (a power-of-two multiple of NB)
    const T* inv = nullptr;  // inverses of the BIG diagonal blocks (FP64-formed, rounded)
    T* tmp = nullptr;        // leaf staging: big x nrhs (left) or nrhs x big (right)
    const T* mtri = nullptr; // masked leaf diagonal blocks (refinement only)

    // Pointer and GEMM op of block M[r0.., c0..] of M = op(A).
    const T* mblk(int r0, int c0) const { return op == 0 ? A + r0 + (long)c0 * lda : A + c0 + (long)r0 * lda; }

    // Solve the diagonal range [o, o+sz) of M against the matching part of B.
    cudaError_t solve(int o, int sz)
    {
        if (sz <= big) {
            // leaf: X = inv(M_oo) * B_o (left) or B_o * inv(M_oo) (right), by GEMM
            const T* ib = inv + (long)(o / big) * big * big;
            cudaError_t e;
            if (left) {
                e = cudaMemcpy2DAsync(tmp, sizeof(T) * sz, B + o, sizeof(T) * ldb, sizeof(T) * sz, nrhs,
                                      cudaMemcpyDeviceToDevice, h->stream);
                if (e != cudaSuccess) return e;
                return Gemm<T>::run(h, ICLBLAS_OP_N, ICLBLAS_OP_N, sz, nrhs, sz, Gemm<T>::one(), ib, big, tmp, sz,
                                    Gemm<T>::zero(), B + o, ldb);
            }
            e = cudaMemcpy2DAsync(tmp, sizeof(T) * nrhs, B + (long)o * ldb, sizeof(T) * ldb, sizeof(T) * nrhs, sz,
                                  cudaMemcpyDeviceToDevice, h->stream);
            if (e != cudaSuccess) return e;
            return Gemm<T>::run(h, ICLBLAS_OP_N, ICLBLAS_OP_N, nrhs, sz, sz, Gemm<T>::one(), tmp, nrhs, ib, big,
                                Gemm<T>::zero(), B + (long)o * ldb, ldb);
        }
        const int nleaf = (sz + big - 1) / big;
        const int h1 = (nleaf / 2) * big;  // first half: a whole number of leaves
        const int o1 = o, s1 = h1, o2 = o + h1, s2 = sz - h1;
        // Forward (first half first) when: left & M lower, or right & M upper.
        const bool forward = left ? m_lower : !m_lower;
        const int fo = forward ? o1 : o2, fs = forward ? s1 : s2;  // solved first
        const int so = forward ? o2 : o1, ss = forward ? s2 : s1;  // updated, solved second
        cudaError_t e = solve(fo, fs);
        if (e != cudaSuccess) return e;
        if (left) {
            // B[so] = B[so] - M[so, fo] * X[fo]
            e = Gemm<T>::run(h, op, ICLBLAS_OP_N, ss, nrhs, fs, Gemm<T>::minus_one(), mblk(so, fo), lda, B + fo, ldb,
                             Gemm<T>::one(), B + so, ldb);
        } else {
            // B[:, so] = B[:, so] - X[:, fo] * M[fo, so]
            e = Gemm<T>::run(h, ICLBLAS_OP_N, op, nrhs, ss, fs, Gemm<T>::minus_one(), B + (long)fo * ldb, ldb,
                             mblk(fo, so), lda, Gemm<T>::one(), B + (long)so * ldb, ldb);
        }
        if (e != cudaSuccess) return e;
        return solve(so, ss);
    }

    // R -= M X over the diagonal range [o, o+sz) (left: rows of R and X;
    // right: columns), with the same recursive split as solve(): leaves use
    // the masked diagonal blocks, the off-diagonal blocks are GEMMs on A.
    cudaError_t residual(int o, int sz, const T* X, long ldx, T* R, long ldr)
    {
        if (sz <= big) {
            const T* mt = mtri + (long)(o / big) * big * big;
            if (left)
                return Gemm<T>::run(h, ICLBLAS_OP_N, ICLBLAS_OP_N, sz, nrhs, sz, Gemm<T>::minus_one(), mt, big, X + o,
                                    (int)ldx, Gemm<T>::one(), R + o, (int)ldr);
            return Gemm<T>::run(h, ICLBLAS_OP_N, ICLBLAS_OP_N, nrhs, sz, sz, Gemm<T>::minus_one(), X + (long)o * ldx,
                                (int)ldx, mt, big, Gemm<T>::one(), R + (long)o * ldr, (int)ldr);
        }
        const int nleaf = (sz + big - 1) / big;
        const int h1 = (nleaf / 2) * big;
        const int o1 = o, s1 = h1, o2 = o + h1, s2 = sz - h1;
        const bool forward = left ? m_lower : !m_lower;
        const int fo = forward ? o1 : o2, fs = forward ? s1 : s2;
        const int so = forward ? o2 : o1, ss = forward ? s2 : s1;
        cudaError_t e = residual(fo, fs, X, ldx, R, ldr);
        if (e == cudaSuccess) e = residual(so, ss, X, ldx, R, ldr);
        if (e != cudaSuccess) return e;
        if (left)
            return Gemm<T>::run(h, op, ICLBLAS_OP_N, ss, nrhs, fs, Gemm<T>::minus_one(), mblk(so, fo), lda, X + fo,
                                (int)ldx, Gemm<T>::one(), R + so, (int)ldr);
        return Gemm<T>::run(h, ICLBLAS_OP_N, op, nrhs, ss, fs, Gemm<T>::minus_one(), X + (long)fo * ldx, (int)ldx,
                            mblk(fo, so), lda, Gemm<T>::one(), R + (long)so * ldr, (int)ldr);
    }
};

// The tensor-core modes on real operands: the solve's GEMMs read operands
// split into BF16 / TF32 planes once per call instead of splitting both
// operands inside every GEMM.  Planes (K-major rows):
//   pa    M = op(A) (left) or M^T (right), masked to its triangle, na x na;
//         split once per call (blocks outside the triangle are never read)
//   pinv  the leaves' FP64-formed inverses rounded to FP32: leaf bb's rows
//         at bb*big (left: rows of inv; right: rows of inv^T); once per call
//   px    the solved blocks of X as the update GEMMs read them (left: row j
//         = right-hand side j, K = row of X; right: row i = row of X, K =
//         column of X); each leaf writes its block once, after its solve
//   pb    one leaf block of the updated B, split just before its leaf GEMM
// Left:  update B[so] -= M[so, fo] X[fo]:    pa rows so, K fo  x  px K fo
//        leaf   X_o = inv_o B_o:              pinv rows o       x  pb
// Right: update B[:, so] -= X[:, fo] M[fo, so]:  px K fo  x  pa rows so, K fo
//        leaf   X_o = B_o inv_o:              pb  x  pinv rows o
struct PlaneSolver {
    iclblasHandle_t h;
    int left, m_lower, nrhs, big;
    float* B;
    long ldb;
    GemmPlanes pa, pinv, px, pb;

    // Leaf block [o, o + sz) of B (left: rows, right: columns) into planes
    // `dst` at K offset k0 (left: L[j][k] = B[o + k, j]; right: L[i][k] =
    // B[i, o + k]).  An odd size writes one zero past the block.
    cudaError_t split_block(const GemmPlanes& dst, long k0, int o, int sz) const
    {
        const long kw = (sz + 1) & ~1;
        if (left) return split_planes(h, B + o, nrhs, sz, ldb, 1, dst, 0, k0, kw);
        return split_planes(h, B + (long)o * ldb, nrhs, sz, 1, ldb, dst, 0, k0, kw);
    }

    cudaError_t solve(int o, int sz) const
    {
        if (sz <= big) {
            const long r0 = (long)(o / big) * big;
            cudaError_t e = split_block(pb, 0, o, sz);
            if (e != cudaSuccess) return e;
            if (left) e = gemm_planes(h, pinv, r0, 0, pb, 0, 0, sz, nrhs, sz, 1.f, 0.f, B + o, (int)ldb);
            else e = gemm_planes(h, pb, 0, 0, pinv, r0, 0, nrhs, sz, sz, 1.f, 0.f, B + (long)o * ldb, (int)ldb);
            if (e != cudaSuccess) return e;
            return split_block(px, o, o, sz);
        }
        const int nleaf = (sz + big - 1) / big;
        const int h1 = (nleaf / 2) * big;
        const int o1 = o, s1 = h1, o2 = o + h1, s2 = sz - h1;
        const bool forward = left ? m_lower : !m_lower;
        const int fo = forward ? o1 : o2, fs = forward ? s1 : s2;
        const int so = forward ? o2 : o1, ss = forward ? s2 : s1;
        cudaError_t e = solve(fo, fs);
        if (e != cudaSuccess) return e;
        if (left) e = gemm_planes(h, pa, so, fo, px, 0, fo, ss, nrhs, fs, -1.f, 1.f, B + so, (int)ldb);
        else e = gemm_planes(h, px, 0, fo, pa, so, fo, nrhs, ss, fs, -1.f, 1.f, B + (long)so * ldb, (int)ldb);
        if (e != cudaSuccess) return e;
        return solve(so, ss);
    }

    // The right-hand sides are independent: with enough of them, the second
    // half (rows of px / pb and columns (left) or rows (right) of B from
    // `cut` on) is solved on the handle's second stream while the first
    // half runs, so the latencies of the small leaf steps of one half
    // overlap the other half's work.
    cudaError_t solve_split(int o, int sz) const
    {
        const int cut = nrhs >= 1024 ? (nrhs / 2) / 64 * 64 : 0;
        if (cut == 0) return solve(o, sz);
        PlaneSolver lo = *this, hi = *this;
        lo.nrhs = cut;
        hi.nrhs = nrhs - cut;
        hi.B = B + (left ? (long)cut * ldb : (long)cut);
        for (GemmPlanes* g : {&hi.px, &hi.pb}) {
            const long esize = g->tf32 ? 4 : 2;
            for (int l = 0; l < g->nlev; ++l) g->plane[l] = (char*)g->plane[l] + (long)cut * g->pitch * esize;
            g->rows -= cut;
        }
        lo.px.rows = lo.pb.rows = cut;
        cudaStream_t side = nullptr;
        cudaError_t e = fork_side(h, &side);
        if (e != cudaSuccess) return e;
        {
            StreamScope on_side(h, side);
            if ((e = hi.solve(o, sz)) != cudaSuccess) return e;
        }
        if ((e = lo.solve(o, sz)) != cudaSuccess) return e;
        return join_side(h);
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
    using W = typename Wide<T>::type;
    constexpr int NB = Solver<T>::NB;
    constexpr int BIG_MAX = sizeof(T) == sizeof(float) ? 512 : 256;
    const int na = s.left ? m : n;
    int big = NB;
    while (big < BIG_MAX && big < na) big *= 2;
    s.big = big;
    const int nbig = ceil_div(na, big);
    const int nsmall = nbig * (big / NB);
    // workspace: FP64 inverses, doubling temporaries, rounded inverses, leaf staging
    const size_t inv_w = (size_t)nbig * big * big;
    const size_t tmp_w = (size_t)nbig * (big / 2) * (big / 2);
    const size_t leaf_t = (size_t)big * s.nrhs;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    // refinement: masked leaf blocks, a copy of B, the residual / correction
    const int steps = h->trsm_refine;
    const size_t mn = (size_t)m * n;
    // tensor-core modes on real data: operand planes split once per call
    const bool planes = std::is_same<T, float>::value && h->math != ICLBLAS_MATH_PLAIN_FP32;
    const int nlev = planes ? plane_levels(h->math) : 0;
    const long esize = planes ? plane_esize(h->math) : 0;
    const long pitch_m = ((long)na + 63) / 64 * 64;
    const size_t pa_b = al((size_t)na * pitch_m * esize), pinv_b = al((size_t)nbig * big * big * esize);
    const size_t px_b = al((size_t)s.nrhs * pitch_m * esize), pb_b = al((size_t)s.nrhs * big * esize);
    const size_t plane_bytes = planes ? nlev * (pa_b + pinv_b + px_b + pb_b) : 0;
    const size_t bytes = al(sizeof(W) * inv_w) + al(sizeof(W) * tmp_w) + al(sizeof(T) * inv_w) +
                         al(sizeof(T) * leaf_t) +
                         (steps > 0 ? al(sizeof(T) * inv_w) + 2 * al(sizeof(T) * mn) : 0) + plane_bytes;
    char* ws = (char*)solver_scratch(h, bytes);
    if (!ws) return cudaErrorMemoryAllocation;
    W* invd = (W*)ws;
    W* dtmp = (W*)(ws + al(sizeof(W) * inv_w));
    T* inv32 = (T*)(ws + al(sizeof(W) * inv_w) + al(sizeof(W) * tmp_w));
    s.tmp = (T*)(ws + al(sizeof(W) * inv_w) + al(sizeof(W) * tmp_w) + al(sizeof(T) * inv_w));
    // the refinement regions exist only when steps > 0; the planes follow
    // whatever was allocated before them
    char* tail = (char*)s.tmp + al(sizeof(T) * leaf_t);
    T *mtri = nullptr, *b0 = nullptr, *res = nullptr;
    if (steps > 0) {
        mtri = (T*)tail;
        tail += al(sizeof(T) * inv_w);
        b0 = (T*)tail;
        tail += al(sizeof(T) * mn);
        res = (T*)tail;
        tail += al(sizeof(T) * mn);
    }
    char* pl = tail;
    PlaneSolver ps{};
    if (planes) {
        ps.h = h;
        ps.left = s.left;
        ps.m_lower = s.m_lower;
        ps.nrhs = s.nrhs;
        ps.big = big;
        ps.B = (float*)B;
        ps.ldb = ldb;
        GemmPlanes* sets[4] = {&ps.pa, &ps.pinv, &ps.px, &ps.pb};
        const size_t sizes[4] = {pa_b, pinv_b, px_b, pb_b};
        const long pitches[4] = {pitch_m, big, pitch_m, big};
        const long rows[4] = {na, (long)nbig * big, s.nrhs, s.nrhs};
        for (int q = 0; q < 4; ++q) {
            sets[q]->rows = rows[q];
            sets[q]->nlev = nlev;
            sets[q]->tf32 = h->math == ICLBLAS_MATH_TF32 ? 1 : 0;
            sets[q]->pitch = pitches[q];
            for (int l = 0; l < nlev; ++l) {
                sets[q]->plane[l] = pl;
                pl += sizes[q];
            }
        }
    }
    // FP64 inverses of the leaves' diagonal blocks, rounded to the working
    // type (and, on the plane path, split into the inverse planes)
    auto form_inverses = [&]() -> cudaError_t {
        cudaError_t e = cudaMemsetAsync(invd, 0, sizeof(W) * inv_w, h->stream);
        if (e != cudaSuccess) return e;
        if constexpr (std::is_same<T, float>::value) {
            if ((e = cudaFuncSetAttribute(trsm_inv_diag64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kInvDiag64Smem)) != cudaSuccess)
                return e;
            trsm_inv_diag64_kernel<<<nsmall, 256, kInvDiag64Smem, h->stream>>>(na, s.op, s.m_lower, s.unit, big, A,
                                                                              lda, (double*)invd);
        } else {
            const size_t sm_inv = sizeof(W) * 2 * NB * (NB + 1);
            if ((e = cudaFuncSetAttribute(trsm_inv_diag_kernel<T, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)sm_inv)) != cudaSuccess)
                return e;
            trsm_inv_diag_kernel<T, NB><<<nsmall, NB, sm_inv, h->stream>>>(na, s.op, s.m_lower, s.unit, big, A,
                                                                            lda, invd);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        constexpr int TS = NB;  // doubling tile: 64 real, 32 complex
        for (int sz = NB; sz < big; sz *= 2) {
            dim3 grid(sz / TS, sz / TS, nbig * (big / (2 * sz)));
            trsm_inv_double_kernel<T, TS, 0><<<grid, 256, 0, h->stream>>>(na, s.op, s.m_lower, sz, big, A, lda, invd,
                                                                           dtmp);
            trsm_inv_double_kernel<T, TS, 1><<<grid, 256, 0, h->stream>>>(na, s.op, s.m_lower, sz, big, A, lda, invd,
                                                                           dtmp);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        const long cnt = (long)inv_w;
        const int g = (int)std::min<long>((cnt + 255) / 256, (long)h->sm_count * 8);
        narrow_kernel<T><<<g, 256, 0, h->stream>>>(cnt, invd, inv32);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (!planes) return cudaSuccess;
        // left: rows of inv; right: rows of inv^T
        return split_planes(h, (const float*)inv32, big, big, s.left ? 1 : big, s.left ? big : 1, ps.pinv, 0, 0, big,
                            0, 0, nbig, (long)big * big, big);
    };
    cudaError_t e;
    if (planes) {
        // the inverses (compute-bound, FP64) form on the second stream while
        // the triangle M (left) or M^T (right), masked, is split (HBM-bound)
        cudaStream_t side = nullptr;
        if ((e = fork_side(h, &side)) != cudaSuccess) return e;
        {
            StreamScope on_side(h, side);
            if ((e = form_inverses()) != cudaSuccess) return e;
        }
        const bool ml = s.m_lower != 0;
        const int tri = s.left ? (ml ? 1 : 2) : (ml ? 2 : 1);
        const bool rows_contig = s.left ? s.op == ICLBLAS_OP_N : s.op != ICLBLAS_OP_N;
        e = split_planes(h, (const float*)A, na, na, rows_contig ? 1 : lda, rows_contig ? lda : 1, ps.pa, 0, 0,
                         (na + 1) & ~1, tri, s.unit);
        if (e == cudaSuccess) e = join_side(h);
        if (e != cudaSuccess) return e;
    } else if ((e = form_inverses()) != cudaSuccess) {
        return e;
    }
    s.inv = inv32;
    if (steps > 0) {
        e = cudaMemcpy2DAsync(b0, sizeof(T) * m, B, sizeof(T) * ldb, sizeof(T) * m, n, cudaMemcpyDeviceToDevice,
                              h->stream);
        if (e != cudaSuccess) return e;
        const long cnt = (long)inv_w;
        const int g = (int)std::min<long>((cnt + 255) / 256, (long)h->sm_count * 8);
        leaf_tri_kernel<T><<<g, 256, 0, h->stream>>>(na, s.op, s.m_lower, s.unit, big, nbig, A, lda, mtri);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        s.mtri = mtri;
    }
    e = planes ? ps.solve_split(0, na) : s.solve(0, na);
    if (e != cudaSuccess) return e;
    for (int it = 0; it < steps; ++it) {
        // R = B0 - M X with FP32-accurate products (6xBF16 on the tensor cores,
        // or the CUDA-core kernel in PLAIN_FP32 mode), then M D = R in the
        // handle's mode with the same inverses, X = X + D (alpha on the last)
        e = cudaMemcpy2DAsync(res, sizeof(T) * m, b0, sizeof(T) * m, sizeof(T) * m, n, cudaMemcpyDeviceToDevice,
                              h->stream);
        if (e != cudaSuccess) return e;
        const iclblasMathMode_t mode = h->math;
        if (mode != ICLBLAS_MATH_PLAIN_FP32) h->math = ICLBLAS_MATH_BF16X6;
        e = s.residual(0, na, B, ldb, res, m);
        h->math = mode;
        if (e != cudaSuccess) return e;
        if (planes) {
            PlaneSolver c = ps;
            c.B = (float*)res;
            c.ldb = m;
            e = c.solve_split(0, na);
        } else {
            Solver<T> c = s;
            c.B = res;
            c.ldb = m;
            e = c.solve(0, na);
        }
        if (e != cudaSuccess) return e;
        const long total = (long)m * n;
        const int grid = (int)std::min<long>((total + 255) / 256, (long)h->sm_count * 8);
        const T sc = it == steps - 1 ? alpha : Gemm<T>::one();
        add_scale_kernel<T><<<grid, 256, 0, h->stream>>>(m, n, sc, B, ldb, res, m);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (steps > 0 || is_one(alpha)) return cudaSuccess;
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
