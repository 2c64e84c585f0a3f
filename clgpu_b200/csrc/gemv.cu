// GEMV: y = alpha*op(A)*x + beta*y for float and complex float.
//
// Replaces the reference's Sgemv_opt_simd16 / Sgemv_opt_simd16_TC /
// Cgemv_naive kernels (libs/blas/funcs/Sgemv/*, Cgemv/*), whose lanes stride
// across columns of a column-major matrix.  Here A is read once, coalesced:
//   op N: each thread owns 16 bytes of consecutive rows (4 floats or 2
//         complex) and walks a slice of columns; slices of columns run in
//         different blocks, their per-row partial sums go to scratch, and the
//         last block of each row tile adds them in slice order (deterministic)
//         and applies alpha/beta;
//   op T/C: one warp per column (a column is contiguous), 128-bit loads down
//         the column, shuffle-tree sum.
// beta == 0 means y is written without being read (Sgemv_naive.cl:34,54).
#include "common.cuh"

namespace iclb {
namespace {

constexpr int kNThreads = 128;  // op N block
constexpr int kTThreads = 256;  // op T block (8 warps = 8 columns)

// ---- element arithmetic
__device__ __forceinline__ float zero_of(float) { return 0.f; }
__device__ __forceinline__ cfloat zero_of(cfloat) { return cfloat{0.f, 0.f}; }

template <bool CONJ>
__device__ __forceinline__ void madd(float& acc, float a, float x) { acc = fmaf(a, x, acc); }
template <bool CONJ>
__device__ __forceinline__ void madd(cfloat& acc, cfloat a, cfloat x)
{
    const float ai = CONJ ? -a.im : a.im;
    acc.re = fmaf(a.re, x.re, acc.re);
    acc.re = fmaf(-ai, x.im, acc.re);
    acc.im = fmaf(a.re, x.im, acc.im);
    acc.im = fmaf(ai, x.re, acc.im);
}
__device__ __forceinline__ float add(float a, float b) { return a + b; }
__device__ __forceinline__ cfloat add(cfloat a, cfloat b) { return cfloat{a.re + b.re, a.im + b.im}; }

// y_out = alpha*s + beta*y (beta == 0: y not read)
__device__ __forceinline__ float axpby(float alpha, float s, float beta, const float* y)
{
    return beta == 0.f ? alpha * s : fmaf(alpha, s, beta * *y);
}
__device__ __forceinline__ cfloat cmulf(cfloat a, cfloat b)
{
    return cfloat{fmaf(a.re, b.re, -a.im * b.im), fmaf(a.re, b.im, a.im * b.re)};
}
__device__ __forceinline__ cfloat axpby(cfloat alpha, cfloat s, cfloat beta, const cfloat* y)
{
    cfloat r = cmulf(alpha, s);
    if (beta.re != 0.f || beta.im != 0.f) r = add(r, cmulf(beta, *y));
    return r;
}

template <class T>
__device__ __forceinline__ T warp_sum_t(T v);
template <>
__device__ __forceinline__ float warp_sum_t<float>(float v) { return warp_sum(v); }
template <>
__device__ __forceinline__ cfloat warp_sum_t<cfloat>(cfloat v)
{
    return cfloat{warp_sum(v.re), warp_sum(v.im)};
}

// ------------------------------------------------------------------ op N
// Block (rt, s): rows [rt*R*128, +R*128), columns [s*cps, min(n, (s+1)*cps)).
// VEC: lda*sizeof(T) and A are 16-byte aligned, so each thread's R rows of a
// column are one 128-bit load.
template <class T, bool VEC>
__global__ void __launch_bounds__(kNThreads) gemv_n_kernel(int m, int n, T alpha, const T* __restrict__ A, long lda,
                                                           const T* __restrict__ x, long incx, T beta,
                                                           T* __restrict__ y, long incy, int cps,
                                                           T* __restrict__ partial, unsigned* counters)
{
    constexpr int R = 16 / sizeof(T);
    constexpr int XC = 256;  // x values staged per chunk
    __shared__ T xs[XC];
    const int splits = gridDim.y;
    const int s = blockIdx.y;
    const long row0 = ((long)blockIdx.x * kNThreads + threadIdx.x) * R;
    const int c0 = s * cps;
    const int c1 = min(n, c0 + cps);

    T acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = zero_of(T());

    for (int cb = c0; cb < c1; cb += XC) {
        const int cn = min(XC, c1 - cb);
        __syncthreads();
        for (int i = threadIdx.x; i < cn; i += kNThreads) xs[i] = x[(long)(cb + i) * incx];
        __syncthreads();
        if (row0 < m) {
            const T* Ac = A + (long)cb * lda + row0;
            if (VEC && row0 + R <= m) {
                int c = 0;
                for (; c + 8 <= cn; c += 8) {
                    float4 v[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) v[u] = ld_stream4((const float4*)(Ac + (long)(c + u) * lda));
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const T* e = (const T*)&v[u];
#pragma unroll
                        for (int r = 0; r < R; ++r) madd<false>(acc[r], e[r], xs[c + u]);
                    }
                }
                for (; c < cn; ++c) {
                    float4 v = ld_stream4((const float4*)(Ac + (long)c * lda));
                    const T* e = (const T*)&v;
#pragma unroll
                    for (int r = 0; r < R; ++r) madd<false>(acc[r], e[r], xs[c]);
                }
            } else {
                for (int c = 0; c < cn; ++c) {
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        if (row0 + r < m) madd<false>(acc[r], Ac[(long)c * lda + r], xs[c]);
                }
            }
        }
    }

    if (splits == 1) {
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (row0 + r < m) {
                T* yp = y + (row0 + r) * incy;
                *yp = axpby(alpha, acc[r], beta, yp);
            }
        return;
    }
    // publish this slice's partial sums; the last slice of the row tile adds them
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (row0 + r < m) partial[(long)s * m + row0 + r] = acc[r];
    if (!last_block_of(counters + blockIdx.x, splits)) return;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const long row = row0 + r;
        if (row >= m) continue;
        T sum = zero_of(T());
        for (int k = 0; k < splits; ++k) sum = add(sum, ((volatile T*)partial)[(long)k * m + row]);
        T* yp = y + row * incy;
        *yp = axpby(alpha, sum, beta, yp);
    }
    if (threadIdx.x == 0) counters[blockIdx.x] = 0u;
}

// ------------------------------------------------------------------ op T / C
// Warp w of the grid handles column col = w / S, row slice w % S of S.
template <class T, bool CONJ, bool VEC>
__global__ void __launch_bounds__(kTThreads) gemv_t_kernel(int m, int n, T alpha, const T* __restrict__ A, long lda,
                                                           const T* __restrict__ x, long incx, T beta,
                                                           T* __restrict__ y, long incy, int S, int rps,
                                                           T* __restrict__ partial, unsigned* counters)
{
    constexpr int R = 16 / sizeof(T);
    const int lane = threadIdx.x & 31;
    const long gw = ((long)blockIdx.x * kTThreads + threadIdx.x) >> 5;
    const long col = gw / S;
    const int s = (int)(gw % S);
    if (col >= n) return;
    const int r0 = s * rps, r1 = min(m, r0 + rps);
    const T* Ac = A + col * lda;
    T acc = zero_of(T());
    if (VEC) {
        // r0 is a multiple of 32*R: every load is one aligned 128-bit vector.
        // Real data: two partial sums (even and odd vectors of the unrolled
        // step) halve the dependent FMA chain and are added in a fixed order
        // after it (complex data keeps one: its four-FMA updates already
        // interleave, and a second sum measured slower).
        T acc2 = zero_of(T());
        int r = r0 + lane * R;
        for (; r + 3 * 32 * R + R <= r1; r += 4 * 32 * R) {
            float4 v[4], xv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                v[u] = ld_stream4((const float4*)(Ac + r + u * 32 * R));
                xv[u] = __ldg((const float4*)(x + r + u * 32 * R));
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const T* e = (const T*)&v[u];
                const T* xe = (const T*)&xv[u];
#pragma unroll
                for (int k = 0; k < R; ++k) madd<CONJ>((sizeof(T) == sizeof(float) && (u & 1)) ? acc2 : acc, e[k], xe[k]);
            }
        }
        acc = add(acc, acc2);
        for (; r + R <= r1; r += 32 * R) {
            float4 v = ld_stream4((const float4*)(Ac + r));
            float4 xv = __ldg((const float4*)(x + r));
            const T* e = (const T*)&v;
            const T* xe = (const T*)&xv;
#pragma unroll
            for (int k = 0; k < R; ++k) madd<CONJ>(acc, e[k], xe[k]);
        }
        for (int k = 0; k < R; ++k)
            if (r + k < r1) madd<CONJ>(acc, Ac[r + k], x[r + k]);
    } else {
        for (int r = r0 + lane; r < r1; r += 32) madd<CONJ>(acc, Ac[r], x[(long)r * incx]);
    }
    acc = warp_sum_t(acc);
    if (S == 1) {
        if (lane == 0) {
            T* yp = y + col * incy;
            *yp = axpby(alpha, acc, beta, yp);
        }
        return;
    }
    if (lane == 0) {
        partial[(long)s * n + col] = acc;
        __threadfence();
        unsigned t = atomicAdd(counters + col, 1u);
        if (t == (unsigned)S - 1) {
            __threadfence();
            T sum = zero_of(T());
            for (int k = 0; k < S; ++k) sum = add(sum, ((volatile T*)partial)[(long)k * n + col]);
            T* yp = y + col * incy;
            *yp = axpby(alpha, sum, beta, yp);
            counters[col] = 0u;
        }
    }
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

template <class T>
cudaError_t gemv_impl(iclblasHandle_t h, int trans, int m, int n, T alpha, const T* A, int lda, const T* x, int incx,
                      T beta, T* y, int incy)
{
    constexpr int R = 16 / sizeof(T);
    const int target = h->sm_count * 8;
    if (trans == ICLBLAS_OP_N) {
        const bool vec = aligned16(A) && ((long)lda * sizeof(T)) % 16 == 0;
        const int rows_per_block = kNThreads * R;
        const int rt = ceil_div(m, rows_per_block);
        int splits = 1;
        if (rt < target && rt <= kCounterWords) {
            splits = ceil_div(target, rt);
            splits = min(splits, max(1, n / 64));
        }
        int cps = ceil_div(n, splits);
        cps = (cps + 7) & ~7;
        splits = ceil_div(n, cps);
        T* partial = nullptr;
        if (splits > 1) {
            partial = (T*)scratch(h, sizeof(T) * (size_t)splits * (size_t)m);
            if (!partial) return cudaErrorMemoryAllocation;
        }
        dim3 grid(rt, splits);
        if (vec)
            gemv_n_kernel<T, true><<<grid, kNThreads, 0, h->stream>>>(m, n, alpha, A, lda, x, incx, beta, y, incy, cps,
                                                                      partial, h->ws.counters);
        else
            gemv_n_kernel<T, false><<<grid, kNThreads, 0, h->stream>>>(m, n, alpha, A, lda, x, incx, beta, y, incy,
                                                                       cps, partial, h->ws.counters);
        return cudaGetLastError();
    }
    // op T / C: columns of A are dot products with x
    const bool vec = aligned16(A) && ((long)lda * sizeof(T)) % 16 == 0 && incx == 1 && aligned16(x);
    const int warps_target = target * (kTThreads / 32);
    int S = 1;
    if (n < warps_target && n <= kCounterWords) S = min(ceil_div(warps_target, n), max(1, m / 1024));
    int rps = ceil_div(m, S);
    rps = (rps + 32 * R - 1) / (32 * R) * (32 * R);
    S = ceil_div(m, rps);
    T* partial = nullptr;
    if (S > 1) {
        partial = (T*)scratch(h, sizeof(T) * (size_t)S * (size_t)n);
        if (!partial) return cudaErrorMemoryAllocation;
    }
    const long warps = (long)n * S;
    const int grid = (int)((warps * 32 + kTThreads - 1) / kTThreads);
    const bool conj = (trans == ICLBLAS_OP_C) && sizeof(T) == sizeof(cfloat);
#define LAUNCH(C, V)                                                                                         \
    gemv_t_kernel<T, C, V><<<grid, kTThreads, 0, h->stream>>>(m, n, alpha, A, lda, x, incx, beta, y, incy, S, \
                                                              rps, partial, h->ws.counters)
    if (conj) { if (vec) LAUNCH(true, true); else LAUNCH(true, false); }
    else { if (vec) LAUNCH(false, true); else LAUNCH(false, false); }
#undef LAUNCH
    return cudaGetLastError();
}

}  // namespace

cudaError_t sgemv(iclblasHandle_t h, int trans, int m, int n, float alpha, const float* A, int lda, const float* x,
                  int incx, float beta, float* y, int incy)
{
    return gemv_impl<float>(h, trans, m, n, alpha, A, lda, x, incx, beta, y, incy);
}

cudaError_t cgemv(iclblasHandle_t h, int trans, int m, int n, cfloat alpha, const cfloat* A, int lda, const cfloat* x,
                  int incx, cfloat beta, cfloat* y, int incy)
{
    return gemv_impl<cfloat>(h, trans, m, n, alpha, A, lda, x, incx, beta, y, incy);
}

}  // namespace iclb
