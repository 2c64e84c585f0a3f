// Rank-1 updates A += alpha x y^T (Sger), alpha x y^T (Cgeru) and
// alpha x y^H (Cgerc).
//
// HBM-bound: every element of A is read and written once (8 B per element
// single, 16 B complex); x and y are read once per CTA from L2.  Aligned
// unit-stride x with a 16-byte aligned A and lda a multiple of the float4
// width takes the 128-bit path: a CTA owns 256 float4 row words (1024 rows
// single, 512 complex) of kColsPerCta columns, keeps its x words in
// registers and streams the columns four at a time.  Everything else uses a
// grid-stride loop over elements.
//
// Per-element arithmetic is the reference kernels' (Sger_naive.cl:16-26:
// prod = x*y rounded, a = fma(alpha, prod, a); Cgeru_naive.cl / Cgerc_naive.cl:
// a += cmul(alpha, cmul(x, y or conj(y))) with complex.h.cl's fma placement),
// so results are bit-exact against a CPU restatement of those expressions.
#include <algorithm>

#include "common.cuh"

namespace iclb {
namespace {

constexpr int kThreads = 256;
constexpr int kColsPerCta = 32;

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

struct SgerOp {
    float alpha;
    __device__ float operator()(float a, float x, float y) const { return fmaf(alpha, __fmul_rn(x, y), a); }
};
template <bool CONJ>
struct CgerOp {
    cfloat alpha;
    __device__ cfloat operator()(cfloat a, cfloat x, cfloat y) const
    {
        const cfloat t = cmul_fma(alpha, cmul_fma(x, CONJ ? cfloat{y.re, -y.im} : y));
        return cfloat{__fadd_rn(a.re, t.re), __fadd_rn(a.im, t.im)};
    }
};

// 128-bit path.  blockIdx.x: row tile of 256 words, blockIdx.y: column group.
template <class T, class Op>
__global__ void __launch_bounds__(kThreads) ger_vec_kernel(int m, int n, const T* __restrict__ x,
                                                           const T* __restrict__ y, long incy, T* A, long lda, Op op)
{
    constexpr int per = (int)(16 / sizeof(T));
    const long r0 = ((long)blockIdx.x * kThreads + threadIdx.x) * per;  // first row of this thread's word
    const int c0 = blockIdx.y * kColsPerCta;
    const int c1 = min(n, c0 + kColsPerCta);
    if (r0 >= m) return;
    if (r0 + per <= m) {
        float4 xw = __ldg((const float4*)(x + r0));
        const T* xe = (const T*)&xw;
        int c = c0;
        for (; c + 4 <= c1; c += 4) {
            float4 w[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) w[u] = ld_stream4((const float4*)(A + (long)(c + u) * lda + r0));
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const T yv = y[(long)(c + u) * incy];
                T* e = (T*)&w[u];
#pragma unroll
                for (int k = 0; k < per; ++k) e[k] = op(e[k], xe[k], yv);
                __stcs((float4*)(A + (long)(c + u) * lda + r0), w[u]);
            }
        }
        for (; c < c1; ++c) {
            float4 w = ld_stream4((const float4*)(A + (long)c * lda + r0));
            const T yv = y[(long)c * incy];
            T* e = (T*)&w;
#pragma unroll
            for (int k = 0; k < per; ++k) e[k] = op(e[k], xe[k], yv);
            __stcs((float4*)(A + (long)c * lda + r0), w);
        }
    } else {
        // the last rows, fewer than one word: element by element
        for (int c = c0; c < c1; ++c) {
            const T yv = y[(long)c * incy];
            for (long r = r0; r < m; ++r) A[(long)c * lda + r] = op(A[(long)c * lda + r], x[r], yv);
        }
    }
}

template <class T, class Op>
__global__ void __launch_bounds__(kThreads) ger_strided_kernel(int m, int n, const T* __restrict__ x, long incx,
                                                               const T* __restrict__ y, long incy, T* A, long lda,
                                                               Op op)
{
    const long total = (long)m * n;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        const long i = e % m, j = e / m;
        A[j * lda + i] = op(A[j * lda + i], x[i * incx], y[j * incy]);
    }
}

template <class T, class Op>
cudaError_t ger_impl(iclblasHandle_t h, int m, int n, const T* x, int incx, const T* y, int incy, T* A, int lda,
                     Op op)
{
    constexpr int per = (int)(16 / sizeof(T));
    const long col_groups = ((long)n + kColsPerCta - 1) / kColsPerCta;
    if (incx == 1 && aligned16(x) && aligned16(A) && lda % per == 0 && col_groups <= 65535) {
        const long words = ((long)m + per - 1) / per;
        dim3 grid((unsigned)((words + kThreads - 1) / kThreads), (unsigned)col_groups);
        ger_vec_kernel<T, Op><<<grid, kThreads, 0, h->stream>>>(m, n, x, y, incy, A, lda, op);
    } else {
        const long total = (long)m * n;
        const long g = std::min<long>((total + kThreads - 1) / kThreads, (long)h->sm_count * 8);
        ger_strided_kernel<T, Op><<<(int)std::max<long>(g, 1), kThreads, 0, h->stream>>>(m, n, x, incx, y, incy, A,
                                                                                          lda, op);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t sger(iclblasHandle_t h, int m, int n, float alpha, const float* x, int incx, const float* y, int incy,
                 float* A, int lda)
{
    return ger_impl<float>(h, m, n, x, incx, y, incy, A, lda, SgerOp{alpha});
}

cudaError_t cger(iclblasHandle_t h, bool conj, int m, int n, cfloat alpha, const cfloat* x, int incx,
                 const cfloat* y, int incy, cfloat* A, int lda)
{
    if (conj) return ger_impl<cfloat>(h, m, n, x, incx, y, incy, A, lda, CgerOp<true>{alpha});
    return ger_impl<cfloat>(h, m, n, x, incx, y, incy, A, lda, CgerOp<false>{alpha});
}

}  // namespace iclb
