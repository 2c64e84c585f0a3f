// Level-1 kernels: axpy, scal, dot, nrm2, asum, iamax, iamin (single and complex).
//
// All of them stream their vectors once from HBM.  Unit-stride vectors whose
// base addresses are 16-byte aligned take 128-bit loads/stores; other
// strides use a scalar grid-stride loop.  Reductions are deterministic: the
// grid size depends only on n and the SM count, every thread accumulates its
// fixed subset of elements in increasing index order in FP64, the block sums
// and the final pass over the per-block partials use fixed trees, and the
// last block to finish (ticket counter) produces the result in the same
// launch.  The FP64 accumulation matches the reference's CPU oracles
// (double accumulators: tests/blas_funcs/test_dot.hpp:22-51,
// test_nrm2.hpp:23-57, test_asum.hpp:23-33); iamax returns the reference's
// 0-based first maximal index (tests/blas_reference/blas_reference.cpp:46-64)
// exactly, for every n (no float-encoded indices).
#include <climits>
#include <mutex>

#include "common.cuh"

namespace iclb {
namespace {

constexpr int kThreads = 256;

// One thread per unit, at most `per_sm` CTAs per SM (grid-stride beyond).
// The cap is per kernel, the best of 3/4/6/8 CTAs per SM measured at
// n = 2^28: 4 for saxpy, 6 for sasum and iamax, 8 for the others (sscal and
// snrm2 lose 15-25% at 4; sdot is flat).
__host__ int l1_grid(iclblasHandle_t h, long units, int per_sm = 8)
{
    long g = (units + kThreads - 1) / kThreads;
    long cap = (long)h->sm_count * per_sm;
    if (g > cap) g = cap;
    return g < 1 ? 1 : (int)g;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// ---------------------------------------------------------------- axpy/scal
// y = fma(alpha, x, y): one rounding of alpha*x + y (the reference kernel
// computes this_y += alpha*this_x, Saxpy_noinc.cl).
__global__ void __launch_bounds__(kThreads) saxpy_vec(long n4, float alpha, const float4* __restrict__ x,
                                                      float4* __restrict__ y)
{
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        float4 a = ld_stream4(x + i), b = ld_stream4(y + i);
        b.x = fmaf(alpha, a.x, b.x);
        b.y = fmaf(alpha, a.y, b.y);
        b.z = fmaf(alpha, a.z, b.z);
        b.w = fmaf(alpha, a.w, b.w);
        __stcs(y + i, b);
    }
}

__global__ void __launch_bounds__(kThreads) saxpy_strided(long n, float alpha, const float* __restrict__ x, long incx,
                                                          float* __restrict__ y, long incy)
{
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        y[i * incy] = fmaf(alpha, x[i * incx], y[i * incy]);
}

__global__ void __launch_bounds__(kThreads) sscal_vec(long n4, float alpha, float4* __restrict__ x)
{
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        float4 a = ld_stream4(x + i);
        a.x *= alpha; a.y *= alpha; a.z *= alpha; a.w *= alpha;
        __stcs(x + i, a);
    }
}

__global__ void __launch_bounds__(kThreads) sscal_strided(long n, float alpha, float* __restrict__ x, long incx)
{
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i * incx] *= alpha;
}

// Complex y += alpha*x and x *= alpha evaluated in double with one rounding
// to float per component (the reference's CPU oracle arithmetic,
// tests/blas_funcs/test_axpy.hpp:22-46, test_scal.hpp:27-39).  The explicit
// _rn intrinsics keep the compiler from contracting into FMAs so the result
// matches that oracle bit for bit.
__device__ __forceinline__ cfloat cmad_d(cfloat a, cfloat x, cfloat y)
{
    double re = __dsub_rn(__dmul_rn(a.re, x.re), __dmul_rn(a.im, x.im));
    double im = __dadd_rn(__dmul_rn(a.re, x.im), __dmul_rn(a.im, x.re));
    return cfloat{(float)__dadd_rn((double)y.re, re), (float)__dadd_rn((double)y.im, im)};
}
__device__ __forceinline__ cfloat cmul_d(cfloat x, cfloat a)
{
    double re = __dsub_rn(__dmul_rn(x.re, a.re), __dmul_rn(x.im, a.im));
    double im = __dadd_rn(__dmul_rn(x.re, a.im), __dmul_rn(x.im, a.re));
    return cfloat{(float)re, (float)im};
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads) caxpy_kernel(long n, cfloat alpha, const cfloat* __restrict__ x, long incx,
                                                         cfloat* __restrict__ y, long incy)
{
    const long stride = (long)gridDim.x * blockDim.x;
    if (VEC) {
        const float4* x4 = (const float4*)x;
        float4* y4 = (float4*)y;
        const long n2 = n >> 1;
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride) {
            float4 a = ld_stream4(x4 + i), b = ld_stream4(y4 + i);
            cfloat r0 = cmad_d(alpha, cfloat{a.x, a.y}, cfloat{b.x, b.y});
            cfloat r1 = cmad_d(alpha, cfloat{a.z, a.w}, cfloat{b.z, b.w});
            __stcs(y4 + i, make_float4(r0.re, r0.im, r1.re, r1.im));
        }
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) y[n - 1] = cmad_d(alpha, x[n - 1], y[n - 1]);
    } else {
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
            y[i * incy] = cmad_d(alpha, x[i * incx], y[i * incy]);
    }
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads) cscal_kernel(long n, cfloat alpha, cfloat* __restrict__ x, long incx)
{
    const long stride = (long)gridDim.x * blockDim.x;
    if (VEC) {
        float4* x4 = (float4*)x;
        const long n2 = n >> 1;
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride) {
            float4 a = ld_stream4(x4 + i);
            cfloat r0 = cmul_d(cfloat{a.x, a.y}, alpha), r1 = cmul_d(cfloat{a.z, a.w}, alpha);
            __stcs(x4 + i, make_float4(r0.re, r0.im, r1.re, r1.im));
        }
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) x[n - 1] = cmul_d(x[n - 1], alpha);
    } else {
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
            x[i * incx] = cmul_d(x[i * incx], alpha);
    }
}

// ---------------------------------------------------------------- real reductions
template <Red OP>
__device__ __forceinline__ double rterm(float a, float b)
{
    if (OP == Red::Dot) return (double)a * (double)b;
    if (OP == Red::Asum) return fabs((double)a);
    return (double)a * (double)a;  // Nrm2: sum of squares, sqrt at the end
}

// Sum over i of term(x[i], y[i]).  VEC: unit stride, 16-byte aligned.
template <Red OP, bool VEC>
__global__ void __launch_bounds__(kThreads) sreduce_kernel(long n, const float* __restrict__ x, long incx,
                                                           const float* __restrict__ y, long incy,
                                                           double* __restrict__ partials, unsigned* counter,
                                                           float* __restrict__ result)
{
    __shared__ double sh[32];
    const long stride = (long)gridDim.x * blockDim.x;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double acc = 0.0, acc2 = 0.0;
    if (VEC) {
        const float4* x4 = (const float4*)x;
        const float4* y4 = (const float4*)y;
        const long n4 = n >> 2;
        long i = tid;
        for (; i + 3 * stride < n4; i += 4 * stride) {
            float4 a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a[u] = ld_stream4(x4 + i + u * stride);
                b[u] = OP == Red::Dot ? ld_stream4(y4 + i + u * stride) : a[u];
            }
            // two partial sums (x,y and z,w components) shorten the dependent
            // FP64 chain; they are combined in a fixed order below
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                acc += rterm<OP>(a[u].x, b[u].x);
                acc2 += rterm<OP>(a[u].z, b[u].z);
                acc += rterm<OP>(a[u].y, b[u].y);
                acc2 += rterm<OP>(a[u].w, b[u].w);
            }
        }
        acc += acc2;
        for (; i < n4; i += stride) {
            float4 a = ld_stream4(x4 + i);
            float4 b = OP == Red::Dot ? ld_stream4(y4 + i) : a;
            acc += rterm<OP>(a.x, b.x);
            acc += rterm<OP>(a.y, b.y);
            acc += rterm<OP>(a.z, b.z);
            acc += rterm<OP>(a.w, b.w);
        }
        if (tid == 0)
            for (long j = n4 * 4; j < n; ++j) acc += rterm<OP>(x[j], OP == Red::Dot ? y[j] : x[j]);
    } else {
        for (long i = tid; i < n; i += stride) {
            float a = x[i * incx];
            acc += rterm<OP>(a, OP == Red::Dot ? y[i * incy] : a);
        }
    }
    double bs = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = bs;
    if (!last_block(counter)) return;
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += ((volatile double*)partials)[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
        *result = OP == Red::Nrm2 ? (float)sqrt(s) : (float)s;
        *counter = 0u;
    }
}

// ---------------------------------------------------------------- complex reductions
// Real-valued reductions of a complex vector: asum = sum |re|+|im|
// (scasum, test_asum.hpp with blas_abs of a complex), nrm2 = sqrt(sum re^2+im^2).
template <Red OP>
__device__ __forceinline__ double cterm(float re, float im)
{
    if (OP == Red::Asum) return fabs((double)re) + fabs((double)im);
    return (double)re * (double)re + (double)im * (double)im;
}

template <Red OP, bool VEC>
__global__ void __launch_bounds__(kThreads) creduce_kernel(long n, const cfloat* __restrict__ x, long incx,
                                                           double* __restrict__ partials, unsigned* counter,
                                                           float* __restrict__ result)
{
    __shared__ double sh[32];
    const long stride = (long)gridDim.x * blockDim.x;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double acc = 0.0;
    if (VEC) {
        const float4* x4 = (const float4*)x;
        const long n2 = n >> 1;
        long i = tid;
        for (; i + 3 * stride < n2; i += 4 * stride) {
            float4 a[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) a[u] = ld_stream4(x4 + i + u * stride);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                acc += cterm<OP>(a[u].x, a[u].y);
                acc += cterm<OP>(a[u].z, a[u].w);
            }
        }
        for (; i < n2; i += stride) {
            float4 a = ld_stream4(x4 + i);
            acc += cterm<OP>(a.x, a.y);
            acc += cterm<OP>(a.z, a.w);
        }
        if (tid == 0 && (n & 1)) acc += cterm<OP>(x[n - 1].re, x[n - 1].im);
    } else {
        for (long i = tid; i < n; i += stride) {
            cfloat v = x[i * incx];
            acc += cterm<OP>(v.re, v.im);
        }
    }
    double bs = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = bs;
    if (!last_block(counter)) return;
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += ((volatile double*)partials)[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
        *result = OP == Red::Nrm2 ? (float)sqrt(s) : (float)s;
        *counter = 0u;
    }
}

// cdotu / cdotc: sum conj?(x)*y in complex double (test_dot.hpp:22-51).
template <bool CONJ, bool VEC>
__global__ void __launch_bounds__(kThreads) cdot_kernel(long n, const cfloat* __restrict__ x, long incx,
                                                        const cfloat* __restrict__ y, long incy,
                                                        double* __restrict__ partials, unsigned* counter,
                                                        cfloat* __restrict__ result)
{
    __shared__ double sh[32];
    const long stride = (long)gridDim.x * blockDim.x;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double re = 0.0, im = 0.0;
    auto term = [&](float xr, float xi, float yr, float yi) {
        double a = xr, b = CONJ ? -(double)xi : (double)xi, c = yr, d = yi;
        re += a * c - b * d;
        im += a * d + b * c;
    };
    if (VEC) {
        const float4* x4 = (const float4*)x;
        const float4* y4 = (const float4*)y;
        const long n2 = n >> 1;
        long i = tid;
        for (; i + 1 * stride < n2; i += 2 * stride) {
            float4 a0 = ld_stream4(x4 + i), b0 = ld_stream4(y4 + i);
            float4 a1 = ld_stream4(x4 + i + stride), b1 = ld_stream4(y4 + i + stride);
            term(a0.x, a0.y, b0.x, b0.y);
            term(a0.z, a0.w, b0.z, b0.w);
            term(a1.x, a1.y, b1.x, b1.y);
            term(a1.z, a1.w, b1.z, b1.w);
        }
        for (; i < n2; i += stride) {
            float4 a = ld_stream4(x4 + i), b = ld_stream4(y4 + i);
            term(a.x, a.y, b.x, b.y);
            term(a.z, a.w, b.z, b.w);
        }
        if (tid == 0 && (n & 1)) term(x[n - 1].re, x[n - 1].im, y[n - 1].re, y[n - 1].im);
    } else {
        for (long i = tid; i < n; i += stride) {
            cfloat a = x[i * incx], b = y[i * incy];
            term(a.re, a.im, b.re, b.im);
        }
    }
    double bre = block_sum(re, sh);
    double bim = block_sum(im, sh);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = bre;
        partials[2 * blockIdx.x + 1] = bim;
    }
    if (!last_block(counter)) return;
    double sr = 0.0, si = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
        sr += ((volatile double*)partials)[2 * i];
        si += ((volatile double*)partials)[2 * i + 1];
    }
    sr = block_sum(sr, sh);
    si = block_sum(si, sh);
    if (threadIdx.x == 0) {
        *result = cfloat{(float)sr, (float)si};
        *counter = 0u;
    }
}

// ---------------------------------------------------------------- iamax
// Candidate (value, index) pairs are ordered by key, then by smaller index;
// NaN never enters (comparisons with NaN are false) and the start key -inf is
// below every other key.  iamax keys are |x|, iamin keys are -|x|.  The
// reduction of that total order gives the first index of the extreme key over
// non-NaN elements, which is what the reference's scans (strict '>' or '<'
// from x[0]) return unless x[0] itself is NaN; that case pins the scan to 0
// and is applied at the end, as is an iamin input made only of infinities
// (no candidate: the scan stays at 0).
struct Cand {
    float v;
    int i;
};
__device__ __forceinline__ void cand_take(Cand& c, float v, int i)
{
    if (v > c.v) { c.v = v; c.i = i; }
}
__device__ __forceinline__ void cand_merge(Cand& c, Cand o)
{
    if (o.v > c.v || (o.v == c.v && o.i < c.i)) c = o;
}
__device__ __forceinline__ Cand warp_cand(Cand c)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        Cand o;
        o.v = __shfl_xor_sync(0xffffffffu, c.v, off);
        o.i = __shfl_xor_sync(0xffffffffu, c.i, off);
        cand_merge(c, o);
    }
    return c;
}
__device__ __forceinline__ Cand block_cand(Cand c, Cand* sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    c = warp_cand(c);
    __syncthreads();
    if (lane == 0) sh[wid] = c;
    __syncthreads();
    Cand r{-INFINITY, INT_MAX};
    if (wid == 0) {
        if (lane < nw) r = sh[lane];
        r = warp_cand(r);
    }
    return r;
}

__device__ __forceinline__ float absval(float v) { return fabsf(v); }
// scabs1 (core/src/ocl/complex.h.cl:54): |re| + |im| in float.
__device__ __forceinline__ float absval(cfloat v) { return fabsf(v.re) + fabsf(v.im); }
__device__ __forceinline__ bool isnan_v(float v) { return isnan(v); }
__device__ __forceinline__ bool isnan_v(cfloat v) { return isnan(fabsf(v.re) + fabsf(v.im)); }

template <bool MIN, class T>
__device__ __forceinline__ float iakey(T v)
{
    return MIN ? -absval(v) : absval(v);
}

template <class T, bool VEC, bool MIN = false>
__global__ void __launch_bounds__(kThreads) iamax_kernel(long n, const T* __restrict__ x, long incx,
                                                         Cand* __restrict__ partials, unsigned* counter,
                                                         int* __restrict__ result)
{
    __shared__ Cand sh[32];
    const long stride = (long)gridDim.x * blockDim.x;
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    Cand c{-INFINITY, INT_MAX};
    constexpr int per = (int)(16 / sizeof(T));  // elements per 128-bit load
    if (VEC) {
        const float4* x4 = (const float4*)x;
        const long nv = n / per;
        long i = tid;
        for (; i + 3 * stride < nv; i += 4 * stride) {
            float4 a[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) a[u] = ld_stream4(x4 + i + u * stride);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const T* e = (const T*)&a[u];
                const int base = (int)((i + u * stride) * per);
#pragma unroll
                for (int k = 0; k < per; ++k) cand_take(c, iakey<MIN>(e[k]), base + k);
            }
        }
        for (; i < nv; i += stride) {
            float4 a = ld_stream4(x4 + i);
            const T* e = (const T*)&a;
#pragma unroll
            for (int k = 0; k < per; ++k) cand_take(c, iakey<MIN>(e[k]), (int)(i * per + k));
        }
        if (tid == 0)
            for (long j = nv * per; j < n; ++j) cand_take(c, iakey<MIN>(x[j]), (int)j);
    } else {
        for (long i = tid; i < n; i += stride) cand_take(c, iakey<MIN>(x[i * incx]), (int)i);
    }
    Cand b = block_cand(c, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = b;
    if (!last_block(counter)) return;
    Cand r{-INFINITY, INT_MAX};
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
        Cand o;
        o.v = ((volatile float*)&partials[i].v)[0];
        o.i = ((volatile int*)&partials[i].i)[0];
        cand_merge(r, o);
    }
    r = block_cand(r, sh);
    if (threadIdx.x == 0) {
        int idx = r.i;
        if (isnan_v(x[0]) || idx == INT_MAX) idx = 0;
        *result = idx;
        *counter = 0u;
    }
}

}  // namespace

// ------------------------------------------------------------------ launchers
cudaError_t saxpy(iclblasHandle_t h, int n, float alpha, const float* x, int incx, float* y, int incy)
{
    if (incx == 1 && incy == 1 && aligned16(x) && aligned16(y)) {
        long n4 = n >> 2;
        if (n4 > 0) saxpy_vec<<<l1_grid(h, n4, 4), kThreads, 0, h->stream>>>(n4, alpha, (const float4*)x, (float4*)y);
        long rem = n - n4 * 4;
        if (rem > 0) saxpy_strided<<<1, 32, 0, h->stream>>>(rem, alpha, x + n4 * 4, 1, y + n4 * 4, 1);
    } else {
        saxpy_strided<<<l1_grid(h, n), kThreads, 0, h->stream>>>(n, alpha, x, incx, y, incy);
    }
    return cudaGetLastError();
}

cudaError_t sscal(iclblasHandle_t h, int n, float alpha, float* x, int incx)
{
    if (incx == 1 && aligned16(x)) {
        long n4 = n >> 2;
        if (n4 > 0) sscal_vec<<<l1_grid(h, n4), kThreads, 0, h->stream>>>(n4, alpha, (float4*)x);
        long rem = n - n4 * 4;
        if (rem > 0) sscal_strided<<<1, 32, 0, h->stream>>>(rem, alpha, x + n4 * 4, 1);
    } else {
        sscal_strided<<<l1_grid(h, n), kThreads, 0, h->stream>>>(n, alpha, x, incx);
    }
    return cudaGetLastError();
}

cudaError_t caxpy(iclblasHandle_t h, int n, cfloat alpha, const cfloat* x, int incx, cfloat* y, int incy)
{
    if (incx == 1 && incy == 1 && aligned16(x) && aligned16(y))
        caxpy_kernel<true><<<l1_grid(h, (long)n / 2 + 1), kThreads, 0, h->stream>>>(n, alpha, x, 1, y, 1);
    else
        caxpy_kernel<false><<<l1_grid(h, n), kThreads, 0, h->stream>>>(n, alpha, x, incx, y, incy);
    return cudaGetLastError();
}

cudaError_t cscal(iclblasHandle_t h, int n, cfloat alpha, cfloat* x, int incx)
{
    if (incx == 1 && aligned16(x))
        cscal_kernel<true><<<l1_grid(h, (long)n / 2 + 1), kThreads, 0, h->stream>>>(n, alpha, x, 1);
    else
        cscal_kernel<false><<<l1_grid(h, n), kThreads, 0, h->stream>>>(n, alpha, x, incx);
    return cudaGetLastError();
}

cudaError_t sreduce(iclblasHandle_t h, Red op, int n, const float* x, int incx, const float* y, int incy,
                    float* result)
{
    const bool vec = incx == 1 && aligned16(x) && (op != Red::Dot || (incy == 1 && aligned16(y)));
    const int grid = l1_grid(h, vec ? ((long)n + 3) / 4 : n, op == Red::Asum ? 6 : 8);
    double* partials = (double*)scratch(h, sizeof(double) * (size_t)grid);
    if (!partials) return cudaErrorMemoryAllocation;
    unsigned* ctr = h->ws.counters;
#define LAUNCH(OP, V) \
    sreduce_kernel<OP, V><<<grid, kThreads, 0, h->stream>>>(n, x, incx, y, incy, partials, ctr, result)
    switch (op) {
    case Red::Dot: if (vec) LAUNCH(Red::Dot, true); else LAUNCH(Red::Dot, false); break;
    case Red::Asum: if (vec) LAUNCH(Red::Asum, true); else LAUNCH(Red::Asum, false); break;
    case Red::Nrm2: if (vec) LAUNCH(Red::Nrm2, true); else LAUNCH(Red::Nrm2, false); break;
    }
#undef LAUNCH
    return cudaGetLastError();
}

// ---------------------------------------------------------------- SDOT without allocation
// Fixed scratch of iclblasSdotNoAlloc: one FP64 partial per thread block and
// the last-block ticket.  It is part of the library image, so every GPU that
// loads the library holds it (32 KiB + 256 B) until the process exits.  In
// host code `g_sdot_noalloc_scratch` names a host-side stand-in, not device
// memory: host code must use the address from cudaGetSymbolAddress.
struct SdotNoAllocScratch {
    double partials[kSdotNoAllocMaxBlocks];
    unsigned counter;
};
static __device__ __align__(256) SdotNoAllocScratch g_sdot_noalloc_scratch;

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
struct NoAllocAddr {
    unsigned long long ctx_id = 0;   // CUDA context the address belongs to (0: none yet)
    SdotNoAllocScratch* ptr = nullptr;
};
NoAllocAddr g_noalloc_addr[kMaxDevices];

// Unique ID of the current CUDA context (cuCtxGetId through the runtime's
// driver entry point; IDs are never reused within a process), 0 if unknown.
unsigned long long current_context_id()
{
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (GetCurrent)p;
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (GetId)p;
        cudaGetLastError();
    });
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of the scratch on `device`, looked up with that device
// current once per device and CUDA context: cudaDeviceReset destroys the
// device's primary context, and the next call looks the address up again
// in the new one.
cudaError_t noalloc_scratch_addr(int device, SdotNoAllocScratch** out)
{
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    DeviceGuard guard(device);
    if (guard.status() != cudaSuccess) return guard.status();
    // (the handle's calls made this device's primary context current; with
    // the context unknown the address is looked up on every call)
    const unsigned long long ctx = current_context_id();
    NoAllocAddr& a = g_noalloc_addr[device];
    if (!a.ptr || ctx == 0 || a.ctx_id != ctx) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_sdot_noalloc_scratch);
        if (e != cudaSuccess) return e;
        a.ptr = (SdotNoAllocScratch*)ptr;
        a.ctx_id = ctx;
    }
    *out = a.ptr;
    return cudaSuccess;
}
}  // namespace

cudaError_t sdot_noalloc(iclblasHandle_t h, int n, const float* x, int incx, const float* y, int incy, float* result)
{
    const bool vec = incx == 1 && aligned16(x) && incy == 1 && aligned16(y);
    const int grid = l1_grid(h, vec ? ((long)n + 3) / 4 : n);
    if (grid > kSdotNoAllocMaxBlocks) return cudaErrorNotSupported;
    SdotNoAllocScratch* sc = nullptr;
    cudaError_t e = noalloc_scratch_addr(h->device, &sc);
    if (e != cudaSuccess) return e;
    // the array keeps the previous call's contents: the ticket must start at 0
    e = cudaMemsetAsync(&sc->counter, 0, sizeof(unsigned), h->stream);
    if (e != cudaSuccess) return e;
    if (vec)
        sreduce_kernel<Red::Dot, true><<<grid, kThreads, 0, h->stream>>>(n, x, incx, y, incy, sc->partials,
                                                                          &sc->counter, result);
    else
        sreduce_kernel<Red::Dot, false><<<grid, kThreads, 0, h->stream>>>(n, x, incx, y, incy, sc->partials,
                                                                           &sc->counter, result);
    return cudaGetLastError();
}

cudaError_t creduce_real(iclblasHandle_t h, Red op, int n, const cfloat* x, int incx, float* result)
{
    const bool vec = incx == 1 && aligned16(x);
    const int grid = l1_grid(h, vec ? ((long)n + 1) / 2 : n);
    double* partials = (double*)scratch(h, sizeof(double) * (size_t)grid);
    if (!partials) return cudaErrorMemoryAllocation;
    unsigned* ctr = h->ws.counters;
    if (op == Red::Asum) {
        if (vec) creduce_kernel<Red::Asum, true><<<grid, kThreads, 0, h->stream>>>(n, x, incx, partials, ctr, result);
        else creduce_kernel<Red::Asum, false><<<grid, kThreads, 0, h->stream>>>(n, x, incx, partials, ctr, result);
    } else {
        if (vec) creduce_kernel<Red::Nrm2, true><<<grid, kThreads, 0, h->stream>>>(n, x, incx, partials, ctr, result);
        else creduce_kernel<Red::Nrm2, false><<<grid, kThreads, 0, h->stream>>>(n, x, incx, partials, ctr, result);
    }
    return cudaGetLastError();
}

cudaError_t cdot(iclblasHandle_t h, bool conj, int n, const cfloat* x, int incx, const cfloat* y, int incy,
                 cfloat* result)
{
    const bool vec = incx == 1 && incy == 1 && aligned16(x) && aligned16(y);
    const int grid = l1_grid(h, vec ? ((long)n + 1) / 2 : n);
    double* partials = (double*)scratch(h, 2 * sizeof(double) * (size_t)grid);
    if (!partials) return cudaErrorMemoryAllocation;
    unsigned* ctr = h->ws.counters;
#define LAUNCH(C, V) cdot_kernel<C, V><<<grid, kThreads, 0, h->stream>>>(n, x, incx, y, incy, partials, ctr, result)
    if (conj) { if (vec) LAUNCH(true, true); else LAUNCH(true, false); }
    else { if (vec) LAUNCH(false, true); else LAUNCH(false, false); }
#undef LAUNCH
    return cudaGetLastError();
}

namespace {
template <class T, bool MIN>
cudaError_t iamax_impl(iclblasHandle_t h, int n, const T* x, int incx, int* result)
{
    const bool vec = incx == 1 && aligned16(x);
    const int grid = l1_grid(h, vec ? ((long)n + (16 / sizeof(T)) - 1) / (16 / sizeof(T)) : n, 6);
    Cand* partials = (Cand*)scratch(h, sizeof(Cand) * (size_t)grid);
    if (!partials) return cudaErrorMemoryAllocation;
    if (vec)
        iamax_kernel<T, true, MIN><<<grid, kThreads, 0, h->stream>>>(n, x, incx, partials, h->ws.counters, result);
    else
        iamax_kernel<T, false, MIN><<<grid, kThreads, 0, h->stream>>>(n, x, incx, partials, h->ws.counters, result);
    return cudaGetLastError();
}
}  // namespace

cudaError_t isamax(iclblasHandle_t h, int n, const float* x, int incx, int* result)
{
    return iamax_impl<float, false>(h, n, x, incx, result);
}
cudaError_t icamax(iclblasHandle_t h, int n, const cfloat* x, int incx, int* result)
{
    return iamax_impl<cfloat, false>(h, n, x, incx, result);
}
// first index of the smallest |x| (scabs1 for complex): the reference's
// Isamin_naive.cl / Icamin_naive.cl scan (strict '<' from x[0])
cudaError_t isamin(iclblasHandle_t h, int n, const float* x, int incx, int* result)
{
    return iamax_impl<float, true>(h, n, x, incx, result);
}
cudaError_t icamin(iclblasHandle_t h, int n, const cfloat* x, int incx, int* result)
{
    return iamax_impl<cfloat, true>(h, n, x, incx, result);
}

}  // namespace iclb
