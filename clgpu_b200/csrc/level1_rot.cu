// Level-1 data movement and plane rotations: copy, swap, rot, rotm (single),
// copy, swap, rot, srot (complex), and the rotation generators rotg, rotmg
// and crotg.
//
// The vector routines stream x and y once from HBM.  Every one of them is a
// per-element map of (x_i, y_i), so they share two kernels: a 128-bit path
// for unit strides with 16-byte aligned bases (the float view of the data,
// four floats or two complex per load), and a scalar grid-stride path for
// everything else.  The 128-bit path runs one wave of 4 CTAs x 256 threads
// per SM over the whole vector: at n = 2^28 that beat 8 CTAs per SM by 5-8%
// on read-modify-write streams (swap, rot), where a narrower window of
// concurrently touched addresses keeps more DRAM row hits; copy, which has
// only one load stream, keeps two words in flight per thread.
//
// Per-element arithmetic follows the reference kernels' expressions and
// their fused multiply-adds exactly (fma where they write fma/mad,
// separately rounded products elsewhere), so results are bit-exact against a
// CPU restatement that evaluates the same expressions.
//
// The generators are scalar: one thread, operands in device memory, so they
// run in stream order with the vector routines that consume their output.
#include <algorithm>

#include "common.cuh"

namespace iclb {
namespace {

constexpr int kThreads = 256;

int grid_for(iclblasHandle_t h, long units)
{
    long g = (units + kThreads - 1) / kThreads;
    long cap = (long)h->sm_count * 8;
    if (g > cap) g = cap;
    return g < 1 ? 1 : (int)g;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }

__device__ __forceinline__ cfloat cmul(cfloat a, cfloat b) { return cmul_fma(a, b); }

// ---------------------------------------------------------------- ops
// Each op maps one (x, y) element pair in registers.  kReadY / kWriteX say
// which streams it touches; prepare() runs once per thread and returns false
// when the call has no work (Srotm with a flag outside {-1, 0, 1}).
struct CopyOp {
    static constexpr bool kReadY = false, kWriteX = false;
    static constexpr int kUnroll = 2;
    __device__ bool prepare() { return true; }
    template <class T>
    __device__ void operator()(T& x, T& y) const { y = x; }
};

struct SwapOp {
    static constexpr bool kReadY = true, kWriteX = true;
    static constexpr int kUnroll = 1;
    __device__ bool prepare() { return true; }
    template <class T>
    __device__ void operator()(T& x, T& y) const
    {
        T t = x;
        x = y;
        y = t;
    }
};

// x' = c x + s y, y' = c y - s x with real c, s (Srot_naive.cl,
// Csrot_naive.cl: the same expression per real component).
struct RotOp {
    static constexpr bool kReadY = true, kWriteX = true;
    static constexpr int kUnroll = 1;
    float c, s;
    __device__ bool prepare() { return true; }
    __device__ void operator()(float& x, float& y) const
    {
        const float sy = mul(s, y), cy = mul(c, y);
        const float nx = fmaf(c, x, sy);
        y = fmaf(-s, x, cy);
        x = nx;
    }
    __device__ void operator()(cfloat& x, cfloat& y) const
    {
        (*this)(x.re, y.re);
        (*this)(x.im, y.im);
    }
};

// x' = c x + s y, y' = c y - conj(s) x with real c, complex s
// (Crot_naive.cl).
struct CrotOp {
    static constexpr bool kReadY = true, kWriteX = true;
    static constexpr int kUnroll = 1;
    float c;
    cfloat s;
    __device__ bool prepare() { return true; }
    __device__ void operator()(cfloat& x, cfloat& y) const
    {
        const cfloat sy = cmul(s, y);
        const cfloat nx{fmaf(x.re, c, sy.re), fmaf(x.im, c, sy.im)};
        const cfloat mx = cmul(cfloat{-s.re, s.im}, x);
        y = cfloat{fmaf(y.re, c, mx.re), fmaf(y.im, c, mx.im)};
        x = nx;
    }
};

// Modified rotation with the reference's param layout
// (Srotm_helpers.h.cl:27-41): flag -1: x' = p1 x + p2 y, y' = p3 x + p4 y;
// flag 0: x' = x + p2 y, y' = p3 x + y; flag 1: x' = p1 x + y,
// y' = p4 y - x.  `dev` (when set) holds the five parameters in device
// memory and is read by every thread; otherwise they are the by-value fields.
struct RotmOp {
    static constexpr bool kReadY = true, kWriteX = true;
    static constexpr int kUnroll = 1;
    float p[5];
    const float* dev;
    __device__ bool prepare()
    {
        if (dev)
#pragma unroll
            for (int k = 0; k < 5; ++k) p[k] = __ldg(dev + k);
        return p[0] == -1.f || p[0] == 0.f || p[0] == 1.f;
    }
    __device__ void operator()(float& x, float& y) const
    {
        float nx, ny;
        if (p[0] == -1.f) {
            nx = fmaf(p[1], x, mul(p[2], y));
            ny = fmaf(p[3], x, mul(p[4], y));
        } else if (p[0] == 0.f) {
            nx = fmaf(p[2], y, x);
            ny = fmaf(p[3], x, y);
        } else {
            nx = fmaf(p[1], x, y);
            ny = fmaf(p[4], y, -x);
        }
        x = nx;
        y = ny;
    }
};

// ---------------------------------------------------------------- kernels
// 128-bit path: n4 float4 words of each vector; T is the element type the
// op is defined on (four floats or two complex per word).  Op::kUnroll words
// per thread per iteration, grid-strided.
template <class T, class Op>
__global__ void __launch_bounds__(kThreads) pair_vec_kernel(long n4, float4* x, float4* y, Op op)
{
    if (!op.prepare()) return;
    constexpr int per = (int)(16 / sizeof(T));
    constexpr int U = Op::kUnroll;
    const long stride = (long)gridDim.x * blockDim.x;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + (U - 1) * stride < n4; i += U * stride) {
        float4 a[U], b[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            a[u] = ld_stream4(x + i + u * stride);
            b[u] = Op::kReadY ? ld_stream4(y + i + u * stride) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            T* ea = (T*)&a[u];
            T* eb = (T*)&b[u];
#pragma unroll
            for (int k = 0; k < per; ++k) op(ea[k], eb[k]);
            if (Op::kWriteX) __stcs(x + i + u * stride, a[u]);
            __stcs(y + i + u * stride, b[u]);
        }
    }
    if (i < n4) {
        float4 a = ld_stream4(x + i);
        float4 b = Op::kReadY ? ld_stream4(y + i) : make_float4(0.f, 0.f, 0.f, 0.f);
        T* ea = (T*)&a;
        T* eb = (T*)&b;
#pragma unroll
        for (int k = 0; k < per; ++k) op(ea[k], eb[k]);
        if (Op::kWriteX) __stcs(x + i, a);
        __stcs(y + i, b);
    }
}

template <class T, class Op>
__global__ void __launch_bounds__(kThreads) pair_strided_kernel(long n, T* x, long incx, T* y, long incy, Op op)
{
    if (!op.prepare()) return;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        T a = x[i * incx];
        T b{};
        if (Op::kReadY) b = y[i * incy];
        op(a, b);
        if (Op::kWriteX) x[i * incx] = a;
        y[i * incy] = b;
    }
}

// Unit strides with both bases 16-byte aligned: the vector path over whole
// words plus a one-warp tail; otherwise the strided path.
template <class T, class Op>
cudaError_t run_pair(iclblasHandle_t h, long n, T* x, long incx, T* y, long incy, Op op)
{
    if (incx == 1 && incy == 1 && aligned16(x) && aligned16(y)) {
        constexpr long per = 16 / sizeof(T);
        const long n4 = n / per;
        if (n4 > 0) {
            long g = (n4 + (long)kThreads * Op::kUnroll - 1) / ((long)kThreads * Op::kUnroll);
            g = std::min<long>(g, 4L * h->sm_count);
            pair_vec_kernel<T, Op><<<(int)g, kThreads, 0, h->stream>>>(n4, (float4*)x, (float4*)y, op);
        }
        const long rem = n - n4 * per;
        if (rem > 0)
            pair_strided_kernel<T, Op><<<1, 32, 0, h->stream>>>(rem, x + n4 * per, 1, y + n4 * per, 1, op);
    } else {
        pair_strided_kernel<T, Op><<<grid_for(h, n), kThreads, 0, h->stream>>>(n, x, incx, y, incy, op);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------- generators
__device__ __forceinline__ float sign_of(float v)  // OpenCL sign(): 0 for 0 and NaN
{
    return v > 0.f ? 1.f : (v < 0.f ? -1.f : 0.f);
}

// Givens rotation of (a, b) as the reference computes it (Srotg_naive.cl),
// including its scale = |a| * |b|: when either input is zero the result is
// c = 1, s = 0, r = z = 0.
__global__ void srotg_kernel(float* a, float* b, float* c, float* s)
{
    const float av = *a, bv = *b;
    const float fa = fabsf(av), fb = fabsf(bv);
    const float roe = fa > fb ? av : bv;
    const float scale = mul(fa, fb);
    float r, z;
    if (scale == 0.f) {
        *c = 1.f;
        *s = 0.f;
        r = 0.f;
        z = 0.f;
    } else {
        const float a2 = __fdiv_rn(av, scale), b2 = __fdiv_rn(bv, scale);
        r = mul(mul(sign_of(roe), scale), __fsqrt_rn(__fadd_rn(mul(a2, a2), mul(b2, b2))));
        const float cv = __fdiv_rn(av, r), sv = __fdiv_rn(bv, r);
        *c = cv;
        *s = sv;
        z = 1.f;
        if (fa > fb) z = sv;
        if (fb >= fa && cv != 0.f) z = __fdiv_rn(1.f, cv);
    }
    *a = r;
    *b = z;
}

__device__ __forceinline__ float cabs_fma(cfloat v)  // complex.h.cl:28-30
{
    return __fsqrt_rn(fmaf(v.re, v.re, mul(v.im, v.im)));
}

// Complex Givens rotation (Crotg_naive.cl).
__global__ void crotg_kernel(cfloat* a, cfloat* b, float* c, cfloat* s)
{
    const cfloat av = *a, bv = *b;
    const float fa = cabs_fma(av), fb = cabs_fma(bv);
    if (fa == 0.f) {
        *c = 0.f;
        *s = cfloat{1.f, 0.f};
        *a = bv;
        return;
    }
    const float scale = __fadd_rn(fa, fb);
    const float da = cabs_fma(cfloat{__fdiv_rn(av.re, scale), __fdiv_rn(av.im, scale)});
    const float db = cabs_fma(cfloat{__fdiv_rn(bv.re, scale), __fdiv_rn(bv.im, scale)});
    const float norm = mul(scale, __fsqrt_rn(__fadd_rn(mul(da, da), mul(db, db))));
    const cfloat alpha{__fdiv_rn(av.re, fa), __fdiv_rn(av.im, fa)};
    *c = __fdiv_rn(fa, norm);
    const cfloat t = cmul(cfloat{bv.re, -bv.im}, alpha);
    *s = cfloat{__fdiv_rn(t.re, norm), __fdiv_rn(t.im, norm)};
    *a = cfloat{mul(alpha.re, norm), mul(alpha.im, norm)};
}

// Modified Givens generator: the reference's host-side checks
// (iclBLAS_S.cpp:101-128) followed by its kernel (Srotmg_naive.cl).  The
// rescaling loops stop after kMaxRescale steps: finite values need at most
// 12 (24 bits of exponent per step), and an infinite d1 or d2 -- on which the
// reference's loop never ends -- is left unscaled.
constexpr int kMaxRescale = 16;

__global__ void srotmg_kernel(float* d1, float* d2, float* x1, const float* y1, float* param)
{
    float dd1 = *d1, dd2 = *d2, bb1 = *x1;
    const float bb2 = *y1;
    if (dd1 < 0.f) {
        param[0] = -1.f;
        param[1] = param[2] = param[3] = param[4] = 0.f;
        return;
    }
    if (dd2 == 0.f || bb2 == 0.f) {
        param[0] = -2.f;
        return;
    }
    if (mul(mul(-dd2, bb2), bb2) >= mul(mul(dd1, bb1), bb1)) {
        param[0] = -1.f;
        param[1] = param[2] = param[3] = param[4] = 0.f;
        return;
    }
    const float p1 = mul(dd1, bb1), p2 = mul(dd2, bb2);
    const float q1 = mul(p1, bb1), q2 = mul(p2, bb2);
    float h11 = 0.f, h12 = 0.f, h21 = 0.f, h22 = 0.f, flag;
    if (q1 > fabsf(q2)) {
        h12 = __fdiv_rn(p2, p1);
        h21 = __fdiv_rn(-bb2, bb1);
        const float u = __fsub_rn(1.f, mul(h12, h21));
        flag = 0.f;
        if (u > 0.f) {
            dd1 = __fdiv_rn(dd1, u);
            dd2 = __fdiv_rn(dd2, u);
            bb1 = mul(bb1, u);
        }
    } else {
        h11 = __fdiv_rn(p1, p2);
        h22 = __fdiv_rn(bb1, bb2);
        const float u = __fadd_rn(1.f, mul(h11, h22));
        const float v = __fdiv_rn(dd1, u);
        flag = 1.f;
        dd1 = __fdiv_rn(dd2, u);
        dd2 = v;
        bb1 = mul(bb2, u);
    }
    const float g = 4096.f, gsq = 4096.f * 4096.f, gmsq = 1.f / (4096.f * 4096.f);
    if (dd1 != 0.f && (fabsf(dd1) < gmsq || fabsf(dd1) > gsq)) {
        if (flag == 0.f) {
            h11 = h22 = 1.f;
        } else {
            h12 = 1.f;
            h21 = -1.f;
        }
        flag = -1.f;
        for (int it = 0; it < kMaxRescale && (fabsf(dd1) < gmsq || fabsf(dd1) > gsq); ++it) {
            if (fabsf(dd1) < gmsq) {
                dd1 = mul(dd1, gsq);
                bb1 = __fdiv_rn(bb1, g);
                h11 = __fdiv_rn(h11, g);
                h12 = __fdiv_rn(h12, g);
            } else {
                dd1 = __fdiv_rn(dd1, gsq);
                bb1 = mul(bb1, g);
                h11 = mul(h11, g);
                h12 = mul(h12, g);
            }
        }
    }
    if (dd2 != 0.f && (fabsf(dd2) < gmsq || fabsf(dd2) > gsq)) {
        if (flag == 0.f) {
            h11 = h22 = 1.f;
            flag = -1.f;
        } else if (flag == 1.f) {
            h12 = 1.f;
            h21 = -1.f;
            flag = -1.f;
        }
        for (int it = 0; it < kMaxRescale && (fabsf(dd2) < gmsq || fabsf(dd2) > gsq); ++it) {
            if (fabsf(dd2) < gmsq) {
                dd2 = mul(dd2, gsq);
                h21 = __fdiv_rn(h21, g);
                h22 = __fdiv_rn(h22, g);
            } else {
                dd2 = __fdiv_rn(dd2, gsq);
                h21 = mul(h21, g);
                h22 = mul(h22, g);
            }
        }
    }
    param[0] = flag;
    if (flag == -1.f) {
        param[1] = h11;
        param[2] = h21;
        param[3] = h12;
        param[4] = h22;
    } else if (flag == 0.f) {
        param[2] = h21;
        param[3] = h12;
    } else {
        param[1] = h11;
        param[4] = h22;
    }
    *d1 = dd1;
    *d2 = dd2;
    *x1 = bb1;
}

}  // namespace

// ------------------------------------------------------------------ launchers
cudaError_t scopy(iclblasHandle_t h, int n, const float* x, int incx, float* y, int incy)
{
    return run_pair<float>(h, n, const_cast<float*>(x), incx, y, incy, CopyOp{});
}
cudaError_t ccopy(iclblasHandle_t h, int n, const cfloat* x, int incx, cfloat* y, int incy)
{
    return run_pair<cfloat>(h, n, const_cast<cfloat*>(x), incx, y, incy, CopyOp{});
}
cudaError_t sswap(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy)
{
    return run_pair<float>(h, n, x, incx, y, incy, SwapOp{});
}
cudaError_t cswap(iclblasHandle_t h, int n, cfloat* x, int incx, cfloat* y, int incy)
{
    return run_pair<cfloat>(h, n, x, incx, y, incy, SwapOp{});
}
cudaError_t srot(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy, float c, float s)
{
    return run_pair<float>(h, n, x, incx, y, incy, RotOp{c, s});
}
cudaError_t csrot(iclblasHandle_t h, int n, cfloat* x, int incx, cfloat* y, int incy, float c, float s)
{
    // unit strides: the same per-float map over 2n floats
    if (incx == 1 && incy == 1) return run_pair<float>(h, 2L * n, (float*)x, 1, (float*)y, 1, RotOp{c, s});
    return run_pair<cfloat>(h, n, x, incx, y, incy, RotOp{c, s});
}
cudaError_t crot(iclblasHandle_t h, int n, cfloat* x, int incx, cfloat* y, int incy, float c, cfloat s)
{
    return run_pair<cfloat>(h, n, x, incx, y, incy, CrotOp{c, s});
}
cudaError_t srotm(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy, const float* host_param,
                  const float* dev_param)
{
    RotmOp op{};
    op.dev = dev_param;
    if (host_param)
        for (int k = 0; k < 5; ++k) op.p[k] = host_param[k];
    return run_pair<float>(h, n, x, incx, y, incy, op);
}
cudaError_t srotg(iclblasHandle_t h, float* a, float* b, float* c, float* s)
{
    srotg_kernel<<<1, 1, 0, h->stream>>>(a, b, c, s);
    return cudaGetLastError();
}
cudaError_t crotg(iclblasHandle_t h, cfloat* a, cfloat* b, float* c, cfloat* s)
{
    crotg_kernel<<<1, 1, 0, h->stream>>>(a, b, c, s);
    return cudaGetLastError();
}
cudaError_t srotmg(iclblasHandle_t h, float* d1, float* d2, float* x1, const float* y1, float* param)
{
    srotmg_kernel<<<1, 1, 0, h->stream>>>(d1, d2, x1, y1, param);
    return cudaGetLastError();
}

}  // namespace iclb
