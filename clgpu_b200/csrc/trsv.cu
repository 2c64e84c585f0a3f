// TRSV: solve op(A) x = b in place (x holds b on entry), float and complex,
// op in {N, T, C}, upper/lower, unit/non-unit.
//
// Replaces Strsv_simd16x16_* (one work-group of 256 serialising every
// 16-column block with barriers) and the serial Strsv_naive / Ctrsv_naive
// (libs/blas/funcs/Strsv/*, Ctrsv/*).  One launch covers the whole solve:
//   - the n rows are cut into blocks of NB = 64; each CTA draws a ticket s
//     from an atomic counter and owns block s of the solve order (forward for
//     a lower op(A), backward for an upper one).  Tickets are handed out in
//     start order, so a CTA only ever waits for CTAs that are already running:
//     no deadlock however many CTAs fit on the GPU at once;
//   - CTA s streams the tiles op(A)[blk s, blk j] for j < s (register
//     prefetch of the next tile while it works on the current one), and for
//     each waits until block j's solution is published (flag j == this call's
//     epoch), then subtracts the tile times x_j;
//   - it then solves its 64x64 diagonal block by substitution in shared
//     memory, writes x_s, fences, and publishes flag s.
// Every wait is bounded: after kSpinLimit polls the CTA records
// kDevWaitTimeout in the device status word and every other CTA, which also
// polls that word, returns; the host reports EXECUTION_FAILED.  Reads of
// other CTAs' results go through L2 (ld.cg) so no stale L1 line is used.
#include "common.cuh"

namespace iclb {
namespace {

constexpr int NB = 64;
constexpr int kThreads = 256;
constexpr long kSpinLimit = 1L << 22;

__device__ __forceinline__ float zero_v(float) { return 0.f; }
__device__ __forceinline__ cfloat zero_v(cfloat) { return cfloat{0.f, 0.f}; }
__device__ __forceinline__ float conj_v(float v) { return v; }
__device__ __forceinline__ cfloat conj_v(cfloat v) { return cfloat{v.re, -v.im}; }
__device__ __forceinline__ float ldcg(const float* p) { return __ldcg(p); }
__device__ __forceinline__ cfloat ldcg(const cfloat* p)
{
    float2 v = __ldcg((const float2*)p);
    return cfloat{v.x, v.y};
}
__device__ __forceinline__ float ldg(const float* p) { return __ldg(p); }
__device__ __forceinline__ cfloat ldg(const cfloat* p)
{
    float2 v = __ldg((const float2*)p);
    return cfloat{v.x, v.y};
}
__device__ __forceinline__ void msub(float& acc, float a, float x) { acc = fmaf(-a, x, acc); }
__device__ __forceinline__ void msub(cfloat& acc, cfloat a, cfloat x)
{
    acc.re = fmaf(-a.re, x.re, acc.re);
    acc.re = fmaf(a.im, x.im, acc.re);
    acc.im = fmaf(-a.re, x.im, acc.im);
    acc.im = fmaf(-a.im, x.re, acc.im);
}
__device__ __forceinline__ float addv(float a, float b) { return a + b; }
__device__ __forceinline__ cfloat addv(cfloat a, cfloat b) { return cfloat{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ float divv(float a, float d) { return a / d; }
// complex quotient through |d|^2 (the reference's cdiv, core/src/ocl/complex.h.cl:36)
__device__ __forceinline__ cfloat divv(cfloat a, cfloat d)
{
    float q = fmaf(d.re, d.re, d.im * d.im);
    return cfloat{fmaf(a.re, d.re, a.im * d.im) / q, fmaf(a.im, d.re, -a.re * d.im) / q};
}
__device__ __forceinline__ float shfl(float v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ __forceinline__ cfloat shfl(cfloat v, int src)
{
    return cfloat{__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src)};
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile(const int* p) { return *(const volatile int*)p; }

// Thread t of the CTA holds tile elements (r, c) for r = t % NB and
// c = t / NB + 4q, q = 0..15.  op N reads A down columns (consecutive r in a
// warp), op T/C reads along rows of A (consecutive c in a warp: the warp
// covers 32 consecutive r of one 4-column group, each thread loading one
// element; A's rows are then strided, but the tile is small and latency, not
// bandwidth, bounds these steps).
template <class T>
struct Tile {
    T v[16];
};

template <class T>
__device__ __forceinline__ void load_tile(Tile<T>& t, const T* __restrict__ A, long lda, int op, int r0, int nr,
                                          int c0, int nc)
{
    const int r = threadIdx.x % NB, cb = threadIdx.x / NB;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int c = cb + 4 * q;
        T val = zero_v(T());
        if (r < nr && c < nc) {
            // element (r, c) of op(A) restricted to the tile
            if (op == 0) val = ldg(A + (long)(c0 + c) * lda + (r0 + r));
            else {
                val = ldg(A + (long)(r0 + r) * lda + (c0 + c));
                if (op == 2) val = conj_v(val);
            }
        }
        t.v[q] = val;
    }
}

template <class T>
__global__ void __launch_bounds__(kThreads) trsv_kernel(int n, int lower_op, int op, int unit, const T* __restrict__ A,
                                                        long lda, T* x, long incx, unsigned* ticket, unsigned* flags,
                                                        unsigned epoch, int* status)
{
    __shared__ T tile[NB][NB + 1];
    __shared__ T xs[NB];
    __shared__ T part[4][NB];
    __shared__ unsigned s_sh;
    __shared__ int abort_sh;

    const int nb = (n + NB - 1) / NB;
    if (threadIdx.x == 0) s_sh = atomicAdd(ticket, 1u);
    __syncthreads();
    const int s = (int)s_sh;
    if (s == nb - 1 && threadIdx.x == 0) *ticket = 0u;  // every ticket of this launch is taken

    // block index in row space for solve-order position p
    auto blk = [&](int p) { return lower_op ? p : nb - 1 - p; };
    const int rb = blk(s);
    const int r0 = rb * NB, nr = min(NB, n - r0);
    const int r = threadIdx.x % NB, cb = threadIdx.x / NB;

    T acc = zero_v(T());  // partial sum of op(A)[r, cols of cb group] * x
    Tile<T> cur;
    {
        const int jb = s > 0 ? blk(0) : rb;
        load_tile(cur, A, lda, op, r0, nr, jb * NB, min(NB, n - jb * NB));
    }
    for (int p = 0; p <= s; ++p) {
        const int jb = blk(p);
        const int c0 = jb * NB, nc = min(NB, n - c0);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 16; ++q) tile[r][cb + 4 * q] = cur.v[q];
        if (p < s) {
            const int nj = blk(p + 1);
            load_tile(cur, A, lda, op, r0, nr, nj * NB, min(NB, n - nj * NB));
        }
        if (p == s) break;  // diagonal tile is in shared memory
        // wait for block p of the solve order
        if (threadIdx.x == 0) {
            int ab = 0;
            long it = 0;
            while (ld_acquire(flags + p) != epoch) {
                if (ld_volatile(status) != kDevOk) { ab = 1; break; }
                if (++it > kSpinLimit) {
                    atomicOr(status, (int)kDevWaitTimeout);
                    ab = 1;
                    break;
                }
                __nanosleep(64);
            }
            abort_sh = ab;
        }
        __syncthreads();
        if (abort_sh) return;
        if (threadIdx.x < nc) xs[threadIdx.x] = ldcg(x + (long)(c0 + threadIdx.x) * incx);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int c = cb + 4 * q;
            if (c < nc) msub(acc, tile[r][c], xs[c]);
        }
    }
    // combine the 4 column-group partials with b, then solve the diagonal block
    part[cb][r] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        // each lane owns rows lane and lane + 32
        T b0 = zero_v(T()), b1 = zero_v(T());
        if (lane < nr) b0 = addv(addv(x[(long)(r0 + lane) * incx], addv(part[0][lane], part[1][lane])),
                                addv(part[2][lane], part[3][lane]));
        if (lane + 32 < nr)
            b1 = addv(addv(x[(long)(r0 + lane + 32) * incx], addv(part[0][lane + 32], part[1][lane + 32])),
                      addv(part[2][lane + 32], part[3][lane + 32]));
        if (lower_op) {
            for (int k = 0; k < nr; ++k) {
                const int owner = k & 31;
                T bk = (k < 32) ? shfl(b0, owner) : shfl(b1, owner);
                if (!unit) bk = divv(bk, tile[k][k]);
                if (lane == owner) { if (k < 32) b0 = bk; else b1 = bk; }
                if (lane > k && lane < nr) msub(b0, tile[lane][k], bk);
                if (lane + 32 > k && lane + 32 < nr) msub(b1, tile[lane + 32][k], bk);
            }
        } else {
            for (int k = nr - 1; k >= 0; --k) {
                const int owner = k & 31;
                T bk = (k < 32) ? shfl(b0, owner) : shfl(b1, owner);
                if (!unit) bk = divv(bk, tile[k][k]);
                if (lane == owner) { if (k < 32) b0 = bk; else b1 = bk; }
                if (lane < k) msub(b0, tile[lane][k], bk);
                if (lane + 32 < k) msub(b1, tile[lane + 32][k], bk);
            }
        }
        if (lane < nr) x[(long)(r0 + lane) * incx] = b0;
        if (lane + 32 < nr) x[(long)(r0 + lane + 32) * incx] = b1;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) st_release(flags + s, epoch);
}

template <class T>
cudaError_t trsv_impl(iclblasHandle_t h, int uplo, int trans, int diag, int n, const T* A, int lda, T* x, int incx)
{
    const int nb = (n + NB - 1) / NB;
    constexpr int kFlagBase = kCounterWords / 2;
    if (nb > kCounterWords / 2 - 1) return cudaErrorInvalidValue;
    const int op = trans;  // 0 N, 1 T, 2 C (C == T for real data)
    const bool lower = uplo == ICLBLAS_FILL_MODE_LOWER;
    const int lower_op = (op == 0) ? lower : !lower;
    unsigned epoch = ++h->ws.epoch;
    if (epoch == 0) epoch = ++h->ws.epoch;
    unsigned* ticket = h->ws.counters;  // zero between launches
    unsigned* flags = h->ws.counters + kFlagBase;
    trsv_kernel<T><<<nb, kThreads, 0, h->stream>>>(n, lower_op, op, diag == ICLBLAS_DIAG_UNIT, A, lda, x, incx,
                                                   ticket, flags, epoch, h->ws.dev_status);
    return cudaGetLastError();
}

}  // namespace

cudaError_t strsv(iclblasHandle_t h, int uplo, int trans, int diag, int n, const float* A, int lda, float* x, int incx)
{
    return trsv_impl<float>(h, uplo, trans == ICLBLAS_OP_C ? ICLBLAS_OP_T : trans, diag, n, A, lda, x, incx);
}

cudaError_t ctrsv(iclblasHandle_t h, int uplo, int trans, int diag, int n, const cfloat* A, int lda, cfloat* x,
                  int incx)
{
    return trsv_impl<cfloat>(h, uplo, trans, diag, n, A, lda, x, incx);
}

}  // namespace iclb
