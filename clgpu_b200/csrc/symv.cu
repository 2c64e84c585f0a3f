// Symmetric / Hermitian matrix-vector products: Ssymv (y = alpha A x + beta y,
// A symmetric) and Chemv (A Hermitian), one triangle of A stored.
//
// HBM-bound on the stored triangle (n(n+1)/2 elements).  Each stored element
// contributes twice -- A(i,j) x_j to y_i and A(i,j) x_i (conjugated for
// Chemv) to y_j -- so the triangle is read once and both contributions are
// formed from registers.  The triangle is cut into TS x TS tiles (TS = 128
// single, 64 complex: 32 lanes x one 16-byte word of rows); one CTA per
// stored tile (I, J):
//   - lane l owns rows [l*per, l*per + per) of the tile, warp w of W the
//     columns w, w+W, ...; A is read in 16-byte words down each column;
//   - row contributions sum in registers across the warp's columns and then
//     across the warps (shared memory);
//   - column contributions sum over the word in registers and over the 32
//     lanes of the column (shuffle tree);
//   - diagonal tiles read only the stored triangle (elements outside it are
//     selected away, never multiplied) and count the diagonal once; Chemv
//     takes the diagonal's real part.
// Tile (I, J) writes its row partial to Q[J][I*TS..] and its column partial
// to Q[I][J*TS..] (a diagonal tile writes their sum to Q[I][I*TS..]), so
// every Q entry is written exactly once and no memset is needed.  A second
// kernel forms y_i = alpha * sum_t Q[t][i] + beta y_i with the sum in FP64 in
// fixed order (deterministic).  Q adds 2 * n * ceil(n/TS) * sizeof(T) bytes
// of traffic: 3 % of the triangle's bytes for single, 6 % for complex.
//
// beta == 0: y is written without being read (the BLAS convention; the
// reference's Chemv_naive.cl:46 always reads it).
#include <algorithm>

#include "common.cuh"

namespace iclb {
namespace {


bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

__device__ __forceinline__ float zero_t(float) { return 0.f; }
__device__ __forceinline__ cfloat zero_t(cfloat) { return cfloat{0.f, 0.f}; }
__device__ __forceinline__ float conj_t(float v) { return v; }
__device__ __forceinline__ cfloat conj_t(cfloat v) { return cfloat{v.re, -v.im}; }
__device__ __forceinline__ float real_part(float v) { return v; }
__device__ __forceinline__ cfloat real_part(cfloat v) { return cfloat{v.re, 0.f}; }
__device__ __forceinline__ void mac(float& acc, float a, float b) { acc = fmaf(a, b, acc); }
__device__ __forceinline__ void mac(cfloat& acc, cfloat a, cfloat b)
{
    acc.re = fmaf(a.re, b.re, acc.re);
    acc.re = fmaf(-a.im, b.im, acc.re);
    acc.im = fmaf(a.re, b.im, acc.im);
    acc.im = fmaf(a.im, b.re, acc.im);
}
__device__ __forceinline__ float add_t(float a, float b) { return a + b; }
__device__ __forceinline__ cfloat add_t(cfloat a, cfloat b) { return cfloat{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ float shfl_xor_t(float v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
__device__ __forceinline__ cfloat shfl_xor_t(cfloat v, int o)
{
    return cfloat{__shfl_xor_sync(0xffffffffu, v.re, o), __shfl_xor_sync(0xffffffffu, v.im, o)};
}

// Tile geometry.  Single: 128 x 128 tiles, 16 warps of 8 columns (512
// threads, 64 registers: two CTAs and 32 warps per SM; 8 warps of 16 columns
// ran at 0.80 of HBM peak instead of 0.84).  Complex: 64 x 64 tiles, 8 warps
// of 8 columns (16 warps of 4 ran at 0.48 instead of 0.61).
template <class T>
struct Tile {
    static constexpr int per = (int)(16 / sizeof(T));  // elements per 16-byte word
    static constexpr int TS = 32 * per;                // tile rows = tile columns
    static constexpr int THREADS = sizeof(T) == 4 ? 512 : 256;
    static constexpr int WARPS = THREADS / 32;
    static constexpr int PASSES = TS / WARPS;          // columns per warp
    static constexpr int MIN_CTAS = sizeof(T) == 4 ? 2 : 5;  // resident CTAs per SM the registers allow
};

// Stored tile number t -> (I, J) with I >= J (row-major over the lower block
// triangle).  Upper storage uses the transposed pair.
__device__ __forceinline__ void tile_of(long t, int& I, int& J)
{
    long i = (long)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((i + 1) * (i + 2) / 2 <= t) ++i;
    while (i * (i + 1) / 2 > t) --i;
    I = (int)i;
    J = (int)(t - i * (i + 1) / 2);
}

// Row and column products of one thread's words of a tile: racc[k] +=
// A(r, c) x_c over the thread's columns, csum[p] = sum_k A(r, c) x_r (or
// conj(A) for HERM).  DIAG: the tile is on the diagonal; only the stored
// triangle counts and the diagonal counts once, as a row term.
template <class T, bool LOWER, bool HERM, bool DIAG>
__device__ __forceinline__ void tile_products(const T (&a)[Tile<T>::PASSES][Tile<T>::per], T (&racc)[Tile<T>::per],
                                              T (&csum)[Tile<T>::PASSES], const T (&xw)[Tile<T>::per], const T* xc,
                                              int w, long r0, long col0)
{
    constexpr int per = Tile<T>::per;
#pragma unroll
    for (int p = 0; p < Tile<T>::PASSES; ++p) {
        const int cl = w + p * Tile<T>::WARPS;
        const T xcv = xc[cl];
        T cs = zero_t(T());
#pragma unroll
        for (int k = 0; k < per; ++k) {
            T v = a[p][k];
            if (DIAG) {
                const long r = r0 + k, c = col0 + cl;
                if (r == c && HERM) v = real_part(v);
                if (LOWER ? (r >= c) : (r <= c)) mac(racc[k], v, xcv);
                if (LOWER ? (r > c) : (r < c)) mac(cs, HERM ? conj_t(v) : v, xw[k]);
            } else {
                mac(racc[k], v, xcv);
                mac(cs, HERM ? conj_t(v) : v, xw[k]);
            }
        }
        csum[p] = cs;
    }
}

template <class T, bool LOWER, bool HERM, bool VEC>
__global__ void __launch_bounds__(Tile<T>::THREADS, Tile<T>::MIN_CTAS) symv_tile_kernel(int n, int nb, const T* __restrict__ A, long lda,
                                                                 const T* __restrict__ x, long incx,
                                                                 T* __restrict__ Q, long qld)
{
    using TL = Tile<T>;
    constexpr int per = TL::per, TS = TL::TS;
    __shared__ T xr[TS];              // x over the tile's rows
    __shared__ T xc[TS];              // x over the tile's columns
    __shared__ T red[TL::WARPS][TS + 1]; // row partials per warp
    __shared__ T colp[TS];

    // Consecutive CTAs take consecutive tiles of one block column (adjacent
    // rows of the same columns: DRAM pages stay open): for upper storage the
    // row-major lower enumeration transposed, for lower storage the same
    // enumeration mirrored through the anti-diagonal.
    // the finishing kernel (launched as a programmatic dependent) may be
    // scheduled once every tile CTA has started; it waits for this grid's
    // completion before reading Q
    asm volatile("griddepcontrol.launch_dependents;");
    int I, J;
    tile_of(blockIdx.x, I, J);
    if (LOWER) {
        const int a = I, b = J;
        I = nb - 1 - b;
        J = nb - 1 - a;
    } else {
        const int t = I;
        I = J;
        J = t;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long row0 = (long)I * TS, col0 = (long)J * TS;
    const bool diag = (I == J);
    const long r0 = row0 + (long)lane * per;  // first row of this lane's word
    const bool full_word = r0 + per <= n;

    // Every word this thread reads is requested before anything else, so a
    // CTA keeps its whole 64 KB (single) / 32 KB (complex) tile in flight.
    T a[TL::PASSES][per];
    if (VEC && row0 + TS <= n && col0 + TS <= n) {
        // interior tile: every word is whole and in range, no conditions
        const T* src = A + (col0 + w) * lda + r0;
        float4 v[TL::PASSES];
#pragma unroll
        for (int p = 0; p < TL::PASSES; ++p) v[p] = ld_stream4((const float4*)(src + (long)p * TL::WARPS * lda));
#pragma unroll
        for (int p = 0; p < TL::PASSES; ++p) {
            const T* e = (const T*)&v[p];
#pragma unroll
            for (int k = 0; k < per; ++k) a[p][k] = e[k];
        }
    } else {
#pragma unroll
    for (int p = 0; p < TL::PASSES; ++p) {
        const long c = col0 + w + (long)p * TL::WARPS;
        if (c < n && r0 < n) {
            const T* src = A + c * lda + r0;
            if (VEC && full_word) {
                float4 v = ld_stream4((const float4*)src);
                const T* e = (const T*)&v;
#pragma unroll
                for (int k = 0; k < per; ++k) a[p][k] = e[k];
            } else {
#pragma unroll
                for (int k = 0; k < per; ++k) a[p][k] = (r0 + k < n) ? src[k] : zero_t(T());
            }
        } else {
#pragma unroll
            for (int k = 0; k < per; ++k) a[p][k] = zero_t(T());
        }
    }
    }
    for (int k = threadIdx.x; k < TS; k += TL::THREADS) {
        xr[k] = (row0 + k < n) ? x[(row0 + k) * incx] : zero_t(T());
        xc[k] = (col0 + k < n) ? x[(col0 + k) * incx] : zero_t(T());
    }
    __syncthreads();

    T racc[per];
    T xw[per];
#pragma unroll
    for (int k = 0; k < per; ++k) {
        racc[k] = zero_t(T());
        xw[k] = xr[lane * per + k];
    }
    T csum[TL::PASSES];
    if (diag)
        tile_products<T, LOWER, HERM, true>(a, racc, csum, xw, xc, w, r0, col0);
    else
        tile_products<T, LOWER, HERM, false>(a, racc, csum, xw, xc, w, r0, col0);
    // column sums over the 32 lanes, all PASSES columns at once: each step
    // halves the values a lane carries (PASSES - 1 shuffles instead of
    // 5 * PASSES), the last steps reduce the one value left
    int bit = 16;
#pragma unroll
    for (int hcount = TL::PASSES / 2; hcount >= 1; hcount /= 2) {
        const bool up = (lane & bit) != 0;
#pragma unroll
        for (int i = 0; i < hcount; ++i) {
            const T send = up ? csum[i] : csum[i + hcount];
            const T keep = up ? csum[i + hcount] : csum[i];
            csum[i] = add_t(keep, shfl_xor_t(send, bit));
        }
        bit >>= 1;
    }
    for (int b = bit; b >= 1; b >>= 1) csum[0] = add_t(csum[0], shfl_xor_t(csum[0], b));
    // lane bits above `bit` name the column this lane's sum belongs to
    if ((lane & (2 * bit - 1)) == 0) {
        int pcol = 0;
#pragma unroll
        for (int b = 16, v = TL::PASSES / 2; v >= 1; b >>= 1, v >>= 1)
            if (lane & b) pcol += v;
        colp[w + pcol * TL::WARPS] = csum[0];
    }
#pragma unroll
    for (int k = 0; k < per; ++k) red[w][lane * per + k] = racc[k];
    __syncthreads();
    for (int k = threadIdx.x; k < TS; k += TL::THREADS) {
        T s = red[0][k];
#pragma unroll
        for (int ww = 1; ww < TL::WARPS; ++ww) s = add_t(s, red[ww][k]);
        if (diag) {
            Q[(long)I * qld + row0 + k] = add_t(s, colp[k]);
        } else {
            Q[(long)J * qld + row0 + k] = s;         // to y over the tile's rows
            Q[(long)I * qld + col0 + k] = colp[k];   // to y over the tile's columns
        }
    }
}

__device__ __forceinline__ void acc_d(double& re, double& im, float v)
{
    re += (double)v;
    (void)im;
}
__device__ __forceinline__ void acc_d(double& re, double& im, cfloat v)
{
    re += (double)v.re;
    im += (double)v.im;
}

// y_i = alpha * sum_t Q[t][i] + beta * y_i, the reference's final expressions
// (Ssymv_naive_lower.cl:34-37, Chemv_naive.cl:45-46) on the FP64 sum rounded
// to T.  The sum runs in a fixed order: kFinChunks contiguous runs of t, each
// summed in order by one thread, then the runs in order.  A CTA takes 32
// rows (a warp per run, consecutive rows in its lanes); one thread per row
// summing all nb partials in sequence left 32 CTAs waiting on their loads
// (10-15 us of a 65-100 us call).
constexpr int kFinChunks = 8;
constexpr int kFinThreads = 32 * kFinChunks;

template <class T>
__device__ __forceinline__ void finish_sums(int n, int nb, const T* __restrict__ Q, long qld, long i, double& re,
                                            double& im)
{
    __shared__ double sre[kFinChunks][32], sim[kFinChunks][32];
    // the tile kernel's partials are complete and visible after this wait
    // (a no-op when the launch was not a programmatic dependent)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
    const int t0 = (int)((long)nb * c / kFinChunks), t1 = (int)((long)nb * (c + 1) / kFinChunks);
    double r = 0.0, m = 0.0;
    if (i < n)
        for (int t = t0; t < t1; ++t) acc_d(r, m, Q[(long)t * qld + i]);
    sre[c][lane] = r;
    sim[c][lane] = m;
    __syncthreads();
    re = 0.0;
    im = 0.0;
#pragma unroll
    for (int cc = 0; cc < kFinChunks; ++cc) {
        re += sre[cc][lane];
        im += sim[cc][lane];
    }
}

__global__ void __launch_bounds__(kFinThreads) symv_finish_kernel(int n, int nb, const float* __restrict__ Q,
                                                                  long qld, float alpha, float beta, float* y,
                                                                  long incy)
{
    const long i = (long)blockIdx.x * 32 + (threadIdx.x & 31);
    double s, unused;
    finish_sums(n, nb, Q, qld, i, s, unused);
    if (threadIdx.x >= 32 || i >= n) return;
    const float r = (float)s;
    float* yp = y + i * incy;
    *yp = (beta != 0.f) ? fmaf(alpha, r, __fmul_rn(beta, *yp)) : __fmul_rn(alpha, r);
}

__global__ void __launch_bounds__(kFinThreads) hemv_finish_kernel(int n, int nb, const cfloat* __restrict__ Q,
                                                                  long qld, cfloat alpha, cfloat beta, cfloat* y,
                                                                  long incy)
{
    const long i = (long)blockIdx.x * 32 + (threadIdx.x & 31);
    double re, im;
    finish_sums(n, nb, Q, qld, i, re, im);
    if (threadIdx.x >= 32 || i >= n) return;
    const cfloat r = cmul_fma(cfloat{(float)re, (float)im}, alpha);
    cfloat* yp = y + i * incy;
    if (beta.re != 0.f || beta.im != 0.f) {
        const cfloat b = cmul_fma(beta, *yp);
        *yp = cfloat{__fadd_rn(b.re, r.re), __fadd_rn(b.im, r.im)};
    } else {
        *yp = r;
    }
}

// launches `kernel` on the handle's stream as a programmatic dependent of the
// kernel before it (its CTAs may be scheduled during that kernel's last wave)
template <class K, class... Args>
cudaError_t launch_dependent(iclblasHandle_t h, K kernel, unsigned grid, unsigned threads, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.stream = h->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <class T, bool HERM>
cudaError_t symv_tiles(iclblasHandle_t h, bool lower, int n, const T* A, int lda, const T* x, int incx, T* Q,
                       long qld, int nb)
{
    const long tiles = (long)nb * (nb + 1) / 2;
    const bool vec = aligned16(A) && lda % Tile<T>::per == 0;
    const unsigned grid = (unsigned)tiles;
#define SYMV_LAUNCH(L, V) \
    symv_tile_kernel<T, L, HERM, V><<<grid, Tile<T>::THREADS, 0, h->stream>>>(n, nb, A, lda, x, incx, Q, qld)
    if (lower) {
        if (vec) SYMV_LAUNCH(true, true); else SYMV_LAUNCH(true, false);
    } else {
        if (vec) SYMV_LAUNCH(false, true); else SYMV_LAUNCH(false, false);
    }
#undef SYMV_LAUNCH
    return cudaGetLastError();
}

}  // namespace

cudaError_t ssymv(iclblasHandle_t h, int uplo, int n, float alpha, const float* A, int lda, const float* x, int incx,
                  float beta, float* y, int incy)
{
    constexpr int TS = Tile<float>::TS;
    const int nb = (n + TS - 1) / TS;
    const long qld = (long)nb * TS;
    float* Q = (float*)scratch(h, sizeof(float) * (size_t)nb * (size_t)qld);
    if (!Q) return cudaErrorMemoryAllocation;
    cudaError_t e = symv_tiles<float, false>(h, uplo == ICLBLAS_FILL_MODE_LOWER, n, A, lda, x, incx, Q, qld, nb);
    if (e != cudaSuccess) return e;
    e = launch_dependent(h, symv_finish_kernel, (unsigned)((n + 31) / 32), (unsigned)kFinThreads, n, nb,
                         (const float*)Q, qld, alpha, beta, y, (long)incy);
    return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t chemv(iclblasHandle_t h, int uplo, int n, cfloat alpha, const cfloat* A, int lda, const cfloat* x,
                  int incx, cfloat beta, cfloat* y, int incy)
{
    constexpr int TS = Tile<cfloat>::TS;
    const int nb = (n + TS - 1) / TS;
    const long qld = (long)nb * TS;
    cfloat* Q = (cfloat*)scratch(h, sizeof(cfloat) * (size_t)nb * (size_t)qld);
    if (!Q) return cudaErrorMemoryAllocation;
    cudaError_t e = symv_tiles<cfloat, true>(h, uplo == ICLBLAS_FILL_MODE_LOWER, n, A, lda, x, incx, Q, qld, nb);
    if (e != cudaSuccess) return e;
    e = launch_dependent(h, hemv_finish_kernel, (unsigned)((n + 31) / 32), (unsigned)kFinThreads, n, nb,
                         (const cfloat*)Q, qld, alpha, beta, y, (long)incy);
    return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace iclb
