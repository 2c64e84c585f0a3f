// Plain FP32 GEMM on the CUDA cores (the drop-in default math mode):
// C = alpha*op(A)*op(B) + beta*C for float and complex float, every
// combination of op in {N, T, C}, any lda/ldb/ldc.
//
// Arithmetic is the reference's (Sgemm_ntransAB.cl:16-40 and the epilogue of
// gemm_n3_template.h.cl:493-511): each output accumulates its k terms in
// increasing k with fused multiply-adds in FP32, then
// C = fma(alpha, acc, beta*C), or alpha*acc without reading C when beta == 0.
// Because every thread keeps whole outputs and walks k in order, a result is
// bit-identical to the serial oracle for the same inputs.
//
// Structure: register-tiled CTA tiles (BM x BN, BK = 8) staged through
// double-buffered shared memory with register prefetch of the next k tile;
// the global loads are arranged so consecutive threads read consecutive
// addresses for each operand layout (op N vs T/C).
#include <algorithm>
#include <type_traits>

#include "common.cuh"

namespace iclb {
namespace {

__device__ __forceinline__ float conj_if(float v, bool) { return v; }
__device__ __forceinline__ cfloat conj_if(cfloat v, bool c) { return c ? cfloat{v.re, -v.im} : v; }
__device__ __forceinline__ float zero_v(float) { return 0.f; }
__device__ __forceinline__ cfloat zero_v(cfloat) { return cfloat{0.f, 0.f}; }

__device__ __forceinline__ void mac(float& acc, float a, float b) { acc = fmaf(a, b, acc); }
__device__ __forceinline__ void mac(cfloat& acc, cfloat a, cfloat b)
{
    acc.re = fmaf(a.re, b.re, acc.re);
    acc.re = fmaf(-a.im, b.im, acc.re);
    acc.im = fmaf(a.re, b.im, acc.im);
    acc.im = fmaf(a.im, b.re, acc.im);
}

// Two FP32 fused multiply-adds in one instruction (fma.rn.f32x2): each lane
// of the pair is rounded exactly as fmaf, so a result keeps its bits; the
// float kernel issues half as many FMA instructions (it is issue-bound)
__device__ __forceinline__ unsigned long long pack2(float lo, float hi)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float half2f(unsigned long long v, int hi)
{
    float lo_v, hi_v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo_v), "=f"(hi_v) : "l"(v));
    return hi ? hi_v : lo_v;
}
__device__ __forceinline__ void mac2(unsigned long long& acc, unsigned long long a, unsigned long long b)
{
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(a), "l"(b));
}

__host__ __device__ __forceinline__ bool is_zero(float v) { return v == 0.f; }
__host__ __device__ __forceinline__ bool is_zero(cfloat v) { return v.re == 0.f && v.im == 0.f; }

__device__ __forceinline__ float epilogue(float alpha, float acc, float beta, const float* c)
{
    return beta == 0.f ? __fmul_rn(alpha, acc) : fmaf(alpha, acc, __fmul_rn(beta, *c));
}
__device__ __forceinline__ cfloat cmul(cfloat a, cfloat b)
{
    return cfloat{fmaf(a.re, b.re, -a.im * b.im), fmaf(a.re, b.im, a.im * b.re)};
}
__device__ __forceinline__ cfloat epilogue(cfloat alpha, cfloat acc, cfloat beta, const cfloat* c)
{
    cfloat r = cmul(acc, alpha);
    if (beta.re != 0.f || beta.im != 0.f) {
        cfloat t = cmul(*c, beta);
        r.re += t.re;
        r.im += t.im;
    }
    return r;
}

// N consecutive elements from shared memory in 16- or 8-byte vector loads
// (the caller guarantees the alignment).
template <class T, int N>
__device__ __forceinline__ void lds_vec(T* dst, const T* src)
{
    constexpr int bytes = N * (int)sizeof(T);
    if constexpr (bytes == 16) {
        union { float4 v; T t[N]; } u;
        u.v = *reinterpret_cast<const float4*>(src);
#pragma unroll
        for (int i = 0; i < N; ++i) dst[i] = u.t[i];
    } else if constexpr (bytes == 8) {
        union { float2 v; T t[N]; } u;
        u.v = *reinterpret_cast<const float2*>(src);
#pragma unroll
        for (int i = 0; i < N; ++i) dst[i] = u.t[i];
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) dst[i] = src[i];
    }
}

// Threads: (BM/TM) x (BN/TN).  Each thread owns TM x TN outputs split in two
// halves along each dimension (rows ty*TM/2 + {0..TM/2-1} and
// BM/2 + ty*TM/2 + ...) so its shared-memory reads are conflict-free vectors.
template <class T, int BM, int BN, int BK, int TM, int TN>
struct Cfg {
    static constexpr int TX = BN / TN, TY = BM / TM, NT = TX * TY;
    static constexpr int A_PER = BM * BK / NT, B_PER = BN * BK / NT;
    static_assert(A_PER * NT == BM * BK && B_PER * NT == BN * BK, "tile/thread mismatch");
};

template <class T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__(Cfg<T, BM, BN, BK, TM, TN>::NT)
    gemm_simt_kernel(int ta, int tb, int m, int n, int k, T alpha, const T* __restrict__ A, long lda,
                     const T* __restrict__ B, long ldb, T beta, T* __restrict__ C, long ldc, int tri)
{
    using CF = Cfg<T, BM, BN, BK, TM, TN>;
    constexpr int NT = CF::NT, TX = CF::TX;
    // rows padded by 4 elements: the k-contiguous operand's stores (consecutive
    // kk in a warp) fall in different banks, and fragment reads stay aligned
    __shared__ __align__(16) T As[2][BK][BM + 4];
    __shared__ __align__(16) T Bs[2][BK][BN + 4];

    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    // tri 1 / 2: only C's lower (row >= col) / upper triangle is formed;
    // tiles wholly outside it have no work
    if ((tri == 1 && m0 + BM - 1 < n0) || (tri == 2 && m0 > n0 + BN - 1)) return;
    const bool a_trans = ta != ICLBLAS_OP_N, a_conj = ta == ICLBLAS_OP_C;
    const bool b_trans = tb != ICLBLAS_OP_N, b_conj = tb == ICLBLAS_OP_C;

    T ra[CF::A_PER], rb[CF::B_PER];

    // Element e of the A tile (BM x BK): op N reads down columns of A
    // (contiguous in i), op T/C along rows (contiguous in kk).
    auto load_a = [&](int k0) {
#pragma unroll
        for (int q = 0; q < CF::A_PER; ++q) {
            const int e = tid + q * NT;
            int i, kk;
            if (!a_trans) { i = e % BM; kk = e / BM; } else { kk = e % BK; i = e / BK; }
            const int gi = m0 + i, gk = k0 + kk;
            T v = zero_v(T());
            if (gi < m && gk < k) v = a_trans ? conj_if(A[(long)gi * lda + gk], a_conj) : A[(long)gk * lda + gi];
            ra[q] = v;
        }
    };
    auto store_a = [&](int buf) {
#pragma unroll
        for (int q = 0; q < CF::A_PER; ++q) {
            const int e = tid + q * NT;
            int i, kk;
            if (!a_trans) { i = e % BM; kk = e / BM; } else { kk = e % BK; i = e / BK; }
            As[buf][kk][i] = ra[q];
        }
    };
    // Element e of the B tile (BK x BN): op N contiguous in kk, op T/C in j.
    auto load_b = [&](int k0) {
#pragma unroll
        for (int q = 0; q < CF::B_PER; ++q) {
            const int e = tid + q * NT;
            int j, kk;
            if (!b_trans) { kk = e % BK; j = e / BK; } else { j = e % BN; kk = e / BN; }
            const int gj = n0 + j, gk = k0 + kk;
            T v = zero_v(T());
            if (gj < n && gk < k) v = b_trans ? conj_if(B[(long)gk * ldb + gj], b_conj) : B[(long)gj * ldb + gk];
            rb[q] = v;
        }
    };
    auto store_b = [&](int buf) {
#pragma unroll
        for (int q = 0; q < CF::B_PER; ++q) {
            const int e = tid + q * NT;
            int j, kk;
            if (!b_trans) { kk = e % BK; j = e / BK; } else { j = e % BN; kk = e / BN; }
            Bs[buf][kk][j] = rb[q];
        }
    };

    // float: accumulators in pairs along j (acc[i][2j], acc[i][2j+1])
    constexpr bool kPair = std::is_same<T, float>::value && TN % 2 == 0;
    using AccT = std::conditional_t<kPair, unsigned long long, T>;
    constexpr int TNA = kPair ? TN / 2 : TN;
    AccT acc[TM][TNA];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TNA; ++j) {
            if constexpr (kPair) acc[i][j] = 0ull;  // (+0.f, +0.f)
            else acc[i][j] = zero_v(T());
        }
    auto acc_at = [&](int i, int j) -> T {
        if constexpr (kPair) return half2f(acc[i][j >> 1], j & 1);
        else return acc[i][j];
    };

    const int ktiles = (k + BK - 1) / BK;
    if (ktiles > 0) {
        load_a(0);
        load_b(0);
        store_a(0);
        store_b(0);
    }
    __syncthreads();
    for (int t = 0; t < ktiles; ++t) {
        const int buf = t & 1;
        if (t + 1 < ktiles) {
            load_a((t + 1) * BK);
            load_b((t + 1) * BK);
        }
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T a[TM], b[TN];
            lds_vec<T, TM / 2>(a, &As[buf][kk][ty * (TM / 2)]);
            lds_vec<T, TM / 2>(a + TM / 2, &As[buf][kk][BM / 2 + ty * (TM / 2)]);
            lds_vec<T, TN / 2>(b, &Bs[buf][kk][tx * (TN / 2)]);
            lds_vec<T, TN / 2>(b + TN / 2, &Bs[buf][kk][BN / 2 + tx * (TN / 2)]);
            if constexpr (kPair) {
                unsigned long long bp[TN / 2];
#pragma unroll
                for (int j = 0; j < TN / 2; ++j) bp[j] = pack2(b[2 * j], b[2 * j + 1]);
#pragma unroll
                for (int i = 0; i < TM; ++i) {
                    const unsigned long long ap = pack2(a[i], a[i]);
#pragma unroll
                    for (int j = 0; j < TN / 2; ++j) mac2(acc[i][j], ap, bp[j]);
                }
            } else {
#pragma unroll
                for (int i = 0; i < TM; ++i)
#pragma unroll
                    for (int j = 0; j < TN; ++j) mac(acc[i][j], a[i], b[j]);
            }
        }
        if (t + 1 < ktiles) {
            store_a(buf ^ 1);
            store_b(buf ^ 1);
        }
        __syncthreads();
    }

    // the row's C values are all loaded before any is stored, so the loads
    // overlap (C is read only when beta != 0)
    const bool read_c = !is_zero(beta);
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int gi = m0 + (i < TM / 2 ? ty * (TM / 2) + i : BM / 2 + ty * (TM / 2) + (i - TM / 2));
        if (gi >= m) continue;
        T cv[TN];
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int gj = n0 + (j < TN / 2 ? tx * (TN / 2) + j : BN / 2 + tx * (TN / 2) + (j - TN / 2));
            const bool in = tri == 0 || (tri == 1 ? gi >= gj : gi <= gj);
            cv[j] = (read_c && gj < n && in) ? C[(long)gj * ldc + gi] : zero_v(T());
        }
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int gj = n0 + (j < TN / 2 ? tx * (TN / 2) + j : BN / 2 + tx * (TN / 2) + (j - TN / 2));
            if (gj >= n) continue;
            if (tri != 0 && (tri == 1 ? gi < gj : gi > gj)) continue;
            C[(long)gj * ldc + gi] = epilogue(alpha, acc_at(i, j), beta, &cv[j]);
        }
    }
}

template <class T, int BM, int BN, int BK, int TM, int TN>
cudaError_t launch(iclblasHandle_t h, int ta, int tb, int m, int n, int k, T alpha, const T* A, int lda, const T* B,
                   int ldb, T beta, T* C, int ldc, int tri)
{
    using CF = Cfg<T, BM, BN, BK, TM, TN>;
    dim3 grid(ceil_div(m, BM), ceil_div(n, BN));
    gemm_simt_kernel<T, BM, BN, BK, TM, TN><<<grid, CF::NT, 0, h->stream>>>(ta, tb, m, n, k, alpha, A, lda, B, ldb,
                                                                            beta, C, ldc, tri);
    return cudaGetLastError();
}

}  // namespace

cudaError_t sgemm_simt(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const float* A, int lda,
                       const float* B, int ldb, float beta, float* C, int ldc, int tri)
{
    // the largest tile that still gives every SM a CTA: 128 x 128 (256
    // threads, 8 x 8 outputs each), 64 x 64 (256 threads, 4 x 4), or for small
    // products 32 x 32 (64 threads, 4 x 4; config 1's 512^3 has 16 tiles of
    // 128 x 128 and 64 of 64 x 64)
    auto tiles = [&](int t) {
        long c = (long)ceil_div(m, t) * ceil_div(n, t);
        if (tri != 0) c = (c + std::min(ceil_div(m, t), ceil_div(n, t))) / 2;
        return c;
    };
    if (tiles(128) >= h->sm_count)
        return launch<float, 128, 128, 16, 8, 8>(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri);
    if (tiles(64) >= h->sm_count)
        return launch<float, 64, 64, 8, 4, 4>(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri);
    return launch<float, 32, 32, 8, 4, 4>(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri);
}

cudaError_t cgemm_simt(iclblasHandle_t h, int ta, int tb, int m, int n, int k, cfloat alpha, const cfloat* A, int lda,
                       const cfloat* B, int ldb, cfloat beta, cfloat* C, int ldc)
{
    const long big_tiles = (long)ceil_div(m, 64) * ceil_div(n, 64);
    if (big_tiles >= h->sm_count)
        return launch<cfloat, 64, 64, 8, 4, 4>(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 0);
    return launch<cfloat, 32, 32, 8, 2, 2>(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 0);
}

}  // namespace iclb
