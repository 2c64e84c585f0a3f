// Uneven batched TRSM and GEMM in one persistent launch each, plus the
// batched TRSM adjoint.  No reference counterpart: the reference has no
// batched routines; these extend its TRSM and GEMM to many independent
// instances of different sizes.
//
// A plan holds, in device memory, each instance's sizes and a work list of
// (instance, tile) items sorted by decreasing cost (longest first, which
// balances the uneven sizes).  A launch runs (SM count x CTAs per SM)
// persistent CTAs that take items from an atomic queue until it is empty.
//   TRSM item: one instance, RC right-hand sides.  Left-looking blocked solve
//     over 64-row blocks of M = op(A) in solve order: the block's RHS rows
//     (scaled by alpha on load) minus M[blk, earlier] * X[earlier] (a 64 x RC
//     register-tiled product per earlier block, operands staged in shared
//     memory), then substitution on the 64 x 64 diagonal block in shared
//     memory, store.  Left side only.
//   GEMM item: one 64 x RC tile of one instance's C.
// The queue head is cleared with cudaMemsetAsync before each launch, so a
// call is a memset node plus a kernel node and can be captured in a CUDA
// graph (the plan, its work lists and its tuning are built before).
// The tile width RC in {32, 64} and the CTAs per SM in {1, 2, 4} are chosen
// by timing the candidates on synthetic operands of the plan's shapes when
// the plan is created; the choice is cached per (kind, shapes, GPU) in memory
// and, when ICLBLAS_TUNE_CACHE names a file, on disk (one "key rc ctas" line
// each).  This is the plain-FP32 path (FP32 FMA on the CUDA cores); a plan
// created while the handle is in the TF32, 3xBF16 or 6xBF16 mode runs the
// tensor-core path of batched_tc.cu instead (no tuning, no work queue).
#include <atomic>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace iclb {

// The tensor-core path of plans created in the TF32 / 3xBF16 / 6xBF16 math
// modes (batched_tc.cu).
bool batch_tc_mode(iclblasMathMode_t mode);
void batch_tc_free(BatchTc* t);
cudaError_t batch_tc_create_trsm(iclblasHandle_t h, iclblasBatchPlan* plan, const std::vector<int>& dims, int right,
                                 int lower_f, int op_f, int tri_lower, int unit);
cudaError_t batch_tc_create_gemm(iclblasHandle_t h, iclblasBatchPlan* plan, const std::vector<int>& dims, int ta,
                                 int tb);
cudaError_t batch_tc_inverses(iclblasHandle_t h, const iclblasBatchPlan* plan, const float* const* A);
cudaError_t batch_tc_solve(iclblasHandle_t h, const iclblasBatchPlan* plan, int adjoint, float alpha,
                           const float* const* A, float* const* B, int operator_ready);
cudaError_t batch_tc_dA(iclblasHandle_t h, const iclblasBatchPlan* plan, float scale, const float* const* P,
                        const float* const* Q, float* const* dA);
cudaError_t batch_tc_gemm(iclblasHandle_t h, const iclblasBatchPlan* plan, float alpha, const float* const* A,
                          const float* const* B, float beta, float* const* C);

namespace {

constexpr int TB = 64;  // row block / tile height

// ---------------------------------------------------------------- diagonal inverses
// Inverse of every 64 x 64 diagonal block of every instance's M = op(A),
// formed in FP64 and stored in FP32, column-major, 4096 floats per block at
// inv + inv_off[instance] + 4096*block; rows and columns beyond the
// instance's size are the identity.  One CTA of 256 threads per (instance,
// block) item, blocked so that no long dependent chain remains:
//   1. the four 16 x 16 diagonal sub-blocks by substitution (64 threads, one
//      column each);
//   2. doubling to 32 and then to 64: for M = [[P, 0], [C, Q]] (lower)
//      inv = [[P^-1, 0], [-Q^-1 C P^-1, Q^-1]], and for M = [[P, C], [0, Q]]
//      (upper) the off-diagonal block is -P^-1 C Q^-1; each step is two small
//      products spread over all threads.
constexpr int kInvThreads = 256;

// One doubling step for every pair of h x h diagonal blocks of the 64 x 64
// block: with ar / ac the first row of the pair's second / first block
// (lower; the other way round for upper),
//   T = D[ar.., ac..] Y[ac.., ac..]   (C P^-1, resp. C Q^-1)
//   Y[ar.., ac..] = -Y[ar.., ar..] T   (-Q^-1 T, resp. -P^-1 T)
// each output an FP64 sum in increasing k; RT x CT outputs per thread.
template <int H, int RT, int CT>
__device__ __forceinline__ void inv_double(double (*Y)[TB + 1], double (*Tm)[TB / 2 + 1], double (*D)[TB + 1],
                                           int lower_op, int t)
{
    constexpr int CTILES = H / CT, TILES = H / RT * CTILES;  // per pair
    static_assert((TB / (2 * H)) * TILES == kInvThreads, "one tile per thread");
    const int pr = t / TILES, e = t % TILES, r0 = (e / CTILES) * RT, c0 = (e % CTILES) * CT;
    const int o = pr * 2 * H;
    const int ar = lower_op ? o + H : o, ac = lower_op ? o : o + H;
    double acc[RT][CT] = {};
    for (int k = 0; k < H; ++k) {
#pragma unroll
        for (int i = 0; i < RT; ++i)
#pragma unroll
            for (int j = 0; j < CT; ++j) acc[i][j] = fma(D[ar + r0 + i][ac + k], Y[ac + k][ac + c0 + j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
        for (int j = 0; j < CT; ++j) Tm[pr * H + r0 + i][c0 + j] = acc[i][j];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
        for (int j = 0; j < CT; ++j) acc[i][j] = 0.0;
    for (int k = 0; k < H; ++k) {
#pragma unroll
        for (int i = 0; i < RT; ++i)
#pragma unroll
            for (int j = 0; j < CT; ++j) acc[i][j] = fma(Y[ar + r0 + i][ar + k], Tm[pr * H + k][c0 + j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
        for (int j = 0; j < CT; ++j) Y[ar + r0 + i][ac + c0 + j] = -acc[i][j];
    __syncthreads();
}

__global__ void __launch_bounds__(kInvThreads) batched_inv_kernel(const int2* __restrict__ inv_items,
                                                                  const int* __restrict__ dims,
                                                                  const long* __restrict__ inv_off, int lower_op,
                                                                  int op, int unit,
                                                                  const float* const* __restrict__ Aptr,
                                                                  float* __restrict__ inv)
{
    extern __shared__ double ysm[];
    double(*Y)[TB + 1] = (double(*)[TB + 1])ysm;              // the inverse being built
    double(*Tm)[TB / 2 + 1] = (double(*)[TB / 2 + 1])(ysm + TB * (TB + 1));  // doubling temporary
    // the block itself, held in FP64 so that the products below convert
    // nothing in their inner loops (FP32 -> FP64 conversions run at a
    // quarter of the FP64 FMA rate)
    double(*D)[TB + 1] = (double(*)[TB + 1])(ysm + TB * (TB + 1) + (TB / 2) * (TB / 2 + 1));
    const int t = threadIdx.x;
    const int2 w = inv_items[blockIdx.x];
    const int* d = dims + 4 * w.x;
    const int m = d[0];
    const long lda = d[2];
    const float* A = Aptr[w.x];
    const int r0 = w.y * TB, nr = min(TB, m - r0);
    {
        // all 16 loads of the thread in flight before the first store
        constexpr int PER = TB * TB / kInvThreads;
        float a[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int idx = t + u * kInvThreads, r = idx % TB, c = idx / TB;  // coalesced down A's columns
            a[u] = (r < nr && c < nr && !(r == c && unit)) ? A[(long)(r0 + c) * lda + r0 + r] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int idx = t + u * kInvThreads, r = idx % TB, c = idx / TB;
            const double v = (r == c && (r >= nr || unit)) ? 1.0 : (double)a[u];
            if (op == 0) D[r][c] = v;
            else D[c][r] = v;
        }
    }
    for (int idx = t; idx < TB * TB; idx += kInvThreads) Y[idx % TB][idx / TB] = 0.0;
    __syncthreads();
    // 1. 16 x 16 diagonal sub-blocks, one column per thread
    if (t < TB) {
        const int b = (t / 16) * 16, j = t % 16;
        if (lower_op) {
            for (int i = 0; i < 16; ++i) {
                double y = (i == j) ? 1.0 : 0.0;
                for (int k = j; k < i; ++k) y = fma(-D[b + i][b + k], Y[b + k][b + j], y);
                Y[b + i][b + j] = (i >= j) ? y / D[b + i][b + i] : 0.0;
            }
        } else {
            for (int i = 15; i >= 0; --i) {
                double y = (i == j) ? 1.0 : 0.0;
                for (int k = i + 1; k <= j; ++k) y = fma(-D[b + i][b + k], Y[b + k][b + j], y);
                Y[b + i][b + j] = (i <= j) ? y / D[b + i][b + i] : 0.0;
            }
        }
    }
    __syncthreads();
    // 2. doubling: blocks of size h combine into 2h (h = 16: two pairs, one
    // row x two columns per thread; h = 32: one pair, 2 x 2 per thread)
    inv_double<16, 1, 2>(Y, Tm, D, lower_op, t);
    inv_double<32, 2, 2>(Y, Tm, D, lower_op, t);
    float* out = inv + inv_off[w.x] + (long)w.y * TB * TB;
    for (int idx = t; idx < TB * TB; idx += kInvThreads) out[idx] = (float)Y[idx % TB][idx / TB];
}

// ---------------------------------------------------------------- TRSM kernel
// Persistent; each item is one instance and RC right-hand sides.  For each
// 64-row block of M = op(A) in solve order:
//   Y = alpha * B[block] - sum over earlier blocks q of M[block, q] X[q]
//       (K slices of 16 staged in shared memory, double-buffered through
//        registers; 4 x RC/16 outputs per thread from float4 reads)
//   X[block] = inv(M[block, block]) Y        (the precomputed FP32 inverse,
//        read transposed when `inv_t`: the adjoint's transposed operator)
// BT: the right-hand sides are the rows of B (element (row, rhs) at
// B[row * ldb + rhs]): the right-side solve X op(A) = alpha B run as
// op(A)^T X^T = alpha B^T.  Loads and stores then run along the rows.
constexpr int KC = 16;

// Two FP32 fused multiply-adds in one instruction (fma.rn.f32x2): each lane
// rounded as fmaf, so results keep their bits; the accumulators are held in
// pairs along the columns
__device__ __forceinline__ unsigned long long pack2(float lo, float hi)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long v)
{
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}
__device__ __forceinline__ void mac2(unsigned long long& acc, unsigned long long a, unsigned long long b)
{
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(a), "l"(b));
}

template <int RC, bool BT>
__global__ void __launch_bounds__(256, 4) batched_trsm_kernel(int nitems, const int2* __restrict__ items,
                                                           const int* __restrict__ dims,
                                                           const long* __restrict__ inv_off,
                                                           const float* __restrict__ inv, int lower_op, int op,
                                                           int inv_t, float alpha,
                                                           const float* const* __restrict__ Aptr,
                                                           float* const* __restrict__ Bptr, unsigned* counter)
{
    constexpr int CPT = RC / 16;        // columns per thread
    constexpr int XPT = KC * RC / 256;  // X slice elements per thread
    __shared__ __align__(16) float Ms[2][KC][TB + 4];
    __shared__ __align__(16) float Xs[2][KC][RC + 4];
    __shared__ __align__(16) float Ys[TB][RC + 4];
    __shared__ int item_sh;
    const int t = threadIdx.x, tx = t % 16, ty = t / 16;
    for (;;) {
        __syncthreads();
        if (t == 0) item_sh = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int it = item_sh;
        if (it >= nitems) break;
        const int2 w = items[it];
        const int* d = dims + 4 * w.x;
        const int m = d[0], nrhs = d[1];
        const long lda = d[2], ldb = d[3];
        const float* A = Aptr[w.x];
        float* B = Bptr[w.x];
        const float* IV = inv + inv_off[w.x];
        const int c0 = w.y * RC, nc = min(RC, nrhs - c0);
        const int nb = (m + TB - 1) / TB;
        for (int p = 0; p < nb; ++p) {
            const int kb = lower_op ? p : nb - 1 - p;
            const int r0 = kb * TB, nr = min(TB, m - r0);
            __syncthreads();
            for (int idx = t; idx < TB * RC; idx += 256) {
                const int r = BT ? idx / RC : idx % TB, c = BT ? idx % RC : idx / TB;
                const long bi = BT ? (long)(r0 + r) * ldb + c0 + c : (long)(c0 + c) * ldb + r0 + r;
                Ys[r][c] = (r < nr && c < nc) ? alpha * B[bi] : 0.f;
            }
            __syncthreads();
            unsigned long long acc[4][CPT / 2];  // column pairs
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < CPT / 2; ++j)
                    acc[i][j] = pack2(Ys[ty * 4 + i][tx * CPT + 2 * j], Ys[ty * 4 + i][tx * CPT + 2 * j + 1]);

            // ---- update by the earlier blocks: K = 64 p in slices of 16
            const int nslices = p * (TB / KC);
            float ra[4], rx[XPT];
            auto load = [&](int sl) {
                const int q = sl / (TB / KC), kk0 = (sl % (TB / KC)) * KC;
                const int j0 = (lower_op ? q : nb - 1 - q) * TB;
                const int nk = min(TB, m - j0) - kk0;  // valid k in this slice: k < nk
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int e = t + 256 * u;
                    int r, k;
                    if (op == 0) { r = e % TB; k = e / TB; } else { k = e % KC; r = e / KC; }
                    float v = 0.f;
                    if (r < nr && k < nk)
                        v = op == 0 ? A[(long)(j0 + kk0 + k) * lda + r0 + r] : A[(long)(r0 + r) * lda + j0 + kk0 + k];
                    ra[u] = v;
                }
#pragma unroll
                for (int u = 0; u < XPT; ++u) {
                    const int e = t + 256 * u;
                    const int k = BT ? e / RC : e % KC, c = BT ? e % RC : e / KC;
                    const long bi = BT ? (long)(j0 + kk0 + k) * ldb + c0 + c : (long)(c0 + c) * ldb + j0 + kk0 + k;
                    rx[u] = (c < nc && k < nk) ? B[bi] : 0.f;
                }
            };
            auto store = [&](int buf) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int e = t + 256 * u;
                    int r, k;
                    if (op == 0) { r = e % TB; k = e / TB; } else { k = e % KC; r = e / KC; }
                    Ms[buf][k][r] = ra[u];
                }
#pragma unroll
                for (int u = 0; u < XPT; ++u) {
                    const int e = t + 256 * u;
                    if (BT) Xs[buf][e / RC][e % RC] = rx[u];
                    else Xs[buf][e % KC][e / KC] = rx[u];
                }
            };
            if (nslices > 0) {
                load(0);
                store(0);
                __syncthreads();
                for (int sl = 0; sl < nslices; ++sl) {
                    const int buf = sl & 1;
                    if (sl + 1 < nslices) load(sl + 1);
#pragma unroll
                    for (int k = 0; k < KC; ++k) {
                        const float4 a = *reinterpret_cast<const float4*>(&Ms[buf][k][ty * 4]);
                        float b[CPT];
                        if (CPT == 4) {
                            const float4 bv = *reinterpret_cast<const float4*>(&Xs[buf][k][tx * 4]);
                            b[0] = bv.x; b[1] = bv.y; b[2] = bv.z; b[3] = bv.w;
                        } else {
                            const float2 bv = *reinterpret_cast<const float2*>(&Xs[buf][k][tx * CPT]);
                            b[0] = bv.x; b[1] = bv.y;
                        }
                        const float av[4] = {a.x, a.y, a.z, a.w};
                        unsigned long long bp[CPT / 2];
#pragma unroll
                        for (int j = 0; j < CPT / 2; ++j) bp[j] = pack2(b[2 * j], b[2 * j + 1]);
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const unsigned long long ap = pack2(-av[i], -av[i]);
#pragma unroll
                            for (int j = 0; j < CPT / 2; ++j) mac2(acc[i][j], ap, bp[j]);
                        }
                    }
                    if (sl + 1 < nslices) store(buf ^ 1);
                    __syncthreads();
                }
            }

            // ---- X = inv(M[block, block]) Y
            __syncthreads();
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < CPT / 2; ++j) {
                    const float2 v = unpack2(acc[i][j]);
                    Ys[ty * 4 + i][tx * CPT + 2 * j] = v.x;
                    Ys[ty * 4 + i][tx * CPT + 2 * j + 1] = v.y;
                }
            unsigned long long out[4][CPT / 2];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < CPT / 2; ++j) out[i][j] = 0ull;  // (+0.f, +0.f)
            const float* IB = IV + (long)kb * TB * TB;
            for (int kk0 = 0; kk0 < TB; kk0 += KC) {
                __syncthreads();
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int e = t + 256 * u;
                    int r, k;
                    if (!inv_t) { r = e % TB; k = e / TB; } else { k = e % KC; r = e / KC; }
                    // inv(r, kk0 + k): column-major block, or its transpose
                    Ms[0][k][r] = inv_t ? IB[(long)r * TB + kk0 + k] : IB[(long)(kk0 + k) * TB + r];
                }
                __syncthreads();
#pragma unroll
                for (int k = 0; k < KC; ++k) {
                    const float4 a = *reinterpret_cast<const float4*>(&Ms[0][k][ty * 4]);
                    float b[CPT];
                    if (CPT == 4) {
                        const float4 bv = *reinterpret_cast<const float4*>(&Ys[kk0 + k][tx * 4]);
                        b[0] = bv.x; b[1] = bv.y; b[2] = bv.z; b[3] = bv.w;
                    } else {
                        const float2 bv = *reinterpret_cast<const float2*>(&Ys[kk0 + k][tx * CPT]);
                        b[0] = bv.x; b[1] = bv.y;
                    }
                    const float av[4] = {a.x, a.y, a.z, a.w};
                    unsigned long long bp[CPT / 2];
#pragma unroll
                    for (int j = 0; j < CPT / 2; ++j) bp[j] = pack2(b[2 * j], b[2 * j + 1]);
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const unsigned long long ap = pack2(av[i], av[i]);
#pragma unroll
                        for (int j = 0; j < CPT / 2; ++j) mac2(out[i][j], ap, bp[j]);
                    }
                }
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < CPT / 2; ++j) {
                    const float2 v = unpack2(out[i][j]);
                    Ys[ty * 4 + i][tx * CPT + 2 * j] = v.x;
                    Ys[ty * 4 + i][tx * CPT + 2 * j + 1] = v.y;
                }
            __syncthreads();
            for (int idx = t; idx < TB * RC; idx += 256) {
                const int r = BT ? idx / RC : idx % TB, cc = BT ? idx % RC : idx / TB;
                const long bi = BT ? (long)(r0 + r) * ldb + c0 + cc : (long)(c0 + cc) * ldb + r0 + r;
                if (r < nr && cc < nc) B[bi] = Ys[r][cc];
            }
        }
    }
}

// ---------------------------------------------------------------- GEMM kernel
// MODE 0: C = alpha*op(A)*op(B) + beta*C, each element's products summed in
// k order by FP32 FMA from zero, then fmaf(alpha, acc, beta*C) (alpha*acc
// when beta == 0), the order of the single-instance plain SGEMM.
// MODE 1 (adjoint of TRSM): C is an m x m block kept on the triangle
// `tri_lower` (strict when `tri_strict`), zero elsewhere.
// Each item is one 64 x RC tile; K slices of 16 are double-buffered through
// registers into shared memory (k-major), 4 x RC/16 outputs per thread.
template <int RC, int MODE>
__global__ void __launch_bounds__(256, 4) batched_gemm_kernel(int nitems, const int2* __restrict__ items,
                                                           const int* __restrict__ dims, int ta, int tb, float alpha,
                                                           float beta, const float* const* __restrict__ Aptr,
                                                           const float* const* __restrict__ Bptr,
                                                           float* const* __restrict__ Cptr, unsigned* counter,
                                                           int tri_lower, int tri_strict)
{
    constexpr int CPT = RC / 16;
    constexpr int BPT = KC * RC / 256;  // B slice elements per thread
    __shared__ __align__(16) float As[2][KC][TB + 4];
    __shared__ __align__(16) float Bs[2][KC][RC + 4];
    __shared__ int item_sh;
    const int t = threadIdx.x, tx = t % 16, ty = t / 16;
    for (;;) {
        __syncthreads();
        if (t == 0) item_sh = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int it = item_sh;
        if (it >= nitems) break;
        const int2 w = items[it];
        const int* d = dims + 6 * w.x;
        const int m = d[0], n = d[1], k = d[2];
        const long lda = d[3], ldb = d[4], ldc = d[5];
        const float* A = Aptr[w.x];
        const float* Bm = Bptr[w.x];
        float* C = Cptr[w.x];
        const int tiles_m = (m + TB - 1) / TB;
        const int tm = w.y % tiles_m, tn = w.y / tiles_m;
        const int i0 = tm * TB, j0 = tn * RC;
        // adjoint tiles entirely off the kept triangle are only zeroed
        bool skip = false;
        if (MODE == 1) skip = tri_lower ? (j0 > i0 + TB - 1) : (i0 > j0 + RC - 1);
        unsigned long long acc[4][CPT / 2];  // column pairs
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < CPT / 2; ++j) acc[i][j] = 0ull;  // (+0.f, +0.f)
        const int nslices = skip ? 0 : (k + KC - 1) / KC;
        float ra[4], rb[BPT];
        auto load = [&](int sl) {
            const int k0 = sl * KC;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = t + 256 * u;
                int r, kk;
                if (ta == 0) { r = e % TB; kk = e / TB; } else { kk = e % KC; r = e / KC; }
                float v = 0.f;
                if (i0 + r < m && k0 + kk < k)
                    v = ta == 0 ? A[(long)(k0 + kk) * lda + i0 + r] : A[(long)(i0 + r) * lda + k0 + kk];
                ra[u] = v;
            }
#pragma unroll
            for (int u = 0; u < BPT; ++u) {
                const int e = t + 256 * u;
                int kk, c;
                if (tb == 0) { kk = e % KC; c = e / KC; } else { c = e % RC; kk = e / RC; }
                float v = 0.f;
                if (k0 + kk < k && j0 + c < n)
                    v = tb == 0 ? Bm[(long)(j0 + c) * ldb + k0 + kk] : Bm[(long)(k0 + kk) * ldb + j0 + c];
                rb[u] = v;
            }
        };
        auto store = [&](int buf) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = t + 256 * u;
                int r, kk;
                if (ta == 0) { r = e % TB; kk = e / TB; } else { kk = e % KC; r = e / KC; }
                As[buf][kk][r] = ra[u];
            }
#pragma unroll
            for (int u = 0; u < BPT; ++u) {
                const int e = t + 256 * u;
                int kk, c;
                if (tb == 0) { kk = e % KC; c = e / KC; } else { c = e % RC; kk = e / RC; }
                Bs[buf][kk][c] = rb[u];
            }
        };
        if (nslices > 0) {
            load(0);
            store(0);
            __syncthreads();
            for (int sl = 0; sl < nslices; ++sl) {
                const int buf = sl & 1;
                if (sl + 1 < nslices) load(sl + 1);
#pragma unroll
                for (int kk = 0; kk < KC; ++kk) {
                    const float4 a = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
                    float b[CPT];
                    if (CPT == 4) {
                        const float4 bv = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
                        b[0] = bv.x; b[1] = bv.y; b[2] = bv.z; b[3] = bv.w;
                    } else {
                        const float2 bv = *reinterpret_cast<const float2*>(&Bs[buf][kk][tx * CPT]);
                        b[0] = bv.x; b[1] = bv.y;
                    }
                    const float av[4] = {a.x, a.y, a.z, a.w};
                    unsigned long long bp[CPT / 2];
#pragma unroll
                    for (int j = 0; j < CPT / 2; ++j) bp[j] = pack2(b[2 * j], b[2 * j + 1]);
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const unsigned long long ap = pack2(av[i], av[i]);
#pragma unroll
                        for (int j = 0; j < CPT / 2; ++j) mac2(acc[i][j], ap, bp[j]);
                    }
                }
                if (sl + 1 < nslices) store(buf ^ 1);
                __syncthreads();
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < CPT; ++j) {
                const int r = i0 + ty * 4 + i, c = j0 + tx * CPT + j;
                if (r >= m || c >= n) continue;
                const float2 v2 = unpack2(acc[i][j / 2]);
                const float v = (j & 1) ? v2.y : v2.x;
                float* cp = C + (long)c * ldc + r;
                if (MODE == 1) {
                    const bool keep = tri_lower ? (r > c || (r == c && !tri_strict))
                                                : (r < c || (r == c && !tri_strict));
                    *cp = keep ? alpha * v : 0.f;
                } else {
                    *cp = beta == 0.f ? alpha * v : fmaf(alpha, v, __fmul_rn(beta, *cp));
                }
            }
    }
}

// Synthetic operand fill for tuning.
__global__ void tune_fill_kernel(long count, float* __restrict__ p, float v)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) p[i] = v;
}

__global__ void tune_ptrs_kernel(int batch, const float** __restrict__ a, const float* pa, const float** __restrict__ b,
                                 const float* pb, const float** __restrict__ c, const float* pc)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x) {
        a[i] = pa;
        b[i] = pb;
        c[i] = pc;
    }
}

// ---------------------------------------------------------------- host: work lists
struct Item {
    double cost;
    int2 w;
};

void sort_items(std::vector<Item>& v)
{
    std::stable_sort(v.begin(), v.end(), [](const Item& a, const Item& b) { return a.cost > b.cost; });
}

// TRSM: one item per (instance, RC-wide column block); cost m^2 * columns.
std::vector<int2> trsm_items(int batch, const std::vector<int>& dims, int rc)
{
    std::vector<Item> v;
    for (int i = 0; i < batch; ++i) {
        const int m = dims[4 * i], n = dims[4 * i + 1];
        if (m == 0 || n == 0) continue;
        for (int c = 0; c * rc < n; ++c) {
            const int nc = std::min(rc, n - c * rc);
            v.push_back({(double)m * m * nc + (double)m * rc, make_int2(i, c)});
        }
    }
    sort_items(v);
    std::vector<int2> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i].w;
    return out;
}

// GEMM: one item per 64 x RC tile of C; cost k (tiles off the kept triangle
// of the adjoint product cost a store only).
std::vector<int2> gemm_items(int batch, const std::vector<int>& dims, int rc, bool masked, bool tri_lower)
{
    std::vector<Item> v;
    for (int i = 0; i < batch; ++i) {
        const int m = dims[6 * i], n = dims[6 * i + 1], k = dims[6 * i + 2];
        if (m == 0 || n == 0) continue;
        const int tm = (m + TB - 1) / TB, tn = (n + rc - 1) / rc;
        for (int b = 0; b < tm * tn; ++b) {
            const int i0 = (b % tm) * TB, j0 = (b / tm) * rc;
            const bool skip = masked && (tri_lower ? (j0 > i0 + TB - 1) : (i0 > j0 + rc - 1));
            v.push_back({skip ? 1.0 : (double)k * TB * rc + TB * rc, make_int2(i, b)});
        }
    }
    sort_items(v);
    std::vector<int2> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i].w;
    return out;
}

cudaError_t upload_items(const std::vector<int2>& items, BatchList& l)
{
    if (l.items) cudaFree(l.items);
    l.items = nullptr;
    l.nitems = (int)items.size();
    if (items.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(&l.items, items.size() * sizeof(int2));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(l.items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice);
}

cudaError_t upload_dims(const std::vector<int>& dims, BatchList& l)
{
    if (dims.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(&l.dims, dims.size() * sizeof(int));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(l.dims, dims.data(), dims.size() * sizeof(int), cudaMemcpyHostToDevice);
}

int grid_of(iclblasHandle_t h, const BatchList& l)
{
    return std::max(1, std::min(l.nitems, h->sm_count * l.ctas_per_sm));
}

// ---------------------------------------------------------------- host: launches
constexpr int kInvSmem = TB * (TB + 1) * (int)(2 * sizeof(double)) + (TB / 2) * (TB / 2 + 1) * (int)sizeof(double);

// The pass forming the diagonal-block inverses of M = op(A).
cudaError_t launch_inv(iclblasHandle_t h, const int2* inv_items, int n_inv, const int* dims, const long* inv_off,
                       int lower_op, int op, int unit, const float* const* A, float* inv)
{
    if (n_inv == 0) return cudaSuccess;
    // the attribute belongs to each device's copy of the kernel (the calls
    // run with the handle's device current)
    static std::atomic<unsigned long long> attr_set{0};
    const unsigned long long bit = 1ull << (h->device & 63);
    if (!(attr_set.load() & bit)) {
        cudaError_t e = cudaFuncSetAttribute(batched_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             kInvSmem);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(bit);
    }
    batched_inv_kernel<<<n_inv, kInvThreads, kInvSmem, h->stream>>>(inv_items, dims, inv_off, lower_op, op, unit, A,
                                                                    inv);
    return cudaGetLastError();
}

// The solve, given the inverses (read transposed when inv_t).
cudaError_t launch_trsm(iclblasHandle_t h, const BatchList& l, unsigned* counter, const long* inv_off,
                        const float* inv, int lower_op, int op, int inv_t, bool bt, float alpha,
                        const float* const* A, float* const* B)
{
    if (l.nitems == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), h->stream);
    if (e != cudaSuccess) return e;
    const int grid = grid_of(h, l);
    auto go = [&](auto kernel) {
        kernel<<<grid, 256, 0, h->stream>>>(l.nitems, l.items, l.dims, inv_off, inv, lower_op, op, inv_t, alpha, A, B,
                                            counter);
    };
    if (l.rc == 32) bt ? go(batched_trsm_kernel<32, true>) : go(batched_trsm_kernel<32, false>);
    else bt ? go(batched_trsm_kernel<64, true>) : go(batched_trsm_kernel<64, false>);
    return cudaGetLastError();
}

cudaError_t launch_gemm(iclblasHandle_t h, const BatchList& l, unsigned* counter, bool masked, int ta, int tb,
                        float alpha, float beta, const float* const* A, const float* const* B, float* const* C,
                        int tri_lower, int tri_strict)
{
    if (l.nitems == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), h->stream);
    if (e != cudaSuccess) return e;
    const int grid = grid_of(h, l);
    if (masked) {
        if (l.rc == 32)
            batched_gemm_kernel<32, 1><<<grid, 256, 0, h->stream>>>(l.nitems, l.items, l.dims, ta, tb, alpha, beta, A,
                                                                    B, C, counter, tri_lower, tri_strict);
        else
            batched_gemm_kernel<64, 1><<<grid, 256, 0, h->stream>>>(l.nitems, l.items, l.dims, ta, tb, alpha, beta, A,
                                                                    B, C, counter, tri_lower, tri_strict);
    } else {
        if (l.rc == 32)
            batched_gemm_kernel<32, 0><<<grid, 256, 0, h->stream>>>(l.nitems, l.items, l.dims, ta, tb, alpha, beta, A,
                                                                    B, C, counter, 0, 0);
        else
            batched_gemm_kernel<64, 0><<<grid, 256, 0, h->stream>>>(l.nitems, l.items, l.dims, ta, tb, alpha, beta, A,
                                                                    B, C, counter, 0, 0);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------- host: tuning cache
struct Choice {
    int rc, ctas;
};
std::mutex g_tune_mu;
std::map<std::string, Choice> g_tune;
bool g_tune_loaded = false;

const char* tune_path()
{
    const char* p = std::getenv("ICLBLAS_TUNE_CACHE");
    return (p && *p) ? p : nullptr;
}

void load_tune_file_locked()
{
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = tune_path();
    if (!path) return;
    std::ifstream f(path);
    std::string key;
    int rc, ctas;
    while (f >> key >> rc >> ctas)
        if ((rc == 32 || rc == 64) && (ctas == 1 || ctas == 2 || ctas == 4)) g_tune[key] = Choice{rc, ctas};
}

bool lookup_tune(const std::string& key, Choice& c)
{
    std::lock_guard<std::mutex> g(g_tune_mu);
    load_tune_file_locked();
    auto it = g_tune.find(key);
    if (it == g_tune.end()) return false;
    c = it->second;
    return true;
}

void store_tune(const std::string& key, Choice c)
{
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune[key] = c;
    if (const char* path = tune_path()) {
        std::ofstream f(path, std::ios::app);
        f << key << ' ' << c.rc << ' ' << c.ctas << '\n';
    }
}

// Key: kind, flags, instance count, FNV-1a hash of the sizes, GPU name and SM count.
std::string tune_key(iclblasHandle_t h, const char* kind, const std::vector<int>& flags, int batch,
                     const std::vector<int>& dims)
{
    uint64_t x = 1469598103934665603ull;
    for (int v : dims)
        for (int b = 0; b < 4; ++b) {
            x ^= (uint64_t)((v >> (8 * b)) & 0xff);
            x *= 1099511628211ull;
        }
    cudaDeviceProp prop;
    std::string name = "gpu";
    if (cudaGetDeviceProperties(&prop, h->device) == cudaSuccess) name = prop.name;
    for (char& ch : name)
        if (ch == ' ' || ch == '\t') ch = '_';
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%016llx", (unsigned long long)x);
    std::string key = std::string(kind);
    for (int f : flags) key += "." + std::to_string(f);
    key += "|b" + std::to_string(batch) + "|" + buf + "|" + name + "|sm" + std::to_string(h->sm_count);
    return key;
}

// Device buffers for timing candidates: every instance points at the same
// operands (sized for the largest instance).  TRSM: A all ones, B zero, so
// every solve writes zeros and concurrent instances store identical values.
// GEMM: A, B, C zero.
struct TuneBuffers {
    float *a = nullptr, *b = nullptr, *c = nullptr;
    const float** ptrs = nullptr;   // 3 x batch pointers
    long* zoff = nullptr;           // batch zero offsets (every instance's inverses at c)
    unsigned* counter = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~TuneBuffers()
    {
        if (zoff) cudaFree(zoff);
        if (a) cudaFree(a);
        if (b) cudaFree(b);
        if (c) cudaFree(c);
        if (ptrs) cudaFree(ptrs);
        if (counter) cudaFree(counter);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
    cudaError_t init(iclblasHandle_t h, int batch, long na, long nb, long nc, float fill_a)
    {
        cudaError_t e;
        if ((e = cudaMalloc(&a, std::max(na, 1L) * sizeof(float))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&b, std::max(nb, 1L) * sizeof(float))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&c, std::max(nc, 1L) * sizeof(float))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&ptrs, 3 * (size_t)batch * sizeof(float*))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&counter, sizeof(unsigned))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&zoff, (size_t)batch * sizeof(long))) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(zoff, 0, (size_t)batch * sizeof(long), h->stream)) != cudaSuccess) return e;
        if ((e = cudaEventCreate(&e0)) != cudaSuccess) return e;
        if ((e = cudaEventCreate(&e1)) != cudaSuccess) return e;
        tune_fill_kernel<<<h->sm_count * 4, 256, 0, h->stream>>>(std::max(na, 1L), a, fill_a);
        tune_fill_kernel<<<h->sm_count * 4, 256, 0, h->stream>>>(std::max(nb, 1L), b, 0.f);
        tune_fill_kernel<<<h->sm_count * 4, 256, 0, h->stream>>>(std::max(nc, 1L), c, 0.f);
        tune_ptrs_kernel<<<(batch + 255) / 256, 256, 0, h->stream>>>(batch, ptrs, a, ptrs + batch, b,
                                                                      ptrs + 2 * batch, c);
        return cudaGetLastError();
    }
};

// Times `run` (one launch of the list) once untimed and 3 times timed; ms per launch.
template <class F>
cudaError_t time_launch(iclblasHandle_t h, TuneBuffers& tb, F&& run, float& ms)
{
    cudaError_t e = run();
    if (e != cudaSuccess) return e;
    if ((e = cudaEventRecord(tb.e0, h->stream)) != cudaSuccess) return e;
    for (int r = 0; r < 3; ++r)
        if ((e = run()) != cudaSuccess) return e;
    if ((e = cudaEventRecord(tb.e1, h->stream)) != cudaSuccess) return e;
    if ((e = cudaEventSynchronize(tb.e1)) != cudaSuccess) return e;
    if ((e = cudaEventElapsedTime(&ms, tb.e0, tb.e1)) != cudaSuccess) return e;
    ms /= 3.f;
    return cudaSuccess;
}

const int kRcs[] = {32, 64};
const int kCtas[] = {1, 2, 4};

// Chooses (rc, ctas) for a TRSM list and fills l.items for the choice.
cudaError_t tune_trsm(iclblasHandle_t h, int batch, const std::vector<int>& dims, int lower_op, int op, int unit,
                      bool bt, BatchList& l)
{
    if (trsm_items(batch, dims, 64).empty()) return upload_items({}, l);   // nothing to solve
    // the key names the kernel generation so that cached choices for an older
    // kernel are not reused
    const std::string key = tune_key(h, "trsm2", {lower_op, op, unit, bt ? 1 : 0}, batch, dims);
    Choice best{64, 1};
    if (!lookup_tune(key, best)) {
        long na = 0, nb = 0, ni = 0;
        for (int i = 0; i < batch; ++i) {
            na = std::max(na, (long)dims[4 * i + 2] * dims[4 * i]);
            nb = std::max(nb, (long)dims[4 * i + 3] * dims[4 * i + (bt ? 0 : 1)]);
            ni = std::max(ni, (long)((dims[4 * i] + TB - 1) / TB) * TB * TB);
        }
        TuneBuffers tb;  // inverses: zeros at c for every instance
        cudaError_t e = tb.init(h, batch, na, nb, ni, 1.f);
        if (e != cudaSuccess) return e;
        float best_ms = 3.4e38f;
        for (int rc : kRcs) {
            BatchList cand;
            cand.dims = l.dims;
            cand.rc = rc;
            if ((e = upload_items(trsm_items(batch, dims, rc), cand)) != cudaSuccess) return e;
            for (int ctas : kCtas) {
                cand.ctas_per_sm = ctas;
                float ms = 0;
                e = time_launch(h, tb, [&]() {
                    return launch_trsm(h, cand, tb.counter, tb.zoff, tb.c, lower_op, op, 0, bt, 1.f, tb.ptrs,
                                       const_cast<float* const*>(tb.ptrs + batch));
                }, ms);
                if (e != cudaSuccess) break;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = Choice{rc, ctas};
                }
            }
            if (cand.items) cudaFree(cand.items);
            if (e != cudaSuccess) return e;
        }
        store_tune(key, best);
    }
    l.rc = best.rc;
    l.ctas_per_sm = best.ctas;
    return upload_items(trsm_items(batch, dims, best.rc), l);
}

cudaError_t tune_gemm(iclblasHandle_t h, int batch, const std::vector<int>& dims, int ta, int tb_, bool masked,
                      int tri_lower, int tri_strict, BatchList& l)
{
    if (gemm_items(batch, dims, 64, masked, tri_lower).empty()) return upload_items({}, l);
    const std::string key = tune_key(h, masked ? "gemm_adj2" : "gemm2", {ta, tb_, tri_lower, tri_strict}, batch, dims);
    Choice best{64, 1};
    if (!lookup_tune(key, best)) {
        long na = 0, nb = 0, nc = 0;
        for (int i = 0; i < batch; ++i) {
            const int m = dims[6 * i], n = dims[6 * i + 1], k = dims[6 * i + 2];
            na = std::max(na, (long)dims[6 * i + 3] * (ta ? m : k));
            nb = std::max(nb, (long)dims[6 * i + 4] * (tb_ ? k : n));
            nc = std::max(nc, (long)dims[6 * i + 5] * n);
        }
        TuneBuffers tb;
        cudaError_t e = tb.init(h, batch, na, nb, nc, 0.f);
        if (e != cudaSuccess) return e;
        float best_ms = 3.4e38f;
        for (int rc : kRcs) {
            BatchList cand;
            cand.dims = l.dims;
            cand.rc = rc;
            if ((e = upload_items(gemm_items(batch, dims, rc, masked, tri_lower), cand)) != cudaSuccess) return e;
            for (int ctas : kCtas) {
                cand.ctas_per_sm = ctas;
                float ms = 0;
                e = time_launch(h, tb, [&]() {
                    return launch_gemm(h, cand, tb.counter, masked, ta, tb_, 1.f, 0.f, tb.ptrs, tb.ptrs + batch,
                                       const_cast<float* const*>(tb.ptrs + 2 * batch), tri_lower, tri_strict);
                }, ms);
                if (e != cudaSuccess) break;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = Choice{rc, ctas};
                }
            }
            if (cand.items) cudaFree(cand.items);
            if (e != cudaSuccess) return e;
        }
        store_tune(key, best);
    }
    l.rc = best.rc;
    l.ctas_per_sm = best.ctas;
    return upload_items(gemm_items(batch, dims, best.rc, masked, tri_lower), l);
}

bool lower_op_of(int uplo, int trans)
{
    return (uplo == ICLBLAS_FILL_MODE_LOWER) != (trans != ICLBLAS_OP_N);
}

}  // namespace

cudaError_t batch_list_free(BatchList& l)
{
    if (l.dims) cudaFree(l.dims);
    if (l.items) cudaFree(l.items);
    l.dims = nullptr;
    l.items = nullptr;
    l.nitems = 0;
    return cudaSuccess;
}

void batch_plan_free(iclblasBatchPlan* p)
{
    if (!p) return;
    batch_list_free(p->main);
    batch_list_free(p->adj);
    batch_tc_free(p->tc);
    p->tc = nullptr;
    if (p->counter) cudaFree(p->counter);
    if (p->inv) cudaFree(p->inv);
    if (p->inv_off) cudaFree(p->inv_off);
    if (p->inv_items) cudaFree(p->inv_items);
    p->tag = 0;
    delete p;
}

cudaError_t batch_plan_create_trsm(iclblasHandle_t h, int side, int uplo, int trans, int diag, int batch,
                                   const int* m, const int* n, const int* lda, const int* ldb,
                                   iclblasBatchPlan** out)
{
    auto* p = new iclblasBatchPlan();
    p->kind = 0;
    p->side = side;
    p->uplo = uplo;
    p->trans = trans;
    p->diag = diag;
    p->batch = batch;
    p->device = h->device;
    // Solve dimension `na` (the triangle) and right-hand-side count `nr` per
    // instance: left side (m, n); right side (n, m), run on B's rows.
    const bool right = side == ICLBLAS_SIDE_RIGHT;
    std::vector<int> dims(4 * (size_t)batch), adims(6 * (size_t)batch);
    for (int i = 0; i < batch; ++i) {
        const int na = right ? n[i] : m[i], nr = right ? m[i] : n[i];
        dims[4 * i] = na;
        dims[4 * i + 1] = nr;
        dims[4 * i + 2] = lda[i];
        dims[4 * i + 3] = ldb[i];
        // adjoint product: dA (na x na, ld lda) from G and X (ld ldb), inner nr
        adims[6 * i] = na;
        adims[6 * i + 1] = na;
        adims[6 * i + 2] = nr;
        adims[6 * i + 3] = ldb[i];
        adims[6 * i + 4] = ldb[i];
        adims[6 * i + 5] = lda[i];
        p->flops += (double)na * na * nr;
    }
    const int op = trans != ICLBLAS_OP_N;
    const int unit = diag == ICLBLAS_DIAG_UNIT;
    // diagonal-block inverses: 64 x 64 FP32 per block of each instance
    std::vector<long> inv_off(batch > 0 ? batch : 1, 0);
    std::vector<int2> inv_items;
    long inv_total = 0;
    for (int i = 0; i < batch; ++i) {
        inv_off[i] = inv_total;
        const int nblk = (dims[4 * i] + TB - 1) / TB;
        if (dims[4 * i + 1] > 0)
            for (int b = 0; b < nblk; ++b) inv_items.push_back(make_int2(i, b));
        inv_total += (long)nblk * TB * TB;
    }
    p->n_inv = (int)inv_items.size();
    cudaError_t e = cudaMalloc(&p->counter, sizeof(unsigned));
    if (e == cudaSuccess && batch > 0) e = cudaMalloc(&p->inv_off, (size_t)batch * sizeof(long));
    if (e == cudaSuccess && batch > 0)
        e = cudaMemcpy(p->inv_off, inv_off.data(), (size_t)batch * sizeof(long), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && inv_total > 0) e = cudaMalloc(&p->inv, (size_t)inv_total * sizeof(float));
    if (e == cudaSuccess && p->n_inv > 0) e = cudaMalloc(&p->inv_items, inv_items.size() * sizeof(int2));
    if (e == cudaSuccess && p->n_inv > 0)
        e = cudaMemcpy(p->inv_items, inv_items.data(), inv_items.size() * sizeof(int2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = upload_dims(dims, p->main);
    if (e == cudaSuccess) e = upload_dims(adims, p->adj);
    // the right side solves op(A)^T X^T = alpha B^T: flipped operator, B's rows
    const int s_lower = right ? !lower_op_of(uplo, trans) : lower_op_of(uplo, trans);
    const int s_op = right ? !op : op;
    if (batch_tc_mode(h->math)) {
        // tensor-core path: 128-row tiles, one persistent CTA per SM
        p->main.rc = 128;
        p->main.ctas_per_sm = 1;
        if (e == cudaSuccess)
            e = batch_tc_create_trsm(h, p, dims, right ? 1 : 0, s_lower, s_op, uplo == ICLBLAS_FILL_MODE_LOWER, unit);
    } else {
        if (e == cudaSuccess) e = tune_trsm(h, batch, dims, s_lower, s_op, unit, right, p->main);
        // dA: left -(1/alpha) dB X^T (op N) or X dB^T; right -(1/alpha) X^T dB (op N) or dB^T X
        if (e == cudaSuccess)
            e = tune_gemm(h, batch, adims, right ? 1 : 0, right ? 0 : 1, true, uplo == ICLBLAS_FILL_MODE_LOWER,
                          unit, p->adj);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        batch_plan_free(p);
        return e;
    }
    p->tag = kBatchPlanTag;
    *out = p;
    return cudaSuccess;
}

cudaError_t batch_plan_create_gemm(iclblasHandle_t h, int transa, int transb, int batch, const int* m, const int* n,
                                   const int* k, const int* lda, const int* ldb, const int* ldc,
                                   iclblasBatchPlan** out)
{
    auto* p = new iclblasBatchPlan();
    p->kind = 1;
    p->transa = transa;
    p->transb = transb;
    p->batch = batch;
    p->device = h->device;
    std::vector<int> dims(6 * (size_t)batch);
    for (int i = 0; i < batch; ++i) {
        dims[6 * i] = m[i];
        dims[6 * i + 1] = n[i];
        dims[6 * i + 2] = k[i];
        dims[6 * i + 3] = lda[i];
        dims[6 * i + 4] = ldb[i];
        dims[6 * i + 5] = ldc[i];
        p->flops += 2.0 * m[i] * n[i] * k[i];
    }
    const int ta = transa != ICLBLAS_OP_N, tb = transb != ICLBLAS_OP_N;
    cudaError_t e = cudaMalloc(&p->counter, sizeof(unsigned));
    if (e == cudaSuccess) e = upload_dims(dims, p->main);
    if (batch_tc_mode(h->math)) {
        p->main.rc = 128;
        p->main.ctas_per_sm = 1;
        if (e == cudaSuccess) e = batch_tc_create_gemm(h, p, dims, ta, tb);
    } else if (e == cudaSuccess) {
        e = tune_gemm(h, batch, dims, ta, tb, false, 0, 0, p->main);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        batch_plan_free(p);
        return e;
    }
    p->tag = kBatchPlanTag;
    *out = p;
    return cudaSuccess;
}

cudaError_t batch_trsm(iclblasHandle_t h, const iclblasBatchPlan* p, float alpha, const float* const* A,
                       float* const* B)
{
    // left: M = op(A) on B's columns; right: M = op(A)^T on B's rows
    const bool right = p->side == ICLBLAS_SIDE_RIGHT;
    const int lower_op = lower_op_of(p->uplo, p->trans) ^ (right ? 1 : 0);
    const int op = (p->trans != ICLBLAS_OP_N) ^ (right ? 1 : 0);
    cudaError_t e = launch_inv(h, p->inv_items, p->n_inv, p->main.dims, p->inv_off, lower_op, op,
                               p->diag == ICLBLAS_DIAG_UNIT, A, p->inv);
    if (e != cudaSuccess) return e;
    if (p->tc) {
        if ((e = batch_tc_inverses(h, p, A)) != cudaSuccess) return e;
        p->inv_formed = true;
        return batch_tc_solve(h, p, 0, alpha, A, B, 0);
    }
    p->inv_formed = true;
    return launch_trsm(h, p->main, p->counter, p->inv_off, p->inv, lower_op, op, 0, right, alpha, A, B);
}

cudaError_t batch_gemm(iclblasHandle_t h, const iclblasBatchPlan* p, float alpha, const float* const* A,
                       const float* const* B, float beta, float* const* C)
{
    if (p->tc) return batch_tc_gemm(h, p, alpha, A, B, beta, C);
    return launch_gemm(h, p->main, p->counter, false, p->transa != ICLBLAS_OP_N, p->transb != ICLBLAS_OP_N, alpha,
                       beta, A, B, C, 0, 0);
}

// Adjoint of X = alpha * op(A)^-1 B for every instance.  G (= dL/dX) becomes
// dB = alpha * op(A)^-T G (the TRSM launch with the transposed operator,
// alpha applied on load); then dA = -W X^T (op N) or -X W^T (op T/C) with
// W = dB / alpha, kept on the stored triangle (the masked GEMM launch, its
// alpha -1/alpha; alpha == 0 gives X == 0 and so dA == 0).
cudaError_t batch_trsm_backward(iclblasHandle_t h, const iclblasBatchPlan* p, float alpha, const float* const* A,
                                const float* const* X, float* const* G, float* const* dA)
{
    const bool right = p->side == ICLBLAS_SIDE_RIGHT;
    const int op = p->trans != ICLBLAS_OP_N;
    const int unit = p->diag == ICLBLAS_DIAG_UNIT;
    // the forward's operator (right side: op(A)^T on B's rows) and its inverses;
    // the adjoint solves with the transposed operator, reading them transposed
    const int f_lower = lower_op_of(p->uplo, p->trans) ^ (right ? 1 : 0);
    const int f_op = op ^ (right ? 1 : 0);
    cudaError_t e = cudaSuccess;
    const bool reuse = p->reuse_inv && p->inv_formed;
    if (!reuse) {
        e = launch_inv(h, p->inv_items, p->n_inv, p->main.dims, p->inv_off, f_lower, f_op, unit, A, p->inv);
        if (e == cudaSuccess && p->tc) e = batch_tc_inverses(h, p, A);
    }
    if (e == cudaSuccess)
        e = p->tc ? batch_tc_solve(h, p, 1, alpha, A, G, reuse ? 1 : 0)
                  : launch_trsm(h, p->main, p->counter, p->inv_off, p->inv, !f_lower, !f_op, 1, right, alpha, A, G);
    if (e != cudaSuccess || !dA) return e;
    const float s = alpha != 0.f ? -1.f / alpha : 0.f;
    const float* const* Gc = const_cast<const float* const*>(G);
    // left: dM = -W X^T; right: dM = -X^T W; dA = dM (op N) or dM^T (op T/C)
    const float* const* P = right ? (op ? Gc : X) : (op ? X : Gc);
    const float* const* Q = right ? (op ? X : Gc) : (op ? Gc : X);
    if (p->tc) return batch_tc_dA(h, p, s, P, Q, dA);
    return launch_gemm(h, p->adj, p->counter, true, right ? 1 : 0, right ? 0 : 1, s, 0.f, P, Q, dA,
                       p->uplo == ICLBLAS_FILL_MODE_LOWER, unit);
}

}  // namespace iclb
