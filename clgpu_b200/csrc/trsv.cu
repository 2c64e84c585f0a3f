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
#include <type_traits>

#include "common.cuh"
#include "tma.cuh"

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

// ---------------------------------------------------------------- STRSV, TMA path
// Float TRSV when A is 16-byte aligned with lda a multiple of 4 and >= n
// (the usual case).  Same ticket-ordered one-launch structure as above, with
// changes that shorten the chain of dependent block solves:
//   - tiles arrive by TMA (one 64 x 64 box per cp.async.bulk.tensor) into a
//     4-stage shared-memory ring, so up to 64 KiB per CTA are in flight while
//     the CTA waits for earlier blocks, and two CTAs fit on an SM;
//   - the first box is the diagonal block D, inverted in FP64 (then kept in
//     FP32) before the CTA needs it; the second box is the tile T next to D
//     (the block solved just before this one), turned into W = inv(D) T
//     while earlier blocks are still being solved; then the remaining tiles
//     in solve order.  Once all but the last earlier block are known, the CTA
//     forms z = inv(D) (b - sum of those tiles' products), so its own step of
//     the chain, when the last block x_prev is published, is
//     x = z - W x_prev: one 64 x 64 product and a publication;
//   - each solved entry is published as one 64-bit word (value, call epoch):
//     a consumer polls the entries it needs directly, with no separate flag.
//     The epoch lives in device memory: each CTA reads the last launch's
//     epoch at its start and uses the next one; the CTA that solves the last
//     block stores it back once everything is published (every other CTA has
//     read it by then), so replays of a captured launch get fresh epochs;
//   - launched as clusters of 8 consecutive blocks (when the GPU can place
//     one), a solved block also goes straight into the shared memory of the
//     later CTAs of its cluster (st.async on a transaction barrier), and the
//     chain step runs on the 64 row threads alone, with no block-wide
//     barrier between the arrival of x_prev and the hand-off of x.  At
//     n = 16384 this took the call from 314 to 265 us, and the blocked FP64
//     inverse below (13 instead of 44 us at the start) to 230 us.
constexpr int FS = 4;
constexpr int TILE_ELEMS = NB * NB;
constexpr int kMaxCluster = 8;
constexpr unsigned long long kTrsvWaitNs = 2000000000ull;  // a wait gives up after 2 s

struct FastSmem {
    float stage[FS][TILE_ELEMS];
    // FP64 inverse while it is formed; then the same bytes hold the FP32
    // inverse and W (two [NB][NB + 1] float arrays)
    double R[NB][NB + 1];
    double Tm[NB / 2][NB / 2 + 1];  // inverse doubling temporary (and 1 / diagonal before it)
    float xs[NB];
    float ys[NB];
    float zs[NB];
    float part[4][NB];
    // cluster launches: the solved blocks of the earlier CTAs of this
    // cluster, delivered into this CTA's shared memory by st.async, one
    // transaction barrier per source rank
    float xin[kMaxCluster][NB];
    uint64_t xbar[kMaxCluster];
    uint64_t full[FS];
    unsigned s, epoch, cl;
    int failed;  // a wait of the chain step gave up
};

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// ---- thread-block-cluster helpers (distributed shared memory)
__device__ __forceinline__ unsigned cluster_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// this CTA's shared address `a` as seen in the shared memory of CTA `rank`
__device__ __forceinline__ uint32_t map_to(const void* a, unsigned rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(tma::smem_u32(a)), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_cluster_u32(uint32_t addr, unsigned v)
{
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
// 4 bytes into another CTA's shared memory, counted as transaction bytes on
// that CTA's barrier
__device__ __forceinline__ void st_async_f32(uint32_t addr, float v, uint32_t bar)
{
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f32 [%0], %1, [%2];" ::"r"(addr), "f"(v),
                 "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// bounded wait, acquiring at cluster scope (the bytes come from another CTA)
__device__ __forceinline__ bool xbar_wait_bounded(uint64_t* bar, unsigned long long limit_ns)
{
    auto try_once = [&]() {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], 0;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(tma::smem_u32(bar))
            : "memory");
        return ok != 0;
    };
    if (try_once()) return true;
    const unsigned long long t0 = tma::global_ns();
    while (!try_once())
        if (tma::global_ns() - t0 > limit_ns) return false;
    return true;
}

// CL = 1: one CTA per block, every solved block handed on through global
// memory.  CL > 1 (a cluster launch): the CTAs of a cluster solve CL
// consecutive blocks and hand each solved block to the later CTAs of the
// cluster directly into their shared memory (st.async, completed on a
// transaction barrier), so CL - 1 of every CL steps of the chain skip the
// global-memory round trip; blocks of earlier clusters still come from the
// published words.  Every CTA of a cluster arrives at a final cluster
// barrier before it exits, so no CTA leaves while another may still write
// into its shared memory.
template <int CL>
__global__ void __launch_bounds__(kThreads, 2)
    strsv_tma_kernel(const __grid_constant__ CUtensorMap amap, int n, int lower_op, int op, int unit, float* x,
                     long incx, unsigned long long* pub, unsigned* ticket, unsigned* epoch_word, int* status)
{
    extern __shared__ unsigned char smem_raw[];
    FastSmem& S = *reinterpret_cast<FastSmem*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    float(*IV)[NB + 1] = reinterpret_cast<float(*)[NB + 1]>(&S.R[0][0]);
    float(*W)[NB + 1] = IV + NB;
    const int t = threadIdx.x;
    const int nb = (n + NB - 1) / NB;
    const unsigned rank = CL > 1 ? cluster_rank() : 0u;
    if (t == 0) {
        unsigned e = *(volatile unsigned*)epoch_word + 1u;
        S.epoch = e == 0u ? 1u : e;
        if (CL == 1) S.s = atomicAdd(ticket, 1u);
        for (int i = 0; i < FS; ++i) tma::mbar_init(&S.full[i], 1);
        S.failed = 0;
        if constexpr (CL > 1) {
            // one arrival (this one, declaring the bytes) plus NB floats per earlier rank
            for (unsigned r = 0; r < (unsigned)CL; ++r) tma::mbar_init(&S.xbar[r], 1);
            tma::mbar_init_fence();
            for (unsigned r = 0; r < rank; ++r) tma::mbar_expect_tx(&S.xbar[r], NB * 4);
        } else {
            tma::mbar_init_fence();
        }
    }
    if constexpr (CL > 1) {
        // every CTA of the cluster has started and set up its barriers before
        // any shared memory of another CTA is written
        __syncthreads();
        cluster_sync_all();
        if (rank == 0 && t == 0) {
            const unsigned c = atomicAdd(ticket, 1u);
            for (unsigned r = 0; r < (unsigned)CL; ++r) st_cluster_u32(map_to(&S.cl, r), c);
            if (c == gridDim.x / CL - 1) *ticket = 0u;  // every ticket of this launch is taken
        }
        cluster_sync_all();
        if (t == 0) S.s = S.cl * CL + rank;
    }
    __syncthreads();
    const int s = (int)S.s;
    const unsigned epoch = S.epoch;
    const int cfirst = CL > 1 ? (int)S.cl * CL : 0;  // first block (solve order) of this cluster
    if (CL == 1 && s == nb - 1 && t == 0) *ticket = 0u;  // every ticket of this launch is taken
    if (CL > 1 && s >= nb) {  // a cluster's spare CTA past the last block
        cluster_sync_all();
        return;
    }
    auto blk = [&](int p) { return lower_op ? p : nb - 1 - p; };
    const int kb = blk(s), r0 = kb * NB, nr = min(NB, n - r0);
    // loads: 0 the diagonal block, 1 the tile of block s-1 (s >= 1), then the
    // tiles of blocks 0 .. s-2 in solve order
    const int nloads = s + 1;
    auto load_block = [&](int i) { return i == 0 ? kb : (i == 1 ? blk(s - 1) : blk(i - 2)); };
    int issued = 0;  // (thread 0)
    auto issue = [&](int i) {
        issued = i + 1;
        const int cb = load_block(i);
        uint64_t* bar = &S.full[i % FS];
        tma::mbar_expect_tx(bar, TILE_ELEMS * 4);
        if (op == 0) tma::load_2d(S.stage[i % FS], &amap, r0, cb * NB, bar);   // A[r0.., cb*NB..]
        else tma::load_2d(S.stage[i % FS], &amap, cb * NB, r0, bar);           // A[cb*NB.., r0..]
    };
    if (t == 0)
        for (int i = 0; i < min(FS, nloads); ++i) issue(i);
    const float b = t < nr ? x[(long)(r0 + t) * incx] : 0.f;
    // on a failed wait: record it, let this CTA's copies still in flight land
    // (each wait bounded), then leave
    auto bail = [&](int consumed) {
        if (t == 0) {
            atomicOr(status, (int)kDevWaitTimeout);
            for (int j = consumed; j < issued; ++j)
                tma::mbar_wait_bounded(&S.full[j % FS], (j / FS) & 1, kTrsvWaitNs);
            // bytes other CTAs of the cluster may still be sending here
            if constexpr (CL > 1)
                for (unsigned r = 0; r < rank; ++r) xbar_wait_bounded(&S.xbar[r], kTrsvWaitNs);
        }
        if constexpr (CL > 1) {
            __syncthreads();
            cluster_sync_all();
        }
    };
    // waits for the solved entries of the block with solve index p (row c0,
    // nc rows): from this CTA's shared memory when an earlier CTA of the
    // cluster solved it, else from the published words (threads t < 64 poll)
    auto fetch_x = [&](int p, int c0, int nc) -> int {
        int bad = 0;
        if (CL > 1 && p >= cfirst) {
            const int src = p - cfirst;
            if (t < NB) {
                if (!xbar_wait_bounded(&S.xbar[src], kTrsvWaitNs)) {
                    atomicOr(status, (int)kDevWaitTimeout);
                    bad = 1;
                }
                S.xs[t] = t < nc ? S.xin[src][t] : 0.f;
            }
            return bad;
        }
        if (t < NB) {
            float v = 0.f;
            if (t < nc) {
                const unsigned long long* src = pub + c0 + t;
                unsigned long long w = ld_relaxed_u64(src);
                if ((unsigned)(w >> 32) != epoch) {
                    const unsigned long long t0 = tma::global_ns();
                    for (;;) {
                        w = ld_relaxed_u64(src);
                        if ((unsigned)(w >> 32) == epoch) break;
                        if (ld_volatile(status) != kDevOk) { bad = 1; break; }
                        if (tma::global_ns() - t0 > kTrsvWaitNs) {
                            atomicOr(status, (int)kDevWaitTimeout);
                            bad = 1;
                            break;
                        }
                    }
                }
                v = __uint_as_float((unsigned)w);
            }
            S.xs[t] = v;
        }
        return bad;
    };
    const int rN = t % NB, gN = t / NB;      // row, group of 16 columns
    // element (r, c) of the op(A) tile in a stage
    auto tile = [&](const float* T, int r, int c) { return op == 0 ? T[c * NB + r] : T[r * NB + c]; };

    // ---- diagonal block: FP64 inverse, then FP32
    int bad = tma::mbar_wait_bounded(&S.full[0], 0, kTrsvWaitNs) ? 0 : 1;
    if (__syncthreads_or(bad)) {
        bail(0);
        return;
    }
    {
        // Blocked FP64 inverse on all threads: the four 16 x 16 diagonal
        // blocks by substitution (one column per thread), then two doubling
        // steps that form the off-diagonal blocks from products of the known
        // inverses (16 -> 32 -> 64).  Rows and columns past nr are an identity
        // (the box holds zeros there) and are cut off when the inverse is
        // stored in FP32.  (One column per thread over all 64 rows took 44 us
        // of every call's start.)
        const float* D = S.stage[0];
        auto d = [&](int r, int c) -> double { return (double)tile(D, r, c); };
        double* rd = &S.Tm[0][0];  // 1 / diagonal, then the doubling temporary
        for (int idx = t; idx < TILE_ELEMS; idx += kThreads) S.R[idx % NB][idx / NB] = 0.0;
        if (t < NB) rd[t] = (unit || t >= nr) ? 1.0 : 1.0 / d(t, t);
        __syncthreads();
        if (t < NB) {
            // thread t owns column j of diagonal block b; the column stays in
            // registers (loops unrolled: the D reads pipeline)
            const int b = (t / 16) * 16, j = t % 16;
            double y[16];
            if (lower_op) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    double acc = (i == j) ? 1.0 : 0.0;
#pragma unroll
                    for (int k = 0; k < i; ++k) acc = fma(-d(b + i, b + k), y[k], acc);
                    y[i] = (i >= j) ? acc * rd[b + i] : 0.0;
                }
            } else {
#pragma unroll
                for (int i = 15; i >= 0; --i) {
                    double acc = (i == j) ? 1.0 : 0.0;
#pragma unroll
                    for (int k = i + 1; k < 16; ++k) acc = fma(-d(b + i, b + k), y[k], acc);
                    y[i] = (i <= j) ? acc * rd[b + i] : 0.0;
                }
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) S.R[b + i][b + j] = y[i];
        }
        __syncthreads();
        // doubling (h = 16, then 32), loops unrolled at compile-time h with two
        // partial sums per output
        auto doubling = [&](auto hc) {
            constexpr int h = decltype(hc)::value;
            constexpr int nout = (NB / (2 * h)) * h * h;
            // T = C Y11 (lower: C the block below Y11) or C Y22 (upper: C right of Y11)
            for (int idx = t; idx < nout; idx += kThreads) {
                const int pr = idx / (h * h), e = idx % (h * h), r = e % h, c = e / h, o = pr * 2 * h;
                double a0 = 0.0, a1 = 0.0;
#pragma unroll
                for (int k = 0; k < h; k += 2) {
                    if (lower_op) {
                        a0 = fma(d(o + h + r, o + k), S.R[o + k][o + c], a0);
                        a1 = fma(d(o + h + r, o + k + 1), S.R[o + k + 1][o + c], a1);
                    } else {
                        a0 = fma(d(o + r, o + h + k), S.R[o + h + k][o + h + c], a0);
                        a1 = fma(d(o + r, o + h + k + 1), S.R[o + h + k + 1][o + h + c], a1);
                    }
                }
                S.Tm[pr * h + r][c] = a0 + a1;
            }
            __syncthreads();
            // the off-diagonal block of the inverse: -Y22 T (lower) or -Y11 T (upper)
            for (int idx = t; idx < nout; idx += kThreads) {
                const int pr = idx / (h * h), e = idx % (h * h), r = e % h, c = e / h, o = pr * 2 * h;
                double a0 = 0.0, a1 = 0.0;
#pragma unroll
                for (int k = 0; k < h; k += 2) {
                    if (lower_op) {
                        a0 = fma(S.R[o + h + r][o + h + k], S.Tm[pr * h + k][c], a0);
                        a1 = fma(S.R[o + h + r][o + h + k + 1], S.Tm[pr * h + k + 1][c], a1);
                    } else {
                        a0 = fma(S.R[o + r][o + k], S.Tm[pr * h + k][c], a0);
                        a1 = fma(S.R[o + r][o + k + 1], S.Tm[pr * h + k + 1][c], a1);
                    }
                }
                if (lower_op) S.R[o + h + r][o + c] = -(a0 + a1);
                else S.R[o + r][o + h + c] = -(a0 + a1);
            }
            __syncthreads();
        };
        doubling(std::integral_constant<int, 16>{});
        doubling(std::integral_constant<int, 32>{});
        // rows and columns past nr: zero
        for (int idx = t; idx < TILE_ELEMS; idx += kThreads) {
            const int r = idx % NB, c = idx / NB;
            if (r >= nr || c >= nr) S.R[r][c] = 0.0;
        }
    }
    __syncthreads();
    {
        float v[TILE_ELEMS / kThreads];
#pragma unroll
        for (int u = 0; u < TILE_ELEMS / kThreads; ++u) {
            const int idx = t + kThreads * u;
            v[u] = (float)S.R[idx % NB][idx / NB];
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < TILE_ELEMS / kThreads; ++u) {
            const int idx = t + kThreads * u;
            IV[idx % NB][idx / NB] = v[u];
        }
    }
    __syncthreads();
    if (t == 0 && FS < nloads) issue(FS);

    // ---- W = inv(D) T for the tile of block s-1
    if (s >= 1) {
        bad = tma::mbar_wait_bounded(&S.full[1], 0, kTrsvWaitNs) ? 0 : 1;
        if (__syncthreads_or(bad)) {
            bail(1);
            return;
        }
        const float* T = S.stage[1];
        float acc[16];
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) acc[jj] = 0.f;
        for (int k = 0; k < NB; ++k) {
            const float a = IV[rN][k];
#pragma unroll
            for (int jj = 0; jj < 16; ++jj) acc[jj] = fmaf(a, tile(T, k, gN * 16 + jj), acc[jj]);
        }
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) W[rN][gN * 16 + jj] = acc[jj];
        __syncthreads();
        if (t == 0 && FS + 1 < nloads) issue(FS + 1);
    }

    // ---- the other earlier blocks, in solve order
    const int lane = t & 31, warp = t >> 5;
    float accN = 0.f;
    float accT[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) accT[i] = 0.f;
    for (int i = 2; i <= s; ++i) {
        const int c0 = blk(i - 2) * NB, nc = min(NB, n - c0);
        bad = tma::mbar_wait_bounded(&S.full[i % FS], (i / FS) & 1, kTrsvWaitNs) ? 0 : 1;
        bad |= fetch_x(i - 2, c0, nc);
        if (__syncthreads_or(bad)) {
            bail(i);
            return;
        }
        const float* T = S.stage[i % FS];
        if (op == 0) {
#pragma unroll
            for (int jj = 0; jj < 16; ++jj) {
                const int c = gN * 16 + jj;
                accN = fmaf(-T[c * NB + rN], S.xs[c], accN);
            }
        } else {
            const float x0 = S.xs[lane], x1 = S.xs[lane + 32];
#pragma unroll
            for (int ii = 0; ii < 8; ++ii) {
                const int r = warp * 8 + ii;
                accT[ii] = fmaf(-T[r * NB + lane], x0, accT[ii]);
                accT[ii] = fmaf(-T[r * NB + lane + 32], x1, accT[ii]);
            }
        }
        __syncthreads();
        if (t == 0 && i + FS < nloads) issue(i + FS);
    }

    // ---- z = inv(D) (b - row sums)
    if (op == 0) {
        S.part[gN][rN] = accN;
    } else {
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) {
            const float v = warp_sum(accT[ii]);
            if (lane == 0) S.part[0][warp * 8 + ii] = v;
        }
    }
    __syncthreads();
    if (t < NB) {
        const float sum = op == 0 ? (S.part[0][t] + S.part[1][t]) + (S.part[2][t] + S.part[3][t]) : S.part[0][t];
        S.ys[t] = t < nr ? b + sum : 0.f;
    }
    __syncthreads();
    {
        float acc = 0.f;
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) acc = fmaf(IV[rN][gN * 16 + jj], S.ys[gN * 16 + jj], acc);
        S.part[gN][rN] = acc;
    }
    __syncthreads();
    if (t < NB) S.zs[t] = (S.part[0][t] + S.part[1][t]) + (S.part[2][t] + S.part[3][t]);

    // ---- this block's step of the chain: x = z - W x_prev, on the 64
    // threads that own the rows: from the arrival of x_prev to the hand-off
    // of x there is no block-wide barrier (the global path synchronises the
    // two warps only)
    if (t < NB) {
        float xf = S.zs[t];
        bool ok = true;
        if (s >= 1) {
            const int p = s - 1, c0 = blk(p) * NB, nc = min(NB, n - c0);
            const float* xp = S.xs;
            if (CL > 1 && p >= cfirst) {
                ok = xbar_wait_bounded(&S.xbar[p - cfirst], kTrsvWaitNs);
                xp = S.xin[p - cfirst];
            } else {
                float v = 0.f;
                if (t < nc) {
                    const unsigned long long* src = pub + c0 + t;
                    unsigned long long w = ld_relaxed_u64(src);
                    if ((unsigned)(w >> 32) != epoch) {
                        const unsigned long long t0 = tma::global_ns();
                        for (;;) {
                            w = ld_relaxed_u64(src);
                            if ((unsigned)(w >> 32) == epoch) break;
                            if (ld_volatile(status) != kDevOk || tma::global_ns() - t0 > kTrsvWaitNs) {
                                ok = false;
                                break;
                            }
                        }
                    }
                    v = __uint_as_float((unsigned)w);
                }
                S.xs[t] = v;
                asm volatile("bar.sync 1, %0;" ::"n"(NB) : "memory");  // the 64 row threads
            }
            float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
            for (int j = 0; j < NB; j += 4) {
                a0 = fmaf(W[t][j], xp[j], a0);
                a1 = fmaf(W[t][j + 1], xp[j + 1], a1);
                a2 = fmaf(W[t][j + 2], xp[j + 2], a2);
                a3 = fmaf(W[t][j + 3], xp[j + 3], a3);
            }
            xf -= (a0 + a1) + (a2 + a3);
        }
        if (ok) {
            if (t < nr) {
                x[(long)(r0 + t) * incx] = xf;
                st_relaxed_u64(pub + r0 + t, ((unsigned long long)epoch << 32) | __float_as_uint(xf));
            }
            // hand the block to the later CTAs of the cluster that have blocks
            if constexpr (CL > 1) {
                const float v = t < nr ? xf : 0.f;
                for (unsigned d = rank + 1u; d < (unsigned)CL && cfirst + (int)d < nb; ++d)
                    st_async_f32(map_to(&S.xin[rank][t], d), v, map_to(&S.xbar[rank], d));
            }
        } else {
            atomicOr(status, (int)kDevWaitTimeout);
            S.failed = 1;
        }
    }
    __syncthreads();
    if (t == 0) {
        // after a failed wait, let bytes other CTAs of the cluster may still
        // send land before leaving (each wait bounded)
        if constexpr (CL > 1)
            if (S.failed)
                for (unsigned r = 0; r < rank; ++r) xbar_wait_bounded(&S.xbar[r], kTrsvWaitNs);
        if (s == nb - 1) *(volatile unsigned*)epoch_word = epoch;
    }
    if constexpr (CL > 1) cluster_sync_all();
}

cudaError_t strsv_tma(iclblasHandle_t h, int uplo, int trans, int diag, int n, const float* A, int lda, float* x,
                      int incx, bool& used)
{
    used = false;
    CUtensorMap map;
    if (lda < n || !tma::map_f32_colmajor(&map, A, n, n, lda, NB, NB)) return cudaSuccess;
    if ((size_t)n > h->ws.pub_elems) {
        if (h->ws.pub) cudaFree(h->ws.pub);
        h->ws.pub = nullptr;
        h->ws.pub_elems = 0;
        cudaError_t e = cudaMalloc(&h->ws.pub, (size_t)n * sizeof(unsigned long long));
        if (e != cudaSuccess) return e;
        e = cudaMemsetAsync(h->ws.pub, 0, (size_t)n * sizeof(unsigned long long), h->stream);
        if (e != cudaSuccess) return e;
        h->ws.pub_elems = n;
    }
    const int smem = (int)sizeof(FastSmem) + 1024;
    static int smem_set = 0;
    if (!smem_set) {
        cudaError_t e = cudaFuncSetAttribute(strsv_tma_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(strsv_tma_kernel<kMaxCluster>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        smem_set = 1;
    }
    const int op = trans == ICLBLAS_OP_N ? 0 : 1;
    const bool lower = uplo == ICLBLAS_FILL_MODE_LOWER;
    const int lower_op = (op == 0) ? lower : !lower;
    const int nb = (n + NB - 1) / NB;
    const int unit = diag == ICLBLAS_DIAG_UNIT;
    unsigned* ticket = h->ws.counters;
    unsigned* epoch_word = h->ws.counters + kCounterWords - 1;
    // clusters of 8 consecutive blocks when the GPU can hold one (and there
    // is more than one block); else one CTA per block
    if (nb > 1) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kMaxCluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3((unsigned)((nb + kMaxCluster - 1) / kMaxCluster * kMaxCluster));
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = h->stream;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, strsv_tma_kernel<kMaxCluster>, &cfg) == cudaSuccess &&
            clusters > 0) {
            cudaError_t e = cudaLaunchKernelEx(&cfg, strsv_tma_kernel<kMaxCluster>, map, n, lower_op, op, unit, x,
                                               (long)incx, h->ws.pub, ticket, epoch_word, h->ws.dev_status);
            if (e != cudaSuccess) return e;
            used = true;
            return cudaGetLastError();
        }
        cudaGetLastError();
    }
    strsv_tma_kernel<1><<<nb, kThreads, smem, h->stream>>>(map, n, lower_op, op, unit, x, incx, h->ws.pub, ticket,
                                                           epoch_word, h->ws.dev_status);
    used = true;
    return cudaGetLastError();
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
    bool used = false;
    cudaError_t e = strsv_tma(h, uplo, trans, diag, n, A, lda, x, incx, used);
    if (e != cudaSuccess || used) return e;
    return trsv_impl<float>(h, uplo, trans == ICLBLAS_OP_C ? ICLBLAS_OP_T : trans, diag, n, A, lda, x, incx);
}

cudaError_t ctrsv(iclblasHandle_t h, int uplo, int trans, int diag, int n, const cfloat* A, int lda, cfloat* x,
                  int incx)
{
    return trsv_impl<cfloat>(h, uplo, trans, diag, n, A, lda, x, incx);
}

}  // namespace iclb
