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
#include <atomic>
#include <cstddef>
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
// blocks of RB = 128 rows, one CTA of 256 threads per block (one CTA per SM),
// and changes that shorten the chain of dependent block solves:
//   - tiles arrive by TMA (boxes of 128 rows x 64 columns of op(A), half a
//     block's columns each) into a 6-stage shared-memory ring, so 192 KiB per
//     CTA are in flight while the CTA waits for earlier blocks;
//   - the first two boxes are the diagonal block D, inverted in FP64: both
//     64 x 64 diagonal halves at once (16 x 16 blocks by substitution, then
//     two doubling steps), then the off-diagonal half from those two
//     (-inv(D22) D21 inv(D11) for a lower D), each product register-tiled.
//     The inverse is kept in FP32 in registers: each thread holds 4 rows x
//     16 columns, so a product with a vector takes 4 16-byte shared-memory
//     reads per thread (not 64 broadcast words: 8 warps reading a vector
//     word by word spend the SM's shared-memory bandwidth) and a butterfly
//     over the 8 lanes sharing the rows.  The FP64 workspace overlays the
//     ring before the ring is used;
//   - the next two boxes are the tile T next to D (the block solved just
//     before this one), kept in registers in the same layout; then the
//     remaining tiles in solve order, consumed with 16-byte reads along the
//     stage's contiguous direction into per-thread partial row sums.  Once
//     all but the last earlier block are known, the CTA holds
//     y = b - (sum of those tiles' products), so its own step of the chain,
//     when the last block x_prev is published, is x = inv(D) (y - T x_prev):
//     two register products with one barrier between them, and the
//     publication;
//   - each solved entry is published as one 64-bit word (value, call epoch):
//     a consumer polls the entries it needs directly, with no separate flag.
//     The epoch lives in device memory: each CTA reads the last launch's
//     epoch at its start and uses the next one; the CTA that solves the last
//     block stores it back once everything is published (every other CTA has
//     read it by then), so replays of a captured launch get fresh epochs;
//   - launched as clusters of CL consecutive blocks, a solved block also goes
//     straight into the shared memory of the later CTAs of its cluster
//     (st.async on a transaction barrier), so CL - 1 of every CL steps of the
//     chain skip the global-memory round trip.  CL is the largest size from
//     8 down to 2 for which the GPU holds every cluster of the launch at once
//     (a cluster that can only start when another has finished starts its
//     own setup late and then streams its tiles alone).
// Against 64-row blocks (two CTAs per SM, n = 16384 in 230 us) the chain has
// half the steps and half the hand-offs between clusters.
constexpr int RB = 128;  // rows (and columns) of a block
constexpr int HB = 64;   // columns of op(A) in one stage
constexpr int STAGE_ELEMS = RB * HB;
constexpr int FS = 6;
constexpr int kMaxCluster = 8;
constexpr int XQ = 8 * 20;  // a block's 128 entries in shared memory: 8 groups of 16, 20 floats apart
constexpr unsigned long long kTrsvWaitNs = 2000000000ull;  // a wait gives up after 2 s

// shared-memory index of entry c (0 .. 127) of a block's entries (the
// padding keeps the 16-byte reads of 8 threads with different groups in
// different banks)
__device__ __forceinline__ int qidx(int c) { return (c >> 4) * 20 + (c & 15); }

// FP64 workspace of the diagonal-block inverse, in doubles: the inverses of
// the two 64 x 64 diagonal halves, the off-diagonal half, and two doubling
// temporaries.  It starts at stage 2 of the ring.
constexpr int kY = HB * (HB + 1);
constexpr int kTm = 32 * 33;
constexpr int kInvDoubles = 3 * kY + 2 * kTm;
static_assert(kInvDoubles * 8 <= (FS - 2) * STAGE_ELEMS * 4, "inverse workspace inside the ring");

struct FastSmem {
    float stage[FS][STAGE_ELEMS];
    // cluster launches: the solved blocks of the earlier CTAs of this
    // cluster, delivered into this CTA's shared memory by st.async, one
    // transaction barrier per source rank
    float xin[kMaxCluster][XQ];
    float xs[XQ];  // entries of the block being streamed, from the published words
    float xp[XQ];  // x_prev, from the published words
    float y[XQ];   // b - the products of the tiles of blocks 0 .. s-2
    float y2[XQ];  // y - T x_prev
    float part[16][RB];  // partial row sums of the streamed tiles
    uint64_t xbar[kMaxCluster];
    uint64_t full[FS];
    unsigned s, epoch, cl;
    int failed;  // a wait of the chain step gave up
};
static_assert(sizeof(FastSmem) + 1024 <= 232448, "STRSV shared memory");
static_assert(offsetof(FastSmem, xin) % 16 == 0 && offsetof(FastSmem, xs) % 16 == 0 &&
                  offsetof(FastSmem, xp) % 16 == 0 && offsetof(FastSmem, y) % 16 == 0 &&
                  offsetof(FastSmem, y2) % 16 == 0,
              "16-byte reads of block entries");

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
// 16 bytes into another CTA's shared memory (16-byte aligned), counted as
// transaction bytes on that CTA's barrier
__device__ __forceinline__ void st_async_f32x4(uint32_t addr, float a, float b, float c, float d, uint32_t bar)
{
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.f32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(
                     addr),
                 "f"(a), "f"(b), "f"(c), "f"(d), "r"(bar)
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
// polls a published (value, epoch) word until it carries `epoch`; false when
// the wait gives up or another CTA has recorded a failure
__device__ __forceinline__ bool poll_word(const unsigned long long* src, unsigned epoch, const int* status,
                                          float& v)
{
    unsigned long long w = ld_relaxed_u64(src);
    if ((unsigned)(w >> 32) != epoch) {
        const unsigned long long t0 = tma::global_ns();
        for (;;) {
            w = ld_relaxed_u64(src);
            if ((unsigned)(w >> 32) == epoch) break;
            if (ld_volatile(status) != kDevOk || tma::global_ns() - t0 > kTrsvWaitNs) return false;
        }
    }
    v = __uint_as_float((unsigned)w);
    return true;
}

// FP64 product tile of the diagonal-block inverse: acc(i, j) = sum_k A(r, k)
// B(k, c) for rows r = r0 + i*rs and columns c = c0 + j*cs (interleaved, so
// that a warp reads consecutive columns of B and few rows of A)
template <int TR, int TC, int K, class FA, class FB>
__device__ __forceinline__ void dtile(double (&acc)[TR][TC], int r0, int rs, int c0, int cs, FA A, FB B)
{
#pragma unroll
    for (int i = 0; i < TR; ++i)
#pragma unroll
        for (int j = 0; j < TC; ++j) acc[i][j] = 0.0;
#pragma unroll 4
    for (int k = 0; k < K; ++k) {
        double a[TR], b[TC];
#pragma unroll
        for (int i = 0; i < TR; ++i) a[i] = A(r0 + i * rs, k);
#pragma unroll
        for (int j = 0; j < TC; ++j) b[j] = B(k, c0 + j * cs);
#pragma unroll
        for (int i = 0; i < TR; ++i)
#pragma unroll
            for (int j = 0; j < TC; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
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
__global__ void __launch_bounds__(kThreads, 1)
    strsv_tma_kernel(const __grid_constant__ CUtensorMap amap, int n, int lower_op, int op, int unit, float* x,
                     long incx, unsigned long long* pub, unsigned* ticket, unsigned* epoch_word, int* status)
{
    extern __shared__ unsigned char smem_raw[];
    // 1024-byte aligned; an offset from the array (not an integer cast) keeps
    // the accesses in the shared address space
    FastSmem& S = *reinterpret_cast<FastSmem*>(smem_raw + ((1024u - (tma::smem_u32(smem_raw) & 1023u)) & 1023u));
    const int t = threadIdx.x;
    const int nb = (n + RB - 1) / RB;
    const unsigned rank = CL > 1 ? cluster_rank() : 0u;
    if (t == 0) {
        unsigned e = *(volatile unsigned*)epoch_word + 1u;
        S.epoch = e == 0u ? 1u : e;
        if (CL == 1) S.s = atomicAdd(ticket, 1u);
        for (int i = 0; i < FS; ++i) tma::mbar_init(&S.full[i], 1);
        S.failed = 0;
        if constexpr (CL > 1) {
            // one arrival (this one, declaring the bytes) plus RB floats per earlier rank
            for (unsigned r = 0; r < (unsigned)CL; ++r) tma::mbar_init(&S.xbar[r], 1);
            tma::mbar_init_fence();
            for (unsigned r = 0; r < rank; ++r) tma::mbar_expect_tx(&S.xbar[r], RB * 4);
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
    const int kb = blk(s), r0 = kb * RB, nr = min(RB, n - r0);
    // loads, numbered: 0 and 1 the two halves of D; 2 and 3 the halves of the
    // tile of block s-1 (s >= 1); then 4 + 2i + h half h of the tile of block
    // i, i = 0 .. s-2 in solve order.  Load L goes to stage L % FS and
    // completes phase L / FS of that stage's barrier; it is issued once load
    // L - FS has been consumed.
    const int nloads = s == 0 ? 2 : 4 + 2 * (s - 1);
    int issued = 0;  // (thread 0)
    auto issue = [&](int L) {
        issued = L + 1;
        const int cb = L < 2 ? kb : (L < 4 ? blk(s - 1) : blk((L - 4) >> 1));
        const int c = cb * RB + (L & 1) * HB;
        uint64_t* bar = &S.full[L % FS];
        tma::mbar_expect_tx(bar, STAGE_ELEMS * 4);
        if (op == 0) tma::load_2d(S.stage[L % FS], &amap, r0, c, bar);  // A[r0 .. +127, c .. +63]
        else tma::load_2d(S.stage[L % FS], &amap, c, r0, bar);          // A[c .. +63, r0 .. +127]
    };
    auto wait_load = [&](int L) { return tma::mbar_wait_bounded(&S.full[L % FS], (L / FS) & 1, kTrsvWaitNs); };
    if (t == 0) {
        issue(0);
        issue(1);
        // the tiles needed first after the inverse (block s-1's, then block
        // 0's) start towards L2 now, while the inverse is formed
        for (int L = 2; L < min(6, nloads); ++L) {
            const int cb = L < 4 ? blk(s - 1) : blk(0);
            const int c = cb * RB + (L & 1) * HB;
            if (op == 0) tma::prefetch_2d(&amap, r0, c);
            else tma::prefetch_2d(&amap, c, r0);
        }
    }
    const float b = (t < nr) ? x[(long)(r0 + t) * incx] : 0.f;  // (threads t < RB)
    // on a failed wait: record it, let this CTA's copies still in flight land
    // (each wait bounded), then leave
    auto bail = [&](int consumed) {
        if (t == 0) {
            atomicOr(status, (int)kDevWaitTimeout);
            for (int L = consumed; L < issued; ++L) wait_load(L);
            // bytes other CTAs of the cluster may still be sending here
            if constexpr (CL > 1)
                for (unsigned r = 0; r < rank; ++r) xbar_wait_bounded(&S.xbar[r], kTrsvWaitNs);
        }
        if constexpr (CL > 1) {
            __syncthreads();
            cluster_sync_all();
        }
    };
    // the solved entries of the block with solve index p: this CTA's own
    // shared memory when an earlier CTA of the cluster solved it (every
    // thread waits on the transaction barrier), else the published words
    // (threads t < RB poll, into `buf`; the caller's barrier publishes them)
    auto fetch_x = [&](int p, float* buf, int& bad) -> const float* {
        if (CL > 1 && p >= cfirst) {
            if (!xbar_wait_bounded(&S.xbar[p - cfirst], kTrsvWaitNs)) {
                atomicOr(status, (int)kDevWaitTimeout);
                bad = 1;
            }
            return S.xin[p - cfirst];
        }
        const int c0 = blk(p) * RB, nc = min(RB, n - c0);
        if (t < RB) {
            float v = 0.f;
            if (t < nc && !poll_word(pub + c0 + t, epoch, status, v)) {
                atomicOr(status, (int)kDevWaitTimeout);
                bad = 1;
            }
            buf[qidx(t)] = v;
        }
        return buf;
    };
    // op(A) element (r, c) of a stage: r < 128, c < 64
    auto el = [&](const float* T, int r, int c) { return op == 0 ? T[c * RB + r] : T[r * HB + c]; };
    // register layout of a 128 x 128 matrix (inv(D), and the tile of block
    // s-1): the thread holds rows R0 .. R0+3, columns cg*16 .. cg*16+15
    const int lane = t & 31, warp = t >> 5;
    const int cg = lane & 7, R0 = warp * 16 + (lane >> 3) * 4;
    // out[k] = row R0+k of M times v (v in the block-entry layout), in every
    // lane of the 8 that share the rows: 4 16-byte reads, 64 FMAs, and a
    // butterfly over the column groups
    auto mv = [&](const float(&m)[4][16], const float* v, float(&out)[4]) {
        const float* vp = v + cg * 20;
        float4 q[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) q[i] = *reinterpret_cast<const float4*>(vp + 4 * i);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float a0 = 0.f, a1 = 0.f;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                a0 = fmaf(m[k][4 * i], q[i].x, a0);
                a1 = fmaf(m[k][4 * i + 1], q[i].y, a1);
                a0 = fmaf(m[k][4 * i + 2], q[i].z, a0);
                a1 = fmaf(m[k][4 * i + 3], q[i].w, a1);
            }
            out[k] = a0 + a1;
        }
#pragma unroll
        for (int o = 1; o < 8; o <<= 1)
#pragma unroll
            for (int k = 0; k < 4; ++k) out[k] += __shfl_xor_sync(0xffffffffu, out[k], o);
    };
    auto pick = [](const float(&o)[4], int k) { return k == 0 ? o[0] : (k == 1 ? o[1] : (k == 2 ? o[2] : o[3])); };

    // ---- diagonal block: FP64 inverse, kept in FP32 registers
    int bad = (wait_load(0) && wait_load(1)) ? 0 : 1;
    if (__syncthreads_or(bad)) {
        bail(0);
        return;
    }
    float iv[4][16];  // inv(D)[R0 + k][cg*16 + j]
    {
        double* ws = reinterpret_cast<double*>(&S.stage[2][0]);
        double(*Y)[HB][HB + 1] = reinterpret_cast<double(*)[HB][HB + 1]>(ws);   // inverses of D11, D22
        double(*Yc)[HB + 1] = reinterpret_cast<double(*)[HB + 1]>(ws + 2 * kY);  // the off-diagonal half
        double(*Tm)[32][33] = reinterpret_cast<double(*)[32][33]>(ws + 3 * kY);  // doubling temporaries
        // element (r, c) of D, r, c < 128; rows and columns past nr are zero (box fill)
        auto d = [&](int r, int c) -> double { return (double)el(S.stage[c >> 6], r, c & (HB - 1)); };
        double* rd = &Tm[0][0][0];  // 1 / diagonal, until the doubling steps use Tm
        for (int idx = t; idx < 2 * kY; idx += kThreads) (&Y[0][0][0])[idx] = 0.0;
        if (t < RB) rd[t] = (unit || t >= nr) ? 1.0 : 1.0 / d(t, t);
        __syncthreads();
        if (t < RB) {
            // thread t owns column j of the 16 x 16 diagonal block at b of
            // half hb; the column stays in registers
            const int hb = t >> 6, b = ((t & (HB - 1)) >> 4) * 16, j = t & 15, o = hb * HB + b;
            double y[16];
            if (lower_op) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    double acc = (i == j) ? 1.0 : 0.0;
#pragma unroll
                    for (int k = 0; k < i; ++k) acc = fma(-d(o + i, o + k), y[k], acc);
                    y[i] = (i >= j) ? acc * rd[o + i] : 0.0;
                }
            } else {
#pragma unroll
                for (int i = 15; i >= 0; --i) {
                    double acc = (i == j) ? 1.0 : 0.0;
#pragma unroll
                    for (int k = i + 1; k < 16; ++k) acc = fma(-d(o + i, o + k), y[k], acc);
                    y[i] = (i <= j) ? acc * rd[o + i] : 0.0;
                }
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) Y[hb][b + i][b + j] = y[i];
        }
        __syncthreads();
        // doubling inside both halves at once (h = 16, then 32): the
        // off-diagonal h x h block of each 2h x 2h diagonal block is
        // -Y22 C Y11 (lower: C below Y11) or -Y11 C Y22 (upper: C right of
        // Y11).  64 / h products of h x h at a time, a TR x TC tile per thread
        auto doubling = [&](auto hc) {
            constexpr int h = decltype(hc)::value;
            constexpr int G = 64 / h, TPG = kThreads / G;  // products, threads per product
            constexpr int TR = 2, TC = h / 8, RS = h / TR;  // 8 thread columns, RS thread rows
            const int gid = t / TPG, u = t % TPG, hb = gid / (G / 2), pr = gid % (G / 2);
            const int ob = hb * HB, o = pr * 2 * h, tr = u / 8, tcl = u % 8;
            double acc[TR][TC];
            if (lower_op)
                dtile<TR, TC, h>(
                    acc, tr, RS, tcl, 8, [&](int r, int k) { return d(ob + o + h + r, ob + o + k); },
                    [&](int k, int c) { return Y[hb][o + k][o + c]; });
            else
                dtile<TR, TC, h>(
                    acc, tr, RS, tcl, 8, [&](int r, int k) { return d(ob + o + r, ob + o + h + k); },
                    [&](int k, int c) { return Y[hb][o + h + k][o + h + c]; });
#pragma unroll
            for (int i = 0; i < TR; ++i)
#pragma unroll
                for (int j = 0; j < TC; ++j) Tm[hb][pr * h + tr + i * RS][tcl + 8 * j] = acc[i][j];
            __syncthreads();
            if (lower_op)
                dtile<TR, TC, h>(
                    acc, tr, RS, tcl, 8, [&](int r, int k) { return Y[hb][o + h + r][o + h + k]; },
                    [&](int k, int c) { return Tm[hb][pr * h + k][c]; });
            else
                dtile<TR, TC, h>(
                    acc, tr, RS, tcl, 8, [&](int r, int k) { return Y[hb][o + r][o + k]; },
                    [&](int k, int c) { return Tm[hb][pr * h + k][c]; });
#pragma unroll
            for (int i = 0; i < TR; ++i)
#pragma unroll
                for (int j = 0; j < TC; ++j) {
                    const int r = tr + i * RS, c = tcl + 8 * j;
                    if (lower_op) Y[hb][o + h + r][o + c] = -acc[i][j];
                    else Y[hb][o + r][o + h + c] = -acc[i][j];
                }
            __syncthreads();
        };
        doubling(std::integral_constant<int, 16>{});
        doubling(std::integral_constant<int, 32>{});
        // the off-diagonal half: lower D: -inv(D22) (D21 inv(D11)); upper D:
        // -inv(D11) (D12 inv(D22)); 4 x 4 outputs per thread
        {
            const int tr = t / 16, tcl = t % 16;
            double acc[4][4];
            if (lower_op)
                dtile<4, 4, HB>(
                    acc, tr, 16, tcl, 16, [&](int r, int k) { return d(HB + r, k); },
                    [&](int k, int c) { return Y[0][k][c]; });
            else
                dtile<4, 4, HB>(
                    acc, tr, 16, tcl, 16, [&](int r, int k) { return d(r, HB + k); },
                    [&](int k, int c) { return Y[1][k][c]; });
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) Yc[tr + 16 * i][tcl + 16 * j] = acc[i][j];
            __syncthreads();
            const int yl = lower_op ? 1 : 0;
            dtile<4, 4, HB>(
                acc, tr, 16, tcl, 16, [&](int r, int k) { return Y[yl][r][k]; },
                [&](int k, int c) { return Yc[k][c]; });
            __syncthreads();
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) Yc[tr + 16 * i][tcl + 16 * j] = -acc[i][j];
        }
        __syncthreads();
        // the inverse in FP32, row-major through stages 0 and 1 (16-byte word
        // f of row R at f ^ ((f >> 2) & 7)), then each thread's 4 x 16 block
        // from it: neither pass has bank conflicts (reading the FP64 pieces
        // straight into the register layout had 8-way conflicts and took 3 us).
        // Rows and columns past nr are cut off.
        {
            float4* Iv = reinterpret_cast<float4*>(&S.stage[0][0]);
            for (int idx = t; idx < RB * 32; idx += kThreads) {
                const int R = idx >> 5, f = idx & 31, C = 4 * f, rr = R & (HB - 1);
                const bool right = C >= HB;  // columns 64 .. 127
                const double* src;           // row R of the 64 x 64 piece holding the columns
                if (lower_op) src = R < HB ? (right ? nullptr : Y[0][rr]) : (right ? Y[1][rr] : Yc[rr]);
                else src = R < HB ? (right ? Yc[rr] : Y[0][rr]) : (right ? Y[1][rr] : nullptr);
                float v[4];
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    v[e] = (src != nullptr && R < nr && C + e < nr) ? (float)src[(C + e) & (HB - 1)] : 0.f;
                Iv[R * 32 + (f ^ (f >> 2 & 7))] = make_float4(v[0], v[1], v[2], v[3]);
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 v = Iv[(R0 + k) * 32 + ((cg * 4 + q) ^ cg)];
                    iv[k][4 * q] = v.x;
                    iv[k][4 * q + 1] = v.y;
                    iv[k][4 * q + 2] = v.z;
                    iv[k][4 * q + 3] = v.w;
                }
        }
        // D (stages 0, 1) and the FP64 workspace (stages 2 on) are free; the
        // stores to them come before the copies that reuse the stages
        tma::fence_proxy_async_smem();
        __syncthreads();
    }
    if (t == 0)
        for (int L = 2; L < min(2 + FS, nloads); ++L) issue(L);

    // ---- the tile T of block s-1, kept in registers in the same layout
    float tc[4][16];
    if (s >= 1) {
        bad = (wait_load(2) && wait_load(3)) ? 0 : 1;
        if (__syncthreads_or(bad)) {
            bail(2);
            return;
        }
        const float* T = S.stage[2 + (cg >> 2)];
        const int c0 = (cg & 3) * 16;  // first column inside the stage
        if (op == 0) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const float4 v = *reinterpret_cast<const float4*>(&T[(c0 + j) * RB + R0]);
                tc[0][j] = v.x;
                tc[1][j] = v.y;
                tc[2][j] = v.z;
                tc[3][j] = v.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 v = *reinterpret_cast<const float4*>(&T[(R0 + k) * HB + c0 + 4 * q]);
                    tc[k][4 * q] = v.x;
                    tc[k][4 * q + 1] = v.y;
                    tc[k][4 * q + 2] = v.z;
                    tc[k][4 * q + 3] = v.w;
                }
        }
        // the registers are not read until the chain step: the reads of
        // stages 2 and 3 must be complete before the copies that reuse them
        tma::fence_proxy_async_smem();
        __syncthreads();
        if (t == 0)
            for (int L = 2 + FS; L < min(4 + FS, nloads); ++L) issue(L);
    }

    // ---- the other earlier blocks, in solve order: y = b - their products.
    // Each thread keeps partial row sums in registers; 16-byte reads run
    // along the stage's contiguous direction.
    //   op N (stage column-major): rows 4*lane .. +3, columns warp*8 .. +7
    //   op T (stage row-major): rows (2*warp + lane/16)*8 .. +7, columns
    //   4*(lane%16) .. +3
    float acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = 0.f;
    for (int i = 0; i + 1 < s; ++i) {
        bad = 0;
        const float* xv = fetch_x(i, S.xs, bad);
        for (int hh = 0; hh < 2; ++hh) {
            const int L = 4 + 2 * i + hh;
            if (!wait_load(L)) bad = 1;
            if (__syncthreads_or(bad)) {
                bail(L);
                return;
            }
            const float* T = S.stage[L % FS];
            if (op == 0) {
                const int c0 = warp * 8;
                const float* xq = xv + qidx(hh * HB + c0);
                const float4 xa = *reinterpret_cast<const float4*>(xq);
                const float4 xb = *reinterpret_cast<const float4*>(xq + 4);
                const float xk[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const float4 v = *reinterpret_cast<const float4*>(&T[(c0 + k) * RB + 4 * lane]);
                    acc[0] = fmaf(-v.x, xk[k], acc[0]);
                    acc[1] = fmaf(-v.y, xk[k], acc[1]);
                    acc[2] = fmaf(-v.z, xk[k], acc[2]);
                    acc[3] = fmaf(-v.w, xk[k], acc[3]);
                }
            } else {
                const int cq = lane & 15, rb = (2 * warp + (lane >> 4)) * 8;
                const float4 xa = *reinterpret_cast<const float4*>(xv + qidx(hh * HB + 4 * cq));
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const float4 v = *reinterpret_cast<const float4*>(&T[(rb + k) * HB + 4 * cq]);
                    acc[k] = fmaf(-v.x, xa.x, acc[k]);
                    acc[k] = fmaf(-v.y, xa.y, acc[k]);
                    acc[k] = fmaf(-v.z, xa.z, acc[k]);
                    acc[k] = fmaf(-v.w, xa.w, acc[k]);
                }
            }
            __syncthreads();
            if (t == 0 && L + FS < nloads) issue(L + FS);
        }
    }
    if (op == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) S.part[warp][4 * lane + k] = acc[k];
    } else {
        const int cq = lane & 15, rb = (2 * warp + (lane >> 4)) * 8;
#pragma unroll
        for (int k = 0; k < 8; ++k) S.part[cq][rb + k] = acc[k];
    }
    __syncthreads();
    if (t < RB) {
        float sum = 0.f;
        const int np = op == 0 ? 8 : 16;
        for (int p = 0; p < np; ++p) sum += S.part[p][t];
        S.y[qidx(t)] = t < nr ? b + sum : 0.f;
    }
    __syncthreads();

    // ---- this block's step of the chain: x = inv(D) (y - T x_prev).  From
    // the arrival of x_prev to the hand-off of x: two register products and
    // one barrier (one more on the global path, after the polls)
    bool ok = true;
    float o[4];
    const int own = cg & 3, row = R0 + own;  // the row this lane publishes
    // hand-off: lane 4 + d sends rows R0 .. R0+3 to the later CTAs rank + 1 + d
    // and rank + 5 + d of the cluster (those that have blocks), 16 bytes
    // each; the remote addresses are formed here, off the critical path
    int ndst = 0;
    uint32_t dx0 = 0, db0 = 0, dx1 = 0, db1 = 0;
    if constexpr (CL > 1) {
        if (cg >= 4) {
            const unsigned d0 = rank + 1u + (unsigned)(cg - 4), d1 = d0 + 4u;
            if (d0 < (unsigned)CL && cfirst + (int)d0 < nb) {
                dx0 = map_to(&S.xin[rank][qidx(R0)], d0);
                db0 = map_to(&S.xbar[rank], d0);
                ndst = 1;
                if (d1 < (unsigned)CL && cfirst + (int)d1 < nb) {
                    dx1 = map_to(&S.xin[rank][qidx(R0)], d1);
                    db1 = map_to(&S.xbar[rank], d1);
                    ndst = 2;
                }
            }
        }
    }
    if (s >= 1) {
        const int p = s - 1;
        const float* xpv;
        if (CL > 1 && p >= cfirst) {
            ok = __all_sync(0xffffffffu, xbar_wait_bounded(&S.xbar[p - cfirst], kTrsvWaitNs));
            xpv = S.xin[p - cfirst];
        } else {
            const int c0 = blk(p) * RB, nc = min(RB, n - c0);
            if (t < RB) {
                float v = 0.f;
                if (t < nc && !poll_word(pub + c0 + t, epoch, status, v)) ok = false;
                S.xp[qidx(t)] = v;
            }
            ok = __syncthreads_and(ok);
            xpv = S.xp;
        }
        mv(tc, xpv, o);
        if (cg < 4) S.y2[qidx(row)] = S.y[qidx(row)] - pick(o, own);
    } else {
        if (cg < 4) S.y2[qidx(row)] = S.y[qidx(row)];
    }
    __syncthreads();
    mv(iv, S.y2, o);
    const float xf = pick(o, own);
    if (ok) {
        // the hand-offs first, then the published words; the output x last
        if (ndst > 0) {
            float v[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) v[k] = R0 + k < nr ? o[k] : 0.f;
            st_async_f32x4(dx0, v[0], v[1], v[2], v[3], db0);
            if (ndst > 1) st_async_f32x4(dx1, v[0], v[1], v[2], v[3], db1);
        }
        if (cg < 4 && row < nr) st_relaxed_u64(pub + r0 + row, ((unsigned long long)epoch << 32) | __float_as_uint(xf));
        if (cg < 4 && row < nr) x[(long)(r0 + row) * incx] = xf;
    } else {
        atomicOr(status, (int)kDevWaitTimeout);
        S.failed = 1;
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

// the number of clusters of CL CTAs of the STRSV kernel the current device
// holds at once (0: none), asked once per device and cluster size
template <int CL>
int strsv_cluster_capacity(int device, int smem)
{
    static std::atomic<int> cap[64];  // capacity + 1; 0: not asked yet
    std::atomic<int>& c = cap[device & 63];
    int v = c.load();
    if (v == 0) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = CL;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(CL);
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, strsv_tma_kernel<CL>, &cfg) != cudaSuccess) {
            cudaGetLastError();
            clusters = 0;
        }
        v = clusters + 1;
        c.store(v);
    }
    return v - 1;
}

template <int CL>
cudaError_t strsv_launch(iclblasHandle_t h, int smem, int nb, const CUtensorMap& map, int n, int lower_op, int op,
                         int unit, float* x, int incx, unsigned* ticket, unsigned* epoch_word)
{
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)((nb + CL - 1) / CL * CL));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = h->stream;
    cfg.attrs = attr;
    cfg.numAttrs = CL > 1 ? 1 : 0;
    cudaError_t e = cudaLaunchKernelEx(&cfg, strsv_tma_kernel<CL>, map, n, lower_op, op, unit, x, (long)incx,
                                       h->ws.pub, ticket, epoch_word, h->ws.dev_status);
    return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t strsv_tma(iclblasHandle_t h, int uplo, int trans, int diag, int n, const float* A, int lda, float* x,
                      int incx, bool& used)
{
    used = false;
    const int op = trans == ICLBLAS_OP_N ? 0 : 1;
    CUtensorMap map;
    // op N: boxes of 128 rows x 64 columns of A; op T: 64 rows x 128 columns
    if (lda < n || !tma::map_f32_colmajor(&map, A, n, n, lda, op == 0 ? RB : HB, op == 0 ? HB : RB))
        return cudaSuccess;
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
    // the attribute belongs to the current device's copy of each kernel
    static std::atomic<unsigned long long> smem_set{0};
    const unsigned long long bit = 1ull << (h->device & 63);
    if (!(smem_set.load() & bit)) {
        const void* kernels[] = {(const void*)strsv_tma_kernel<1>, (const void*)strsv_tma_kernel<2>,
                                 (const void*)strsv_tma_kernel<3>, (const void*)strsv_tma_kernel<4>,
                                 (const void*)strsv_tma_kernel<5>, (const void*)strsv_tma_kernel<6>,
                                 (const void*)strsv_tma_kernel<7>, (const void*)strsv_tma_kernel<8>};
        for (const void* k : kernels) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) return e;
        }
        smem_set.fetch_or(bit);
    }
    const bool lower = uplo == ICLBLAS_FILL_MODE_LOWER;
    const int lower_op = (op == 0) ? lower : !lower;
    const int nb = (n + RB - 1) / RB;
    const int unit = diag == ICLBLAS_DIAG_UNIT;
    unsigned* ticket = h->ws.counters;
    unsigned* epoch_word = h->ws.counters + kCounterWords - 1;
    used = true;
    if (nb > 1) {
        // the largest cluster size, 8 down to 2, for which every cluster of
        // the launch is resident at once (sizes need not be powers of two: a
        // GPC that holds two clusters of 8 may hold three of 6); if none is,
        // clusters of 8 (the most DSMEM hand-offs), else one CTA per block
        const int caps[9] = {0,
                             0,
                             strsv_cluster_capacity<2>(h->device, smem),
                             strsv_cluster_capacity<3>(h->device, smem),
                             strsv_cluster_capacity<4>(h->device, smem),
                             strsv_cluster_capacity<5>(h->device, smem),
                             strsv_cluster_capacity<6>(h->device, smem),
                             strsv_cluster_capacity<7>(h->device, smem),
                             strsv_cluster_capacity<8>(h->device, smem)};
        int cl = 0;
        for (int c = 8; c >= 2 && !cl; --c)
            if (caps[c] > 0 && caps[c] * c >= nb) cl = c;
        if (!cl && caps[8] > 0) cl = 8;
        switch (cl) {
        case 8: return strsv_launch<8>(h, smem, nb, map, n, lower_op, op, unit, x, incx, ticket, epoch_word);
        case 7: return strsv_launch<7>(h, smem, nb, map, n, lower_op, op, unit, x, incx, ticket, epoch_word);
        case 6: return strsv_launch<6>(h, smem, nb, map, n, lower_op, op, unit, x, incx, ticket, epoch_word);
        case 5: return strsv_launch<5>(h, smem, nb, map, n, lower_op, op, unit, x, incx, ticket, epoch_word);
        case 4: return strsv_launch<4>(h, smem, nb, map, n, lower_op, op, unit, x, incx, ticket, epoch_word);
        case 3: return strsv_launch<3>(h, smem, nb, map, n, lower_op, op, unit, x, incx, ticket, epoch_word);
        case 2: return strsv_launch<2>(h, smem, nb, map, n, lower_op, op, unit, x, incx, ticket, epoch_word);
        default: break;
        }
    }
    return strsv_launch<1>(h, smem, nb, map, n, lower_op, op, unit, x, incx, ticket, epoch_word);
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
