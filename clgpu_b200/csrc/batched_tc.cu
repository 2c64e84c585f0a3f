// Uneven batched TRSM and GEMM on the tensor cores: the TF32, 3xBF16 and
// 6xBF16 math modes of the batched plans.  No reference counterpart (the
// reference has no batched routines); the plain-FP32 plans run the
// CUDA-core kernels of batched.cu.
//
// Operands live in "tiled planes": FP32 values split into BF16 levels (hi,
// mid, lo; 3xBF16 reads two, 6xBF16 three) or rounded to TF32 (one FP32
// level), stored as 16 KiB tiles of 128 rows x 128 bytes (64 BF16 or 32
// TF32 K values per row), each tile laid out exactly as the tensor core
// reads it from shared memory (128-byte swizzle: the 16-byte chunk c of row
// r sits at chunk c ^ (r % 8)).  A tile is then fetched with one plain bulk
// copy (cp.async.bulk, no tensor map), so the per-instance operands of an
// uneven batch need no per-instance descriptors: a plan stores, per
// instance and plane set, the index of its first tile and the number of K
// tiles per row of tiles.
//
// One kernel (btc_mma_kernel) runs every product: a launch is a list of
// items, each one 128 x N output tile of one instance, C = c_alpha * A B^T
// + c_beta * C over a range of K tiles (N = the instance's column count in
// the tile, rounded up to 16).  Persistent CTAs (one per SM) take items
// round-robin; warp 0 issues the bulk copies into a ring of stages (all
// levels of one A and one B K tile per stage), one thread of warp 1 issues
// tcgen05.mma (M = 128, N, K = 32 bytes per instruction; products
// smallest first, as in the single-instance engine) into one of two TMEM
// accumulators, and 16 epilogue warps (a 32-column group of one TMEM lane
// quarter each) drain the other: C (column- or row-major, per-instance
// leading dimension), an optional triangle mask, and optionally the result
// split straight into tiled planes again, so that the next launch reads it
// as an operand.  6xBF16 drains the accumulator after every K tile and sums
// the parts in FP32 (the tensor core's FP32 accumulation loses a fraction
// of an ulp per step); the other modes accumulate the item's K range.
//
// TRSM, op(A) X = alpha B per instance, is solved by blocks of 128 rows in
// the operator's order, level-synchronously over the batch:
//   step q:  Y_s = B_s - sum_{r before s} M_sr X_r   (one launch over every
//                                          instance with more than q blocks,
//                                          K = the q solved blocks; writes
//                                          the planes of Y_s only)
//            X_s = inv(M_ss) Y_s          (one launch; C = B block s gets
//                                          alpha X_s, the planes get X_s)
// with M's off-diagonal tiles split once per call and the 128 x 128
// diagonal-block inverses formed from the 64 x 64 FP64-formed FP32
// inverses of batched.cu (one doubling step: off-diagonal block
// -Q^-1 C P^-1 for lower, -P^-1 C Q^-1 for upper; FP64 accumulation for
// 6xBF16, FP32 for the modes whose planes keep fewer bits), written as
// planes of inv and of inv^T (the adjoint's operator).  The adjoint solves
// with M^T the same way, reading M's tiles MN-major in the BF16 modes (TF32
// splits M^T), and forms dA = -(1/alpha) dB X^T on the stored triangle with
// one masked product launch (tiles off the triangle store zeros).
//
// Every wait is bounded (2 s); on timeout the kernel records
// kDevWaitTimeout in the handle's status word, waits (bounded) for its own
// copies and MMAs, frees TMEM and returns.  All copies are issued by a CTA
// into its own shared memory; no cluster, no multicast.
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <vector>

#include "common.cuh"
#include "tma.cuh"

namespace iclb {

namespace {

constexpr int TR = 128;                        // tile rows; one MMA is 128 x N
constexpr int ROWB = 128;                      // bytes per tile row
constexpr int TILE_BYTES = TR * ROWB;          // 16 KiB
constexpr int RING_BYTES = 192 * 1024;         // the stage ring
constexpr int MAX_STAGES = 6;
constexpr int EPI_WARPS = 16;                  // four per TMEM lane quarter
constexpr int THREADS = 64 + 32 * EPI_WARPS;   // producer, MMA, epilogue
constexpr int SMEM_BYTES = RING_BYTES + 1024 /*barriers*/ + 1024 /*alignment*/;
constexpr unsigned long long kWaitNs = 2000000000ull;

// A set of tiled planes: level l of tile `ti` at base + l * lstride + ti *
// TILE_BYTES; instance i's tile (row tile rt, K tile kt) is off[i] + rt *
// nkt + kt, nkt = nkt_arr[i] (or nkt_c when nkt_arr is null).
struct Opnd {
    char* base;
    long lstride;
    const long* off;
    const int* nkt_arr;
    int nkt_c;
};

__device__ __forceinline__ long tile_index(const Opnd& o, int inst, int rt, int kt)
{
    const long nk = o.nkt_arr ? o.nkt_arr[inst] : o.nkt_c;
    return o.off[inst] + (long)rt * nk + kt;
}

// Item: x instance; y (row tile << 16) | column tile; z (A K tile << 16) |
// B K tile; w K tiles << 16.
struct MmaLaunch {
    const int4* items;
    int nitems;
    Opnd a, b;
    int nlev, nprod;
    int pa[6], pb[6];   // split level of A and B for each product, smallest first
    float* const* C;
    const int4* cinfo;  // per instance: rows, columns, leading dimension
    int ct;             // 0: C[row + col * ld]; 1: C[col + row * ld]
    float c_alpha, c_beta;
    Opnd w;             // planes of the result: row = C column, K = C row
    int mask;           // kEpiMask: 1 keep row >= col, 2 keep row <= col; +4 strict
    int a_mn;           // A read MN-major from the tiles of its transpose (BF16 only)
    int kpb;            // K tiles per 128-row block
    int* status;
};

// ---------------------------------------------------------------- PTX helpers
using tma::global_ns;
using tma::mbar_expect_tx;
using tma::mbar_init;
using tma::mbar_try_wait;
using tma::smem_u32;

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait: false when 2 s passed or another role gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort_flag) return false;
        if (global_ns() - t0 > kWaitNs) {
            *abort_flag = 1;
            return false;
        }
    }
    return true;
}

// Wait without the abort shortcut, bounded by 2 s (drains own async work).
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity)
{
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity) && global_ns() - t0 < kWaitNs) {}
}

// Contiguous global -> own shared memory copy, completion counted in bytes
// on `bar` (16-byte aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"((unsigned long long)__cvta_generic_to_global(src)), "r"(bytes),
                 "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

template <bool TF32>
__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                     uint32_t accumulate)
{
    if (TF32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
    }
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 lanes x 32 consecutive columns of FP32 from TMEM (one column per register).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor, K-major, 128-byte swizzle: rows of 128 B,
// 8-row groups 1024 B apart, version 1, layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

// Shared-memory matrix descriptor, MN-major, 128-byte swizzle: rows of 128 B
// hold 64 consecutive M indices of one K index; 8-K groups 1024 B apart
// (SBO); the next 64 M indices 8 KiB further (LBO).  One MMA (K = 16) spans
// two 8-K groups: the start address advances by 2048 B per MMA.
__device__ __forceinline__ uint64_t desc_mn_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)(8192u >> 4) << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

// Instruction descriptor: FP32 accumulator, A/B format (1 BF16, 2 TF32),
// A K-major or MN-major (bit 15), B K-major, N = n, M = 128.
__device__ __forceinline__ uint32_t idesc_of(uint32_t fmt, int n, int a_mn)
{
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(TR >> 4) << 24);
}

__device__ __forceinline__ float to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// hi = bf16(x), mid = bf16(x - hi), lo = bf16(x - hi - mid); each
// difference is exact in FP32.
__device__ __forceinline__ void split3(float x, __nv_bfloat16& hi, __nv_bfloat16& mid, __nv_bfloat16& lo)
{
    hi = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(hi);
    mid = __float2bfloat16_rn(r1);
    lo = __float2bfloat16_rn(r1 - __bfloat162float(mid));
}

// Byte offset of (row, K element e) inside a tile (esize bytes per element).
__device__ __forceinline__ int swz(int row, int e, int esize)
{
    const int b = e * esize;
    return row * ROWB + ((((b >> 4) ^ (row & 7))) << 4) + (b & 15);
}

__device__ __forceinline__ int b_rows(int cols, int ct)
{
    const int c = min(TR, cols - ct * TR);
    return max(16, (c + 15) & ~15);
}

// ---------------------------------------------------------------- epilogue
// What the epilogue does with one accumulator tile (a template argument, so
// that the per-element code has no branches on the kind):
//   kEpiInv   C = alpha * acc; planes of acc            (X_s = inv Y_s)
//   kEpiUpd   planes of C - acc; C only read            (Y_s = B_s - sum)
//   kEpiGemm  C = alpha * acc + beta * C (C not read when beta == 0)
//   kEpiMask  C = alpha * acc on the kept triangle, 0 elsewhere (dA)
enum EpiKind { kEpiInv = 0, kEpiUpd = 1, kEpiGemm = 2, kEpiMask = 3 };

// One thread's 32 consecutive columns col0.. of its row (v = acc): element
// (row, col) of C at C[row + col * ld] (ct 0) or C[col + row * ld]; the
// planes, when written, get (row j = column within the column tile, K =
// row) in tile (column tile, row / KT).
template <bool TF32, int EK>
__device__ __forceinline__ void epilogue_group(const MmaLaunch& p, float (&v)[32], int inst, int row, int ct,
                                               int c0, const int4 ci)
{
    constexpr int KT = TF32 ? 32 : 64;
    constexpr int ESIZE = TF32 ? 4 : 2;
    const int rows = ci.x, cols = ci.y, col0 = ct * TR + c0;
    const long ld = ci.z;
    const bool rv = row < rows;
    const int ncv = rv ? min(32, cols - col0) : 0;  // columns of this thread inside C
    float* const cp = p.C[inst] + (p.ct ? (long)row * ld + col0 : (long)col0 * ld + row);
    const long cs = p.ct ? 1 : ld;
    // v becomes the value stored (C) or split (planes)
    if constexpr (EK == kEpiUpd || EK == kEpiGemm) {
        const bool load = EK == kEpiUpd || p.c_beta != 0.f;
#pragma unroll
        for (int h = 0; h < 32; h += 16) {  // two halves: 16 loads in flight, fewer live registers
            float x[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) x[j] = (load && h + j < ncv) ? cp[(h + j) * cs] : 0.f;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                if constexpr (EK == kEpiUpd) {
                    v[h + j] = x[j] - v[h + j];
                } else {  // stored at once: v is not needed after
                    const float y = load ? fmaf(p.c_alpha, v[h + j], p.c_beta * x[j]) : p.c_alpha * v[h + j];
                    if (h + j < ncv) cp[(h + j) * cs] = y;
                }
            }
        }
    } else if constexpr (EK == kEpiMask) {
        const bool strict = (p.mask & 4) != 0, lower = (p.mask & 3) == 1;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const int col = col0 + j;
            const bool keep = lower ? (strict ? row > col : row >= col) : (strict ? row < col : row <= col);
            v[j] = keep ? p.c_alpha * v[j] : 0.f;
        }
    }
    if constexpr (EK == kEpiInv) {
#pragma unroll
        for (int j = 0; j < 32; ++j)
            if (j < ncv) cp[j * cs] = p.c_alpha * v[j];
    } else if constexpr (EK == kEpiMask) {
#pragma unroll
        for (int j = 0; j < 32; ++j)
            if (j < ncv) cp[j * cs] = v[j];
    }
    if constexpr (EK == kEpiInv || EK == kEpiUpd) {
        // planes of acc (X_s) or C - acc (Y_s), zero outside C: row j = C
        // column c0 + j of this column tile, K = this thread's row (a warp
        // writes 32 consecutive K values of one tile row per store); the
        // tile row's swizzle phase is j % 8 (c0 is a multiple of 8)
        char* const tile = p.w.base + tile_index(p.w, inst, ct, row / KT) * TILE_BYTES;
        const int b = (row % KT) * ESIZE;
        char* const base = tile + (long)c0 * ROWB + (b & 15);
        const int chunk = (b >> 4) << 4;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const float pv = j < ncv ? v[j] : 0.f;
            char* const a = base + j * ROWB + (chunk ^ ((j & 7) << 4));
            if (TF32) {
                *(float*)a = to_tf32(pv);
            } else {
                __nv_bfloat16 hi, mid, lo;
                split3(pv, hi, mid, lo);
                *(__nv_bfloat16*)a = hi;
                if (p.nlev > 1) *(__nv_bfloat16*)(a + p.w.lstride) = mid;
                if (p.nlev > 2) *(__nv_bfloat16*)(a + 2 * p.w.lstride) = lo;
            }
        }
    }
}

// ---------------------------------------------------------------- product kernel
template <bool TF32, int EK>
__global__ void __launch_bounds__(THREADS, 1) btc_mma_kernel(const __grid_constant__ MmaLaunch p)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* ring = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int stage_bytes = 2 * p.nlev * TILE_BYTES;
    const int nstages = RING_BYTES / stage_bytes;  // 6 (TF32), 3 (3xBF16), 2 (6xBF16)
    uint64_t* full = (uint64_t*)(ring + RING_BYTES);
    uint64_t* empty = full + MAX_STAGES;
    uint64_t* tfull = empty + MAX_STAGES;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = (uint32_t*)(tempty + 2);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

    if (threadIdx.x == 0) {
        for (int s = 0; s < nstages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], EPI_WARPS);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * TR));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ---------------------------------------------------------- bulk-copy producer
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            for (int it = blockIdx.x; it < p.nitems && ok; it += gridDim.x) {
                const int4 w = p.items[it];
                const int inst = w.x, rt = w.y >> 16, ct = w.y & 0xffff, nk = w.w >> 16;
                if (nk == 0) continue;
                const uint32_t bbytes = (uint32_t)b_rows(p.cinfo[inst].y, ct) * ROWB;
                const int akt = w.z >> 16;
                const long ta = p.a_mn ? 0 : tile_index(p.a, inst, rt, akt), tb = tile_index(p.b, inst, ct, w.z & 0xffff);
                for (int kt = 0; kt < nk; ++kt) {
                    if (!mbar_wait(&empty[s], ph ^ 1, abort_flag)) { ok = false; break; }
                    uint8_t* st = ring + s * stage_bytes;
                    mbar_expect_tx(&full[s], (uint32_t)p.nlev * (TILE_BYTES + bbytes));
                    // MN-major A: K tile k of the transpose = rows (k % kpb) * 64.. of
                    // its row block k / kpb, the two 64-column tiles of block rt
                    const int kg = akt + kt, sb = kg / p.kpb, half = (kg % p.kpb) * (TILE_BYTES / 2);
                    const long tm = p.a_mn ? tile_index(p.a, inst, sb, 2 * rt) : 0;
                    for (int l = 0; l < p.nlev; ++l) {
                        const char* const a = p.a.base + l * p.a.lstride;
                        if (p.a_mn) {
                            bulk_load(st + l * TILE_BYTES, a + tm * TILE_BYTES + half, TILE_BYTES / 2, &full[s]);
                            bulk_load(st + l * TILE_BYTES + TILE_BYTES / 2, a + (tm + 1) * TILE_BYTES + half,
                                      TILE_BYTES / 2, &full[s]);
                        } else {
                            bulk_load(st + l * TILE_BYTES, a + (ta + kt) * TILE_BYTES, TILE_BYTES, &full[s]);
                        }
                        bulk_load(st + (p.nlev + l) * TILE_BYTES, p.b.base + l * p.b.lstride + (tb + kt) * TILE_BYTES,
                                  bbytes, &full[s]);
                    }
                    if (++s == nstages) { s = 0; ph ^= 1; }
                }
            }
            if (!ok) {
                // wait (bounded) for the copies this thread issued, then leave
                for (int i = 0; i < nstages; ++i) mbar_drain(&full[(s + i) % nstages], ph);
            }
        }
    } else if (warp == 1) {
        // ---------------------------------------------------------- MMA issuer
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            int acc = 0;
            uint32_t acc_ph = 0;
            bool ok = true;
            // TMEM chunk: 6xBF16 one K tile (drained and summed in FP32 by
            // the epilogue: the tensor core's accumulation loses a fraction
            // of an ulp per step), the other modes the whole K range
            const bool per_tile = p.nprod == 6;
            for (int it = blockIdx.x; it < p.nitems && ok; it += gridDim.x) {
                const int4 w = p.items[it];
                const int inst = w.x, ct = w.y & 0xffff, nk = w.w >> 16;
                if (nk == 0) continue;
                const uint32_t idesc = idesc_of(TF32 ? 2u : 1u, b_rows(p.cinfo[inst].y, ct), p.a_mn);
                const uint64_t a_step = p.a_mn ? 128 : 2;  // per MMA, 16-byte units
                uint32_t d = 0;
                bool open = false;  // MMAs issued into the current chunk, not yet committed
                for (int kt = 0; kt < nk; ++kt) {
                    if (kt == 0 || per_tile) {
                        if (!mbar_wait(&tempty[acc], acc_ph ^ 1, abort_flag)) { ok = false; break; }
                        tc_fence_after();
                        d = tmem_base + (uint32_t)(acc * TR);
                    }
                    if (!mbar_wait(&full[s], ph, abort_flag)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t st = smem_u32(ring + s * stage_bytes);
                    for (int pr = 0; pr < p.nprod; ++pr) {
                        const uint32_t sa = st + p.pa[pr] * TILE_BYTES;
                        const uint64_t da = p.a_mn ? desc_mn_sw128(sa) : desc_sw128(sa);
                        const uint64_t db = desc_sw128(st + (p.nlev + p.pb[pr]) * TILE_BYTES);
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk)  // 4 x 32 bytes of K per tile row
                            umma<TF32>(d, da + a_step * kk, db + 2 * kk, idesc,
                                       ((kt > 0 && !per_tile) || pr > 0 || kk > 0) ? 1u : 0u);
                    }
                    open = true;
                    umma_commit(&empty[s]);
                    if (++s == nstages) { s = 0; ph ^= 1; }
                    if (per_tile || kt == nk - 1) {
                        // chunk done: the epilogue may read this accumulator
                        umma_commit(&tfull[acc]);
                        open = false;
                        if (++acc == 2) { acc = 0; acc_ph ^= 1; }
                    }
                }
                if (!ok && open) {
                    umma_commit(&tfull[acc]);
                    mbar_drain(&tfull[acc], acc_ph);  // every issued MMA done before TMEM is freed
                }
            }
        }
    } else {
        // ---------------------------------------------------------- epilogue
        // 16 warps: TMEM lane quarter q (rows 32q..), 32-column group cg
        const int q = warp & 3, cg = (warp - 2) >> 2;
        const int r = q * 32 + lane;  // tile row = TMEM lane
        int acc = 0;
        uint32_t acc_ph = 0;
        for (int it = blockIdx.x; it < p.nitems; it += gridDim.x) {
            const int4 w = p.items[it];
            const int inst = w.x, rt = w.y >> 16, ct = w.y & 0xffff, nk = w.w >> 16;
            const int4 ci = p.cinfo[inst];
            const int c0 = cg * 32;
            const bool active = c0 < b_rows(ci.y, ct);
            float v[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = 0.f;
            // the item's chunks (one per K tile in 6xBF16), summed in FP32 in K order
            const int nchunks = nk == 0 ? 0 : (p.nprod == 6 ? nk : 1);
            bool ok = true;
            for (int c = 0; c < nchunks; ++c) {
                int okw = 1;
                if (lane == 0) okw = mbar_wait(&tfull[acc], acc_ph, abort_flag) ? 1 : 0;
                if (!__shfl_sync(0xffffffffu, okw, 0)) { ok = false; break; }
                tc_fence_after();
                if (active) {
                    float u[32];
                    tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * TR + c0), u);
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] += u[j];
                }
                // the values are in registers: the accumulator is free
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[acc]);
                if (++acc == 2) { acc = 0; acc_ph ^= 1; }
            }
            if (!ok) break;
            if (active) epilogue_group<TF32, EK>(p, v, inst, rt * TR + r, ct, c0, ci);
        }
    }

    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicOr(p.status, (int)kDevWaitTimeout);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(2 * TR));
    }
}

// ---------------------------------------------------------------- split kernel
// One tile per CTA: L[r][k] = S[r * ld + k] (rmajor) or S[r + k * ld], r < R,
// k < K (zero elsewhere), staged through shared memory so that the reads run
// along the source's contiguous dimension, then written as 16-byte chunks
// of every level (a warp writes four whole 128-byte tile rows).
struct SplitKind {
    const float* const* src;
    const int4* info;   // per instance: R, K, ld
    int rmajor;
    Opnd dst;
};
struct SplitLaunch {
    const int4* items;  // (kind, instance, row tile, K tile)
    SplitKind kind[2];
    int nlev;
};

template <bool TF32>
__global__ void __launch_bounds__(256) btc_split_kernel(const __grid_constant__ SplitLaunch p)
{
    constexpr int KT = TF32 ? 32 : 64;
    __shared__ float tile[TR][KT + 1];
    const int4 w = p.items[blockIdx.x];
    const SplitKind& k = p.kind[w.x];
    const int inst = w.y, rt = w.z, kt = w.w;
    const int4 in = k.info[inst];
    const int R = in.x, K = in.y;
    const long ld = in.z;
    const float* S = k.src[inst];
    const int r0 = rt * TR, k0 = kt * KT, t = threadIdx.x;
    // every load of the thread is issued before the first shared-memory store
    constexpr int PER = TR * KT / 256;
    float v[PER];
    if (k.rmajor) {
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int idx = t + u * 256, rr = idx / KT, kk = idx % KT;
            const int r = r0 + rr, c = k0 + kk;
            v[u] = (r < R && c < K) ? S[(long)r * ld + c] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int idx = t + u * 256;
            tile[idx / KT][idx % KT] = v[u];
        }
    } else {
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int idx = t + u * 256, rr = idx % TR, kk = idx / TR;
            const int r = r0 + rr, c = k0 + kk;
            v[u] = (r < R && c < K) ? S[r + (long)c * ld] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int idx = t + u * 256;
            tile[idx % TR][idx / TR] = v[u];
        }
    }
    __syncthreads();
    char* dst = k.dst.base + tile_index(k.dst, inst, rt, kt) * TILE_BYTES;
    for (int idx = t; idx < TR * 8; idx += 256) {
        const int rr = idx >> 3, c = idx & 7;
        const int o = rr * ROWB + ((c ^ (rr & 7)) << 4);
        if (TF32) {
            const float* s = &tile[rr][c * 4];
            *(float4*)(dst + o) = make_float4(to_tf32(s[0]), to_tf32(s[1]), to_tf32(s[2]), to_tf32(s[3]));
        } else {
            const float* s = &tile[rr][c * 8];
            uint32_t hv[4], mv[4], lv[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                __nv_bfloat16 h0, m0, l0, h1, m1, l1;
                split3(s[2 * e], h0, m0, l0);
                split3(s[2 * e + 1], h1, m1, l1);
                hv[e] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
                mv[e] = (uint32_t)__bfloat16_as_ushort(m0) | ((uint32_t)__bfloat16_as_ushort(m1) << 16);
                lv[e] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
            }
            *(uint4*)(dst + o) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
            if (p.nlev > 1) *(uint4*)(dst + k.dst.lstride + o) = make_uint4(mv[0], mv[1], mv[2], mv[3]);
            if (p.nlev > 2) *(uint4*)(dst + 2 * k.dst.lstride + o) = make_uint4(lv[0], lv[1], lv[2], lv[3]);
        }
    }
}

// ---------------------------------------------------------------- 128 x 128 inverses
// One CTA (256 threads) per (instance, 128-row block) of M = op(A): from the
// FP32 inverses P^-1, Q^-1 of its two 64 x 64 diagonal blocks (identity for a
// missing second block) and the off-diagonal block C of M,
//   lower: inv = [[P^-1, 0], [-Q^-1 (C P^-1), Q^-1]]
//   upper: inv = [[P^-1, -P^-1 (C Q^-1)], [0, Q^-1]]
// with both products accumulated in FP64 for 6xBF16, whose three planes
// keep every bit of the FP32 inverse, and in FP32 for 3xBF16 and TF32, whose
// planes keep about 16 and 11 bits of it (4 x 4 outputs per thread; T held
// in the accumulation type); the block is written as tiled planes of inv
// (row r, K c) and of inv^T straight from its quadrants (a 16-byte chunk
// never crosses one).
struct InvLaunch {
    const int2* items;       // (instance, 128-row block)
    const int* dims;         // per instance: na, nr, lda, ldb
    const long* inv64_off;   // per instance: offset of its 64 x 64 inverses
    const float* inv64;      // column-major 64 x 64 blocks, identity past the size
    const float* const* A;
    int lower, op;
    Opnd w, wt;
    int nlev;
};
constexpr int kInvLd = 65;
template <class Acc>
constexpr int inv_smem_bytes()
{
    return 3 * 64 * kInvLd * (int)sizeof(float) + 64 * kInvLd * (int)sizeof(Acc);
}

template <bool TF32, class Acc>
__global__ void __launch_bounds__(256) btc_inv_kernel(const __grid_constant__ InvLaunch p)
{
    constexpr int KT = TF32 ? 32 : 64;
    constexpr int ESIZE = TF32 ? 4 : 2;
    constexpr int EPC = 16 / ESIZE;  // elements per 16-byte chunk
    constexpr int CPR = TR / EPC;    // chunks per 128-element row
    extern __shared__ double inv_smem[];
    Acc(*T)[kInvLd] = (Acc(*)[kInvLd])inv_smem;
    float(*P)[kInvLd] = (float(*)[kInvLd])((Acc*)inv_smem + 64 * kInvLd);
    float(*Q)[kInvLd] = P + 64;
    float(*Cm)[kInvLd] = Q + 64;  // C, then the off-diagonal block of the inverse
    const int t = threadIdx.x;
    const int2 it = p.items[blockIdx.x];
    const int inst = it.x, b = it.y;
    const int* d = p.dims + 4 * inst;
    const int na = d[0];
    const long lda = d[2];
    const int nb64 = (na + 63) / 64;
    const float* A = p.A[inst];
    const float* inv = p.inv64 + p.inv64_off[inst];
    const int r0 = b * TR;
    const bool has_q = 2 * b + 1 < nb64;
    {
        // every load of the thread in flight before the first store
        float vp[16], vq[16], vc[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            const int idx = t + u * 256, rr = idx % 64, cc = idx / 64;  // column-major: coalesced
            vp[u] = inv[(long)(2 * b) * 4096 + idx];
            vq[u] = has_q ? inv[(long)(2 * b + 1) * 4096 + idx] : (rr == cc ? 1.f : 0.f);
            // off-diagonal block of M (local rows i, columns j of the 128 block)
            const int i = p.lower ? 64 + rr : rr, j = p.lower ? cc : 64 + cc;
            vc[u] = (r0 + i < na && r0 + j < na)
                        ? (p.op ? A[(long)(r0 + j) + (long)(r0 + i) * lda] : A[(long)(r0 + i) + (long)(r0 + j) * lda])
                        : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            const int idx = t + u * 256, rr = idx % 64, cc = idx / 64;
            P[rr][cc] = vp[u];
            Q[rr][cc] = vq[u];
            Cm[rr][cc] = vc[u];
        }
    }
    __syncthreads();
    const int tr = (t >> 4) * 4, tc = (t & 15) * 4;
    {
        // T = C P^-1 (lower) or C Q^-1 (upper)
        float(*R)[kInvLd] = p.lower ? P : Q;
        Acc acc[4][4] = {};
        for (int k = 0; k < 64; ++k) {
            Acc a[4], bb[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = Cm[tr + i][k];
#pragma unroll
            for (int j = 0; j < 4; ++j) bb[j] = R[k][tc + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) T[tr + i][tc + j] = acc[i][j];
    }
    __syncthreads();
    {
        // off-diagonal block of the inverse: -Q^-1 T (lower) or -P^-1 T (upper), into Cm
        float(*L)[kInvLd] = p.lower ? Q : P;
        Acc acc[4][4] = {};
        for (int k = 0; k < 64; ++k) {
            Acc a[4], bb[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = L[tr + i][k];
#pragma unroll
            for (int j = 0; j < 4; ++j) bb[j] = T[k][tc + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
        }
        // Cm is read only by the first product, which every thread has finished
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) Cm[tr + i][tc + j] = (float)(-acc[i][j]);
    }
    __syncthreads();
    // planes: pass 0 inv (threads along a row's chunks), pass 1 inv^T
    // (consecutive threads take consecutive rows: reading down a column of
    // the quadrant without bank conflicts)
    for (int pass = 0; pass < 2; ++pass) {
        const Opnd& o = pass ? p.wt : p.w;
        for (int idx = t; idx < TR * CPR; idx += 256) {
            const int r = pass ? idx % TR : idx / CPR, ch = pass ? idx / TR : idx % CPR;
            const int c0 = ch * EPC;
            // element (r, c0 + e) of inv (pass 0) or inv^T (pass 1)
            const int gr = pass ? c0 : r, gc = pass ? r : c0;  // quadrant of inv holding it
            const int hr = gr >> 6, hc = gc >> 6;
            const float(*S)[kInvLd] = hr == hc ? (hr ? Q : P) : Cm;
            const bool zero = hr != hc && (p.lower ? hr == 0 : hr == 1);
            float x[EPC];
#pragma unroll
            for (int e = 0; e < EPC; ++e)
                x[e] = zero ? 0.f : (pass ? S[(c0 + e) & 63][r & 63] : S[r & 63][(c0 + e) & 63]);
            char* tile = o.base + tile_index(o, inst, b, c0 / KT) * TILE_BYTES;
            const int off16 = swz(r, c0 % KT, ESIZE);
            if (TF32) {
                *(float4*)(tile + off16) = make_float4(to_tf32(x[0]), to_tf32(x[1]), to_tf32(x[2]), to_tf32(x[3]));
            } else {
                uint32_t hv[EPC / 2], mv[EPC / 2], lv[EPC / 2];
#pragma unroll
                for (int e = 0; e < EPC / 2; ++e) {
                    __nv_bfloat16 h0, m0, l0, h1, m1, l1;
                    split3(x[2 * e], h0, m0, l0);
                    split3(x[2 * e + 1], h1, m1, l1);
                    hv[e] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
                    mv[e] = (uint32_t)__bfloat16_as_ushort(m0) | ((uint32_t)__bfloat16_as_ushort(m1) << 16);
                    lv[e] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
                }
                *(uint4*)(tile + off16) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
                if (p.nlev > 1) *(uint4*)(tile + o.lstride + off16) = make_uint4(mv[0], mv[1], mv[2], mv[3]);
                if (p.nlev > 2) *(uint4*)(tile + 2 * o.lstride + off16) = make_uint4(lv[0], lv[1], lv[2], lv[3]);
            }
        }
    }
}

// ---------------------------------------------------------------- host
// Split level of A and B of each product, smallest first (the orders of the
// single-instance engine): 3xBF16 mid*hi, hi*mid, hi*hi; 6xBF16 lo*hi,
// hi*lo, mid*mid, mid*hi, hi*mid, hi*hi.
void mode_products(iclblasMathMode_t mode, int& tf32, int& nlev, int& nprod, int* pa, int* pb)
{
    tf32 = mode == ICLBLAS_MATH_TF32;
    if (tf32) {
        nlev = 1;
        nprod = 1;
        pa[0] = pb[0] = 0;
    } else if (mode == ICLBLAS_MATH_BF16X3) {
        nlev = 2;
        nprod = 3;
        const int a[3] = {1, 0, 0}, b[3] = {0, 1, 0};
        for (int i = 0; i < 3; ++i) { pa[i] = a[i]; pb[i] = b[i]; }
    } else {
        nlev = 3;
        nprod = 6;
        const int a[6] = {2, 0, 1, 1, 0, 0}, b[6] = {0, 2, 1, 0, 1, 0};
        for (int i = 0; i < 6; ++i) { pa[i] = a[i]; pb[i] = b[i]; }
    }
}

int4 mk_item(int inst, int rt, int ct, int akt, int bkt, int nk)
{
    return make_int4(inst, (rt << 16) | ct, (akt << 16) | bkt, nk << 16);
}

template <class T>
cudaError_t upload(T** dst, const std::vector<T>& v)
{
    *dst = nullptr;
    if (v.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(dst, v.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

cudaError_t alloc_planes(char** dst, long tiles, int nlev, long& lstride)
{
    lstride = std::max(tiles, 1L) * TILE_BYTES;
    return cudaMalloc(dst, (size_t)lstride * nlev);
}

// Kernel attributes, once per device.
cudaError_t set_attrs(int device)
{
    static std::atomic<unsigned long long> done{0};
    const unsigned long long bit = 1ull << (device & 63);
    if (done.load() & bit) return cudaSuccess;
    cudaError_t e;
    const void* kernels[8] = {
        (const void*)btc_mma_kernel<true, kEpiInv>,   (const void*)btc_mma_kernel<true, kEpiUpd>,
        (const void*)btc_mma_kernel<true, kEpiGemm>,  (const void*)btc_mma_kernel<true, kEpiMask>,
        (const void*)btc_mma_kernel<false, kEpiInv>,  (const void*)btc_mma_kernel<false, kEpiUpd>,
        (const void*)btc_mma_kernel<false, kEpiGemm>, (const void*)btc_mma_kernel<false, kEpiMask>};
    for (const void* k : kernels)
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES)) != cudaSuccess)
            return e;
    if ((e = cudaFuncSetAttribute(btc_inv_kernel<true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  inv_smem_bytes<float>())) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(btc_inv_kernel<false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  inv_smem_bytes<float>())) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(btc_inv_kernel<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  inv_smem_bytes<double>())) != cudaSuccess)
        return e;
    done.fetch_or(bit);
    return cudaSuccess;
}

}  // namespace

// A contiguous range of a plan's item array: one launch.
struct TcRange {
    int off = 0, count = 0;
};

// Everything a tensor-core batched plan owns (device memory and the launch
// lists, fixed at plan creation).
struct BatchTc {
    int tf32 = 0, nlev = 0, nprod = 0, pa[6] = {}, pb[6] = {};
    int kpb = 0;     // K tiles per 128-row block (2 BF16, 4 TF32)
    std::vector<void*> allocs;
    int4* items = nullptr;       // every launch's items, one array
    // TRSM plans
    char *sp = nullptr, *inv = nullptr, *invt = nullptr, *xp = nullptr, *wp = nullptr, *xq = nullptr;
    long sp_l = 0, inv_l = 0, xp_l = 0, d_l = 0;
    long *off_s = nullptr, *off_inv = nullptr, *off_x = nullptr, *off_d = nullptr;
    int *nkt_s = nullptr, *nkt_x = nullptr, *nkt_d = nullptr;
    int4 *info_a = nullptr, *info_y = nullptr, *info_p = nullptr;
    int2* inv_items = nullptr;
    int n_inv = 0;
    int right = 0, lower_f = 0, op_f = 0, tri_lower = 0, unit = 0;
    // split launches: forward (first block + operator tiles); adjoint with
    // the operator tiles (the forward's, read MN-major, in the BF16 modes;
    // the transpose's in TF32) or, when the forward call's are reused, the
    // first block only
    TcRange split_f, split_b, split_b_first, split_d, gemm_d;
    int a_mn_b = 0;  // the adjoint's updates read the forward's operator tiles MN-major
    std::vector<TcRange> inv_f, upd_f, inv_b, upd_b;
    // GEMM plans
    char *ap = nullptr, *bp = nullptr;
    long ap_l = 0, bp_l = 0;
    long *off_ga = nullptr, *off_gb = nullptr;
    int* nkt_g = nullptr;
    int4 *info_ga = nullptr, *info_gb = nullptr, *info_gc = nullptr;
    int ta = 0, tb = 0;
    TcRange split_g, gemm_g;
};

namespace {

Opnd opnd(char* base, long lstride, const long* off, const int* nkt_arr, int nkt_c = 0)
{
    return Opnd{base, lstride, off, nkt_arr, nkt_c};
}

cudaError_t run_split(iclblasHandle_t h, const BatchTc& t, TcRange r, const SplitKind& k0, const SplitKind& k1)
{
    if (r.count == 0) return cudaSuccess;
    SplitLaunch p{};
    p.items = t.items + r.off;
    p.kind[0] = k0;
    p.kind[1] = k1;
    p.nlev = t.nlev;
    if (t.tf32) btc_split_kernel<true><<<r.count, 256, 0, h->stream>>>(p);
    else btc_split_kernel<false><<<r.count, 256, 0, h->stream>>>(p);
    return cudaGetLastError();
}

struct MmaArgs {
    int kind = kEpiGemm;
    Opnd a, b;
    float* const* C;
    const int4* cinfo;
    int ct = 0;
    float c_alpha = 1.f, c_beta = 0.f;
    Opnd w{};
    int mask = 0;
    int a_mn = 0;
};

template <bool TF32>
void launch_mma(const MmaLaunch& p, int kind, int grid, cudaStream_t st)
{
    switch (kind) {
    case kEpiInv: btc_mma_kernel<TF32, kEpiInv><<<grid, THREADS, SMEM_BYTES, st>>>(p); break;
    case kEpiUpd: btc_mma_kernel<TF32, kEpiUpd><<<grid, THREADS, SMEM_BYTES, st>>>(p); break;
    case kEpiMask: btc_mma_kernel<TF32, kEpiMask><<<grid, THREADS, SMEM_BYTES, st>>>(p); break;
    default: btc_mma_kernel<TF32, kEpiGemm><<<grid, THREADS, SMEM_BYTES, st>>>(p); break;
    }
}

cudaError_t run_mma(iclblasHandle_t h, const BatchTc& t, TcRange r, const MmaArgs& m)
{
    if (r.count == 0) return cudaSuccess;
    MmaLaunch p{};
    p.items = t.items + r.off;
    p.nitems = r.count;
    p.a = m.a;
    p.b = m.b;
    p.nlev = t.nlev;
    p.nprod = t.nprod;
    for (int i = 0; i < 6; ++i) {
        p.pa[i] = t.pa[i];
        p.pb[i] = t.pb[i];
    }
    p.C = m.C;
    p.cinfo = m.cinfo;
    p.ct = m.ct;
    p.c_alpha = m.c_alpha;
    p.c_beta = m.c_beta;
    p.w = m.w;
    p.mask = m.mask;
    p.a_mn = m.a_mn;
    p.kpb = t.kpb;
    p.status = h->ws.dev_status;
    const int grid = std::min(r.count, h->sm_count);
    if (t.tf32) launch_mma<true>(p, m.kind, grid, h->stream);
    else launch_mma<false>(p, m.kind, grid, h->stream);
    return cudaGetLastError();
}

// Level-synchronous items of a blocked solve with operator S (lower: blocks
// in increasing order) for instances (na, nr): per step q, the update of
// that step's block s of every instance from all blocks solved before it
// (one item per column tile, K = q blocks; it writes the planes of
// Y_s = B_s - sum M_sq X_q), then the inverse products X_s = inv(S_ss) Y_s.
void solve_items(const std::vector<int>& dims, int batch, int lower, int kpb, std::vector<int4>& all,
                 std::vector<TcRange>& invs, std::vector<TcRange>& upds)
{
    int qmax = 0;
    for (int i = 0; i < batch; ++i)
        if (dims[4 * i] > 0 && dims[4 * i + 1] > 0) qmax = std::max(qmax, (dims[4 * i] + TR - 1) / TR);
    invs.assign(qmax, TcRange{});
    upds.assign(qmax, TcRange{});
    for (int q = 0; q < qmax; ++q) {
        // update of step q's block s from the q blocks solved before it (K
        // tiles contiguous: lower, blocks 0..s-1; upper, blocks s+1..)
        upds[q].off = (int)all.size();
        for (int i = 0; i < batch && q > 0; ++i) {
            const int na = dims[4 * i], nr = dims[4 * i + 1];
            const int nblk = (na + TR - 1) / TR, nct = (nr + TR - 1) / TR;
            if (na == 0 || nr == 0 || nblk <= q) continue;
            const int s = lower ? q : nblk - 1 - q;
            const int k0 = lower ? 0 : (s + 1) * kpb;
            for (int c = 0; c < nct; ++c) all.push_back(mk_item(i, s, c, k0, k0, q * kpb));
        }
        upds[q].count = (int)all.size() - upds[q].off;
        invs[q].off = (int)all.size();
        for (int i = 0; i < batch; ++i) {
            const int na = dims[4 * i], nr = dims[4 * i + 1];
            const int nblk = (na + TR - 1) / TR, nct = (nr + TR - 1) / TR;
            if (na == 0 || nr == 0 || nblk <= q) continue;
            const int s = lower ? q : nblk - 1 - q;
            for (int c = 0; c < nct; ++c) all.push_back(mk_item(i, s, c, 0, s * kpb, kpb));
        }
        invs[q].count = (int)all.size() - invs[q].off;
    }
}

// Split items: the operator's tiles strictly off the diagonal blocks on
// the side `lower` names (kind 0), and the first block, in the solve order
// of `lower`, of the right-hand sides (kind 1).
void operator_items(const std::vector<int>& dims, int batch, int lower, int kpb, std::vector<int4>& all)
{
    for (int i = 0; i < batch; ++i) {
        const int na = dims[4 * i], nr = dims[4 * i + 1];
        if (na == 0 || nr == 0) continue;
        const int nblk = (na + TR - 1) / TR;
        for (int tt = 0; tt < nblk; ++tt) {
            const int k0 = lower ? 0 : (tt + 1) * kpb, k1 = lower ? tt * kpb : nblk * kpb;
            for (int kt = k0; kt < k1; ++kt) all.push_back(make_int4(0, i, tt, kt));
        }
    }
}

void first_block_items(const std::vector<int>& dims, int batch, int lower, int kpb, std::vector<int4>& all)
{
    for (int i = 0; i < batch; ++i) {
        const int na = dims[4 * i], nr = dims[4 * i + 1];
        if (na == 0 || nr == 0) continue;
        const int nblk = (na + TR - 1) / TR, nct = (nr + TR - 1) / TR;
        const int s0 = lower ? 0 : nblk - 1;
        for (int c = 0; c < nct; ++c)
            for (int kt = s0 * kpb; kt < (s0 + 1) * kpb; ++kt) all.push_back(make_int4(1, i, c, kt));
    }
}

template <class T>
cudaError_t track(BatchTc* t, T** p, const std::vector<T>& v)
{
    cudaError_t e = upload(p, v);
    if (*p) t->allocs.push_back(*p);
    return e;
}

cudaError_t track_planes(BatchTc* t, char** p, long tiles, long& lstride)
{
    cudaError_t e = alloc_planes(p, tiles, t->nlev, lstride);
    if (*p) t->allocs.push_back(*p);
    return e;
}

}  // namespace

void batch_tc_free(BatchTc* t)
{
    if (!t) return;
    for (void* p : t->allocs) cudaFree(p);
    delete t;
}

bool batch_tc_mode(iclblasMathMode_t mode)
{
    return mode == ICLBLAS_MATH_TF32 || mode == ICLBLAS_MATH_BF16X3 || mode == ICLBLAS_MATH_BF16X6;
}

cudaError_t batch_tc_create_trsm(iclblasHandle_t h, iclblasBatchPlan* plan, const std::vector<int>& dims, int right,
                                 int lower_f, int op_f, int tri_lower, int unit)
{
    cudaError_t e = set_attrs(h->device);
    if (e != cudaSuccess) return e;
    auto* t = new BatchTc();
    plan->tc = t;
    mode_products(h->math, t->tf32, t->nlev, t->nprod, t->pa, t->pb);
    const int KT = t->tf32 ? 32 : 64;
    t->kpb = TR / KT;
    t->right = right;
    t->lower_f = lower_f;
    t->op_f = op_f;
    t->tri_lower = tri_lower;
    t->unit = unit;
    const int batch = plan->batch;
    std::vector<long> off_s(batch), off_inv(batch), off_x(batch), off_d(batch);
    std::vector<int> nkt_s(batch), nkt_x(batch), nkt_d(batch);
    std::vector<int4> info_a(batch), info_y(batch), info_p(batch);
    std::vector<int2> inv_items;
    long ts = 0, ti = 0, tx = 0, td = 0;
    for (int i = 0; i < batch; ++i) {
        const int na = dims[4 * i], nr = dims[4 * i + 1], lda = dims[4 * i + 2], ldb = dims[4 * i + 3];
        const int nblk = (na + TR - 1) / TR, nct = (nr + TR - 1) / TR, nkd = (nr + KT - 1) / KT;
        off_s[i] = ts;
        nkt_s[i] = nblk * t->kpb;
        ts += (long)nblk * nblk * t->kpb;
        off_inv[i] = ti;
        ti += (long)nblk * t->kpb;
        off_x[i] = tx;
        nkt_x[i] = nblk * t->kpb;
        tx += (long)nct * nblk * t->kpb;
        off_d[i] = td;
        nkt_d[i] = nkd;
        td += (long)nblk * nkd;
        info_a[i] = make_int4(na, na, lda, 0);
        info_y[i] = make_int4(nr, na, ldb, 0);
        info_p[i] = make_int4(na, nr, ldb, 0);
        if (na > 0 && nr > 0)
            for (int b = 0; b < nblk; ++b) inv_items.push_back(make_int2(i, b));
    }
    t->n_inv = (int)inv_items.size();
    std::vector<int4> all;
    // forward: operator M (lower_f); adjoint: M^T (!lower_f).  Item order
    // [first block fwd][M's tiles][M^T's tiles, TF32 only][first block adj]
    // keeps every split launch one contiguous range.
    t->a_mn_b = t->tf32 ? 0 : 1;
    t->split_f.off = (int)all.size();
    first_block_items(dims, batch, lower_f, t->kpb, all);
    const int op_off = (int)all.size();
    operator_items(dims, batch, lower_f, t->kpb, all);
    t->split_f.count = (int)all.size() - t->split_f.off;
    t->split_b.off = t->a_mn_b ? op_off : (int)all.size();
    if (!t->a_mn_b) operator_items(dims, batch, !lower_f, t->kpb, all);
    t->split_b_first.off = (int)all.size();
    first_block_items(dims, batch, !lower_f, t->kpb, all);
    t->split_b_first.count = (int)all.size() - t->split_b_first.off;
    t->split_b.count = (int)all.size() - t->split_b.off;
    solve_items(dims, batch, lower_f, t->kpb, all, t->inv_f, t->upd_f);
    solve_items(dims, batch, !lower_f, t->kpb, all, t->inv_b, t->upd_b);
    // dA: operands P (kind 0, rows na, K nr) and Q (kind 1), then the masked product
    t->split_d.off = (int)all.size();
    for (int kind = 0; kind < 2; ++kind)
        for (int i = 0; i < batch; ++i) {
            const int na = dims[4 * i], nr = dims[4 * i + 1];
            if (na == 0 || nr == 0) continue;
            for (int rt = 0; rt < (na + TR - 1) / TR; ++rt)
                for (int kt = 0; kt < nkt_d[i]; ++kt) all.push_back(make_int4(kind, i, rt, kt));
        }
    t->split_d.count = (int)all.size() - t->split_d.off;
    {
        std::vector<std::pair<int, int4>> g;
        for (int i = 0; i < batch; ++i) {
            const int na = dims[4 * i];
            const int nblk = (na + TR - 1) / TR;
            for (int rt = 0; rt < nblk; ++rt)
                for (int c = 0; c < nblk; ++c) {
                    const bool on = tri_lower ? rt >= c : rt <= c;
                    const int nk = on ? nkt_d[i] : 0;
                    g.push_back({nk, mk_item(i, rt, c, 0, 0, nk)});
                }
        }
        std::stable_sort(g.begin(), g.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        t->gemm_d.off = (int)all.size();
        for (auto& x : g) all.push_back(x.second);
        t->gemm_d.count = (int)all.size() - t->gemm_d.off;
    }
    if ((e = track(t, &t->items, all)) != cudaSuccess) return e;
    if ((e = track(t, &t->off_s, off_s)) != cudaSuccess) return e;
    if ((e = track(t, &t->off_inv, off_inv)) != cudaSuccess) return e;
    if ((e = track(t, &t->off_x, off_x)) != cudaSuccess) return e;
    if ((e = track(t, &t->off_d, off_d)) != cudaSuccess) return e;
    if ((e = track(t, &t->nkt_s, nkt_s)) != cudaSuccess) return e;
    if ((e = track(t, &t->nkt_x, nkt_x)) != cudaSuccess) return e;
    if ((e = track(t, &t->nkt_d, nkt_d)) != cudaSuccess) return e;
    if ((e = track(t, &t->info_a, info_a)) != cudaSuccess) return e;
    if ((e = track(t, &t->info_y, info_y)) != cudaSuccess) return e;
    if ((e = track(t, &t->info_p, info_p)) != cudaSuccess) return e;
    if ((e = track(t, &t->inv_items, inv_items)) != cudaSuccess) return e;
    if ((e = track_planes(t, &t->sp, ts, t->sp_l)) != cudaSuccess) return e;
    if ((e = track_planes(t, &t->inv, ti, t->inv_l)) != cudaSuccess) return e;
    if ((e = track_planes(t, &t->invt, ti, t->inv_l)) != cudaSuccess) return e;
    if ((e = track_planes(t, &t->xp, tx, t->xp_l)) != cudaSuccess) return e;
    if ((e = track_planes(t, &t->wp, td, t->d_l)) != cudaSuccess) return e;
    if ((e = track_planes(t, &t->xq, td, t->d_l)) != cudaSuccess) return e;
    return cudaSuccess;
}

// The 128 x 128 inverses (and their transposes) from the plan's 64 x 64
// FP32 inverses, which the caller has formed.
cudaError_t batch_tc_inverses(iclblasHandle_t h, const iclblasBatchPlan* plan, const float* const* A)
{
    const BatchTc& t = *plan->tc;
    if (t.n_inv == 0) return cudaSuccess;
    InvLaunch p{};
    p.items = t.inv_items;
    p.dims = plan->main.dims;
    p.inv64_off = plan->inv_off;
    p.inv64 = plan->inv;
    p.A = A;
    p.lower = t.lower_f;
    p.op = t.op_f;
    p.w = opnd(t.inv, t.inv_l, t.off_inv, nullptr, t.kpb);
    p.wt = opnd(t.invt, t.inv_l, t.off_inv, nullptr, t.kpb);
    p.nlev = t.nlev;
    if (t.tf32) btc_inv_kernel<true, float><<<t.n_inv, 256, inv_smem_bytes<float>(), h->stream>>>(p);
    else if (t.nlev == 3) btc_inv_kernel<false, double><<<t.n_inv, 256, inv_smem_bytes<double>(), h->stream>>>(p);
    else btc_inv_kernel<false, float><<<t.n_inv, 256, inv_smem_bytes<float>(), h->stream>>>(p);
    return cudaGetLastError();
}

// One blocked solve, in place on B: the forward operator (adjoint = 0) or
// its transpose, with the inverse planes already formed; operator_ready:
// the operator tiles of the plan's last forward call are still valid
// (same A), so the adjoint (BF16 modes) splits only its first block.
cudaError_t batch_tc_solve(iclblasHandle_t h, const iclblasBatchPlan* plan, int adjoint, float alpha,
                           const float* const* A, float* const* B, int operator_ready)
{
    const BatchTc& t = *plan->tc;
    // operator tiles: L[r][k] = S[r][k], S = M = op(A) (forward, and the
    // adjoint in the BF16 modes, which reads them MN-major) or M^T (TF32
    // adjoint); M[i][j] = A[i + j*lda] (op N) or A[j + i*lda]
    const int s_rmajor = (adjoint && !t.a_mn_b) ? !t.op_f : t.op_f;
    const SplitKind ks{A, t.info_a, s_rmajor, opnd(t.sp, t.sp_l, t.off_s, t.nkt_s)};
    // right-hand sides: row j = right-hand side j, K = solve row (left: B's
    // columns, L[j][k] = B[k + j*ldb]; right: B's rows, L[j][k] = B[j + k*ldb])
    const Opnd xp = opnd(t.xp, t.xp_l, t.off_x, t.nkt_x);
    const SplitKind ky{const_cast<const float* const*>(B), t.info_y, t.right ? 0 : 1, xp};
    const TcRange sr = !adjoint ? t.split_f : ((operator_ready && t.a_mn_b) ? t.split_b_first : t.split_b);
    cudaError_t e = run_split(h, t, sr, ks, ky);
    if (e != cudaSuccess) return e;
    const std::vector<TcRange>& invs = adjoint ? t.inv_b : t.inv_f;
    const std::vector<TcRange>& upds = adjoint ? t.upd_b : t.upd_f;
    MmaArgs mi;
    mi.kind = kEpiInv;
    mi.a = opnd(adjoint ? t.invt : t.inv, t.inv_l, t.off_inv, nullptr, t.kpb);
    mi.b = xp;
    mi.C = B;
    mi.cinfo = t.info_p;  // rows na, columns nr, ld ldb
    mi.ct = t.right;
    mi.c_alpha = alpha;
    mi.w = xp;
    MmaArgs mu = mi;
    mu.kind = kEpiUpd;  // planes of Y_s = B_s - acc; B_s is only read
    mu.a = opnd(t.sp, t.sp_l, t.off_s, t.nkt_s);
    mu.a_mn = adjoint ? t.a_mn_b : 0;
    for (size_t q = 0; q < invs.size(); ++q) {
        if ((e = run_mma(h, t, upds[q], mu)) != cudaSuccess) return e;
        if ((e = run_mma(h, t, invs[q], mi)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// dA = scale * op(P) op(Q)^T on the stored triangle (zero elsewhere), the
// operands given as the batched adjoint chooses them (left: P, Q are
// na x nr with ld ldb; right: nr x na).
cudaError_t batch_tc_dA(iclblasHandle_t h, const iclblasBatchPlan* plan, float scale, const float* const* P,
                        const float* const* Q, float* const* dA)
{
    const BatchTc& t = *plan->tc;
    const Opnd wp = opnd(t.wp, t.d_l, t.off_d, t.nkt_d), xq = opnd(t.xq, t.d_l, t.off_d, t.nkt_d);
    // left: L[i][k] = P[i + k*ldb]; right: L[i][k] = P[k + i*ldb]
    const SplitKind kp{P, t.info_p, t.right ? 1 : 0, wp}, kq{Q, t.info_p, t.right ? 1 : 0, xq};
    cudaError_t e = run_split(h, t, t.split_d, kp, kq);
    if (e != cudaSuccess) return e;
    MmaArgs m;
    m.kind = kEpiMask;
    m.a = wp;
    m.b = xq;
    m.C = dA;
    m.cinfo = t.info_a;  // rows na, columns na, ld lda
    m.ct = 0;
    m.c_alpha = scale;
    m.c_beta = 0.f;
    m.mask = (t.tri_lower ? 1 : 2) | (t.unit ? 4 : 0);
    m.w = Opnd{};
    return run_mma(h, t, t.gemm_d, m);
}

cudaError_t batch_tc_create_gemm(iclblasHandle_t h, iclblasBatchPlan* plan, const std::vector<int>& dims, int ta,
                                 int tb)
{
    cudaError_t e = set_attrs(h->device);
    if (e != cudaSuccess) return e;
    auto* t = new BatchTc();
    plan->tc = t;
    mode_products(h->math, t->tf32, t->nlev, t->nprod, t->pa, t->pb);
    const int KT = t->tf32 ? 32 : 64;
    t->kpb = TR / KT;
    t->ta = ta;
    t->tb = tb;
    const int batch = plan->batch;
    std::vector<long> off_a(batch), off_b(batch);
    std::vector<int> nkt(batch);
    std::vector<int4> ia(batch), ib(batch), ic(batch);
    std::vector<int4> all;
    std::vector<std::pair<long, int4>> g;
    long na_t = 0, nb_t = 0;
    t->split_g.off = 0;
    for (int i = 0; i < batch; ++i) {
        const int m = dims[6 * i], n = dims[6 * i + 1], k = dims[6 * i + 2];
        const int nmt = (m + TR - 1) / TR, nnt = (n + TR - 1) / TR, nk = (k + KT - 1) / KT;
        off_a[i] = na_t;
        off_b[i] = nb_t;
        nkt[i] = nk;
        na_t += (long)nmt * nk;
        nb_t += (long)nnt * nk;
        ia[i] = make_int4(m, k, dims[6 * i + 3], 0);
        ib[i] = make_int4(n, k, dims[6 * i + 4], 0);
        ic[i] = make_int4(m, n, dims[6 * i + 5], 0);
        if (m == 0 || n == 0) continue;
        for (int rt = 0; rt < nmt; ++rt)
            for (int kt = 0; kt < nk; ++kt) all.push_back(make_int4(0, i, rt, kt));
        for (int rt = 0; rt < nnt; ++rt)
            for (int kt = 0; kt < nk; ++kt) all.push_back(make_int4(1, i, rt, kt));
        for (int rt = 0; rt < nmt; ++rt)
            for (int c = 0; c < nnt; ++c) g.push_back({(long)nk, mk_item(i, rt, c, 0, 0, nk)});
    }
    t->split_g.count = (int)all.size();
    std::stable_sort(g.begin(), g.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    t->gemm_g.off = (int)all.size();
    for (auto& x : g) all.push_back(x.second);
    t->gemm_g.count = (int)all.size() - t->gemm_g.off;
    if ((e = track(t, &t->items, all)) != cudaSuccess) return e;
    if ((e = track(t, &t->off_ga, off_a)) != cudaSuccess) return e;
    if ((e = track(t, &t->off_gb, off_b)) != cudaSuccess) return e;
    if ((e = track(t, &t->nkt_g, nkt)) != cudaSuccess) return e;
    if ((e = track(t, &t->info_ga, ia)) != cudaSuccess) return e;
    if ((e = track(t, &t->info_gb, ib)) != cudaSuccess) return e;
    if ((e = track(t, &t->info_gc, ic)) != cudaSuccess) return e;
    if ((e = track_planes(t, &t->ap, na_t, t->ap_l)) != cudaSuccess) return e;
    if ((e = track_planes(t, &t->bp, nb_t, t->bp_l)) != cudaSuccess) return e;
    return cudaSuccess;
}

// C_i = alpha op(A_i) op(B_i) + beta C_i: both operands split into planes,
// then one product launch over every instance's tiles.
cudaError_t batch_tc_gemm(iclblasHandle_t h, const iclblasBatchPlan* plan, float alpha, const float* const* A,
                          const float* const* B, float beta, float* const* C)
{
    const BatchTc& t = *plan->tc;
    const Opnd ap = opnd(t.ap, t.ap_l, t.off_ga, t.nkt_g), bp = opnd(t.bp, t.bp_l, t.off_gb, t.nkt_g);
    // A: L[i][k] = op(A)[i][k] (op N: A[i + k*lda]); B: L[j][k] = op(B)[k][j]
    // (op N: B[k + j*ldb])
    const SplitKind ka{A, t.info_ga, t.ta ? 1 : 0, ap}, kb{B, t.info_gb, t.tb ? 0 : 1, bp};
    cudaError_t e = run_split(h, t, t.split_g, ka, kb);
    if (e != cudaSuccess) return e;
    MmaArgs m;
    m.a = ap;
    m.b = bp;
    m.C = C;
    m.cinfo = t.info_gc;
    m.c_alpha = alpha;
    m.c_beta = beta;
    m.w = Opnd{};
    return run_mma(h, t, t.gemm_g, m);
}

}  // namespace iclb
