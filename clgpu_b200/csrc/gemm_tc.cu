// Tensor-core GEMM for the TF32 / 3xBF16 / 6xBF16 math modes and HGEMM
// (sm_100a).
//
// C = alpha*op(A)*op(B) + beta*C in FP32 (and complex FP32, or IEEE half for
// HGEMM) computed on the 5th-generation tensor cores.  No reference
// counterpart: the reference's GEMMs are FP32 SIMD kernels; these are the
// library's split-precision math modes (FP32 accuracy from BF16 products)
// and its half-precision GEMM.
//
// 1. Pre-pass (split kernel): each operand op(X) is rewritten K-major (row r
//    holds its K values contiguously, zero-padded to a multiple of the
//    K block) as
//      TF32:  one FP32 plane rounded to TF32 (cvt.rna.tf32.f32);
//      BF16:  hi = bf16(x), mid = bf16(x - hi), lo = bf16(x - hi - mid)
//             (each difference is exact in FP32).
//    Complex operands are embedded in a real GEMM with the same flop count:
//    A' = [re A | im A] (M x 2K) and, for each column j of op(B), the rows
//    2j = [re b_j | -im b_j] and 2j+1 = [im b_j | re b_j] of B'' (2N x 2K), so
//    C'' = A' B''^T holds re C(:,j) in column 2j and im C(:,j) in 2j+1.
// 2. Main kernel: persistent, one CTA per SM, CTA tile 128 x 256, 6 warps:
//      warp 0     TMA producer: 128-byte-swizzled tiles of the split planes
//                 into a 4-stage shared-memory ring (mbarrier expect-tx);
//      warp 1     allocates 512 TMEM columns (two 128x256 FP32 accumulators)
//                 and one thread issues tcgen05.mma (M=128, N=256, K=32 bytes
//                 per instruction, 4 per stage) and tcgen05.commit;
//      warps 2-9  epilogue: two warps per 32-lane TMEM quarter, 128 columns
//                 each (two halves of four warps).
//    Each pipeline stage is one (K block, product) pair.  The BF16 modes run
//    the products of every K block small-first -- 3xBF16: mid*hi, hi*mid,
//    hi*hi; 6xBF16: lo*hi, hi*lo, mid*mid, mid*hi, hi*mid, hi*hi -- into a
//    fresh accumulator per chunk of one K block.  The tensor core's FP32
//    accumulation loses a fraction of an ulp of the running value at every
//    update; starting each chunk from zero and adding the largest term last
//    keeps that loss at the chunk's size, and the chunks are summed in FP32
//    in registers (the two accumulator buffers let the next chunk's MMAs run
//    while the previous chunk is drained).  TF32 uses one chunk per tile.
// 3. Epilogue.  Single-chunk tiles (TF32, HGEMM) are read from TMEM 16
//    columns at a time; each half of the epilogue warps writes alpha*acc
//    (+ beta*C) into a 128 x 16 shared-memory box laid out like C and one
//    thread stores it with TMA (C read by TMA for beta != 0), double
//    buffered.  Column-at-a-time stores of a warp's 32 rows (64 or 128 B per
//    column) ran these kernels at a fifth of the HBM write rate when the
//    epilogue, not the MMA, bounds the tile (small K).  A TMA store clips the
//    contiguous dimension only at 16-byte granularity, so the C map stops at
//    M rounded down to 16 bytes and the last few rows are stored directly.
//    The BF16 modes with several chunks keep their running sum in registers
//    and stage it the same way once the last chunk is drained; triangular
//    output and a C that TMA cannot address (16-byte alignment) are stored
//    directly.
// 4. HGEMM operands are read in place in either layout: K-major (op T of A,
//    op N of B) through the plane descriptors, MN-major (op N of A, op T of
//    B) as boxes of 64 rows x 64 K with an MN-major shared-memory descriptor;
//    only an operand TMA cannot address is packed first.
// Every mbarrier wait is bounded; on timeout the kernel records
// kDevWaitTimeout, waits (bounded) for its own TMA copies, frees TMEM and
// returns.  Every TMA load targets the issuing CTA's own shared memory.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <type_traits>

#include "common.cuh"

namespace iclb {
namespace tc {
namespace {

constexpr int BM = 128;
constexpr int ROW_BYTES = 128;                  // one K block per tile row
constexpr int A_TILE = BM * ROW_BYTES;          // 16 KiB
constexpr int RING_BYTES = 192 * 1024;          // the stage ring
constexpr int EPI_GROUP = 16;                  // FP32 output columns per staged store (half: 32)
// Output element type of a kernel instantiation: FP32, IEEE half (HGEMM),
// or complex FP32 with the real GEMM's columns 2j, 2j+1 holding (re, im) of
// column j.
enum : int { OUT_F32 = 0, OUT_F16 = 1, OUT_C64 = 2 };
// output columns per staged store: one 8 KiB buffer of 128 rows
template <int OUT>
constexpr int group_cols() { return OUT == OUT_F16 ? 32 : EPI_GROUP; }
constexpr int EPI_BUF_BYTES = 8192;             // one staging buffer: 128 rows x 16 FP32 columns
constexpr int EPI_STAGE_BYTES = 4 * EPI_BUF_BYTES;  // two buffers for each half of the epilogue warps
constexpr int MN_CHUNK_BYTES = 8192;            // MN-major operand: 64 rows x 64 K of 16-bit values
constexpr int SMEM_BYTES = RING_BYTES + 1024 /*barriers*/ + EPI_STAGE_BYTES + 1024 /*alignment*/;
static_assert(SMEM_BYTES <= 232448, "shared memory per CTA");
// Output tile 128 x BN: 256 columns, or 128 when the 256-wide tiles would
// leave a quarter or more of the SMs idle (more, smaller tiles).
template <int BN_>
struct Tile {
    static constexpr int BN = BN_;
    static constexpr int B_TILE = BN * ROW_BYTES;             // 32 or 16 KiB
    static constexpr int STAGE_BYTES = A_TILE + B_TILE;       // 48 or 32 KiB
    static constexpr int STAGES = RING_BYTES / STAGE_BYTES;   // 4 or 6
    static constexpr int TMEM_COLS = 2 * BN;                  // two accumulators
    static constexpr int EPI_COLS = BN / 2;                   // columns per epilogue warp
};
constexpr int EPI_WARPS = 8;                    // two per TMEM lane quarter
constexpr int THREADS = 64 + 32 * EPI_WARPS;    // producer, MMA, epilogue
constexpr int GROUP_M = 16;                     // tile raster: 16 M-tiles per band
constexpr unsigned long long kWaitNs = 2000000000ull;  // a wait gives up after 2 s

struct Params {
    int M, N;          // output rows / columns of the (real) GEMM
    int kblocks;       // K_pad / elements-per-row-block
    int nprod;         // products per K block (1, 3 or 6)
    int chunk;         // K blocks per TMEM chunk (drained into registers)
    int pa[6], pb[6];  // split level of A and B for each product
    int complex_out;   // columns come in (re, im) pairs
    float alpha_re, alpha_im, beta_re, beta_im;
    float* C;
    long ldc;          // in elements of the output type
    int* status;
    int tri;           // 0: full C; 1: only row >= col is written; 2: only row <= col (real C)
    int ab_fmt;        // kind::f16 operand format: 1 bf16 (split planes), 0 f16 (HGEMM)
    int out_half;      // real C stored as IEEE half (HGEMM)
    int a_mn, b_mn;    // operand stored MN-major (its rows contiguous; 16-bit operands only)
    int c_tma;         // C written (and, for beta != 0, read) through the C tensor map
    int m_tma;         // rows the C tensor map covers (M rounded down to 16 bytes)
};

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
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

__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, int x, int y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(smem_dst)), "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
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

// 32 lanes x 16 consecutive columns of FP32 from TMEM.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor, K-major, 128-byte swizzle: rows of 128 B,
// 8-row groups 1024 B apart (SBO), version 1, layout type 2.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;           // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32; // stride byte offset: next 8-row group
    d |= (uint64_t)1u << 46;           // descriptor version
    d |= (uint64_t)2u << 61;           // SWIZZLE_128B
    return d;
}

// Shared-memory matrix descriptor, MN-major, 128-byte swizzle: rows of 128 B
// hold 64 consecutive M (or N) indices of one K index; 8-K groups 1024 B
// apart (SBO); the next 64 M indices 8 KiB further (LBO: one TMA box of
// 64 x 64).  One MMA (K = 16) spans two 8-K groups, so the start address
// advances by 2048 B per MMA.
__device__ __forceinline__ uint64_t smem_desc_mn_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)(MN_CHUNK_BYTES >> 4) << 16;  // leading byte offset: next 64 rows
    d |= (uint64_t)(1024u >> 4) << 32;           // stride byte offset: next 8 K indices
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

// Instruction descriptor: FP32 accumulator, A/B format (0 = F16, 1 = BF16,
// 2 = TF32), A / B K-major or MN-major (bits 15, 16), N = bn, M = 128.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t ab_format, int bn, int a_mn = 0, int b_mn = 0)
{
    return (1u << 4) | (ab_format << 7) | (ab_format << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void tile_coords(int t, int tiles_m, int tiles_n, int& tm, int& tn)
{
    const int per_band = GROUP_M * tiles_n;
    const int band = t / per_band;
    const int first_m = band * GROUP_M;
    const int rows = min(GROUP_M, tiles_m - first_m);
    const int in_band = t - band * per_band;
    tm = first_m + in_band % rows;
    tn = in_band / rows;
}

// Tile rows [lo, hi) of tile column tn that hold an element of C's triangle
// (tiles of bm x bn outputs).
__device__ __forceinline__ void tri_rows(int tri, int tn, int tiles_m, int bm, int bn, int& lo, int& hi)
{
    if (tri == 1) {  // some row >= some column: last row of the tile >= first column
        lo = (tn * bn) / bm;
        hi = tiles_m;
    } else {         // first row of the tile <= last column
        lo = 0;
        hi = min(tiles_m, (tn * bn + bn - 1) / bm + 1);
    }
    if (lo > hi) lo = hi;
}

// Number of tiles a CTA loop visits: all, or only those meeting C's triangle.
__device__ __forceinline__ int tile_count(int tri, int tiles_m, int tiles_n, int bm, int bn)
{
    if (tri == 0) return tiles_m * tiles_n;
    int c = 0;
    for (int tn = 0; tn < tiles_n; ++tn) {
        int lo, hi;
        tri_rows(tri, tn, tiles_m, bm, bn, lo, hi);
        c += hi - lo;
    }
    return c;
}

// Tile t of that visit order: the grouped order for a full C, column by
// column over the triangle's tiles otherwise.
__device__ __forceinline__ void tile_at(int tri, int t, int tiles_m, int tiles_n, int bm, int bn, int& tm, int& tn)
{
    if (tri == 0) {
        tile_coords(t, tiles_m, tiles_n, tm, tn);
        return;
    }
    for (tn = 0; tn < tiles_n; ++tn) {
        int lo, hi;
        tri_rows(tri, tn, tiles_m, bm, bn, lo, hi);
        if (t < hi - lo) {
            tm = lo + t;
            return;
        }
        t -= hi - lo;
    }
    tm = 0;
}

__device__ __forceinline__ bool in_tri(int tri, int row, int col)
{
    return tri == 0 || (tri == 1 ? row >= col : row <= col);
}

// One operand tile (rows x one K block) into shared memory: a single box for
// K-major storage, boxes of 64 rows x 64 K at 8 KiB steps for MN-major.
__device__ __forceinline__ void load_operand(uint8_t* dst, const CUtensorMap* map, int mn, int rows, int kx, int r0,
                                             uint64_t* bar)
{
    if (mn) {
        for (int i = 0; i < rows / 64; ++i) tma_load_2d(dst + i * MN_CHUNK_BYTES, map, r0 + i * 64, kx, bar);
    } else {
        tma_load_2d(dst, map, kx, r0, bar);
    }
}

// ---------------------------------------------------------------- epilogue stores
// The four epilogue warps that share one half of the tile's columns
// synchronise on a named barrier of their own (ids 1 and 2; 0 is
// __syncthreads).
__device__ __forceinline__ void group_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
// true when v holds in every thread of the group
__device__ __forceinline__ bool group_all(int id, bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.b32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, 128, p;\n\t"
        "selp.b32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, const void* smem_src, int x, int y)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
                 ::"l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(smem_src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// State of one half's staged stores.
struct EpiGroup {
    uint8_t* buf;   // two staging buffers of EPI_BUF_BYTES
    uint64_t* bar;  // their load barriers (beta != 0)
    int id;         // named barrier of the half
    bool leader;    // the thread that issues the copies
    int gi;         // groups staged so far: buffer gi & 1, barrier parity (gi >> 1) & 1
};

// alpha * v + beta * c with the rounding of the reference's real GEMM
// epilogue (beta == 0: C is not read)
__device__ __forceinline__ float axpby(const Params& p, bool beta_zero, float v, float c)
{
    return beta_zero ? __fmul_rn(p.alpha_re, v) : fmaf(p.alpha_re, v, __fmul_rn(p.beta_re, c));
}
__device__ __forceinline__ float2 caxpby(const Params& p, bool beta_zero, float re, float im, float2 c)
{
    float2 o;
    o.x = fmaf(p.alpha_re, re, -p.alpha_im * im);
    o.y = fmaf(p.alpha_re, im, p.alpha_im * re);
    if (!beta_zero) {
        o.x += fmaf(p.beta_re, c.x, -p.beta_im * c.y);
        o.y += fmaf(p.beta_re, c.y, p.beta_im * c.x);
    }
    return o;
}

// Direct epilogue, one group of 16 columns of one row (C not reachable by
// TMA, triangular output, or the rows a TMA store cannot clip exactly); C
// is read before any of the group is stored, so the loads overlap (columns
// of C never alias for ldc >= M).
template <int OUT, int W>
__device__ __forceinline__ void direct_group(const float (&v)[W], const Params& p, int row, int cx)
{
    if (row >= p.M) return;
    const bool beta_zero = p.beta_re == 0.f && p.beta_im == 0.f;
    if constexpr (OUT == OUT_C64) {
        float2* const C2 = (float2*)p.C;
        float2 cv[W / 2];
#pragma unroll
        for (int j = 0; j < W / 2; ++j) {
            const int col = cx + 2 * j;
            cv[j] = (!beta_zero && col < p.N) ? C2[(long)(col >> 1) * p.ldc + row] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < W / 2; ++j) {
            const int col = cx + 2 * j;
            if (col < p.N) C2[(long)(col >> 1) * p.ldc + row] = caxpby(p, beta_zero, v[2 * j], v[2 * j + 1], cv[j]);
        }
    } else {
        using T = typename std::conditional<OUT == OUT_F16, __half, float>::type;
        T* const Ct = (T*)p.C;
        float cv[W];
#pragma unroll
        for (int j = 0; j < W; ++j) {
            const int col = cx + j;
            cv[j] = (!beta_zero && col < p.N && in_tri(p.tri, row, col)) ? (float)Ct[(long)col * p.ldc + row] : 0.f;
        }
#pragma unroll
        for (int j = 0; j < W; ++j) {
            const int col = cx + j;
            if (col < p.N && in_tri(p.tri, row, col)) Ct[(long)col * p.ldc + row] = (T)axpby(p, beta_zero, v[j], cv[j]);
        }
    }
}

// Staged epilogue, one group of 16 columns of one half of a CTA's tile
// (128 rows): the half's four warps write alpha*v (+ beta*C) into a buffer
// laid out as C's own column-major box, and one thread stores the box with
// TMA, which clips columns past C's edge.  Along the rows a TMA store clips
// only at 16-byte granularity, so the map covers the first m_tma rows (M
// rounded down to 16 bytes) and the rows in [m_tma, M) are stored directly
// by their threads.  For beta != 0 the same box of C is first loaded into
// the buffer by TMA.  A buffer is refilled once the store that last read it
// has finished reading.  The arithmetic is that of the direct stores.
// Returns false (in every thread of the half) when a wait gave up; the
// leader's load into the current buffer may then still be in flight.
template <int OUT>
__device__ __forceinline__ bool stage_group(const float (&v)[group_cols<OUT>()], const Params& p, const CUtensorMap* mC,
                                            EpiGroup& eg, int r, int row0, int cx, volatile int* abort_flag)
{
    constexpr int GW = group_cols<OUT>();
    constexpr uint32_t box_bytes = EPI_BUF_BYTES;
    const bool beta_zero = p.beta_re == 0.f && p.beta_im == 0.f;
    const int b = eg.gi & 1;
    const uint32_t ph = (uint32_t)(eg.gi >> 1) & 1u;
    uint8_t* buf = eg.buf + b * EPI_BUF_BYTES;
    const int x = OUT == OUT_C64 ? 2 * row0 : row0, y = OUT == OUT_C64 ? cx / 2 : cx;
    // this thread's row of the group into the buffer (C from the buffer for
    // beta != 0), or straight to C for the rows past the map
    auto fill = [&]() {
        if (row0 + r < p.m_tma) {
            if constexpr (OUT == OUT_C64) {
                float2* const sb = (float2*)buf + r;
#pragma unroll
                for (int j = 0; j < GW / 2; ++j)
                    sb[j * 128] = caxpby(p, beta_zero, v[2 * j], v[2 * j + 1], beta_zero ? make_float2(0.f, 0.f) : sb[j * 128]);
            } else {
                using T = typename std::conditional<OUT == OUT_F16, __half, float>::type;
                T* const sb = (T*)buf + r;
#pragma unroll
                for (int j = 0; j < GW; ++j)
                    sb[j * 128] = (T)axpby(p, beta_zero, v[j], beta_zero ? 0.f : (float)sb[j * 128]);
            }
        } else {
            direct_group<OUT, GW>(v, p, row0 + r, cx);  // rows past the map (none past M)
        }
    };
    if (beta_zero) {
        // One barrier per group.  This group's buffer was last read by the
        // store two groups back, which the leader saw finish reading before
        // the previous group's barrier; before this group's barrier it waits
        // for the previous group's store, whose buffer the next group fills.
        fill();
        fence_async_smem();
        if (eg.leader) bulk_wait_read0();
        group_sync(eg.id);
        if (eg.leader) {
            tma_store_2d(mC, buf, x, y);
            bulk_commit();
        }
        ++eg.gi;
        return true;
    }
    if (eg.leader) {
        bulk_wait_read1();
        mbar_expect_tx(&eg.bar[b], box_bytes);
        tma_load_2d(buf, mC, x, y, &eg.bar[b]);
    }
    group_sync(eg.id);
    const bool lok = mbar_wait(&eg.bar[b], ph, abort_flag);
    if (lok) fill();
    fence_async_smem();
    if (!group_all(eg.id, lok)) return false;
    if (eg.leader) {
        tma_store_2d(mC, buf, x, y);
        bulk_commit();
    }
    ++eg.gi;
    return true;
}

// The epilogue warps' loops over a CTA's tiles (tiles of tile_rows x BN;
// this CTA's rows start row_off into each).  Warp w serves TMEM lane quarter
// w % 4 and one half (EPI_COLS columns) of the tile.
//
// Single chunk (the whole K in one accumulator: TF32, HGEMM): 16 columns at a
// time straight from TMEM into the staged (or direct) stores; the
// accumulator is released after the last group.
template <int OUT, int BN, int EPI_COLS, class Arrive>
__device__ __forceinline__ void epilogue_single(const Params& p, const CUtensorMap* mC, int t0, int tstep, int ntiles,
                                                int tiles_m, int tiles_n, int tile_rows, int row_off,
                                                uint32_t tmem_base, uint64_t* tfull, Arrive arrive, uint8_t* epi_buf,
                                                uint64_t* cbar, volatile int* abort_flag)
{
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int q = warp & 3, half = (warp - 2) / 4;
    const int r = q * 32 + lane;  // row within the CTA's 128
    constexpr int GW = group_cols<OUT>();
    static_assert(EPI_COLS % GW == 0, "epilogue columns");
    EpiGroup eg{epi_buf + half * 2 * EPI_BUF_BYTES, cbar + half * 2, 1 + half, q == 0 && lane == 0, 0};
    int acc = 0;
    uint32_t acc_ph = 0;
    for (int t = t0; t < ntiles; t += tstep) {
        int w = 1;
        if (lane == 0) w = mbar_wait(&tfull[acc], acc_ph, abort_flag) ? 1 : 0;
        // the half's four warps leave together (a warp that gave up has set
        // the abort flag, so the others' waits end too)
        if (!group_all(eg.id, __shfl_sync(0xffffffffu, w, 0) != 0)) break;
        tc_fence_after();
        int tm, tn;
        tile_at(p.tri, t, tiles_m, tiles_n, tile_rows, BN, tm, tn);
        const int row0 = tm * tile_rows + row_off, col0 = tn * BN + half * EPI_COLS;
        const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN + half * EPI_COLS);
        bool stored = true;
#pragma unroll 1
        for (int g = 0; g < EPI_COLS / GW && stored; ++g) {
            float v[GW];
            if constexpr (GW == 32)
                tmem_ld32(taddr + (uint32_t)(g * GW), v);
            else
                tmem_ld16(taddr + (uint32_t)(g * GW), v);
            if (p.c_tma)
                stored = stage_group<OUT>(v, p, mC, eg, r, row0, col0 + g * GW, abort_flag);
            else
                direct_group<OUT, GW>(v, p, row0 + r, col0 + g * GW);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) arrive(acc);
        if (++acc == 2) { acc = 0; acc_ph ^= 1; }
        if (!stored) {
            if (eg.leader) mbar_drain(&eg.bar[eg.gi & 1], (uint32_t)(eg.gi >> 1) & 1u);
            break;
        }
    }
    if (eg.leader) bulk_wait_all();
}

// Several chunks (the BF16 modes): each chunk is drained into FP32 registers
// and released at once; only the running sum stays live across the chunk
// loop.  The sum is stored through the staged TMA path when C allows it
// (direct column-at-a-time stores of a 128-row tile took 5.5 us, a third of
// a 512 x 4096 x 512 3xBF16 call), else directly.
template <int OUT, int BN, int EPI_COLS, class Arrive>
__device__ __forceinline__ void epilogue_multi(const Params& p, const CUtensorMap* mC, int t0, int tstep, int ntiles,
                                               int tiles_m, int tiles_n, int tile_rows, int row_off,
                                               uint32_t tmem_base, uint64_t* tfull, Arrive arrive, uint8_t* epi_buf,
                                               uint64_t* cbar, volatile int* abort_flag)
{
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int q = warp & 3, half = (warp - 2) / 4;
    const int r = q * 32 + lane;  // row within the CTA's 128
    constexpr int GW = group_cols<OUT>();
    static_assert(EPI_COLS % GW == 0 && EPI_COLS % 8 == 0, "epilogue columns");
    EpiGroup eg{epi_buf + half * 2 * EPI_BUF_BYTES, cbar + half * 2, 1 + half, q == 0 && lane == 0, 0};
    const int nchunks = (p.kblocks + p.chunk - 1) / p.chunk;
    int acc = 0;
    uint32_t acc_ph = 0;
    bool ok = true;
    for (int t = t0; t < ntiles && ok; t += tstep) {
        float sum[EPI_COLS];
#pragma unroll
        for (int j = 0; j < EPI_COLS; ++j) sum[j] = 0.f;
        for (int c = 0; c < nchunks; ++c) {
            int w = 1;
            if (lane == 0) w = mbar_wait(&tfull[acc], acc_ph, abort_flag) ? 1 : 0;
            ok = __shfl_sync(0xffffffffu, w, 0) != 0;
            if (!ok) break;
            tc_fence_after();
            const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN + half * EPI_COLS);
#pragma unroll
            for (int g = 0; g < EPI_COLS / 32; ++g) {
                float v[32];
                tmem_ld32(taddr + (uint32_t)(g * 32), v);
#pragma unroll
                for (int j = 0; j < 32; ++j) sum[g * 32 + j] += v[j];
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) arrive(acc);
            if (++acc == 2) { acc = 0; acc_ph ^= 1; }
        }
        // the half's four warps go on together (a warp that gave up has set
        // the abort flag, so the others' waits end too)
        ok = group_all(eg.id, ok);
        if (!ok) break;
        int tm, tn;
        tile_at(p.tri, t, tiles_m, tiles_n, tile_rows, BN, tm, tn);
        const int row0 = tm * tile_rows + row_off;
        const int col0 = tn * BN + half * EPI_COLS;
        if (p.c_tma) {
#pragma unroll
            for (int g = 0; g < EPI_COLS / GW; ++g) {
                float v[GW];
#pragma unroll
                for (int j = 0; j < GW; ++j) v[j] = sum[g * GW + j];
                if (ok) ok = stage_group<OUT>(v, p, mC, eg, r, row0, col0 + g * GW, abort_flag);
            }
            if (!ok) {
                if (eg.leader) mbar_drain(&eg.bar[eg.gi & 1], (uint32_t)(eg.gi >> 1) & 1u);
                break;
            }
        } else if (row0 + r < p.M) {
#pragma unroll
            for (int g = 0; g < EPI_COLS / 8; ++g) {
                float v[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) v[j] = sum[g * 8 + j];
                direct_group<OUT, 8>(v, p, row0 + r, col0 + g * 8);
            }
        }
    }
    if (eg.leader) bulk_wait_all();
}

template <bool TF32, int BN_, int OUT, bool SINGLE>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_tc_kernel(const __grid_constant__ CUtensorMap mA0, const __grid_constant__ CUtensorMap mA1,
                   const __grid_constant__ CUtensorMap mA2, const __grid_constant__ CUtensorMap mB0,
                   const __grid_constant__ CUtensorMap mB1, const __grid_constant__ CUtensorMap mB2,
                   const __grid_constant__ CUtensorMap mC, Params p)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* tiles = smem;
    using TC = Tile<BN_>;
    constexpr int BN = TC::BN, STAGES = TC::STAGES, STAGE_BYTES = TC::STAGE_BYTES, EPI_COLS = TC::EPI_COLS;
    uint64_t* full = (uint64_t*)(smem + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* tfull = empty + STAGES;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = (uint32_t*)(tempty + 2);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    uint64_t* cbar = (uint64_t*)(smem + RING_BYTES + 512);  // [half][buffer] C-load barriers
    uint8_t* epi_buf = smem + RING_BYTES + 1024;             // [half][buffer] staging

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int tiles_m = (p.M + BM - 1) / BM, tiles_n = (p.N + BN - 1) / BN;
    const int ntiles = tile_count(p.tri, tiles_m, tiles_n, BM, BN);
    const int steps = p.kblocks * p.nprod;
    constexpr bool MN_OK = OUT == OUT_F16;  // MN-major operands: HGEMM only

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], EPI_WARPS);  // one arrive per epilogue warp
        }
        for (int i = 0; i < 4; ++i) mbar_init(&cbar[i], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, TC::TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ---------------------------------------------------------- TMA producer
        if (lane == 0) {
            const CUtensorMap* ma[3] = {&mA0, &mA1, &mA2};
            const CUtensorMap* mb[3] = {&mB0, &mB1, &mB2};
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                int tm, tn;
                tile_at(p.tri, t, tiles_m, tiles_n, BM, BN, tm, tn);
                for (int st = 0; st < steps && ok; ++st) {
                    const int kb = st / p.nprod, pr = st % p.nprod;
                    if (!mbar_wait(&empty[s], ph ^ 1, abort_flag)) { ok = false; break; }
                    uint8_t* sa = tiles + s * STAGE_BYTES;
                    uint8_t* sb = sa + A_TILE;
                    mbar_expect_tx(&full[s], STAGE_BYTES);
                    const int kx = kb * (TF32 ? 32 : 64);
                    load_operand(sa, ma[p.pa[pr]], MN_OK && p.a_mn, BM, kx, tm * BM, &full[s]);
                    load_operand(sb, mb[p.pb[pr]], MN_OK && p.b_mn, BN, kx, tn * BN, &full[s]);
                    if (++s == STAGES) { s = 0; ph ^= 1; }
                }
            }
            if (!ok) {
                // wait (bounded) for the copies this thread issued, then leave
                for (int i = 0; i < STAGES; ++i) mbar_drain(&full[(s + i) % STAGES], ph);
            }
        }
    } else if (warp == 1) {
        // ---------------------------------------------------------- MMA issuer
        if (lane == 0) {
            const int a_mn = MN_OK && p.a_mn, b_mn = MN_OK && p.b_mn;
            const uint32_t idesc = instr_desc(TF32 ? 2u : (uint32_t)p.ab_fmt, BN, a_mn, b_mn);
            const uint64_t a_step = a_mn ? 128 : 2, b_step = b_mn ? 128 : 2;  // per MMA, 16-byte units
            int s = 0;
            uint32_t ph = 0;
            int acc = 0;
            uint32_t acc_ph = 0;
            bool ok = true;
            const int chunk_steps = p.chunk * p.nprod;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                for (int c0 = 0; c0 < steps && ok; c0 += chunk_steps) {
                    if (!mbar_wait(&tempty[acc], acc_ph ^ 1, abort_flag)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t d = tmem_base + (uint32_t)(acc * BN);
                    const int c1 = min(steps, c0 + chunk_steps);
                    for (int st = c0; st < c1; ++st) {
                        if (!mbar_wait(&full[s], ph, abort_flag)) { ok = false; break; }
                        tc_fence_after();
                        const uint32_t sa = smem_u32(tiles + s * STAGE_BYTES);
                        const uint32_t sb = sa + A_TILE;
                        const uint64_t da = a_mn ? smem_desc_mn_sw128(sa) : smem_desc_sw128(sa);
                        const uint64_t db = b_mn ? smem_desc_mn_sw128(sb) : smem_desc_sw128(sb);
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk)  // 4 x 32 bytes of K per stage
                            umma<TF32>(d, da + a_step * kk, db + b_step * kk, idesc, (st > c0 || kk > 0) ? 1u : 0u);
                        umma_commit(&empty[s]);
                        if (++s == STAGES) { s = 0; ph ^= 1; }
                    }
                    // chunk done (or aborted): the epilogue may read this accumulator
                    umma_commit(&tfull[acc]);
                    if (!ok) {
                        mbar_drain(&tfull[acc], acc_ph);  // every issued MMA done before TMEM is freed
                        break;
                    }
                    if (++acc == 2) { acc = 0; acc_ph ^= 1; }
                }
            }
        }
    } else {
        // ---------------------------------------------------------- epilogue
        auto arrive = [&](int a) { mbar_arrive(&tempty[a]); };
        if constexpr (SINGLE)
            epilogue_single<OUT, BN, EPI_COLS>(p, &mC, blockIdx.x, gridDim.x, ntiles, tiles_m, tiles_n, BM, 0,
                                                tmem_base, tfull, arrive, epi_buf, cbar, abort_flag);
        else
            epilogue_multi<OUT, BN, EPI_COLS>(p, &mC, blockIdx.x, gridDim.x, ntiles, tiles_m, tiles_n, BM, 0,
                                               tmem_base, tfull, arrive, epi_buf, cbar, abort_flag);
    }

    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicOr(p.status, (int)kDevWaitTimeout);
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, TC::TMEM_COLS);
    }
}

// ---------------------------------------------------------------- 2-SM variant
// The same GEMM on CTA pairs (cluster of 2, tcgen05 cta_group::2): the pair
// computes a 256 x 256 output tile; each CTA holds its own 128 rows of the A
// tile and one half (128 rows) of the B tile in shared memory, so B is
// fetched once per pair instead of once per CTA.  The even CTA (the leader)
// issues the MMAs (M = 256, N = 256), which read A and B from both CTAs'
// shared memory at the same offsets and accumulate each CTA's 128 rows into
// its own TMEM.  Both CTAs issue their own TMA loads (each into its own
// shared memory), completing on the leader's stage barrier, on which only the
// leader arrives (expecting both CTAs' bytes); the leader's MMA commits arrive
// on both CTAs' "stage free" and "accumulator ready" barriers; both CTAs'
// epilogue warps report a drained accumulator to the leader.
namespace two_sm {
constexpr int BN = 256;                     // pair tile columns; each CTA stores 128 rows of B
constexpr int B_HALF = 128 * ROW_BYTES;     // 16 KiB
constexpr int STAGE_BYTES = A_TILE + B_HALF;  // 32 KiB
constexpr int STAGES = RING_BYTES / STAGE_BYTES;  // 6

__device__ __forceinline__ uint32_t cta_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// shared::cluster address of the same variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t map_rank(const void* p, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}
__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void tma_load_2d_pair(void* smem_dst, const CUtensorMap* map, int x, int y,
                                                 uint32_t bar_cluster)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(smem_dst)), "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar_cluster)
        : "memory");
}
template <bool TF32>
__device__ __forceinline__ void umma_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    if (TF32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
    }
}
// arrive on the barrier at this offset in both CTAs of the pair when the
// leader's MMAs issued so far have completed (one commit per CTA's barrier)
__device__ __forceinline__ void commit_to(uint32_t bar_cluster)
{
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_cluster)
                 : "memory");
}
__device__ __forceinline__ void commit_both(uint64_t* bar)
{
    commit_to(map_rank(bar, 0));
    commit_to(map_rank(bar, 1));
}
__device__ __forceinline__ void arrive_remote(uint32_t bar_cluster)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}
__device__ __forceinline__ void alloc_pair(uint32_t* dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols));
}
__device__ __forceinline__ void relinquish_pair()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
}
__device__ __forceinline__ void dealloc_pair(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
}  // namespace two_sm

template <bool TF32, int OUT, bool SINGLE>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_tc2_kernel(const __grid_constant__ CUtensorMap mA0, const __grid_constant__ CUtensorMap mA1,
                    const __grid_constant__ CUtensorMap mA2, const __grid_constant__ CUtensorMap mB0,
                    const __grid_constant__ CUtensorMap mB1, const __grid_constant__ CUtensorMap mB2,
                    const __grid_constant__ CUtensorMap mC, Params p)
{
    using namespace two_sm;
    constexpr int EPI_COLS = BN / 2;  // columns per epilogue warp
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* tiles = smem;
    uint64_t* full = (uint64_t*)(smem + RING_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* tfull = empty + STAGES;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = (uint32_t*)(tempty + 2);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    uint64_t* cbar = (uint64_t*)(smem + RING_BYTES + 512);  // [half][buffer] C-load barriers
    uint8_t* epi_buf = smem + RING_BYTES + 1024;             // [half][buffer] staging

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint32_t rank = cta_rank();
    const bool leader = rank == 0;
    const int pair = blockIdx.x / 2, npairs = gridDim.x / 2;
    const int tiles_m = (p.M + 2 * BM - 1) / (2 * BM), tiles_n = (p.N + BN - 1) / BN;
    const int ntiles = tile_count(p.tri, tiles_m, tiles_n, 2 * BM, BN);
    const int steps = p.kblocks * p.nprod;
    constexpr bool MN_OK = OUT == OUT_F16;  // MN-major operands: HGEMM only

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);    // the leader's producer (bytes of both CTAs)
            mbar_init(&empty[s], 1);   // the leader's MMA commit
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], 2 * EPI_WARPS);  // every epilogue warp of both CTAs
        }
        for (int i = 0; i < 4; ++i) mbar_init(&cbar[i], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        alloc_pair(tmem_slot, 512);
        relinquish_pair();
    }
    tc_fence_before();
    cluster_sync();  // both CTAs' barriers and TMEM are set up
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ---------------------------------------------------------- TMA producer (both CTAs)
        if (lane == 0) {
            const CUtensorMap* ma[3] = {&mA0, &mA1, &mA2};
            const CUtensorMap* mb[3] = {&mB0, &mB1, &mB2};
            int s = 0;
            uint32_t ph = 0;
            bool ok = true;
            for (int t = pair; t < ntiles && ok; t += npairs) {
                int tm, tn;
                tile_at(p.tri, t, tiles_m, tiles_n, 2 * BM, BN, tm, tn);
                for (int st = 0; st < steps && ok; ++st) {
                    const int kb = st / p.nprod, pr = st % p.nprod;
                    if (!mbar_wait(&empty[s], ph ^ 1, abort_flag)) { ok = false; break; }
                    uint8_t* sa = tiles + s * STAGE_BYTES;
                    uint8_t* sb = sa + A_TILE;
                    if (leader) mbar_expect_tx(&full[s], 2 * STAGE_BYTES);
                    const uint32_t bar = map_rank(&full[s], 0);
                    const int kx = kb * (TF32 ? 32 : 64);
                    const int ra = tm * 2 * BM + (int)rank * BM, rb = tn * BN + (int)rank * 128;
                    if (MN_OK && p.a_mn) {
                        for (int i = 0; i < BM / 64; ++i)
                            tma_load_2d_pair(sa + i * MN_CHUNK_BYTES, ma[p.pa[pr]], ra + i * 64, kx, bar);
                    } else {
                        tma_load_2d_pair(sa, ma[p.pa[pr]], kx, ra, bar);
                    }
                    if (MN_OK && p.b_mn) {
                        for (int i = 0; i < 128 / 64; ++i)
                            tma_load_2d_pair(sb + i * MN_CHUNK_BYTES, mb[p.pb[pr]], rb + i * 64, kx, bar);
                    } else {
                        tma_load_2d_pair(sb, mb[p.pb[pr]], kx, rb, bar);
                    }
                    if (++s == STAGES) { s = 0; ph ^= 1; }
                }
            }
            if (!ok && leader) {
                // wait (bounded) for the copies in flight to this CTA's barriers, then leave
                for (int i = 0; i < STAGES; ++i) mbar_drain(&full[(s + i) % STAGES], ph);
            }
        }
    } else if (warp == 1) {
        // ---------------------------------------------------------- MMA issuer (leader only)
        if (lane == 0 && leader) {
            const uint32_t fmt = TF32 ? 2u : (uint32_t)p.ab_fmt;
            const int a_mn = MN_OK && p.a_mn, b_mn = MN_OK && p.b_mn;
            const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)a_mn << 15) |
                                   ((uint32_t)b_mn << 16) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)((2 * BM) >> 4) << 24);
            const uint64_t a_step = a_mn ? 128 : 2, b_step = b_mn ? 128 : 2;  // per MMA, 16-byte units
            int s = 0;
            uint32_t ph = 0;
            int acc = 0;
            uint32_t acc_ph = 0;
            bool ok = true;
            const int chunk_steps = p.chunk * p.nprod;
            for (int t = pair; t < ntiles && ok; t += npairs) {
                for (int c0 = 0; c0 < steps && ok; c0 += chunk_steps) {
                    if (!mbar_wait(&tempty[acc], acc_ph ^ 1, abort_flag)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t d = tmem_base + (uint32_t)(acc * BN);
                    const int c1 = min(steps, c0 + chunk_steps);
                    for (int st = c0; st < c1; ++st) {
                        if (!mbar_wait(&full[s], ph, abort_flag)) { ok = false; break; }
                        tc_fence_after();
                        const uint32_t sa = smem_u32(tiles + s * STAGE_BYTES);
                        const uint32_t sb = sa + A_TILE;
                        const uint64_t da = a_mn ? smem_desc_mn_sw128(sa) : smem_desc_sw128(sa);
                        const uint64_t db = b_mn ? smem_desc_mn_sw128(sb) : smem_desc_sw128(sb);
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk)
                            umma_pair<TF32>(d, da + a_step * kk, db + b_step * kk, idesc,
                                            (st > c0 || kk > 0) ? 1u : 0u);
                        commit_both(&empty[s]);
                        if (++s == STAGES) { s = 0; ph ^= 1; }
                    }
                    commit_both(&tfull[acc]);
                    if (!ok) {
                        mbar_drain(&tfull[acc], acc_ph);  // every issued MMA done
                        break;
                    }
                    if (++acc == 2) { acc = 0; acc_ph ^= 1; }
                }
            }
        }
    } else {
        // ---------------------------------------------------------- epilogue (both CTAs)
        const uint32_t tempty_leader[2] = {map_rank(&tempty[0], 0), map_rank(&tempty[1], 0)};
        auto arrive = [&](int a) { arrive_remote(tempty_leader[a]); };
        if constexpr (SINGLE)
            epilogue_single<OUT, BN, EPI_COLS>(p, &mC, pair, npairs, ntiles, tiles_m, tiles_n, 2 * BM,
                                                (int)rank * BM, tmem_base, tfull, arrive, epi_buf, cbar, abort_flag);
        else
            epilogue_multi<OUT, BN, EPI_COLS>(p, &mC, pair, npairs, ntiles, tiles_m, tiles_n, 2 * BM,
                                               (int)rank * BM, tmem_base, tfull, arrive, epi_buf, cbar, abort_flag);
    }

    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicOr(p.status, (int)kDevWaitTimeout);
    // the leader's MMAs write both CTAs' TMEM: free it only when both are done
    tc_fence_before();
    cluster_sync();
    tc_fence_after();
    if (warp == 1) dealloc_pair(tmem_base, 512);
}

// ---------------------------------------------------------------- split pre-pass
// Logical operand L (R x K): L[r][k] = S[r*rs + k*ks] (conj if requested).
// Output planes are K-major with row pitch kpad elements.
// Real:    plane[l][r*kpad + k]            (k >= K: zero)
// Complex A: plane[l][r*kpad + k] = re, [r*kpad + K + k] = im       (kpad >= 2K)
// Complex B: plane[l][(2r)*kpad + k] = re, [(2r)*kpad + K + k] = -im,
//            plane[l][(2r+1)*kpad + k] = im, [(2r+1)*kpad + K + k] = re
enum SplitMode { kReal = 0, kCplxA = 1, kCplxB = 2 };

__device__ __forceinline__ void split3(float x, __nv_bfloat16& hi, __nv_bfloat16& mid, __nv_bfloat16& lo)
{
    hi = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(hi);
    mid = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(mid);
    lo = __float2bfloat16_rn(r2);
}

__device__ __forceinline__ float to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

struct SplitOut {
    void* plane[3];
    int nlev;  // planes to write (TF32: 1 FP32 plane)
    int tf32;
    long kpad;
};

__device__ __forceinline__ void put(const SplitOut& o, long idx, float x)
{
    if (o.tf32) {
        ((float*)o.plane[0])[idx] = to_tf32(x);
        return;
    }
    __nv_bfloat16 h, m, l;
    split3(x, h, m, l);
    ((__nv_bfloat16*)o.plane[0])[idx] = h;
    if (o.nlev > 1) ((__nv_bfloat16*)o.plane[1])[idx] = m;
    if (o.nlev > 2) ((__nv_bfloat16*)o.plane[2])[idx] = l;
}

// Real operands: 32 rows x 64 K per block (256 threads).  Reads are coalesced
// along the source's contiguous dimension (through shared memory); each
// thread then writes two consecutive K values: one bfloat162 per plane, or a
// float2 for TF32 (128- or 256-byte rows per warp).  Row r goes to
// plane + r * o.kpad, K values [0, kw) (zeros for k >= K; kw even).
// `tri` masks L to a triangle (1: keep k <= r, 2: keep k >= r; `unit` puts 1
// on the diagonal); tiles wholly outside the kept triangle are left
// unwritten.  blockIdx.z selects one of several equal operands: source
// + z * szs, destination row offset + z * dzs.
__global__ void __launch_bounds__(256) split_real_kernel(int R, int K, const float* __restrict__ S, long rs, long ks,
                                                         SplitOut o, long kw, int tri, int unit, long szs, long dzs)
{
    __shared__ float tile[32][65];
    const int k0 = blockIdx.x * 64, r0 = blockIdx.y * 32, t = threadIdx.x;
    if ((tri == 1 && k0 > r0 + 31) || (tri == 2 && k0 + 63 < r0)) return;
    S += (long)blockIdx.z * szs;
    const long dz = (long)blockIdx.z * dzs;
    if (rs == 1) {  // contiguous along r
        for (int idx = t; idx < 32 * 64; idx += 256) {
            const int rr = idx % 32, kk = idx / 32;
            const int r = r0 + rr, k = k0 + kk;
            tile[rr][kk] = (r < R && k < K) ? S[(long)r + (long)k * ks] : 0.f;
        }
    } else {        // contiguous along k (ks == 1)
        for (int idx = t; idx < 32 * 64; idx += 256) {
            const int kk = idx % 64, rr = idx / 64;
            const int r = r0 + rr, k = k0 + kk;
            tile[rr][kk] = (r < R && k < K) ? S[(long)r * rs + k] : 0.f;
        }
    }
    __syncthreads();
    for (int idx = t; idx < 32 * 32; idx += 256) {
        const int kp = idx % 32, rr = idx / 32;
        const int r = r0 + rr, k = k0 + 2 * kp;
        if (r >= R || k >= kw) continue;
        float a = tile[rr][2 * kp], b = tile[rr][2 * kp + 1];
        if (tri) {
            const bool ka = tri == 1 ? k <= r : k >= r, kb = tri == 1 ? k + 1 <= r : k + 1 >= r;
            a = ka ? ((unit && k == r) ? 1.f : a) : 0.f;
            b = kb ? ((unit && k + 1 == r) ? 1.f : b) : 0.f;
        }
        const long off = ((long)r + dz) * o.kpad + k;  // even: 4- and 8-byte aligned pairs
        if (o.tf32) {
            *reinterpret_cast<float2*>((float*)o.plane[0] + off) = make_float2(to_tf32(a), to_tf32(b));
        } else {
            __nv_bfloat16 ha, ma, la, hb, mb, lb;
            split3(a, ha, ma, la);
            split3(b, hb, mb, lb);
            *reinterpret_cast<__nv_bfloat162*>((__nv_bfloat16*)o.plane[0] + off) = __halves2bfloat162(ha, hb);
            if (o.nlev > 1)
                *reinterpret_cast<__nv_bfloat162*>((__nv_bfloat16*)o.plane[1] + off) = __halves2bfloat162(ma, mb);
            if (o.nlev > 2)
                *reinterpret_cast<__nv_bfloat162*>((__nv_bfloat16*)o.plane[2] + off) = __halves2bfloat162(la, lb);
        }
    }
}

// IEEE half operands (HGEMM): the same 32 x 64 tiling, values copied into
// the K-major padded plane unchanged (zeros past K).
__global__ void __launch_bounds__(256) pack_half_kernel(int R, int K, const __half* __restrict__ S, long rs, long ks,
                                                        __half* __restrict__ plane, long kpad)
{
    __shared__ __half tile[32][66];
    const int k0 = blockIdx.x * 64, r0 = blockIdx.y * 32, t = threadIdx.x;
    const __half zero = __float2half_rn(0.f);
    if (rs == 1) {
        for (int idx = t; idx < 32 * 64; idx += 256) {
            const int rr = idx % 32, kk = idx / 32;
            const int r = r0 + rr, k = k0 + kk;
            tile[rr][kk] = (r < R && k < K) ? S[(long)r + (long)k * ks] : zero;
        }
    } else {
        for (int idx = t; idx < 32 * 64; idx += 256) {
            const int kk = idx % 64, rr = idx / 64;
            const int r = r0 + rr, k = k0 + kk;
            tile[rr][kk] = (r < R && k < K) ? S[(long)r * rs + k] : zero;
        }
    }
    __syncthreads();
    for (int idx = t; idx < 32 * 32; idx += 256) {
        const int kp = idx % 32, rr = idx / 32;
        const int r = r0 + rr, k = k0 + 2 * kp;
        if (r >= R || k >= kpad) continue;
        *reinterpret_cast<__half2*>(plane + (long)r * kpad + k) = __halves2half2(tile[rr][2 * kp], tile[rr][2 * kp + 1]);
    }
}

// Complex operands: 32 x 32 tile of L per block (blockDim 32 x 8), transposed
// through shared memory when the source is contiguous along r, so that both
// the reads of S and the K-contiguous writes are coalesced.
template <class T>
__global__ void __launch_bounds__(256) split_kernel(int R, int K, const T* __restrict__ S, long rs, long ks, int conj,
                                                    int mode, SplitOut o)
{
    __shared__ T tile[32][33];
    const int k0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    // load tile[rr][kk] = L[r0+rr][k0+kk]
    if (rs == 1) {  // contiguous along r
        for (int kk = ty; kk < 32; kk += 8) {
            const int r = r0 + tx, k = k0 + kk;
            T v{};
            if (r < R && k < K) v = S[(long)r + (long)k * ks];
            tile[tx][kk] = v;
        }
    } else {
        for (int rr = ty; rr < 32; rr += 8) {
            const int r = r0 + rr, k = k0 + tx;
            T v{};
            if (r < R && k < K) v = S[(long)r * rs + (long)k];
            tile[rr][tx] = v;
        }
    }
    __syncthreads();
    for (int rr = ty; rr < 32; rr += 8) {
        const int r = r0 + rr, k = k0 + tx;
        if (r >= R) continue;
        const T v = tile[rr][tx];
        if constexpr (sizeof(T) == sizeof(float)) {
            // real: K is padded to a multiple of the block by the grid; k >= K writes zeros
            if (k < o.kpad) put(o, (long)r * o.kpad + k, k < K ? (float)*(const float*)&v : 0.f);
        } else {
            const float re = ((const float*)&v)[0];
            const float im = (conj ? -1.f : 1.f) * ((const float*)&v)[1];
            if (k >= K) continue;
            if (mode == kCplxA) {
                put(o, (long)r * o.kpad + k, re);
                put(o, (long)r * o.kpad + K + k, im);
            } else {
                put(o, (long)(2 * r) * o.kpad + k, re);
                put(o, (long)(2 * r) * o.kpad + K + k, -im);
                put(o, (long)(2 * r + 1) * o.kpad + k, im);
                put(o, (long)(2 * r + 1) * o.kpad + K + k, re);
            }
        }
    }
}

// zero the K padding columns [kfrom, kpad) of every row (complex layouts)
__global__ void zero_pad_kernel(long rows, long kfrom, SplitOut o)
{
    const long w = o.kpad - kfrom;
    const long total = rows * w;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long r = e / w, k = kfrom + e % w;
        const long idx = r * o.kpad + k;
        if (o.tf32) ((float*)o.plane[0])[idx] = 0.f;
        else
            for (int l = 0; l < o.nlev; ++l) ((__nv_bfloat16*)o.plane[l])[idx] = __float2bfloat16_rn(0.f);
    }
}

// ---------------------------------------------------------------- host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

// One operand as the engine reads it: a prepared K-major plane, or the
// caller's own 16-bit array in either layout.
struct Operand {
    const void* base;
    long rows;  // M (A) or N (B)
    long kext;  // K extent; the copies zero-fill past it
    long ld;    // elements between consecutive rows (K-major) or consecutive K indices (MN-major)
    bool mn;    // MN-major: the rows are contiguous
};

bool make_operand_map(CUtensorMap* m, const Operand& o, bool tf32, int box_rows)
{
    EncodeTiledFn f = encode_fn();
    if (!f) return false;
    const int esize = tf32 ? 4 : 2;
    const cuuint32_t kbox = ROW_BYTES / esize;
    cuuint64_t dims[2] = {(cuuint64_t)o.kext, (cuuint64_t)o.rows};
    cuuint32_t box[2] = {kbox, (cuuint32_t)box_rows};
    if (o.mn) {  // boxes of 64 rows x 64 K (16-bit operands only)
        if (tf32) return false;
        dims[0] = (cuuint64_t)o.rows;
        dims[1] = (cuuint64_t)o.kext;
        box[1] = kbox;
    }
    cuuint64_t strides[1] = {(cuuint64_t)(o.ld * esize)};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = f(m, tf32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                   const_cast<void*>(o.base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// C as boxes of 128 rows x 16 columns (complex: 8 columns of (re, im)
// pairs), unswizzled, for the staged epilogue.  False when C cannot be
// addressed that way (alignment, triangular output).
bool make_c_map(CUtensorMap* m, Params& p)
{
    EncodeTiledFn f = encode_fn();
    if (!f || p.tri != 0 || !p.C || p.M <= 0 || p.N <= 0 || ((uintptr_t)p.C & 15) != 0) return false;
    const int esize = p.out_half ? 2 : (p.complex_out ? 8 : 4);
    const long pitch = p.ldc * esize;
    if (pitch % 16 != 0 || pitch >= (1L << 40)) return false;
    // a store clips rows only at 16-byte granularity: the map stops at the
    // last whole 16 bytes of each column, the rest are stored directly
    p.m_tma = p.M - p.M % (16 / esize);
    if (p.m_tma == 0) return false;
    cuuint64_t dims[2] = {(cuuint64_t)p.m_tma, (cuuint64_t)p.N};
    cuuint32_t box[2] = {128, (cuuint32_t)(p.out_half ? 32 : EPI_GROUP)};
    if (p.complex_out) {
        dims[0] = 2 * (cuuint64_t)p.m_tma;
        dims[1] = (cuuint64_t)(p.N / 2);
        box[0] = 256;
        box[1] = EPI_GROUP / 2;
    }
    cuuint64_t strides[1] = {(cuuint64_t)pitch};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = f(m, p.out_half ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)p.C,
                   dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

struct ModeInfo {
    bool tf32;
    int nlev;
    int nprod;
    int pa[6], pb[6];
};

ModeInfo mode_info(iclblasMathMode_t mode)
{
    ModeInfo mi{};
    if (mode == ICLBLAS_MATH_TF32) {
        mi.tf32 = true;
        mi.nlev = 1;
        mi.nprod = 1;
        mi.pa[0] = mi.pb[0] = 0;
    } else if (mode == ICLBLAS_MATH_BF16X3) {
        mi.nlev = 2;
        mi.nprod = 3;  // mid*hi, hi*mid, hi*hi: smallest first (levels: 0 hi, 1 mid)
        const int a[3] = {1, 0, 0}, b[3] = {0, 1, 0};
        for (int i = 0; i < 3; ++i) { mi.pa[i] = a[i]; mi.pb[i] = b[i]; }
    } else {
        mi.nlev = 3;
        mi.nprod = 6;  // lo*hi, hi*lo, mid*mid, mid*hi, hi*mid, hi*hi: smallest first
        const int a[6] = {2, 0, 1, 1, 0, 0}, b[6] = {0, 2, 1, 0, 1, 0};
        for (int i = 0; i < 6; ++i) { mi.pa[i] = a[i]; mi.pb[i] = b[i]; }
    }
    return mi;
}

// The mode's share of the kernel parameters for a K extent of kext elements:
// K blocks, products per block (in the small-first order) and TMEM chunking.
// 6xBF16 drains the accumulator every K block (its FP32-level accuracy
// needs it: 2 blocks per chunk measured 5.9e-7 instead of 2.2e-7 at
// 8192^3); 3xBF16 every 4 blocks (its dropped products dominate: 3.84e-6
// instead of 3.78e-6, 9 % faster); TF32 accumulates the whole K in TMEM.
void set_mode_params(Params& p, const ModeInfo& mi, long kext)
{
    const int kblk = ROW_BYTES / (mi.tf32 ? 4 : 2);
    p.kblocks = (int)((kext + kblk - 1) / kblk);
    p.nprod = mi.nprod;
    p.chunk = mi.tf32 ? p.kblocks : (mi.nprod == 3 ? 4 : 1);
    for (int i = 0; i < 6; ++i) {
        p.pa[i] = mi.pa[i];
        p.pb[i] = mi.pb[i];
    }
}

template <class T>
cudaError_t run_split(iclblasHandle_t h, const T* S, int R, int K, long rs, long ks, int conj, int mode,
                      const SplitOut& o, long out_rows)
{
    if (std::is_same<T, float>::value) {
        dim3 grid((unsigned)ceil_div(o.kpad, 64L), (unsigned)ceil_div(R, 32));
        split_real_kernel<<<grid, 256, 0, h->stream>>>(R, K, (const float*)S, rs, ks, o, o.kpad, 0, 0, 0, 0);
        return cudaGetLastError();
    }
    dim3 grid(ceil_div(K, 32), ceil_div(R, 32));
    split_kernel<T><<<grid, dim3(32, 8), 0, h->stream>>>(R, K, S, rs, ks, conj, mode, o);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (!std::is_same<T, float>::value && o.kpad > 2L * K) {
        const long total = out_rows * (o.kpad - 2L * K);
        const int g = (int)std::min<long>((total + 255) / 256, (long)h->sm_count * 8);
        zero_pad_kernel<<<g, 256, 0, h->stream>>>(out_rows, 2L * K, o);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace

// Launch facts that are fixed per kernel and device, found once: the
// dynamic shared-memory opt-in is set, and (CTA-pair kernels) the number of
// clusters that fit at once is queried (0 for single-CTA kernels).
struct KernelFacts {
    cudaError_t status;
    int max_clusters;
};

template <class K>
KernelFacts kernel_facts(K kernel, int smem, bool pairs, iclblasHandle_t h)
{
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, KernelFacts> known;
    const std::pair<const void*, int> key((const void*)kernel, h->device);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = known.find(key);
        if (it != known.end()) return it->second;
    }
    // the attribute and the occupancy query apply to the current device
    DeviceGuard guard(h->device);
    if (guard.status() != cudaSuccess) return KernelFacts{guard.status(), 0};
    KernelFacts f{cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), 0};
    if (f.status == cudaSuccess && pairs) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.blockDim = dim3(THREADS);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = h->stream;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cfg.gridDim = dim3(2 * std::max(1, h->sm_count / 2));
        if (cudaOccupancyMaxActiveClusters(&f.max_clusters, kernel, &cfg) != cudaSuccess || f.max_clusters < 1) {
            cudaGetLastError();
            f.max_clusters = std::max(1, h->sm_count / 2);
        }
    }
    if (f.status == cudaSuccess) {
        std::lock_guard<std::mutex> lock(mu);
        known[key] = f;
    }
    return f;
}

// Launches the persistent tcgen05 kernel over the operands (one per split
// level): CTA pairs (256 x 256 tiles) when there are enough pair tiles to
// fill the GPU; else single CTAs, with 128-wide tiles when 256-wide ones
// would leave a quarter of the SMs idle.
cudaError_t launch_engine(iclblasHandle_t h, const ModeInfo& mi, const Operand* a, const Operand* b, Params& p)
{
    const long rows_a = a[0].rows, rows_b = b[0].rows;
    const int m = (int)rows_a;
    const int pair_tiles = ceil_div(m, 2 * BM) * ceil_div((long)rows_b, 256);
    const bool pairs = pair_tiles * 2 >= h->sm_count;
    const int tiles256 = ceil_div(m, BM) * ceil_div((long)rows_b, 256);
    const int bn = pairs ? 128 : (tiles256 * 4 < h->sm_count * 3 ? 128 : 256);  // B box rows
    CUtensorMap ma[3], mb[3], mc;
    for (int l = 0; l < 3; ++l) {
        const int ll = l < mi.nlev ? l : 0;
        if (!make_operand_map(&ma[l], a[ll], mi.tf32, BM)) return cudaErrorInvalidValue;
        if (!make_operand_map(&mb[l], b[ll], mi.tf32, bn)) return cudaErrorInvalidValue;
    }
    p.a_mn = a[0].mn ? 1 : 0;
    p.b_mn = b[0].mn ? 1 : 0;
    // single-chunk kernels hold the whole K in one accumulator (TF32, HGEMM,
    // and the BF16 modes when K fits one chunk); both forms store C through
    // TMA boxes whenever C allows it
    const bool single = mi.tf32 || p.out_half || p.kblocks <= p.chunk;
    p.c_tma = make_c_map(&mc, p) ? 1 : 0;
    const int smem = SMEM_BYTES;
    if (!p.c_tma) mc = ma[0];  // unused by the kernel
    if (pairs) {
        auto run2 = [&](auto kernel) -> cudaError_t {
            const KernelFacts f = kernel_facts(kernel, smem, true, h);
            if (f.status != cudaSuccess) return f.status;
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = 2;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.blockDim = dim3(THREADS);
            cfg.dynamicSmemBytes = smem;
            cfg.stream = h->stream;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            // as many pairs as can be resident at once (persistent), at most one per tile
            cfg.gridDim = dim3(2 * std::min(pair_tiles, f.max_clusters));
            const cudaError_t r = cudaLaunchKernelEx(&cfg, kernel, ma[0], ma[1], ma[2], mb[0], mb[1], mb[2], mc, p);
            if (r != cudaSuccess) return r;
            return cudaGetLastError();
        };
        if (p.out_half) return run2(gemm_tc2_kernel<false, OUT_F16, true>);
        if (mi.tf32)
            return p.complex_out ? run2(gemm_tc2_kernel<true, OUT_C64, true>) : run2(gemm_tc2_kernel<true, OUT_F32, true>);
        if (p.complex_out)
            return single ? run2(gemm_tc2_kernel<false, OUT_C64, true>) : run2(gemm_tc2_kernel<false, OUT_C64, false>);
        return single ? run2(gemm_tc2_kernel<false, OUT_F32, true>) : run2(gemm_tc2_kernel<false, OUT_F32, false>);
    }
    const int tiles = ceil_div(m, BM) * ceil_div((long)rows_b, bn);
    const int grid = std::min(tiles, h->sm_count);
    auto run = [&](auto kernel) -> cudaError_t {
        const KernelFacts f = kernel_facts(kernel, smem, false, h);
        if (f.status != cudaSuccess) return f.status;
        kernel<<<grid, THREADS, smem, h->stream>>>(ma[0], ma[1], ma[2], mb[0], mb[1], mb[2], mc, p);
        return cudaGetLastError();
    };
    // instantiations: TF32 and HGEMM always single-chunk; the BF16 modes
    // single-chunk when the whole K fits one chunk (K <= 64 * chunk)
    auto pick = [&](auto k128, auto k256) { return bn == 128 ? run(k128) : run(k256); };
    if (p.out_half) return pick(gemm_tc_kernel<false, 128, OUT_F16, true>, gemm_tc_kernel<false, 256, OUT_F16, true>);
    if (mi.tf32) {
        if (p.complex_out) return pick(gemm_tc_kernel<true, 128, OUT_C64, true>, gemm_tc_kernel<true, 256, OUT_C64, true>);
        return pick(gemm_tc_kernel<true, 128, OUT_F32, true>, gemm_tc_kernel<true, 256, OUT_F32, true>);
    }
    if (p.complex_out) {
        if (single) return pick(gemm_tc_kernel<false, 128, OUT_C64, true>, gemm_tc_kernel<false, 256, OUT_C64, true>);
        return pick(gemm_tc_kernel<false, 128, OUT_C64, false>, gemm_tc_kernel<false, 256, OUT_C64, false>);
    }
    if (single) return pick(gemm_tc_kernel<false, 128, OUT_F32, true>, gemm_tc_kernel<false, 256, OUT_F32, true>);
    return pick(gemm_tc_kernel<false, 128, OUT_F32, false>, gemm_tc_kernel<false, 256, OUT_F32, false>);
}

// Real or complex GEMM on the tensor cores.  `cplx` selects complex operands
// (T = cfloat); the real GEMM then has M rows, 2N columns and 2K depth.
template <class T>
cudaError_t gemm_tc(iclblasHandle_t h, int ta, int tb, int m, int n, int k, T alpha, const T* A, int lda,
                    const T* B, int ldb, T beta, T* C, int ldc, int tri)
{
    constexpr bool cplx = sizeof(T) == sizeof(cfloat);
    const ModeInfo mi = mode_info(h->math);
    const int esize = mi.tf32 ? 4 : 2;
    const int kblk = ROW_BYTES / esize;
    const long kreal = cplx ? 2L * k : (long)k;
    const long kpad = (kreal + kblk - 1) / kblk * kblk;
    const long rows_a = m, rows_b = cplx ? 2L * n : (long)n;
    const size_t plane_a = (size_t)rows_a * kpad * esize, plane_b = (size_t)rows_b * kpad * esize;
    const size_t align = 1024;
    const size_t pa_al = (plane_a + align - 1) / align * align, pb_al = (plane_b + align - 1) / align * align;
    char* ws = (char*)scratch(h, (pa_al + pb_al) * mi.nlev);
    if (!ws) return cudaErrorMemoryAllocation;
    SplitOut oa{}, ob{};
    oa.nlev = ob.nlev = mi.nlev;
    oa.tf32 = ob.tf32 = mi.tf32 ? 1 : 0;
    oa.kpad = ob.kpad = kpad;
    for (int l = 0; l < mi.nlev; ++l) {
        oa.plane[l] = ws + l * pa_al;
        ob.plane[l] = ws + mi.nlev * pa_al + l * pb_al;
    }
    // A: L[r=m][k] ; op N: S[m + k*lda] ; op T/C: S[k + m*lda]
    const bool at = ta != ICLBLAS_OP_N, bt = tb != ICLBLAS_OP_N;
    cudaError_t e = run_split<T>(h, A, m, k, at ? lda : 1, at ? 1 : lda, ta == ICLBLAS_OP_C, kCplxA, oa, rows_a);
    if (e != cudaSuccess) return e;
    // B: L[r=n][k] = op(B)[k][n] ; op N: S[k + n*ldb] ; op T/C: S[n + k*ldb]
    e = run_split<T>(h, B, n, k, bt ? 1 : ldb, bt ? ldb : 1, tb == ICLBLAS_OP_C, kCplxB, ob, rows_b);
    if (e != cudaSuccess) return e;

    Params p{};
    p.M = m;
    p.N = (int)rows_b;
    set_mode_params(p, mi, kpad);
    p.complex_out = cplx ? 1 : 0;
    const float* al = (const float*)&alpha;
    const float* be = (const float*)&beta;
    p.alpha_re = al[0];
    p.alpha_im = cplx ? al[1] : 0.f;
    p.beta_re = be[0];
    p.beta_im = cplx ? be[1] : 0.f;
    p.C = (float*)C;
    p.ldc = ldc;
    p.status = h->ws.dev_status;
    p.tri = cplx ? 0 : tri;
    p.ab_fmt = 1;
    p.out_half = 0;
    Operand pa[3], pb[3];
    for (int l = 0; l < 3; ++l) {
        pa[l] = Operand{oa.plane[l], rows_a, kpad, kpad, false};
        pb[l] = Operand{ob.plane[l], rows_b, kpad, kpad, false};
    }
    return launch_engine(h, mi, pa, pb, p);
}

// HGEMM: IEEE half operands and result, products on the tensor cores with
// the f16 operand format, the whole K accumulated in FP32 in TMEM, one
// rounding of alpha * acc + beta * C to half.  The tensor core reads either
// operand layout, so each operand is read in place (A: MN-major for op N,
// K-major for op T / C; B the other way round) when TMA can address it
// (16-byte aligned base and leading dimension); otherwise it is first
// packed K-major into scratch.
cudaError_t hgemm_tc(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const __half* A, int lda,
                     const __half* B, int ldb, float beta, __half* C, int ldc)
{
    const int kblk = ROW_BYTES / 2;
    const long kpad = std::max<long>(kblk, ((long)k + kblk - 1) / kblk * kblk);
    const bool at = ta != ICLBLAS_OP_N, bt = tb != ICLBLAS_OP_N;
    auto in_place = [&](const __half* X, int ld) { return k > 0 && ((uintptr_t)X & 15) == 0 && ld % 8 == 0; };
    const bool a_direct = in_place(A, lda), b_direct = in_place(B, ldb);
    Operand oa{A, m, k, lda, !at}, ob{B, n, k, ldb, bt};
    if (!a_direct || !b_direct) {
        const size_t align = 1024;
        const size_t plane_a = a_direct ? 0 : ((size_t)m * kpad * 2 + align - 1) / align * align;
        const size_t plane_b = b_direct ? 0 : ((size_t)n * kpad * 2 + align - 1) / align * align;
        char* ws = (char*)scratch(h, plane_a + plane_b);
        if (!ws) return cudaErrorMemoryAllocation;
        if (!a_direct) {
            __half* la = (__half*)ws;
            // A: L[r=m][k] ; op N: S[m + k*lda] ; op T/C: S[k + m*lda]
            pack_half_kernel<<<dim3((unsigned)ceil_div(kpad, 64L), (unsigned)ceil_div(m, 32)), 256, 0, h->stream>>>(
                m, k, A, at ? lda : 1, at ? 1 : lda, la, kpad);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
            oa = Operand{la, m, kpad, kpad, false};
        }
        if (!b_direct) {
            __half* lb = (__half*)(ws + plane_a);
            // B: L[r=n][k] = op(B)[k][n] ; op N: S[k + n*ldb] ; op T/C: S[n + k*ldb]
            pack_half_kernel<<<dim3((unsigned)ceil_div(kpad, 64L), (unsigned)ceil_div(n, 32)), 256, 0, h->stream>>>(
                n, k, B, bt ? 1 : ldb, bt ? ldb : 1, lb, kpad);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
            ob = Operand{lb, n, kpad, kpad, false};
        }
    }
    ModeInfo mi{};
    mi.tf32 = false;
    mi.nlev = 1;
    mi.nprod = 1;
    Params p{};
    p.M = m;
    p.N = n;
    p.kblocks = (int)(kpad / kblk);
    p.nprod = 1;
    p.chunk = p.kblocks;
    p.complex_out = 0;
    p.alpha_re = alpha;
    p.beta_re = beta;
    p.C = (float*)C;
    p.ldc = ldc;
    p.status = h->ws.dev_status;
    p.tri = 0;
    p.ab_fmt = 0;
    p.out_half = 1;
    const Operand pa[3] = {oa, oa, oa}, pb[3] = {ob, ob, ob};
    return launch_engine(h, mi, pa, pb, p);
}

// Products of pre-split operands (declared in internal.h): the engine over
// sub-boxes of plane sets split once by the caller.
cudaError_t gemm_planes_tc(iclblasHandle_t h, const GemmPlanes& a, long ar0, long ak0, const GemmPlanes& b, long br0,
                           long bk0, int m, int n, int k, float alpha, float beta, float* C, int ldc)
{
    const ModeInfo mi = mode_info(h->math);
    if (h->math == ICLBLAS_MATH_PLAIN_FP32 || k <= 0 || a.tf32 != (mi.tf32 ? 1 : 0) ||
        b.tf32 != (mi.tf32 ? 1 : 0) || a.nlev < mi.nlev || b.nlev < mi.nlev)
        return cudaErrorInvalidValue;
    // the tensor maps cover exactly the sub-boxes: keep them inside the planes
    if (ar0 < 0 || ak0 < 0 || br0 < 0 || bk0 < 0 || ar0 + m > a.rows || br0 + n > b.rows || ak0 + k > a.pitch ||
        bk0 + k > b.pitch || (ak0 & 7) || (bk0 & 7))
        return cudaErrorInvalidValue;
    const long esize = mi.tf32 ? 4 : 2;
    Params p{};
    p.M = m;
    p.N = n;
    set_mode_params(p, mi, k);
    p.alpha_re = alpha;
    p.beta_re = beta;
    p.C = C;
    p.ldc = ldc;
    p.status = h->ws.dev_status;
    p.ab_fmt = 1;
    Operand oa[3], ob[3];
    for (int l = 0; l < 3; ++l) {
        const int la = l < a.nlev ? l : 0, lb = l < b.nlev ? l : 0;
        oa[l] = Operand{(const char*)a.plane[la] + (ar0 * a.pitch + ak0) * esize, m, k, a.pitch, false};
        ob[l] = Operand{(const char*)b.plane[lb] + (br0 * b.pitch + bk0) * esize, n, k, b.pitch, false};
    }
    return launch_engine(h, mi, oa, ob, p);
}

cudaError_t split_planes_tc(iclblasHandle_t h, const float* S, int R, int K, long rs, long ks, const GemmPlanes& dst,
                            long row0, long k0, long kw, int tri, int unit, int nz, long szs, long dzs)
{
    if (R <= 0 || kw <= 0 || nz <= 0) return cudaSuccess;
    if ((kw & 1) || (k0 & 1) || nz > 65535 || row0 < 0 || k0 < 0 || k0 + kw > dst.pitch ||
        row0 + (long)(nz - 1) * dzs + R > dst.rows)
        return cudaErrorInvalidValue;
    const long esize = dst.tf32 ? 4 : 2;
    SplitOut o{};
    o.nlev = dst.nlev;
    o.tf32 = dst.tf32;
    o.kpad = dst.pitch;
    for (int l = 0; l < dst.nlev; ++l) o.plane[l] = (char*)dst.plane[l] + (row0 * dst.pitch + k0) * esize;
    dim3 grid((unsigned)ceil_div(kw, 64L), (unsigned)ceil_div(R, 32), (unsigned)nz);
    split_real_kernel<<<grid, 256, 0, h->stream>>>(R, K, S, rs, ks, o, kw, tri, unit, szs, dzs);
    return cudaGetLastError();
}

template cudaError_t gemm_tc<float>(iclblasHandle_t, int, int, int, int, int, float, const float*, int, const float*,
                                    int, float, float*, int, int);
template cudaError_t gemm_tc<cfloat>(iclblasHandle_t, int, int, int, int, int, cfloat, const cfloat*, int,
                                     const cfloat*, int, cfloat, cfloat*, int, int);

}  // namespace tc

int plane_esize(iclblasMathMode_t mode) { return mode == ICLBLAS_MATH_TF32 ? 4 : 2; }
int plane_levels(iclblasMathMode_t mode) { return tc::mode_info(mode).nlev; }

cudaError_t split_planes(iclblasHandle_t h, const float* S, int R, int K, long rs, long ks, const GemmPlanes& dst,
                         long row0, long k0, long kw, int tri, int unit, int nz, long szs, long dzs)
{
    return tc::split_planes_tc(h, S, R, K, rs, ks, dst, row0, k0, kw, tri, unit, nz, szs, dzs);
}

cudaError_t gemm_planes(iclblasHandle_t h, const GemmPlanes& a, long ar0, long ak0, const GemmPlanes& b, long br0,
                        long bk0, int m, int n, int k, float alpha, float beta, float* C, int ldc)
{
    if (m <= 0 || n <= 0) return cudaSuccess;
    return tc::gemm_planes_tc(h, a, ar0, ak0, b, br0, bk0, m, n, k, alpha, beta, C, ldc);
}
}  // namespace iclb
