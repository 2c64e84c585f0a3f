// Internal declarations of the B200 iclBLAS library: the handle, device
// workspace management, error plumbing and the kernel launchers that the
// C-ABI layer (api.cu) dispatches to.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "../../include/iclBLAS.h"

namespace iclb {

// Complex single as two packed floats; layout-identical to oclComplex_t.
struct cfloat {
    float re, im;
};

constexpr uint32_t kHandleTag = 0xB1A5B200u;

// Device-side status word bits (written by kernels, read by the host).
enum DeviceStatus : int {
    kDevOk = 0,
    kDevWaitTimeout = 1,   // a bounded spin-wait ran out
};

// Per-handle device workspace.  Grows on demand; never shrinks until the
// handle is destroyed.  `counters` is a small zero-initialised area for
// last-block-done tickets and flags; kernels that use a counter leave it at
// zero (or, for epoch flags, monotonically increasing) when they finish.
struct Workspace {
    void* scratch = nullptr;   // general scratch (partials, GEMM operand planes)
    size_t scratch_bytes = 0;
    void* solver = nullptr;    // solver workspace (TRSM diagonal inverses), kept
    size_t solver_bytes = 0;   // apart so the GEMMs inside a solve can grow `scratch`
    unsigned* counters = nullptr;   // kCounterWords words, zeroed at creation
    int* dev_status = nullptr;      // one int, DeviceStatus bits
    unsigned epoch = 0;             // host-side epoch for flag-based kernels
    unsigned long long* pub = nullptr;   // TRSV: published solution entries (value, epoch), zeroed when grown
    size_t pub_elems = 0;
};
constexpr int kCounterWords = 1 << 16;

// ---------------------------------------------------------------- adjoints
cudaError_t strsm_backward(iclblasHandle_t h, int side, int uplo, int trans, int diag, int m, int n, float alpha,
                           const float* A, int lda, const float* X, int ldx, float* G, int ldg, float* dA, int ldda);
cudaError_t sgemm_backward(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const float* A, int lda,
                           const float* B, int ldb, float beta, const float* G, int ldg, float* dA, int ldda,
                           float* dB, int lddb, float* dC, int lddc);

// ---------------------------------------------------------------- pre-split GEMM operands
// Real operands of the tensor-core modes held as split planes, for products
// whose operands are reused (TRSM splits its triangle once per call and
// each solved block once).  A plane set stores rows of K values contiguously
// (K-major), `pitch` elements per row (a multiple of 64 elements for BF16,
// 32 for TF32), in `nlev` planes: BF16 hi, mid, lo (3xBF16 reads two, 6xBF16
// three) or one TF32-rounded FP32 plane.
struct GemmPlanes {
    void* plane[3] = {nullptr, nullptr, nullptr};
    int nlev = 0;
    int tf32 = 0;
    long pitch = 0;
    long rows = 0;   // rows each plane holds: every access stays below rows x pitch
};
// Element size and levels of the planes of `mode` (a tensor-core mode).
int plane_esize(iclblasMathMode_t mode);
int plane_levels(iclblasMathMode_t mode);
// Splits the real operand L[r][k] = S[r*rs + k*ks] (r < R, k < K) into rows
// row0.. of `dst`, K values [k0, k0 + kw) (zeros past K; kw even, k0 even).
// tri: 1 keeps k <= r, 2 keeps k >= r (unit: 1 on the diagonal); blocks
// wholly outside the triangle are not written.  nz operands at source
// stride szs and destination row stride dzs are split in one launch.  A
// write range outside dst (rows x pitch) returns cudaErrorInvalidValue
// before any launch.
cudaError_t split_planes(iclblasHandle_t h, const float* S, int R, int K, long rs, long ks, const GemmPlanes& dst,
                         long row0, long k0, long kw, int tri = 0, int unit = 0, int nz = 1, long szs = 0,
                         long dzs = 0);
// C (m x n, column-major) = alpha * A' B'^T + beta * C in the handle's math
// mode, A' = rows [ar0, ar0 + m) x K [ak0, ak0 + k) of planes a and B' =
// rows [br0, br0 + n) x the same K range [bk0, bk0 + k) of planes b.  K
// offsets and the row pitch keep every sub-box 16-byte aligned when ak0 and
// bk0 are multiples of 8.  A sub-box outside its plane set (rows x pitch)
// returns cudaErrorInvalidValue before any launch.
cudaError_t gemm_planes(iclblasHandle_t h, const GemmPlanes& a, long ar0, long ak0, const GemmPlanes& b, long br0,
                        long bk0, int m, int n, int k, float alpha, float beta, float* C, int ldc);

}  // namespace iclb

struct iclblasContext {
    uint32_t tag = 0;
    int device = 0;
    int sm_count = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    iclblasMathMode_t math = ICLBLAS_MATH_PLAIN_FP32;
    int trsm_refine = 0;   // TRSM residual-refinement steps (0..2)
    iclb::Workspace ws;
    // Device staging for host-pointer arguments (grows on demand).
    void* stage = nullptr;
    size_t stage_bytes = 0;
    // Pinned host bounce buffer for reduction results.
    void* pinned = nullptr;
    // Second stream and per-chunk events for pipelined host-operand calls
    // (created on first use).
    cudaStream_t aux_stream = nullptr;
    static constexpr int kMaxChunks = 32;
    cudaEvent_t chunk_ev[kMaxChunks] = {};
    // Fork / join of work on the second stream within one call (created on
    // first use).
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    // Two pinned bounce buffers for copies of pageable host memory, each with
    // the event of the last copy that used it (allocated on first use).
    void* bounce[2] = {nullptr, nullptr};
    cudaEvent_t bounce_ev[2] = {nullptr, nullptr};
    bool bounce_busy[2] = {false, false};
};

namespace iclb {

// Makes `device` current for a scope and restores the previous device.
class DeviceGuard {
public:
    explicit DeviceGuard(int device)
    {
        status_ = cudaGetDevice(&prev_);
        if (status_ == cudaSuccess && prev_ != device) {
            status_ = cudaSetDevice(device);
            switched_ = status_ == cudaSuccess;
        }
    }
    ~DeviceGuard()
    {
        if (switched_) cudaSetDevice(prev_);
    }
    cudaError_t status() const { return status_; }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;

private:
    int prev_ = 0;
    bool switched_ = false;
    cudaError_t status_ = cudaSuccess;
};

// Work of one call on two streams: fork() makes the handle's second stream
// wait for everything issued so far on the handle's stream; join() makes the
// handle's stream wait for everything issued so far on the second stream.
// Both streams and the events are created on first use.
cudaError_t fork_side(iclblasHandle_t h, cudaStream_t* side);
cudaError_t join_side(iclblasHandle_t h);
// Issues the launches of a scope on another stream (restored at scope exit).
class StreamScope {
public:
    StreamScope(iclblasHandle_t h, cudaStream_t s);
    ~StreamScope();
    StreamScope(const StreamScope&) = delete;
    StreamScope& operator=(const StreamScope&) = delete;

private:
    iclblasHandle_t h_;
    cudaStream_t saved_;
};

// Copies between pageable host memory and the device through the handle's
// pinned bounce buffers (host_copy.cu), on the handle's stream: h2d returns
// once every chunk has been handed to the DMA engine (later work on the
// stream sees the data), d2h once the data is in host memory.
cudaError_t copy_pageable_h2d(iclblasHandle_t h, void* dst_dev, const void* src_host, size_t bytes);
cudaError_t copy_pageable_d2h(iclblasHandle_t h, void* dst_host, const void* src_dev, size_t bytes);
cudaError_t free_bounce(iclblasHandle_t h);
// memcpy between host buffers on the process-wide pool of copy threads.
void host_copy(void* dst, const void* src, size_t bytes);

// Returns scratch of at least `bytes` (256-byte aligned) or nullptr.
void* scratch(iclblasHandle_t h, size_t bytes);
// Same for the solver workspace.
void* solver_scratch(iclblasHandle_t h, size_t bytes);

// ---------------------------------------------------------------- level 1
// All pointers are device pointers; n > 0, inc > 0.  Reduction results are
// written to device memory `result` in stream order.
cudaError_t saxpy(iclblasHandle_t h, int n, float alpha, const float* x, int incx, float* y, int incy);
cudaError_t sscal(iclblasHandle_t h, int n, float alpha, float* x, int incx);
cudaError_t caxpy(iclblasHandle_t h, int n, cfloat alpha, const cfloat* x, int incx, cfloat* y, int incy);
cudaError_t cscal(iclblasHandle_t h, int n, cfloat alpha, cfloat* x, int incx);

enum class Red { Dot, Asum, Nrm2 };
cudaError_t sreduce(iclblasHandle_t h, Red op, int n, const float* x, int incx, const float* y, int incy,
                    float* result);
cudaError_t creduce_real(iclblasHandle_t h, Red op, int n, const cfloat* x, int incx, float* result);
cudaError_t cdot(iclblasHandle_t h, bool conj, int n, const cfloat* x, int incx, const cfloat* y, int incy,
                 cfloat* result);
cudaError_t isamax(iclblasHandle_t h, int n, const float* x, int incx, int* result);
// SDOT whose scratch is a fixed array in the library image (no allocation);
// device pointers only.  cudaErrorNotSupported when the launch would need
// more than kSdotNoAllocMaxBlocks per-block partials.
constexpr int kSdotNoAllocMaxBlocks = 4096;
cudaError_t sdot_noalloc(iclblasHandle_t h, int n, const float* x, int incx, const float* y, int incy,
                         float* result);
cudaError_t icamax(iclblasHandle_t h, int n, const cfloat* x, int incx, int* result);
cudaError_t isamin(iclblasHandle_t h, int n, const float* x, int incx, int* result);
cudaError_t icamin(iclblasHandle_t h, int n, const cfloat* x, int incx, int* result);

// copy, swap, plane rotations and their generators (level1_rot.cu)
cudaError_t scopy(iclblasHandle_t h, int n, const float* x, int incx, float* y, int incy);
cudaError_t ccopy(iclblasHandle_t h, int n, const cfloat* x, int incx, cfloat* y, int incy);
cudaError_t sswap(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy);
cudaError_t cswap(iclblasHandle_t h, int n, cfloat* x, int incx, cfloat* y, int incy);
cudaError_t srot(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy, float c, float s);
cudaError_t csrot(iclblasHandle_t h, int n, cfloat* x, int incx, cfloat* y, int incy, float c, float s);
cudaError_t crot(iclblasHandle_t h, int n, cfloat* x, int incx, cfloat* y, int incy, float c, cfloat s);
// Exactly one of host_param (read now) and dev_param (read by the kernel) is set.
cudaError_t srotm(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy, const float* host_param,
                  const float* dev_param);
// Generators: every pointer is device memory.
cudaError_t srotg(iclblasHandle_t h, float* a, float* b, float* c, float* s);
cudaError_t crotg(iclblasHandle_t h, cfloat* a, cfloat* b, float* c, cfloat* s);
cudaError_t srotmg(iclblasHandle_t h, float* d1, float* d2, float* x1, const float* y1, float* param);

// ---------------------------------------------------------------- level 2
cudaError_t sgemv(iclblasHandle_t h, int trans, int m, int n, float alpha, const float* A, int lda,
                  const float* x, int incx, float beta, float* y, int incy);
cudaError_t cgemv(iclblasHandle_t h, int trans, int m, int n, cfloat alpha, const cfloat* A, int lda,
                  const cfloat* x, int incx, cfloat beta, cfloat* y, int incy);
cudaError_t strsv(iclblasHandle_t h, int uplo, int trans, int diag, int n, const float* A, int lda, float* x,
                  int incx);
cudaError_t ctrsv(iclblasHandle_t h, int uplo, int trans, int diag, int n, const cfloat* A, int lda, cfloat* x,
                  int incx);

// rank-1 updates (ger.cu) and symmetric / Hermitian products (symv.cu)
cudaError_t sger(iclblasHandle_t h, int m, int n, float alpha, const float* x, int incx, const float* y, int incy,
                 float* A, int lda);
cudaError_t cger(iclblasHandle_t h, bool conj, int m, int n, cfloat alpha, const cfloat* x, int incx,
                 const cfloat* y, int incy, cfloat* A, int lda);
cudaError_t ssymv(iclblasHandle_t h, int uplo, int n, float alpha, const float* A, int lda, const float* x, int incx,
                  float beta, float* y, int incy);
cudaError_t chemv(iclblasHandle_t h, int uplo, int n, cfloat alpha, const cfloat* A, int lda, const cfloat* x,
                  int incx, cfloat beta, cfloat* y, int incy);

// ---------------------------------------------------------------- level 3
cudaError_t sgemm(iclblasHandle_t h, int transa, int transb, int m, int n, int k, float alpha, const float* A,
                  int lda, const float* B, int ldb, float beta, float* C, int ldc);
// GEMM on IEEE half storage (A, B and C hold 16-bit halves): tensor-core
// products, FP32 accumulation, alpha * acc + beta * C rounded once to half.
cudaError_t hgemm(iclblasHandle_t h, int transa, int transb, int m, int n, int k, float alpha, const void* A, int lda,
                  const void* B, int ldb, float beta, void* C, int ldc);
// S GEMM forming only one triangle of C: tri 1 writes (and reads, for beta)
// only row >= col, tri 2 only row <= col; tiles outside the triangle are not
// computed.  tri 0 is the plain GEMM.
cudaError_t sgemm_tri(iclblasHandle_t h, int tri, int transa, int transb, int m, int n, int k, float alpha,
                      const float* A, int lda, const float* B, int ldb, float beta, float* C, int ldc);
cudaError_t cgemm(iclblasHandle_t h, int transa, int transb, int m, int n, int k, cfloat alpha, const cfloat* A,
                  int lda, const cfloat* B, int ldb, cfloat beta, cfloat* C, int ldc);
cudaError_t strsm(iclblasHandle_t h, int side, int uplo, int trans, int diag, int m, int n, float alpha,
                  const float* A, int lda, float* B, int ldb);
cudaError_t ctrsm(iclblasHandle_t h, int side, int uplo, int trans, int diag, int m, int n, cfloat alpha,
                  const cfloat* A, int lda, cfloat* B, int ldb);

// GEMM-shaped level-3 routines (level3_ext.cu)
cudaError_t ssyrk(iclblasHandle_t h, int uplo, int trans, int n, int k, float alpha, const float* A, int lda,
                  float beta, float* C, int ldc);
cudaError_t ssyr2k(iclblasHandle_t h, int uplo, int trans, int n, int k, float alpha, const float* A, int lda,
                   const float* B, int ldb, float beta, float* C, int ldc);
cudaError_t ssymm(iclblasHandle_t h, int side, int uplo, int m, int n, float alpha, const float* A, int lda,
                  const float* B, int ldb, float beta, float* C, int ldc);
cudaError_t strmm(iclblasHandle_t h, int side, int uplo, int transa, int diag, int m, int n, float alpha,
                  const float* A, int lda, const float* B, int ldb, float* C, int ldc);

// ---------------------------------------------------------------- adjoints
cudaError_t strsm_backward(iclblasHandle_t h, int side, int uplo, int trans, int diag, int m, int n, float alpha,
                           const float* A, int lda, const float* X, int ldx, float* G, int ldg, float* dA, int ldda);
cudaError_t sgemm_backward(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const float* A, int lda,
                           const float* B, int ldb, float beta, const float* G, int ldg, float* dA, int ldda,
                           float* dB, int lddb, float* dC, int lddc);

// ---------------------------------------------------------------- batched
// A plan for uneven batched TRSM (left side) or GEMM: per-instance sizes and
// a cost-sorted work list in device memory, plus the tuned launch shape.
struct BatchList {
    int* dims = nullptr;     // per instance: TRSM (m, n, lda, ldb); GEMM (m, n, k, lda, ldb, ldc)
    int2* items = nullptr;   // (instance, tile) work items, most expensive first
    int nitems = 0;
    int rc = 64;             // tile width (right-hand sides / C columns per item)
    int ctas_per_sm = 1;
};
cudaError_t batch_list_free(BatchList& l);
struct BatchTc;  // a plan's tensor-core path (batched_tc.cu)

}  // namespace iclb

constexpr uint32_t kBatchPlanTag = 0xBA7C4001u;
struct iclblasBatchPlan {
    uint32_t tag = 0;
    int kind = 0;   // 0 = TRSM, 1 = GEMM
    int side = 0, uplo = 0, trans = 0, diag = 0;
    int transa = 0, transb = 0;
    int batch = 0;
    int device = 0;
    double flops = 0;
    iclb::BatchList main;   // the TRSM (forward and the adjoint's solve) or the GEMM
    iclb::BatchList adj;    // TRSM plans: the masked dA product of the adjoint
    unsigned* counter = nullptr;   // work-queue head, cleared before each launch
    // TRSM plans: FP32 inverses of every 64 x 64 diagonal block of every
    // instance (formed by each call), their per-instance offsets and the
    // (instance, block) list of the pass that forms them
    float* inv = nullptr;
    long* inv_off = nullptr;
    int2* inv_items = nullptr;
    int n_inv = 0;
    // the backward call may use the inverses of the last forward call
    // (iclblasBatchPlanSetInverseReuse); inv_formed: a forward call formed them
    bool reuse_inv = false;
    mutable bool inv_formed = false;
    // plans created in a tensor-core math mode (TF32, 3xBF16, 6xBF16): the
    // tiled operand planes and launch lists of that path; null in PLAIN_FP32
    iclb::BatchTc* tc = nullptr;
};

namespace iclb {
cudaError_t batch_plan_create_trsm(iclblasHandle_t h, int side, int uplo, int trans, int diag, int batch,
                                   const int* m, const int* n, const int* lda, const int* ldb,
                                   iclblasBatchPlan** out);
cudaError_t batch_plan_create_gemm(iclblasHandle_t h, int transa, int transb, int batch, const int* m, const int* n,
                                   const int* k, const int* lda, const int* ldb, const int* ldc,
                                   iclblasBatchPlan** out);
void batch_plan_free(iclblasBatchPlan* p);
cudaError_t batch_trsm(iclblasHandle_t h, const iclblasBatchPlan* p, float alpha, const float* const* A,
                       float* const* B);
cudaError_t batch_gemm(iclblasHandle_t h, const iclblasBatchPlan* p, float alpha, const float* const* A,
                       const float* const* B, float beta, float* const* C);
cudaError_t batch_trsm_backward(iclblasHandle_t h, const iclblasBatchPlan* p, float alpha, const float* const* A,
                                const float* const* X, float* const* G, float* const* dA);

}  // namespace iclb
