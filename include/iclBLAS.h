/*
 * iclBLAS C API -- B200 (sm_100a) implementation.
 *
 * Call-compatible drop-in for the hot-path subset of Intel clGPU's
 * include/iclBLAS/iclBLAS.h: the same type names, enum values, function names
 * and parameter order, so code written against the reference header compiles
 * and links against libiclblas_b200.so unchanged.  Every prototype below cites
 * the reference declaration it replaces (include/iclBLAS/iclBLAS.h:<line>).
 *
 * Semantics kept from the reference:
 *   - column-major storage, element (i,j) of a matrix at A[j*lda + i];
 *   - scalars (alpha, beta) are host pointers read at call time;
 *   - array arguments may be HOST pointers (as in the reference: the call
 *     copies them to the device, runs, copies outputs back and returns when
 *     the results are in host memory) or DEVICE pointers (extension: the call
 *     is enqueued on the handle's stream and returns without waiting);
 *     device memory must belong to the GPU the handle was created on (or be
 *     managed memory): another GPU's memory gives INVALID_VALUE, before any
 *     copy or launch;
 *   - result arguments of reductions (dot/nrm2/asum/iamax) follow the same
 *     rule: a host pointer is written before return, a device pointer is
 *     written by the device in stream order;
 *   - iclblasIsamax / iclblasIcamax return a 0-based index;
 *   - the error and early-return rules of libs/blas/shlib/iclBLAS_S.cpp,
 *     iclBLAS_C.cpp and iclBLASImpl.hpp (validation order n, m, k, x, incx,
 *     y, incy, A, lda, B, ldb, C, ldc; negative increments NOT_SUPPORTED).
 *
 * A handle owns one CUDA stream; it is not thread-safe, separate handles are
 * independent (the reference has the same contract: one queue per handle).
 */
#ifndef ICLBLAS_B200_H
#define ICLBLAS_B200_H

#if defined(__GNUC__)
#   define ICLBLAS_API __attribute__((visibility("default")))
#else
#   define ICLBLAS_API
#endif

#if defined(__GNUC__) || defined(__clang__)
#   define ICLBLAS_ALWAYS_INLINE static inline __attribute__((always_inline))
#else
#   define ICLBLAS_ALWAYS_INLINE static inline
#endif

/* Complex single: two packed floats, {re, im}.  Same layout as the
 * reference's oclComplex_t (iclBLAS.h:71-86), float2 and cuFloatComplex. */
#ifdef __cplusplus
#   include <complex>
    typedef std::complex<float> oclComplex_t;
    inline float Creal(const oclComplex_t& a)       { return a.real(); }
    inline float Cimag(const oclComplex_t& a)       { return a.imag(); }
    inline void  Csetreal(oclComplex_t* a, float r) { a->real(r); }
    inline void  Csetimag(oclComplex_t* a, float i) { a->imag(i); }
#else
    typedef struct _oclComplex_t { float val[2]; } oclComplex_t;
    ICLBLAS_ALWAYS_INLINE float Creal(struct _oclComplex_t a)              { return a.val[0]; }
    ICLBLAS_ALWAYS_INLINE float Cimag(struct _oclComplex_t a)              { return a.val[1]; }
    ICLBLAS_ALWAYS_INLINE void  Csetreal(struct _oclComplex_t* a, float r) { a->val[0] = r; }
    ICLBLAS_ALWAYS_INLINE void  Csetimag(struct _oclComplex_t* a, float i) { a->val[1] = i; }
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: values of iclBLAS.h:104-117 (ERROR follows LICENSE_ERROR). */
typedef enum {
    ICLBLAS_STATUS_SUCCESS          = 0,
    ICLBLAS_STATUS_NOT_INITIALIZED  = 1,
    ICLBLAS_STATUS_ALLOC_FAILED     = 3,
    ICLBLAS_STATUS_INVALID_VALUE    = 7,
    ICLBLAS_STATUS_ARCH_MISMATCH    = 8,
    ICLBLAS_STATUS_MAPPING_ERROR    = 11,
    ICLBLAS_STATUS_EXECUTION_FAILED = 13,
    ICLBLAS_STATUS_INTERNAL_ERROR   = 14,
    ICLBLAS_STATUS_NOT_SUPPORTED    = 15,
    ICLBLAS_STATUS_LICENSE_ERROR    = 16,
    ICLBLAS_STATUS_ERROR            = 17
} iclblasStatus_t;

/* Opaque library context (iclBLAS.h:123). */
typedef struct iclblasContext* iclblasHandle_t;

/* Enumerations: values of iclBLAS.h:128-158. */
typedef enum { ICLBLAS_OP_N = 0, ICLBLAS_OP_T = 1, ICLBLAS_OP_C = 2 } iclblasOperation_t;
typedef enum { ICLBLAS_FILL_MODE_UPPER = 0, ICLBLAS_FILL_MODE_LOWER = 1 } iclblasFillMode_t;
typedef enum { ICLBLAS_DIAG_NON_UNIT = 0, ICLBLAS_DIAG_UNIT = 1 } iclblasDiagType_t;
typedef enum { ICLBLAS_SIDE_LEFT = 0, ICLBLAS_SIDE_RIGHT = 1 } iclblasSideMode_t;

/* ---- utilities ---- */
/* replaces iclBLAS.h:172 */
ICLBLAS_API iclblasStatus_t iclblasCreate(iclblasHandle_t* handle);
/* replaces iclBLAS.h:179 */
ICLBLAS_API iclblasStatus_t iclblasDestroy(iclblasHandle_t handle);

/* ---- level 1, single ---- */
/* replaces iclBLAS.h:219 */
ICLBLAS_API iclblasStatus_t iclblasSscal(iclblasHandle_t handle, int n, const float* alpha, float* x, int incx);
/* replaces iclBLAS.h:237 */
ICLBLAS_API iclblasStatus_t iclblasSaxpy(iclblasHandle_t handle, int n, const float* alpha, float* x, int incx, float* y, int incy);
/* replaces iclBLAS.h:250 */
ICLBLAS_API iclblasStatus_t iclblasSnrm2(iclblasHandle_t handle, int n, float* x, int incx, float* result);
/* replaces iclBLAS.h:275 (0-based index) */
ICLBLAS_API iclblasStatus_t iclblasIsamax(iclblasHandle_t handle, int n, float* x, int incx, int* result);
/* replaces iclBLAS.h:345 */
ICLBLAS_API iclblasStatus_t iclblasSasum(iclblasHandle_t handle, int n, float* x, int incx, float* result);
/* replaces iclBLAS.h:371 */
ICLBLAS_API iclblasStatus_t iclblasSdot(iclblasHandle_t handle, int n, float* x, int incx, float* y, int incy, float* result);
/* No counterpart in the reference: SDOT that allocates no device memory.
 * For callers that cannot call cudaMalloc: code whose device memory is owned
 * by another allocator (a framework's caching pool that has reserved the free
 * memory, so a private cudaMalloc would fail), and latency-critical paths
 * that must not call cudaMalloc/cudaFree because those can synchronize the
 * device and serialize with other host threads.  iclblasSdot may grow the
 * handle's workspace with cudaMalloc/cudaFree; this variant instead keeps its
 * scratch (one FP64 partial per thread block, at most 4096, and a ticket
 * counter: 32 KiB + 256 B) in a fixed array compiled into the library, which
 * every GPU that loads the library holds until the process exits.
 *   - x, y and result must be device pointers on the handle's GPU
 *     (INVALID_VALUE otherwise: staging host data would allocate, and a
 *     kernel cannot read another GPU's memory); the call is asynchronous on the
 *     handle's stream and its result equals iclblasSdot's;
 *   - a call needing more than 4096 partials -- one per block, with
 *     min(ceil(n/1024), 8 x SM count) blocks for unit-stride 16-byte-aligned
 *     operands and min(ceil(n/256), 8 x SM count) otherwise -- returns
 *     NOT_SUPPORTED;
 *   - the first call on each device looks up the array's device address
 *     (cudaGetSymbolAddress) in the CUDA runtime's context of that device
 *     (its primary context; a context made current through the driver API is
 *     not supported), and looks it up again once that context has changed
 *     (after cudaDeviceReset); make that first call before any stream capture;
 *   - all calls share the one array, which keeps the previous call's
 *     contents (the counter is cleared at the start of each call): calls that
 *     overlap on the GPU (other streams or handles at the same time) race and
 *     give wrong results, so serialize them. */
ICLBLAS_API iclblasStatus_t iclblasSdotNoAlloc(iclblasHandle_t handle, int n, const float* x, int incx, const float* y,
                                               int incy, float* result);

/* ---- level 1, single: copy, swap, rotations, iamin ----
 * Vector arguments follow the same host/device rule as above.  Srot's c and
 * s are passed by value; Srotm's param may be a host pointer (read at call
 * time; flag -2 returns at once) or a device pointer (read by the kernel,
 * which leaves x and y unchanged for any flag outside {-1, 0, 1}).  param
 * uses the reference's layout {flag, p1, p2, p3, p4} with
 *   flag -1: x' = p1 x + p2 y, y' = p3 x + p4 y
 *   flag  0: x' = x + p2 y,    y' = p3 x + y
 *   flag  1: x' = p1 x + y,    y' = p4 y - x
 * (libs/blas/funcs/Srotm/Srotm_helpers.h.cl).  The generators (Srotg,
 * Srotmg, Crotg) accept all-host or all-device operands and reproduce the
 * reference kernels' formulas, including Srotg's zero result when a or b is
 * 0 and Srotmg's partial writes of param for flags 0, 1 and -2. */
/* replaces iclBLAS.h:203 */
ICLBLAS_API iclblasStatus_t iclblasScopy(iclblasHandle_t handle, int n, float* x, int incx, float* y, int incy);
/* replaces iclBLAS.h:262 */
ICLBLAS_API iclblasStatus_t iclblasSrotmg(iclblasHandle_t handle, float* d1, float* d2, float* x1, const float* y1, float* params);
/* replaces iclBLAS.h:288 (0-based index of the first smallest |x_i|) */
ICLBLAS_API iclblasStatus_t iclblasIsamin(iclblasHandle_t handle, int n, float* x, int incx, int* result);
/* replaces iclBLAS.h:305 */
ICLBLAS_API iclblasStatus_t iclblasSswap(iclblasHandle_t handle, int n, float* x, int incx, float* y, int incy);
/* replaces iclBLAS.h:319 */
ICLBLAS_API iclblasStatus_t iclblasSrot(iclblasHandle_t handle, int n, float* x, int incx, float* y, int incy, float c, float s);
/* replaces iclBLAS.h:332 */
ICLBLAS_API iclblasStatus_t iclblasSrotm(iclblasHandle_t handle, int n, float* x, int incx, float* y, int incy, float* param);
/* replaces iclBLAS.h:356 */
ICLBLAS_API iclblasStatus_t iclblasSrotg(iclblasHandle_t handle, float* a, float* b, float* c, float* s);

/* ---- level 1, complex ---- */
/* replaces iclBLAS.h:411 */
ICLBLAS_API iclblasStatus_t iclblasCscal(iclblasHandle_t handle, int n, const oclComplex_t* alpha, oclComplex_t* x, int incx);
/* replaces iclBLAS.h:427 */
ICLBLAS_API iclblasStatus_t iclblasCsscal(iclblasHandle_t handle, int n, const float* alpha, oclComplex_t* x, int incx);
/* replaces iclBLAS.h:462 */
ICLBLAS_API iclblasStatus_t iclblasCdotu(iclblasHandle_t handle, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy, oclComplex_t* result);
/* replaces iclBLAS.h:475 */
ICLBLAS_API iclblasStatus_t iclblasScnrm2(iclblasHandle_t handle, int n, oclComplex_t* x, int incx, float* result);
/* replaces iclBLAS.h:488 (0-based index) */
ICLBLAS_API iclblasStatus_t iclblasIcamax(iclblasHandle_t handle, int n, oclComplex_t* x, int incx, int* result);
/* replaces iclBLAS.h:519 */
ICLBLAS_API iclblasStatus_t iclblasCaxpy(iclblasHandle_t handle, int n, const oclComplex_t* alpha, oclComplex_t* x, int incx, oclComplex_t* y, int incy);
/* replaces iclBLAS.h:549 */
ICLBLAS_API iclblasStatus_t iclblasCdotc(iclblasHandle_t handle, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy, oclComplex_t* result);
/* replaces iclBLAS.h:590 */
ICLBLAS_API iclblasStatus_t iclblasScasum(iclblasHandle_t handle, int n, oclComplex_t* x, int incx, float* result);

/* ---- level 1, complex: copy, swap, rotations, iamin ----
 * Crot and Csrot read c and s through host pointers at call time. */
/* replaces iclBLAS.h:395 */
ICLBLAS_API iclblasStatus_t iclblasCcopy(iclblasHandle_t handle, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy);
/* replaces iclBLAS.h:444 */
ICLBLAS_API iclblasStatus_t iclblasCswap(iclblasHandle_t handle, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy);
/* replaces iclBLAS.h:501 (0-based index of the first smallest |re| + |im|) */
ICLBLAS_API iclblasStatus_t iclblasIcamin(iclblasHandle_t handle, int n, oclComplex_t* x, int incx, int* result);
/* replaces iclBLAS.h:530 */
ICLBLAS_API iclblasStatus_t iclblasCrotg(iclblasHandle_t handle, oclComplex_t* a, oclComplex_t* b, float* c, oclComplex_t* s);
/* replaces iclBLAS.h:563 */
ICLBLAS_API iclblasStatus_t iclblasCrot(iclblasHandle_t handle, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy,
                                        const float* c, const oclComplex_t* s);
/* replaces iclBLAS.h:577 */
ICLBLAS_API iclblasStatus_t iclblasCsrot(iclblasHandle_t handle, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy,
                                         const float* c, const float* s);

/* ---- level 2 ---- */
/* replaces iclBLAS.h:630 */
ICLBLAS_API iclblasStatus_t iclblasStrsv(iclblasHandle_t handle, iclblasFillMode_t uplo, iclblasOperation_t trans, iclblasDiagType_t diag,
                                         int n, float* A, int lda, float* x, int incx);
/* replaces iclBLAS.h:1049 */
ICLBLAS_API iclblasStatus_t iclblasSgemv(iclblasHandle_t handle, iclblasOperation_t trans, int m, int n, const float* alpha,
                                         float* A, int lda, float* x, int incx, const float* beta, float* y, int incy);
/* replaces iclBLAS.h:1164 */
ICLBLAS_API iclblasStatus_t iclblasCgemv(iclblasHandle_t handle, iclblasOperation_t trans, int m, int n, const oclComplex_t* alpha,
                                         oclComplex_t* A, int lda, oclComplex_t* x, int incx, const oclComplex_t* beta,
                                         oclComplex_t* y, int incy);
/* replaces iclBLAS.h:1463 */
ICLBLAS_API iclblasStatus_t iclblasCtrsv(iclblasHandle_t handle, iclblasFillMode_t uplo, iclblasOperation_t trans, iclblasDiagType_t diag,
                                         int n, oclComplex_t* A, int lda, oclComplex_t* x, int incx);

/* ---- level 2: rank-1 updates, symmetric / Hermitian products ----
 * Ssymv / Chemv read only the uplo triangle of A (Chemv takes the real part
 * of its diagonal); beta == 0 writes y without reading it. */
/* replaces iclBLAS.h:727 */
ICLBLAS_API iclblasStatus_t iclblasSger(iclblasHandle_t handle, int m, int n, const float* alpha, float* x, int incx, float* y, int incy,
                                        float* A, int lda);
/* replaces iclBLAS.h:1018 */
ICLBLAS_API iclblasStatus_t iclblasSsymv(iclblasHandle_t handle, iclblasFillMode_t uplo, int n, const float* alpha, float* A, int lda,
                                         float* x, int incx, const float* beta, float* y, int incy);
/* replaces iclBLAS.h:1112 */
ICLBLAS_API iclblasStatus_t iclblasCgeru(iclblasHandle_t handle, int m, int n, const oclComplex_t* alpha, oclComplex_t* x, int incx,
                                         oclComplex_t* y, int incy, oclComplex_t* A, int lda);
/* replaces iclBLAS.h:1133 */
ICLBLAS_API iclblasStatus_t iclblasCgerc(iclblasHandle_t handle, int m, int n, const oclComplex_t* alpha, oclComplex_t* x, int incx,
                                         oclComplex_t* y, int incy, oclComplex_t* A, int lda);
/* replaces iclBLAS.h:1205 */
ICLBLAS_API iclblasStatus_t iclblasChemv(iclblasHandle_t handle, iclblasFillMode_t uplo, int n, const oclComplex_t* alpha,
                                         oclComplex_t* A, int lda, oclComplex_t* x, int incx, const oclComplex_t* beta,
                                         oclComplex_t* y, int incy);

/* ---- level 3 ---- */
/* replaces iclBLAS.h:1685 */
ICLBLAS_API iclblasStatus_t iclblasSgemm(iclblasHandle_t handle, iclblasOperation_t transa, iclblasOperation_t transb, int m, int n, int k,
                                         const float* alpha, float* A, int lda, float* B, int ldb, const float* beta, float* C, int ldc);
/* replaces iclBLAS.h:1719 */
ICLBLAS_API iclblasStatus_t iclblasStrsm(iclblasHandle_t handle, iclblasSideMode_t side, iclblasFillMode_t uplo, iclblasOperation_t trans,
                                         iclblasDiagType_t diag, int m, int n, const float* alpha, float* A, int lda, float* B, int ldb);
/* replaces iclBLAS.h:1799 */
ICLBLAS_API iclblasStatus_t iclblasCgemm(iclblasHandle_t handle, iclblasOperation_t transa, iclblasOperation_t transb, int m, int n, int k,
                                         const oclComplex_t* alpha, oclComplex_t* A, int lda, oclComplex_t* B, int ldb,
                                         const oclComplex_t* beta, oclComplex_t* C, int ldc);
/* replaces iclBLAS.h:1925 */
ICLBLAS_API iclblasStatus_t iclblasCtrsm(iclblasHandle_t handle, iclblasSideMode_t side, iclblasFillMode_t uplo, iclblasOperation_t trans,
                                         iclblasDiagType_t diag, int m, int n, const oclComplex_t* alpha, oclComplex_t* A, int lda,
                                         oclComplex_t* B, int ldb);

/* ---- level 3 on the GEMM engine (the handle's math mode applies) ----
 * Ssyrk / Ssyr2k update only the uplo triangle of C; Ssymm reads only the
 * uplo triangle of A.  beta == 0 writes C without reading it.  Strmm computes
 * the documented C = alpha op(A) B (left) or alpha B op(A) (right) with A
 * triangular (uplo, diag) into a separate C, which may be B itself: an
 * overlapping C gets the product of the original B. */
/* replaces iclBLAS.h:1579 */
ICLBLAS_API iclblasStatus_t iclblasSsymm(iclblasHandle_t handle, iclblasSideMode_t side, iclblasFillMode_t uplo, int m, int n,
                                         const float* alpha, float* A, int lda, float* B, int ldb, const float* beta, float* C, int ldc);
/* replaces iclBLAS.h:1608 */
ICLBLAS_API iclblasStatus_t iclblasSsyrk(iclblasHandle_t handle, iclblasFillMode_t uplo, iclblasOperation_t trans, int n, int k,
                                         const float* alpha, float* A, int lda, const float* beta, float* C, int ldc);
/* replaces iclBLAS.h:1645 */
ICLBLAS_API iclblasStatus_t iclblasSsyr2k(iclblasHandle_t handle, iclblasFillMode_t uplo, iclblasOperation_t trans, int n, int k,
                                          const float* alpha, float* A, int lda, float* B, int ldb, const float* beta, float* C, int ldc);
/* replaces iclBLAS.h:1753 */
ICLBLAS_API iclblasStatus_t iclblasStrmm(iclblasHandle_t handle, iclblasSideMode_t side, iclblasFillMode_t uplo, iclblasOperation_t transa,
                                         iclblasDiagType_t diag, int m, int n, const float* alpha, float* A, int lda, float* B, int ldb,
                                         float* C, int ldc);

/* ======================================================================== */
/* Extensions (new symbols; no reference counterpart).                      */
/* ======================================================================== */

/* Half-precision GEMM: C = alpha op(A) op(B) + beta C with A, B and C in IEEE
 * 754 binary16 (each element an unsigned short holding the bit pattern),
 * column-major as the other routines.  Products run on the tensor cores,
 * the K sum accumulates in FP32 and alpha * acc + beta * C is rounded to
 * half once (round to nearest even).  alpha and beta are FP32 host scalars;
 * beta == 0 writes C without reading it.  The reference ships FP16 GEMM only
 * as stand-alone experimental OpenCL kernels (experimental/kernels/
 * hgemm_buf_*.cl, for ResNet-50 1x1 convolutions), not through its API. */
ICLBLAS_API iclblasStatus_t iclblasHgemm(iclblasHandle_t handle, iclblasOperation_t transa, iclblasOperation_t transb,
                                         int m, int n, int k, const float* alpha, const unsigned short* A, int lda,
                                         const unsigned short* B, int ldb, const float* beta, unsigned short* C, int ldc);

/* Arithmetic used by S/C GEMM and by the trailing updates of S/C TRSM.
 *   PLAIN_FP32: FP32 FFMA on the CUDA cores (the drop-in default);
 *   TF32:       one TF32 product on the tensor cores, FP32 accumulate;
 *   BF16X3:     FP32 operands split into three BF16 terms, the three leading
 *               cross products on the tensor cores, FP32 accumulate;
 *   BF16X6:     as BF16X3 with all six products of split order <= 2. */
typedef enum {
    ICLBLAS_MATH_PLAIN_FP32 = 0,
    ICLBLAS_MATH_TF32       = 1,
    ICLBLAS_MATH_BF16X3     = 2,
    ICLBLAS_MATH_BF16X6     = 3
} iclblasMathMode_t;

/* Stream of the handle (a cudaStream_t passed as void*; NULL = the legacy
 * default stream).  A new handle uses a stream of its own.  Device-pointer
 * calls are enqueued on the handle's stream. */
ICLBLAS_API iclblasStatus_t iclblasSetStream(iclblasHandle_t handle, void* stream);
ICLBLAS_API iclblasStatus_t iclblasGetStream(iclblasHandle_t handle, void** stream);
ICLBLAS_API iclblasStatus_t iclblasSetMathMode(iclblasHandle_t handle, iclblasMathMode_t mode);
ICLBLAS_API iclblasStatus_t iclblasGetMathMode(iclblasHandle_t handle, iclblasMathMode_t* mode);
/* TRSM residual refinement, no reference counterpart.  With steps = 1 or 2
 * (0, the default, turns it off), S/C TRSM follows its solve X by `steps`
 * rounds of: R = B - op(A) X with FP32-accurate products (6xBF16 on the tensor
 * cores in the tensor-core modes, FP32 on the CUDA cores in PLAIN_FP32),
 * D = solve(R) in the handle's math mode with the same FP64-formed diagonal
 * inverses, X = X + D.  Each round costs about one extra solve plus one
 * triangle product and needs workspace for two copies of B. */
ICLBLAS_API iclblasStatus_t iclblasSetTrsmRefinement(iclblasHandle_t handle, int steps);
ICLBLAS_API iclblasStatus_t iclblasGetTrsmRefinement(iclblasHandle_t handle, int* steps);
/* Wait for all work enqueued on the handle's stream; reports a device-side
 * error flag (a bounded wait that ran out) as EXECUTION_FAILED. */
ICLBLAS_API iclblasStatus_t iclblasSynchronize(iclblasHandle_t handle);

/* Adjoints (reverse-mode derivatives), no reference counterpart.
 * iclblasStrsm_backward: given the TRSM inputs A, the solution X (= the B that
 * iclblasStrsm returned) and G = dL/dX, overwrites G with dL/dB and writes
 * dL/dA into dA on the stored triangle of A (zero elsewhere; zero diagonal for
 * a unit diagonal).  dA may be NULL.  Left side: W = op(A)^-T G, dB = alpha W,
 * d op(A) = -W X^T; right side: W = G op(A)^-T, dB = alpha W,
 * d op(A) = -X^T W. */
ICLBLAS_API iclblasStatus_t iclblasStrsm_backward(iclblasHandle_t handle, iclblasSideMode_t side, iclblasFillMode_t uplo,
                                                  iclblasOperation_t trans, iclblasDiagType_t diag, int m, int n,
                                                  const float* alpha, const float* A, int lda, const float* X, int ldx,
                                                  float* G, int ldg, float* dA, int ldda);
/* iclblasSgemm_backward: for C = alpha*op(A)*op(B) + beta*C_in and G = dL/dC,
 * writes dL/dA (shape of A), dL/dB (shape of B) and dL/dC_in = beta*G; any of
 * dA, dB, dC may be NULL. */
ICLBLAS_API iclblasStatus_t iclblasSgemm_backward(iclblasHandle_t handle, iclblasOperation_t transa,
                                                  iclblasOperation_t transb, int m, int n, int k, const float* alpha,
                                                  const float* A, int lda, const float* B, int ldb, const float* beta,
                                                  const float* G, int ldg, float* dA, int ldda, float* dB, int lddb,
                                                  float* dC, int lddc);

/* Uneven batched TRSM and GEMM, no reference counterpart.  A plan is built
 * once for a list of instance sizes (host arrays of `batch` ints) and takes
 * the handle's math mode at creation.  PLAIN_FP32 plans: each call runs
 * every instance in one persistent launch per stage (a memset of the plan's
 * work-queue head plus one kernel) with FP32 FMA on the CUDA cores; plan
 * creation times the launch-shape candidates on synthetic operands (the
 * choice is cached per shapes and GPU, and in the file named by the
 * environment variable ICLBLAS_TUNE_CACHE when set).  TF32 / 3xBF16 / 6xBF16
 * plans: the products run on the tensor cores over operands split into
 * planes once per call, TRSM by 128-row block steps (two launches per step
 * of the largest instance); the plan holds the planes (about 2.8 GB for
 * 512 instances of order up to 1024 in 6xBF16).  Either way the calls only
 * launch kernels on the handle's stream and can be captured in a CUDA graph;
 * plan creation is synchronous and allocates device memory: do not create a
 * plan during stream capture.  The calls take device arrays of `batch`
 * device pointers, one per instance; a plan serves one stream at a time.
 * TRSM: instance i solves op(A_i) X_i = alpha B_i (left side, A_i m_i x m_i,
 * lda_i >= max(1, m_i)) or X_i op(A_i) = alpha B_i (right side, A_i n_i x n_i,
 * lda_i >= max(1, n_i)); B_i is m_i x n_i with ldb_i >= max(1, m_i).
 * GEMM: C_i = alpha op(A_i) op(B_i) + beta C_i, leading dimensions at least
 * the stored row counts; in a PLAIN_FP32 plan each element is bit-identical
 * to iclblasSgemm in PLAIN_FP32 mode. */
typedef struct iclblasBatchPlan* iclblasBatchPlan_t;
ICLBLAS_API iclblasStatus_t iclblasStrsmBatchedPlanCreate(iclblasHandle_t handle, iclblasSideMode_t side,
                                                          iclblasFillMode_t uplo, iclblasOperation_t trans,
                                                          iclblasDiagType_t diag, int batch, const int* m,
                                                          const int* n, const int* lda, const int* ldb,
                                                          iclblasBatchPlan_t* plan);
ICLBLAS_API iclblasStatus_t iclblasSgemmBatchedPlanCreate(iclblasHandle_t handle, iclblasOperation_t transa,
                                                          iclblasOperation_t transb, int batch, const int* m,
                                                          const int* n, const int* k, const int* lda, const int* ldb,
                                                          const int* ldc, iclblasBatchPlan_t* plan);
ICLBLAS_API iclblasStatus_t iclblasBatchPlanDestroy(iclblasBatchPlan_t plan);
/* Algorithmic flops of one call (TRSM sum m^2 n, GEMM sum 2mnk) and the
 * launch shape (tile width, CTAs per SM: the tuner's choice in a PLAIN_FP32
 * plan, 128 and 1 in a tensor-core plan); any output may be NULL. */
ICLBLAS_API iclblasStatus_t iclblasBatchPlanGetInfo(iclblasBatchPlan_t plan, double* flops, int* tile_width,
                                                    int* ctas_per_sm);
/* TRSM plans: with reuse = 1, iclblasStrsmBatchedUnevenBackward uses the
 * diagonal-block inverses formed by the plan's most recent
 * iclblasStrsmBatchedUneven call instead of forming them again (it forms
 * them when no forward call has run yet); a tensor-core plan in the BF16
 * modes also reuses that call's split operator tiles.  The caller promises that the
 * triangles A_i are unchanged since that forward call and that the two
 * calls run in order on one stream.  0 (the default) forms them in every
 * call.  INVALID_VALUE for a GEMM plan or another value. */
ICLBLAS_API iclblasStatus_t iclblasBatchPlanSetInverseReuse(iclblasBatchPlan_t plan, int reuse);
ICLBLAS_API iclblasStatus_t iclblasStrsmBatchedUneven(iclblasHandle_t handle, iclblasBatchPlan_t plan,
                                                      const float* alpha, const float* const* A, float* const* B);
ICLBLAS_API iclblasStatus_t iclblasSgemmBatchedUneven(iclblasHandle_t handle, iclblasBatchPlan_t plan,
                                                      const float* alpha, const float* const* A,
                                                      const float* const* B, const float* beta, float* const* C);
/* Batched iclblasStrsm_backward for a TRSM plan: X_i and G_i use ldb_i, dA_i
 * uses lda_i; G_i is overwritten with dL/dB_i, dA_i receives dL/dA_i on the
 * stored triangle (zero elsewhere).  dA may be NULL (then only dB). */
ICLBLAS_API iclblasStatus_t iclblasStrsmBatchedUnevenBackward(iclblasHandle_t handle, iclblasBatchPlan_t plan,
                                                              const float* alpha, const float* const* A,
                                                              const float* const* X, float* const* G,
                                                              float* const* dA);

#ifdef __cplusplus
}
#endif
#endif /* ICLBLAS_B200_H */
