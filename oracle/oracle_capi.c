/*
 * The iclBLAS C API implemented on the CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * Links the reference's own C-API known-answer suite (tests/iclBLAS/test_*.cpp
 * of the clGPU tree, compiled by oracle/Makefile) against the oracle, which is
 * how the oracle is pinned to the reference's golden vectors.  Host pointers
 * only.  Argument checks restate the reference's rules:
 *   - per-routine early returns (libs/blas/shlib/iclBLAS_S.cpp, iclBLAS_C.cpp);
 *   - validate_params: n, m, k, x, incx, y, incy, A, lda, B, ldb, C, ldc in
 *     that order, n == 0 or m == 0 ends the call successfully before the
 *     handle is looked at (libs/blas/shlib/iclBLASImpl.hpp:218-245);
 *   - handle tag check (libs/blas/shlib/iclBLAS.cpp:35-39).
 */
#include <stdlib.h>

#include "iclBLAS.h"
#include "oracle.h"

struct iclblasContext { int tag; };
#define ORC_TAG 0x0AC1

enum {
    P_N = 1 << 0, P_M = 1 << 1, P_K = 1 << 2, P_X = 1 << 3, P_INCX = 1 << 4,
    P_Y = 1 << 5, P_INCY = 1 << 6, P_A = 1 << 7, P_LDA = 1 << 8, P_B = 1 << 9,
    P_LDB = 1 << 10, P_C = 1 << 11, P_LDC = 1 << 12
};

typedef struct {
    unsigned present;
    int n, m, k, incx, incy, lda, ldb, ldc;
    const void *x, *y, *A, *B, *C;
} vparams;

/* Returns 0 to run the routine, 1 to return SUCCESS without work, or an
 * error status (>1). */
static int validate(const vparams* p, iclblasHandle_t h)
{
    unsigned f = p->present;
    if (f & P_N) { if (p->n < 0) return ICLBLAS_STATUS_INVALID_VALUE; if (p->n == 0) return 1; }
    if (f & P_M) { if (p->m < 0) return ICLBLAS_STATUS_INVALID_VALUE; if (p->m == 0) return 1; }
    if (f & P_K) { if (p->k < 0) return ICLBLAS_STATUS_INVALID_VALUE; }
    if ((f & P_X) && !p->x) return ICLBLAS_STATUS_INVALID_VALUE;
    if (f & P_INCX) { if (p->incx == 0) return ICLBLAS_STATUS_INVALID_VALUE; if (p->incx < 0) return ICLBLAS_STATUS_NOT_SUPPORTED; }
    if ((f & P_Y) && !p->y) return ICLBLAS_STATUS_INVALID_VALUE;
    if (f & P_INCY) { if (p->incy == 0) return ICLBLAS_STATUS_INVALID_VALUE; if (p->incy < 0) return ICLBLAS_STATUS_NOT_SUPPORTED; }
    if ((f & P_A) && !p->A) return ICLBLAS_STATUS_INVALID_VALUE;
    if ((f & P_LDA) && p->lda <= 0) return ICLBLAS_STATUS_INVALID_VALUE;
    if ((f & P_B) && !p->B) return ICLBLAS_STATUS_INVALID_VALUE;
    if ((f & P_LDB) && p->ldb <= 0) return ICLBLAS_STATUS_INVALID_VALUE;
    if ((f & P_C) && !p->C) return ICLBLAS_STATUS_INVALID_VALUE;
    if ((f & P_LDC) && p->ldc <= 0) return ICLBLAS_STATUS_INVALID_VALUE;
    if (!h || h->tag != ORC_TAG) return ICLBLAS_STATUS_INVALID_VALUE;
    return 0;
}

#define CHECK(p, h) do { int v_ = validate(&(p), (h)); if (v_ == 1) return ICLBLAS_STATUS_SUCCESS; \
                         if (v_) return (iclblasStatus_t)v_; } while (0)

static orc_c32 c32(const oclComplex_t* a) { orc_c32 r = { a->val[0], a->val[1] }; return r; }

iclblasStatus_t iclblasCreate(iclblasHandle_t* handle)
{
    if (!handle) return ICLBLAS_STATUS_INVALID_VALUE;
    *handle = (iclblasHandle_t)malloc(sizeof(struct iclblasContext));
    if (!*handle) return ICLBLAS_STATUS_ALLOC_FAILED;
    (*handle)->tag = ORC_TAG;
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasDestroy(iclblasHandle_t handle)
{
    if (!handle || handle->tag != ORC_TAG) return ICLBLAS_STATUS_INVALID_VALUE;
    handle->tag = 0;
    free(handle);
    return ICLBLAS_STATUS_SUCCESS;
}

/* ---- level 1, single (iclBLAS_S.cpp:66-228) ---- */
iclblasStatus_t iclblasSscal(iclblasHandle_t h, int n, const float* alpha, float* x, int incx)
{
    vparams p = { P_N | P_X | P_INCX, .n = n, .x = x, .incx = incx };
    CHECK(p, h);
    orc_sscal(n, *alpha, x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSaxpy(iclblasHandle_t h, int n, const float* alpha, float* x, int incx, float* y, int incy)
{
    if (n <= 0 || *alpha == 0.f) return ICLBLAS_STATUS_SUCCESS;
    vparams p = { P_N | P_X | P_INCX | P_Y | P_INCY, .n = n, .x = x, .incx = incx, .y = y, .incy = incy };
    CHECK(p, h);
    orc_saxpy(n, *alpha, x, incx, y, incy);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSnrm2(iclblasHandle_t h, int n, float* x, int incx, float* result)
{
    if (n <= 0 || incx <= 0) { result[0] = 0.f; return ICLBLAS_STATUS_SUCCESS; }
    vparams p = { P_N | P_X | P_INCX, .n = n, .x = x, .incx = incx };
    CHECK(p, h);
    *result = orc_snrm2(n, x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasIsamax(iclblasHandle_t h, int n, float* x, int incx, int* result)
{
    if (n <= 0 || incx <= 0) { *result = 0; return ICLBLAS_STATUS_SUCCESS; }
    vparams p = { P_N | P_X | P_INCX, .n = n, .x = x, .incx = incx };
    CHECK(p, h);
    *result = orc_isamax(n, x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSasum(iclblasHandle_t h, int n, float* x, int incx, float* result)
{
    if (n <= 0 || incx <= 0) { result[0] = 0.f; return ICLBLAS_STATUS_SUCCESS; }
    vparams p = { P_N | P_X | P_INCX, .n = n, .x = x, .incx = incx };
    CHECK(p, h);
    *result = orc_sasum(n, x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSdot(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy, float* result)
{
    if (n <= 0) return ICLBLAS_STATUS_SUCCESS;
    vparams p = { P_N | P_X | P_INCX | P_Y | P_INCY, .n = n, .x = x, .incx = incx, .y = y, .incy = incy };
    CHECK(p, h);
    *result = orc_sdot(n, x, incx, y, incy);
    return ICLBLAS_STATUS_SUCCESS;
}

/* ---- level 1, complex (iclBLAS_C.cpp:69-307) ---- */
iclblasStatus_t iclblasCscal(iclblasHandle_t h, int n, const oclComplex_t* alpha, oclComplex_t* x, int incx)
{
    vparams p = { P_N | P_X | P_INCX, .n = n, .x = x, .incx = incx };
    CHECK(p, h);
    orc_cscal(n, c32(alpha), (orc_c32*)x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCsscal(iclblasHandle_t h, int n, const float* alpha, oclComplex_t* x, int incx)
{
    vparams p = { P_N | P_X | P_INCX, .n = n, .x = x, .incx = incx };
    CHECK(p, h);
    orc_c32 a = { *alpha, 0.f };
    orc_cscal(n, a, (orc_c32*)x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCdotu(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy, oclComplex_t* result)
{
    if (n <= 0) { result->val[0] = 0.f; result->val[1] = 0.f; return ICLBLAS_STATUS_SUCCESS; }
    vparams p = { P_N | P_X | P_INCX | P_Y | P_INCY, .n = n, .x = x, .incx = incx, .y = y, .incy = incy };
    CHECK(p, h);
    orc_c32 r = orc_cdot(n, (const orc_c32*)x, incx, (const orc_c32*)y, incy, 0);
    result->val[0] = r.re; result->val[1] = r.im;
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCdotc(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy, oclComplex_t* result)
{
    if (n <= 0) { result->val[0] = 0.f; result->val[1] = 0.f; return ICLBLAS_STATUS_SUCCESS; }
    vparams p = { P_N | P_X | P_INCX | P_Y | P_INCY, .n = n, .x = x, .incx = incx, .y = y, .incy = incy };
    CHECK(p, h);
    orc_c32 r = orc_cdot(n, (const orc_c32*)x, incx, (const orc_c32*)y, incy, 1);
    result->val[0] = r.re; result->val[1] = r.im;
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasScnrm2(iclblasHandle_t h, int n, oclComplex_t* x, int incx, float* result)
{
    if (n <= 0 || incx <= 0) { *result = 0.f; return ICLBLAS_STATUS_SUCCESS; }
    vparams p = { P_N | P_X | P_INCX, .n = n, .x = x, .incx = incx };
    CHECK(p, h);
    *result = orc_scnrm2(n, (const orc_c32*)x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasScasum(iclblasHandle_t h, int n, oclComplex_t* x, int incx, float* result)
{
    /* no early return in the reference (iclBLAS_C.cpp:112-118) */
    vparams p = { P_N | P_X | P_INCX, .n = n, .x = x, .incx = incx };
    CHECK(p, h);
    *result = orc_scasum(n, (const orc_c32*)x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasIcamax(iclblasHandle_t h, int n, oclComplex_t* x, int incx, int* result)
{
    if (n <= 0 || incx <= 0) { *result = 0; return ICLBLAS_STATUS_SUCCESS; }
    vparams p = { P_N | P_X | P_INCX, .n = n, .x = x, .incx = incx };
    CHECK(p, h);
    *result = orc_icamax(n, (const orc_c32*)x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCaxpy(iclblasHandle_t h, int n, const oclComplex_t* alpha, oclComplex_t* x, int incx, oclComplex_t* y, int incy)
{
    if (n <= 0 || (alpha->val[0] == 0.f && alpha->val[1] == 0.f)) return ICLBLAS_STATUS_SUCCESS;
    vparams p = { P_N | P_X | P_INCX | P_Y | P_INCY, .n = n, .x = x, .incx = incx, .y = y, .incy = incy };
    CHECK(p, h);
    orc_caxpy(n, c32(alpha), (const orc_c32*)x, incx, (orc_c32*)y, incy);
    return ICLBLAS_STATUS_SUCCESS;
}

/* ---- level 2 ---- */
iclblasStatus_t iclblasStrsv(iclblasHandle_t h, iclblasFillMode_t uplo, iclblasOperation_t trans, iclblasDiagType_t diag,
                             int n, float* A, int lda, float* x, int incx)
{
    if (n == 0) return ICLBLAS_STATUS_SUCCESS;
    if (n < 0 || incx == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    vparams p = { P_N | P_A | P_LDA | P_X | P_INCX, .n = n, .A = A, .lda = lda, .x = x, .incx = incx };
    CHECK(p, h);
    orc_strsv(uplo, trans, diag, n, A, lda, x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCtrsv(iclblasHandle_t h, iclblasFillMode_t uplo, iclblasOperation_t trans, iclblasDiagType_t diag,
                             int n, oclComplex_t* A, int lda, oclComplex_t* x, int incx)
{
    if (n == 0) return ICLBLAS_STATUS_SUCCESS;
    if (n < 0 || incx == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    vparams p = { P_N | P_A | P_LDA | P_X | P_INCX, .n = n, .A = A, .lda = lda, .x = x, .incx = incx };
    CHECK(p, h);
    orc_ctrsv(uplo, trans, diag, n, (const orc_c32*)A, lda, (orc_c32*)x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSgemv(iclblasHandle_t h, iclblasOperation_t trans, int m, int n, const float* alpha,
                             float* A, int lda, float* x, int incx, const float* beta, float* y, int incy)
{
    if (m == 0 || n == 0 || (*alpha == 0.f && *beta == 1.f)) return ICLBLAS_STATUS_SUCCESS;
    if (m < 0 || n < 0 || incx == 0 || incy == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    vparams p = { P_N | P_M | P_A | P_LDA | P_X | P_INCX | P_Y | P_INCY,
                  .n = n, .m = m, .A = A, .lda = lda, .x = x, .incx = incx, .y = y, .incy = incy };
    CHECK(p, h);
    orc_sgemv(trans, m, n, *alpha, A, lda, x, incx, *beta, y, incy);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCgemv(iclblasHandle_t h, iclblasOperation_t trans, int m, int n, const oclComplex_t* alpha,
                             oclComplex_t* A, int lda, oclComplex_t* x, int incx, const oclComplex_t* beta,
                             oclComplex_t* y, int incy)
{
    int alpha_zero = alpha->val[0] == 0.f && alpha->val[1] == 0.f;
    int beta_one = beta->val[0] == 1.f && beta->val[1] == 0.f;
    if (m == 0 || n == 0 || (alpha_zero && beta_one)) return ICLBLAS_STATUS_SUCCESS;
    if (m < 0 || n < 0 || incx == 0 || incy == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    vparams p = { P_N | P_M | P_A | P_LDA | P_X | P_INCX | P_Y | P_INCY,
                  .n = n, .m = m, .A = A, .lda = lda, .x = x, .incx = incx, .y = y, .incy = incy };
    CHECK(p, h);
    orc_cgemv(trans, m, n, c32(alpha), (const orc_c32*)A, lda, (const orc_c32*)x, incx, c32(beta), (orc_c32*)y, incy);
    return ICLBLAS_STATUS_SUCCESS;
}

/* ---- level 3 ---- */
iclblasStatus_t iclblasSgemm(iclblasHandle_t h, iclblasOperation_t transa, iclblasOperation_t transb, int m, int n, int k,
                             const float* alpha, float* A, int lda, float* B, int ldb, const float* beta, float* C, int ldc)
{
    if (m < 0 || n < 0 || k < 0) return ICLBLAS_STATUS_INVALID_VALUE;
    vparams p = { P_N | P_M | P_K | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC,
                  .n = n, .m = m, .k = k, .A = A, .lda = lda, .B = B, .ldb = ldb, .C = C, .ldc = ldc };
    CHECK(p, h);
    orc_sgemm(transa, transb, m, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCgemm(iclblasHandle_t h, iclblasOperation_t transa, iclblasOperation_t transb, int m, int n, int k,
                             const oclComplex_t* alpha, oclComplex_t* A, int lda, oclComplex_t* B, int ldb,
                             const oclComplex_t* beta, oclComplex_t* C, int ldc)
{
    if (m < 0 || n < 0 || k < 0) return ICLBLAS_STATUS_INVALID_VALUE;
    vparams p = { P_N | P_M | P_K | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC,
                  .n = n, .m = m, .k = k, .A = A, .lda = lda, .B = B, .ldb = ldb, .C = C, .ldc = ldc };
    CHECK(p, h);
    orc_cgemm(transa, transb, m, n, k, c32(alpha), (const orc_c32*)A, lda, (const orc_c32*)B, ldb, c32(beta),
              (orc_c32*)C, ldc);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasStrsm(iclblasHandle_t h, iclblasSideMode_t side, iclblasFillMode_t uplo, iclblasOperation_t trans,
                             iclblasDiagType_t diag, int m, int n, const float* alpha, float* A, int lda, float* B, int ldb)
{
    if (m == 0 || n == 0) return ICLBLAS_STATUS_SUCCESS;
    vparams p = { P_N | P_M | P_A | P_LDA | P_B | P_LDB, .n = n, .m = m, .A = A, .lda = lda, .B = B, .ldb = ldb };
    CHECK(p, h);
    orc_strsm(side, uplo, trans, diag, m, n, *alpha, A, lda, B, ldb);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCtrsm(iclblasHandle_t h, iclblasSideMode_t side, iclblasFillMode_t uplo, iclblasOperation_t trans,
                             iclblasDiagType_t diag, int m, int n, const oclComplex_t* alpha, oclComplex_t* A, int lda,
                             oclComplex_t* B, int ldb)
{
    if (m == 0 || n == 0) return ICLBLAS_STATUS_SUCCESS;
    vparams p = { P_N | P_M | P_A | P_LDA | P_B | P_LDB, .n = n, .m = m, .A = A, .lda = lda, .B = B, .ldb = ldb };
    CHECK(p, h);
    orc_ctrsm(side, uplo, trans, diag, m, n, c32(alpha), (const orc_c32*)A, lda, (orc_c32*)B, ldb);
    return ICLBLAS_STATUS_SUCCESS;
}

/* ---- level 1: iamin, copy, swap, rotations (iclBLAS_S.cpp:54-62, 101-246;
 *      iclBLAS_C.cpp:58-95, 151-190, 309-333) ---- */
iclblasStatus_t iclblasIsamin(iclblasHandle_t h, int n, float* x, int incx, int* result)
{
    if (n <= 0 || incx <= 0) { *result = 0; return ICLBLAS_STATUS_SUCCESS; }
    vparams p = { P_N | P_X | P_INCX, .n = n, .x = x, .incx = incx };
    CHECK(p, h);
    *result = orc_isamin(n, x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasIcamin(iclblasHandle_t h, int n, oclComplex_t* x, int incx, int* result)
{
    if (n <= 0 || incx <= 0) { *result = 0; return ICLBLAS_STATUS_SUCCESS; }
    vparams p = { P_N | P_X | P_INCX, .n = n, .x = x, .incx = incx };
    CHECK(p, h);
    *result = orc_icamin(n, (const orc_c32*)x, incx);
    return ICLBLAS_STATUS_SUCCESS;
}

static iclblasStatus_t pair_check(iclblasHandle_t h, int n, const void* x, int incx, const void* y, int incy)
{
    vparams p = { P_N | P_X | P_INCX | P_Y | P_INCY, .n = n, .x = x, .incx = incx, .y = y, .incy = incy };
    int v = validate(&p, h);
    return v == 1 ? ICLBLAS_STATUS_SUCCESS : (iclblasStatus_t)v;
}
#define PAIR(h, n, x, incx, y, incy) do { if ((n) <= 0) return ICLBLAS_STATUS_SUCCESS; \
    iclblasStatus_t s_ = pair_check(h, n, x, incx, y, incy); if (s_) return s_; } while (0)

iclblasStatus_t iclblasScopy(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy)
{
    PAIR(h, n, x, incx, y, incy);
    orc_copy(n, x, incx, y, incy, (int)sizeof(float));
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCcopy(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy)
{
    PAIR(h, n, x, incx, y, incy);
    orc_copy(n, x, incx, y, incy, (int)sizeof(oclComplex_t));
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSswap(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy)
{
    PAIR(h, n, x, incx, y, incy);
    orc_swap(n, x, incx, y, incy, (int)sizeof(float));
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCswap(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy)
{
    PAIR(h, n, x, incx, y, incy);
    orc_swap(n, x, incx, y, incy, (int)sizeof(oclComplex_t));
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSrot(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy, float c, float s)
{
    if (c == 1.f && s == 0.f) return ICLBLAS_STATUS_SUCCESS;
    PAIR(h, n, x, incx, y, incy);
    orc_srot(n, x, incx, y, incy, c, s);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSrotm(iclblasHandle_t h, int n, float* x, int incx, float* y, int incy, float* param)
{
    if (n <= 0 || param[0] == -2.f) return ICLBLAS_STATUS_SUCCESS;
    PAIR(h, n, x, incx, y, incy);
    orc_srotm(n, x, incx, y, incy, param);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCrot(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy,
                            const float* c, const oclComplex_t* s)
{
    if (n <= 0 || (*c == 1.f && s->val[0] == 0.f && s->val[1] == 0.f)) return ICLBLAS_STATUS_SUCCESS;
    PAIR(h, n, x, incx, y, incy);
    orc_crot(n, (orc_c32*)x, incx, (orc_c32*)y, incy, *c, c32(s));
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCsrot(iclblasHandle_t h, int n, oclComplex_t* x, int incx, oclComplex_t* y, int incy,
                             const float* c, const float* s)
{
    if (n <= 0 || (*c == 1.f && *s == 0.f)) return ICLBLAS_STATUS_SUCCESS;
    PAIR(h, n, x, incx, y, incy);
    orc_csrot(n, (orc_c32*)x, incx, (orc_c32*)y, incy, *c, *s);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSrotg(iclblasHandle_t h, float* a, float* b, float* c, float* s)
{
    if (!h || h->tag != ORC_TAG || !a || !b || !c || !s) return ICLBLAS_STATUS_INVALID_VALUE;
    orc_srotg(a, b, c, s);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCrotg(iclblasHandle_t h, oclComplex_t* a, oclComplex_t* b, float* c, oclComplex_t* s)
{
    if (!h || h->tag != ORC_TAG || !a || !b || !c || !s) return ICLBLAS_STATUS_INVALID_VALUE;
    orc_crotg((orc_c32*)a, (orc_c32*)b, c, (orc_c32*)s);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSrotmg(iclblasHandle_t h, float* d1, float* d2, float* x1, const float* y1, float* param)
{
    if (!h || h->tag != ORC_TAG || !d1 || !d2 || !x1 || !y1 || !param) return ICLBLAS_STATUS_INVALID_VALUE;
    orc_srotmg(d1, d2, x1, *y1, param);
    return ICLBLAS_STATUS_SUCCESS;
}

/* ---- rank-1 updates and symmetric / Hermitian products (iclBLAS_S.cpp,
 *      iclBLAS_C.cpp: Sger, Ssymv, Cgeru, Cgerc, Chemv) ---- */
iclblasStatus_t iclblasSger(iclblasHandle_t h, int m, int n, const float* alpha, float* x, int incx, float* y, int incy,
                            float* A, int lda)
{
    if (m == 0 || n == 0 || *alpha == 0.f) return ICLBLAS_STATUS_SUCCESS;
    if (m < 0 || n < 0 || incx == 0 || incy == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    vparams p = { P_N | P_M | P_X | P_INCX | P_Y | P_INCY | P_A | P_LDA, .n = n, .m = m, .incx = incx, .incy = incy,
                  .lda = lda, .x = x, .y = y, .A = A };
    CHECK(p, h);
    orc_sger(m, n, *alpha, x, incx, y, incy, A, lda);
    return ICLBLAS_STATUS_SUCCESS;
}

static iclblasStatus_t cger_orc(iclblasHandle_t h, int conj, int m, int n, const oclComplex_t* alpha, oclComplex_t* x,
                                int incx, oclComplex_t* y, int incy, oclComplex_t* A, int lda)
{
    if (m == 0 || n == 0 || (alpha->val[0] == 0.f && alpha->val[1] == 0.f)) return ICLBLAS_STATUS_SUCCESS;
    if (m < 0 || n < 0 || incx == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    vparams p = { P_N | P_M | P_X | P_INCX | P_Y | P_INCY | P_A | P_LDA, .n = n, .m = m, .incx = incx, .incy = incy,
                  .lda = lda, .x = x, .y = y, .A = A };
    CHECK(p, h);
    orc_cger(conj, m, n, c32(alpha), (const orc_c32*)x, incx, (const orc_c32*)y, incy, (orc_c32*)A, lda);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasCgeru(iclblasHandle_t h, int m, int n, const oclComplex_t* alpha, oclComplex_t* x, int incx,
                             oclComplex_t* y, int incy, oclComplex_t* A, int lda)
{
    return cger_orc(h, 0, m, n, alpha, x, incx, y, incy, A, lda);
}

iclblasStatus_t iclblasCgerc(iclblasHandle_t h, int m, int n, const oclComplex_t* alpha, oclComplex_t* x, int incx,
                             oclComplex_t* y, int incy, oclComplex_t* A, int lda)
{
    return cger_orc(h, 1, m, n, alpha, x, incx, y, incy, A, lda);
}

iclblasStatus_t iclblasSsymv(iclblasHandle_t h, iclblasFillMode_t uplo, int n, const float* alpha, float* A, int lda,
                             float* x, int incx, const float* beta, float* y, int incy)
{
    if (n == 0 || (*alpha == 0.f && *beta == 1.f)) return ICLBLAS_STATUS_SUCCESS;
    if (n < 0 || incx == 0 || incy == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    vparams p = { P_N | P_X | P_INCX | P_Y | P_INCY | P_A | P_LDA, .n = n, .incx = incx, .incy = incy, .lda = lda,
                  .x = x, .y = y, .A = A };
    CHECK(p, h);
    orc_ssymv(uplo, n, *alpha, A, lda, x, incx, *beta, y, incy);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasChemv(iclblasHandle_t h, iclblasFillMode_t uplo, int n, const oclComplex_t* alpha,
                             oclComplex_t* A, int lda, oclComplex_t* x, int incx, const oclComplex_t* beta,
                             oclComplex_t* y, int incy)
{
    if (n == 0 || (alpha->val[0] == 0.f && alpha->val[1] == 0.f && beta->val[0] == 1.f && beta->val[1] == 0.f))
        return ICLBLAS_STATUS_SUCCESS;
    if (n < 0 || incx == 0 || incy == 0) return ICLBLAS_STATUS_INVALID_VALUE;
    vparams p = { P_N | P_X | P_INCX | P_Y | P_INCY | P_A | P_LDA, .n = n, .incx = incx, .incy = incy, .lda = lda,
                  .x = x, .y = y, .A = A };
    CHECK(p, h);
    orc_chemv(uplo, n, c32(alpha), (const orc_c32*)A, lda, (const orc_c32*)x, incx, c32(beta), (orc_c32*)y, incy);
    return ICLBLAS_STATUS_SUCCESS;
}

/* ---- level 3 (iclBLAS_S.cpp: Ssymm, Ssyrk, Ssyr2k, Strmm) ---- */
iclblasStatus_t iclblasSsyrk(iclblasHandle_t h, iclblasFillMode_t uplo, iclblasOperation_t trans, int n, int k,
                             const float* alpha, float* A, int lda, const float* beta, float* C, int ldc)
{
    if (n == 0 || k == 0 || (*alpha == 0.f && *beta == 1.f)) return ICLBLAS_STATUS_SUCCESS;
    vparams p = { P_N | P_K | P_A | P_LDA | P_C | P_LDC, .n = n, .k = k, .lda = lda, .ldc = ldc, .A = A, .C = C };
    CHECK(p, h);
    orc_ssyrk(uplo, trans != ICLBLAS_OP_N, n, k, *alpha, A, lda, *beta, C, ldc);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSsyr2k(iclblasHandle_t h, iclblasFillMode_t uplo, iclblasOperation_t trans, int n, int k,
                              const float* alpha, float* A, int lda, float* B, int ldb, const float* beta, float* C,
                              int ldc)
{
    if (n == 0 || k == 0 || (*alpha == 0.f && *beta == 1.f)) return ICLBLAS_STATUS_SUCCESS;
    vparams p = { P_N | P_K | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC, .n = n, .k = k, .lda = lda, .ldb = ldb,
                  .ldc = ldc, .A = A, .B = B, .C = C };
    CHECK(p, h);
    orc_ssyr2k(uplo, trans != ICLBLAS_OP_N, n, k, *alpha, A, lda, B, ldb, *beta, C, ldc);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasSsymm(iclblasHandle_t h, iclblasSideMode_t side, iclblasFillMode_t uplo, int m, int n,
                             const float* alpha, float* A, int lda, float* B, int ldb, const float* beta, float* C,
                             int ldc)
{
    if (n == 0 || m == 0 || (*alpha == 0.f && *beta == 1.f)) return ICLBLAS_STATUS_SUCCESS;
    vparams p = { P_N | P_M | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC, .n = n, .m = m, .lda = lda, .ldb = ldb,
                  .ldc = ldc, .A = A, .B = B, .C = C };
    CHECK(p, h);
    orc_ssymm(side, uplo, m, n, *alpha, A, lda, B, ldb, *beta, C, ldc);
    return ICLBLAS_STATUS_SUCCESS;
}

iclblasStatus_t iclblasStrmm(iclblasHandle_t h, iclblasSideMode_t side, iclblasFillMode_t uplo,
                             iclblasOperation_t transa, iclblasDiagType_t diag, int m, int n, const float* alpha,
                             float* A, int lda, float* B, int ldb, float* C, int ldc)
{
    vparams p = { P_N | P_M | P_A | P_LDA | P_B | P_LDB | P_C | P_LDC, .n = n, .m = m, .lda = lda, .ldb = ldb,
                  .ldc = ldc, .A = A, .B = B, .C = C };
    CHECK(p, h);
    orc_strmm(side, uplo, transa, diag, m, n, *alpha, A, lda, B, ldb, C, ldc);
    return ICLBLAS_STATUS_SUCCESS;
}
