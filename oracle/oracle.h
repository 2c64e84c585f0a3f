/*
 * CPU oracle for the iclBLAS hot path (test infrastructure only).
 *
 * This header declares a plain-C restatement of the reference's CPU
 * algorithms for the S/C gemm, gemv, trsv, trsm, dot, nrm2, asum, iamax,
 * axpy and scal routines, and for iamin, copy, swap, rot, rotm, rotg, rotmg.  It is the checker the GPU library is compared
 * against; nothing in the shipped library links it.  Each function names the
 * reference source it restates (paths are relative to the clGPU tree).
 *
 * Conventions (same as the reference): column-major storage, element (i,j)
 * at j*ld+i (libs/blas/funcs/iclblas_common.h.cl:47); positive strides only;
 * complex numbers are two packed floats {re, im}.
 *
 * Arithmetic: like the reference test oracles (tests/blas_funcs/test_*.hpp,
 * accumulator_type<float> = double, tests/blas_funcs/test_helpers.hpp:216-232)
 * every accumulation runs in double and is rounded to float once at the end,
 * except SGEMM, which follows the reference kernels' FP32 FMA order, and the
 * copy/swap/rotation family, which restates the reference kernels' FP32
 * expressions (their fma placement included) exactly.
 */
#ifndef ICLB_ORACLE_H
#define ICLB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float re, im; } orc_c32;

/* ---- level 1, single ---- */
void  orc_saxpy(int n, float alpha, const float* x, int incx, float* y, int incy);
void  orc_sscal(int n, float alpha, float* x, int incx);
float orc_sdot(int n, const float* x, int incx, const float* y, int incy);
float orc_snrm2(int n, const float* x, int incx);
float orc_sasum(int n, const float* x, int incx);
int   orc_isamax(int n, const float* x, int incx);

/* ---- level 1, complex ---- */
void    orc_caxpy(int n, orc_c32 alpha, const orc_c32* x, int incx, orc_c32* y, int incy);
void    orc_cscal(int n, orc_c32 alpha, orc_c32* x, int incx);
orc_c32 orc_cdot(int n, const orc_c32* x, int incx, const orc_c32* y, int incy, int conj_x);
float   orc_scnrm2(int n, const orc_c32* x, int incx);
float   orc_scasum(int n, const orc_c32* x, int incx);
int     orc_icamax(int n, const orc_c32* x, int incx);

/* ---- level 1: iamin, copy, swap, plane rotations ---- */
int   orc_isamin(int n, const float* x, int incx);
int   orc_icamin(int n, const orc_c32* x, int incx);
void  orc_copy(int n, const void* x, int incx, void* y, int incy, int esize);
void  orc_swap(int n, void* x, int incx, void* y, int incy, int esize);
void  orc_srot(int n, float* x, int incx, float* y, int incy, float c, float s);
void  orc_csrot(int n, orc_c32* x, int incx, orc_c32* y, int incy, float c, float s);
void  orc_crot(int n, orc_c32* x, int incx, orc_c32* y, int incy, float c, orc_c32 s);
void  orc_srotm(int n, float* x, int incx, float* y, int incy, const float* param);
void  orc_srotg(float* a, float* b, float* c, float* s);
void  orc_crotg(orc_c32* a, orc_c32* b, float* c, orc_c32* s);
void  orc_srotmg(float* d1, float* d2, float* x1, float y1, float* param);

/* ---- rank-1 updates, symmetric / Hermitian products, level 3 on GEMM ---- */
void orc_sger(int m, int n, float alpha, const float* x, int incx, const float* y, int incy, float* A, int lda);
void orc_cger(int conj, int m, int n, orc_c32 alpha, const orc_c32* x, int incx, const orc_c32* y, int incy,
              orc_c32* A, int lda);
void orc_ssymv(int uplo, int n, float alpha, const float* A, int lda, const float* x, int incx, float beta, float* y,
               int incy);
void orc_chemv(int uplo, int n, orc_c32 alpha, const orc_c32* A, int lda, const orc_c32* x, int incx, orc_c32 beta,
               orc_c32* y, int incy);
void orc_ssyrk(int uplo, int trans, int n, int k, float alpha, const float* A, int lda, float beta, float* C, int ldc);
void orc_ssyr2k(int uplo, int trans, int n, int k, float alpha, const float* A, int lda, const float* B, int ldb,
                float beta, float* C, int ldc);
void orc_ssymm(int side, int uplo, int m, int n, float alpha, const float* A, int lda, const float* B, int ldb,
               float beta, float* C, int ldc);
void orc_strmm(int side, int uplo, int transa, int diag, int m, int n, float alpha, const float* A, int lda,
               const float* B, int ldb, float* C, int ldc);

/* ---- half-precision GEMM (library extension; binary16 bit patterns) ---- */
void orc_hgemm(int transa, int transb, int m, int n, int k, float alpha, const uint16_t* A, int lda,
               const uint16_t* B, int ldb, float beta, uint16_t* C, int ldc);

/* ---- level 2 ---- */
void orc_sgemv(int trans, int m, int n, float alpha, const float* A, int lda,
               const float* x, int incx, float beta, float* y, int incy);
void orc_cgemv(int trans, int m, int n, orc_c32 alpha, const orc_c32* A, int lda,
               const orc_c32* x, int incx, orc_c32 beta, orc_c32* y, int incy);
void orc_strsv(int uplo, int trans, int diag, int n, const float* A, int lda, float* x, int incx);
void orc_ctrsv(int uplo, int trans, int diag, int n, const orc_c32* A, int lda, orc_c32* x, int incx);

/* ---- level 3 ---- */
void orc_sgemm(int transa, int transb, int m, int n, int k, float alpha,
               const float* A, int lda, const float* B, int ldb, float beta, float* C, int ldc);
void orc_cgemm(int transa, int transb, int m, int n, int k, orc_c32 alpha,
               const orc_c32* A, int lda, const orc_c32* B, int ldb, orc_c32 beta, orc_c32* C, int ldc);
void orc_strsm(int side, int uplo, int trans, int diag, int m, int n, float alpha,
               const float* A, int lda, float* B, int ldb);
void orc_ctrsm(int side, int uplo, int trans, int diag, int m, int n, orc_c32 alpha,
               const orc_c32* A, int lda, orc_c32* B, int ldb);

/* FP64 variants used as the error reference for the precision study
 * (double in, double out; same semantics as the float versions). */
void orc_dgemm(int transa, int transb, int m, int n, int k, double alpha,
               const double* A, int lda, const double* B, int ldb, double beta, double* C, int ldc);
void orc_dtrsm(int side, int uplo, int trans, int diag, int m, int n, double alpha,
               const double* A, int lda, double* B, int ldb);

#ifdef __cplusplus
}
#endif
#endif
