// The reference's serial OpenCL kernels compiled as C++ -- TEST INFRASTRUCTURE.
//
// Each kernel is #included from its .cl file in the clGPU tree (built by
// oracle/Makefile into oracle/_ref/) behind clshim.hpp and exported with an
// extern "C" wrapper.  They give CPU results of the reference's own GEMV,
// TRSV, TRSM and CGEMM algorithms, which its tests have no template for, and
// of its iamin, rotation and rotation-generator kernels.
#include "clshim.hpp"

namespace ref_sgemv {
#include "Sgemv/Sgemv_naive.cl"
}
#undef MAT_ACCESS
#undef ICLBLAS_OP_N
#undef ICLBLAS_OP_T
#undef ICLBLAS_OP_C
namespace ref_cgemv {
#include "Cgemv/Cgemv_naive.cl"
}
namespace ref_strsv {
#include "Strsv/Strsv_naive.cl"
}
namespace ref_ctrsv {
#include "Ctrsv/Ctrsv_naive.cl"
}
namespace ref_strsm {
#include "Strsm/Strsm_naive.cl"
}
#undef ACCESS
namespace ref_ctrsm {
#include "Ctrsm/Ctrsm_naive.cl"
}
#undef ACCESS
namespace ref_sgemm {
#include "Sgemm/Sgemm_naive.cl"
}
namespace ref_cgemm {
#include "Cgemm/Cgemm_naive.cl"
}

namespace ref_isamin {
#include "Isamin/Isamin_naive.cl"
}
namespace ref_icamin {
#include "Icamin/Icamin_naive.cl"
}
namespace ref_srot {
#include "Srot/Srot_naive.cl"
}
namespace ref_csrot {
#include "Csrot/Csrot_naive.cl"
}
namespace ref_crot {
#include "Crot/Crot_naive.cl"
}
namespace ref_srotm {
#include "Srotm/Srotm_naive.cl"
}
namespace ref_srotg {
#include "Srotg/Srotg_naive.cl"
}
namespace ref_crotg {
#include "Crotg/Crotg_naive.cl"
}
namespace ref_srotmg {
#include "Srotmg/Srotmg_naive.cl"
}

namespace ref_sger {
#include "Sger/Sger_naive.cl"
}
namespace ref_cgeru {
#include "Cgeru/Cgeru_naive.cl"
}
#undef IDX
namespace ref_cgerc {
#include "Cgerc/Cgerc_naive.cl"
}
#undef IDX
namespace ref_ssymv_lower {
#include "Ssymv/Ssymv_naive_lower.cl"
}
#undef MAT_ACCESS
namespace ref_ssymv_upper {
#include "Ssymv/Ssymv_naive_upper.cl"
}
#undef MAT_ACCESS
namespace ref_chemv {
#include "Chemv/Chemv_naive.cl"
}
#undef ACCESS
namespace ref_ssyrk {
#include "Ssyrk/Ssyrk_naive.cl"
}
#undef ACCESS
namespace ref_ssyr2k {
#include "Ssyr2k/Ssyr2k_naive.cl"
}
#undef ACCESS
namespace ref_ssymm {
#include "Ssymm/Ssymm_naive.cl"
}
#undef ACCESS
namespace ref_strmm {
#include "Strmm/Strmm_naive.cl"
}

static complex_t c2(const float* p) { return complex_t(p[0], p[1]); }

extern "C" {

// Sgemv_naive: one work-item runs the whole product (Sgemv_naive.cpp launch of 1)
void ref_naive_sgemv(int trans, int m, int n, float alpha, float* A, int lda, float* x, int incx, float beta,
                     float* y, int incy)
{
    ref_sgemv::Sgemv_naive(trans, m, n, alpha, A, lda, x, incx, beta, y, incy);
}

// Cgemv_naive: one work-item per output element (Cgemv_naive.cpp:66)
void ref_naive_cgemv(int trans, int m, int n, const float* alpha, float* A, int lda, float* x, int incx,
                     const float* beta, float* y, int incy)
{
    size_t gws = (trans == 0) ? (size_t)m : (size_t)n;
    clshim::run_ndrange(gws, [&] {
        ref_cgemv::Cgemv_naive(trans, m, n, c2(alpha), (complex_t*)A, lda, (complex_t*)x, incx, c2(beta),
                               (complex_t*)y, incy);
    });
}

void ref_naive_strsv(int uplo, int trans, int diag, int n, const float* A, int lda, float* x, int incx)
{
    ref_strsv::Strsv_naive(uplo, trans, diag, n, A, lda, x, incx);
}

void ref_naive_ctrsv(int uplo, int trans, int diag, int n, float* A, int lda, float* x, int incx)
{
    ref_ctrsv::Ctrsv_naive(uplo, trans, diag, n, (complex_t*)A, lda, (complex_t*)x, incx);
}

void ref_naive_strsm(int side, int uplo, int trans, int diag, int m, int n, float alpha, float* A, int lda,
                     float* B, int ldb)
{
    ref_strsm::Strsm_naive(side, uplo, trans, diag, m, n, alpha, A, lda, B, ldb);
}

void ref_naive_ctrsm(int side, int uplo, int trans, int diag, int m, int n, const float* alpha, float* A, int lda,
                     float* B, int ldb)
{
    ref_ctrsm::Ctrsm_naive(side, uplo, trans, diag, m, n, c2(alpha), (complex_t*)A, lda, (complex_t*)B, ldb);
}

void ref_naive_sgemm(int ta, int tb, int m, int n, int k, float alpha, float* A, int lda, float* B, int ldb,
                     float beta, float* C, int ldc)
{
    ref_sgemm::Sgemm_naive(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

void ref_naive_cgemm(int ta, int tb, int m, int n, int k, const float* alpha, float* A, int lda, float* B, int ldb,
                     const float* beta, float* C, int ldc)
{
    ref_cgemm::Cgemm_naive(ta, tb, m, n, k, c2(alpha), (complex_t*)A, lda, (complex_t*)B, ldb, c2(beta),
                           (complex_t*)C, ldc);
}

// Level-1 kernels: each one is launched with a single work-item
// (Isamin_naive.cpp, Icamin_naive.cpp, Srot_naive.cpp:45, Crot_naive.cpp:46,
// Csrot_naive.cpp, Srotm_naive.cpp, Srotg_naive.cpp:44, Crotg_naive.cpp:44,
// Srotmg_naive.cpp:45).
int ref_naive_isamin(int n, float* x, int incx)
{
    int r = -1;
    ref_isamin::Isamin_naive(n, x, incx, &r);
    return r;
}

int ref_naive_icamin(int n, float* x, int incx)
{
    int r = -1;
    ref_icamin::Icamin_naive(n, (complex_t*)x, incx, &r);
    return r;
}

void ref_naive_srot(int n, float* x, int incx, float* y, int incy, float c, float s)
{
    ref_srot::Srot_naive((uint)n, x, incx, y, incy, c, s);
}

void ref_naive_csrot(int n, float* x, int incx, float* y, int incy, float c, float s)
{
    ref_csrot::Csrot_naive(n, (complex_t*)x, incx, (complex_t*)y, incy, c, s);
}

void ref_naive_crot(int n, float* x, int incx, float* y, int incy, float c, const float* s)
{
    ref_crot::Crot_naive(n, (complex_t*)x, incx, (complex_t*)y, incy, c, c2(s));
}

void ref_naive_srotm(int n, float* x, int incx, float* y, int incy, float* param)
{
    ref_srotm::Srotm_naive((uint)n, x, (uint)incx, y, (uint)incy, param);
}

void ref_naive_srotg(float* a, float* b, float* c, float* s)
{
    ref_srotg::Srotg_naive(a, b, c, s);
}

// Compare only for a != 0: the a == 0 branch writes an OpenCL vector literal.
void ref_naive_crotg(float* a, float* b, float* c, float* s)
{
    ref_crotg::Crotg_naive((complex_t*)a, (complex_t*)b, c, (complex_t*)s);
}

// The kernel alone; the caller applies the host-side checks of
// iclBLAS_S.cpp:101-128 first.  Inputs whose rescaling loops would not end
// (an infinite d1 or d2) must not be passed.
void ref_naive_srotmg(float* d1, float* d2, float* x1, float y1, float* param)
{
    ref_srotmg::Srotmg_naive(d1, d2, x1, y1, param);
}

// Level-2/3 kernels with their NDRanges: Sger/Cgeru/Cgerc (m, n), Ssymv one
// work-item, Chemv (n), Ssyrk/Ssyr2k (n, n), Ssymm/Strmm (m, n).
void ref_naive_sger(int m, int n, float alpha, float* x, int incx, float* y, int incy, float* A, int lda)
{
    clshim::run_ndrange2(m, n, [&] { ref_sger::Sger_naive(alpha, x, incx, y, incy, A, lda); });
}

void ref_naive_cger(int conj, int m, int n, const float* alpha, float* x, int incx, float* y, int incy, float* A,
                    int lda)
{
    clshim::run_ndrange2(m, n, [&] {
        if (conj)
            ref_cgerc::Cgerc_naive(c2(alpha), (complex_t*)x, incx, (complex_t*)y, incy, (complex_t*)A, lda);
        else
            ref_cgeru::Cgeru_naive(c2(alpha), (complex_t*)x, incx, (complex_t*)y, incy, (complex_t*)A, lda);
    });
}

void ref_naive_ssymv(int uplo, int n, float alpha, float* A, int lda, float* x, int incx, float beta, float* y,
                     int incy)
{
    if (uplo == 1) ref_ssymv_lower::Ssymv_naive_lower(n, alpha, A, lda, x, incx, beta, y, incy);
    else ref_ssymv_upper::Ssymv_naive_upper(n, alpha, A, lda, x, incx, beta, y, incy);
}

void ref_naive_chemv(int uplo, int n, const float* alpha, float* A, int lda, float* x, int incx, const float* beta,
                     float* y, int incy)
{
    clshim::run_ndrange(n, [&] {
        ref_chemv::Chemv_naive(uplo, n, c2(alpha), (complex_t*)A, lda, (complex_t*)x, incx, c2(beta), (complex_t*)y,
                               incy);
    });
}

void ref_naive_ssyr2k(int uplo, int trans, int n, int k, float alpha, float* A, int lda, float* B, int ldb, float beta,
                      float* C, int ldc)
{
    clshim::run_ndrange2(n, n, [&] {
        if (B) ref_ssyr2k::Ssyr2k_naive(uplo, trans, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
        else ref_ssyrk::Ssyrk_naive(uplo, trans, n, k, alpha, A, lda, beta, C, ldc);
    });
}

void ref_naive_ssymm(int side, int uplo, int m, int n, float alpha, float* A, int lda, float* B, int ldb, float beta,
                     float* C, int ldc)
{
    clshim::run_ndrange2(m, n, [&] { ref_ssymm::Ssymm_naive(side, uplo, m, n, alpha, A, lda, B, ldb, beta, C, ldc); });
}

void ref_naive_strmm(int side, int uplo, int transa, int diag, int m, int n, float alpha, float* A, int lda, float* B,
                     int ldb, float* C, int ldc)
{
    clshim::run_ndrange2(m, n, [&] {
        ref_strmm::Strmm_naive(side, uplo, transa, diag, m, n, alpha, A, lda, B, ldb, C, ldc);
    });
}

}  // extern "C"
