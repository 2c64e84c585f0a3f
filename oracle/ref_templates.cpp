// Reference CPU oracles compiled from their own sources -- TEST INFRASTRUCTURE.
//
// Wraps the reference's header-only CPU templates (tests/blas_funcs/*.hpp)
// and tests/blas_reference/blas_reference.cpp behind extern "C" entry points
// so that the oracle restatement (oracle.c) can be checked against them and
// the CPU baseline can time the reference's own code.  Built only by
// oracle/Makefile into oracle/_ref/, from the files where they lie in the
// clGPU tree; nothing here is a copy of them.
#include <complex>
#include "test_gemm.hpp"
#include "test_dot.hpp"
#include "test_nrm2.hpp"
#include "test_asum.hpp"
#include "test_axpy.hpp"
#include "test_scal.hpp"
#include "test_amax.hpp"
#include "test_symv.hpp"

using cf = std::complex<float>;
using namespace iclgpu::tests;

extern "C" {

void ref_cpu_sgemm(int ta, int tb, int m, int n, int k, float alpha, const float* A, int lda,
                   const float* B, int ldb, float beta, float* C, int ldc)
{
    cpu_gemm<float>((iclblasOperation_t)ta, (iclblasOperation_t)tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

// cpu_gemm in double with a double accumulator: ties the FP64 products used
// as the error reference of the precision studies to the reference's GEMM.
void ref_cpu_dgemm(int ta, int tb, int m, int n, int k, double alpha, const double* A, int lda,
                   const double* B, int ldb, double beta, double* C, int ldc)
{
    cpu_gemm<double, double>((iclblasOperation_t)ta, (iclblasOperation_t)tb, m, n, k, alpha, A, lda, B, ldb, beta, C,
                             ldc);
}

void ref_cpu_cgemm(int ta, int tb, int m, int n, int k, const float* alpha, const float* A, int lda,
                   const float* B, int ldb, const float* beta, float* C, int ldc)
{
    cpu_gemm<cf>((iclblasOperation_t)ta, (iclblasOperation_t)tb, m, n, k, cf(alpha[0], alpha[1]),
                 (const cf*)A, lda, (const cf*)B, ldb, cf(beta[0], beta[1]), (cf*)C, ldc);
}

float ref_cpu_sdot(int n, const float* x, int incx, const float* y, int incy)
{
    float r = 0.f;
    cpu_dot<float>(n, x, incx, y, incy, &r);
    return r;
}

void ref_cpu_cdot(int n, const float* x, int incx, const float* y, int incy, int conj, float* out)
{
    cf r;
    if (conj) cpu_dot<cf, true>(n, (const cf*)x, incx, (const cf*)y, incy, &r);
    else cpu_dot<cf, false>(n, (const cf*)x, incx, (const cf*)y, incy, &r);
    out[0] = r.real();
    out[1] = r.imag();
}

float ref_cpu_snrm2(int n, const float* x, int incx) { float r; cpu_nrm2<float>(n, x, incx, &r); return r; }
float ref_cpu_scnrm2(int n, const float* x, int incx) { float r; cpu_nrm2<cf>(n, (const cf*)x, incx, &r); return r; }
float ref_cpu_sasum(int n, const float* x, int incx) { float r; cpu_asum<float>(n, x, incx, &r); return r; }
float ref_cpu_scasum(int n, const float* x, int incx) { float r; cpu_asum<cf>(n, (const cf*)x, incx, &r); return r; }

void ref_cpu_saxpy(int n, float alpha, const float* x, int incx, float* y, int incy)
{
    cpu_axpy<float>(n, alpha, x, incx, y, incy);
}

// Caxpy_reference (tests/blas_reference/blas_reference.cpp:38-43)
void ref_caxpy_reference(int n, const float* alpha, float* x, int incx, float* y, int incy)
{
    Caxpy_reference(n, cf(alpha[0], alpha[1]), array_ref<cf>((cf*)x, (size_t)n * incx), incx,
                    array_ref<cf>((cf*)y, (size_t)n * incy), incy);
}

void ref_cpu_sscal(int n, float alpha, float* x, int incx) { cpu_scal<float, float>(n, alpha, x, incx); }
void ref_cpu_cscal(int n, const float* alpha, float* x, int incx)
{
    cpu_scal<cf, cf>(n, cf(alpha[0], alpha[1]), (cf*)x, incx);
}

// cpu_amax<float> = Isamax_reference - 1 (0-based)
int ref_cpu_isamax(int n, const float* x, int incx) { int r = 0; cpu_amax<float>(n, x, incx, &r); return r; }
int ref_cpu_icamax(int n, const float* x, int incx) { int r = 0; cpu_amax<cf>(n, (const cf*)x, incx, &r); return r; }

// cpu_symv (tests/blas_funcs/test_symv.hpp:21-87), double accumulation
void ref_cpu_ssymv(int uplo, int n, float alpha, const float* A, int lda, const float* x, int incx, float beta, float* y,
                   int incy)
{
    cpu_symv<float>((iclblasFillMode_t)uplo, n, alpha, A, lda, x, incx, beta, y, incy);
}

void ref_cpu_chemv(int uplo, int n, const float* alpha, const float* A, int lda, const float* x, int incx,
                   const float* beta, float* y, int incy)
{
    cpu_symv<cf, true>((iclblasFillMode_t)uplo, n, cf(alpha[0], alpha[1]), (const cf*)A, lda, (const cf*)x, incx,
                       cf(beta[0], beta[1]), (cf*)y, incy);
}

}  // extern "C"
