// GEMM dispatch by the handle's math mode.
//
// The reference picks among seven SGEMM implementations by summed accept()
// scores (include/iclgpu/functions_base.hpp:164-223); here the routine maps
// directly: PLAIN_FP32 runs the CUDA-core FFMA kernel (bit-identical to the
// reference's FP32 FMA order), the tensor-core modes run the tcgen05 kernel.
#include <cuda_fp16.h>

#include "common.cuh"

namespace iclb {

cudaError_t sgemm_simt(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const float* A, int lda,
                       const float* B, int ldb, float beta, float* C, int ldc, int tri);
cudaError_t cgemm_simt(iclblasHandle_t h, int ta, int tb, int m, int n, int k, cfloat alpha, const cfloat* A, int lda,
                       const cfloat* B, int ldb, cfloat beta, cfloat* C, int ldc);
namespace tc {
cudaError_t hgemm_tc(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const __half* A, int lda,
                     const __half* B, int ldb, float beta, __half* C, int ldc);
template <class T>
cudaError_t gemm_tc(iclblasHandle_t h, int ta, int tb, int m, int n, int k, T alpha, const T* A, int lda, const T* B,
                    int ldb, T beta, T* C, int ldc, int tri);
}

cudaError_t sgemm_tri(iclblasHandle_t h, int tri, int ta, int tb, int m, int n, int k, float alpha, const float* A,
                      int lda, const float* B, int ldb, float beta, float* C, int ldc)
{
    if (m == 0 || n == 0) return cudaSuccess;
    // k == 0 (C = beta*C) needs no products: the CUDA-core kernel handles it in every mode
    if (h->math != ICLBLAS_MATH_PLAIN_FP32 && k > 0)
        return tc::gemm_tc<float>(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri);
    return sgemm_simt(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri);
}

cudaError_t sgemm(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const float* A, int lda,
                  const float* B, int ldb, float beta, float* C, int ldc)
{
    return sgemm_tri(h, 0, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

cudaError_t hgemm(iclblasHandle_t h, int ta, int tb, int m, int n, int k, float alpha, const void* A, int lda,
                  const void* B, int ldb, float beta, void* C, int ldc)
{
    if (m == 0 || n == 0) return cudaSuccess;
    return tc::hgemm_tc(h, ta, tb, m, n, k, alpha, (const __half*)A, lda, (const __half*)B, ldb, beta, (__half*)C,
                        ldc);
}

cudaError_t cgemm(iclblasHandle_t h, int ta, int tb, int m, int n, int k, cfloat alpha, const cfloat* A, int lda,
                  const cfloat* B, int ldb, cfloat beta, cfloat* C, int ldc)
{
    if (m == 0 || n == 0) return cudaSuccess;
    if (h->math != ICLBLAS_MATH_PLAIN_FP32 && k > 0)
        return tc::gemm_tc<cfloat>(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 0);
    return cgemm_simt(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

}  // namespace iclb
