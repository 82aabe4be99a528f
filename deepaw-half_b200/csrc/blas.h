// Thin typed wrappers over the cuBLAS / cuSOLVER calls the solvers make.
// Complex FP64 maps to Z routines; complex FP32 to C routines (with cuBLAS's
// BF16x9 math mode) or, for large products, to the split BF16 path.
#pragma once

#include "context.h"

namespace hb {

inline void gemm(Runtime& rt, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, double2 alpha,
                 const double2* A, long long lda, const double2* B, long long ldb, double2 beta, double2* C,
                 long long ldc) {
  if (m <= 0 || n <= 0) return;
  cublas_check(cublasZgemm(rt.blas, ta, tb, m, n, k, reinterpret_cast<const cuDoubleComplex*>(&alpha),
                           reinterpret_cast<const cuDoubleComplex*>(A), int(lda),
                           reinterpret_cast<const cuDoubleComplex*>(B), int(ldb),
                           reinterpret_cast<const cuDoubleComplex*>(&beta), reinterpret_cast<cuDoubleComplex*>(C),
                           int(ldc)),
               "zgemm");
}

void gemm_c32_split(Runtime& rt, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, float2 alpha,
                    const float2* A, long long lda, const float2* B, long long ldb, float2 beta, float2* C,
                    long long ldc);   // blas_split.cu

// Complex FP32: GEMMs of at least 5e9 complex multiply-adds go to the split
// BF16 tensor-core path (blas_split.cu); smaller ones to CGEMM.
inline void gemm(Runtime& rt, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, float2 alpha,
                 const float2* A, long long lda, const float2* B, long long ldb, float2 beta, float2* C,
                 long long ldc) {
  if (m <= 0 || n <= 0) return;
  if (rt.tc_split && k > 0 && double(m) * n * k >= 5e9) {
    gemm_c32_split(rt, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    return;
  }
  cublas_check(cublasCgemm(rt.blas, ta, tb, m, n, k, reinterpret_cast<const cuComplex*>(&alpha),
                           reinterpret_cast<const cuComplex*>(A), int(lda), reinterpret_cast<const cuComplex*>(B),
                           int(ldb), reinterpret_cast<const cuComplex*>(&beta), reinterpret_cast<cuComplex*>(C),
                           int(ldc)),
               "cgemm");
}

template <typename R>
inline cplx_t<R> cval(double x, double y = 0) {
  cplx_t<R> c;
  c.x = R(x);
  c.y = R(y);
  return c;
}

}  // namespace hb
