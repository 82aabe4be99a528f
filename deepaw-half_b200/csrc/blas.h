// Typed GEMM entry used by the solvers.  Complex FP64 (the FP64 mode and the
// refinement phase) maps to cuBLAS ZGEMM, the reference's own call
// (src/half_cuda_iterative_solver.cuf:163-194); complex FP32 (the mixed
// mode's iterations) runs on the library's tcgen05 kernel with in-kernel
// bf16 hi/lo splitting (tc_gemm.cu).  Environment HALF_TC_GEMM=0 sends the
// FP32 products to cuBLAS CGEMM instead, for A/B measurements.
#pragma once

#include "context.h"
#include "tc_gemm.h"

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

inline void gemm(Runtime& rt, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, float2 alpha,
                 const float2* A, long long lda, const float2* B, long long ldb, float2 beta, float2* C,
                 long long ldc) {
  if (m <= 0 || n <= 0) return;
  if (rt.tc_gemm) {
    tc_cgemm(rt, tc_dense_a(ta, A, lda, m, k), tc_dense_b(tb, B, ldb, k, n), m, n, k,
             make_double2(alpha.x, alpha.y), make_double2(beta.x, beta.y), C, false, ldc);
    return;
  }
  cublas_check(cublasCgemm(rt.blas, ta, tb, m, n, k, reinterpret_cast<const cuComplex*>(&alpha),
                           reinterpret_cast<const cuComplex*>(A), int(lda), reinterpret_cast<const cuComplex*>(B),
                           int(ldb), reinterpret_cast<const cuComplex*>(&beta), reinterpret_cast<cuComplex*>(C),
                           int(ldc)),
               "cgemm");
}

// Complex FP32 product written as complex FP64 (the FP32 phase's projected
// matrices, which feed the FP64 small eigensolves).
inline void gemm_to64(Runtime& rt, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
                      const float2* A, long long lda, const float2* B, long long ldb, double2* C, long long ldc) {
  if (m <= 0 || n <= 0) return;
  tc_cgemm(rt, tc_dense_a(ta, A, lda, m, k), tc_dense_b(tb, B, ldb, k, n), m, n, k, make_double2(1, 0),
           make_double2(0, 0), C, true, ldc);
}

template <typename R>
inline cplx_t<R> cval(double x, double y = 0) {
  cplx_t<R> c;
  c.x = R(x);
  c.y = R(y);
  return c;
}

}  // namespace hb
