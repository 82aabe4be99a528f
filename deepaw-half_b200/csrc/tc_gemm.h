// Complex FP32 GEMM on the sm_100a tensor cores (tc_gemm.cu).
//
// C = alpha op(A) op(B) + beta C with op(A) M x K and op(B) K x N complex.
// Every operand element is split into bf16 planes, x = x_hi + x_lo
// (x_hi = bf16(x), x_lo = bf16(x - x_hi)), and each real product is taken as
// x_hi y_hi + x_hi y_lo + x_lo y_hi with FP32 accumulation in Tensor Memory
// (relative error about 2^-16).  Operands are dense complex FP32 matrices,
// the projector matrix B of a k point generated from its radial-angular
// table, plane-wave indices and atom phases, or planes split beforehand
// (tc_presplit_a) and reused across products.
#pragma once

#include <climits>

#include "context.h"

namespace hb {

struct TcOperand {
  enum Kind : int {
    kDenseK = 0,      // element (r, k) at p[k + r ld]: k contiguous
    kDenseMN = 1,     // element (r, k) at p[r + k ld]: r contiguous
    kProjConj = 2,    // conj(B[g = k, col = r]): rows = projector columns, k = plane waves
    kProj = 3,        // B[g = r, col = k]: rows = plane waves, k = projector columns
    kPlanes = 4       // pre-split bf16 planes in global memory (tc_presplit_a, or tc_cgemm itself)
  };
  int kind = kDenseK;
  int rows = 0, kdim = 0;
  const float2* p = nullptr;
  const float2* p2 = nullptr;   // dense: rows >= split read p2 at row - split
  int split = INT_MAX;
  long long ld = 0;
  int conj = 0;
  // projector generation: B[g, col] = ftab[frow][g] (-i)^l exp(-2 pi i sum_j (n_j(g) + k_j) f_j(atom))
  const float* ftab = nullptr;  // [frow][npw]: Omega^-1/2 beta_l(|q|) Y_lm(q^)
  const int* gpack = nullptr;   // npw: (n1, n2, n3) as three signed 10-bit fields
  const int* pcol = nullptr;    // per projector column: (atom << 16) | (frow << 2) | l
  const double* afrac = nullptr;   // per atom: (q.R) / (2 pi) = sum_j (n_j + k_j) afrac[3 a + j]
  double kf0 = 0, kf1 = 0, kf2 = 0;
  int npw = 0;
  // kPlanes: plane p (Re hi, Re lo, Im hi, Im lo) at planes + p plane_bytes;
  // k block kb at kb rows_pad 32 bytes, in the tile's shared-memory layout
  const unsigned char* planes = nullptr;
  long long plane_bytes = 0;
  int rows_pad = 0;
};

// op(A) (M x K) and op(B) (K x N) from cuBLAS-style operations on column-major storage.
TcOperand tc_dense_a(cublasOperation_t op, const float2* A, long long lda, int M, int K);
TcOperand tc_dense_b(cublasOperation_t op, const float2* B, long long ldb, int K, int N);

// C (column-major, ldc; complex FP32, or FP64 when c_fp64) = alpha op(A) op(B) + beta C.
// With C2 set, output columns j >= split_col go to C2 column j - split_col (same ldc).
void tc_cgemm(Runtime& rt, const TcOperand& A, const TcOperand& B, int M, int N, int K, double2 alpha,
              double2 beta, void* C, bool c_fp64, long long ldc, void* C2 = nullptr, int split_col = INT_MAX);

// Splits `op`, used as the A operand of later products (M = op.rows,
// K = op.kdim), into bf16 planes in `store` (grown when too small) and
// returns the kPlanes operand that reads them; asynchronous on rt.stream.
TcOperand tc_presplit_a(Runtime& rt, const TcOperand& op, DeviceBuffer<unsigned char>& store);

// Raises kInternal if a tensor-core GEMM on this runtime gave up on a pipeline
// wait (synchronises the stream).
void tc_check(Runtime& rt);

}  // namespace hb
