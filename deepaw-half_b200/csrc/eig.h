// Device-resident small Hermitian eigensolvers (see eig.cu).
#pragma once

#include <vector>

#include "context.h"

namespace hb {

struct SmallEigen {
  // Orders the one-CTA kernels serve; above it cuSOLVER's zhegvd is faster
  // (order 320: 4.7 against 5.9 ms; order 1080: 20 against 37 ms).
  static constexpr int kOwnMaxOrder = 164;
  int cap = 0;
  DeviceBuffer<double> d, e, Z, scratch, lam;
  DeviceBuffer<double2> tau, V, work;
  DeviceBuffer<int> info;   // zhetrd status (reports illegal arguments only)
  void reserve(Runtime& rt, int nmax);
  // A (n x n, upper triangle) -> nev lowest eigenpairs; vectors overwrite
  // A[:, :nev].  *status (device) becomes nonzero if inverse iteration failed.
  void heev(Runtime& rt, double2* A, int n, int nev, double* w, int* status);
  // A y = lambda B y, B Hermitian positive definite; Y^H B Y = I.
  // *chol_status (device) is zpotrf's info (> 0: B not positive definite).
  void hegv(Runtime& rt, double2* A, double2* B, int n, int nev, double* w, int* status, int* chol_status);
  // ACC correction metric: M = P^H S P (m x m) -> U, upper triangular, with
  // (P U)^H S (P U) = I; returns false (nothing launched) when m is too large.
  bool metric_normalize(Runtime& rt, double2* M, int m, int* status);
};

// Selected eigenvalues of a large Hermitian matrix A (n x n, column-major,
// upper triangle used and destroyed): Householder tridiagonalisation
// (cuSOLVER zhetrd), then multisection on Sturm counts for the index ranges
// [k0s[r], k0s[r] + counts[r]), written one range after another to lam
// (device).  Synchronises the stream.
void hermitian_eigenvalues_large(Runtime& rt, double2* A, long long n, const std::vector<int>& k0s,
                                 const std::vector<int>& counts, double* lam);

}  // namespace hb
