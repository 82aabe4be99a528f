// Device-resident small Hermitian eigensolvers (see eig.cu).
#pragma once

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

}  // namespace hb
