// Reciprocal-space indexing of the full charge box, shared by the set-up and
// ion-force kernels.  Box index i = (i1 * n2 + i2) * n3 + i3 (C order); the
// integer frequencies follow the reference's fft_integer
// (src/half_local_forces.F90:209-212): i <= (n-1)/2 -> i, else i - n.
#pragma once

#include "common.h"

namespace hb {

struct Grid3 {
  int n1, n2, n3;
  double rec[9];   // reciprocal rows b_i (2 pi inv(lattice)^T), A^-1
  __host__ __device__ long long size() const { return (long long)n1 * n2 * n3; }
};

__device__ __forceinline__ void gvector(long long idx, const Grid3& g, double& qx, double& qy, double& qz) {
  int i3 = int(idx % g.n3);
  long long t = idx / g.n3;
  int i2 = int(t % g.n2);
  int i1 = int(t / g.n2);
  int k1 = i1 <= (g.n1 - 1) / 2 ? i1 : i1 - g.n1;
  int k2 = i2 <= (g.n2 - 1) / 2 ? i2 : i2 - g.n2;
  int k3 = i3 <= (g.n3 - 1) / 2 ? i3 : i3 - g.n3;
  qx = k1 * g.rec[0] + k2 * g.rec[3] + k3 * g.rec[6];
  qy = k1 * g.rec[1] + k2 * g.rec[4] + k3 * g.rec[7];
  qz = k1 * g.rec[2] + k2 * g.rec[5] + k3 * g.rec[8];
}

inline int blocks_for(long long n, int t = 256) { return int((n + t - 1) / t); }

}  // namespace hb
