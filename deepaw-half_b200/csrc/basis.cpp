// Plane-wave basis of one k point (src/half_basis.F90:9-55): the box loop
// n1 -> n2 -> n3 over [-n/2, (n-1)/2], kept when hbar^2/2m |k+G|^2 < ENCUT.
// The G order is ABI-visible through half_get_basis and must match exactly.
#include "context.h"

namespace hb {

Basis build_basis(const Crystal& c, const std::array<int, 3>& shape, double encut, const double k[3]) {
  if (!(encut > 0)) fail(kInvalidArgument, "ENCUT must be positive");
  Basis b;
  b.shape = shape;
  for (int j = 0; j < 3; ++j) b.kpoint[j] = k[j];
  auto rec = c.reciprocal();
  const int s1 = shape[0], s2 = shape[1], s3 = shape[2];
  for (int n1 = -(s1 / 2); n1 <= (s1 - 1) / 2; ++n1)
    for (int n2 = -(s2 / 2); n2 <= (s2 - 1) / 2; ++n2)
      for (int n3 = -(s3 / 2); n3 <= (s3 - 1) / 2; ++n3) {
        double f0 = n1 + k[0], f1 = n2 + k[1], f2 = n3 + k[2];
        double q[3];
        for (int j = 0; j < 3; ++j) q[j] = f0 * rec[0 * 3 + j] + f1 * rec[1 * 3 + j] + f2 * rec[2 * 3 + j];
        double kin = kHsqdtm * (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
        if (kin < encut) {
          b.gvec.push_back(n1);
          b.gvec.push_back(n2);
          b.gvec.push_back(n3);
          b.qvec.insert(b.qvec.end(), {q[0], q[1], q[2]});
          b.kinetic.push_back(kin);
          long long i1 = ((n1 % s1) + s1) % s1, i2 = ((n2 % s2) + s2) % s2, i3 = ((n3 % s3) + s3) % s3;
          b.fft_index.push_back((i1 * s2 + i2) * s3 + i3);
        }
      }
  return b;
}

}  // namespace hb
