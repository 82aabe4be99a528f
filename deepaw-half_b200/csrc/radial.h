// Radial and angular helper math shared by host set-up and device kernels:
// the reference's uniform-grid cubic spline (src/half_paw.F90:78-107), its
// associated Legendre recursion and real spherical harmonics (:109-143).
#pragma once

#include <cmath>
#include <vector>

#ifdef __CUDACC__
#define HALF_HD __host__ __device__
#else
#define HALF_HD
#endif

namespace hb {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kAutoa = 0.529177249;
constexpr double kRytoev = 13.605826;
constexpr double kHatoev = 2.0 * kRytoev;
constexpr double kFelect = 2.0 * kRytoev * kAutoa;
constexpr double kEdeps = 4.0 * kPi * kFelect;
constexpr double kHsqdtm = kRytoev * kAutoa * kAutoa;

// Second-derivative table of the reference's spline on x_k = k * xmax / n.
std::vector<double> spline_second(const std::vector<double>& y, double xmax);

// Evaluate the spline at x (k clamped to [1, n-1] in 1-based terms).
HALF_HD inline double spline_eval(const double* y, const double* m2, int n, double xmax, double x) {
  double h = xmax / n;
  int k = int(floor(x / h)) + 1;
  k = k < 1 ? 1 : (k > n - 1 ? n - 1 : k);
  double t = (x - (k - 1) * h) / h;
  double u = 1 - t;
  return u * y[k - 1] + t * y[k] + h * h * ((u * u * u - u) * m2[k - 1] + (t * t * t - t) * m2[k]) / 6;
}

HALF_HD inline double factorial_d(int n) {
  double v = 1;
  for (int i = 2; i <= n; ++i) v *= i;
  return v;
}

HALF_HD inline double assoc_legendre(int l, int m, double x) {
  double pmm = 1;
  if (m > 0) {
    double fact = 1, s = sqrt(fmax(0.0, (1 - x) * (1 + x)));
    for (int i = 1; i <= m; ++i) { pmm = -pmm * fact * s; fact += 2; }
  }
  if (l == m) return pmm;
  double pmmp1 = x * (2 * m + 1) * pmm;
  if (l == m + 1) return pmmp1;
  double pll = 0;
  for (int ll = m + 2; ll <= l; ++ll) {
    pll = ((2 * ll - 1) * x * pmmp1 - (ll + m - 1) * pmm) / (ll - m);
    pmm = pmmp1;
    pmmp1 = pll;
  }
  return pmmp1;
}

// Real harmonic of the reference from x = cos(theta) and phi.
HALF_HD inline double real_ylm(int l, int m, double x, double phi) {
  int am = m < 0 ? -m : m;
  double p = assoc_legendre(l, am, x);
  double norm = sqrt((2 * l + 1) / (4 * kPi) * factorial_d(l - am) / factorial_d(l + am));
  double sgn = (am % 2) ? -1.0 : 1.0;
  if (m > 0) return sqrt(2.0) * sgn * norm * p * cos(am * phi);
  if (m < 0) return sqrt(2.0) * sgn * norm * p * sin(am * phi);
  return norm * p;
}

// Per-species QDEP tables (src/half_uspp.F90:137-200): radial weights,
// compensation shapes g_l, multipoles, quadrature directions and weights.
struct QdepTables {
  int nlm = 0, naug = 0, nrad = 0, lmax = 0;
  std::vector<int> laug;            // naug
  std::vector<double> rgrid;        // nrad
  std::vector<double> wr2g;         // [k][ir] = rw * r^2 * g_{l_k}(r)
  std::vector<double> multipole;    // [a][b][k]
  std::vector<double> dirs;         // [ip][3], 288 directions
  std::vector<double> yweight;      // [ip][k]
  std::vector<double> dion_lm;      // [a][b]
  std::vector<double> qij_lm;       // [a][b]
  // g_l(r) = c1 j_l(z1 r / rc) + c2 j_l(z2 r / rc) for r <= paw_rmax
  // (src/half_uspp.F90:163-171): [l][4] = {z1, z2, c1, c2}
  std::vector<double> shape_coeff;
};

// Spherical Bessel j_l (src/half_uspp.F90:307-319): power series below
// x = l + 2, upward recurrence above.
HALF_HD inline double sph_bessel(int l, double x) {
  if (fabs(x) < l + 2) {
    double den = 1;
    for (int i = 1; i <= l; ++i) den *= 2 * i + 1;
    double x2 = x * x, term = pow(x, double(l)) / den, v = term;
    for (int k = 0; k <= 30; ++k) {
      term = -term * x2 / (2.0 * (k + 1) * (2 * l + 2 * k + 3));
      v += term;
      if (fabs(term) < 1e-16 * fmax(1.0, fabs(v))) break;
    }
    return v;
  }
  double jm = sin(x) / x;
  if (l == 0) return jm;
  double j = sin(x) / (x * x) - cos(x) / x;
  if (l == 1) return j;
  for (int n = 1; n <= l - 1; ++n) {
    double jn = (2 * n + 1) * j / x - jm;
    jm = j;
    j = jn;
  }
  return j;
}

struct Potcar;
QdepTables build_qdep_tables(const Potcar& pot);
void species_lm_tables(const Potcar& pot, std::vector<double>& dij, std::vector<double>& qij);

}  // namespace hb
