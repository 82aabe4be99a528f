// Band occupations for the band-energy force workload, restating
// compute_occupations (src/half_energy.F90:41-120): zero width fills
// degenerate levels fractionally in ascending order; otherwise bisection on
// the chemical potential (256 steps) with Gaussian (ISMEAR=0, erfc) or
// Fermi-Dirac (ISMEAR=-1) occupations and the matching entropy term.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "common.h"

namespace hb {

void compute_occupations(const std::vector<double>& eig, int nk, int nb, const double* w, double nelect, double sigma,
                         int ismear, std::vector<double>& occ, double& mu, double& band, double& entropy) {
  double wsum = 0;
  for (int k = 0; k < nk; ++k) wsum += w[k];
  if (std::fabs(wsum - 1.0) > 1e-10) fail(kInvalidArgument, "k-point weights must sum to one");
  if (nelect < -1e-12 || nelect > 2.0 * nb + 1e-12) fail(kInvalidArgument, "electrons do not fit in requested bands");
  if (!(sigma >= 0)) fail(kInvalidArgument, "sigma must be finite and non-negative");
  if (ismear != -1 && ismear != 0) fail(kInvalidArgument, "supported ISMEAR values are -1 and 0");
  occ.assign((size_t)nk * nb, 0.0);
  const double emin = *std::min_element(eig.begin(), eig.end());
  const double emax = *std::max_element(eig.begin(), eig.end());
  entropy = 0;
  if (sigma == 0.0) {
    int ns = nk * nb;
    std::vector<int> order(ns);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return eig[a] < eig[b]; });
    double remaining = nelect;
    mu = emin;
    int pos = 0;
    while (pos < ns && remaining > 1e-13) {
      double level = eig[order[pos]];
      int stop = pos + 1;
      double tol = 1e-10 * std::max(1.0, std::fabs(level));
      while (stop < ns && std::fabs(eig[order[stop]] - level) <= tol) ++stop;
      double capacity = 0;
      for (int i = pos; i < stop; ++i) capacity += 2.0 * w[order[i] / nb];
      double frac = std::min(1.0, std::max(0.0, remaining / capacity));
      for (int i = pos; i < stop; ++i) occ[order[i]] = 2.0 * frac;
      double filled = frac * capacity;
      if (filled > 0) mu = level;
      remaining -= filled;
      pos = stop;
    }
    if (remaining > 1e-9) fail(kInvalidArgument, "not enough bands for electron count");
  } else {
    auto count = [&](double m) {
      double v = 0;
      for (int k = 0; k < nk; ++k)
        for (int b = 0; b < nb; ++b) {
          double x = (eig[(size_t)k * nb + b] - m) / sigma;
          if (ismear == 0) v += w[k] * std::erfc(x);
          else { x = std::max(-700.0, std::min(700.0, x)); v += w[k] * 2.0 / (1.0 + std::exp(x)); }
        }
      return v;
    };
    double lo = emin - std::max(10.0, 100.0 * sigma), hi = emax + std::max(10.0, 100.0 * sigma);
    for (int i = 0; i < 256; ++i) {
      double mid = 0.5 * (lo + hi);
      if (count(mid) < nelect) lo = mid; else hi = mid;
      if (hi - lo < 1e-13 * std::max(1.0, std::fabs(mid))) break;
    }
    mu = 0.5 * (lo + hi);
    for (int k = 0; k < nk; ++k)
      for (int b = 0; b < nb; ++b) {
        double x = (eig[(size_t)k * nb + b] - mu) / sigma;
        if (ismear == 0) {
          occ[(size_t)k * nb + b] = std::erfc(x);
          if (std::fabs(x) < 20.0) entropy -= sigma * w[k] * std::exp(-x * x) / std::sqrt(3.141592653589793238462643383279502884);
        } else {
          x = std::max(-700.0, std::min(700.0, x));
          double p = 1.0 / (1.0 + std::exp(x));
          occ[(size_t)k * nb + b] = 2.0 * p;
          p = std::max(1e-300, std::min(1.0 - 1e-16, p));
          entropy += 2.0 * sigma * w[k] * (p * std::log(p) + (1 - p) * std::log(1 - p));
        }
      }
  }
  band = 0;
  for (int k = 0; k < nk; ++k)
    for (int b = 0; b < nb; ++b) band += w[k] * occ[(size_t)k * nb + b] * eig[(size_t)k * nb + b];
}

}  // namespace hb
