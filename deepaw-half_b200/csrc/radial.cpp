// Host-side radial tables for the projector splines and the MIMIC_US QDEP
// correction.  Each routine restates the cited reference routine; these run
// once per context on the host (a few thousand operations per species).
#include "radial.h"

#include <algorithm>

#include "common.h"
#include "io.h"

namespace hb {

// src/half_paw.F90:78-99 (the reference's end conditions on a uniform grid)
std::vector<double> spline_second(const std::vector<double>& y, double xmax) {
  int n = int(y.size());
  if (n < 4) fail(kIO, "spline table too short");
  double h = xmax / n;
  std::vector<double> diag(n, 0.0), rhs(n, 0.0), upper(n, 0.0), m2(n, 0.0);
  diag[1] = 1;
  rhs[1] = ((y[2] - y[1]) / h - (y[1] - y[0]) / h) / h;
  for (int i = 2; i <= n - 3; ++i) {
    diag[i] = 4 * h;
    upper[i] = h;
    rhs[i] = 6 * ((y[i + 1] - y[i]) / h - (y[i] - y[i - 1]) / h);
  }
  diag[n - 2] = 1;
  rhs[n - 2] = ((y[n - 1] - y[n - 2]) / h - (y[n - 2] - y[n - 3]) / h) / h;
  for (int i = 2; i <= n - 2; ++i) {
    double w = (i <= n - 3 ? h : 0.0) / diag[i - 1];
    diag[i] -= w * upper[i - 1];
    rhs[i] -= w * rhs[i - 1];
  }
  m2[n - 2] = rhs[n - 2] / diag[n - 2];
  for (int i = n - 3; i >= 1; --i) m2[i] = (rhs[i] - upper[i] * m2[i + 1]) / diag[i];
  m2[0] = 2 * m2[1] - m2[2];
  m2[n - 1] = 2 * m2[n - 2] - m2[n - 3];
  return m2;
}

namespace {

// src/half_uspp.F90:292-305
std::vector<double> radial_weights(const std::vector<double>& r) {
  int n = int(r.size());
  std::vector<double> w(n, 0.0);
  int last = (n % 2 == 1) ? n : n - 1;
  for (int i = 0; i <= last - 3; i += 2) {
    double h0 = r[i + 1] - r[i], h1 = r[i + 2] - r[i + 1], s = (h0 + h1) / 6;
    w[i] += s * (2 - h1 / h0);
    w[i + 1] += s * (h0 + h1) * (h0 + h1) / (h0 * h1);
    w[i + 2] += s * (2 - h0 / h1);
  }
  if (n % 2 == 0) {
    double h0 = r[n - 2] - r[n - 3], h1 = r[n - 1] - r[n - 2];
    w[n - 1] += (2 * h1 * h1 + 3 * h0 * h1) / (6 * (h0 + h1));
    w[n - 2] += (h1 * h1 + 3 * h0 * h1) / (6 * h0);
    w[n - 3] -= h1 * h1 * h1 / (6 * h0 * (h0 + h1));
  }
  return w;
}

double sph_bessel_deriv(int l, double x) {
  if (l == 0) return -sph_bessel(1, x);
  return sph_bessel(l - 1, x) - (l + 1) / x * sph_bessel(l, x);
}

// src/half_uspp.F90:321-333
double bessel_root(int l, int which) {
  double x0 = 1e-4, f0 = sph_bessel(l, x0), x1 = x0, f1;
  int found = 0;
  while (found < which) {
    x1 = x0 + 0.05;
    f1 = sph_bessel(l, x1);
    if (f0 * f1 < 0) {
      ++found;
      if (found == which) break;
    }
    x0 = x1;
    f0 = f1;
  }
  while (x1 - x0 > 1e-13) {
    double root = 0.5 * (x0 + x1);
    if (f0 * sph_bessel(l, root) <= 0) x1 = root;
    else { x0 = root; f0 = sph_bessel(l, x0); }
  }
  return 0.5 * (x0 + x1);
}

// src/half_uspp.F90:363-375
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  int m = (n + 1) / 2;
  for (int i = 1; i <= m; ++i) {
    double z = std::cos(kPi * (i - 0.25) / (n + 0.5)), z1, pp, p1, p2, p3;
    while (true) {
      p1 = 1; p2 = 0;
      for (int j = 1; j <= n; ++j) {
        p3 = p2; p2 = p1;
        p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1);
      z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1e-15) break;
    }
    x[i - 1] = -z;
    x[n - i] = z;
    w[i - 1] = 2 / ((1 - z * z) * pp * pp);
    w[n - i] = w[i - 1];
  }
}

// src/half_uspp.F90:335-342
void compensation_coefficients(int l, double rc, double z1, double z2, double& c1, double& c2) {
  double a11 = z1 / rc * sph_bessel_deriv(l, z1), a12 = z2 / rc * sph_bessel_deriv(l, z2);
  std::vector<double> xg, wg;
  gauss_legendre(32, xg, wg);
  double a21 = 0, a22 = 0;
  for (int i = 0; i < 32; ++i) {
    double rg = 0.5 * rc * (xg[i] + 1), w = 0.5 * rc * wg[i];
    a21 += w * sph_bessel(l, z1 * rg / rc) * std::pow(rg, l + 2);
    a22 += w * sph_bessel(l, z2 * rg / rc) * std::pow(rg, l + 2);
  }
  double det = a11 * a22 - a12 * a21;
  c1 = -a12 / det;
  c2 = a11 / det;
}

// src/half_uspp.F90:353-361
double gaunt_numeric(int l1, int m1, int l2, int m2, int l3, int m3) {
  std::vector<double> xg, wg;
  gauss_legendre(12, xg, wg);
  double g = 0;
  for (int it = 0; it < 12; ++it)
    for (int ip = 0; ip < 24; ++ip) {
      double phi = 2 * kPi * ip / 24;
      g += wg[it] * 2 * kPi / 24 * real_ylm(l1, m1, xg[it], phi) * real_ylm(l2, m2, xg[it], phi) *
           real_ylm(l3, m3, xg[it], phi);
    }
  return g;
}

}  // namespace

// Expanded per-species DION / QPAW: nonzero only for equal (l, m)
// (src/half_paw.F90:39-51).  Row-major [a][b].
void species_lm_tables(const Potcar& pot, std::vector<double>& dij, std::vector<double>& qij) {
  int nlm = pot.nlm(), nch = pot.channels();
  dij.assign(size_t(nlm) * nlm, 0.0);
  qij.assign(size_t(nlm) * nlm, 0.0);
  int a = 0;
  for (int ia = 0; ia < nch; ++ia)
    for (int ma = -pot.lps[ia]; ma <= pot.lps[ia]; ++ma, ++a) {
      int b = 0;
      for (int ib = 0; ib < nch; ++ib)
        for (int mb = -pot.lps[ib]; mb <= pot.lps[ib]; ++mb, ++b)
          if (pot.lps[ia] == pot.lps[ib] && ma == mb) {
            dij[a * nlm + b] = pot.dion[ia * nch + ib];
            qij[a * nlm + b] = pot.qpaw[ia * nch + ib];
          }
    }
}

QdepTables build_qdep_tables(const Potcar& pot) {
  QdepTables t;
  int nch = pot.channels();
  std::vector<int> chan, lv, mv;
  for (int ich = 0; ich < nch; ++ich)
    for (int m = -pot.lps[ich]; m <= pot.lps[ich]; ++m) {
      chan.push_back(ich);
      lv.push_back(pot.lps[ich]);
      mv.push_back(m);
    }
  t.nlm = int(chan.size());
  t.lmax = 0;
  for (int l : pot.lps) t.lmax = std::max(t.lmax, 2 * l);
  t.naug = (t.lmax + 1) * (t.lmax + 1);
  t.nrad = pot.nmax;
  t.rgrid = pot.rgrid;
  std::vector<int> maug;
  for (int l = 0; l <= t.lmax; ++l)
    for (int m = -l; m <= l; ++m) { t.laug.push_back(l); maug.push_back(m); }
  auto rw = radial_weights(pot.rgrid);
  std::vector<double> gshape(size_t(t.nrad) * (t.lmax + 1), 0.0);   // [l][ir]
  for (int l = 0; l <= t.lmax; ++l) {
    double z1 = bessel_root(l, 1), z2 = bessel_root(l, 2), c1, c2;
    compensation_coefficients(l, pot.paw_rmax, z1, z2, c1, c2);
    t.shape_coeff.insert(t.shape_coeff.end(), {z1, z2, c1, c2});
    for (int ir = 0; ir < t.nrad; ++ir) {
      double r = pot.rgrid[ir];
      if (r <= pot.paw_rmax)
        gshape[size_t(l) * t.nrad + ir] = c1 * sph_bessel(l, z1 * r / pot.paw_rmax) + c2 * sph_bessel(l, z2 * r / pot.paw_rmax);
    }
  }
  t.wr2g.assign(size_t(t.naug) * t.nrad, 0.0);
  for (int k = 0; k < t.naug; ++k)
    for (int ir = 0; ir < t.nrad; ++ir) {
      double r = pot.rgrid[ir];
      t.wr2g[size_t(k) * t.nrad + ir] = rw[ir] * r * r * gshape[size_t(t.laug[k]) * t.nrad + ir];
    }
  // multipoles (src/half_uspp.F90:176-187)
  t.multipole.assign(size_t(t.nlm) * t.nlm * t.naug, 0.0);
  for (int a = 0; a < t.nlm; ++a)
    for (int b = 0; b < t.nlm; ++b)
      for (int k = 0; k < t.naug; ++k) {
        int l = t.laug[k];
        if (std::abs(lv[a] - lv[b]) <= l && l <= lv[a] + lv[b] && (lv[a] + lv[b] + l) % 2 == 0) {
          double moment = 0;
          const double* wa = &pot.wae[size_t(chan[a]) * t.nrad];
          const double* wb = &pot.wae[size_t(chan[b]) * t.nrad];
          const double* pa = &pot.wps[size_t(chan[a]) * t.nrad];
          const double* pb = &pot.wps[size_t(chan[b]) * t.nrad];
          for (int ir = 0; ir < t.nrad; ++ir)
            moment += rw[ir] * (wa[ir] * wb[ir] - pa[ir] * pb[ir]) * std::pow(pot.rgrid[ir], l);
          t.multipole[(size_t(a) * t.nlm + b) * t.naug + k] = gaunt_numeric(lv[a], mv[a], lv[b], mv[b], l, maug[k]) * moment;
        }
      }
  // directions and harmonic weights (src/half_uspp.F90:188-200)
  std::vector<double> xg, wg;
  gauss_legendre(12, xg, wg);
  for (int it = 0; it < 12; ++it)
    for (int m = 0; m < 24; ++m) {
      double ph = 2 * kPi * m / 24, st = std::sqrt(std::max(0.0, 1.0 - xg[it] * xg[it]));
      t.dirs.push_back(st * std::cos(ph));
      t.dirs.push_back(st * std::sin(ph));
      t.dirs.push_back(xg[it]);
      for (int k = 0; k < t.naug; ++k)
        t.yweight.push_back(real_ylm(t.laug[k], maug[k], xg[it], ph) * wg[it] * 2 * kPi / 24);
    }
  species_lm_tables(pot, t.dion_lm, t.qij_lm);
  return t;
}

}  // namespace hb
