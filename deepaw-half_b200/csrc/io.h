// Host-side input model: crystal, smooth density grid and POTCAR datasets.
#pragma once

#include <array>
#include <string>
#include <vector>

namespace hb {

// crystal_t of the reference (src/half_types.F90:9-21): lattice rows are the
// lattice vectors (Angstrom), positions fractional in type-major order.
struct Crystal {
  std::string name;
  std::array<double, 9> lattice{};     // row-major [vector][xyz]
  std::vector<std::string> species;    // element per type
  std::vector<int> counts;             // atoms per type
  std::vector<double> positions;       // nions*3 fractional
  int nions() const { int n = 0; for (int c : counts) n += c; return n; }
  int ntypes() const { return int(counts.size()); }
  double volume() const;
  std::array<double, 9> reciprocal() const;   // 2 pi inv(lattice)^T, rows b_i
  std::array<double, 9> inverse_lattice() const;
  std::array<double, 3> cartesian(int ion) const;
};

// potcar_t (src/half_types.F90:41-56), only the fields the path reads.
struct Potcar {
  std::string header, element;
  double zval = 0, psp_gmax = 0, pspnl_gmax = 0, paw_rmax = 0;
  std::vector<double> psp_local, pspcor, psprho;
  std::vector<int> lps;                 // l per channel
  std::vector<double> dion;             // channels x channels, row-major
  std::vector<double> pspnl;            // [channel][100]
  std::vector<double> qpaw;             // channels x channels, row-major
  int nmax = 0;
  std::vector<double> rgrid;
  std::vector<double> wae, wps;         // [channel][nmax]
  bool has_core() const { return !pspcor.empty(); }
  int channels() const { return int(lps.size()); }
  int nlm() const { int n = 0; for (int l : lps) n += 2 * l + 1; return n; }
};

struct ChargeGrid {
  std::array<int, 3> shape{};
  std::vector<double> values;           // file order, x fastest (rho * Omega)
};

// src/half_chgcar.F90:133-219
void read_chgcar(const std::string& path, Crystal& crystal, ChargeGrid& charge);
// src/half_potcar.F90:24-205
std::vector<Potcar> read_potcar(const std::string& path);
// src/half_potcar.F90:12-22
void validate_potcar_structure(const std::vector<Potcar>& pots, const Crystal& c);

bool file_exists(const std::string& path);

}  // namespace hb
