// Text readers for the reference's input formats.
//
// CHGCAR: POSCAR header (scale, three lattice rows, optional element line,
// counts, optional Selective line, Direct/Cartesian, positions), blank
// line(s), grid line, then nx*ny*nz values x fastest (src/half_chgcar.F90:
// 133-219).  POTCAR: one or more datasets, each header, ZVAL, PSCTR tags up to
// "END of PSCTR", local part (1000 points) with optional sections, non-local
// projector blocks (DION + 100-point reciprocal / real tables) and the PAW
// radial sets (src/half_potcar.F90:24-205).  Numbers are read Fortran
// list-directed style: whitespace separated, continuing across lines.
#include "io.h"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <sys/stat.h>

#include "common.h"

namespace hb {

double Crystal::volume() const {
  const auto& a = lattice;
  double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
               a[2] * (a[3] * a[7] - a[4] * a[6]);
  return std::fabs(det);
}

std::array<double, 9> Crystal::inverse_lattice() const {
  const auto& a = lattice;
  double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
               a[2] * (a[3] * a[7] - a[4] * a[6]);
  if (std::fabs(det) < 1e-18) fail(kInvalidArgument, "singular lattice");
  std::array<double, 9> inv{};
  inv[0] = (a[4] * a[8] - a[5] * a[7]) / det;
  inv[1] = -(a[1] * a[8] - a[2] * a[7]) / det;
  inv[2] = (a[1] * a[5] - a[2] * a[4]) / det;
  inv[3] = -(a[3] * a[8] - a[5] * a[6]) / det;
  inv[4] = (a[0] * a[8] - a[2] * a[6]) / det;
  inv[5] = -(a[0] * a[5] - a[2] * a[3]) / det;
  inv[6] = (a[3] * a[7] - a[4] * a[6]) / det;
  inv[7] = -(a[0] * a[7] - a[1] * a[6]) / det;
  inv[8] = (a[0] * a[4] - a[1] * a[3]) / det;
  return inv;
}

std::array<double, 9> Crystal::reciprocal() const {
  auto inv = inverse_lattice();
  const double twopi = 2.0 * 3.141592653589793238462643383279502884;
  std::array<double, 9> b{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) b[i * 3 + j] = twopi * inv[j * 3 + i];
  return b;
}

std::array<double, 3> Crystal::cartesian(int ion) const {
  std::array<double, 3> r{};
  for (int j = 0; j < 3; ++j)
    r[j] = positions[ion * 3 + 0] * lattice[0 * 3 + j] + positions[ion * 3 + 1] * lattice[1 * 3 + j] +
           positions[ion * 3 + 2] * lattice[2 * 3 + j];
  return r;
}

bool file_exists(const std::string& path) {
  struct stat st;
  return ::stat(path.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

namespace {

std::vector<std::string> read_lines(const std::string& path, const char* what) {
  std::ifstream in(path, std::ios::binary);
  if (!in) fail(kIO, std::string("cannot open ") + what);
  std::stringstream ss;
  ss << in.rdbuf();
  std::string all = ss.str();
  std::vector<std::string> lines;
  size_t start = 0;
  while (start <= all.size()) {
    size_t nl = all.find('\n', start);
    if (nl == std::string::npos) {
      if (start < all.size()) lines.push_back(all.substr(start));
      break;
    }
    std::string l = all.substr(start, nl - start);
    if (!l.empty() && l.back() == '\r') l.pop_back();
    lines.push_back(l);
    start = nl + 1;
  }
  return lines;
}

std::string lower(std::string s) {
  for (auto& c : s) c = char(std::tolower((unsigned char)c));
  return s;
}

std::vector<std::string> words(const std::string& line) {
  std::vector<std::string> w;
  std::istringstream is(line);
  std::string t;
  while (is >> t) w.push_back(t);
  return w;
}

bool trimmed_empty(const std::string& s) {
  for (char c : s)
    if (!std::isspace((unsigned char)c)) return false;
  return true;
}

double parse_real(const std::string& tok, const char* what) {
  std::string t = tok;
  for (auto& c : t)
    if (c == 'D' || c == 'd') c = 'E';
  char* end = nullptr;
  double v = std::strtod(t.c_str(), &end);
  if (end == t.c_str()) fail(kIO, std::string("failed to read ") + what);
  return v;
}

bool parse_int(const std::string& tok, int& v) {
  char* end = nullptr;
  long x = std::strtol(tok.c_str(), &end, 10);
  if (end == tok.c_str() || *end != '\0') return false;
  v = int(x);
  return true;
}

struct Cursor {
  const std::vector<std::string>& lines;
  size_t pos = 0;
  const char* file;
  explicit Cursor(const std::vector<std::string>& l, const char* f) : lines(l), file(f) {}
  bool eof() const { return pos >= lines.size(); }
  const std::string& line(const char* what) {
    if (eof()) fail(kIO, std::string("failed to read ") + file + " " + what);
    return lines[pos++];
  }
  const std::string& nonblank(const char* what) {
    while (true) {
      const std::string& l = line(what);
      if (!trimmed_empty(l)) return l;
    }
  }
  // list-directed read of n reals continuing across lines
  std::vector<double> values(size_t n, const char* what) {
    std::vector<double> v;
    v.reserve(n);
    while (v.size() < n) {
      const std::string& l = line(what);
      const char* p = l.c_str();
      while (*p && v.size() < n) {
        while (*p && (std::isspace((unsigned char)*p) || *p == ',')) ++p;
        if (!*p) break;
        const char* q = p;
        while (*q && !std::isspace((unsigned char)*q) && *q != ',') ++q;
        v.push_back(parse_real(std::string(p, q), what));
        p = q;
      }
    }
    return v;
  }
};

}  // namespace

void read_chgcar(const std::string& path, Crystal& c, ChargeGrid& g) {
  auto lines = read_lines(path, "CHGCAR");
  Cursor cur(lines, "CHGCAR");
  c = Crystal();
  c.name = cur.line("system name");
  double scale = cur.values(1, "lattice scale")[0];
  if (!(scale > 0)) fail(kIO, "only positive POSCAR scale is supported");
  for (int i = 0; i < 3; ++i) {
    auto w = words(cur.line("lattice vector"));
    if (w.size() < 3) fail(kIO, "failed to read lattice vector");
    for (int j = 0; j < 3; ++j) c.lattice[i * 3 + j] = scale * parse_real(w[j], "lattice vector");
  }
  auto w = words(cur.line("species or counts"));
  if (w.empty()) fail(kIO, "empty species/count line");
  bool all_int = true;
  for (auto& t : w) { int v; if (!parse_int(t, v)) all_int = false; }
  if (all_int) {
    for (size_t i = 0; i < w.size(); ++i) {
      c.species.push_back("Type" + std::to_string(i + 1));
      int v; parse_int(w[i], v); c.counts.push_back(v);
    }
  } else {
    c.species = w;
    auto cw = words(cur.line("ion counts"));
    if (cw.size() != w.size()) fail(kIO, "invalid ion counts");
    for (auto& t : cw) { int v; if (!parse_int(t, v)) fail(kIO, "invalid ion counts"); c.counts.push_back(v); }
  }
  for (int n : c.counts)
    if (n < 1) fail(kIO, "invalid ion counts");
  // the reference tests the first column only (line(1:1)), not the first word
  std::string mode = cur.line("coordinate mode");
  char m0 = mode.empty() ? ' ' : char(std::tolower((unsigned char)mode[0]));
  if (m0 == 's') {
    mode = cur.line("coordinate mode after selective dynamics");
    m0 = mode.empty() ? ' ' : char(std::tolower((unsigned char)mode[0]));
  }
  bool cart = (m0 == 'c' || m0 == 'k');
  int nions = c.nions();
  c.positions.assign(size_t(nions) * 3, 0.0);
  for (int i = 0; i < nions; ++i) {
    auto pw = words(cur.line("atomic position"));
    if (pw.size() < 3) fail(kIO, "failed to read atomic position values");
    for (int j = 0; j < 3; ++j) c.positions[i * 3 + j] = parse_real(pw[j], "atomic position values");
  }
  if (cart) {
    auto inv = c.inverse_lattice();
    for (int i = 0; i < nions; ++i) {
      double x[3] = {c.positions[i * 3], c.positions[i * 3 + 1], c.positions[i * 3 + 2]};
      for (int j = 0; j < 3; ++j) c.positions[i * 3 + j] = x[0] * inv[0 * 3 + j] + x[1] * inv[1 * 3 + j] + x[2] * inv[2 * 3 + j];
    }
  }
  auto gw = words(cur.nonblank("FFT grid"));
  if (gw.size() < 3) fail(kIO, "failed to read FFT grid dimensions");
  for (int j = 0; j < 3; ++j) {
    int v;
    if (!parse_int(gw[j], v) || v <= 0) fail(kIO, "invalid FFT grid dimensions");
    g.shape[j] = v;
  }
  size_t ngrid = size_t(g.shape[0]) * g.shape[1] * g.shape[2];
  g.values = cur.values(ngrid, "smooth charge grid");
}

namespace {

bool tag_value(const std::string& line, const char* tag, std::string& part) {
  size_t at = line.find(tag);
  if (at == std::string::npos) return false;
  size_t eq = line.find('=', at);
  if (eq == std::string::npos) return false;
  part = line.substr(eq + 1);
  size_t s = part.find_first_not_of(" \t");
  part = (s == std::string::npos) ? std::string() : part.substr(s);
  return true;
}

Potcar read_dataset(Cursor& cur, const std::string& header) {
  Potcar p;
  p.header = header;
  auto hw = words(header);
  p.element = hw.size() >= 2 ? hw[1] : "";
  p.zval = cur.values(1, "POTCAR ZVAL")[0];
  while (true) {  // PSCTR (half_potcar.F90:65-78)
    const std::string& l = cur.line("POTCAR PSCTR");
    if (lower(l).find("end of psctr") != std::string::npos) break;
    std::string part;
    if (tag_value(l, "ZVAL", part)) {
      size_t semi = part.find(';');
      if (semi != std::string::npos) part = part.substr(0, semi);
      auto pw = words(part);
      if (!pw.empty()) {
        char* end = nullptr;
        double v = std::strtod(pw[0].c_str(), &end);
        if (end != pw[0].c_str()) p.zval = v;
      }
    }
    if (tag_value(l, "VRHFIN", part)) {
      size_t last = part.find_first_of(" :;\t");
      p.element = part.substr(0, last);
    }
  }
  if (lower(cur.nonblank("POTCAR local header")).find("local part") == std::string::npos)
    fail(kIO, "expected POTCAR local part");
  p.psp_gmax = cur.values(1, "POTCAR local grid")[0];
  p.psp_local = cur.values(1000, "POTCAR local potential");
  while (true) {  // half_potcar.F90:90-106
    std::string l = lower(cur.nonblank("POTCAR local optional data"));
    if (l.find("gradient") != std::string::npos) {
      cur.line("POTCAR gradient selector");
    } else if (l.find("core charge-density (partial)") != std::string::npos) {
      p.pspcor = cur.values(1000, "POTCAR partial core charge");
    } else if (l.find("kinetic energy density") != std::string::npos) {
      cur.values(1000, "POTCAR kinetic density");
    } else if (l.find("atomic pseudo charge-density") != std::string::npos) {
      p.psprho = cur.values(1000, "POTCAR atomic pseudo charge");
      break;
    } else {
      fail(kIO, "unknown POTCAR local-data selector");
    }
  }
  p.pspnl_gmax = cur.values(1, "POTCAR projector grid")[0];
  std::vector<std::pair<int, std::vector<double>>> dblocks;
  std::vector<std::vector<double>> gcols;
  while (true) {  // half_potcar.F90:119-144
    std::string l = lower(cur.nonblank("POTCAR projector header"));
    if (l.find("paw radial sets") != std::string::npos) break;
    if (l.find("non local part") == std::string::npos) fail(kIO, "expected non-local projector block");
    auto hdr = cur.values(3, "POTCAR projector channels");
    int lval = int(hdr[0]), npro = int(hdr[1]);
    if (npro < 1 || lval < 0 || lval > 3) fail(kIO, "invalid POTCAR projector channels");
    dblocks.push_back({int(p.lps.size()), cur.values(size_t(npro) * npro, "POTCAR DION")});
    for (int i = 0; i < npro; ++i) {
      p.lps.push_back(lval);
      if (lower(cur.nonblank("POTCAR reciprocal header")).find("reciprocal space part") == std::string::npos)
        fail(kIO, "expected reciprocal projector");
      gcols.push_back(cur.values(100, "POTCAR reciprocal projector"));
      if (lower(cur.nonblank("POTCAR real header")).find("real space part") == std::string::npos)
        fail(kIO, "expected real projector");
      cur.values(100, "POTCAR real projector");
    }
  }
  int n = p.channels();
  if (n == 0) fail(kIO, "POTCAR dataset has no projectors");
  p.dion.assign(size_t(n) * n, 0.0);
  for (auto& b : dblocks) {
    int off = b.first;
    int k = int(std::lround(std::sqrt(double(b.second.size()))));
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j) p.dion[(off + i) * n + off + j] = b.second[i * k + j];
  }
  p.pspnl.clear();
  for (auto& col : gcols) p.pspnl.insert(p.pspnl.end(), col.begin(), col.end());
  auto hdr = cur.values(2, "POTCAR PAW grid header");  // half_potcar.F90:154
  p.nmax = int(hdr[0]);
  p.paw_rmax = hdr[1];
  if (p.nmax < 4) fail(kIO, "invalid POTCAR PAW grid");
  cur.line("POTCAR PAW format");
  if (lower(cur.nonblank("POTCAR augmentation header")).find("augmentation charges") == std::string::npos)
    fail(kIO, "expected augmentation charges");
  p.qpaw = cur.values(size_t(n) * n, "POTCAR QPAW");
  p.rgrid.assign(p.nmax, 0.0);
  p.wae.assign(size_t(n) * p.nmax, 0.0);
  p.wps.assign(size_t(n) * p.nmax, 0.0);
  while (true) {  // half_potcar.F90:163-200
    std::string raw = cur.nonblank("POTCAR PAW selector");
    size_t s0 = raw.find_first_not_of(" \t");
    std::string key = lower(raw.substr(s0));
    while (!key.empty() && std::isspace((unsigned char)key.back())) key.pop_back();
    auto has = [&](const char* t) { return key.find(t) != std::string::npos; };
    if (has("occupancies in atom") || has("uccopancies in atom")) {
      cur.values(size_t(n) * n, "POTCAR QATO");
    } else if (key == "grid") {
      p.rgrid = cur.values(p.nmax, "POTCAR radial grid");
    } else if (key == "aepotential") {
      cur.values(p.nmax, "POTCAR AE potential");
    } else if (has("core charge-density (pseudized)")) {
      cur.values(p.nmax, "POTCAR pseudo core charge");
    } else if (has("core charge-density")) {
      cur.values(p.nmax, "POTCAR AE core charge");
    } else if (has("local pseudopotential core")) {
      cur.values(p.nmax, "POTCAR core potential");
    } else if (has("pspotential valence only")) {
      cur.values(p.nmax, "POTCAR valence potential");
    } else if (has("kinetic energy-density") || has("mkinetic energy-density")) {
      cur.values(p.nmax, "POTCAR kinetic radial data");
    } else if (has("pseudo wavefunction")) {
      auto v = cur.values(p.nmax, "POTCAR pseudo wavefunction");
      std::copy(v.begin(), v.end(), p.wps.begin());
      cur.nonblank("POTCAR AE wavefunction header");
      v = cur.values(p.nmax, "POTCAR AE wavefunction");
      std::copy(v.begin(), v.end(), p.wae.begin());
      for (int i = 1; i < n; ++i) {
        cur.nonblank("POTCAR pseudo wavefunction header");
        v = cur.values(p.nmax, "POTCAR pseudo wavefunction");
        std::copy(v.begin(), v.end(), p.wps.begin() + size_t(i) * p.nmax);
        cur.nonblank("POTCAR AE wavefunction header");
        v = cur.values(p.nmax, "POTCAR AE wavefunction");
        std::copy(v.begin(), v.end(), p.wae.begin() + size_t(i) * p.nmax);
      }
      break;
    } else if (!key.empty() && key[0] == 't') {
      cur.values(size_t(n) * n, "POTCAR total charge");
    } else {
      fail(kIO, "unknown POTCAR PAW selector");
    }
  }
  while (!cur.eof()) {
    if (cur.line("end").find("End of Dataset") != std::string::npos) break;
  }
  return p;
}

}  // namespace

std::vector<Potcar> read_potcar(const std::string& path) {
  auto lines = read_lines(path, "POTCAR");
  Cursor cur(lines, "POTCAR");
  std::vector<Potcar> out;
  while (true) {
    while (!cur.eof() && trimmed_empty(lines[cur.pos])) ++cur.pos;
    if (cur.eof()) break;
    std::string header = cur.line("header");
    if (header.find("End of Dataset") != std::string::npos) continue;
    size_t s0 = header.find_first_not_of(" \t");
    size_t s1 = header.find_last_not_of(" \t");
    out.push_back(read_dataset(cur, header.substr(s0, s1 - s0 + 1)));
    if (out.size() > 32) fail(kIO, "too many POTCAR datasets");
  }
  return out;
}

void validate_potcar_structure(const std::vector<Potcar>& pots, const Crystal& c) {
  if (int(pots.size()) != c.ntypes())
    fail(kInvalidArgument, "POTCAR dataset count does not match structure species count");
  for (int i = 0; i < c.ntypes(); ++i) {
    std::string s = lower(c.species[i]);
    if (s.rfind("type", 0) == 0) continue;
    if (lower(pots[i].element) != s)
      fail(kInvalidArgument, "POTCAR dataset order does not match structure species order");
  }
}

}  // namespace hb
