// Standard mode of HPhi (`HPhi -s stan.in`, src/HPhiMain.c:212-214, which hands the file to
// the StdFace library's StdFace_main): a keyword file that names a lattice, a model and a
// method becomes the expert-mode input that the engine reads (namelist.def, calcmod.def,
// modpara.def, locspn.def, trans.def, interall.def, coulombintra.def, coulombinter.def,
// greenone.def, greentwo.def, pair.def / single.def for spectra, teone.def / tetwo.def for time
// evolution, and geometry.dat for the Fourier utility).
//
// StdFace's own sources are an empty submodule of the reference tree.  The conventions below
// follow the reference's documentation (doc/en/source/filespecification/standardmode_en/*.rst,
// doc/en/source/fourier/format.rst) and lattice figures (doc/figs/chap04_1_lattice.png,
// chap04_1_honeycomb.png, kagome.png, ladder.png), and the reference's test/*.sh outputs pin
// them (energies, site-resolved correlation functions, and the default frequency window of
// the spectra, which is the coefficient sum below):
//  - the numerical cell is spanned by a0 = (a0W, a0L) and a1 = (a1W, a1L) in units of the
//    primitive vectors (W and L alone give a0 = (W, 0), a1 = (0, L)); its unit cells are
//    numbered with the W coordinate running fastest, and site = cell * orbitals + orbital;
//  - a chain runs along W; a ladder's legs are its orbitals (site = L index * W + leg);
//  - Kondo lattices number the local spins first (0..N-1), then the conduction orbitals
//    (N..2N-1); local spin n couples to conduction orbital N + n;
//  - H = -mu n - t c+c + U n n + V n n (Hubbard); -h Sz - Gamma Sx + D Sz Sz + S J S (spin);
//    the Kondo coupling is J S.s with s = c+ sigma c / 2;
//  - the default LargeValue is (sum of |coefficients|) / Nsite, counting each one-body entry
//    of trans.def, each |U|, each |V|, and per spin bond the magnitudes of its terms (for two
//    S = 1/2 spins with a diagonal coupling: 5/4 |Jz| + |Jx + Jy| / 2 + |Jx - Jy| / 2);
//    OmegaMax / OmegaMin default to +-LargeValue * Nsite and OmegaIm to LargeValue / 100.
#include "stdface.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace hphi {
namespace stdface {
namespace {

using cplx = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;

struct Fail : std::runtime_error {
  explicit Fail(const std::string &m) : std::runtime_error(m) {}
};

std::string lower(std::string s) {
  for (auto &c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

// ----------------------------------------------------------------------------- keywords
// One "key = value" per line; blanks are dropped everywhere, keys are case-insensitive, and
// string values lose their double quotes and case.  A key given twice is an error, and so is
// a key that nothing reads (checked at the end).
class Keys {
 public:
  void load(const std::string &path) {
    std::ifstream f(path);
    if (!f.is_open()) throw Fail("cannot open " + path);
    std::string line;
    int n = 0;
    while (std::getline(f, line)) {
      n++;
      const auto hash = line.find('#');
      if (hash != std::string::npos) line.erase(hash);
      const auto sl = line.find("//");
      if (sl != std::string::npos) line.erase(sl);
      std::string s;
      for (char c : line)
        if (!std::isspace((unsigned char)c)) s += c;
      if (s.empty()) continue;
      const auto eq = s.find('=');
      if (eq == std::string::npos || eq == 0) throw Fail(path + ":" + std::to_string(n) + ": expected key = value");
      const std::string k = lower(s.substr(0, eq));
      std::string v;
      for (char c : s.substr(eq + 1))
        if (c != '"') v += c;
      if (kv_.count(k)) throw Fail(path + ": keyword given twice: " + k);
      kv_[k] = Entry{v, false};
    }
  }
  bool has(const std::string &k) const { return kv_.count(k) != 0; }
  bool str(const std::string &k, std::string *out) {
    auto it = kv_.find(k);
    if (it == kv_.end()) return false;
    it->second.used = true;
    *out = lower(it->second.value);
    return true;
  }
  std::string str_or(const std::string &k, const std::string &def) {
    std::string s;
    return str(k, &s) ? s : def;
  }
  bool real(const std::string &k, double *out) {
    auto it = kv_.find(k);
    if (it == kv_.end()) return false;
    it->second.used = true;
    *out = parse_real(k, it->second.value);
    return true;
  }
  double real_or(const std::string &k, double def) {
    double v;
    return real(k, &v) ? v : def;
  }
  bool integer(const std::string &k, long *out) {
    double v;
    if (!real(k, &v)) return false;
    if (v != std::floor(v)) throw Fail("keyword " + k + " needs an integer");
    *out = (long)v;
    return true;
  }
  long int_or(const std::string &k, long def) {
    long v;
    return integer(k, &v) ? v : def;
  }
  // "re" or "re,im"
  bool complex(const std::string &k, cplx *out) {
    auto it = kv_.find(k);
    if (it == kv_.end()) return false;
    it->second.used = true;
    const std::string &s = it->second.value;
    const auto comma = s.find(',');
    if (comma == std::string::npos) *out = cplx(parse_real(k, s), 0.0);
    else *out = cplx(parse_real(k, s.substr(0, comma)), parse_real(k, s.substr(comma + 1)));
    return true;
  }
  void check_all_used() const {
    for (const auto &e : kv_)
      if (!e.second.used) throw Fail("keyword not supported for this lattice / model / method: " + e.first);
  }

 private:
  struct Entry {
    std::string value;
    bool used;
  };
  static double parse_real(const std::string &k, const std::string &s) {
    char *end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (s.empty() || *end != '\0') throw Fail("keyword " + k + ": not a number: " + s);
    return v;
  }
  std::map<std::string, Entry> kv_;
};

// ----------------------------------------------------------------------------- lattice
// A bond type: from orbital si of cell R to orbital sj of cell R + (dw, dl).  `label` is the
// direction index of the parameter (t0 / t1 / t2), `order` the neighbour order (t, t', t'').
struct BondType {
  int dw, dl, si, sj, label, order;
};

struct Lattice {
  std::string kind;  // chain ladder square triangular honeycomb kagome
  int nsub = 1;
  long a[2][2] = {{0, 0}, {0, 0}};  // a0 = (a[0][0], a[0][1]), a1 = (a[1][0], a[1][1])
  long det = 0;
  std::vector<std::array<long, 2>> cells;
  std::map<std::array<long, 2>, int> index;
  std::vector<BondType> bonds;
  double cart[2][2] = {{1, 0}, {0, 1}};  // primitive vectors (for wave numbers and pulses)
  double tau[3][2] = {{0, 0}, {0, 0}, {0, 0}};  // orbital positions, fractional

  static long floor_div(long a, long b) {
    long q = a / b, r = a % b;
    if (r != 0 && ((r < 0) != (b < 0))) q--;
    return q;
  }
  void frac(long w, long l, long *f0, long *f1) const {  // det * fractional coordinates
    *f0 = w * a[1][1] - l * a[1][0];
    *f1 = -w * a[0][1] + l * a[0][0];
  }
  void build_cells() {
    det = a[0][0] * a[1][1] - a[0][1] * a[1][0];
    if (det == 0) throw Fail("the vectors a0 and a1 of the numerical cell are parallel");
    long lo[2] = {0, 0}, hi[2] = {0, 0};
    const long corner[4][2] = {{0, 0}, {a[0][0], a[0][1]}, {a[1][0], a[1][1]},
                               {a[0][0] + a[1][0], a[0][1] + a[1][1]}};
    for (auto &c : corner)
      for (int d = 0; d < 2; d++) {
        lo[d] = std::min(lo[d], c[d]);
        hi[d] = std::max(hi[d], c[d]);
      }
    for (long l = lo[1]; l <= hi[1]; l++)
      for (long w = lo[0]; w <= hi[0]; w++) {
        long f0, f1;
        frac(w, l, &f0, &f1);
        if (floor_div(f0, det) == 0 && floor_div(f1, det) == 0) {
          index[{w, l}] = (int)cells.size();
          cells.push_back({w, l});
        }
      }
    if ((long)cells.size() != std::labs(det)) throw Fail("internal error: numerical cell enumeration");
  }
  // Cell index of (w, l) folded into the numerical cell; n0 / n1 count the a0 / a1 shifts.
  int fold(long w, long l, long *n0, long *n1) const {
    long f0, f1;
    frac(w, l, &f0, &f1);
    *n0 = floor_div(f0, det);
    *n1 = floor_div(f1, det);
    const long ww = w - *n0 * a[0][0] - *n1 * a[1][0];
    const long ll = l - *n0 * a[0][1] - *n1 * a[1][1];
    return index.at({ww, ll});
  }
  int ncell() const { return (int)cells.size(); }
  // Cartesian position of orbital s in cell c (unfolded cell coordinates w, l).
  void position(double w, double l, int s, double *x, double *y) const {
    const double fw = w + tau[s][0], fl = l + tau[s][1];
    *x = fw * cart[0][0] + fl * cart[1][0];
    *y = fw * cart[0][1] + fl * cart[1][1];
  }
};

const char *primes(int order) { return order == 0 ? "" : (order == 1 ? "'" : "''"); }

void set_box(Keys &k, Lattice *lat, bool one_d) {
  long W, L;
  const bool hw = k.has("w"), hl = k.has("l");
  const bool hbox = k.has("a0w") || k.has("a0l") || k.has("a1w") || k.has("a1l");
  if (one_d) {
    if (hbox || hw) throw Fail("a one-dimensional lattice takes its length from L only");
    if (!k.integer("l", &L) || L < 1) throw Fail("L is needed (a positive integer)");
    lat->a[0][0] = L;
    lat->a[0][1] = 0;
    lat->a[1][0] = 0;
    lat->a[1][1] = 1;
    return;
  }
  if (hbox && (hw || hl)) throw Fail("give either W and L or a0W, a0L, a1W, a1L, not both");
  if (hbox) {
    lat->a[0][0] = k.int_or("a0w", 0);
    lat->a[0][1] = k.int_or("a0l", 0);
    lat->a[1][0] = k.int_or("a1w", 0);
    lat->a[1][1] = k.int_or("a1l", 0);
  } else {
    if (!k.integer("w", &W) || !k.integer("l", &L) || W < 1 || L < 1) throw Fail("W and L are needed");
    lat->a[0][0] = W;
    lat->a[0][1] = 0;
    lat->a[1][0] = 0;
    lat->a[1][1] = L;
  }
}

Lattice make_lattice(Keys &k, const std::string &name) {
  Lattice lat;
  const double h = std::sqrt(3.0) / 2.0;
  if (name == "chain" || name == "chainlattice") {
    lat.kind = "chain";
    set_box(k, &lat, true);
    lat.bonds = {{1, 0, 0, 0, 0, 0}, {2, 0, 0, 0, 0, 1}, {3, 0, 0, 0, 0, 2}};
  } else if (name == "ladder" || name == "ladderlattice") {
    lat.kind = "ladder";
    long W, L;
    if (!k.integer("w", &W) || !k.integer("l", &L) || W < 1 || L < 1) throw Fail("W and L are needed");
    lat.nsub = (int)W;
    lat.a[0][0] = L;
    lat.a[1][1] = 1;
    lat.cart[1][0] = 0.0;
    lat.cart[1][1] = 1.0;
    for (int w = 0; w < W; w++) {
      if (w + 1 < W) lat.bonds.push_back({0, 0, w, w + 1, 0, 0});  // rung J0
      lat.bonds.push_back({1, 0, w, w, 1, 0});                       // leg J1
      lat.bonds.push_back({2, 0, w, w, 1, 1});                       // leg, second neighbour J1'
      if (w + 1 < W) {
        lat.bonds.push_back({1, 0, w + 1, w, 2, 0});  // diagonal J2
        lat.bonds.push_back({1, 0, w, w + 1, 2, 1});  // other diagonal J2'
      }
    }
    if (W > 3) throw Fail("ladder: more than three legs is not supported");
  } else if (name == "square" || name == "squarelattice" || name == "tetragonal" || name == "tetragonallattice") {
    lat.kind = "square";
    set_box(k, &lat, false);
    lat.bonds = {{1, 0, 0, 0, 0, 0}, {0, 1, 0, 0, 1, 0}, {1, 1, 0, 0, 0, 1},
                 {1, -1, 0, 0, 1, 1}, {2, 0, 0, 0, 0, 2}, {0, 2, 0, 0, 1, 2}};
  } else if (name == "triangular" || name == "triangularlattice") {
    lat.kind = "triangular";
    set_box(k, &lat, false);
    lat.cart[1][0] = 0.5;
    lat.cart[1][1] = h;
    lat.bonds = {{1, 0, 0, 0, 0, 0},  {0, 1, 0, 0, 1, 0}, {-1, 1, 0, 0, 2, 0},
                 {-1, 2, 0, 0, 0, 1}, {2, -1, 0, 0, 1, 1}, {1, 1, 0, 0, 2, 1},
                 {2, 0, 0, 0, 0, 2},  {0, 2, 0, 0, 1, 2}, {-2, 2, 0, 0, 2, 2}};
  } else if (name == "honeycomb" || name == "honeycomblattice") {
    lat.kind = "honeycomb";
    set_box(k, &lat, false);
    lat.nsub = 2;
    lat.cart[1][0] = 0.5;
    lat.cart[1][1] = h;
    lat.tau[1][0] = lat.tau[1][1] = 1.0 / 3.0;
    // J0 from orbital 0 to 1 of the same cell; J1 and J2 from orbital 1 to orbital 0 of the
    // next cell along a0 / a1 (the direction matters for couplings J^{ab} != J^{ba})
    lat.bonds = {{0, 0, 0, 1, 0, 0}, {1, 0, 1, 0, 1, 0}, {0, 1, 1, 0, 2, 0}};
    for (int s = 0; s < 2; s++) {
      lat.bonds.push_back({-1, 1, s, s, 0, 1});
      lat.bonds.push_back({0, 1, s, s, 1, 1});
      lat.bonds.push_back({1, 0, s, s, 2, 1});
    }
    lat.bonds.push_back({-1, -1, 0, 1, 0, 2});
    lat.bonds.push_back({1, -1, 0, 1, 1, 2});
    lat.bonds.push_back({-1, 1, 0, 1, 2, 2});
  } else if (name == "kagome" || name == "kagomelattice") {
    lat.kind = "kagome";
    set_box(k, &lat, false);
    lat.nsub = 3;
    lat.cart[1][0] = 0.5;
    lat.cart[1][1] = h;
    lat.tau[1][0] = 0.5;
    lat.tau[2][1] = 0.5;
    lat.bonds = {{0, 0, 1, 2, 0, 0}, {-1, 1, 2, 1, 0, 0},   // J0: orbitals 1-2
                 {0, 0, 0, 2, 1, 0}, {0, -1, 0, 2, 1, 0},   // J1: orbitals 0-2
                 {0, 0, 0, 1, 2, 0}, {1, 0, 1, 0, 2, 0},    // J2: orbitals 0-1
                 {0, 1, 2, 1, 0, 1}, {1, 0, 1, 2, 0, 1},    // J0'
                 {1, -1, 0, 2, 1, 1}, {1, 0, 2, 0, 1, 1},   // J1'
                 {1, -1, 1, 0, 2, 1}, {0, 1, 1, 0, 2, 1}};  // J2'
  } else {
    throw Fail("lattice not supported: " + name +
               " (chain, ladder, square / tetragonal, triangular, honeycomb, kagome are)");
  }
  lat.build_cells();
  return lat;
}

// ----------------------------------------------------------------------------- model terms
struct Terms {
  int nsite = 0;
  std::vector<int> two_s;   // per site: 2S of a local spin, 0 for an electron orbital
  std::vector<std::tuple<int, int, int, int, cplx>> trans;
  std::map<std::array<int, 4>, size_t> trans_at;
  std::vector<std::pair<std::array<int, 8>, cplx>> intr;
  std::map<std::array<int, 8>, size_t> intr_at;
  std::vector<std::pair<int, double>> cintra;
  std::vector<std::tuple<int, int, double>> cinter;
  double weight = 0.0;      // coefficient sum behind the default LargeValue

  // H += -T c+_{i si} c_{j sj} (the sign convention of trans.def)
  void add_trans(int i, int si, int j, int sj, cplx T) {
    if (T == 0.0) return;
    weight += std::abs(T);
    const std::array<int, 4> key{i, si, j, sj};
    auto it = trans_at.find(key);
    if (it != trans_at.end()) {
      std::get<4>(trans[it->second]) += T;
    } else {
      trans_at[key] = trans.size();
      trans.emplace_back(i, si, j, sj, T);
    }
  }
  // H += X c+_{i a} c_{i b} c+_{j c} c_{j d}; `count` false leaves the coefficient sum alone
  void add_intr(int i, int a, int ib, int b, int j, int c, int jd, int d, cplx X, bool count = true) {
    if (std::abs(X) < 1e-15) return;
    if (count) weight += std::abs(X);
    const std::array<int, 8> key{i, a, ib, b, j, c, jd, d};
    auto it = intr_at.find(key);
    if (it != intr_at.end()) {
      intr[it->second].second += X;
    } else {
      intr_at[key] = intr.size();
      intr.emplace_back(key, X);
    }
  }
};

using JMat = std::array<std::array<double, 3>, 3>;  // J[a][b] of S_i^a S_j^b, a, b = x, y, z

bool jmat_zero(const JMat &J) {
  for (auto &r : J)
    for (double x : r)
      if (x != 0.0) return false;
  return true;
}

// m of spin state s (s = 0 is m = S) and the ladder factors.
double m_of(int two_s, int s) { return 0.5 * two_s - s; }
double raise_amp(int two_s, int s) {  // <s-1| S+ |s>
  const double S = 0.5 * two_s, m = m_of(two_s, s);
  return std::sqrt(S * (S + 1.0) - m * (m + 1.0));
}
double lower_amp(int two_s, int s) {  // <s+1| S- |s>
  const double S = 0.5 * two_s, m = m_of(two_s, s);
  return std::sqrt(S * (S + 1.0) - m * (m - 1.0));
}

// H += sum_ab J[a][b] S_i^a S_j^b between spins 2S = ti, tj (an electron orbital enters with
// tj = 1 and its spin s = c+ sigma c / 2), written as InterAll terms.  Each off-diagonal term
// X c+_{i a} c_{i b} c+_{j c} c_{j d} is followed by its Hermitian partner in reversed order,
// X* c+_{j d} c_{j c} c+_{i b} c_{i a}, the pairing the reference's InterAll check expects
// (src/readdef.c:2257-2320).
void add_spin_coupling(Terms *T, int i, int ti, int j, int tj, const JMat &J) {
  if (i == j) {
    // a bond from a site to itself (a period-1 direction): the one-site operator
    // sum_ab J[a][b] S^a S^b, written as transfers between the spin states
    const int n = ti + 1;
    auto S = [&](int a, int r, int c) -> cplx {  // <r| S^a |c>
      const double mc = m_of(ti, c);
      const double up = (r == c - 1) ? raise_amp(ti, c) : 0.0;   // S+
      const double dn = (r == c + 1) ? lower_amp(ti, c) : 0.0;   // S-
      if (a == 0) return 0.5 * (up + dn);
      if (a == 1) return cplx(0.0, -0.5) * (up - dn);
      return r == c ? mc : 0.0;
    };
    for (int r = 0; r < n; r++)
      for (int c = 0; c < n; c++) {
        cplx m = 0.0;
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) {
            if (J[a][b] == 0.0) continue;
            for (int q = 0; q < n; q++) m += J[a][b] * S(a, r, q) * S(b, q, c);
          }
        if (std::abs(m) > 1e-15) T->add_trans(i, r, i, c, -m);
      }
    return;
  }
  const double xx = J[0][0], yy = J[1][1], zz = J[2][2];
  const double xy = J[0][1], yx = J[1][0], xz = J[0][2], zx = J[2][0], yz = J[1][2], zy = J[2][1];
  const cplx I(0.0, 1.0);
  const cplx pm = 0.25 * (xx + yy + I * (xy - yx));   // S+_i S-_j (partner S-_i S+_j)
  const cplx pp = 0.25 * (xx - yy - I * (xy + yx));   // S+_i S+_j (partner S-_i S-_j)
  const cplx pz = 0.5 * (xz - I * yz);                // S+_i Sz_j (partner S-_i Sz_j)
  const cplx zp = 0.5 * (zx - I * zy);                // Sz_i S+_j (partner Sz_i S-_j)
  const bool diag_half = ti == 1 && tj == 1 && xy == 0 && yx == 0 && xz == 0 && zx == 0 && yz == 0 && zy == 0;
  if (diag_half) T->weight += 1.25 * std::abs(zz) + 0.5 * std::abs(xx + yy) + 0.5 * std::abs(xx - yy);
  const bool count = !diag_half;
  auto pair = [&](int a, int b, int c, int d, cplx X) {
    T->add_intr(i, a, i, b, j, c, j, d, X, count);
    T->add_intr(j, d, j, c, i, b, i, a, std::conj(X), count);
  };
  for (int a = 0; a <= ti; a++) {
    const double mi = m_of(ti, a);
    for (int b = 0; b <= tj; b++) {
      const double mj = m_of(tj, b);
      T->add_intr(i, a, i, a, j, b, j, b, zz * mi * mj, count);
      if (a > 0 && b < tj) pair(a - 1, a, b + 1, b, pm * raise_amp(ti, a) * lower_amp(tj, b));
      if (a > 0 && b > 0) pair(a - 1, a, b - 1, b, pp * raise_amp(ti, a) * raise_amp(tj, b));
      if (a > 0) pair(a - 1, a, b, b, pz * raise_amp(ti, a) * mj);
      if (b > 0) pair(a, a, b - 1, b, zp * mi * raise_amp(tj, b));
    }
  }
}

// The coupling matrix of bond direction `label`, neighbour order `order`: J<label><primes> and
// its components J<label><primes><x|y|z|xy|...>, else the direction-free forms J<primes>...
JMat bond_jmat(Keys &k, int label, int order, bool simplified_ok) {
  static const char *comp[9] = {"x", "y", "z", "xy", "yx", "xz", "zx", "yz", "zy"};
  static const int ab[9][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {1, 0}, {0, 2}, {2, 0}, {1, 2}, {2, 1}};
  const std::string p = primes(order);
  auto read = [&](const std::string &base, JMat *J) {
    bool any = false;
    double v;
    const bool iso = k.real(base, &v);
    if (iso) {
      (*J)[0][0] = (*J)[1][1] = (*J)[2][2] = v;
      any = true;
    }
    for (int c = 0; c < 9; c++) {
      double x;
      if (k.real(base + comp[c], &x)) {
        if (iso && c < 3) throw Fail("give either " + base + " or its diagonal components, not both");
        (*J)[ab[c][0]][ab[c][1]] = x;
        any = true;
      }
    }
    return any;
  };
  JMat J{}, Js{};
  const bool have = read("j" + std::to_string(label) + p, &J);
  const bool have_s = simplified_ok && read("j" + p, &Js);
  if (have && have_s) throw Fail("give either J" + p + " or the direction-resolved J0" + p + ", J1" + p + "..., not both");
  return have ? J : Js;
}

cplx bond_complex(Keys &k, const std::string &base, int label, int order, bool simplified_ok) {
  const std::string p = primes(order);
  cplx v(0.0), vs(0.0);
  const bool have = k.complex(base + std::to_string(label) + p, &v);
  const bool have_s = simplified_ok && k.complex(base + p, &vs);
  if (have && have_s) throw Fail("give either " + base + p + " or " + base + "0" + p + ", " + base + "1" + p + "..., not both");
  return have ? v : vs;
}

// ----------------------------------------------------------------------------- writers
void write_table_head(FILE *f, const char *what, size_t n) {
  std::fprintf(f, "========================\n%s %zu\n========================\n"
                  "========================\n========================\n", what, n);
}

FILE *open_out(const std::string &dir, const std::string &name) {
  FILE *f = std::fopen((dir + "/" + name).c_str(), "w");
  if (!f) throw Fail("cannot write " + dir + "/" + name);
  return f;
}

enum ModelKind { kHubbardM, kSpinM, kKondoM };

struct Plan {
  ModelKind model;
  bool gc = false;
  int calc_type = 0;
  Lattice lat;
  Terms terms;
  int nc = 0;                 // orbitals of the lattice (= cells * orbitals per cell)
  int two_s = 1;
  std::vector<std::tuple<int, int, int, cplx>> single;          // i, s, type (0: c, 1: c+), coefficient
  std::vector<std::tuple<int, int, int, int, int, cplx>> pair;  // i, s1, j, s2, type (1: c+c, 0: c c+), coefficient
  std::vector<std::array<int, 4>> green1;
  std::vector<std::array<int, 8>> green2;
  bool full_green = false;
  bool no_green = false;
  // local spins of a Kondo lattice come first: itinerant orbital n is site nc + n
  int orb_site(int n) const { return model == kKondoM ? nc + n : n; }
  bool is_local(int site) const { return terms.two_s[site] != 0; }
  int nstates(int site) const { return is_local(site) ? terms.two_s[site] + 1 : 2; }
};

// ----------------------------------------------------------------------------- spectra
// The excitation operator A of a dynamical Green's function <A+ (z - H)^-1 A>:
// A = sum_i exp(i q.r_i) O_i with q = 2 pi (SpectrumQW, SpectrumQL) in units of the reciprocal
// lattice and r_i the fractional position of site i: cell plus orbital offset (honeycomb
// orbital 1 at (1/3, 1/3); kagome orbitals 1, 2 at (1/2, 0), (0, 1/2)); for a ladder, the rung
// index along the legs and leg / W across them; for a chain, the site along it (SpectrumQL).
// O_i = S^z_i (SzSz), S^-_i (S+S-), n_i (Density; the identity of a spin site), c_{i up} (Up),
// c_{i down} (Down); a Kondo lattice's spin operators act on its local spins and conduction
// orbitals together.
void make_excitation(Plan *P, const std::string &type, double qw, double ql) {
  const Lattice &lat = P->lat;
  auto phase = [&](int n) {  // n: orbital index of the lattice (cell * nsub + orbital)
    const int c = n / lat.nsub, s = n % lat.nsub;
    double x;
    if (lat.kind == "chain") x = ql * lat.cells[c][0];
    else if (lat.kind == "ladder") x = ql * lat.cells[c][0] + qw * s / (double)lat.nsub;
    else x = qw * (lat.cells[c][0] + lat.tau[s][0]) + ql * (lat.cells[c][1] + lat.tau[s][1]);
    return std::polar(1.0, 2.0 * kPi * x);
  };
  for (int n = 0; n < P->nc; n++) {
    const cplx f = phase(n);
    const bool spin_site = P->model != kHubbardM;  // spins, and the local spins of a Kondo lattice
    const int o = P->orb_site(n);
    if (type == "szsz") {
      if (spin_site)
        for (int a = 0; a <= P->two_s; a++) P->pair.emplace_back(n, a, n, a, 1, f * m_of(P->two_s, a));
      if (P->model != kSpinM)
        for (int a = 0; a < 2; a++) P->pair.emplace_back(o, a, o, a, 1, f * (a == 0 ? 0.5 : -0.5));
    } else if (type == "s+s-") {
      if (spin_site)
        for (int a = 0; a < P->two_s; a++) P->pair.emplace_back(n, a + 1, n, a, 1, f * lower_amp(P->two_s, a));
      if (P->model != kSpinM) P->pair.emplace_back(o, 1, o, 0, 1, f);
    } else if (type == "density") {
      if (P->model == kSpinM)
        for (int a = 0; a <= P->two_s; a++) P->pair.emplace_back(n, a, n, a, 1, f);
      else
        for (int a = 0; a < 2; a++) P->pair.emplace_back(o, a, o, a, 1, f);
    } else if (type == "up" || type == "down") {
      if (P->model == kSpinM) throw Fail("SpectrumType " + type + " needs electrons");
      P->single.emplace_back(o, type == "up" ? 0 : 1, 0, f);
    } else {
      throw Fail("SpectrumType: SzSz, S+S-, Density, Up or Down");
    }
  }
}

// ----------------------------------------------------------------------------- correlation lists
void make_green(Plan *P) {
  const int N = P->terms.nsite;
  if (P->no_green) return;
  if (P->full_green) {
    // every <c+_{i s1} c_{j s2}> (spins: i == j; Kondo: no pair of two different local spins)
    for (int i = 0; i < N; i++)
      for (int s1 = 0; s1 < P->nstates(i); s1++)
        for (int j = 0; j < N; j++) {
          if (i != j && (P->model == kSpinM || (P->is_local(i) && P->is_local(j)))) continue;
          for (int s2 = 0; s2 < P->nstates(j); s2++) P->green1.push_back({i, s1, j, s2});
        }
    for (const auto &g : P->green1)
      for (const auto &h : P->green1) P->green2.push_back({g[0], g[1], g[2], g[3], h[0], h[1], h[2], h[3]});
    return;
  }
  // Correlation functions of the Fourier utility (doc/en/source/fourier/format.rst): from the
  // orbitals of the first unit cell to every site, <c+_{0a s} c_{Rb s}>, <n_{0a s} n_{Rb s'}>
  // and <c+_{0a s} c_{0a -s} c+_{Rb -s} c_{Rb s}>.
  const int per_cell = P->lat.nsub;
  std::vector<int> first;
  for (int a = 0; a < per_cell; a++) {
    if (P->model == kKondoM) first.push_back(a);
    first.push_back(P->orb_site(a));
  }
  std::sort(first.begin(), first.end());
  for (int i : first)
    for (int j = 0; j < N; j++) {
      if (P->is_local(i) != P->is_local(j)) continue;
      if (P->is_local(i) && i != j) continue;
      for (int s = 0; s < std::min(P->nstates(i), P->nstates(j)); s++) P->green1.push_back({i, s, j, s});
    }
  for (int i : first)
    for (int j = 0; j < N; j++) {
      if (P->is_local(i) != P->is_local(j)) continue;
      for (int s = 0; s < P->nstates(i); s++)
        for (int t = 0; t < P->nstates(j); t++) P->green2.push_back({i, s, i, s, j, t, j, t});
      if (P->nstates(i) == 2 && P->nstates(j) == 2)
        for (int s = 0; s < 2; s++) P->green2.push_back({i, s, i, 1 - s, j, 1 - s, j, s});
    }
}

}  // namespace

int generate(const std::string &stan_in, const std::string &dir, std::string *err) {
  try {
    Keys k;
    k.load(stan_in);
    Plan P;
    // ---------------------------------------------------------------- model / method
    const std::string model = k.str_or("model", "");
    if (model == "hubbard" || model == "fermionhubbard") P.model = kHubbardM;
    else if (model == "hubbardgc" || model == "fermionhubbardgc") { P.model = kHubbardM; P.gc = true; }
    else if (model == "spin") P.model = kSpinM;
    else if (model == "spingc" || model == "spingccma") {
      // SpinGCCMA is the SpinGC Hamiltonian computed by the reference's cluster-multiplication
      // algorithm; the engine's general kernel computes the same system
      P.model = kSpinM;
      P.gc = true;
    }
    else if (model == "kondo" || model == "kondolattice") P.model = kKondoM;
    else if (model == "kondogc" || model == "kondolatticegc") { P.model = kKondoM; P.gc = true; }
    else throw Fail("model not supported: '" + model + "' (Hubbard, Spin, Kondo, their GC forms and SpinGCCMA are)");
    const std::string method = k.str_or("method", "");
    if (method == "lanczos") P.calc_type = 0;
    else if (method == "tpq") P.calc_type = 1;
    else if (method == "fulldiag" || method == "alldiag") P.calc_type = 2;
    else if (method == "cg" || method == "lobcg" || method == "lobpcg") P.calc_type = 3;
    else if (method == "timeevolution" || method == "time-evolution") P.calc_type = 4;
    else if (method == "ctpq") P.calc_type = 5;
    else throw Fail("method not supported: '" + method + "'");
    const std::string lattice = k.str_or("lattice", "");
    P.lat = make_lattice(k, lattice);
    const Lattice &lat = P.lat;
    const int ncell = lat.ncell();
    P.nc = ncell * lat.nsub;
    P.two_s = (int)k.int_or("2s", 1);
    if (P.two_s < 1) throw Fail("2S must be positive");
    if (P.model == kKondoM && P.two_s != 1) throw Fail("Kondo lattices with local spins 2S > 1 are not supported");
    if (P.model == kHubbardM && k.has("2s")) throw Fail("2S is a parameter of spin and Kondo models");
    Terms &T = P.terms;
    T.nsite = P.model == kKondoM ? 2 * P.nc : P.nc;
    T.two_s.assign(T.nsite, 0);
    if (P.model == kSpinM) std::fill(T.two_s.begin(), T.two_s.end(), P.two_s);
    if (P.model == kKondoM) std::fill(T.two_s.begin(), T.two_s.begin() + P.nc, P.two_s);

    const double phase[2] = {k.real_or("phase0", 0.0), k.real_or("phase1", 0.0)};
    const bool simplified_ok = lat.kind != "ladder";
    // Time evolution: PumpType "Quench" adds U_quench sum_i n_i,up n_i,down to H for t >= 0;
    // the lasers replace every hopping by its Peierls-substituted form at each time step.
    std::string pump;
    if (P.calc_type == 4) {
      pump = k.str_or("pumptype", "quench");
      if (pump != "quench" && pump != "pulselaser" && pump != "aclaser" && pump != "dclaser")
        throw Fail("PumpType: Quench, Pulse Laser, AC Laser or DC Laser");
      if (P.model == kSpinM) throw Fail("time evolution from the standard mode needs electrons");
    }
    const bool laser = P.calc_type == 4 && pump != "quench";
    struct Hop {
      int oi, oj;      // H gets -t c+_{oj s} c_{oi s} + h.c.
      cplx t;
      double dr[2];    // r_oj - r_oi, fractional
    };
    std::vector<Hop> hops;

    // ---------------------------------------------------------------- one-site terms
    const double mu = (P.model == kSpinM) ? 0.0 : k.real_or("mu", 0.0);
    const double U = (P.model == kSpinM) ? 0.0 : k.real_or("u", 0.0);
    const double hfield = k.real_or("h", 0.0);
    const double gamma = k.real_or("gamma", 0.0);
    const double D = (P.model == kSpinM) ? k.real_or("d", 0.0) : 0.0;
    for (int n = 0; n < P.nc; n++) {
      if (P.model != kHubbardM) {  // spins, and the local spins of a Kondo lattice
        const int ts = P.two_s;
        for (int s = 0; s <= ts; s++) {
          const double m = m_of(ts, s);
          T.add_trans(n, s, n, s, hfield * m - D * m * m);
        }
        for (int s = 1; s <= ts; s++) {
          T.add_trans(n, s - 1, n, s, 0.5 * gamma * raise_amp(ts, s));
          T.add_trans(n, s, n, s - 1, 0.5 * gamma * lower_amp(ts, s - 1));
        }
      }
      if (P.model != kSpinM) {
        const int o = P.orb_site(n);
        T.add_trans(o, 0, o, 0, mu + 0.5 * hfield);
        T.add_trans(o, 1, o, 1, mu - 0.5 * hfield);
        T.add_trans(o, 0, o, 1, 0.5 * gamma);
        T.add_trans(o, 1, o, 0, 0.5 * gamma);
        if (U != 0.0) {
          T.cintra.emplace_back(o, U);
          T.weight += std::abs(U);
        }
      }
    }
    if (P.model == kKondoM) {
      // Kondo coupling J S_n . s_n between local spin n and its conduction orbital
      JMat J{};
      static const char *comp[9] = {"x", "y", "z", "xy", "yx", "xz", "zx", "yz", "zy"};
      static const int ab[9][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {1, 0}, {0, 2}, {2, 0}, {1, 2}, {2, 1}};
      double v;
      const bool iso = k.real("j", &v);
      if (iso) J[0][0] = J[1][1] = J[2][2] = v;
      for (int c = 0; c < 9; c++) {
        double x;
        if (k.real(std::string("j") + comp[c], &x)) {
          if (iso && c < 3) throw Fail("give either J or Jx, Jy, Jz, not both");
          J[ab[c][0]][ab[c][1]] = x;
        }
      }
      if (!jmat_zero(J))
        for (int n = 0; n < P.nc; n++) add_spin_coupling(&T, n, P.two_s, P.orb_site(n), 1, J);
    }

    // ---------------------------------------------------------------- bonds
    for (int c = 0; c < ncell; c++) {
      const long w = lat.cells[c][0], l = lat.cells[c][1];
      for (const BondType &b : lat.bonds) {
        long n0, n1;
        const int c2 = lat.fold(w + b.dw, l + b.dl, &n0, &n1);
        const int i = c * lat.nsub + b.si, j = c2 * lat.nsub + b.sj;
        if (P.model == kSpinM) {
          const JMat J = bond_jmat(k, b.label, b.order, simplified_ok);
          if (!jmat_zero(J)) add_spin_coupling(&T, i, P.two_s, j, P.two_s, J);
        } else {
          const cplx t = bond_complex(k, "t", b.label, b.order, simplified_ok);
          const double th = (phase[0] * n0 + phase[1] * n1) * kPi / 180.0;
          const cplx te = t * std::polar(1.0, th);
          const int oi = P.orb_site(i), oj = P.orb_site(j);
          if (laser && te != 0.0) {
            const double dr0 = b.dw + lat.tau[b.sj][0] - lat.tau[b.si][0];
            const double dr1 = b.dl + lat.tau[b.sj][1] - lat.tau[b.si][1];
            hops.push_back({oi, oj, te, {dr0, dr1}});
            continue;
          }
          for (int s = 0; s < 2; s++) {
            T.add_trans(oj, s, oi, s, te);
            T.add_trans(oi, s, oj, s, std::conj(te));
          }
          const cplx V = bond_complex(k, "v", b.label, b.order, simplified_ok);
          if (V.imag() != 0.0) throw Fail("V is real");
          if (V.real() != 0.0) {
            T.cinter.emplace_back(oi, oj, V.real());
            T.weight += std::abs(V.real());
          }
        }
      }
    }
    // parameters read for other models are errors rather than silently unused
    if (P.model != kSpinM) {
      for (int lbl = 0; lbl < 3; lbl++)
        for (int o = 0; o < 3; o++) {
          JMat J = bond_jmat(k, lbl, o, simplified_ok && !(P.model == kKondoM && o == 0));
          if (!jmat_zero(J)) throw Fail("bond spin couplings J0, J1, ... belong to the spin model");
        }
    }

    // ---------------------------------------------------------------- numerical conditions
    const int nsite = T.nsite;
    double large_value = T.weight / nsite;
    k.real("largevalue", &large_value);
    long lanczos_max = k.int_or("lanczos_max", 2000);
    const long initial_iv = k.int_or("initial_iv", -1);
    const long exct = k.int_or("exct", 1);
    const long lanczos_eps = k.int_or("lanczoseps", 14);
    const long lanczos_target = k.int_or("lanczostarget", 2);
    const long num_ave = k.int_or("numave", 5);
    const long expec_interval = k.int_or("expecinterval", 20);
    const long n_omega = k.int_or("nomega", 200);
    const long expand_coef = k.int_or("expandcoef", 10);
    const double omega_max = k.real_or("omegamax", large_value * nsite);
    const double omega_min = k.real_or("omegamin", -large_value * nsite);
    const double omega_org = k.real_or("omegaorg", 0.0);
    const double omega_im = k.real_or("omegaim", 0.01 * large_value);

    long nelec = -1, two_sz = 0;
    const bool have_nelec = k.integer("nelec", &nelec) || k.integer("ncond", &nelec);
    const bool have_2sz = k.integer("2sz", &two_sz);
    if (P.gc && (have_nelec || have_2sz)) throw Fail("nelec and 2Sz are not parameters of grand-canonical models");
    if (!P.gc) {
      if (P.model == kSpinM) {
        if (have_nelec) throw Fail("nelec is not a parameter of the spin model");
        if (!have_2sz) throw Fail("2Sz is needed for the canonical spin model");
      } else if (!have_nelec) {
        throw Fail("nelec is needed for canonical Hubbard and Kondo models");
      } else if (P.model == kKondoM && !have_2sz) {
        throw Fail("2Sz is needed for the canonical Kondo model");
      }
    }
    const std::string outputmode = k.str_or("outputmode", "corr");
    if (outputmode == "none") P.no_green = true;
    else if (outputmode == "all" || outputmode == "full" || outputmode == "raw") P.full_green = true;
    else if (outputmode != "corr" && outputmode != "correlation") throw Fail("OutputMode: none, correlation or full");

    auto pick = [&](const std::string &key, const std::map<std::string, int> &m, int def) {
      std::string s;
      if (!k.str(key, &s)) return def;
      auto it = m.find(s);
      if (it == m.end()) throw Fail("keyword " + key + ": unknown value " + s);
      return it->second;
    };
    const int restart = pick("restart", {{"none", 0}, {"restart_out", 1}, {"save", 1}, {"restartsave", 2},
                                         {"restart", 2}, {"restart_in", 3}}, 0);
    const int calc_spec = pick("calcspec", {{"none", 0}, {"normal", 1}, {"noiteration", 2}, {"restart_out", 3},
                                            {"restart_in", 4}, {"restartsave", 5}, {"restart", 5}}, 0);
    const int ivtype = pick("initialvectype", {{"c", 0}, {"r", 1}}, 0);
    const int eigio = pick("eigenvecio", {{"none", 0}, {"in", 1}, {"out", 2}}, 0);
    const int hamio = pick("hamio", {{"none", 0}, {"in", 1}, {"out", 2}}, 0);
    const int exvec = pick("outputexcitedvec", {{"none", 0}, {"out", 1}}, 0);

    // time-dependent terms, one list per step at t = step * dt (src/CalcByTEM.c:141-165 reads
    // them as TETime / TEOneBody / TETwoBody); the vector potential of a laser is
    // A0 exp(-(t - t0)^2 / (2 tdump^2)) cos(freq (t - t0)) (Pulse), A0 sin(freq (t - t0)) (AC) or
    // A0 t (DC), with A0 = (VecPotW, VecPotL) and t0 = tshift
    std::vector<std::pair<double, std::vector<std::tuple<int, int, int, int, cplx>>>> te_one;
    std::vector<std::pair<double, std::vector<std::pair<std::array<int, 8>, cplx>>>> te_two;
    if (P.calc_type == 4) {
      const double dt = k.real_or("dt", 0.1), tshift = k.real_or("tshift", 0.0), tdump = k.real_or("tdump", 0.1);
      const double freq = k.real_or("freq", 0.1), uquench = k.real_or("uquench", 0.0);
      const double A0[2] = {k.real_or("vecpotw", 0.0), k.real_or("vecpotl", 0.0)};
      for (long step = 0; step < lanczos_max; step++) {
        const double t = dt * step;
        const double ta = t;
        if (!laser) {
          std::vector<std::pair<std::array<int, 8>, cplx>> rows;
          if (uquench != 0.0)
            for (int n = 0; n < P.nc; n++) {
              const int o = P.orb_site(n);
              rows.push_back({{o, 0, o, 0, o, 1, o, 1}, uquench});
            }
          te_two.push_back({t, rows});
          continue;
        }
        double a;  // A(t) / A0
        if (pump == "pulselaser") a = std::exp(-(ta - tshift) * (ta - tshift) / (2.0 * tdump * tdump)) * std::cos(freq * (ta - tshift));
        else if (pump == "aclaser") a = std::sin(freq * (ta - tshift));
        else a = ta;
        std::vector<std::tuple<int, int, int, int, cplx>> rows;
        for (const Hop &h : hops) {
          // A(t) = A0 a(t) in units of the reciprocal lattice vectors: the hop from r_i to r_j
          // picks up exp(i A(t).(r_j - r_i) / 2 pi) = exp(i a(t) (A0W dr_W + A0L dr_L))
          const cplx te = h.t * std::polar(1.0, a * (A0[0] * h.dr[0] + A0[1] * h.dr[1]));
          for (int s = 0; s < 2; s++) {
            rows.emplace_back(h.oj, s, h.oi, s, te);
            rows.emplace_back(h.oi, s, h.oj, s, std::conj(te));
          }
        }
        te_one.push_back({t, rows});
      }
    }
    const std::string spectrum_type = k.str_or("spectrumtype", "szsz");
    const double qw = k.real_or("spectrumqw", 0.0), ql = k.real_or("spectrumql", 0.0);
    if (calc_spec != 0) make_excitation(&P, spectrum_type, qw, ql);

    make_green(&P);
    k.check_all_used();

    // ---------------------------------------------------------------- files
    std::vector<std::pair<std::string, std::string>> names;
    names.push_back({"ModPara", "modpara.def"});
    names.push_back({"LocSpin", "locspn.def"});
    {
      FILE *f = open_out(dir, "locspn.def");
      int nloc = 0;
      for (int s : T.two_s) nloc += s != 0;
      write_table_head(f, "NlocalSpin", nloc);
      for (int i = 0; i < nsite; i++) std::fprintf(f, "%5d %5d\n", i, T.two_s[i]);
      std::fclose(f);
    }
    {
      std::vector<std::tuple<int, int, int, int, cplx>> tr;
      for (const auto &e : T.trans)
        if (std::abs(std::get<4>(e)) > 1e-15) tr.push_back(e);
      FILE *f = open_out(dir, "trans.def");
      write_table_head(f, "NTransfer", tr.size());
      for (const auto &e : tr)
        std::fprintf(f, "%5d %5d %5d %5d %25.15f %25.15f\n", std::get<0>(e), std::get<1>(e), std::get<2>(e),
                     std::get<3>(e), std::get<4>(e).real(), std::get<4>(e).imag());
      std::fclose(f);
      names.push_back({"Trans", "trans.def"});
    }
    if (!T.cintra.empty()) {
      FILE *f = open_out(dir, "coulombintra.def");
      write_table_head(f, "NCoulombIntra", T.cintra.size());
      for (const auto &e : T.cintra) std::fprintf(f, "%5d %25.15f\n", e.first, e.second);
      std::fclose(f);
      names.push_back({"CoulombIntra", "coulombintra.def"});
    }
    if (!T.cinter.empty()) {
      FILE *f = open_out(dir, "coulombinter.def");
      write_table_head(f, "NCoulombInter", T.cinter.size());
      for (const auto &e : T.cinter)
        std::fprintf(f, "%5d %5d %25.15f\n", std::get<0>(e), std::get<1>(e), std::get<2>(e));
      std::fclose(f);
      names.push_back({"CoulombInter", "coulombinter.def"});
    }
    {
      std::vector<std::pair<std::array<int, 8>, cplx>> in;
      for (const auto &e : T.intr)
        if (std::abs(e.second) > 1e-15) in.push_back(e);
      if (!in.empty()) {
        FILE *f = open_out(dir, "interall.def");
        write_table_head(f, "NInterAll", in.size());
        for (const auto &e : in) {
          for (int q = 0; q < 8; q++) std::fprintf(f, "%5d ", e.first[q]);
          std::fprintf(f, "%25.15f %25.15f\n", e.second.real(), e.second.imag());
        }
        std::fclose(f);
        names.push_back({"InterAll", "interall.def"});
      }
    }
    if (!P.no_green) {
      FILE *f = open_out(dir, "greenone.def");
      write_table_head(f, "NCisAjs", P.green1.size());
      for (const auto &g : P.green1) std::fprintf(f, "%5d %5d %5d %5d\n", g[0], g[1], g[2], g[3]);
      std::fclose(f);
      f = open_out(dir, "greentwo.def");
      write_table_head(f, "NCisAjsCktAltDC", P.green2.size());
      for (const auto &g : P.green2)
        std::fprintf(f, "%5d %5d %5d %5d %5d %5d %5d %5d\n", g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7]);
      std::fclose(f);
      names.push_back({"OneBodyG", "greenone.def"});
      names.push_back({"TwoBodyG", "greentwo.def"});
    }
    names.push_back({"CalcMod", "calcmod.def"});
    if (!P.single.empty()) {
      FILE *f = open_out(dir, "single.def");
      write_table_head(f, "NSingle", P.single.size());
      for (const auto &e : P.single)
        std::fprintf(f, "%5d %5d %5d %25.15f %25.15f\n", std::get<0>(e), std::get<1>(e), std::get<2>(e),
                     std::get<3>(e).real(), std::get<3>(e).imag());
      std::fclose(f);
      names.push_back({"SingleExcitation", "single.def"});
    }
    if (!P.pair.empty()) {
      FILE *f = open_out(dir, "pair.def");
      write_table_head(f, "NPair", P.pair.size());
      for (const auto &e : P.pair)
        std::fprintf(f, "%5d %5d %5d %5d %5d %25.15f %25.15f\n", std::get<0>(e), std::get<1>(e), std::get<2>(e),
                     std::get<3>(e), std::get<4>(e), std::get<5>(e).real(), std::get<5>(e).imag());
      std::fclose(f);
      names.push_back({"PairExcitation", "pair.def"});
    }
    if (!te_one.empty()) {
      FILE *f = open_out(dir, "teone.def");
      write_table_head(f, "AllTimeStep", te_one.size());
      for (const auto &st : te_one) {
        std::fprintf(f, "%.15f %zu\n", st.first, st.second.size());
        for (const auto &e : st.second)
          std::fprintf(f, "%5d %5d %5d %5d %25.15f %25.15f\n", std::get<0>(e), std::get<1>(e), std::get<2>(e),
                       std::get<3>(e), std::get<4>(e).real(), std::get<4>(e).imag());
      }
      std::fclose(f);
      names.push_back({"TEOneBody", "teone.def"});
    }
    if (!te_two.empty()) {
      FILE *f = open_out(dir, "tetwo.def");
      write_table_head(f, "AllTimeStep", te_two.size());
      for (const auto &st : te_two) {
        std::fprintf(f, "%.15f %zu\n", st.first, st.second.size());
        for (const auto &e : st.second) {
          for (int q = 0; q < 8; q++) std::fprintf(f, "%5d ", e.first[q]);
          std::fprintf(f, "%25.15f %25.15f\n", e.second.real(), e.second.imag());
        }
      }
      std::fclose(f);
      names.push_back({"TETwoBody", "tetwo.def"});
    }
    if (calc_spec != 0 || P.calc_type == 4) names.push_back({"SpectrumVec", "zvo_eigenvec_0"});
    {
      int calc_model;
      if (P.model == kHubbardM) calc_model = P.gc ? 3 : 0;
      else if (P.model == kSpinM) calc_model = P.gc ? 4 : 1;
      else calc_model = P.gc ? 5 : 2;
      FILE *f = open_out(dir, "calcmod.def");
      std::fprintf(f, "#CalcType = 0:Lanczos, 1:TPQCalc, 2:FullDiag, 3:CG, 4:Time-evolution, 5:cTPQ\n");
      std::fprintf(f, "#CalcModel = 0:Hubbard, 1:Spin, 2:Kondo, 3:HubbardGC, 4:SpinGC, 5:KondoGC\n");
      std::fprintf(f, "#Restart = 0:None, 1:Save, 2:Restart&Save, 3:Restart\n");
      std::fprintf(f, "#CalcSpec = 0:None, 1:Normal, 2:No H*Phi, 3:Save, 4:Restart, 5:Restart&Save\n");
      std::fprintf(f, "CalcType %3d\nCalcModel %3d\nReStart %3d\nCalcSpec %3d\n", P.calc_type, calc_model, restart,
                   calc_spec);
      std::fprintf(f, "CalcEigenVec %3d\nInitialVecType %3d\nInputEigenVec %3d\nOutputEigenVec %3d\n", 0, ivtype,
                   eigio == 1 ? 1 : 0, eigio == 2 ? 1 : 0);
      std::fprintf(f, "InputHam %3d\nOutputHam %3d\nOutputExVec %3d\n", hamio == 1 ? 1 : 0, hamio == 2 ? 1 : 0,
                   exvec);
      std::fclose(f);
    }
    {
      FILE *f = open_out(dir, "modpara.def");
      std::fprintf(f, "--------------------\nModel_Parameters   0\n--------------------\nHPhi_Cal_Parameters\n"
                      "--------------------\nCDataFileHead  zvo\nCParaFileHead  zqp\n--------------------\n");
      std::fprintf(f, "Nsite          %d\n", nsite);
      if (!P.gc && P.model != kSpinM) std::fprintf(f, "Ncond          %ld\n", nelec);
      if (!P.gc && have_2sz) std::fprintf(f, "2Sz            %ld\n", two_sz);
      std::fprintf(f, "Lanczos_max    %ld\ninitial_iv     %ld\nexct           %ld\nLanczosEps     %ld\n", lanczos_max,
                   initial_iv, exct, lanczos_eps);
      std::fprintf(f, "LanczosTarget  %ld\nLargeValue     %.15e\nNumAve         %ld\nExpecInterval  %ld\n",
                   lanczos_target, large_value, num_ave, expec_interval);
      std::fprintf(f, "NOmega         %ld\n", n_omega);
      std::fprintf(f, "ExpandCoef     %ld\n", expand_coef);
      std::fprintf(f, "OmegaMax       %.15e %.15e\n", omega_max + omega_org, omega_im);
      std::fprintf(f, "OmegaMin       %.15e %.15e\n", omega_min + omega_org, omega_im);
      std::fprintf(f, "OmegaOrg       %.15e %.15e\n", omega_org, 0.0);
      std::fclose(f);
    }
    {
      // geometry.dat for HPhi's Fourier utility (doc/en/source/fourier/format.rst): the unit
      // lattice vectors, the boundary phases, the three integer vectors of the numerical cell
      // and, per site, its cell (W, L, H) and orbital (a Kondo lattice's conduction orbitals
      // follow its local spins as orbitals nsub .. 2 nsub - 1).  The k path the utility also
      // reads is the user's to append.
      FILE *f = open_out(dir, "geometry.dat");
      for (int d = 0; d < 2; d++) std::fprintf(f, "%25.15e %25.15e %25.15e\n", lat.cart[d][0], lat.cart[d][1], 0.0);
      std::fprintf(f, "%25.15e %25.15e %25.15e\n", 0.0, 0.0, 1.0);
      std::fprintf(f, "%25.15e %25.15e %25.15e\n", phase[0], phase[1], 0.0);
      for (int d = 0; d < 2; d++) std::fprintf(f, "%ld %ld %d\n", lat.a[d][0], lat.a[d][1], 0);
      std::fprintf(f, "0 0 1\n");
      const int copies = P.model == kKondoM ? 2 : 1;
      for (int k = 0; k < copies; k++)
        for (int c = 0; c < ncell; c++)
          for (int o = 0; o < lat.nsub; o++)
            std::fprintf(f, "%ld %ld 0 %d\n", lat.cells[c][0], lat.cells[c][1], o + k * lat.nsub);
      std::fclose(f);
    }
    {
      FILE *f = open_out(dir, "namelist.def");
      for (const auto &n : names) std::fprintf(f, "%16s  %s\n", n.first.c_str(), n.second.c_str());
      std::fclose(f);
    }
    return 0;
  } catch (const std::exception &e) {
    *err = std::string("standard mode: ") + e.what();
    return -1;
  }
}

}  // namespace stdface
}  // namespace hphi
