// Expert-mode reader and term compiler (host C++).
//
// File formats follow the reference reader (src/readdef.c):
//   namelist.def   "Keyword file" lines; keywords src/readdef.c:46-71
//   calcmod.def    "Key int" lines                          src/readdef.c:233-386
//   modpara.def    8 header lines, then "Key value" lines   src/readdef.c:513-640
//   locspn.def     5 header lines (2nd: "NlocalSpin n"), then "i S2" lines
//   interactions   5 header lines (2nd: "N<kind> n"), then one entry per line
// Sector parameters (Nup, Ndown, Ne, Total2Sz) are derived as in
// src/readdef.c:880-960.  Hamiltonian semantics of each keyword:
//   Trans        H += -t c+_{i s1} c_{j s2}               (src/mltplyHubbard.c:202; diagonal
//                                                          entries become EDChemi, src/readdef.c:2185-2233)
//   CoulombIntra H += U n_{i0} n_{i1}                     (src/diagonalcalc.c:260-355)
//   CoulombInter H += V n_i n_j                           (src/diagonalcalc.c:543-787)
//   Hund         H += -J (n_{i0} n_{j0} + n_{i1} n_{j1})   (src/diagonalcalc.c:788-1112)
//   Ising        Hund(-J/2) + CoulombInter(-J/4)          (src/readdef.c:1320-1327)
//   Exchange     Hubbard/Kondo: J (c+_{i0}c_{j0}c+_{j1}c_{i1} + h.c.) (src/mltplyHubbardCore.c:197-218, 472-526)
//                Spin: J (|10><01| + |01><10|) on (i,j)   (src/mltplySpinCore.c:35-56, 273-307)
//   PairHop      J (c+_{i0}c_{j0}c+_{i1}c_{j1}), stored with its (j,i) partner (src/readdef.c:1262-1283,
//                src/mltplyHubbardCore.c:533-575)
//   PairLift     SpinGC: J (|11><00| + |00><11|) on (i,j)  (src/mltplySpinCore.c:352-382)
//   InterAll     V c+_{i s1} c_{j s2} c+_{k s3} c_{l s4}   (src/readdef.c:1373-1400, 2415-2549)
// Spin models label a site's state by its bit value (sigma == bit), as the spin
// element routines do (src/mltplySpinCore.c:239-266, src/diagonalcalc.c SetDiagonalChemi).
#include "model.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <tuple>

namespace hphi {
namespace {

std::string lower(std::string s) {
  for (auto &ch : s) ch = (char)std::tolower((unsigned char)ch);
  return s;
}

bool open_def(const Model &m, const std::string &name, std::ifstream *f) {
  f->open(name);
  if (f->is_open()) return true;
  if (!name.empty() && name[0] != '/' && !m.base_dir.empty()) {
    f->clear();
    f->open(m.base_dir + "/" + name);
    return f->is_open();
  }
  return false;
}

int parity64(uint64_t x) { return __builtin_popcountll(x) & 1; }

// Reads the count on the 2nd header line of an interaction file and the entry lines.
bool read_table(const Model &m, const std::string &fname, std::vector<std::vector<double>> *rows,
                int ncol, std::string *err) {
  std::ifstream f;
  if (!open_def(m, fname, &f)) { *err = "cannot open " + fname; return false; }
  std::string line;
  int count = -1;
  for (int i = 0; i < 5; i++) {
    if (!std::getline(f, line)) { *err = fname + ": truncated header"; return false; }
    if (i == 1) {
      std::istringstream ss(line);
      std::string kw;
      ss >> kw >> count;
      if (ss.fail()) { *err = fname + ": bad header line 2"; return false; }
    }
  }
  rows->clear();
  while ((int)rows->size() < count && std::getline(f, line)) {
    if (line.find_first_not_of(" \t\r\n") == std::string::npos) continue;
    std::istringstream ss(line);
    std::vector<double> r(ncol, 0.0);
    int got = 0;
    for (; got < ncol; got++) {
      if (!(ss >> r[got])) break;
    }
    if (got < ncol) {
      // Trans/InterAll may omit the imaginary part.
      if (!(got == ncol - 1)) { *err = fname + ": malformed line: " + line; return false; }
      r[ncol - 1] = 0.0;
    }
    rows->push_back(r);
  }
  if ((int)rows->size() != count) { *err = fname + ": fewer entries than the header count"; return false; }
  return true;
}

// Reads an integer table (OneBodyG / TwoBodyG): the count on the 2nd header line, then that
// many lines of ncol integers.
bool read_int_table(const Model &m, const std::string &fname, int ncol, std::vector<std::vector<int>> *rows,
                    std::string *err) {
  std::ifstream f;
  if (!open_def(m, fname, &f)) { *err = "cannot open " + fname; return false; }
  std::string line;
  int count = -1;
  for (int i = 0; i < 5; i++) {
    if (!std::getline(f, line)) { *err = fname + ": truncated header"; return false; }
    if (i == 1) {
      std::istringstream ss(line);
      std::string kw;
      ss >> kw >> count;
      if (ss.fail() || count < 0) { *err = fname + ": bad header line 2"; return false; }
    }
  }
  rows->clear();
  while ((int)rows->size() < count && std::getline(f, line)) {
    if (line.find_first_not_of(" \t\r\n") == std::string::npos) continue;
    std::istringstream ss(line);
    std::vector<int> r(ncol, 0);
    for (int q = 0; q < ncol; q++)
      if (!(ss >> r[q])) { *err = fname + ": malformed line: " + line; return false; }
    rows->push_back(r);
  }
  if ((int)rows->size() != count) { *err = fname + ": fewer entries than the header count"; return false; }
  return true;
}

// Compiles a fermion operator string (ops applied right to left) in the
// Jordan-Wigner ordering of configuration bits.  Push form: a source s with
// (s & req_mask) == req_val maps to s ^ flip with sign (-1)^(sign0 + popc(s & sm)).
bool compile_fermion(const std::vector<FermionOp> &ops, uint64_t *req_mask, uint64_t *req_val,
                     uint64_t *flip, uint64_t *sm, int *sign0) {
  uint64_t rm = 0, rv = 0, fl = 0, s = 0;
  int sg = 0;
  for (int k = (int)ops.size() - 1; k >= 0; k--) {
    const uint64_t b = 1ull << ops[k].bit;
    const int need_now = ops[k].dag ? 0 : 1;
    const int need_orig = need_now ^ ((fl & b) ? 1 : 0);
    if (rm & b) {
      if ((int)((rv & b) ? 1 : 0) != need_orig) return false;
    } else {
      rm |= b;
      if (need_orig) rv |= b;
    }
    const uint64_t below = b - 1;
    s ^= below;
    sg ^= parity64(fl & below);
    fl ^= b;
  }
  *req_mask = rm; *req_val = rv; *flip = fl; *sm = s; *sign0 = sg;
  return true;
}

// Spin strings on packed digit fields (site_bits bits per site; 1 for S = 1/2): each
// |to><from| requires the site's current digit to be `from` and sets it to `to`.  Push form:
// a source s with (s & req_mask) == req_val maps to s ^ flip (the fields it touches go from
// their required values to their final values).
bool compile_spin(const std::vector<SpinOp> &ops, int site_bits, uint64_t *req_mask, uint64_t *req_val,
                  uint64_t *flip) {
  uint64_t rm = 0, rv = 0;
  std::map<int, int> cur;  // current digit of each touched site
  for (int k = (int)ops.size() - 1; k >= 0; k--) {
    const int sh = site_bits * ops[k].site;
    const uint64_t fm = ((1ull << site_bits) - 1) << sh;
    auto it = cur.find(ops[k].site);
    if (it != cur.end()) {
      if (it->second != ops[k].from) return false;
    } else {
      rm |= fm;
      rv |= (uint64_t)ops[k].from << sh;
    }
    cur[ops[k].site] = ops[k].to;
  }
  uint64_t fl = 0;
  for (const auto &kv : cur) {
    const int sh = site_bits * kv.first;
    fl |= (((rv >> sh) ^ (uint64_t)kv.second) & ((1ull << site_bits) - 1)) << sh;
  }
  *req_mask = rm; *req_val = rv; *flip = fl;
  return true;
}

void push_term(Model *m, uint64_t rm, uint64_t rv, uint64_t fl, uint64_t sm, int sign0,
               std::complex<double> coef) {
  if (sign0) coef = -coef;
  if (fl == 0) {
    m->diag.push_back(DiagTerm{rm, rv, coef.real()});
    return;
  }
  // Pull form for the output configuration t = s ^ fl.
  const uint64_t cv = rv ^ (fl & rm);
  if (parity64(fl & sm)) coef = -coef;
  m->offdiag.push_back(BitTerm{rm, cv, fl, sm, coef.real(), coef.imag()});
}

}  // namespace

bool add_fermion_string(Model *m, const std::vector<FermionOp> &ops, std::complex<double> coef) {
  uint64_t rm, rv, fl, sm;
  int s0;
  if (!compile_fermion(ops, &rm, &rv, &fl, &sm, &s0)) return false;
  push_term(m, rm, rv, fl, sm, s0, coef);
  return true;
}

bool add_spin_string(Model *m, const std::vector<SpinOp> &ops, std::complex<double> coef) {
  uint64_t rm, rv, fl;
  if (!compile_spin(ops, m->site_bits, &rm, &rv, &fl)) return false;
  push_term(m, rm, rv, fl, 0, 0, coef);
  return true;
}

int compile_green(const Model &m, int body, const int *rows, int n, std::vector<GreenTerm> *terms,
                  std::vector<char> *trailing_space, std::string *err) {
  terms->assign((size_t)n, GreenTerm{0, 0, 0, 0, 0.0, 0.0});
  trailing_space->assign((size_t)n, 0);
  const bool spin = m.is_spin();
  const bool kondo = m.is_kondo();
  // Hubbard-type dispatch of both functions (HubbardNConserved runs as Hubbard after sz,
  // src/sz.c:802-806); iFlgSzConserved is set by a 2Sz line (src/readdef.c:570-573)
  const bool canonical_fermion = m.calc_model == kHubbard || m.calc_model == kHubbardNConserved || kondo;
  const int stride = 4 * (body == 1 ? 1 : body == 2 ? 2 : body);  // 4 integers per site pair
  auto fbit = [](int site, int s) { return 2 * site + s; };
  auto bad = [&](int site, int g) {
    return site < 0 || site >= m.nsite || g < 0 || g > (spin ? m.locspn[site] : 1);
  };
  auto set_fermion = [&](int e, const std::vector<FermionOp> &ops) {
    uint64_t rm, rv, fl, sm;
    int s0;
    if (compile_fermion(ops, &rm, &rv, &fl, &sm, &s0)) (*terms)[e] = GreenTerm{rm, rv, fl, sm, s0 ? -1.0 : 1.0, 0.0};
  };
  auto set_spin = [&](int e, const std::vector<SpinOp> &ops) {
    uint64_t rm, rv, fl;
    if (compile_spin(ops, m.site_bits, &rm, &rv, &fl)) (*terms)[e] = GreenTerm{rm, rv, fl, 0, 1.0, 0.0};
  };
  for (int e = 0; e < n; e++) {
    const int *r = rows + (size_t)stride * e;
    for (int q = 0; q < stride / 2; q++)
      if (bad(r[2 * q], r[2 * q + 1])) {
        *err = "Green's function entry " + std::to_string(e) + ": site or spin index out of range";
        return -1;
      }
    if (body >= 3) {
      // expec_Threebody / Fourbody / Sixbody_SpinGCHalf (src/expec_cisajscktaltdc.c:901-1420):
      // spin-1/2 SpinGC only; the last pairs act first through mltplyHalfSpinGC_mini
      // (src/mltplySpin.c:416-500, nothing for a pair on two sites), the first two pairs go
      // through Rearray_Interactions (:274-391) and the SpinGC element routines
      if (m.calc_model != kSpinGC || m.general_spin) continue;
      int a[4], g[4];
      for (int q = 0; q < 4; q++) { a[q] = r[2 * q]; g[q] = r[2 * q + 1]; }
      int p1, q1, q2, p3, q3, q4;  // pairs (site, to, from) after Rearray
      double V;
      if (a[0] == a[1] && a[2] == a[3]) {
        V = 1.0;
        if (a[0] > a[2]) { p1 = a[2]; q1 = g[2]; q2 = g[3]; p3 = a[0]; q3 = g[0]; q4 = g[1]; }
        else { p1 = a[0]; q1 = g[0]; q2 = g[1]; p3 = a[2]; q3 = g[2]; q4 = g[3]; }
      } else if (a[0] == a[3] && a[2] == a[1]) {
        V = -1.0;
        if (a[0] > a[2]) { p1 = a[2]; q1 = g[2]; q2 = g[1]; p3 = a[0]; q3 = g[0]; q4 = g[3]; }
        else { p1 = a[0]; q1 = g[0]; q2 = g[3]; p3 = a[2]; q3 = g[2]; q4 = g[1]; }
      } else {
        (*trailing_space)[e] = 1;  // printed with its first 8 indices only
        continue;
      }
      std::vector<SpinOp> ops = {{p1, q1, q2}, {p3, q3, q4}};
      bool onsite = true;
      for (int k = 2; k < body; k++) {  // pair k: (r[4k], r[4k+1]) created, (r[4k+2], r[4k+3]) annihilated
        if (r[4 * k] != r[4 * k + 2]) { onsite = false; break; }
        ops.push_back({r[4 * k], r[4 * k + 1], r[4 * k + 3]});
      }
      if (!onsite) continue;
      uint64_t rm, rv, fl;
      if (compile_spin(ops, m.site_bits, &rm, &rv, &fl)) (*terms)[e] = GreenTerm{rm, rv, fl, 0, V, 0.0};
      continue;
    }
    if (body == 1) {
      const int i = r[0], s1 = r[1], j = r[2], s2 = r[3];
      if (spin) {
        // spin sites never hop (src/expec_cisajs.c:349-398, 446-450, 526-530, 626-629)
        if (i != j) continue;
        if (s1 == s2) set_spin(e, {{i, s1, s1}});                  // longitudinal: [digit == s1]
        else if (m.calc_model == kSpinGC) set_spin(e, {{i, s1, s2}});  // transverse |s1><s2| (:512-521, :609-621)
        continue;                                                   // canonical: zero
      }
      if (canonical_fermion && m.sz_conserved && s1 != s2) continue;  // :276-282
      if (kondo && ((m.locspn[i] == 1 && m.locspn[j] == 0) || (m.locspn[i] == 0 && m.locspn[j] == 1)))
        continue;                                                   // :284-293
      // c+_{i s1} c_{j s2} (general_hopp / GC_general_hopp, CisAjt src/mltplyHubbardCore.c:305-347)
      set_fermion(e, {{fbit(i, s1), true}, {fbit(j, s2), false}});
    } else {
      const int i = r[0], s1 = r[1], j = r[2], s2 = r[3], k = r[4], s3 = r[5], l = r[6], s4 = r[7];
      if (spin) {
        // on-site pairs (the reader enforces i == j, k == l); Rearray_Interactions orders the
        // pairs by site (:274-391), which commute on different sites.  Every spin branch
        // prints "value \n" (:682-886, :1423-1647).
        (*trailing_space)[e] = 1;
        // a canonical sector holds one Sz: rows that change it are zero without a lookup
        // (the 2Sz test of SpinGeneral :801-817; SpinHalf reaches its lookups only through
        // Sz-conserving branches :700-760), since the half tables would map such a
        // configuration to an unrelated row
        if (m.calc_model == kSpin && (s1 - s2) + (s3 - s4) != 0) continue;
        set_spin(e, {{i, s1, s2}, {k, s3, s4}});
        continue;
      }
      if (canonical_fermion && m.sz_conserved && s1 + s3 != s2 + s4) {  // :535-541
        (*trailing_space)[e] = 1;
        continue;
      }
      // c+_{i s1} c_{j s2} c+_{k s3} c_{l s4}, right pair first (CisAjtCkuAlv_element and
      // relatives, src/mltplyHubbardCore.c:689-1000)
      set_fermion(e, {{fbit(i, s1), true}, {fbit(j, s2), false}, {fbit(k, s3), true}, {fbit(l, s4), false}});
    }
  }
  return 0;
}

void canonicalize_terms(Model *m) {
  std::map<std::tuple<uint64_t, uint64_t, uint64_t, uint64_t>, std::complex<double>> off;
  std::vector<std::tuple<uint64_t, uint64_t, uint64_t, uint64_t>> order;
  for (const auto &t : m->offdiag) {
    auto key = std::make_tuple(t.flip, t.cm, t.cv, t.sm);
    auto it = off.find(key);
    if (it == off.end()) { off[key] = {t.re, t.im}; order.push_back(key); }
    else it->second += std::complex<double>(t.re, t.im);
  }
  m->offdiag.clear();
  m->complex_terms = false;
  for (const auto &key : order) {
    const auto c = off[key];
    if (c == std::complex<double>(0.0, 0.0)) continue;
    m->offdiag.push_back(BitTerm{std::get<1>(key), std::get<2>(key), std::get<0>(key),
                                 std::get<3>(key), c.real(), c.imag()});
    if (c.imag() != 0.0) m->complex_terms = true;
  }
  // Diagonal terms are summed in their input order by the device (no merging, so the
  // per-configuration sum follows the reference's term order as closely as possible).
  std::vector<DiagTerm> d;
  for (const auto &t : m->diag)
    if (t.v != 0.0) d.push_back(t);
  m->diag.swap(d);
}

int read_expert(const std::string &namelist, Model *m, std::string *err) {
  *m = Model();
  {
    const auto pos = namelist.find_last_of('/');
    m->base_dir = (pos == std::string::npos) ? std::string(".") : namelist.substr(0, pos);
  }
  std::ifstream nl(namelist);
  if (!nl.is_open()) { *err = "cannot open " + namelist; return -1; }
  std::map<std::string, std::string> files;
  std::string line;
  static const char *known[] = {"calcmod", "modpara", "locspin", "trans", "coulombintra", "coulombinter",
                                "hund", "pairhop", "exchange", "interall", "onebodyg", "twobodyg",
                                "pairlift", "ising", "boost", "singleexcitation", "pairexcitation",
                                "spectrumvec", "laser", "teonebody", "tetwobody", "threebodyg",
                                "fourbodyg", "sixbodyg"};
  while (std::getline(nl, line)) {
    std::istringstream ss(line);
    std::string kw, fn;
    if (!(ss >> kw)) continue;
    if (kw[0] == '#') continue;
    if (!(ss >> fn)) { *err = "namelist.def: keyword without file: " + kw; return -1; }
    const std::string k = lower(kw);
    if (std::find(std::begin(known), std::end(known), k) == std::end(known)) {
      *err = "namelist.def: unknown keyword " + kw;
      return -1;
    }
    if (files.count(k)) { *err = "namelist.def: duplicate keyword " + kw; return -1; }
    files[k] = fn;
  }
  for (const char *must : {"calcmod", "modpara", "locspin"})
    if (!files.count(must)) { *err = std::string("namelist.def: missing ") + must; return -1; }
  for (const char *unsupported : {"boost", "laser"})
    if (files.count(unsupported)) {
      *err = std::string("namelist.def: keyword not supported by this engine: ") + unsupported;
      return -1;
    }

  // ---- calcmod.def
  {
    std::ifstream f;
    if (!open_def(*m, files["calcmod"], &f)) { *err = "cannot open " + files["calcmod"]; return -1; }
    while (std::getline(f, line)) {
      std::istringstream ss(line);
      std::string kw;
      long v;
      if (!(ss >> kw) || kw[0] == '#' || kw[0] == '=' || kw[0] == '-') continue;
      if (!(ss >> v)) continue;
      const std::string k = lower(kw);
      if (k == "calctype") m->calc_type = (int)v;
      else if (k == "calcmodel") m->calc_model = (int)v;
      else if (k == "outputmode") m->output_mode = (int)v;
      else if (k == "calceigenvec") m->calc_eigenvec = (int)v;
      else if (k == "initialvectype") m->initial_vec_type = (int)v;
      else if (k == "outputeigenvec" || k == "oev") m->output_eigenvec = (int)v;
      else if (k == "inputeigenvec" || k == "iev") m->input_eigenvec = (int)v;
      else if (k == "restart") m->restart = (int)v;
      else if (k == "flgfinitetemperature") m->flg_finite_temperature = (int)v;
      else if (k == "calcspec" || k == "calcspectrum") {
        if (v != 0 && v != 1) {
          *err = "calcmod.def: " + kw + " " + std::to_string(v) +
                 " is not supported by this engine (0, or 1: spectrum from an input vector)";
          return -1;
        }
        m->calc_spec = (int)v;
      } else if (k == "outputexcitedvec" || k == "outputexvec") {
        m->output_exvec = (int)v;
      } else if (k == "outputham" || k == "inputham" || k == "ngpu" || k == "scalapack") {
        if (k == "inputham" && v != 0) {
          *err = "calcmod.def: " + kw + " is not supported by this engine";
          return -1;
        }
      } else {
        *err = "calcmod.def: unknown keyword " + kw;
        return -1;
      }
    }
    if (m->calc_model < 0 || m->calc_model > 5) { *err = "calcmod.def: CalcModel out of range"; return -1; }
    if (m->calc_type < 0 || m->calc_type > 5) { *err = "calcmod.def: CalcType out of range"; return -1; }
  }
  // ---- modpara.def
  {
    std::ifstream f;
    if (!open_def(*m, files["modpara"], &f)) { *err = "cannot open " + files["modpara"]; return -1; }
    for (int i = 0; i < 8; i++) {
      if (!std::getline(f, line)) { *err = "modpara.def: truncated header"; return -1; }
      std::istringstream ss(line);
      std::string kw, v;
      if (i == 5 && (ss >> kw >> v)) m->data_head = v;
      if (i == 6 && (ss >> kw >> v)) m->para_head = v;
    }
    while (std::getline(f, line)) {
      std::istringstream ss(line);
      std::string kw;
      double v = 0.0, v2 = 0.0;
      if (!(ss >> kw)) continue;
      if (!(ss >> v)) { *err = "modpara.def: malformed line: " + line; return -1; }
      if (!(ss >> v2)) v2 = 0.0;  // second number (imaginary part of OmegaMax / OmegaMin / OmegaOrg)
      const std::string k = lower(kw);
      if (k == "nsite") m->nsite = (int)v;
      else if (k == "nup") m->nup = (int)v;
      else if (k == "ndown") { m->ndown = (int)v; m->total_2sz = m->nup - m->ndown; }
      else if (k == "2sz") { m->total_2sz = (int)v; m->sz_conserved = true; }
      else if (k == "ncond") {
        if ((int)v < 0) { *err = "modpara.def: Ncond must be non-negative"; return -1; }
        m->ncond = (int)v; m->read_ncond = true;
      }
      else if (k == "lanczos_max") m->lanczos_max = (int)v;
      else if (k == "initial_iv") m->initial_iv = (int)v;
      else if (k == "nvec") m->nvec = (int)v;
      else if (k == "exct") m->k_exct = (int)v;
      else if (k == "lanczoseps") m->lanczos_eps = (int)v;
      else if (k == "lanczostarget") m->lanczos_target = (int)v;
      else if (k == "largevalue") m->large_value = v;
      else if (k == "numave") m->num_ave = (int)v;
      else if (k == "expecinterval") m->expec_interval = (int)v;
      else if (k == "calchs") m->read_hacker = (int)v;
      else if (k == "precg") m->pre_cg = (int)v;
      else if (k == "expandcoef") m->expand_coef = (int)v;
      else if (k == "outputinterval") m->output_interval = (int)v;
      else if (k == "omegamax") { m->omega_max[0] = v; m->omega_max[1] = v2; m->omega_max_set = true; }
      else if (k == "omegamin") { m->omega_min[0] = v; m->omega_min[1] = v2; m->omega_min_set = true; }
      else if (k == "omegaim") { m->omega_org[1] += v; m->omega_org_set = true; }
      else if (k == "omegaorg") { m->omega_org[0] += v; m->omega_org[1] += v2; m->omega_org_set = true; }
      else if (k == "nomega") m->n_omega = (int)v;
      else if (k == "timeslice" || k == "tinit" || k == "targettpqrand") {
        // accepted and ignored: parameters of modes outside this engine
      } else {
        *err = "modpara.def: unknown keyword " + kw;
        return -1;
      }
    }
  }
  // ---- locspn.def
  {
    std::ifstream f;
    if (!open_def(*m, files["locspin"], &f)) { *err = "cannot open " + files["locspin"]; return -1; }
    for (int i = 0; i < 5; i++) {
      if (!std::getline(f, line)) { *err = "locspn.def: truncated header"; return -1; }
      if (i == 1) {
        std::istringstream ss(line);
        std::string kw;
        ss >> kw >> m->nlocspn;
      }
    }
    if (m->nsite <= 0) { *err = "modpara.def: Nsite must be positive"; return -1; }
    m->locspn.assign(m->nsite, -1);
    int idx = 0;
    while (std::getline(f, line)) {
      std::istringstream ss(line);
      int i, s;
      if (!(ss >> i >> s)) continue;
      if (idx == m->nsite || i < 0 || i >= m->nsite) { *err = "locspn.def: bad site index"; return -1; }
      m->locspn[i] = s;
      idx++;
    }
    for (int i = 0; i < m->nsite; i++)
      if (m->locspn[i] < 0) { *err = "locspn.def: missing site"; return -1; }
    for (int i = 0; i < m->nsite; i++) {
      // CheckLocSpin (src/readdef.c:2725-2765): spin sites have 2S >= 1; 2S > 1 anywhere
      // makes the model a general-spin one
      if (m->is_spin() && m->locspn[i] < 1) {
        *err = "locspn.def: spin sites need 2S >= 1";
        return -1;
      }
      if (m->is_spin() && m->locspn[i] > 1) m->general_spin = true;
      if ((m->calc_model == kHubbard || m->calc_model == kHubbardGC) && m->locspn[i] != 0) {
        *err = "locspn.def: Hubbard models need itinerant sites (0)";
        return -1;
      }
    }
  }
  // ---- sector parameters (src/readdef.c:880-960)
  switch (m->calc_model) {
    case kSpin: case kHubbard: case kKondo:
      if (m->read_ncond) {
        if (m->calc_model == kSpin) { *err = "modpara.def: Ncond is not allowed for Spin"; return -1; }
        if (m->sz_conserved) {
          m->nup = (m->nlocspn + m->ncond + m->total_2sz) / 2;
          m->ndown = (m->nlocspn + m->ncond - m->total_2sz) / 2;
        } else if (m->calc_model == kHubbard) {
          m->ne = m->ncond;
          if (m->ne < 1) { *err = "modpara.def: Ncond must be positive"; return -1; }
          m->calc_model = kHubbardNConserved;
        } else {
          *err = "modpara.def: Kondo needs 2Sz"; return -1;
        }
      } else if (m->sz_conserved) {
        if (m->calc_model != kSpin) { *err = "modpara.def: Ncond is required"; return -1; }
        m->nup = (m->nlocspn + m->total_2sz) / 2;
        m->ndown = (m->nlocspn - m->total_2sz) / 2;
      } else if (m->nup == 0 && m->ndown == 0) {
        *err = "modpara.def: sector (2Sz / Ncond / Nup, Ndown) is not given"; return -1;
      }
      if (m->calc_model == kSpin) m->ne = m->nup;
      else if (m->ne == 0) m->ne = m->nup + m->ndown;
      break;
    default:
      break;
  }
  if (m->lanczos_max <= 0) { *err = "modpara.def: Lanczos_max must be positive"; return -1; }
  if (m->lanczos_eps <= 0) { *err = "modpara.def: LanczosEps must be positive"; return -1; }
  if (m->num_ave <= 0) { *err = "modpara.def: NumAve must be positive"; return -1; }
  if (m->expec_interval <= 0) { *err = "modpara.def: ExpecInterval must be positive"; return -1; }
  if (m->nvec == 0) m->nvec = m->lanczos_max;
  if (m->nvec < m->k_exct) m->nvec = m->k_exct;
  if (m->lanczos_target < m->k_exct) m->lanczos_target = m->k_exct;
  if (m->k_exct < 1 || m->k_exct > m->nvec) { *err = "modpara.def: exct out of range"; return -1; }
  if (m->calc_model == kKondo || m->calc_model == kKondoGC) {
    // Local spins are S = 1/2 sites held singly occupied by the sector (src/sz.c:1110-1220,
    // 1342-1420).  An odd number of sites splits one site across the two halves of the
    // configuration; the engine supports even Nsite.
    if (m->nsite % 2 != 0) { *err = "Kondo models with an odd number of sites are not supported by this engine"; return -1; }
    for (int i = 0; i < m->nsite; i++)
      if (m->locspn[i] != 0 && m->locspn[i] != 1) {
        *err = "locspn.def: Kondo local spins must be S=1/2 (2S=1)"; return -1;
      }
  }
  const bool spin = m->is_spin();
  if (m->general_spin) {
    int maxs = 1;
    for (int i = 0; i < m->nsite; i++) maxs = std::max(maxs, m->locspn[i]);
    m->site_bits = 1;
    while ((1 << m->site_bits) < maxs + 1) m->site_bits++;
  }
  m->nbits = spin ? m->site_bits * m->nsite : 2 * m->nsite;
  if (m->nbits > 64) { *err = "too many sites for 64-bit configurations"; return -1; }
  // two-spin-state index range of a site (0 .. 2S_i; 0 .. 1 for fermions)
  auto sigma_ok = [&](int site, int g) { return g >= 0 && g <= (spin ? m->locspn[site] : 1); };

  auto fbit = [&](int site, int s) { return 2 * site + s; };
  auto check_site = [&](int i) { return i >= 0 && i < m->nsite; };
  std::vector<std::vector<double>> rows;

  // ---- Trans
  if (files.count("trans")) {
    if (!read_table(*m, files["trans"], &rows, 6, err)) return -1;
    // Merge duplicates (src/readdef.c:1139-1156), then check Hermiticity (CheckTransferHermite).
    std::map<std::tuple<int, int, int, int>, std::complex<double>> tr;
    std::vector<std::tuple<int, int, int, int>> order;
    for (const auto &r : rows) {
      const int i = (int)r[0], s1 = (int)r[1], j = (int)r[2], s2 = (int)r[3];
      if (!check_site(i) || !check_site(j) || !sigma_ok(i, s1) || !sigma_ok(j, s2)) {
        *err = files["trans"] + ": bad site or spin index"; return -1;
      }
      if (i == j && s1 == s2 && std::fabs(r[5]) > 1e-12) {
        *err = files["trans"] + ": diagonal transfer with an imaginary part"; return -1;
      }
      if (m->calc_model == kSpin && i != j) { *err = files["trans"] + ": Spin needs site-diagonal transfers"; return -1; }
      if (m->calc_model == kSpinGC && i != j) { *err = files["trans"] + ": SpinGC needs site-diagonal transfers"; return -1; }
      if ((m->calc_model == kKondo || m->calc_model == kKondoGC) && i != j && (m->locspn[i] != 0 || m->locspn[j] != 0)) {
        *err = files["trans"] + ": Kondo transfers touching a local spin must be site-diagonal"; return -1;
      }
      auto key = std::make_tuple(i, s1, j, s2);
      if (!tr.count(key)) order.push_back(key);
      tr[key] += std::complex<double>(r[4], r[5]);
    }
    for (const auto &key : order) {
      int i, s1, j, s2;
      std::tie(i, s1, j, s2) = key;
      if (i == j && s1 == s2) continue;
      auto it = tr.find(std::make_tuple(j, s2, i, s1));
      if (it == tr.end() || std::abs(it->second - std::conj(tr[key])) > 1e-12) {
        *err = files["trans"] + ": transfer integrals are not Hermitian"; return -1;
      }
    }
    for (const auto &key : order) {
      int i, s1, j, s2;
      std::tie(i, s1, j, s2) = key;
      const std::complex<double> t = tr[key];
      // A canonical spin sector keeps Sz: the reference's multiply absorbs only the diagonal
      // transfers and never applies spin-flip ones (src/mltplySpin.c:208-211, 327-329).
      if (m->calc_model == kSpin && s1 != s2) continue;
      if (spin) add_spin_string(m, {{i, s1, s2}}, -t);
      else add_fermion_string(m, {{fbit(i, s1), true}, {fbit(j, s2), false}}, -t);
    }
    m->n_trans = (int)rows.size();
  }
  // General spin takes its interactions as InterAll only (src/readdef.c:2027-2044).
  if (m->general_spin)
    for (const char *k : {"coulombintra", "coulombinter", "hund", "pairhop", "exchange", "ising", "pairlift"})
      if (files.count(k)) { *err = std::string(k) + ": general spin takes interactions as InterAll only"; return -1; }
  // ---- CoulombIntra
  if (files.count("coulombintra")) {
    if (!read_table(*m, files["coulombintra"], &rows, 2, err)) return -1;
    for (const auto &r : rows) {
      const int i = (int)r[0];
      if (!check_site(i)) { *err = files["coulombintra"] + ": bad site"; return -1; }
      if (!spin) {
        const uint64_t msk = (1ull << fbit(i, 0)) | (1ull << fbit(i, 1));
        m->diag.push_back(DiagTerm{msk, msk, r[1]});
      }
    }
    m->n_coulomb_intra = (int)rows.size();
  }
  auto add_inter = [&](int i, int j, double V) {
    if (spin) { m->diag.push_back(DiagTerm{0, 0, V}); return; }
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++) {
        const uint64_t msk = (1ull << fbit(i, a)) | (1ull << fbit(j, b));
        m->diag.push_back(DiagTerm{msk, msk, V});
      }
  };
  auto add_hund = [&](int i, int j, double J) {  // H += -J (n_i0 n_j0 + n_i1 n_j1)
    if (spin) {
      const uint64_t msk = (1ull << i) | (1ull << j);
      m->diag.push_back(DiagTerm{msk, msk, -J});
      m->diag.push_back(DiagTerm{msk, 0, -J});
      return;
    }
    for (int a = 0; a < 2; a++) {
      const uint64_t msk = (1ull << fbit(i, a)) | (1ull << fbit(j, a));
      m->diag.push_back(DiagTerm{msk, msk, -J});
    }
  };
  // ---- CoulombInter
  if (files.count("coulombinter")) {
    if (!read_table(*m, files["coulombinter"], &rows, 3, err)) return -1;
    for (const auto &r : rows) {
      if (!check_site((int)r[0]) || !check_site((int)r[1])) { *err = files["coulombinter"] + ": bad site"; return -1; }
      add_inter((int)r[0], (int)r[1], r[2]);
    }
    m->n_coulomb_inter = (int)rows.size();
  }
  // ---- Hund
  if (files.count("hund")) {
    if (!read_table(*m, files["hund"], &rows, 3, err)) return -1;
    for (const auto &r : rows) {
      if (!check_site((int)r[0]) || !check_site((int)r[1])) { *err = files["hund"] + ": bad site"; return -1; }
      add_hund((int)r[0], (int)r[1], r[2]);
    }
    m->n_hund = (int)rows.size();
  }
  // ---- Ising: Hund(-J/2) + CoulombInter(-J/4)
  if (files.count("ising")) {
    if (!read_table(*m, files["ising"], &rows, 3, err)) return -1;
    for (const auto &r : rows) {
      if (!check_site((int)r[0]) || !check_site((int)r[1])) { *err = files["ising"] + ": bad site"; return -1; }
      add_hund((int)r[0], (int)r[1], -r[2] / 2.0);
      add_inter((int)r[0], (int)r[1], -r[2] / 4.0);
    }
    m->n_ising = (int)rows.size();
  }
  // ---- Exchange
  if (files.count("exchange")) {
    if (!read_table(*m, files["exchange"], &rows, 3, err)) return -1;
    for (const auto &r : rows) {
      const int i = (int)r[0], j = (int)r[1];
      if (!check_site(i) || !check_site(j)) { *err = files["exchange"] + ": bad site"; return -1; }
      if (i == j) continue;
      const std::complex<double> J(r[2], 0.0);
      if (spin) {
        add_spin_string(m, {{i, 1, 0}, {j, 0, 1}}, J);
        add_spin_string(m, {{i, 0, 1}, {j, 1, 0}}, J);
      } else {
        add_fermion_string(m, {{fbit(i, 0), true}, {fbit(j, 0), false}, {fbit(j, 1), true}, {fbit(i, 1), false}}, J);
        add_fermion_string(m, {{fbit(j, 0), true}, {fbit(i, 0), false}, {fbit(i, 1), true}, {fbit(j, 1), false}}, J);
      }
    }
    m->n_exchange = (int)rows.size();
  }
  // ---- PairHop
  if (files.count("pairhop")) {
    if (spin) { *err = "PairHop is not active in Spin and SpinGC"; return -1; }
    if (!read_table(*m, files["pairhop"], &rows, 3, err)) return -1;
    for (const auto &r : rows) {
      const int i = (int)r[0], j = (int)r[1];
      if (!check_site(i) || !check_site(j)) { *err = files["pairhop"] + ": bad site"; return -1; }
      if (i == j) continue;
      const std::complex<double> J(r[2], 0.0);
      add_fermion_string(m, {{fbit(i, 0), true}, {fbit(j, 0), false}, {fbit(i, 1), true}, {fbit(j, 1), false}}, J);
      add_fermion_string(m, {{fbit(j, 0), true}, {fbit(i, 0), false}, {fbit(j, 1), true}, {fbit(i, 1), false}}, J);
    }
    m->n_pairhop = (int)rows.size();
  }
  // ---- PairLift
  if (files.count("pairlift")) {
    if (!read_table(*m, files["pairlift"], &rows, 3, err)) return -1;
    if (!rows.empty() && m->calc_model != kSpinGC) { *err = "PairLift is active only in SpinGC"; return -1; }
    for (const auto &r : rows) {
      const int i = (int)r[0], j = (int)r[1];
      if (!check_site(i) || !check_site(j)) { *err = files["pairlift"] + ": bad site"; return -1; }
      if (i == j) continue;
      const std::complex<double> J(r[2], 0.0);
      add_spin_string(m, {{i, 1, 0}, {j, 1, 0}}, J);
      add_spin_string(m, {{i, 0, 1}, {j, 0, 1}}, J);
    }
    m->n_pairlift = (int)rows.size();
  }
  // ---- InterAll
  if (files.count("interall")) {
    if (!read_table(*m, files["interall"], &rows, 10, err)) return -1;
    for (const auto &r : rows) {
      int s[4], g[4];
      for (int q = 0; q < 4; q++) { s[q] = (int)r[2 * q]; g[q] = (int)r[2 * q + 1]; }
      for (int q = 0; q < 4; q++)
        if (!check_site(s[q]) || !sigma_ok(s[q], g[q])) { *err = files["interall"] + ": bad index"; return -1; }
      if (m->general_spin && m->calc_model == kSpin && (g[0] - g[1]) + (g[2] - g[3]) != 0) {
        *err = files["interall"] + ": a canonical general-spin InterAll term must conserve Sz"; return -1;
      }
      const std::complex<double> V(r[8], r[9]);
      if (m->calc_model == kKondo || m->calc_model == kKondoGC) {  // CheckFormatForKondoInt (src/readdef.c:2665-2684)
        if (((m->locspn[s[0]] != 0 || m->locspn[s[1]] != 0) && s[0] != s[1]) ||
            ((m->locspn[s[2]] != 0 || m->locspn[s[3]] != 0) && s[2] != s[3])) {
          *err = files["interall"] + ": Kondo InterAll on a local spin must pair operators of the same site"; return -1;
        }
      }
      if (spin) {
        if (s[0] != s[1] || s[2] != s[3]) {
          *err = files["interall"] + ": spin InterAll needs i==j and k==l"; return -1;
        }
        add_spin_string(m, {{s[0], g[0], g[1]}, {s[2], g[2], g[3]}}, V);
      } else {
        add_fermion_string(m, {{fbit(s[0], g[0]), true}, {fbit(s[1], g[1]), false},
                               {fbit(s[2], g[2]), true}, {fbit(s[3], g[3]), false}}, V);
      }
    }
    m->n_interall = (int)rows.size();
  }
  // ---- Green's function requests (src/readdef.c:1441-1523)
  if (files.count("onebodyg")) {
    std::vector<std::vector<int>> g;
    if (!read_int_table(*m, files["onebodyg"], 4, &g, err)) return -1;
    for (const auto &r : g) {
      if (!check_site(r[0]) || !check_site(r[2]) || !sigma_ok(r[0], r[1]) || !sigma_ok(r[2], r[3])) {
        *err = files["onebodyg"] + ": bad index"; return -1;
      }
      if (m->calc_model == kSpin && r[0] != r[2]) {
        // the reference skips the row (cWarningIncorrectFormatForSpin2, src/readdef.c:1455-1460)
        printf("Warning: Site component of (i, j) =(%d, %d) is ignored.\n", r[0], r[2]);
        continue;
      }
      m->green_one.push_back({r[0], r[1], r[2], r[3]});
    }
  }
  if (files.count("twobodyg")) {
    std::vector<std::vector<int>> g;
    if (!read_int_table(*m, files["twobodyg"], 8, &g, err)) return -1;
    for (const auto &r : g) {
      if (spin && (r[0] != r[2] || r[4] != r[6])) {
        // CheckFormatForSpinInt (src/readdef.c:2637-2651): a fatal input error in the reference
        *err = files["twobodyg"] + ": Site component of (i, j, k, l) =(" + std::to_string(r[0]) + ", " +
               std::to_string(r[2]) + ", " + std::to_string(r[4]) + ", " + std::to_string(r[6]) +
               ") is not correct; i=j and k=l must be satisfied.";
        return -1;
      }
      for (int q = 0; q < 4; q++)
        if (!check_site(r[2 * q]) || !sigma_ok(r[2 * q], r[2 * q + 1])) {
          *err = files["twobodyg"] + ": bad index"; return -1;
        }
      m->green_two.push_back({r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]});
    }
  }
  // three-, four- and six-body rows: read as written (the reference's format check of these
  // rows is disabled, src/readdef.c:1547-1555); indices must be in range here
  const std::pair<const char *, std::vector<std::vector<int>> *> multi[] = {
      {"threebodyg", &m->green_three}, {"fourbodyg", &m->green_four}, {"sixbodyg", &m->green_six}};
  const int multi_pairs[] = {3, 4, 6};
  for (int q = 0; q < 3; q++) {
    if (!files.count(multi[q].first)) continue;
    std::vector<std::vector<int>> g;
    const std::string fn = files[multi[q].first];
    if (!read_int_table(*m, fn, 4 * multi_pairs[q], &g, err)) return -1;
    for (const auto &r : g) {
      for (int k = 0; k < 2 * multi_pairs[q]; k++)
        if (!check_site(r[2 * k]) || !sigma_ok(r[2 * k], r[2 * k + 1])) { *err = fn + ": bad index"; return -1; }
      multi[q].second->push_back(r);
    }
  }
  if (files.count("spectrumvec")) m->spectrum_vec = files["spectrumvec"];
  // ---- TEOneBody / TETwoBody, read for CalcType 4 only (src/readdef.c:755-797, 1752-1840):
  // 5 header lines (the 2nd: "AllTimeStep n"), then per time index a line "time count"
  // followed by count transfer rows (i s1 j s2 re im) or InterAll rows (8 indices, re im)
  if (m->calc_type == kTimeEvolution && (files.count("teonebody") || files.count("tetwobody"))) {
    if (files.count("teonebody") && files.count("tetwobody")) {
      *err = "Time Evolution mode does not support TEOneBody and TETwoBody at the same time";
      return -1;
    }
    const bool one = files.count("teonebody") > 0;
    const std::string fn = files[one ? "teonebody" : "tetwobody"];
    const int ncol = one ? 6 : 10;
    std::ifstream f;
    if (!open_def(*m, fn, &f)) { *err = "cannot open " + fn; return -1; }
    int nsteps = -1;
    for (int i = 0; i < 5; i++) {
      if (!std::getline(f, line)) { *err = fn + ": truncated header"; return -1; }
      std::istringstream ss(line);
      std::string kw;
      if (i == 1 && !(ss >> kw >> nsteps)) { *err = fn + ": bad step count line"; return -1; }
    }
    if (nsteps < 0) { *err = fn + ": negative step count"; return -1; }
    Model scratch = *m;
    auto next_line = [&](std::string *out) {
      while (std::getline(f, *out))
        if (out->find_first_not_of(" \t\r") != std::string::npos) return true;
      return false;
    };
    // a canonical sector admits only terms that keep its particle numbers (and Sz where fixed)
    const uint64_t up_bits = 0x5555555555555555ull, dn_bits = 0xAAAAAAAAAAAAAAAAull;
    auto delta = [](const BitTerm &t, uint64_t mask) {
      return 2 * __builtin_popcountll(t.cv & t.flip & mask) - __builtin_popcountll(t.flip & mask);
    };
    auto keeps_sector = [&](const BitTerm &t) {
      if (m->is_gc() || m->general_spin) return true;
      if (spin) return delta(t, ~0ull) == 0;
      if (m->calc_model == kHubbardNConserved) return delta(t, ~0ull) == 0;
      return delta(t, up_bits) == 0 && delta(t, dn_bits) == 0;
    };
    for (int step = 0; step < nsteps; step++) {
      if (!next_line(&line)) break;
      std::istringstream hs(line);
      double time;
      int count;
      if (!(hs >> time >> count) || count < 0) { *err = fn + ": bad time line: " + line; return -1; }
      std::vector<std::vector<double>> trows;
      for (int q = 0; q < count; q++) {
        std::string row;
        if (!next_line(&row)) { *err = fn + ": truncated at time index " + std::to_string(step); return -1; }
        std::istringstream rs(row);
        std::vector<double> r(ncol);
        for (double &x : r)
          if (!(rs >> x)) { *err = fn + ": malformed line: " + row; return -1; }
        trows.push_back(r);
      }
      scratch.offdiag.clear();
      scratch.diag.clear();
      if (one) {
        // CheckTETransferHermite (src/readdef.c:3100-3220): every row needs its conjugate
        // partner; a site-diagonal row keeps its real part
        for (const auto &r : trows) {
          const int i = (int)r[0], s1 = (int)r[1], j = (int)r[2], s2 = (int)r[3];
          if (!check_site(i) || !check_site(j) || !sigma_ok(i, s1) || !sigma_ok(j, s2)) {
            *err = fn + ": bad site or spin index"; return -1;
          }
          if (spin && i != j) { *err = fn + ": spin models need site-diagonal transfers"; return -1; }
          bool partner = false;
          for (const auto &p : trows)
            if ((int)p[0] == j && (int)p[1] == s2 && (int)p[2] == i && (int)p[3] == s1 &&
                std::abs(std::complex<double>(r[4], r[5]) - std::complex<double>(p[4], -p[5])) <= 1e-12)
              partner = true;
          if (!partner) { *err = fn + ": transfer integrals are not Hermitian"; return -1; }
          std::complex<double> t(r[4], r[5]);
          if (i == j && s1 == s2) t = t.real();
          if (spin) add_spin_string(&scratch, {{i, s1, s2}}, -t);
          else add_fermion_string(&scratch, {{fbit(i, s1), true}, {fbit(j, s2), false}}, -t);
        }
      } else {
        for (const auto &r : trows) {
          int s[4], g[4];
          for (int q = 0; q < 4; q++) { s[q] = (int)r[2 * q]; g[q] = (int)r[2 * q + 1]; }
          for (int q = 0; q < 4; q++)
            if (!check_site(s[q]) || !sigma_ok(s[q], g[q])) { *err = fn + ": bad index"; return -1; }
          const std::complex<double> V(r[8], r[9]);
          if (spin) {
            if (s[0] != s[1] || s[2] != s[3]) { *err = fn + ": spin InterAll needs i==j and k==l"; return -1; }
            add_spin_string(&scratch, {{s[0], g[0], g[1]}, {s[2], g[2], g[3]}}, V);
          } else {
            add_fermion_string(&scratch, {{fbit(s[0], g[0]), true}, {fbit(s[1], g[1]), false},
                                          {fbit(s[2], g[2]), true}, {fbit(s[3], g[3]), false}}, V);
          }
        }
      }
      canonicalize_terms(&scratch);
      for (const auto &t : scratch.offdiag)
        if (!keeps_sector(t)) {
          *err = fn + ": a term at time index " + std::to_string(step) + " leaves the sector";
          return -1;
        }
      m->te_time.push_back(time);
      m->te_offdiag.push_back(scratch.offdiag);
      m->te_diag.push_back(scratch.diag);
    }
    if ((int)m->te_time.size() != nsteps) { *err = fn + ": fewer time indices than AllTimeStep"; return -1; }
    m->te_kind = one ? 1 : 2;
  }
  // ---- SingleExcitation / PairExcitation (src/readdef.c:1943-2007): operators of the
  // excited state A|v> for the dynamical Green's function, compiled in gather form on the
  // excited sector's configurations.  Single: c+_{i s} (type 1) or c_{i s} (type 0), Hubbard
  // models only.  Pair: c+_{i s1} c_{j s2} (type 1) or c_{i s1} c+_{j s2} (type 0; the
  // reference stores it as -c+_{j s2} c_{i s1}, or 1 - n for i = j, s1 = s2); on spins the
  // sites must agree and the pair is the one-site transition |s1><s2| (type 1), 1 - n_{s1}
  // (type 0, s1 = s2) or -|s2><s1| (type 0, s1 != s2) (src/PairExSpin.c:251-330).
  if (files.count("singleexcitation") || files.count("pairexcitation")) {
    if (files.count("singleexcitation") && files.count("pairexcitation")) {
      *err = "Error: Both single and pair excitation operators exist.";
      return -1;
    }
    const bool spin = m->is_spin();
    const bool single = files.count("singleexcitation") > 0;
    const std::string fn = files[single ? "singleexcitation" : "pairexcitation"];
    if (!read_table(*m, fn, &rows, single ? 5 : 7, err)) return -1;
    if (single && spin) { *err = "SingleExcitation is not allowed for spin system."; return -1; }
    auto fbit = [](int site, int sg) { return 2 * site + sg; };
    const uint64_t even = 0x5555555555555555ull;
    int dup = 0, ddn = 0;
    bool first = true;
    for (const auto &r : rows) {
      const int i = (int)r[0], s1 = (int)r[1];
      uint64_t rm = 0, rv = 0, fl = 0, sm = 0;
      int s0 = 0;
      std::complex<double> coef;
      bool ok;
      if (single) {
        const int type = (int)r[2];
        coef = std::complex<double>(r[3], r[4]);
        if (!check_site(i) || s1 < 0 || s1 > 1 || (type != 0 && type != 1)) { *err = fn + ": bad line"; return -1; }
        // the reference's single-operator sign counts the occupied modes above the mode
        // (child_Cis / child_Ajt, GC_Cis / GC_Ajt: src/mltplyHubbardCore.c:980-1180)
        const uint64_t b = 1ull << fbit(i, s1);
        rm = b;
        rv = (type == 1) ? 0 : b;
        fl = b;
        sm = ~((b << 1) - 1);
        ok = true;
      } else {
        const int j = (int)r[2], s2 = (int)r[3], type = (int)r[4];
        coef = std::complex<double>(r[5], r[6]);
        const int smax = spin ? m->locspn[i] : 1;
        if (!check_site(i) || !check_site(j) || s1 < 0 || s1 > smax || s2 < 0 || s2 > smax || (type != 0 && type != 1)) {
          *err = fn + ": bad line";
          return -1;
        }
        if (spin && m->general_spin) {
          // general spin (src/PairExSpin.c:353-440): |s1><s2| whatever the type when s1 != s2;
          // n_{s1} (type 1) or -(1 - n_{s1}) (type 0) when s1 == s2
          if (i != j) { *err = "ERROR: hopping is not allowed in localized spin system"; return -1; }
          std::vector<std::pair<int, std::complex<double>>> ops;  // (state, coefficient) of diagonal parts
          if (s1 != s2) {
            uint64_t grm, grv, gfl;
            if (compile_spin({SpinOp{i, s1, s2}}, m->site_bits, &grm, &grv, &gfl))
              m->excitation.push_back(BitTerm{grm, grv ^ (gfl & grm), gfl, 0, coef.real(), coef.imag()});
          } else if (type == 1) {
            ops.push_back({s1, coef});
          } else {
            for (int t = 0; t <= m->locspn[i]; t++)
              if (t != s1) ops.push_back({t, -coef});
          }
          for (const auto &o : ops) {
            uint64_t grm, grv, gfl;
            if (compile_spin({SpinOp{i, o.first, o.first}}, m->site_bits, &grm, &grv, &gfl))
              m->excitation.push_back(BitTerm{grm, grv ^ (gfl & grm), gfl, 0, o.second.real(), o.second.imag()});
          }
          // Sz change of the operator: a spin state's digit counts up from m = -S, so
          // |s1><s2| changes 2Sz by 2 (s1 - s2) (src/CalcSpectrum.c:588-589)
          const int d2 = s1 - s2;
          if (first) { dup = d2; ddn = 0; first = false; }
          else if (!m->is_gc() && d2 != dup) { *err = fn + ": the operators lead to different sectors"; return -1; }
          continue;
        }
        if (spin) {
          if (i != j) { *err = "Error: isite1 must be equal to isite2 for Spin system."; return -1; }
          SpinOp op{i, s1, s2};
          if (type == 0) {
            if (s1 == s2) op = SpinOp{i, 1 - s1, 1 - s1};
            else { op = SpinOp{i, s2, s1}; coef = -coef; }
          }
          ok = compile_spin({op}, 1, &rm, &rv, &fl);
        } else if (type == 1) {
          ok = compile_fermion({{fbit(i, s1), true}, {fbit(j, s2), false}}, &rm, &rv, &fl, &sm, &s0);
        } else {
          ok = compile_fermion({{fbit(i, s1), false}, {fbit(j, s2), true}}, &rm, &rv, &fl, &sm, &s0);
        }
      }
      if (!ok) continue;  // identically zero (e.g. c c on one mode)
      // particle change of the operator: the flipped bits before (rv & fl) and after
      const uint64_t before = rv & fl, after = (rv ^ fl) & fl;
      const int du = spin ? __builtin_popcountll(after) - __builtin_popcountll(before)
                          : __builtin_popcountll(after & even) - __builtin_popcountll(before & even);
      const int dd = spin ? 0 : __builtin_popcountll(after & ~even) - __builtin_popcountll(before & ~even);
      // HubbardNConserved keeps only the particle number (src/CalcSpectrum.c:521-527)
      const bool n_only = m->calc_model == kHubbardNConserved;
      if (first) { dup = du; ddn = dd; first = false; }
      else if (!m->is_gc() && (n_only ? du + dd != dup + ddn : (du != dup || dd != ddn))) {
        *err = fn + ": the operators lead to different sectors";
        return -1;
      }
      if (s0) coef = -coef;
      if (parity64(fl & sm)) coef = -coef;
      m->excitation.push_back(BitTerm{rm, rv ^ (fl & rm), fl, sm, coef.real(), coef.imag()});
    }
    (single ? m->n_single_ex : m->n_pair_ex) = (int)rows.size();
    m->ex_nup = m->nup;
    m->ex_ndown = m->ndown;
    m->ex_ne = m->ne;
    m->ex_2sz = m->total_2sz;
    if (m->calc_model == kHubbardNConserved) {
      m->ex_ne += dup + ddn;
    } else if (!m->is_gc()) {
      m->ex_nup += dup;
      m->ex_ndown += ddn;
      m->ex_ne += spin ? dup : dup + ddn;
      m->ex_2sz += spin ? 2 * dup : dup - ddn;
    }
  }
  canonicalize_terms(m);
  return 0;
}

}  // namespace hphi
