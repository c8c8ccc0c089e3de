// Host-side model description: HPhi expert-mode input compiled to bit-operator terms.
//
// Every Hamiltonian term that HPhi reads from its expert-mode .def files (Trans,
// CoulombIntra, CoulombInter, Hund, Ising, Exchange, PairHop, PairLift, InterAll;
// reader in src/readdef.c:1006-2059) is an operator string acting on the occupation
// bits of a configuration.  On a basis configuration c such a string either gives
// zero or a single configuration c ^ flip with a coefficient whose sign is
// (-1)^popcount(c & sign_mask) times a constant.  That closed form is what the GPU
// kernels evaluate; it reproduces the per-term element routines of
// src/mltplyHubbardCore.c and src/mltplySpinCore.c (masks from the *_GetInfo
// functions, fermion signs from SgnBit, src/bitcalc.c:338-352).
#pragma once
#include <array>
#include <complex>
#include <cstdint>
#include <string>
#include <vector>

namespace hphi {

// CalcModel values of calcmod.def (include/DefCommon.h:21-39).  HubbardNConserved is
// the internal model HPhi switches to when Hubbard is given Ncond without 2Sz
// (src/readdef.c:905-912).
enum CalcModel : int {
  kHubbard = 0, kSpin = 1, kKondo = 2, kHubbardGC = 3, kSpinGC = 4, kKondoGC = 5,
  kHubbardNConserved = 6
};
// CalcType values (include/DefCommon.h).
enum CalcType : int { kLanczos = 0, kTPQ = 1, kFullDiag = 2, kCG = 3, kTimeEvolution = 4, kcTPQ = 5 };

// Off-diagonal term in gather ("pull") form, for an output configuration t:
//   applies iff (t & cm) == cv; source configuration s = t ^ flip;
//   contribution = (re + i im) * (-1)^popcount(t & sm) * v[index(s)].
struct BitTerm {
  uint64_t cm, cv, flip, sm;
  double re, im;
};

// Diagonal projector term: adds v iff (c & cm) == cv.
struct DiagTerm {
  uint64_t cm, cv;
  double v;
};

struct Model {
  // calcmod.def
  int calc_type = 0, calc_model = 0, output_mode = 0, calc_eigenvec = 0, initial_vec_type = 0;
  int output_eigenvec = 0, input_eigenvec = 0, restart = 0, flg_finite_temperature = 0;
  // modpara.def
  int nsite = 0, nup = 0, ndown = 0, ne = 0, total_2sz = 0, ncond = 0;
  bool sz_conserved = false, read_ncond = false;
  int lanczos_max = 0, initial_iv = 0, nvec = 0, k_exct = 0, lanczos_eps = 0, lanczos_target = 0;
  int num_ave = 1, expec_interval = 1, read_hacker = 1;
  int pre_cg = 0;               // PreCG: point-Jacobi preconditioning in LOBPCG (src/readdef.c:646)
  int expand_coef = 0;          // ExpandCoef: Taylor order of the cTPQ step (0: 10, src/CalcByCanonicalTPQ.c:81-86)
  double large_value = 0.0;
  std::string data_head = "zvo", para_head = "zqp";
  // locspn.def
  int nlocspn = 0;
  std::vector<int> locspn;
  // Compiled Hamiltonian.
  std::vector<BitTerm> offdiag;
  std::vector<DiagTerm> diag;
  bool complex_terms = false;   // any off-diagonal coefficient with a non-zero imaginary part
  int nbits = 0;                // configuration bits: 2*Nsite (Hubbard/Kondo) or Nsite (spin)
  // General spin (some site with 2S > 1, src/readdef.c:2735-2760): site i holds a digit
  // 0 .. 2S_i (2Sz_i = 2*digit - 2S_i, GetLocal2Sz src/bitcalc.c:447-461) in a field of
  // site_bits bits at bit site_bits * i, so configurations are packed digit strings whose
  // numeric order is HPhi's mixed-radix order.  Spin-1/2 models have site_bits = 1.
  bool general_spin = false;
  int site_bits = 1;
  // Green's function requests as read (0-based sites): OneBodyG rows (i, s1, j, s2) and
  // TwoBodyG rows (i, s1, j, s2, k, s3, l, s4) (src/readdef.c:1441-1523).  A canonical Spin
  // model drops one-body rows with i != j, as the reference does with a warning.
  std::vector<std::array<int, 4>> green_one;
  std::vector<std::array<int, 8>> green_two;
  // ThreeBodyG / FourBodyG / SixBodyG rows (3, 4, 6 site pairs of 4 integers each,
  // src/readdef.c:1525-1700);
  // the reference evaluates them for spin-1/2 SpinGC only.
  std::vector<std::vector<int>> green_three, green_four, green_six;
  // Time evolution (CalcType 4, src/CalcByTEM.c:52-234): the terms of TEOneBody (te_kind 1,
  // transfers) or TETwoBody (te_kind 2, InterAll) at each time index, compiled like the static
  // terms and added to H at that step (MakeTEDTransfer / MakeTEDInterAll :237-279 for the
  // off-diagonal part, diagonalcalcForTE src/diagonalcalc.c:195-245 for the diagonal part).
  int te_kind = 0;
  std::vector<double> te_time;                   // TETime[step]
  std::vector<std::vector<BitTerm>> te_offdiag;  // per step
  std::vector<std::vector<DiagTerm>> te_diag;    // per step
  std::string spectrum_vec;                      // SpectrumVec: head of the input vector file
  // Dynamical Green's function (CalcSpec 1, src/CalcSpectrum.c:90-312): the SingleExcitation or
  // PairExcitation operators compiled in gather form on the excited sector (flip 0 allowed),
  // that sector's particle numbers (MakeExcitedList, :438-634) and the frequency grid
  // (modpara OmegaMax / OmegaMin / OmegaIm / OmegaOrg / NOmega, src/readdef.c:624-642).
  int calc_spec = 0;
  int output_exvec = 0;
  int n_single_ex = 0, n_pair_ex = 0;
  std::vector<BitTerm> excitation;
  int ex_nup = 0, ex_ndown = 0, ex_ne = 0, ex_2sz = 0;
  bool omega_max_set = false, omega_min_set = false, omega_org_set = false;
  double omega_max[2] = {0.0, 0.0}, omega_min[2] = {0.0, 0.0}, omega_org[2] = {0.0, 0.0};
  int n_omega = 1000;
  int output_interval = 0;                       // OutputInterval (eigenvector files)
  // Raw term counts as read (for logs).
  int n_trans = 0, n_coulomb_intra = 0, n_coulomb_inter = 0, n_hund = 0, n_exchange = 0;
  int n_ising = 0, n_pairhop = 0, n_pairlift = 0, n_interall = 0;
  std::string base_dir;

  bool is_gc() const {
    return calc_model == kHubbardGC || calc_model == kSpinGC || calc_model == kKondoGC;
  }
  bool is_spin() const { return calc_model == kSpin || calc_model == kSpinGC; }
  // Grand-canonical models whose basis is every configuration (row index == configuration);
  // KondoGC keeps lists because its local spins must stay singly occupied.
  bool rows_are_configs() const { return calc_model == kHubbardGC || (calc_model == kSpinGC && !general_spin); }
  bool is_kondo() const { return calc_model == kKondo || calc_model == kKondoGC; }
};

// Reads namelist.def and every file it names (expert mode).  Returns 0 on success,
// -1 with a message in *err otherwise.  Mirrors ReadDefFileNInt / ReadDefFileIdxPara
// (src/readdef.c:463, 1006) for the keywords this engine supports.
int read_expert(const std::string &namelist, Model *m, std::string *err);

// Adds a literal operator string to the compiled model.  Fermion strings are lists
// of (bit, dagger) applied right to left; spin strings are lists of (site, to, from)
// single-site transitions |to><from|.  Returns false for an identically-zero string.
struct FermionOp { int bit; bool dag; };
struct SpinOp { int site, to, from; };
bool add_fermion_string(Model *m, const std::vector<FermionOp> &ops, std::complex<double> coef);
bool add_spin_string(Model *m, const std::vector<SpinOp> &ops, std::complex<double> coef);

// Merges duplicate terms (same masks) by adding their coefficients, drops zeros.
void canonicalize_terms(Model *m);

// One Green's function entry <v| O |v> in push form: a row whose configuration c has
// (c & cm) == cv contributes coef * (-1)^popcount(c & sm) * conj(v[row(c ^ flip)]) * v[row(c)]
// (no contribution when c ^ flip is outside the sector).  coef == 0 marks an entry that is
// zero by the reference's rules.
struct GreenTerm {
  uint64_t cm, cv, flip, sm;
  double coef, unused;
};

// Compiles Green's function rows (body 1: OneBodyG rows i s1 j s2; body 2: TwoBodyG rows
// i s1 j s2 k s3 l s4; body 3 / 4 / 6: ThreeBodyG / FourBodyG / SixBodyG rows of 3 / 4 / 6
// site pairs; 0-based sites) following expec_cisajs (src/expec_cisajs.c:66-641) and
// expec_cisajscktaltdc (src/expec_cisajscktaltdc.c:87-1647).  flag[e] (bodies 1, 2):
// the reference prints the entry's line with a space before the newline; (bodies 3, 4, 6):
// the reference prints only the first 8 indices (its Rearray_Interactions rejected the row).
// Returns 0, or -1 with a message for an index out of range.
int compile_green(const Model &m, int body, const int *rows, int n, std::vector<GreenTerm> *terms,
                  std::vector<char> *trailing_space, std::string *err);

}  // namespace hphi
