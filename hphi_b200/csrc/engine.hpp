// Device-resident sector ("Hilbert space") and the kernels that act on it.
//
// One Sector replaces HPhi's globally allocated state for one Hamiltonian
// (list_1, list_2_1, list_2_2, list_Diagonal; src/include/global.h:34-50, allocated by
// setmem_large, src/xsetmem.c:153-249).  Vectors are 0-based device arrays of length
// dim (HPhi's 1-based host arrays carry an unused slot 0; the C-ABI converts at the
// boundary).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "model.hpp"

namespace hphi {

struct HubPlan;
struct ProdPlan;
struct RowBlockPlan;

// Real or complex double scalar for host/device code.
struct cplx { double x, y; };

enum VecType : int { kReal64 = 0, kComplex128 = 1 };

// Upper-half entry of the split-term plan: source row = row + delta (grand-canonical
// models: row ^ delta) with coefficient index k.
struct HiEnt {
  int64_t delta;
  uint32_t k, pad;
};

// Split-term plan of the general kernels (split.cuh): per lower half the applicable
// lower-half terms, per upper half the applicable upper-half terms, the rest generic.
// Device pointers; lo_ptr == nullptr means no plan (every term generic).
struct SplitPlan {
  uint32_t *lo_ptr = nullptr, *lo_ent = nullptr, *hi_ptr = nullptr;
  HiEnt *hi_ent = nullptr;
  double *coef = nullptr;
  BitTerm *gen = nullptr;  // terms left to the generic path
  int ngen = 0;
  int64_t n_lo_ent = 0, n_hi_ent = 0;
};

struct Sector {
  Model model;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool gc = false;                 // grand-canonical: configuration == row index
  int64_t dim = 0;                 // idim_max (src/check.c:51-209)
  int lo_bits = 0, hi_bits = 0;    // HPhi's half split: ihfbit = 2^lo_bits (src/bitcalc.c:45-62)
  uint64_t ihfbit = 0, sdim = 0;   // sdim = number of upper-half configurations (src/check.c:296-328)
  int64_t size_list_2_1 = 0, size_list_2_2 = 0;  // HPhi's allocation sizes (src/xsetmem.c:284-318)

  // Device tables (canonical models).  list_2_1 / list_2_2 hold HPhi's values: the
  // 0-based row of configuration c is list_2_1[c & (ihfbit-1)] + list_2_2[c >> lo_bits] - 3
  // and a zero entry means "not in the sector" (src/bitcalc.c:195-223).
  uint64_t *d_list_1 = nullptr;    // [dim] configurations in HPhi order
  uint32_t *d_list_2_1 = nullptr;  // [ihfbit]
  uint32_t *d_list_2_2 = nullptr;  // [sdim]
  double *d_diag = nullptr;        // [dim] list_Diagonal
  BitTerm *d_terms = nullptr;
  int nterms = 0;
  DiagTerm *d_dterms = nullptr;
  int ndterms = 0;
  double *d_red = nullptr;         // reduction partials
  double *d_scal = nullptr;        // small device scalars (dot results)
  int red_blocks = 0;
  int num_sms = 0;
  // Optional specialised plan (canonical Hubbard).  When present, the drivers keep
  // vectors in the plan's native order; see hv_native / to_native.
  HubPlan *hub = nullptr;
  // Product-layout plan (canonical Hubbard); preferred over the block plan when both apply.
  ProdPlan *prod = nullptr;
  // Row-block plan (spin models, HPhi order): row pass + column pass over the blocks of
  // rows that share an upper half (hv_rowblock.cu).
  RowBlockPlan *rb = nullptr;
  SplitPlan split;
  // General spin: the device tables above are indexed by packed digit codes; HPhi's own
  // mixed-radix lists (src/sz.c:795-830, 1564-1590) are kept here for export.
  std::vector<uint64_t> gs_list_1, gs_list_2_1, gs_list_2_2;
};

// Builds the split-term plan of the term list T into *plan (device arrays; coefficients from
// T).  tab_out: the tabulated terms in coefficient-table order (term tab[i] has entries 4i..4i+3:
// re, im, -re, -im); gen_out: the terms left generic (plan->gen holds them in that order).  A
// plan whose lo_ptr stays null tabulates nothing.  split_plan_free releases it.
int split_plan_for_terms(Sector *s, const std::vector<BitTerm> &T, SplitPlan *plan, std::vector<int> *tab_out,
                         std::vector<int> *gen_out, std::string *err);
void split_plan_free(SplitPlan *p);

// specialise = false skips the specialised kernel plans (the batched engine uses the
// general row kernel only).
int sector_build(const Model &m, int device, Sector **out, std::string *err, bool specialise = true);
// idim_max of the model's sector, computed on the host (src/check.c:51-209).
int64_t sector_dim(const Model &m);
void sector_free(Sector *s);

// v0 = acc * v0 + s * (H v1) with (acc, s) = d_coef[0..1] read on the device, and the raw
// sum_r conj(v1[r]) (H v1)[r] written to d_out[0..1] (re, im).  HPhi's mltply
// (src/mltply.c:56-132) is acc = s = 1, prdct = d_out.  acc == 0 never reads v0.
int hv_launch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out);

// Native vector order: HPhi order unless a specialised plan defines its own (then an
// exact per-block permutation of it).  hv_native runs the fastest kernel on native
// vectors; to_native / from_native convert (they copy when the orders coincide).
bool has_native_order(const Sector *s);
// Block H*V over nb <= kHvBlockMax vectors at d_v1 + b * stride (general kernel path only,
// hv_block_applies): v0_b = acc_b * v0_b + scale_b * H v1_b with (acc_b, scale_b) at
// d_coef + b * cstride and <v1_b|H v1_b> at d_out + b * ostride; d_part holds
// 2 * nb * red_blocks doubles.
constexpr int kHvBlockMax = 8;
bool hv_block_applies(const Sector *s, VecType vt);
int hv_block_native(Sector *s, VecType vt, int nb, int64_t stride, const void *d_v1, void *d_v0,
                    const double *d_coef, int cstride, double *d_out, int ostride, double *d_part);
int hv_native(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
              bool acc_read = true);
int to_native(Sector *s, VecType vt, const void *d_hphi, void *d_native);
int from_native(Sector *s, VecType vt, const void *d_native, void *d_hphi);
// hv_native with caller-provided scratch: d_part receives the per-block partial sums
// (hv_scratch_doubles(s, vt) doubles), d_counter the block counters (2 ints, zeroed on the stream).
int hv_native_scratch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                      double *d_part, int *d_counter);
size_t hv_scratch_doubles(const Sector *s, VecType vt);

// Diagonal observables of a native-order vector (as vec_diag_observables).
int native_observables(Sector *s, VecType vt, const void *d_v, double *d_out);

// ---- vector kernels (vecops.cu); all reductions are deterministic (fixed grid).
// d_out[0] = sum |x|^2
int vec_norm2(Sector *s, VecType vt, const void *d_x, double *d_out);
// d_out[0..1] = sum conj(x) y
int vec_dot(Sector *s, VecType vt, const void *d_x, const void *d_y, double *d_out);
// y = a*x + b*y  (real a, b)
int vec_axpby(Sector *s, VecType vt, double a, const void *d_x, double b, void *d_y);
// x *= a
int vec_scale(Sector *s, VecType vt, double a, void *d_x);
// Lanczos sweep: p = p - alpha*sq*q in place and d_out[0] = |p|^2 (one pass).
int vec_lanczos_sweep(Sector *s, VecType vt, const double *d_alpha_scale, void *d_p, const void *d_q,
                      double *d_out);
// Diagonal observables of a vector: d_out[0] = sum |v|^2 n_up n_dn over sites (doublon),
// d_out[1] = sum |v|^2 * Sz, d_out[2] = sum |v|^2 * N.
int vec_diag_observables(Sector *s, VecType vt, const void *d_v, double *d_out);

// Device-side Lanczos scalar update (see vecops.cu); st is a device array of >= 6 doubles.
int lanczos_scalars(Sector *s, int phase, int k, double *st, double *alpha, double *beta);
// p = p - a_sq*q; vg += c_over_b * p  (eigenvector replay)
int vec_replay_sweep(Sector *s, VecType vt, double a_sq, double c_over_b, void *p, const void *q, void *vg);
// v = cv*v - ch*h and d_out[0] = |v|^2 (TPQ step before normalisation)
int vec_tpq_sweep(Sector *s, VecType vt, double cv, double ch, void *v, const void *h, double *d_out);

// CG sweep (eigenvector refinement): x += a*p; r -= a*(hp + shift*p); d_out[0] = |r|^2.
int vec_cg_sweep(Sector *s, VecType vt, double a, double shift, const void *p, const void *hp, void *x, void *r,
                 double *d_out);
// x = the hashed start vector start_value(seed, configuration of row i, part) (HPhi order, not
// normalised; imaginary parts only for complex vectors).
int vec_fill_hashed(Sector *s, VecType vt, uint64_t seed, void *d_x);
// x[i] += amp * start_value(seed, configuration of row i, 0) on the real part (HPhi order).
int vec_add_hashed(Sector *s, VecType vt, uint64_t seed, double amp, void *d_x);
// <v| O_e |v> of compiled Green's function entries (compile_green) on a device vector in
// HPhi's row order; out = (re, im) per entry (green.cu).
int green_expect(Sector *s, VecType vt, const void *d_v, const std::vector<GreenTerm> &terms,
                 std::vector<double> *out);
// Uploads a host vector in HPhi's layout for green_expect: real parts only (*vt = kReal64)
// when every imaginary part is zero, else complex.  *d_vec is the caller's to cudaFree.
int green_stage_host_vector(Sector *s, const double *h_v_1based, void **d_vec, VecType *vt);

// Real-time evolution (te.cu), complex vectors in HPhi's row order:
// v0 += (terms of one time index) v1, the terms compiled like the static ones;
// y += (a_re + i a_im) x.
// plan: split-term plan of the union of every time index's off-diagonal terms, with d_coef the
// index's coefficient table (plan->coef is not read); d_off / noff: the index's generic terms.
int te_terms_apply(Sector *s, const SplitPlan &plan, const double *d_coef, const BitTerm *d_off, int noff,
                   const DiagTerm *d_diag, int ndiag, const void *d_v1, void *d_v0);
int vec_caxpy(Sector *s, double a_re, double a_im, const void *d_x, void *d_y);

// complex128 <-> real and imaginary parts (n = dim); y[0, n) += x[0, n) on stream st.
int vec_split_c128(Sector *s, const void *d_c, double *d_re, double *d_im);
int vec_join_c128(Sector *s, const double *d_re, const double *d_im, void *d_c);
int vec_add_c128(Sector *s, cudaStream_t st, int64_t n, void *d_y, const void *d_x);

// Copies between HPhi's 1-based complex128 host layout and a device vector.
int vec_from_host_c128(Sector *s, VecType vt, const double *h_v_1based, void *d_v);
int vec_to_host_c128(Sector *s, VecType vt, const void *d_v, double *h_v_1based);

void set_error(const std::string &msg);
const char *get_error();

}  // namespace hphi
