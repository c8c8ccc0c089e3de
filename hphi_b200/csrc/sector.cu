// Sector enumeration and diagonal on the device.
//
// Replaces sz() (src/sz.c:62-832, hacker paths omp_sz_hacker :993-1094 and
// omp_sz_spin_hacker :1495-1546) and diagonalcalc() (src/diagonalcalc.c:84-187).
//
// HPhi orders the canonical sector by upper half ib (bits >= lo_bits) and, inside
// a block, by increasing lower half ia.  Which ia are allowed depends only on the
// particle-number class of ib, so
//   list_2_1[ia] = rank of ia among lower halves of its class + 2   (0 if the class
//                  is never needed by any ib),
//   list_2_2[ib] = (number of rows in blocks before ib) + 1          (0 for empty blocks),
//   list_1[jb + ja] = unrank(class, ja) | ib << lo_bits.
// The serial list_jb prefix loop of the reference becomes a device scan; the per-block
// snoob enumeration becomes a gather from a per-class unrank table.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>

#include "engine.hpp"
#include "hv_hubbard.hpp"
#include "hv_rowblock.hpp"
#include "hv_product.hpp"
#include "split.cuh"

namespace hphi {
namespace {

#define CK(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      *err = std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call; \
      return -1;                                                                  \
    }                                                                             \
  } while (0)

__constant__ uint64_t c_binom[65][65];

// Class of a half configuration: (n_even, n_odd) by global bit parity for Hubbard
// (even bit = up, src/sz.c:1006-1015), popcount otherwise.  class id = a*(D+1)+b.
__device__ __forceinline__ void half_counts(uint64_t x, int offset, int hubbard, int *a, int *b) {
  if (!hubbard) { *a = __popcll(x); *b = 0; return; }
  // global position offset + p is even (up) iff p has the parity of offset.
  const uint64_t even_local = (offset & 1) ? 0xAAAAAAAAAAAAAAAAull : 0x5555555555555555ull;
  *a = __popcll(x & even_local);
  *b = __popcll(x & ~even_local);
}

// Rank of x among half configurations of the same class (increasing order).
__device__ uint64_t half_rank(uint64_t x, int nbits, int offset, int hubbard) {
  const uint64_t even_local = (offset & 1) ? 0xAAAAAAAAAAAAAAAAull : 0x5555555555555555ull;
  uint64_t r = 0;
  int need_a = 0, need_b = 0;  // class counts of x restricted to positions <= p
  // walk from low to high so that need_* are the counts at and below p
  for (int p = 0; p < nbits; p++) {
    const uint64_t bit = 1ull << p;
    const bool is_a = !hubbard || (even_local & bit);
    if (x & bit) {
      if (is_a) need_a++; else need_b++;
      const uint64_t below = bit - 1;
      int na, nb;
      if (!hubbard) { na = p; nb = 0; }
      else { na = __popcll(below & even_local); nb = __popcll(below & ~even_local); }
      if (need_a <= na && need_b <= nb) r += c_binom[na][need_a] * c_binom[nb][need_b];
    }
  }
  return r;
}

__global__ void lo_tables_kernel(uint64_t ihfbit, int lo_bits, int hubbard, int D,
                                 const unsigned char *__restrict__ valid_cls,
                                 const uint64_t *__restrict__ cls_off, uint32_t *__restrict__ list_2_1,
                                 uint32_t *__restrict__ unrank) {
  const uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (x >= ihfbit) return;
  int a, b;
  half_counts(x, 0, hubbard, &a, &b);
  const int cls = a * (D + 1) + b;
  const uint64_t r = half_rank(x, lo_bits, 0, hubbard);
  list_2_1[x] = valid_cls[cls] ? (uint32_t)(r + 2) : 0u;
  unrank[cls_off[cls] + r] = (uint32_t)x;
}

__global__ void hi_count_kernel(uint64_t sdim, int lo_bits, int hubbard, int D_lo, int ta, int tb,
                                const uint64_t *__restrict__ cls_cnt, int max_a, int max_b,
                                uint64_t *__restrict__ cnt, int *__restrict__ need) {
  const uint64_t ib = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (ib >= sdim) return;
  int a, b;
  half_counts(ib, lo_bits, hubbard, &a, &b);
  const int na = ta - a, nb = tb - b;
  if (na < 0 || nb < 0 || na > max_a || nb > max_b) { cnt[ib] = 0; need[ib] = -1; return; }
  const int cls = na * (D_lo + 1) + nb;
  cnt[ib] = cls_cnt[cls];
  need[ib] = cls;
}

// Exclusive scan of cnt into jb (single block, deterministic), total into *total.
__global__ void scan_kernel(uint64_t n, const uint64_t *__restrict__ cnt, uint64_t *__restrict__ jb,
                            uint64_t *__restrict__ total) {
  __shared__ uint64_t warp_sums[32];
  __shared__ uint64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (uint64_t base = 0; base < n; base += blockDim.x) {
    const uint64_t i = base + threadIdx.x;
    const uint64_t v = (i < n) ? cnt[i] : 0;
    uint64_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      const int nw = blockDim.x >> 5;
      uint64_t w = (lane < nw) ? warp_sums[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const uint64_t t = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += t;
      }
      if (lane < nw) warp_sums[lane] = w;
    }
    __syncthreads();
    const uint64_t warp_prefix = (wid > 0) ? warp_sums[wid - 1] : 0;
    if (i < n) jb[i] = carry + warp_prefix + incl - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += warp_prefix + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void list_2_2_kernel(uint64_t sdim, const uint64_t *__restrict__ cnt, const uint64_t *__restrict__ jb,
                                uint32_t *__restrict__ list_2_2) {
  const uint64_t ib = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (ib >= sdim) return;
  list_2_2[ib] = cnt[ib] ? (uint32_t)(jb[ib] + 1) : 0u;
}

// One block per upper half ib (grid-strided), threads over the block's rows.
__global__ void list_1_kernel(uint64_t sdim, int lo_bits, const uint64_t *__restrict__ cnt,
                              const uint64_t *__restrict__ jb, const int *__restrict__ need,
                              const uint64_t *__restrict__ cls_off, const uint32_t *__restrict__ unrank,
                              uint64_t *__restrict__ list_1) {
  for (uint64_t ib = blockIdx.x; ib < sdim; ib += gridDim.x) {
    const uint64_t n = cnt[ib];
    if (!n) continue;
    const uint64_t base = jb[ib];
    const uint32_t *u = unrank + cls_off[need[ib]];
    const uint64_t hi = ib << lo_bits;
    for (uint64_t ja = threadIdx.x; ja < n; ja += blockDim.x) list_1[base + ja] = (uint64_t)u[ja] | hi;
  }
}

__global__ void diag_kernel(int64_t dim, int gc, const uint64_t *__restrict__ list_1,
                            const DiagTerm *__restrict__ terms, int nterms, double *__restrict__ diag) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = gc ? (uint64_t)r : list_1[r];
    double d = 0.0;
    for (int k = 0; k < nterms; k++) {
      const DiagTerm t = terms[k];
      if ((c & t.cm) == t.cv) d += t.v;
    }
    diag[r] = d;
  }
}

uint64_t binom_host(int n, int k) {
  if (k < 0 || n < 0 || k > n) return 0;
  uint64_t r = 1;
  for (int i = 1; i <= k; i++) r = r * (uint64_t)(n - k + i) / (uint64_t)i;
  return r;
}

}  // namespace

static int split_plan_build(Sector *s, std::string *err) {
  return split_plan_for_terms(s, s->model.offdiag, &s->split, nullptr, nullptr, err);
}

// Split-term plan (split.cuh): classifies the compiled terms by which half of the
// configuration their masks touch and tabulates the lower-half and upper-half ones.
// Skipped (every term generic) when a half has more than 18 bits or the entry fields
// would overflow.
int split_plan_for_terms(Sector *s, const std::vector<BitTerm> &T, SplitPlan *plan, std::vector<int> *tab_out,
                         std::vector<int> *gen_out, std::string *err) {
  SplitPlan &P = *plan;
  const uint64_t lo_mask = s->ihfbit - 1;
  std::vector<int> lo_t, hi_t, gen_t;
  for (int q = 0; q < (int)T.size(); q++) {
    const uint64_t all = T[q].cm | T[q].flip | T[q].sm;
    if ((all & ~lo_mask) == 0) lo_t.push_back(q);
    else if ((all & lo_mask) == 0) hi_t.push_back(q);
    else gen_t.push_back(q);
  }
  const bool usable = s->lo_bits <= 18 && s->hi_bits <= 18 && 2 * (lo_t.size() + hi_t.size()) < 4096 &&
                      (s->gc || s->dim < (int64_t)(1ll << 40));
  if (!usable) {
    lo_t.clear();
    hi_t.clear();
    gen_t.clear();
    for (int q = 0; q < (int)T.size(); q++) gen_t.push_back(q);
  }
  std::vector<BitTerm> gen;
  for (int q : gen_t) gen.push_back(T[q]);
  if (gen_out) *gen_out = gen_t;
  if (tab_out) tab_out->clear();
  P.ngen = (int)gen.size();
  if (P.ngen) {
    CK(cudaMalloc(&P.gen, sizeof(BitTerm) * gen.size()));
    CK(cudaMemcpy(P.gen, gen.data(), sizeof(BitTerm) * gen.size(), cudaMemcpyHostToDevice));
  }
  if (!usable) return 0;
  // coefficient table: index 2i / 2i+1 = +/- coefficient of the i-th tabulated term
  std::vector<int> tab;
  for (int q : lo_t) tab.push_back(q);
  for (int q : hi_t) tab.push_back(q);
  if (tab_out) *tab_out = tab;
  std::vector<double> coef(4 * tab.size() + 2, 0.0);
  for (size_t i = 0; i < tab.size(); i++) {
    coef[4 * i] = T[tab[i]].re;
    coef[4 * i + 1] = T[tab[i]].im;
    coef[4 * i + 2] = -T[tab[i]].re;
    coef[4 * i + 3] = -T[tab[i]].im;
  }
  std::vector<uint32_t> l21, l22;
  if (!s->gc) {
    l21.resize(s->ihfbit);
    l22.resize(s->sdim);
    CK(cudaMemcpy(l21.data(), s->d_list_2_1, sizeof(uint32_t) * s->ihfbit, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(l22.data(), s->d_list_2_2, sizeof(uint32_t) * s->sdim, cudaMemcpyDeviceToHost));
  }
  const uint64_t nlo = s->ihfbit, nhi = s->sdim;
  std::vector<uint32_t> lo_ptr(nlo + 1, 0), lo_ent;
  for (uint64_t ia = 0; ia < nlo; ia++) {
    lo_ptr[ia] = (uint32_t)lo_ent.size();
    if (!s->gc && l21[ia] == 0) continue;
    for (size_t i = 0; i < lo_t.size(); i++) {
      const BitTerm &t = T[lo_t[i]];
      if ((ia & t.cm) != t.cv) continue;
      const uint64_t src = ia ^ t.flip;
      const uint64_t val = s->gc ? src : l21[src];
      if (!s->gc && val == 0) continue;
      if (val >= (1ull << kSplitTargetBits)) {
        *err = "split plan: lower-half value out of range";
        return -1;
      }
      const uint32_t k = 2 * (uint32_t)i + (uint32_t)(__builtin_popcountll(ia & t.sm) & 1);
      lo_ent.push_back((uint32_t)val | (k << kSplitTargetBits));
    }
    if (lo_ent.size() > 0xFFFFFFF0ull) { *err = "split plan: too many entries"; return -1; }
  }
  lo_ptr[nlo] = (uint32_t)lo_ent.size();
  std::vector<uint32_t> hi_ptr(nhi + 1, 0);
  std::vector<HiEnt> hi_ent;
  for (uint64_t ib = 0; ib < nhi; ib++) {
    hi_ptr[ib] = (uint32_t)hi_ent.size();
    if (!s->gc && l22[ib] == 0) continue;
    const uint64_t cfg = ib << s->lo_bits;
    for (size_t i = 0; i < hi_t.size(); i++) {
      const BitTerm &t = T[hi_t[i]];
      if ((cfg & t.cm) != t.cv) continue;
      HiEnt h{};
      if (s->gc) {
        h.delta = (int64_t)t.flip;
      } else {
        const uint64_t src = (cfg ^ t.flip) >> s->lo_bits;
        if (l22[src] == 0) continue;
        h.delta = (int64_t)l22[src] - (int64_t)l22[ib];
      }
      h.k = 2 * (uint32_t)(lo_t.size() + i) + (uint32_t)(__builtin_popcountll(cfg & t.sm) & 1);
      hi_ent.push_back(h);
    }
    if (hi_ent.size() > 0xFFFFFFF0ull) { *err = "split plan: too many entries"; return -1; }
  }
  hi_ptr[nhi] = (uint32_t)hi_ent.size();
  P.n_lo_ent = (int64_t)lo_ent.size();
  P.n_hi_ent = (int64_t)hi_ent.size();
  CK(cudaMalloc(&P.lo_ptr, sizeof(uint32_t) * lo_ptr.size()));
  CK(cudaMalloc(&P.lo_ent, sizeof(uint32_t) * std::max<size_t>(1, lo_ent.size())));
  CK(cudaMalloc(&P.hi_ptr, sizeof(uint32_t) * hi_ptr.size()));
  CK(cudaMalloc(&P.hi_ent, sizeof(HiEnt) * std::max<size_t>(1, hi_ent.size())));
  CK(cudaMalloc(&P.coef, sizeof(double) * coef.size()));
  CK(cudaMemcpy(P.lo_ptr, lo_ptr.data(), sizeof(uint32_t) * lo_ptr.size(), cudaMemcpyHostToDevice));
  if (!lo_ent.empty()) CK(cudaMemcpy(P.lo_ent, lo_ent.data(), sizeof(uint32_t) * lo_ent.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(P.hi_ptr, hi_ptr.data(), sizeof(uint32_t) * hi_ptr.size(), cudaMemcpyHostToDevice));
  if (!hi_ent.empty()) CK(cudaMemcpy(P.hi_ent, hi_ent.data(), sizeof(HiEnt) * hi_ent.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(P.coef, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice));
  return 0;
}

void split_plan_free(SplitPlan *p) {
  cudaFree(p->lo_ptr); cudaFree(p->lo_ent); cudaFree(p->hi_ptr); cudaFree(p->hi_ent);
  cudaFree(p->coef); cudaFree(p->gen);
  *p = SplitPlan();
}

int64_t sector_dim(const Model &m) {
  if (m.calc_model == kKondoGC) {  // 4^Ncond * 2^NLocSpn (src/check.c:160-168)
    const int nloc = m.nlocspn, ncond = m.nsite - m.nlocspn;
    return (int64_t)1 << (2 * ncond + nloc);
  }
  if (m.calc_model == kKondo) {  // src/check.c:134-158
    const int nloc = m.nlocspn, ncond = m.nsite - m.nlocspn;
    uint64_t sum = 0;
    for (int ul = 0; ul <= m.nup; ul++)
      sum += binom_host(nloc, ul) * binom_host(ncond, m.nup - ul) * binom_host(ncond, m.ndown + ul - nloc);
    return (int64_t)sum;
  }
  if (m.general_spin) {
    // check.c:171-200 / 102-111: configurations of the mixed-radix space with total 2Sz
    // (every configuration in the grand-canonical case), counted by a sum over sites
    std::map<int, uint64_t> cnt{{0, 1}};
    for (int i = 0; i < m.nsite; i++) {
      std::map<int, uint64_t> nx;
      for (const auto &kv : cnt)
        for (int d = 0; d <= m.locspn[i]; d++) nx[kv.first + 2 * d - m.locspn[i]] += kv.second;
      cnt.swap(nx);
    }
    if (m.is_gc()) {
      uint64_t t = 0;
      for (const auto &kv : cnt) t += kv.second;
      return (int64_t)t;
    }
    auto it = cnt.find(m.total_2sz);
    return it == cnt.end() ? 0 : (int64_t)it->second;
  }
  if (m.is_gc()) return (int64_t)(1ull << m.nbits);
  if (m.calc_model == kHubbard) return (int64_t)(binom_host(m.nsite, m.nup) * binom_host(m.nsite, m.ndown));
  if (m.calc_model == kHubbardNConserved) return (int64_t)binom_host(2 * m.nsite, m.ne);
  return (int64_t)binom_host(m.nsite, m.ne);
}

int sector_build(const Model &m, int device, Sector **out, std::string *err, bool specialise) {
  CK(cudaSetDevice(device));
  Sector *s = new Sector();
  s->model = m;
  s->device = device;
  CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  int nsm = 0;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  s->num_sms = nsm;
  s->red_blocks = nsm * 8;
  CK(cudaMalloc(&s->d_red, sizeof(double) * 8 * (size_t)s->red_blocks));
  CK(cudaMalloc(&s->d_scal, sizeof(double) * 64));

  const int nbits = m.nbits;
  s->gc = m.rows_are_configs();
  // GetSplitBit (src/bitcalc.c:45-62): ihfbit = 2^((Nbits+1)/2).
  s->lo_bits = (nbits + 1) / 2;
  s->hi_bits = nbits - s->lo_bits;
  s->ihfbit = 1ull << s->lo_bits;
  s->sdim = 1ull << s->hi_bits;
  // HPhi's list_2_* allocation sizes (GetlistSize, src/xsetmem.c:284-318).
  s->size_list_2_2 = (int64_t)s->sdim + 2;
  s->size_list_2_1 = (int64_t)s->ihfbit + 2;

  if (s->gc) {
    s->dim = (int64_t)(1ull << nbits);
  } else if (m.general_spin) {
    // General spin (src/sz.c:795-830, 1564-1590; GetSplitBitForGeneralSpin src/bitcalc.c:
    // 124-150).  HPhi splits the mixed-radix configuration at the first prefix of sites whose
    // product ihfbit reaches floor(sqrt(total)); blocks by increasing upper index ib, inside a
    // block the lower indices ia whose 2Sz completes Total2Sz (every ia when grand-canonical),
    // list_2_1[ia] = rank within its 2Sz class + 2, list_2_2[ib] = block offset + 1.  The
    // engine's configurations are packed digit codes split at the same site; its device tables
    // hold HPhi's values at the packed codes (0 for codes with an out-of-range digit).
    const int N = m.nsite, b = m.site_bits;
    const bool gcs = m.is_gc();
    std::vector<uint64_t> radix(N), tpow(N + 1, 1);
    for (int i = 0; i < N; i++) { radix[i] = (uint64_t)m.locspn[i] + 1; tpow[i + 1] = tpow[i] * radix[i]; }
    const uint64_t total = tpow[N];
    const int64_t isq = (int64_t)std::sqrt((double)(int64_t)total);
    int k = 0;
    uint64_t hf = 1;
    for (int i = 0; i < N; i++) {
      hf *= radix[i];
      k = i + 1;
      if ((int64_t)hf >= isq) break;
    }
    const uint64_t nlo = hf, nhi = total / hf;
    s->lo_bits = b * k;
    s->hi_bits = nbits - s->lo_bits;
    if (s->lo_bits > 26 || s->hi_bits > 26) { *err = "general-spin sector too large for the packed tables"; return -1; }
    s->ihfbit = 1ull << s->lo_bits;
    s->sdim = 1ull << s->hi_bits;
    s->size_list_2_1 = (int64_t)nlo + 2;     // GetlistSize (src/xsetmem.c:305-310)
    s->size_list_2_2 = (int64_t)nhi + 2;
    auto digits_sz = [&](uint64_t x, int site0, int nsites, uint64_t *packed) {
      int sz = 0;
      uint64_t pk = 0;
      for (int j = 0; j < nsites; j++) {
        const int d = (int)(x % radix[site0 + j]);
        x /= radix[site0 + j];
        sz += 2 * d - m.locspn[site0 + j];
        pk |= (uint64_t)d << (b * j);
      }
      *packed = pk;
      return sz;
    };
    std::vector<int> sz_lo(nlo), sz_hi(nhi);
    std::vector<uint64_t> pk_lo(nlo), pk_hi(nhi);
    for (uint64_t ia = 0; ia < nlo; ia++) sz_lo[ia] = digits_sz(ia, 0, k, &pk_lo[ia]);
    for (uint64_t ib = 0; ib < nhi; ib++) sz_hi[ib] = digits_sz(ib, k, N - k, &pk_hi[ib]);
    std::map<int, std::vector<uint64_t>> cls;  // 2Sz of the lower part -> its ia, increasing
    for (uint64_t ia = 0; ia < nlo; ia++) cls[gcs ? 0 : sz_lo[ia]].push_back(ia);
    std::vector<uint64_t> h21(nlo + 2, 0), h22(nhi + 2, 0), h1(1, 0), l1;
    std::vector<uint32_t> d21(s->ihfbit, 0), d22(s->sdim, 0);
    std::map<int, bool> used;
    uint64_t jb = 0;
    for (uint64_t ib = 0; ib < nhi; ib++) {
      auto it = cls.find(gcs ? 0 : m.total_2sz - sz_hi[ib]);
      if (it == cls.end()) continue;
      used[it->first] = true;
      h22[ib] = jb + 1;
      d22[pk_hi[ib]] = (uint32_t)(jb + 1);
      for (uint64_t ia : it->second) {
        h1.push_back(ia + ib * nlo);
        l1.push_back(pk_lo[ia] | (pk_hi[ib] << s->lo_bits));
      }
      jb += it->second.size();
    }
    for (const auto &kv : cls)
      if (used.count(kv.first))
        for (size_t r = 0; r < kv.second.size(); r++) {
          h21[kv.second[r]] = r + 2;
          d21[pk_lo[kv.second[r]]] = (uint32_t)(r + 2);
        }
    const int64_t expect = sector_dim(m);
    if ((int64_t)jb != expect || jb == 0) {
      *err = "general-spin sector size mismatch: enumerated " + std::to_string(jb) + ", expected " +
             std::to_string(expect);
      return -1;
    }
    if (jb > 0xFFFFFFF0ull) { *err = "sector too large for 32-bit list_2 tables"; return -1; }
    s->dim = (int64_t)jb;
    if (!gcs) {
      s->gs_list_1.swap(h1);
      s->gs_list_2_1.swap(h21);
      s->gs_list_2_2.swap(h22);
    }
    CK(cudaMalloc(&s->d_list_2_1, sizeof(uint32_t) * s->ihfbit));
    CK(cudaMalloc(&s->d_list_2_2, sizeof(uint32_t) * s->sdim));
    CK(cudaMalloc(&s->d_list_1, sizeof(uint64_t) * jb));
    CK(cudaMemcpy(s->d_list_2_1, d21.data(), sizeof(uint32_t) * s->ihfbit, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->d_list_2_2, d22.data(), sizeof(uint32_t) * s->sdim, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->d_list_1, l1.data(), sizeof(uint64_t) * jb, cudaMemcpyHostToDevice));
  } else if (m.is_kondo()) {
    // Kondo / KondoGC (src/sz.c:541-635, 1110-1220, 1342-1420): a half is admissible when
    // its local spins are singly occupied; blocks by increasing upper half ib, inside a block
    // the admissible lower halves ia of the needed (up, down) counts (KondoGC: all of them)
    // in increasing order; list_2_1[ia] = rank + 2, list_2_2[ib] = block offset + 1.
    const int N = m.nsite, half = N / 2;
    const uint64_t nh = 1ull << N;
    if (s->lo_bits != N || s->hi_bits != N) { *err = "Kondo sector: unexpected half split"; return -1; }
    auto admissible = [&](uint64_t x, int site0) {
      for (int j = 0; j < half; j++)
        if (m.locspn[site0 + j] != 0 && ((x >> (2 * j)) & 1ull) == ((x >> (2 * j + 1)) & 1ull)) return false;
      return true;
    };
    const uint64_t even = 0x5555555555555555ull;
    const bool gck = (m.calc_model == kKondoGC);
    std::vector<std::vector<uint32_t>> members((half + 1) * (half + 1));
    std::vector<uint32_t> l21(nh, 0), l22(nh, 0);
    std::vector<char> used(members.size(), 0);
    for (uint64_t ia = 0; ia < nh; ia++) {
      if (!admissible(ia, 0)) continue;
      const int key = gck ? 0 : __builtin_popcountll(ia & even) * (half + 1) + __builtin_popcountll(ia & ~even);
      members[key].push_back((uint32_t)ia);
    }
    std::vector<uint64_t> l1;
    uint64_t jb = 0;
    for (uint64_t ib = 0; ib < nh; ib++) {
      if (!admissible(ib, half)) continue;
      int key = 0;
      if (!gck) {
        const int nu = m.nup - __builtin_popcountll(ib & even), nd = m.ndown - __builtin_popcountll(ib & ~even);
        if (nu < 0 || nd < 0 || nu > half || nd > half) continue;
        key = nu * (half + 1) + nd;
      }
      const std::vector<uint32_t> &mem = members[key];
      if (mem.empty()) continue;
      used[key] = 1;
      l22[ib] = (uint32_t)(jb + 1);
      for (uint32_t ia : mem) l1.push_back((uint64_t)ia | (ib << N));
      jb += mem.size();
    }
    // list_2_1 holds a rank only for lower halves some block uses (the reference writes it
    // while filling the blocks)
    for (size_t key = 0; key < members.size(); key++)
      if (used[key])
        for (size_t r = 0; r < members[key].size(); r++) l21[members[key][r]] = (uint32_t)r + 2u;
    const int64_t expect = sector_dim(m);
    if ((int64_t)jb != expect || jb == 0) {
      *err = "Kondo sector size mismatch: enumerated " + std::to_string(jb) + ", expected " + std::to_string(expect);
      return -1;
    }
    if (jb > 0xFFFFFFF0ull) { *err = "sector too large for 32-bit list_2 tables"; return -1; }
    s->dim = (int64_t)jb;
    CK(cudaMalloc(&s->d_list_2_1, sizeof(uint32_t) * nh));
    CK(cudaMalloc(&s->d_list_2_2, sizeof(uint32_t) * nh));
    CK(cudaMalloc(&s->d_list_1, sizeof(uint64_t) * jb));
    CK(cudaMemcpy(s->d_list_2_1, l21.data(), sizeof(uint32_t) * nh, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->d_list_2_2, l22.data(), sizeof(uint32_t) * nh, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->d_list_1, l1.data(), sizeof(uint64_t) * jb, cudaMemcpyHostToDevice));
  } else {
    const int hubbard = (m.calc_model == kHubbard) ? 1 : 0;
    // Targets and class geometry.
    int ta, tb, Dlo, Dhi, Alo, Ahi;
    if (hubbard) {
      ta = m.nup; tb = m.ndown;
      Alo = (s->lo_bits + 1) / 2; Dlo = s->lo_bits / 2;  // lo half starts at an even position
      const int off_odd = s->lo_bits & 1;
      Ahi = off_odd ? s->hi_bits / 2 : (s->hi_bits + 1) / 2;
      Dhi = s->hi_bits - Ahi;
    } else {
      ta = m.ne; tb = 0;
      Alo = s->lo_bits; Dlo = 0; Ahi = s->hi_bits; Dhi = 0;
    }
    (void)Dhi; (void)Ahi;
    const int ncls = (Alo + 1) * (Dlo + 1);
    std::vector<uint64_t> cls_cnt(ncls), cls_off(ncls + 1, 0);
    for (int a = 0; a <= Alo; a++)
      for (int b = 0; b <= Dlo; b++) cls_cnt[a * (Dlo + 1) + b] = binom_host(Alo, a) * binom_host(Dlo, b);
    for (int c = 0; c < ncls; c++) cls_off[c + 1] = cls_off[c] + cls_cnt[c];
    // A lower-half class is used iff some upper half needs it.
    std::vector<unsigned char> valid(ncls, 0);
    for (int a = 0; a <= Ahi; a++)
      for (int b = 0; b <= Dhi; b++) {
        const int na = ta - a, nb = tb - b;
        if (na < 0 || nb < 0 || na > Alo || nb > Dlo) continue;
        if (!hubbard && b != 0) continue;
        valid[na * (Dlo + 1) + nb] = 1;
      }
    std::vector<uint64_t> binom(65 * 65, 0);
    for (int n = 0; n <= 64; n++)
      for (int k = 0; k <= n; k++) binom[n * 65 + k] = binom_host(n, k);
    CK(cudaMemcpyToSymbol(c_binom, binom.data(), sizeof(uint64_t) * 65 * 65));

    unsigned char *d_valid;
    uint64_t *d_cls_off, *d_cls_cnt, *d_cnt, *d_jb, *d_total;
    uint32_t *d_unrank;
    int *d_need;
    CK(cudaMalloc(&d_valid, ncls));
    CK(cudaMalloc(&d_cls_off, sizeof(uint64_t) * (ncls + 1)));
    CK(cudaMalloc(&d_cls_cnt, sizeof(uint64_t) * ncls));
    CK(cudaMalloc(&d_unrank, sizeof(uint32_t) * s->ihfbit));
    CK(cudaMalloc(&d_cnt, sizeof(uint64_t) * s->sdim));
    CK(cudaMalloc(&d_jb, sizeof(uint64_t) * s->sdim));
    CK(cudaMalloc(&d_total, sizeof(uint64_t)));
    CK(cudaMalloc(&d_need, sizeof(int) * s->sdim));
    CK(cudaMalloc(&s->d_list_2_1, sizeof(uint32_t) * s->ihfbit));
    CK(cudaMalloc(&s->d_list_2_2, sizeof(uint32_t) * s->sdim));
    CK(cudaMemcpyAsync(d_valid, valid.data(), ncls, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(d_cls_off, cls_off.data(), sizeof(uint64_t) * (ncls + 1), cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(d_cls_cnt, cls_cnt.data(), sizeof(uint64_t) * ncls, cudaMemcpyHostToDevice, s->stream));
    const int T = 256;
    lo_tables_kernel<<<(unsigned)((s->ihfbit + T - 1) / T), T, 0, s->stream>>>(
        s->ihfbit, s->lo_bits, hubbard, Dlo, d_valid, d_cls_off, s->d_list_2_1, d_unrank);
    hi_count_kernel<<<(unsigned)((s->sdim + T - 1) / T), T, 0, s->stream>>>(
        s->sdim, s->lo_bits, hubbard, Dlo, ta, tb, d_cls_cnt, Alo, Dlo, d_cnt, d_need);
    scan_kernel<<<1, 1024, 0, s->stream>>>(s->sdim, d_cnt, d_jb, d_total);
    list_2_2_kernel<<<(unsigned)((s->sdim + T - 1) / T), T, 0, s->stream>>>(s->sdim, d_cnt, d_jb, s->d_list_2_2);
    CK(cudaGetLastError());
    uint64_t total = 0;
    CK(cudaMemcpyAsync(&total, d_total, sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->dim = (int64_t)total;
    // idim_max from check() (src/check.c:102-150).
    uint64_t expect;
    if (m.calc_model == kHubbard) expect = binom_host(m.nsite, m.nup) * binom_host(m.nsite, m.ndown);
    else if (m.calc_model == kHubbardNConserved) expect = binom_host(2 * m.nsite, m.ne);
    else expect = binom_host(m.nsite, m.ne);
    if (total != expect || total == 0) {
      *err = "sector size mismatch: enumerated " + std::to_string(total) + ", expected " + std::to_string(expect);
      return -1;
    }
    if (total > 0xFFFFFFF0ull) { *err = "sector too large for 32-bit list_2 tables"; return -1; }
    CK(cudaMalloc(&s->d_list_1, sizeof(uint64_t) * total));
    const unsigned nb = (unsigned)std::min<uint64_t>(s->sdim, (uint64_t)nsm * 64);
    list_1_kernel<<<nb, 256, 0, s->stream>>>(s->sdim, s->lo_bits, d_cnt, d_jb, d_need, d_cls_off, d_unrank,
                                             s->d_list_1);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    cudaFree(d_valid); cudaFree(d_cls_off); cudaFree(d_cls_cnt); cudaFree(d_unrank);
    cudaFree(d_cnt); cudaFree(d_jb); cudaFree(d_total); cudaFree(d_need);
  }

  // Terms.
  s->nterms = (int)m.offdiag.size();
  s->ndterms = (int)m.diag.size();
  if (s->nterms) {
    CK(cudaMalloc(&s->d_terms, sizeof(BitTerm) * s->nterms));
    CK(cudaMemcpyAsync(s->d_terms, m.offdiag.data(), sizeof(BitTerm) * s->nterms, cudaMemcpyHostToDevice, s->stream));
  }
  if (s->ndterms) {
    CK(cudaMalloc(&s->d_dterms, sizeof(DiagTerm) * s->ndterms));
    CK(cudaMemcpyAsync(s->d_dterms, m.diag.data(), sizeof(DiagTerm) * s->ndterms, cudaMemcpyHostToDevice, s->stream));
  }
  if (split_plan_build(s, err) != 0) return -1;
  CK(cudaMalloc(&s->d_diag, sizeof(double) * (size_t)s->dim));
  diag_kernel<<<nsm * 8, 256, 0, s->stream>>>(s->dim, s->gc ? 1 : 0, s->d_list_1, s->d_dterms, s->ndterms, s->d_diag);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s->stream));
  // Specialised kernels (HPHI_B200_KERNEL=general keeps the general kernel).
  const char *kern = getenv("HPHI_B200_KERNEL");
  // HPHI_B200_KERNEL=general keeps the general kernel, =block the block plan; by default the
  // product-layout plan is used where it applies, else the block plan.
  const std::string kname = kern ? kern : "";
  if (specialise && kname != "general" && kname != "block") {
    if (prod_plan_build(s, err) != 0) return -1;
  }
  if (specialise && kname != "general" && !s->prod) {
    if (hub_plan_build(s, err) != 0) return -1;
  }
  // Row-block plan (spin sectors): from 2^24 rows up, where the vectors no longer stay in L2
  // and the general kernel's scattered gathers go to memory (below that the general kernel is
  // faster); HPHI_B200_KERNEL=rowblock builds it at any size.
  if (specialise && kname != "general" && !s->prod && !s->hub && (kname == "rowblock" || s->dim >= (1ll << 24))) {
    if (rb_plan_build(s, err) != 0) return -1;
  }
  *out = s;
  return 0;
}

void sector_free(Sector *s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  cudaFree(s->d_list_1); cudaFree(s->d_list_2_1); cudaFree(s->d_list_2_2); cudaFree(s->d_diag);
  cudaFree(s->d_terms); cudaFree(s->d_dterms); cudaFree(s->d_red); cudaFree(s->d_scal);
  cudaFree(s->split.lo_ptr); cudaFree(s->split.lo_ent); cudaFree(s->split.hi_ptr); cudaFree(s->split.hi_ent);
  cudaFree(s->split.coef); cudaFree(s->split.gen);
  hub_plan_free(s->hub);
  prod_plan_free(s->prod);
  rb_plan_free(s->rb);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

}  // namespace hphi
