// Block kernel for canonical Hubbard Hamiltonians: H*v with every operand access
// coalesced or conflict-free.
//
// Applies when every off-diagonal term is a spin-conserving single hop c+_{i s} c_{j s}
// (the Trans terms of a Hubbard model, src/mltplyHubbard.c:174-209 with the element
// routine CisAjt, src/mltplyHubbardCore.c:305-347) and Nsite is even; diagonal terms
// of any kind are allowed (src/diagonalcalc.c).  Other inputs use the general kernel.
//
// Layout ("native" order).  HPhi orders the sector by upper half ib and, inside a
// block, by increasing lower half ia (src/sz.c:993-1094).  The native order keeps
// HPhi's block offsets (list_2_2) but stores each block as a dense matrix
//   pos = rank(ua) * C(L, pop(da)) + rank(da),
// ua / da = the up / down occupations of the lower half (L = Nsite/2 sites).  The
// kernel then applies, per output block ib (one CTA at a time, block staged in SMEM):
//   lower-half up hops    rows of the staged block, warp-uniform CSR rows (conflict-free)
//   lower-half down hops  columns within a row of the staged block (small CSR per column)
//   upper-half hops       the same position in block ib ^ flip (coalesced global stream)
//   cross hops (up)       one row of block ib ^ bit, row rank(ua ^ bit)   (coalesced)
//   cross hops (down)     one row of block ib ^ bit, columns rank(da ^ bit)
// Fermion signs are (-1)^popcount(c & sign_mask) on the full configuration c, exactly
// as in the general kernel (SgnBit, src/bitcalc.c:338-352).  HPhi order is restored by
// the permutation kernels at the boundary (hv_to_native / hv_from_native).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "device_util.cuh"
#include "engine.hpp"
#include "hv_hubbard.hpp"

namespace hphi {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlockTerms = 128;   // per-block hi / cross term lists

struct HubTermDev {       // upper-half or cross hop (pull form on the full configuration)
  uint64_t cm, cv, flip, sm;
  double re, im;
  int lo_bit;             // cross: bit index inside ua / da (-1 for upper-half hops)
  int lo_need;            // cross: required value of that bit in the output configuration
  int spin;               // 0 up, 1 down
  int pad;
};

struct HubArgs {
  int nsite, L, N;                 // N = Nsite = bits per half
  int nup, ndn;
  uint64_t sdim;
  const uint32_t *list_2_2;        // block offsets + 1 (HPhi's list_2_2), 0 = empty block
  const uint16_t *rank;            // [2^L] rank of x among L-bit numbers of its popcount
  const uint16_t *unrank;          // [2^L] grouped by popcount, offsets unrank_off
  const int *unrank_off;           // [L+2]
  const int *binom;                // [L+1] C(L, k)
  const uint32_t *spread;          // [2^L] bits of x moved to even positions
  const int *csr_up_ptr;           // [2^L + 1] rows ordered (k, r) like unrank
  const uint32_t *csr_up;          // entries: r' | term << 16
  const int *csr_dn_ptr;
  const uint32_t *csr_dn;
  const double *lo_coef;           // [n_lo_terms][2]
  const uint64_t *lo_sm;           // [n_lo_terms]
  const HubTermDev *hi_terms;      // upper-half hops
  int n_hi;
  const HubTermDev *cross_terms;   // cross hops
  int n_cross;
  const double *d_lo;              // diagonal, lower-half terms, per class pair in native order
  const int *d_lo_off;             // [(L+1)*(L+1)] offset of class pair (ku, kd)
  const double *d_hi;              // [2^N] diagonal, upper-half terms
  const DiagTerm *d_cross;         // diagonal terms spanning both halves
  int n_dcross;
};

struct BlockTerm {  // a term resolved for the current output block
  uint64_t sm;
  double re, im;
  int64_t src;      // first element of the source block
  int lo_bit, lo_need, spin, nsrc;  // nsrc: C(L, k') of the changed species in the source block
};

template <typename T>
__device__ __forceinline__ T coef_mul(double re, double im, T x);
template <>
__device__ __forceinline__ double coef_mul<double>(double re, double, double x) { return re * x; }
template <>
__device__ __forceinline__ cplx coef_mul<cplx>(double re, double im, cplx x) {
  return cplx{re * x.x - im * x.y, re * x.y + im * x.x};
}

template <typename T>
__global__ void __launch_bounds__(kThreads) hv_hub_kernel(HubArgs a, const T *__restrict__ v1, T *__restrict__ v0,
                                                          const double *__restrict__ coef, double *__restrict__ part) {
  extern __shared__ unsigned char smem_raw[];
  T *xs = reinterpret_cast<T *>(smem_raw);
  __shared__ BlockTerm hi_list[kMaxBlockTerms];
  __shared__ BlockTerm cr_list[kMaxBlockTerms];
  __shared__ int n_hi_blk, n_cr_blk;
  const double acc = coef[0], scale = coef[1];
  const int N = a.N, L = a.L;
  const uint64_t even_mask = 0x5555555555555555ull & ((N >= 64) ? ~0ull : ((1ull << N) - 1));
  double pr[2] = {0.0, 0.0};

  for (uint64_t ib = blockIdx.x; ib < a.sdim; ib += gridDim.x) {
    const uint32_t l22 = a.list_2_2[ib];
    if (l22 == 0u) continue;
    const int64_t jb = (int64_t)l22 - 1;
    const int pu = __popcll(ib & even_mask), pd = __popcll(ib & (even_mask << 1));
    const int nu = a.nup - pu, nd = a.ndn - pd;
    const int nua = a.binom[nu], nda = a.binom[nd];
    const int n = nua * nda;
    const uint64_t chi = ib << N;
    // stage the source block
    for (int p = threadIdx.x; p < n; p += blockDim.x) xs[p] = v1[jb + p];
    // resolve the block's upper-half and cross terms
    if (threadIdx.x < 32) {
      int nh = 0, nc = 0;
      for (int base = 0; base < a.n_hi + a.n_cross; base += 32) {
        const int t = base + (int)threadIdx.x;
        bool take = false;
        const HubTermDev *tt = nullptr;
        if (t < a.n_hi + a.n_cross) {
          tt = (t < a.n_hi) ? &a.hi_terms[t] : &a.cross_terms[t - a.n_hi];
          const uint64_t cm_hi = tt->cm & ~((N >= 64) ? ~0ull : ((1ull << N) - 1));
          const uint64_t cv_hi = tt->cv & cm_hi;
          take = (chi & cm_hi) == cv_hi;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, take && t < a.n_hi);
        const unsigned maskc = __ballot_sync(0xffffffffu, take && t >= a.n_hi);
        if (take) {
          const uint64_t src_ib = ib ^ (tt->flip >> N);
          const uint32_t sl = a.list_2_2[src_ib];
          BlockTerm bt;
          bt.sm = tt->sm; bt.re = tt->re; bt.im = tt->im;
          bt.src = (sl == 0u) ? -1 : (int64_t)sl - 1;
          bt.lo_bit = tt->lo_bit; bt.lo_need = tt->lo_need; bt.spin = tt->spin;
          if (t < a.n_hi) {
            bt.nsrc = 0;
            const int slot = nh + __popc(mask & ((1u << threadIdx.x) - 1));
            if (slot < kMaxBlockTerms) hi_list[slot] = bt;
          } else {
            // source class of the changed species: one particle more or fewer in the lower half
            const int k_src = (tt->spin == 0 ? nu : nd) + (tt->lo_need ? -1 : 1);
            bt.nsrc = (k_src >= 0 && k_src <= L) ? a.binom[k_src] : 0;
            const int slot = nc + __popc(maskc & ((1u << threadIdx.x) - 1));
            if (slot < kMaxBlockTerms) cr_list[slot] = bt;
          }
        }
        nh += __popc(mask);
        nc += __popc(maskc);
      }
      if (threadIdx.x == 0) {
        n_hi_blk = min(nh, kMaxBlockTerms);
        n_cr_blk = min(nc, kMaxBlockTerms);
      }
    }
    __syncthreads();
    const int nhb = n_hi_blk, ncb = n_cr_blk;
    const int off_u = a.unrank_off[nu], off_d = a.unrank_off[nd];
    const uint32_t magic = (uint32_t)(0xFFFFFFFFull / (uint32_t)nda + 1ull);
    const double dhi = a.d_hi[ib];
    const double *dlo = a.d_lo + a.d_lo_off[nu * (L + 1) + nd];
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
      const int ra = (nda == 1) ? p : (int)__umulhi((uint32_t)p, magic);
      const int rd = p - ra * nda;
      const uint32_t ua = a.unrank[off_u + ra], da = a.unrank[off_d + rd];
      const uint64_t c = chi | (uint64_t)a.spread[ua] | ((uint64_t)a.spread[da] << 1);
      const T x = xs[p];
      double dg = dlo[p] + dhi;
      for (int k = 0; k < a.n_dcross; k++) {
        const DiagTerm dt = a.d_cross[k];
        if ((c & dt.cm) == dt.cv) dg += dt.v;
      }
      T y = VT<T>::scale(dg, x);
      // lower-half up hops: rows of the staged block
      {
        const int r0 = a.csr_up_ptr[off_u + ra], r1 = a.csr_up_ptr[off_u + ra + 1];
        for (int e = r0; e < r1; e++) {
          const uint32_t ent = a.csr_up[e];
          const int rs = (int)(ent & 0xFFFFu), t = (int)(ent >> 16);
          const double s = (__popcll(c & a.lo_sm[t]) & 1) ? -1.0 : 1.0;
          y = VT<T>::add(y, coef_mul<T>(s * a.lo_coef[2 * t], s * a.lo_coef[2 * t + 1], xs[rs * nda + rd]));
        }
      }
      // lower-half down hops: columns within the row
      {
        const int r0 = a.csr_dn_ptr[off_d + rd], r1 = a.csr_dn_ptr[off_d + rd + 1];
        const T *row = xs + ra * nda;
        for (int e = r0; e < r1; e++) {
          const uint32_t ent = a.csr_dn[e];
          const int rs = (int)(ent & 0xFFFFu), t = (int)(ent >> 16);
          const double s = (__popcll(c & a.lo_sm[t]) & 1) ? -1.0 : 1.0;
          y = VT<T>::add(y, coef_mul<T>(s * a.lo_coef[2 * t], s * a.lo_coef[2 * t + 1], row[rs]));
        }
      }
      // upper-half hops: same position in another block of the same class
      for (int k = 0; k < nhb; k++) {
        const BlockTerm &bt = hi_list[k];
        if (bt.src < 0) continue;
        const double s = (__popcll(c & bt.sm) & 1) ? -1.0 : 1.0;
        y = VT<T>::add(y, coef_mul<T>(s * bt.re, s * bt.im, v1[bt.src + p]));
      }
      // cross hops: one particle moves between the halves
      for (int k = 0; k < ncb; k++) {
        const BlockTerm &bt = cr_list[k];
        const uint32_t own = bt.spin == 0 ? ua : da;
        if ((int)((own >> bt.lo_bit) & 1u) != bt.lo_need || bt.src < 0) continue;
        const int r_new = a.rank[own ^ (1u << bt.lo_bit)];
        const int64_t j = (bt.spin == 0) ? bt.src + (int64_t)r_new * nda + rd
                                         : bt.src + (int64_t)ra * bt.nsrc + r_new;
        const double s = (__popcll(c & bt.sm) & 1) ? -1.0 : 1.0;
        y = VT<T>::add(y, coef_mul<T>(s * bt.re, s * bt.im, v1[j]));
      }
      pr[0] += VT<T>::conj_mul_re(x, y);
      pr[1] += VT<T>::conj_mul_im(x, y);
      y = VT<T>::scale(scale, y);
      v0[jb + p] = (acc == 0.0) ? y : VT<T>::add(VT<T>::scale(acc, v0[jb + p]), y);
    }
    __syncthreads();
  }
  block_sum<2>(pr);
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = pr[0]; part[2 * blockIdx.x + 1] = pr[1]; }
}

// ---- HPhi order <-> native order (per row r of HPhi's list_1)
template <typename T, bool TO_NATIVE>
__global__ void permute_kernel(int64_t dim, int N, int L, const uint64_t *__restrict__ list_1,
                               const uint32_t *__restrict__ list_2_2, const uint16_t *__restrict__ rank,
                               const int *__restrict__ binom, const T *__restrict__ in, T *__restrict__ out) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = list_1[r];
    const uint64_t ib = c >> N;
    const uint64_t ia = c & ((1ull << N) - 1);
    uint32_t ua = 0, da = 0;
    for (int s = 0; s < L; s++) {
      ua |= (uint32_t)((ia >> (2 * s)) & 1ull) << s;
      da |= (uint32_t)((ia >> (2 * s + 1)) & 1ull) << s;
    }
    const int64_t jb = (int64_t)list_2_2[ib] - 1;
    const int64_t pos = jb + (int64_t)rank[ua] * binom[__popc(da)] + rank[da];
    if (TO_NATIVE) out[pos] = in[r];
    else out[r] = in[pos];
  }
}

// Diagonal observables in native order (expec_energy_flct_Hubbard, src/expec_energy_flct.c).
template <typename T>
__global__ void native_obs_kernel(HubArgs a, const T *__restrict__ v, double *__restrict__ part) {
  double o[6] = {0, 0, 0, 0, 0, 0};
  const int N = a.N, L = a.L;
  const uint64_t even_mask = 0x5555555555555555ull & ((1ull << N) - 1);
  for (uint64_t ib = blockIdx.x; ib < a.sdim; ib += gridDim.x) {
    const uint32_t l22 = a.list_2_2[ib];
    if (l22 == 0u) continue;
    const int64_t jb = (int64_t)l22 - 1;
    const int nu = a.nup - __popcll(ib & even_mask), nd = a.ndn - __popcll(ib & (even_mask << 1));
    const int nda = a.binom[nd], n = a.binom[nu] * nda;
    const int off_u = a.unrank_off[nu], off_d = a.unrank_off[nd];
    (void)L;
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
      const int ra = p / nda, rd = p - ra * nda;
      const uint64_t c = (ib << N) | (uint64_t)a.spread[a.unrank[off_u + ra]] |
                         ((uint64_t)a.spread[a.unrank[off_d + rd]] << 1);
      const double w = VT<T>::abs2(v[jb + p]);
      const uint64_t ev = 0x5555555555555555ull;
      const int up = __popcll(c & ev), dn = __popcll(c & ~ev);
      const double D = (double)__popcll(c & (c >> 1) & ev), Nn = (double)(up + dn), Sz = 0.5 * (double)(up - dn);
      o[0] += w * D; o[1] += w * D * D; o[2] += w * Nn; o[3] += w * Nn * Nn; o[4] += w * Sz; o[5] += w * Sz * Sz;
    }
  }
  block_sum<6>(o);
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; k++) part[6 * blockIdx.x + k] = o[k];
}

uint64_t binom_u(int n, int k) {
  if (k < 0 || k > n) return 0;
  uint64_t r = 1;
  for (int i = 1; i <= k; i++) r = r * (uint64_t)(n - k + i) / (uint64_t)i;
  return r;
}

template <typename V>
int upload(const std::vector<V> &h, V **d, std::string *err) {
  if (h.empty()) { *d = nullptr; return 0; }
  if (cudaMalloc(d, sizeof(V) * h.size()) != cudaSuccess ||
      cudaMemcpy(*d, h.data(), sizeof(V) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    *err = "hubbard plan: device allocation failed";
    return -1;
  }
  return 0;
}

}  // namespace

struct HubPlan {
  HubArgs args;
  std::vector<void *> allocs;
  size_t smem_real = 0, smem_cplx = 0;
  int grid = 0;
  int n_lo_terms = 0;
};

void hub_plan_free(HubPlan *p) {
  if (!p) return;
  for (void *q : p->allocs) cudaFree(q);
  delete p;
}

int hub_plan_build(Sector *s, std::string *err) {
  const Model &m = s->model;
  s->hub = nullptr;
  if (m.calc_model != kHubbard || m.nsite % 2 != 0 || m.nsite > 30 || s->gc) return 0;
  const int N = m.nsite, L = N / 2;
  const uint64_t lo_mask = (1ull << N) - 1;
  // classify off-diagonal terms; any term that is not a spin-conserving single hop
  // keeps the general kernel
  struct Hop { uint64_t cm, cv, flip, sm; double re, im; int p, q; };
  std::vector<Hop> lo_up, lo_dn, hi, cross;
  for (const BitTerm &t : m.offdiag) {
    if (__builtin_popcountll(t.flip) != 2 || t.cm != t.flip) return 0;
    const int p = __builtin_ctzll(t.flip), q = 63 - __builtin_clzll(t.flip);
    if ((p & 1) != (q & 1)) return 0;
    if (t.cv != (1ull << p) && t.cv != (1ull << q)) return 0;
    Hop h{t.cm, t.cv, t.flip, t.sm, t.re, t.im, p, q};
    if (q < N) ((p & 1) ? lo_dn : lo_up).push_back(h);
    else if (p >= N) hi.push_back(h);
    else cross.push_back(h);
  }
  if ((int)(hi.size()) > kMaxBlockTerms || (int)cross.size() > kMaxBlockTerms) return 0;
  const int nx = 1 << L;
  // rank / unrank / spread tables for L-bit half-species configurations
  std::vector<uint16_t> rank(nx), unrank(nx);
  std::vector<int> unrank_off(L + 2, 0), binom(L + 1);
  for (int k = 0; k <= L; k++) binom[k] = (int)binom_u(L, k);
  for (int k = 0; k <= L; k++) unrank_off[k + 1] = unrank_off[k] + binom[k];
  {
    std::vector<int> fill(L + 1, 0);
    for (int x = 0; x < nx; x++) {
      const int k = __builtin_popcount(x);
      rank[x] = (uint16_t)fill[k];
      unrank[unrank_off[k] + fill[k]] = (uint16_t)x;
      fill[k]++;
    }
  }
  std::vector<uint32_t> spread(nx);
  for (int x = 0; x < nx; x++) {
    uint32_t v = 0;
    for (int b = 0; b < L; b++)
      if (x >> b & 1) v |= 1u << (2 * b);
    spread[x] = v;
  }
  if ((uint64_t)binom[L / 2] * (uint64_t)binom[L / 2] >= 65536ull) return 0;  // 16-bit positions
  // lower-half CSR: for species spin (0 up / 1 down), row = (class k, rank r) of that species;
  // entries reference the lower-half hop table lo_coef / lo_sm (ups first, then downs)
  std::vector<double> lo_coef;
  std::vector<uint64_t> lo_sm;
  for (const auto *hops : {&lo_up, &lo_dn})
    for (const Hop &h : *hops) {
      lo_coef.push_back(h.re);
      lo_coef.push_back(h.im);
      lo_sm.push_back(h.sm);
    }
  auto build_csr = [&](const std::vector<Hop> &hops, int spin, int id0, std::vector<int> *ptr,
                       std::vector<uint32_t> *ent) {
    ptr->assign(nx + 1, 0);
    ent->clear();
    for (int k = 0; k <= L; k++)
      for (int r = 0; r < binom[k]; r++) {
        const int row = unrank_off[k] + r;
        const uint32_t x = unrank[row];
        const uint64_t cfg = (uint64_t)spread[x] << spin;  // this species' bits in the lower half
        for (size_t hi_ = 0; hi_ < hops.size(); hi_++) {
          const Hop &h = hops[hi_];
          if ((cfg & h.cm) != h.cv) continue;
          const uint64_t src = cfg ^ h.flip;
          uint32_t xs = 0;
          for (int b = 0; b < L; b++) xs |= (uint32_t)((src >> (2 * b + spin)) & 1ull) << b;
          ent->push_back((uint32_t)rank[xs] | ((uint32_t)(id0 + hi_) << 16));
        }
        (*ptr)[row + 1] = (int)ent->size();
      }
  };
  std::vector<int> up_ptr, dn_ptr;
  std::vector<uint32_t> up_ent, dn_ent;
  build_csr(lo_up, 0, 0, &up_ptr, &up_ent);
  build_csr(lo_dn, 1, (int)lo_up.size(), &dn_ptr, &dn_ent);
  if (lo_coef.size() / 2 >= 65536) return 0;
  auto to_dev = [&](const std::vector<Hop> &hops, bool is_cross) {
    std::vector<HubTermDev> out;
    for (const Hop &h : hops) {
      HubTermDev d{};
      d.cm = h.cm; d.cv = h.cv; d.flip = h.flip; d.sm = h.sm; d.re = h.re; d.im = h.im;
      d.spin = h.p & 1;
      d.lo_bit = -1; d.lo_need = 0;
      if (is_cross) {
        d.lo_bit = h.p >> 1;  // p is the lower-half end (p < N <= q)
        d.lo_need = (int)((h.cv >> h.p) & 1ull);
      }
      out.push_back(d);
    }
    return out;
  };
  std::vector<HubTermDev> hi_dev = to_dev(hi, false), cross_dev = to_dev(cross, true);
  // diagonal split
  std::vector<DiagTerm> dlo_t, dhi_t, dcross;
  for (const DiagTerm &t : m.diag) {
    if ((t.cm & ~lo_mask) == 0) dlo_t.push_back(t);
    else if ((t.cm & lo_mask) == 0) dhi_t.push_back(t);
    else dcross.push_back(t);
  }
  if (dcross.size() > 4096) return 0;
  std::vector<double> dhi(1ull << N, 0.0);
  for (uint64_t ib = 0; ib < (1ull << N); ib++) {
    const uint64_t c = ib << N;
    double v = 0.0;
    for (const DiagTerm &t : dhi_t)
      if ((c & t.cm) == t.cv) v += t.v;
    dhi[ib] = v;
  }
  std::vector<int> dlo_off((L + 1) * (L + 1), 0);
  std::vector<double> dlo;
  for (int ku = 0; ku <= L; ku++)
    for (int kd = 0; kd <= L; kd++) {
      dlo_off[ku * (L + 1) + kd] = (int)dlo.size();
      for (int ra = 0; ra < binom[ku]; ra++)
        for (int rd = 0; rd < binom[kd]; rd++) {
          const uint64_t c = (uint64_t)spread[unrank[unrank_off[ku] + ra]] |
                             ((uint64_t)spread[unrank[unrank_off[kd] + rd]] << 1);
          double v = 0.0;
          for (const DiagTerm &t : dlo_t)
            if ((c & t.cm) == t.cv) v += t.v;
          dlo.push_back(v);
        }
    }

  HubPlan *plan = new HubPlan();
  HubArgs &a = plan->args;
  a.nsite = N; a.L = L; a.N = N; a.nup = m.nup; a.ndn = m.ndown; a.sdim = s->sdim;
  a.list_2_2 = s->d_list_2_2;
  auto up = [&](auto &vec, auto **dst) -> int {
    if (upload(vec, dst, err)) return -1;
    plan->allocs.push_back((void *)*dst);
    return 0;
  };
  uint16_t *d_rank, *d_unrank;
  int *d_uoff, *d_binom, *d_up_ptr, *d_dn_ptr, *d_dlo_off;
  uint32_t *d_spread, *d_up_ent, *d_dn_ent;
  double *d_lo_coef, *d_dlo, *d_dhi;
  uint64_t *d_lo_sm;
  HubTermDev *d_hi, *d_cross;
  DiagTerm *d_dcross;
  if (up(rank, &d_rank) || up(unrank, &d_unrank) || up(unrank_off, &d_uoff) || up(binom, &d_binom) ||
      up(spread, &d_spread) || up(up_ptr, &d_up_ptr) || up(up_ent, &d_up_ent) || up(dn_ptr, &d_dn_ptr) ||
      up(dn_ent, &d_dn_ent) || up(lo_coef, &d_lo_coef) || up(lo_sm, &d_lo_sm) || up(hi_dev, &d_hi) ||
      up(cross_dev, &d_cross) || up(dlo, &d_dlo) || up(dlo_off, &d_dlo_off) || up(dhi, &d_dhi) ||
      up(dcross, &d_dcross)) {
    hub_plan_free(plan);
    return -1;
  }
  a.rank = d_rank; a.unrank = d_unrank; a.unrank_off = d_uoff; a.binom = d_binom; a.spread = d_spread;
  a.csr_up_ptr = d_up_ptr; a.csr_up = d_up_ent; a.csr_dn_ptr = d_dn_ptr; a.csr_dn = d_dn_ent;
  a.lo_coef = d_lo_coef; a.lo_sm = d_lo_sm;
  a.hi_terms = d_hi; a.n_hi = (int)hi_dev.size();
  a.cross_terms = d_cross; a.n_cross = (int)cross_dev.size();
  a.d_lo = d_dlo; a.d_lo_off = d_dlo_off; a.d_hi = d_dhi; a.d_cross = d_dcross; a.n_dcross = (int)dcross.size();
  plan->n_lo_terms = (int)lo_coef.size() / 2;
  int maxn = 0;
  for (int ku = 0; ku <= L; ku++)
    for (int kd = 0; kd <= L; kd++) maxn = std::max(maxn, binom[ku] * binom[kd]);
  plan->smem_real = sizeof(double) * (size_t)maxn;
  plan->smem_cplx = sizeof(cplx) * (size_t)maxn;
  cudaFuncSetAttribute((const void *)hv_hub_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)plan->smem_real);
  cudaFuncSetAttribute((const void *)hv_hub_kernel<cplx>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)plan->smem_cplx);
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hv_hub_kernel<double>, kThreads, plan->smem_real);
  plan->grid = std::max(1, per_sm) * s->num_sms;
  if (plan->grid > s->red_blocks) plan->grid = s->red_blocks;
  if (cudaGetLastError() != cudaSuccess) {
    *err = "hubbard plan: kernel configuration failed";
    hub_plan_free(plan);
    return -1;
  }
  s->hub = plan;
  return 0;
}

int hub_hv_launch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                  bool acc_read) {
  HubPlan *p = s->hub;
  (void)acc_read;
  if (vt == kReal64 && s->model.complex_terms) {
    set_error("H has complex coefficients: real vectors are not allowed");
    return -1;
  }
  if (vt == kReal64)
    hv_hub_kernel<double><<<p->grid, kThreads, p->smem_real, s->stream>>>(p->args, (const double *)d_v1,
                                                                          (double *)d_v0, d_coef, s->d_red);
  else
    hv_hub_kernel<cplx><<<p->grid, kThreads, p->smem_cplx, s->stream>>>(p->args, (const cplx *)d_v1, (cplx *)d_v0,
                                                                        d_coef, s->d_red);
  finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(s->d_red, p->grid, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("hubbard hv launch failed: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

int hub_permute(Sector *s, VecType vt, const void *in, void *out, bool to_native) {
  HubPlan *p = s->hub;
  const HubArgs &a = p->args;
  const int grid = s->red_blocks;
  if (vt == kReal64) {
    if (to_native)
      permute_kernel<double, true><<<grid, kThreads, 0, s->stream>>>(s->dim, a.N, a.L, s->d_list_1, a.list_2_2, a.rank,
                                                                     a.binom, (const double *)in, (double *)out);
    else
      permute_kernel<double, false><<<grid, kThreads, 0, s->stream>>>(s->dim, a.N, a.L, s->d_list_1, a.list_2_2,
                                                                      a.rank, a.binom, (const double *)in, (double *)out);
  } else {
    if (to_native)
      permute_kernel<cplx, true><<<grid, kThreads, 0, s->stream>>>(s->dim, a.N, a.L, s->d_list_1, a.list_2_2, a.rank,
                                                                   a.binom, (const cplx *)in, (cplx *)out);
    else
      permute_kernel<cplx, false><<<grid, kThreads, 0, s->stream>>>(s->dim, a.N, a.L, s->d_list_1, a.list_2_2, a.rank,
                                                                    a.binom, (const cplx *)in, (cplx *)out);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("permute failed: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

int hub_observables(Sector *s, VecType vt, const void *v, double *d_out) {
  HubPlan *p = s->hub;
  if (vt == kReal64) native_obs_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(p->args, (const double *)v, s->d_red);
  else native_obs_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(p->args, (const cplx *)v, s->d_red);
  finalize_partials_kernel<6><<<1, 256, 0, s->stream>>>(s->d_red, s->red_blocks, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("observables failed: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

}  // namespace hphi
