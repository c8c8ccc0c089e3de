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
  uint32_t cm_hi, cv_hi;  // condition on the upper half (bits of c >> N)
  uint32_t flip_hi;       // flip of the upper half
  uint32_t sm;            // sign mask on the full configuration
  double re, im;
  int lo_bit;             // cross hops: bit of ua / da that moves (-1 for upper-half hops)
  int lo_need;            // cross hops: value of that bit in the output configuration
};

struct HubArgs {
  int L, N;                        // N = Nsite = bits per half, L = N/2 sites per half
  int nup, ndn;
  int nblocks;                     // non-empty blocks
  const uint32_t *order[2];        // block processing order: [0] by (db, ub), [1] by (ub, db)
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
  int n_csr_up, n_csr_dn, n_lo;
  const double *lo_coef;           // [n_lo][2]
  const uint32_t *lo_sm;           // [n_lo]
  const HubTermDev *terms[2];      // [0] up-spin upper-half + cross hops, [1] down-spin
  int n_hi[2], n_cross[2];         // terms[s] = n_hi[s] upper-half hops, then n_cross[s] cross hops
  const double *d_lo;              // diagonal, lower-half terms, per class pair in native order
  const int *d_lo_off;             // [(L+1)*(L+1)] offset of class pair (ku, kd)
  const double *d_hi;              // [2^N] diagonal, upper-half terms
  const DiagTerm *d_cross;         // diagonal terms spanning both halves
  int n_dcross;
};

template <typename T>
__device__ __forceinline__ T coef_mul(double re, double im, T x);
template <>
__device__ __forceinline__ double coef_mul<double>(double re, double, double x) { return re * x; }
template <>
__device__ __forceinline__ cplx coef_mul<cplx>(double re, double im, cplx x) {
  return cplx{re * x.x - im * x.y, re * x.y + im * x.x};
}
__device__ __forceinline__ double sgn_of(uint32_t c, uint32_t sm) { return (__popc(c & sm) & 1) ? -1.0 : 1.0; }

// Per-block resolved terms (SoA in shared memory).
struct BlockTerms {
  int64_t src[kMaxBlockTerms];
  uint32_t sm[kMaxBlockTerms];
  double re[kMaxBlockTerms], im[kMaxBlockTerms];
  int bit[kMaxBlockTerms], need[kMaxBlockTerms], nsrc[kMaxBlockTerms];
  int n_hi, n_cr;
};

// Phase 0 (up spin) and phase 1 (down spin) of the native-order Hubbard H*v.
//   phase 0: v0 = acc*v0 + scale*(D + H_lo + H_up,hi + H_up,cross) v1   blocks in (db, ub) order
//   phase 1: v0 += scale*(H_dn,hi + H_dn,cross) v1                       blocks in (ub, db) order
// The up-spin hops of a block only reach blocks with the same down part db (and the
// down-spin hops only blocks with the same ub), so in each phase the source blocks of the
// CTAs in flight form a few L2-resident columns (rows) of the block grid.
template <typename T, int PHASE>
__global__ void __launch_bounds__(kThreads) hv_hub_phase(HubArgs a, const T *__restrict__ v1, T *__restrict__ v0,
                                                         const double *__restrict__ coef, double *__restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ BlockTerms bl;
  const int L = a.L, N = a.N, nx = 1 << L;
  // shared tables: rank, unrank, spread (+ lower-half CSR in phase 0), then the staged block
  unsigned char *sp = smem_raw;
  uint32_t *s_spread = reinterpret_cast<uint32_t *>(sp); sp += sizeof(uint32_t) * nx;
  uint16_t *s_rank = reinterpret_cast<uint16_t *>(sp); sp += sizeof(uint16_t) * nx;
  uint16_t *s_unrank = reinterpret_cast<uint16_t *>(sp); sp += sizeof(uint16_t) * nx;
  int *s_uoff = reinterpret_cast<int *>(sp); sp += sizeof(int) * 32;
  int *s_binom = reinterpret_cast<int *>(sp); sp += sizeof(int) * 32;
  int *s_up_ptr = nullptr, *s_dn_ptr = nullptr;
  uint32_t *s_up = nullptr, *s_dn = nullptr, *s_losm = nullptr;
  double *s_locoef = nullptr;
  T *xs = nullptr;
  if (PHASE == 0) {
    s_up_ptr = reinterpret_cast<int *>(sp); sp += sizeof(int) * (nx + 1);
    s_dn_ptr = reinterpret_cast<int *>(sp); sp += sizeof(int) * (nx + 1);
    s_up = reinterpret_cast<uint32_t *>(sp); sp += sizeof(uint32_t) * a.n_csr_up;
    s_dn = reinterpret_cast<uint32_t *>(sp); sp += sizeof(uint32_t) * a.n_csr_dn;
    s_losm = reinterpret_cast<uint32_t *>(sp); sp += sizeof(uint32_t) * a.n_lo;
    sp = smem_raw + (((sp - smem_raw) + 15) & ~(size_t)15);
    s_locoef = reinterpret_cast<double *>(sp); sp += sizeof(double) * 2 * a.n_lo;
    xs = reinterpret_cast<T *>(sp);
  }
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    s_spread[i] = a.spread[i]; s_rank[i] = a.rank[i]; s_unrank[i] = a.unrank[i];
  }
  for (int i = threadIdx.x; i <= L + 1 && i < 32; i += blockDim.x) {
    s_uoff[i] = a.unrank_off[i];
    if (i <= L) s_binom[i] = a.binom[i];
  }
  if (PHASE == 0) {
    for (int i = threadIdx.x; i <= nx; i += blockDim.x) { s_up_ptr[i] = a.csr_up_ptr[i]; s_dn_ptr[i] = a.csr_dn_ptr[i]; }
    for (int i = threadIdx.x; i < a.n_csr_up; i += blockDim.x) s_up[i] = a.csr_up[i];
    for (int i = threadIdx.x; i < a.n_csr_dn; i += blockDim.x) s_dn[i] = a.csr_dn[i];
    for (int i = threadIdx.x; i < a.n_lo; i += blockDim.x) {
      s_losm[i] = a.lo_sm[i]; s_locoef[2 * i] = a.lo_coef[2 * i]; s_locoef[2 * i + 1] = a.lo_coef[2 * i + 1];
    }
  }
  __syncthreads();
  const double acc = coef[0], scale = coef[1];
  const uint32_t even_mask = 0x55555555u & ((N >= 32) ? 0xFFFFFFFFu : ((1u << N) - 1u));
  const HubTermDev *terms = a.terms[PHASE];
  const int n_hi = a.n_hi[PHASE], n_all = a.n_hi[PHASE] + a.n_cross[PHASE];
  double pr[2] = {0.0, 0.0};

  for (int bi = blockIdx.x; bi < a.nblocks; bi += gridDim.x) {
    const uint32_t ib = a.order[PHASE][bi];
    const int64_t jb = (int64_t)a.list_2_2[ib] - 1;
    const int nu = a.nup - __popc(ib & even_mask), nd = a.ndn - __popc(ib & (even_mask << 1));
    const int nua = s_binom[nu], nda = s_binom[nd];
    const int n = nua * nda;
    const uint32_t chi = ib << N;
    if (PHASE == 0)
      for (int p = threadIdx.x; p < n; p += blockDim.x) xs[p] = v1[jb + p];
    if (threadIdx.x < 32) {
      int nh = 0, nc = 0;
      for (int base = 0; base < n_all; base += 32) {
        const int t = base + (int)threadIdx.x;
        bool take = false;
        HubTermDev tt;
        if (t < n_all) {
          tt = terms[t];
          take = (ib & tt.cm_hi) == tt.cv_hi;
        }
        const bool is_hi = t < n_hi;
        const unsigned mh = __ballot_sync(0xffffffffu, take && is_hi);
        const unsigned mc = __ballot_sync(0xffffffffu, take && !is_hi);
        if (take) {
          const uint32_t sl = a.list_2_2[ib ^ tt.flip_hi];
          const int slot = is_hi ? nh + __popc(mh & ((1u << threadIdx.x) - 1))
                                 : kMaxBlockTerms - 1 - (nc + __popc(mc & ((1u << threadIdx.x) - 1)));
          bl.src[slot] = (sl == 0u) ? -1 : (int64_t)sl - 1;
          bl.sm[slot] = tt.sm; bl.re[slot] = tt.re; bl.im[slot] = tt.im;
          bl.bit[slot] = tt.lo_bit; bl.need[slot] = tt.lo_need;
          const int k_src = (PHASE == 0 ? nu : nd) + (tt.lo_need ? -1 : 1);
          bl.nsrc[slot] = (!is_hi && k_src >= 0 && k_src <= L) ? s_binom[k_src] : 0;
        }
        nh += __popc(mh);
        nc += __popc(mc);
      }
      if (threadIdx.x == 0) { bl.n_hi = nh; bl.n_cr = nc; }
    }
    __syncthreads();
    const int nhb = bl.n_hi, ncb = bl.n_cr;
    const int off_u = s_uoff[nu], off_d = s_uoff[nd];
    const uint32_t magic = (uint32_t)(0xFFFFFFFFull / (uint32_t)nda + 1ull);
    const double dhi = (PHASE == 0) ? a.d_hi[ib] : 0.0;
    const double *dlo = a.d_lo + a.d_lo_off[nu * (L + 1) + nd];
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
      const int ra = (nda == 1) ? p : (int)__umulhi((uint32_t)p, magic);
      const int rd = p - ra * nda;
      const uint32_t ua = s_unrank[off_u + ra], da = s_unrank[off_d + rd];
      const uint32_t c = chi | s_spread[ua] | (s_spread[da] << 1);
      T x, y;
      if (PHASE == 0) {
        x = xs[p];
        double dg = dlo[p] + dhi;
        for (int k = 0; k < a.n_dcross; k++) {
          const DiagTerm dt = a.d_cross[k];
          if (((uint64_t)c & dt.cm) == dt.cv) dg += dt.v;
        }
        y = VT<T>::scale(dg, x);
        {  // lower-half up hops: rows of the staged block
          const int r0 = s_up_ptr[off_u + ra], r1 = s_up_ptr[off_u + ra + 1];
          for (int e = r0; e < r1; e++) {
            const uint32_t ent = s_up[e];
            const int t = (int)(ent >> 16);
            const double sg = sgn_of(c, s_losm[t]);
            y = VT<T>::add(y, coef_mul<T>(sg * s_locoef[2 * t], sg * s_locoef[2 * t + 1], xs[(int)(ent & 0xFFFFu) * nda + rd]));
          }
        }
        {  // lower-half down hops: columns within the row
          const int r0 = s_dn_ptr[off_d + rd], r1 = s_dn_ptr[off_d + rd + 1];
          const T *row = xs + ra * nda;
          for (int e = r0; e < r1; e++) {
            const uint32_t ent = s_dn[e];
            const int t = (int)(ent >> 16);
            const double sg = sgn_of(c, s_losm[t]);
            y = VT<T>::add(y, coef_mul<T>(sg * s_locoef[2 * t], sg * s_locoef[2 * t + 1], row[ent & 0xFFFFu]));
          }
        }
      } else {
        x = v1[jb + p];
        y = VT<T>::zero();
      }
      // upper-half hops of this phase's spin: the same position in a block of the same class
      for (int k = 0; k < nhb; k++) {
        const int64_t src = bl.src[k];
        if (src < 0) continue;
        const double sg = sgn_of(c, bl.sm[k]);
        y = VT<T>::add(y, coef_mul<T>(sg * bl.re[k], sg * bl.im[k], v1[src + p]));
      }
      // cross hops of this phase's spin
      const uint32_t own = (PHASE == 0) ? ua : da;
      for (int q = 0; q < ncb; q++) {
        const int k = kMaxBlockTerms - 1 - q;
        if ((int)((own >> bl.bit[k]) & 1u) != bl.need[k]) continue;
        const int64_t src = bl.src[k];
        if (src < 0) continue;
        const int r_new = s_rank[own ^ (1u << bl.bit[k])];
        const int64_t j = (PHASE == 0) ? src + (int64_t)r_new * nda + rd : src + (int64_t)ra * bl.nsrc[k] + r_new;
        const double sg = sgn_of(c, bl.sm[k]);
        y = VT<T>::add(y, coef_mul<T>(sg * bl.re[k], sg * bl.im[k], v1[j]));
      }
      pr[0] += VT<T>::conj_mul_re(x, y);
      pr[1] += VT<T>::conj_mul_im(x, y);
      y = VT<T>::scale(scale, y);
      if (PHASE == 0) v0[jb + p] = (acc == 0.0) ? y : VT<T>::add(VT<T>::scale(acc, v0[jb + p]), y);
      else v0[jb + p] = VT<T>::add(v0[jb + p], y);
    }
    __syncthreads();
  }
  block_sum<2>(pr);
  if (threadIdx.x == 0) {
    part[2 * (PHASE * gridDim.x + blockIdx.x)] = pr[0];
    part[2 * (PHASE * gridDim.x + blockIdx.x) + 1] = pr[1];
  }
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
  for (int bi = blockIdx.x; bi < a.nblocks; bi += gridDim.x) {
    const uint64_t ib = a.order[0][bi];
    const int64_t jb = (int64_t)a.list_2_2[ib] - 1;
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
  size_t smem[2][2] = {{0, 0}, {0, 0}};  // [phase][real, complex]
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
  if (m.calc_model != kHubbard || m.nsite % 2 != 0 || m.nsite > 16 || s->gc) return 0;
  const int N = m.nsite, L = N / 2;
  const uint64_t lo_mask = (1ull << N) - 1;
  // classify off-diagonal terms; any term that is not a spin-conserving single hop
  // keeps the general kernel
  struct Hop { uint64_t cm, cv, flip, sm; double re, im; int p, q; };
  std::vector<Hop> lo_up, lo_dn, hi[2], cross[2];
  for (const BitTerm &t : m.offdiag) {
    if (__builtin_popcountll(t.flip) != 2 || t.cm != t.flip) return 0;
    const int p = __builtin_ctzll(t.flip), q = 63 - __builtin_clzll(t.flip);
    if ((p & 1) != (q & 1)) return 0;
    if (t.cv != (1ull << p) && t.cv != (1ull << q)) return 0;
    Hop h{t.cm, t.cv, t.flip, t.sm, t.re, t.im, p, q};
    const int spin = p & 1;
    if (q < N) (spin ? lo_dn : lo_up).push_back(h);
    else if (p >= N) hi[spin].push_back(h);
    else cross[spin].push_back(h);
  }
  for (int sp = 0; sp < 2; sp++)
    if ((int)(hi[sp].size() + cross[sp].size()) > kMaxBlockTerms) return 0;
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
  // lower-half CSR: for species spin (0 up / 1 down), row = (class k, rank r) of that species;
  // entries reference the lower-half hop table lo_coef / lo_sm (ups first, then downs)
  std::vector<double> lo_coef;
  std::vector<uint32_t> lo_sm;
  for (const auto *hops : {&lo_up, &lo_dn})
    for (const Hop &h : *hops) {
      lo_coef.push_back(h.re);
      lo_coef.push_back(h.im);
      lo_sm.push_back((uint32_t)h.sm);
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
  // upper-half and cross hops per spin: hi first, then cross
  std::vector<HubTermDev> terms[2];
  for (int sp = 0; sp < 2; sp++) {
    for (int pass = 0; pass < 2; pass++)
      for (const Hop &h : (pass == 0 ? hi[sp] : cross[sp])) {
        HubTermDev d{};
        d.cm_hi = (uint32_t)(h.cm >> N);
        d.cv_hi = (uint32_t)(h.cv >> N);
        d.flip_hi = (uint32_t)(h.flip >> N);
        d.sm = (uint32_t)h.sm;
        d.re = h.re; d.im = h.im;
        d.lo_bit = -1; d.lo_need = 0;
        if (pass == 1) {
          d.lo_bit = h.p >> 1;  // h.p is the lower-half end (p < N <= q)
          d.lo_need = (int)((h.cv >> h.p) & 1ull);
        }
        terms[sp].push_back(d);
      }
  }
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
  // block processing orders: phase 0 walks the block grid by columns (fixed db),
  // phase 1 by rows (fixed ub)
  std::vector<uint32_t> l22(s->sdim);
  if (cudaMemcpy(l22.data(), s->d_list_2_2, sizeof(uint32_t) * s->sdim, cudaMemcpyDeviceToHost) != cudaSuccess) {
    *err = "hubbard plan: cannot read list_2_2";
    return -1;
  }
  auto compress = [&](uint32_t x, int shift) {
    uint32_t v = 0;
    for (int b = 0; b < L; b++) v |= ((x >> (2 * b + shift)) & 1u) << b;
    return v;
  };
  std::vector<uint32_t> ord0, ord1;
  for (uint32_t ib = 0; ib < (uint32_t)s->sdim; ib++)
    if (l22[ib]) ord0.push_back(ib);
  ord1 = ord0;
  std::stable_sort(ord0.begin(), ord0.end(), [&](uint32_t x, uint32_t y) {
    const uint32_t dx = compress(x, 1), dy = compress(y, 1);
    return dx != dy ? dx < dy : compress(x, 0) < compress(y, 0);
  });
  std::stable_sort(ord1.begin(), ord1.end(), [&](uint32_t x, uint32_t y) {
    const uint32_t ux = compress(x, 0), uy = compress(y, 0);
    return ux != uy ? ux < uy : compress(x, 1) < compress(y, 1);
  });

  HubPlan *plan = new HubPlan();
  HubArgs &a = plan->args;
  a.L = L; a.N = N; a.nup = m.nup; a.ndn = m.ndown;
  a.nblocks = (int)ord0.size();
  a.list_2_2 = s->d_list_2_2;
  auto up = [&](auto &vec, auto **dst) -> int {
    if (upload(vec, dst, err)) return -1;
    plan->allocs.push_back((void *)*dst);
    return 0;
  };
  uint16_t *d_rank, *d_unrank;
  int *d_uoff, *d_binom, *d_up_ptr, *d_dn_ptr, *d_dlo_off;
  uint32_t *d_spread, *d_up_ent, *d_dn_ent, *d_lo_sm, *d_ord0, *d_ord1;
  double *d_lo_coef, *d_dlo, *d_dhi;
  HubTermDev *d_t0, *d_t1;
  DiagTerm *d_dcross;
  if (up(rank, &d_rank) || up(unrank, &d_unrank) || up(unrank_off, &d_uoff) || up(binom, &d_binom) ||
      up(spread, &d_spread) || up(up_ptr, &d_up_ptr) || up(up_ent, &d_up_ent) || up(dn_ptr, &d_dn_ptr) ||
      up(dn_ent, &d_dn_ent) || up(lo_coef, &d_lo_coef) || up(lo_sm, &d_lo_sm) || up(terms[0], &d_t0) ||
      up(terms[1], &d_t1) || up(dlo, &d_dlo) || up(dlo_off, &d_dlo_off) || up(dhi, &d_dhi) ||
      up(dcross, &d_dcross) || up(ord0, &d_ord0) || up(ord1, &d_ord1)) {
    hub_plan_free(plan);
    return -1;
  }
  a.rank = d_rank; a.unrank = d_unrank; a.unrank_off = d_uoff; a.binom = d_binom; a.spread = d_spread;
  a.csr_up_ptr = d_up_ptr; a.csr_up = d_up_ent; a.csr_dn_ptr = d_dn_ptr; a.csr_dn = d_dn_ent;
  a.n_csr_up = (int)up_ent.size(); a.n_csr_dn = (int)dn_ent.size(); a.n_lo = (int)lo_sm.size();
  a.lo_coef = d_lo_coef; a.lo_sm = d_lo_sm;
  a.terms[0] = d_t0; a.terms[1] = d_t1;
  for (int sp = 0; sp < 2; sp++) { a.n_hi[sp] = (int)hi[sp].size(); a.n_cross[sp] = (int)cross[sp].size(); }
  a.d_lo = d_dlo; a.d_lo_off = d_dlo_off; a.d_hi = d_dhi; a.d_cross = d_dcross; a.n_dcross = (int)dcross.size();
  a.order[0] = d_ord0; a.order[1] = d_ord1;
  plan->n_lo_terms = a.n_lo;
  int maxn = 0;
  for (int ku = 0; ku <= L; ku++)
    for (int kd = 0; kd <= L; kd++) maxn = std::max(maxn, binom[ku] * binom[kd]);
  // dynamic shared memory: tables (+ lower-half CSR and the staged block in phase 0)
  const size_t tables = sizeof(uint32_t) * nx + 2 * sizeof(uint16_t) * nx + 2 * sizeof(int) * 32;
  size_t p0 = tables + 2 * sizeof(int) * (nx + 1) + sizeof(uint32_t) * (up_ent.size() + dn_ent.size() + lo_sm.size());
  p0 = (p0 + 15) & ~(size_t)15;
  p0 += sizeof(double) * 2 * lo_sm.size();
  plan->smem[0][0] = p0 + sizeof(double) * (size_t)maxn;
  plan->smem[0][1] = p0 + sizeof(cplx) * (size_t)maxn;
  plan->smem[1][0] = plan->smem[1][1] = tables;
  if (plan->smem[0][1] > 200 * 1024) { hub_plan_free(plan); return 0; }
  cudaFuncSetAttribute((const void *)hv_hub_phase<double, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan->smem[0][0]);
  cudaFuncSetAttribute((const void *)hv_hub_phase<cplx, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan->smem[0][1]);
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hv_hub_phase<double, 0>, kThreads, plan->smem[0][0]);
  plan->grid = std::max(1, per_sm) * s->num_sms;
  if (2 * plan->grid > 4 * s->red_blocks) plan->grid = 2 * s->red_blocks;
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
  if (vt == kReal64) {
    hv_hub_phase<double, 0><<<p->grid, kThreads, p->smem[0][0], s->stream>>>(p->args, (const double *)d_v1,
                                                                             (double *)d_v0, d_coef, s->d_red);
    hv_hub_phase<double, 1><<<p->grid, kThreads, p->smem[1][0], s->stream>>>(p->args, (const double *)d_v1,
                                                                             (double *)d_v0, d_coef, s->d_red);
  } else {
    hv_hub_phase<cplx, 0><<<p->grid, kThreads, p->smem[0][1], s->stream>>>(p->args, (const cplx *)d_v1,
                                                                           (cplx *)d_v0, d_coef, s->d_red);
    hv_hub_phase<cplx, 1><<<p->grid, kThreads, p->smem[1][1], s->stream>>>(p->args, (const cplx *)d_v1,
                                                                           (cplx *)d_v0, d_coef, s->d_red);
  }
  finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(s->d_red, 2 * p->grid, d_out);
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
