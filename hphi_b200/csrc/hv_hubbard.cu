// Block kernel for canonical Hubbard Hamiltonians.
//
// Applies when every off-diagonal term is a spin-conserving single hop c+_{i s} c_{j s}
// (the Trans terms of a Hubbard model, src/mltplyHubbard.c:174-209, element routine
// CisAjt src/mltplyHubbardCore.c:305-347) and Nsite is even and at most 16; diagonal
// terms of any kind are allowed (src/diagonalcalc.c).  Other inputs use hv.cu.
//
// Native vector order.  HPhi orders the sector by upper half ib and, inside a block,
// by increasing lower half ia (src/sz.c:993-1094).  The native order keeps HPhi's block
// offsets (list_2_2) but stores block ib as a dense matrix
//   pos = rank(ua) * C(L, pop(da)) + rank(da),
// ua / da = up / down occupations of the lower half (L = Nsite/2 sites, ranks among
// L-bit numbers of equal popcount).  The native basis also orders fermion modes
// species-first (all up modes, then all down modes) instead of HPhi's interleaved bit
// order; the two bases differ by a diagonal sign
//   sigma(c) = (-1)^#{(down at i, up at j) : i < j},
// applied by the boundary permutation.  In the species-first basis the sign of a hop
// only counts occupied modes of its own species between its two sites, so every sign
// is a property of the row (ua or da) or of the block (ub or db) and is folded into
// precomputed coefficients.
//
// H*v runs in two passes over the block grid (ub, db):
//   pass 0 (blocks ordered by db, then ub): v0 = acc*v0 + scale*(D + H_lower + H_up) v1
//     lower-half up hops:    rows of the block staged in shared memory
//     lower-half down hops:  entries within a row of the staged block
//     upper-half up hops:    the same position in block (ub', db)        (coalesced)
//     cross up hops:         row rank(ua ^ bit) of block (ub ^ bit, db)   (coalesced)
//   pass 1 (blocks ordered by ub, then db): v0 += scale * H_down,upper+cross v1
// Up hops never change db and down hops never change ub, so the source blocks of a
// pass are the current column (row) of the block grid, a few MB that stay in L2.
// Blocks are handed out through an atomic counter so the CTAs in flight stay within a
// compact window of that order.
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
constexpr int kMaxBlockTerms = 96;  // upper-half + cross hops of one spin
constexpr int kCols = 3;            // columns per lane: C(L, L/2) <= 96 for L <= 8

struct HubTermDev {    // upper-half or cross hop of one spin
  uint32_t cm_hi, cv_hi, flip_hi;  // condition / flip on the upper half (bits of ib)
  uint32_t btw_hi;                 // upper-half sites (as bits of ub or db) counted by the sign
  double re, im;                   // operator coefficient
  int lo_bit;                      // cross hops: lower-half site (bit of ua / da); -1 otherwise
  int lo_need;                     // cross hops: occupation of that site in the output
};

struct HubArgs {
  int L, N, nup, ndn;
  int nblocks;
  const uint32_t *order[2];        // block processing order of pass 0 / pass 1
  int *counter;                    // [2] block dispenser of each pass
  const uint32_t *list_2_2;        // HPhi's list_2_2 (block offsets + 1)
  const uint16_t *rank;            // [2^L]
  const uint16_t *unrank;          // [2^L], grouped by popcount (offsets unrank_off)
  const int *unrank_off;           // [L+2]
  const int *binom;                // [L+1]
  const uint32_t *spread;          // [2^L] site bits -> even bit positions (HPhi layout)
  const int *csr_ptr[2];           // [2^L + 1] lower-half hops of each spin, rows (k, r)
  const uint16_t *csr[2];          // entry: source rank | hop << 8 | sign << 15
  int n_csr[2];
  const double *hop_coef[2];       // [n_lo_hops[s]][2] operator coefficients of lower-half hops
  int n_lo_hops[2];
  const uint16_t *cross_tab;       // [L][2^L]: rank(x ^ bit) | occupation << 14 | sign << 15
  const HubTermDev *terms[2];      // per spin: n_hi upper-half hops, then n_cross cross hops
  int n_hi[2], n_cross[2];
  const double *d_lo;              // diagonal (lower-half terms) per class pair, native order
  const int *d_lo_off;             // [(L+1)^2]
  const double *d_hi;              // [2^N] diagonal (upper-half terms)
  const DiagTerm *d_cross;         // diagonal terms spanning both halves (HPhi bit layout)
  int n_dcross;
};

struct BlockTerms {  // the current block's upper-half and cross hops, signs resolved
  int64_t src[kMaxBlockTerms];
  double re[kMaxBlockTerms], im[kMaxBlockTerms];
  int nsrc[kMaxBlockTerms];
  unsigned char bit[kMaxBlockTerms], need[kMaxBlockTerms];
  int n_hi, n_cr, bi;
};

template <typename T>
__device__ __forceinline__ T cfma(double re, double im, T x, T y);
template <>
__device__ __forceinline__ double cfma<double>(double re, double, double x, double y) { return fma(re, x, y); }
template <>
__device__ __forceinline__ cplx cfma<cplx>(double re, double im, cplx x, cplx y) {
  return cplx{fma(re, x.x, fma(-im, x.y, y.x)), fma(re, x.y, fma(im, x.x, y.y))};
}

__host__ __device__ __forceinline__ uint32_t compress_bits(uint32_t x, int shift, int L) {
  uint32_t v = 0;
  for (int b = 0; b < L; b++) v |= ((x >> (2 * b + shift)) & 1u) << b;
  return v;
}

template <typename T, int PASS>
__global__ void __launch_bounds__(kThreads, PASS == 0 ? 3 : 4) hv_hub_pass(HubArgs a, const T *__restrict__ v1, T *__restrict__ v0,
                                                        const double *__restrict__ coef, double *__restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ BlockTerms bl;
  const int L = a.L, N = a.N, nx = 1 << L;
  // shared tables (pass 0 also holds the lower-half CSR of both spins and the staged block)
  unsigned char *sp = smem_raw;
  double *s_hop[2] = {nullptr, nullptr};
  int *s_ptr[2] = {nullptr, nullptr};
  uint16_t *s_csr[2] = {nullptr, nullptr};
  uint16_t *s_ctab = nullptr;
  if (PASS == 0) {
    s_hop[0] = reinterpret_cast<double *>(sp); sp += sizeof(double) * 2 * a.n_lo_hops[0];
    s_hop[1] = reinterpret_cast<double *>(sp); sp += sizeof(double) * 2 * a.n_lo_hops[1];
    s_ptr[0] = reinterpret_cast<int *>(sp); sp += sizeof(int) * (nx + 1);
    s_ptr[1] = reinterpret_cast<int *>(sp); sp += sizeof(int) * (nx + 1);
  }
  int *s_uoff = reinterpret_cast<int *>(sp); sp += sizeof(int) * 32;
  int *s_binom = reinterpret_cast<int *>(sp); sp += sizeof(int) * 32;
  uint16_t *s_rank = reinterpret_cast<uint16_t *>(sp); sp += sizeof(uint16_t) * nx;
  uint16_t *s_unrank = reinterpret_cast<uint16_t *>(sp); sp += sizeof(uint16_t) * nx;
  if (PASS == 0) {
    s_csr[0] = reinterpret_cast<uint16_t *>(sp); sp += sizeof(uint16_t) * a.n_csr[0];
    s_csr[1] = reinterpret_cast<uint16_t *>(sp); sp += sizeof(uint16_t) * a.n_csr[1];
  } else {
    s_ctab = reinterpret_cast<uint16_t *>(sp); sp += sizeof(uint16_t) * L * nx;
  }
  sp = smem_raw + (((sp - smem_raw) + 15) & ~(size_t)15);
  T *xs = reinterpret_cast<T *>(sp);
  for (int i = threadIdx.x; i < nx; i += blockDim.x) { s_rank[i] = a.rank[i]; s_unrank[i] = a.unrank[i]; }
  for (int i = threadIdx.x; i < 32; i += blockDim.x) {
    s_uoff[i] = (i <= L + 1) ? a.unrank_off[i] : 0;
    s_binom[i] = (i <= L) ? a.binom[i] : 0;
  }
  if (PASS == 0) {
    for (int q = 0; q < 2; q++) {
      for (int i = threadIdx.x; i <= nx; i += blockDim.x) s_ptr[q][i] = a.csr_ptr[q][i];
      for (int i = threadIdx.x; i < a.n_csr[q]; i += blockDim.x) s_csr[q][i] = a.csr[q][i];
      for (int i = threadIdx.x; i < 2 * a.n_lo_hops[q]; i += blockDim.x) s_hop[q][i] = a.hop_coef[q][i];
    }
  } else {
    for (int i = threadIdx.x; i < L * nx; i += blockDim.x) s_ctab[i] = a.cross_tab[i];
  }
  __syncthreads();
  const double acc = coef[0], scale = coef[1];
  const uint32_t even_mask = 0x55555555u & ((1u << N) - 1u);
  const HubTermDev *terms = a.terms[PASS];
  const int n_hi = a.n_hi[PASS], n_all = a.n_hi[PASS] + a.n_cross[PASS];
  double pr[2] = {0.0, 0.0};

  while (true) {
    if (threadIdx.x == 0) bl.bi = atomicAdd(&a.counter[PASS], 1);
    __syncthreads();
    const int bi = bl.bi;
    if (bi >= a.nblocks) break;
    const uint32_t ib = a.order[PASS][bi];
    const int64_t jb = (int64_t)a.list_2_2[ib] - 1;
    const int nu = a.nup - __popc(ib & even_mask), nd = a.ndn - __popc(ib & (even_mask << 1));
    const int nua = s_binom[nu], nda = s_binom[nd];
    const int n = nua * nda;
    if (PASS == 0)
      for (int p = threadIdx.x; p < n; p += blockDim.x) xs[p] = v1[jb + p];
    if (threadIdx.x < 32) {
      // resolve this block's hops of the pass's spin: source block and block-level sign
      const uint32_t own_hi = compress_bits(ib, PASS, L);  // ub (pass 0) or db (pass 1)
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
          const double sg = (__popc(own_hi & tt.btw_hi) & 1) ? -1.0 : 1.0;
          bl.src[slot] = (sl == 0u) ? -1 : (int64_t)sl - 1;
          bl.re[slot] = sg * tt.re;
          bl.im[slot] = sg * tt.im;
          bl.bit[slot] = tt.lo_bit;
          bl.need[slot] = tt.lo_need;
          const int k_src = (PASS == 0 ? nu : nd) + (tt.lo_need ? -1 : 1);
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
    const double dhi = (PASS == 0) ? a.d_hi[ib] : 0.0;
    const double *dlo = a.d_lo + a.d_lo_off[nu * (L + 1) + nd];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    // per-lane columns rd = lane + 32 r of the block rows
    uint32_t da[kCols];
#pragma unroll
    for (int r = 0; r < kCols; r++) da[r] = (lane + 32 * r < nda) ? s_unrank[off_d + lane + 32 * r] : 0u;
    // a warp owns a block row ra (ua uniform across the warp)
    for (int ra = warp; ra < nua; ra += nwarps) {
      const uint32_t ua = s_unrank[off_u + ra];
      const int row0 = ra * nda;
      T x[kCols], y[kCols];
#pragma unroll
      for (int r = 0; r < kCols; r++) {
        const int rd = lane + 32 * r;
        if (rd < nda) {
          if (PASS == 0) {
            x[r] = xs[row0 + rd];
            double dg = dlo[row0 + rd] + dhi;
            if (a.n_dcross) {
              const uint64_t c = ((uint64_t)ib << N) | a.spread[ua] | ((uint64_t)a.spread[da[r]] << 1);
              for (int k = 0; k < a.n_dcross; k++) {
                const DiagTerm dt = a.d_cross[k];
                if ((c & dt.cm) == dt.cv) dg += dt.v;
              }
            }
            y[r] = VT<T>::scale(dg, x[r]);
          } else {
            x[r] = v1[jb + row0 + rd];
            y[r] = VT<T>::zero();
          }
        } else {
          x[r] = VT<T>::zero();
          y[r] = VT<T>::zero();
        }
      }
      if (PASS == 0) {
        // lower-half up hops: warp-uniform CSR row of ua, source rows of the staged block
        const int r0 = s_ptr[0][off_u + ra], r1 = s_ptr[0][off_u + ra + 1];
        for (int e = r0; e < r1; e++) {
          const uint32_t ent = s_csr[0][e];
          const int h = (ent >> 8) & 0x7F;
          const double sg = (ent >> 15) ? -1.0 : 1.0;
          const double cre = sg * s_hop[0][2 * h], cim = sg * s_hop[0][2 * h + 1];
          const T *srow = xs + (int)(ent & 0xFF) * nda;
#pragma unroll
          for (int r = 0; r < kCols; r++)
            if (lane + 32 * r < nda) y[r] = cfma<T>(cre, cim, srow[lane + 32 * r], y[r]);
        }
        // lower-half down hops: per-column CSR rows within the staged row
        const T *row = xs + row0;
#pragma unroll
        for (int r = 0; r < kCols; r++) {
          const int rd = lane + 32 * r;
          if (rd < nda) {
            const int q0 = s_ptr[1][off_d + rd], q1 = s_ptr[1][off_d + rd + 1];
            for (int e = q0; e < q1; e++) {
              const uint32_t ent = s_csr[1][e];
              const int h = (ent >> 8) & 0x7F;
              const double sg = (ent >> 15) ? -1.0 : 1.0;
              y[r] = cfma<T>(sg * s_hop[1][2 * h], sg * s_hop[1][2 * h + 1], row[ent & 0xFF], y[r]);
            }
          }
        }
      }
      // upper-half hops: the same positions in a block of the same class
      for (int k = 0; k < nhb; k++) {
        const T *src = v1 + bl.src[k] + row0;
        const double cre = bl.re[k], cim = bl.im[k];
#pragma unroll
        for (int r = 0; r < kCols; r++)
          if (lane + 32 * r < nda) y[r] = cfma<T>(cre, cim, src[lane + 32 * r], y[r]);
      }
      // cross hops: one particle of this pass's spin changes half
      for (int q = 0; q < ncb; q++) {
        const int k = kMaxBlockTerms - 1 - q;
        const int b = bl.bit[k], need = bl.need[k];
        if (PASS == 0) {
          // condition, source row and sign depend on ua only: uniform across the warp
          if ((int)((ua >> b) & 1u) != need) continue;
          const double sg = (__popc(ua >> (b + 1)) & 1) ? -1.0 : 1.0;
          const double cre = sg * bl.re[k], cim = sg * bl.im[k];
          const T *src = v1 + bl.src[k] + (int64_t)s_rank[ua ^ (1u << b)] * nda;
#pragma unroll
          for (int r = 0; r < kCols; r++)
            if (lane + 32 * r < nda) y[r] = cfma<T>(cre, cim, src[lane + 32 * r], y[r]);
        } else {
          const T *src = v1 + bl.src[k] + (int64_t)ra * bl.nsrc[k];
          const uint16_t *tab = s_ctab + b * nx;
          const double cre = bl.re[k], cim = bl.im[k];
#pragma unroll
          for (int r = 0; r < kCols; r++) {
            const uint32_t e = tab[da[r]];
            if (lane + 32 * r < nda && (int)((e >> 14) & 1u) == need) {
              const double sg = (e >> 15) ? -1.0 : 1.0;
              y[r] = cfma<T>(sg * cre, sg * cim, src[e & 0x3FFF], y[r]);
            }
          }
        }
      }
#pragma unroll
      for (int r = 0; r < kCols; r++) {
        const int rd = lane + 32 * r;
        if (rd < nda) {
          pr[0] += VT<T>::conj_mul_re(x[r], y[r]);
          pr[1] += VT<T>::conj_mul_im(x[r], y[r]);
          const T yy = VT<T>::scale(scale, y[r]);
          T *dst = v0 + jb + row0 + rd;
          if (PASS == 0) *dst = (acc == 0.0) ? yy : VT<T>::add(VT<T>::scale(acc, *dst), yy);
          else *dst = VT<T>::add(*dst, yy);
        }
      }
    }
    __syncthreads();
  }
  block_sum<2>(pr);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = pr[0];
    part[2 * blockIdx.x + 1] = pr[1];
  }
}

// sigma(c) of the species-first basis: (-1)^#{(down at i, up at j) : i < j}.
__device__ __forceinline__ int species_sign(uint64_t c, int nsite) {
  int cnt = 0, downs = 0;
  for (int s = 0; s < nsite; s++) {
    if ((c >> (2 * s)) & 1ull) cnt += downs;
    downs += (int)((c >> (2 * s + 1)) & 1ull);
  }
  return cnt & 1;
}

// HPhi order <-> native order, per row r of HPhi's list_1 (sign sigma applied both ways).
template <typename T, bool TO_NATIVE>
__global__ void permute_kernel(int64_t dim, int N, int L, const uint64_t *__restrict__ list_1,
                               const uint32_t *__restrict__ list_2_2, const uint16_t *__restrict__ rank,
                               const int *__restrict__ binom, const T *__restrict__ in, T *__restrict__ out) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = list_1[r];
    const uint64_t ib = c >> N;
    const uint32_t ia = (uint32_t)(c & ((1ull << N) - 1));
    const uint32_t ua = compress_bits(ia, 0, L), da = compress_bits(ia, 1, L);
    const int64_t pos = (int64_t)list_2_2[ib] - 1 + (int64_t)rank[ua] * binom[__popc(da)] + rank[da];
    const double sg = species_sign(c, N) ? -1.0 : 1.0;
    if (TO_NATIVE) out[pos] = VT<T>::scale(sg, in[r]);
    else out[r] = VT<T>::scale(sg, in[pos]);
  }
}

// Diagonal observables in native order (expec_energy_flct_Hubbard, src/expec_energy_flct.c:259-330).
template <typename T>
__global__ void native_obs_kernel(HubArgs a, const T *__restrict__ v, double *__restrict__ part) {
  double o[6] = {0, 0, 0, 0, 0, 0};
  const int N = a.N;
  const uint32_t even_mask = 0x55555555u & ((1u << N) - 1u);
  for (int bi = blockIdx.x; bi < a.nblocks; bi += gridDim.x) {
    const uint32_t ib = a.order[0][bi];
    const int64_t jb = (int64_t)a.list_2_2[ib] - 1;
    const int nu = a.nup - __popc(ib & even_mask), nd = a.ndn - __popc(ib & (even_mask << 1));
    const int nda = a.binom[nd], n = a.binom[nu] * nda;
    const int off_u = a.unrank_off[nu], off_d = a.unrank_off[nd];
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
      const int ra = p / nda, rd = p - ra * nda;
      const uint64_t c = ((uint64_t)ib << N) | (uint64_t)a.spread[a.unrank[off_u + ra]] |
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
  const size_t bytes = h.empty() ? 16 : sizeof(V) * h.size();  // empty tables keep a valid pointer
  if (cudaMalloc(d, bytes) != cudaSuccess) {
    *err = "hubbard plan: device allocation failed";
    return -1;
  }
  if (!h.empty() && cudaMemcpy(*d, h.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    *err = "hubbard plan: copy failed";
    return -1;
  }
  return 0;
}

}  // namespace

struct HubPlan {
  HubArgs args;
  std::vector<void *> allocs;
  size_t smem[2][2] = {{0, 0}, {0, 0}};  // [pass][real, complex]
  int grid[2] = {0, 0};                  // CTAs of each pass (shared-memory bound differs)
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
  // Hops: site i (created) <- site j (annihilated), spin, operator coefficient.  The
  // compiled term carries HPhi's interleaved-order sign; its operator coefficient is the
  // amplitude on the configuration holding only the created particle (no modes between).
  struct Hop { int i, j, spin; double re, im; uint64_t cm, cv, flip; };
  std::vector<Hop> lo[2], hi[2], cross[2];
  for (const BitTerm &t : m.offdiag) {
    if (__builtin_popcountll(t.flip) != 2 || t.cm != t.flip) return 0;
    const int p = __builtin_ctzll(t.flip), q = 63 - __builtin_clzll(t.flip);
    if ((p & 1) != (q & 1)) return 0;
    if (t.cv != (1ull << p) && t.cv != (1ull << q)) return 0;
    const int created = __builtin_ctzll(t.cv), annihilated = (created == p) ? q : p;
    const double sg = (__builtin_popcountll(t.cv & t.sm) & 1) ? -1.0 : 1.0;
    Hop h{created >> 1, annihilated >> 1, p & 1, sg * t.re, sg * t.im, t.cm, t.cv, t.flip};
    if (q < N) lo[h.spin].push_back(h);
    else if (p >= N) hi[h.spin].push_back(h);
    else cross[h.spin].push_back(h);
  }
  for (int sp = 0; sp < 2; sp++)
    if ((int)(hi[sp].size() + cross[sp].size()) > kMaxBlockTerms) return 0;
  if (binom_u(L, L / 2) > 255) return 0;  // ranks fit the 8-bit CSR field
  const int nx = 1 << L;
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
  auto between = [](int i, int j) -> uint32_t {  // sites strictly between i and j (as bits)
    const int lo_ = std::min(i, j), hi_ = std::max(i, j);
    return (uint32_t)(((1ull << hi_) - 1) ^ ((1ull << (lo_ + 1)) - 1));
  };
  // lower-half CSR per spin: row = (class k, rank r) of that spin's lower-half occupation x;
  // entry = source rank | hop << 8 | sign << 15 (species-first sign: modes of x between i, j)
  std::vector<int> ptr[2];
  std::vector<uint16_t> csr[2];
  std::vector<double> hop_coef[2];
  for (int sp = 0; sp < 2; sp++) {
    if (lo[sp].size() > 127) return 0;
    for (const Hop &h : lo[sp]) { hop_coef[sp].push_back(h.re); hop_coef[sp].push_back(h.im); }
    ptr[sp].assign(nx + 1, 0);
    for (int k = 0; k <= L; k++)
      for (int r = 0; r < binom[k]; r++) {
        const int row = unrank_off[k] + r;
        const uint32_t x = unrank[row];
        for (size_t hh = 0; hh < lo[sp].size(); hh++) {
          const Hop &h = lo[sp][hh];
          if (!((x >> h.i) & 1u) || ((x >> h.j) & 1u)) continue;  // output: i occupied, j empty
          const uint32_t src = x ^ (1u << h.i) ^ (1u << h.j);
          const uint32_t neg = __builtin_popcount(x & between(h.i, h.j)) & 1;
          csr[sp].push_back((uint16_t)(rank[src] | (hh << 8) | (neg << 15)));
        }
        ptr[sp][row + 1] = (int)csr[sp].size();
      }
  }
  // cross-hop table: for site b and occupation x of one spin's lower half
  std::vector<uint16_t> cross_tab((size_t)L * nx);
  for (int b = 0; b < L; b++)
    for (int x = 0; x < nx; x++) {
      const uint32_t occ = (x >> b) & 1, neg = __builtin_popcount((uint32_t)x >> (b + 1)) & 1;
      cross_tab[(size_t)b * nx + x] = (uint16_t)(rank[x ^ (1 << b)] | (occ << 14) | (neg << 15));
    }
  // upper-half and cross hops per spin (upper-half first, then cross)
  std::vector<HubTermDev> terms[2];
  for (int sp = 0; sp < 2; sp++) {
    for (int pass = 0; pass < 2; pass++)
      for (const Hop &h : (pass == 0 ? hi[sp] : cross[sp])) {
        HubTermDev d{};
        d.cm_hi = (uint32_t)(h.cm >> N);
        d.cv_hi = (uint32_t)(h.cv >> N);
        d.flip_hi = (uint32_t)(h.flip >> N);
        d.re = h.re;
        d.im = h.im;
        if (pass == 0) {
          d.btw_hi = between(h.i - L, h.j - L);
          d.lo_bit = -1;
          d.lo_need = 0;
        } else {
          const int lo_site = std::min(h.i, h.j), hi_site = std::max(h.i, h.j);
          d.btw_hi = (uint32_t)((1ull << (hi_site - L)) - 1);  // upper-half sites below hi_site
          d.lo_bit = lo_site;  // the kernel adds the lower-half sites above lo_site
          d.lo_need = (lo_site == h.i) ? 1 : 0;
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
  // block orders: pass 0 by (db, ub), pass 1 by (ub, db)
  std::vector<uint32_t> l22(s->sdim);
  if (cudaMemcpy(l22.data(), s->d_list_2_2, sizeof(uint32_t) * s->sdim, cudaMemcpyDeviceToHost) != cudaSuccess) {
    *err = "hubbard plan: cannot read list_2_2";
    return -1;
  }
  std::vector<uint32_t> ord0, ord1;
  for (uint32_t ib = 0; ib < (uint32_t)s->sdim; ib++)
    if (l22[ib]) ord0.push_back(ib);
  for (int sp = 0; sp < 2; sp++)
    for (int t = 0; t < (int)hi[sp].size(); t++) {
      const HubTermDev &d = terms[sp][t];
      for (uint32_t ib : ord0)
        if ((ib & d.cm_hi) == d.cv_hi && l22[ib ^ d.flip_hi] == 0) return 0;  // keep the general kernel
    }
  ord1 = ord0;
  std::stable_sort(ord0.begin(), ord0.end(), [&](uint32_t x, uint32_t y) {
    const uint32_t dx = compress_bits(x, 1, L), dy = compress_bits(y, 1, L);
    return dx != dy ? dx < dy : compress_bits(x, 0, L) < compress_bits(y, 0, L);
  });
  std::stable_sort(ord1.begin(), ord1.end(), [&](uint32_t x, uint32_t y) {
    const uint32_t ux = compress_bits(x, 0, L), uy = compress_bits(y, 0, L);
    return ux != uy ? ux < uy : compress_bits(x, 1, L) < compress_bits(y, 1, L);
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
  uint16_t *d_rank, *d_unrank, *d_csr0, *d_csr1, *d_ctab;
  int *d_uoff, *d_binom, *d_ptr0, *d_ptr1, *d_dlo_off;
  uint32_t *d_spread, *d_ord0, *d_ord1;
  double *d_hop0, *d_hop1, *d_dlo, *d_dhi;
  HubTermDev *d_t0, *d_t1;
  DiagTerm *d_dcross;
  std::vector<int> ctr(2, 0);
  int *d_ctr;
  if (up(rank, &d_rank) || up(unrank, &d_unrank) || up(unrank_off, &d_uoff) || up(binom, &d_binom) ||
      up(spread, &d_spread) || up(ptr[0], &d_ptr0) || up(ptr[1], &d_ptr1) || up(csr[0], &d_csr0) ||
      up(csr[1], &d_csr1) || up(hop_coef[0], &d_hop0) || up(hop_coef[1], &d_hop1) || up(cross_tab, &d_ctab) ||
      up(terms[0], &d_t0) ||
      up(terms[1], &d_t1) || up(dlo, &d_dlo) || up(dlo_off, &d_dlo_off) || up(dhi, &d_dhi) ||
      up(dcross, &d_dcross) || up(ord0, &d_ord0) || up(ord1, &d_ord1) || up(ctr, &d_ctr)) {
    hub_plan_free(plan);
    return -1;
  }
  a.rank = d_rank; a.unrank = d_unrank; a.unrank_off = d_uoff; a.binom = d_binom; a.spread = d_spread;
  a.csr_ptr[0] = d_ptr0; a.csr_ptr[1] = d_ptr1; a.csr[0] = d_csr0; a.csr[1] = d_csr1;
  a.n_csr[0] = (int)csr[0].size(); a.n_csr[1] = (int)csr[1].size();
  a.hop_coef[0] = d_hop0; a.hop_coef[1] = d_hop1;
  a.n_lo_hops[0] = (int)lo[0].size(); a.n_lo_hops[1] = (int)lo[1].size();
  a.cross_tab = d_ctab;
  a.terms[0] = d_t0; a.terms[1] = d_t1;
  for (int sp = 0; sp < 2; sp++) { a.n_hi[sp] = (int)hi[sp].size(); a.n_cross[sp] = (int)cross[sp].size(); }
  a.d_lo = d_dlo; a.d_lo_off = d_dlo_off; a.d_hi = d_dhi; a.d_cross = d_dcross; a.n_dcross = (int)dcross.size();
  a.order[0] = d_ord0; a.order[1] = d_ord1;
  a.counter = d_ctr;
  int maxn = 0;
  for (int ku = 0; ku <= L; ku++)
    for (int kd = 0; kd <= L; kd++) maxn = std::max(maxn, binom[ku] * binom[kd]);
  // dynamic shared memory of each pass (layout as in hv_hub_pass)
  const size_t base = sizeof(int) * 64 + 2 * sizeof(uint16_t) * nx;
  size_t p0 = sizeof(double) * 2 * (lo[0].size() + lo[1].size()) + 2 * sizeof(int) * (nx + 1) + base +
              sizeof(uint16_t) * (csr[0].size() + csr[1].size());
  p0 = (p0 + 15) & ~(size_t)15;
  plan->smem[0][0] = p0 + sizeof(double) * (size_t)maxn;
  plan->smem[0][1] = p0 + sizeof(cplx) * (size_t)maxn;
  plan->smem[1][0] = plan->smem[1][1] = (base + sizeof(uint16_t) * L * nx + 15) & ~(size_t)15;
  if (plan->smem[0][1] > 200 * 1024) { hub_plan_free(plan); return 0; }
  raise_smem_limit((const void *)hv_hub_pass<double, 0>, plan->smem[0][0]);
  raise_smem_limit((const void *)hv_hub_pass<cplx, 0>, plan->smem[0][1]);
  int per_sm0 = 1, per_sm1 = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm0, hv_hub_pass<double, 0>, kThreads, plan->smem[0][0]);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm1, hv_hub_pass<double, 1>, kThreads, plan->smem[1][0]);
  // partial sums: pass p writes records [p * grid[0] + block]; both fit 4 * red_blocks records
  plan->grid[0] = std::min(std::max(1, per_sm0) * s->num_sms, 2 * s->red_blocks);
  plan->grid[1] = std::min(std::max(1, per_sm1) * s->num_sms, 2 * s->red_blocks);
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
  cudaMemsetAsync(p->args.counter, 0, 2 * sizeof(int), s->stream);
  if (vt == kReal64) {
    hv_hub_pass<double, 0><<<p->grid[0], kThreads, p->smem[0][0], s->stream>>>(p->args, (const double *)d_v1,
                                                                               (double *)d_v0, d_coef, s->d_red);
    hv_hub_pass<double, 1><<<p->grid[1], kThreads, p->smem[1][0], s->stream>>>(p->args, (const double *)d_v1,
                                                                               (double *)d_v0, d_coef,
                                                                               s->d_red + 2 * p->grid[0]);
  } else {
    hv_hub_pass<cplx, 0><<<p->grid[0], kThreads, p->smem[0][1], s->stream>>>(p->args, (const cplx *)d_v1,
                                                                             (cplx *)d_v0, d_coef, s->d_red);
    hv_hub_pass<cplx, 1><<<p->grid[1], kThreads, p->smem[1][1], s->stream>>>(p->args, (const cplx *)d_v1,
                                                                             (cplx *)d_v0, d_coef,
                                                                             s->d_red + 2 * p->grid[0]);
  }
  finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(s->d_red, p->grid[0] + p->grid[1], d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("hubbard hv launch failed: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

size_t hub_scratch_doubles(const Sector *s) { return 2 * (size_t)(s->hub->grid[0] + s->hub->grid[1]); }

int hub_hv_launch_scratch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                          double *d_part, int *d_counter) {
  HubPlan *p = s->hub;
  if (vt == kReal64 && s->model.complex_terms) {
    set_error("H has complex coefficients: real vectors are not allowed");
    return -1;
  }
  HubArgs args = p->args;
  args.counter = d_counter;
  if (cudaMemsetAsync(d_counter, 0, 2 * sizeof(int), s->stream) != cudaSuccess) {
    set_error("hubbard hv: clearing the block counters failed");
    return -1;
  }
  if (vt == kReal64) {
    hv_hub_pass<double, 0><<<p->grid[0], kThreads, p->smem[0][0], s->stream>>>(args, (const double *)d_v1,
                                                                               (double *)d_v0, d_coef, d_part);
    hv_hub_pass<double, 1><<<p->grid[1], kThreads, p->smem[1][0], s->stream>>>(args, (const double *)d_v1,
                                                                               (double *)d_v0, d_coef,
                                                                               d_part + 2 * p->grid[0]);
  } else {
    hv_hub_pass<cplx, 0><<<p->grid[0], kThreads, p->smem[0][1], s->stream>>>(args, (const cplx *)d_v1,
                                                                             (cplx *)d_v0, d_coef, d_part);
    hv_hub_pass<cplx, 1><<<p->grid[1], kThreads, p->smem[1][1], s->stream>>>(args, (const cplx *)d_v1,
                                                                             (cplx *)d_v0, d_coef,
                                                                             d_part + 2 * p->grid[0]);
  }
  finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(d_part, p->grid[0] + p->grid[1], d_out);
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
  if (vt == kReal64)
    native_obs_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(p->args, (const double *)v, s->d_red);
  else
    native_obs_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(p->args, (const cplx *)v, s->d_red);
  finalize_partials_kernel<6><<<1, 256, 0, s->stream>>>(s->d_red, s->red_blocks, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("observables failed: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

}  // namespace hphi
