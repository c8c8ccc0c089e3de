// Row-block kernels for spin models (canonical Spin with a fixed Sz, and the grand-canonical
// models whose rows are their configurations: SpinGC, HubbardGC).
//
// HPhi stores these sectors as blocks of consecutive rows that share the upper half of the
// configuration (sz, src/sz.c:993-1094 and omp_sz_spin_hacker :1495-1546): block ib holds
// the lower halves ia whose particle count completes the sector, in increasing order, at
// row list_2_2[ib] - 1 + list_2_1[ia] - 2 (grand-canonical: row = configuration).  A term
// of the Hamiltonian is
//   lower-half: every mask in the lower half; it maps a row to a row of the same block,
//   upper-half: every mask in the upper half; it maps a whole block to a block of the same
//               size, position for position (src/mltplySpinCore.c:273-307 in gather form),
//   crossing:   masks in both halves (a bond across the split).
// The split-term plan (split.cuh) lists the first two kinds per lower / upper half and keeps
// the crossing ones as generic terms.  H*v is done in two passes over the vectors:
//   row pass:    one CTA per block; the block of v1 is staged in shared memory, every row
//                applies the diagonal, its lower-half terms as gathers inside the staged
//                block and its crossing terms as gathers from global memory (few per row:
//                a lattice cut across the split), v0 = acc * v0 + scale * (...);
//   column pass: upper-half terms, the same for every row of a block: a warp takes one
//                block and 64 positions and reads each source block's 64 positions as
//                whole 256/512-byte pieces; tasks run class by class and chunk by chunk so
//                the pieces being gathered stay in L2; v0 += scale * (...).
// Both passes keep per-CTA partial sums of <v1|H v1> (static work assignment, so results are
// reproducible); the vectors stay in HPhi's order.
//
// Fast row pass (canonical Spin, real vectors, every lower-half term of one magnitude, e.g.
// the Heisenberg exchange): the lower-half operator depends only on the block's class (the
// popcount of its lower halves), so each class gets the edge-coloured gather table of the
// Hubbard row pass (hv_product.cu: 16-bit entries position | sign << 15, every 8-byte gather
// of a half-warp on its own shared-memory bank pair); a CTA of 1024 threads stages two blocks
// of one class at once and every table entry serves both.  The crossing terms whose
// upper-half condition the block meets are listed once per block; each then walks its source
// block in increasing order (a flip of one lower-half bit keeps the order of the positions),
// through a per-class table of source positions.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <string>
#include <vector>

#include "device_util.cuh"
#include "engine.hpp"
#include "hv_product.hpp"
#include "hv_rowblock.hpp"
#include "split.cuh"
#include "tma.cuh"

namespace hphi {
namespace {

constexpr int kRowThreads = 512;
constexpr int kColThreads = 256;
constexpr int kColBatch = 4;       // upper-half terms per batch of loads
constexpr int kRowTermMax = 256;   // crossing terms staged in shared memory
constexpr size_t kSmemLimit = 227 * 1024;

struct RBArgs {
  int nblk;                      // blocks
  const uint32_t *rb_ib;         // [nblk] row pass order (largest first): upper half
  const int64_t *rb_start;       // first row
  const int *rb_n;               // rows
  const int *rb_uoff;            // offset of the block's lower halves in unrank (canonical)
  const uint32_t *unrank;        // lower halves of each class in position order
  int nclass;
  const int *cl_nblk;            // blocks of the class
  const int *cl_boff;            // offset of the class's blocks in cb_*
  const uint32_t *cb_ib;         // blocks grouped by class
  const int64_t *cb_start;
  const int *cb_n;
  const int *cb_key;             // class of each block (canonical: popcount of its lower halves)
  int lo_bits;
  uint64_t lo_mask;
  int lo_base;                   // position of a lower half = its lower-term target - lo_base
};

// Row pass.  part[blockIdx] = (re, im) of sum conj(v1) (diagonal + lower + crossing) v1 over
// the CTA's blocks.
template <typename T, bool GC>
__global__ void __launch_bounds__(kRowThreads) rb_row_kernel(RBArgs p, SplitView sv, const BitTerm *__restrict__ gterms,
                                                            int ngen, const uint32_t *__restrict__ l21,
                                                            const uint32_t *__restrict__ l22,
                                                            const double *__restrict__ diag, const T *__restrict__ v1,
                                                            T *__restrict__ v0, const double *__restrict__ coef,
                                                            double *__restrict__ part) {
  extern __shared__ __align__(16) unsigned char rb_smem[];
  BitTerm *terms = reinterpret_cast<BitTerm *>(rb_smem);
  T *row = reinterpret_cast<T *>(rb_smem + sizeof(BitTerm) * (size_t)ngen);
  const double acc = coef[0], scale = coef[1];
  for (int k = threadIdx.x; k < ngen; k += blockDim.x) terms[k] = gterms[k];
  const double2 *cf = reinterpret_cast<const double2 *>(sv.coef);
  double pr[2] = {0.0, 0.0};
  for (int b = blockIdx.x; b < p.nblk; b += gridDim.x) {
    const uint64_t ib = p.rb_ib[b];
    const int64_t start = p.rb_start[b];
    const int n = p.rb_n[b];
    __syncthreads();  // the previous block is no longer read (and the terms are staged)
    for (int a = threadIdx.x; a < n; a += blockDim.x) row[a] = v1[start + a];
    __syncthreads();
    const uint32_t *un = GC ? nullptr : p.unrank + p.rb_uoff[b];
    const uint64_t hi = ib << p.lo_bits;
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
      const int64_t r = start + a;
      const uint32_t ia = GC ? (uint32_t)a : __ldg(un + a);
      const uint64_t c = hi | ia;
      const T x = row[a];
      T y = VT<T>::scale(__ldg(diag + r), x);
      const uint32_t e0 = __ldg(sv.lo_ptr + ia), e1 = __ldg(sv.lo_ptr + ia + 1);
      for (uint32_t e = e0; e < e1; e++) {
        const uint32_t v = __ldg(sv.lo_ent + e);
        const int src = (int)(v & ((1u << kSplitTargetBits) - 1u)) - p.lo_base;
        const double2 w = __ldg(cf + (v >> kSplitTargetBits));
        y = VT<T>::add(y, VT<T>::cmul_re_im(w.x, w.y, row[src]));
      }
      for (int k = 0; k < ngen; k++) {
        const BitTerm t = terms[k];
        if ((c & t.cm) != t.cv) continue;
        const uint64_t s = c ^ t.flip;
        int64_t j;
        if (GC) {
          j = (int64_t)s;
        } else {
          const uint32_t a1 = __ldg(l21 + (s & p.lo_mask)), b1 = __ldg(l22 + (s >> p.lo_bits));
          if (a1 == 0u || b1 == 0u) continue;
          j = (int64_t)a1 + (int64_t)b1 - 3;
        }
        const bool neg = __popcll(c & t.sm) & 1;
        y = VT<T>::add(y, VT<T>::cmul_re_im(neg ? -t.re : t.re, neg ? -t.im : t.im, v1[j]));
      }
      pr[0] += VT<T>::conj_mul_re(x, y);
      pr[1] += VT<T>::conj_mul_im(x, y);
      const T ys = VT<T>::scale(scale, y);
      v0[r] = (acc == 0.0) ? ys : VT<T>::add(VT<T>::scale(acc, v0[r]), ys);
    }
  }
  block_sum<2>(pr);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = pr[0];
    part[2 * blockIdx.x + 1] = pr[1];
  }
}

// h[q] += sum over the block's upper-half terms of c * v1[row r[q] shifted by the term]:
// every lane reads the term (row shift and coefficient index) at the same address, kColBatch
// terms per batch of loads.
template <typename T, bool GC>
__device__ __forceinline__ int64_t rb_shift(int64_t r, int64_t delta) {
  return GC ? (int64_t)((uint64_t)r ^ (uint64_t)delta) : r + delta;
}

template <typename T, bool GC, int P>
__device__ __forceinline__ void rb_upper_terms(const SplitView &sv, uint32_t ib, const T *__restrict__ v1,
                                               const int64_t (&r)[P], T (&h)[P]) {
  const double2 *cf = reinterpret_cast<const double2 *>(sv.coef);
  const uint32_t e0 = __ldg(sv.hi_ptr + ib), e1 = __ldg(sv.hi_ptr + ib + 1);
  uint32_t e = e0;
  for (; e + kColBatch <= e1; e += kColBatch) {
    HiEnt hh[kColBatch];
    T w[kColBatch][P];
#pragma unroll
    for (int b = 0; b < kColBatch; b++) hh[b] = sv.hi_ent[e + b];
#pragma unroll
    for (int b = 0; b < kColBatch; b++)
#pragma unroll
      for (int q = 0; q < P; q++) w[b][q] = v1[rb_shift<T, GC>(r[q], hh[b].delta)];
#pragma unroll
    for (int b = 0; b < kColBatch; b++) {
      const double2 cw = __ldg(cf + hh[b].k);
#pragma unroll
      for (int q = 0; q < P; q++) h[q] = VT<T>::add(h[q], VT<T>::cmul_re_im(cw.x, cw.y, w[b][q]));
    }
  }
  for (; e < e1; e++) {
    const HiEnt hh = sv.hi_ent[e];
    const double2 cw = __ldg(cf + hh.k);
#pragma unroll
    for (int q = 0; q < P; q++) h[q] = VT<T>::add(h[q], VT<T>::cmul_re_im(cw.x, cw.y, v1[rb_shift<T, GC>(r[q], hh.delta)]));
  }
}

// Column pass: warp tasks (block, 32 * P positions: lane l owns l + 32 q, q < P), class by
// class, chunk by chunk; cl_task holds the task offsets of each class for this chunk size.
template <typename T, bool GC, int P>
__global__ void __launch_bounds__(kColThreads) rb_col_kernel(RBArgs p, const int64_t *__restrict__ cl_task, SplitView sv,
                                                            const T *__restrict__ v1, T *__restrict__ v0,
                                                            const double *__restrict__ coef, double *__restrict__ part) {
  constexpr int CH = 32 * P;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t)((blockIdx.x * (unsigned)kColThreads + threadIdx.x) >> 5);
  const int64_t nwarps = (int64_t)(gridDim.x * (unsigned)kColThreads) >> 5;
  const int64_t ntask = cl_task[p.nclass];
  const double scale = coef[1];
  double pr[2] = {0.0, 0.0};
  int g = 0;
  for (int64_t t = warp; t < ntask; t += nwarps) {
    while (t >= cl_task[g + 1]) g++;   // tasks only move forward within a warp
    const int64_t tt = t - cl_task[g];
    const int nb = p.cl_nblk[g];
    const int c = (int)(tt / nb), bj = (int)(tt - (int64_t)c * nb);
    const int bidx = p.cl_boff[g] + bj;
    const uint32_t ib = p.cb_ib[bidx];
    const int64_t start = p.cb_start[bidx];
    const int n = p.cb_n[bidx];
    int64_t r[P];
    bool ok[P];
#pragma unroll
    for (int q = 0; q < P; q++) {
      const int a = c * CH + lane + 32 * q;
      ok[q] = a < n;
      r[q] = start + (ok[q] ? a : 0);  // lanes past the block's end read its first position and discard it
    }
    T h[P];
#pragma unroll
    for (int q = 0; q < P; q++) h[q] = VT<T>::zero();
    rb_upper_terms<T, GC, P>(sv, ib, v1, r, h);
#pragma unroll
    for (int q = 0; q < P; q++)
      if (ok[q]) {
        const T x = v1[r[q]];
        pr[0] += VT<T>::conj_mul_re(x, h[q]);
        pr[1] += VT<T>::conj_mul_im(x, h[q]);
        v0[r[q]] = VT<T>::add(v0[r[q]], VT<T>::scale(scale, h[q]));
      }
  }
  block_sum<2>(pr);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = pr[0];
    part[2 * blockIdx.x + 1] = pr[1];
  }
}

constexpr int kSpinThreads = 1024;
constexpr int kSpinRow2 = 103168;   // shared-memory offset of the second block (>= (12880 + 16) * 8)
constexpr int kSpinGenMax = 64;     // crossing terms of the fast row pass

struct SpinRowArgs {
  int ntask;
  const int64_t *t_start;   // [2 * ntask] first rows of the two blocks (second -1: one block)
  const uint32_t *t_ib;     // [2 * ntask] their upper halves
  const int *t_cls;         // [ntask] class
  const int *c_n;           // per class: positions (block size)
  const int *c_groups;      // slot groups per warp in the class's table
  const int *c_uoff;        // offset of the class's lower halves in unrank
  const int64_t *c_gat;     // offset of the class's table in gat (16-byte units)
  const int *c_ws;          // offset of the class's slot counts in wslots
  const uint4 *gat;
  const uint8_t *wslots;
  const uint32_t *unrank;
  double t_lo;              // magnitude of every lower-half term
  int lo_bits;
  uint64_t lo_mask;
  const uint16_t *xt;       // per class and lower site j: position of ia ^ (1 << j) in its class
  const int64_t *c_xt;      // per class: offset of its [lo_bits][n] part of xt
  const int8_t *g_xbit;     // per crossing term: its single lower-half flip bit (-1: several)
};

__device__ __forceinline__ double rb_flip(double x, uint32_t sg) {
  return __hiloint2double(__double2hiint(x) ^ (int)sg, __double2loint(x));
}

// A crossing term that acts on rows of a staged block, prepared once per block: it acts on
// the row of lower half ia iff (ia & cm) == cv; the source row is src + xt[xt_off + position]
// (one lower-half flip bit) or src + list_2_1[ia ^ flo] - 2; its coefficient is c times
// (-1)^popcount(ia & sm).
struct XRec {
  int64_t src, xt_off;   // xt_off < 0: the source position comes from list_2_1
  double c;
  uint32_t cm, cv, sm, flo;
};

// Fast row pass: v0 = acc * v0 + scale * (diagonal + lower-half + crossing terms) v1 for two
// blocks of one class at a time; part[blockIdx] = sum of v1 . (...) v1 over the CTA's blocks.
// The gathers of the lower-half terms come first (one sweep over the columns); the crossing
// terms follow term by term over the thread's columns (their fields read once per term), each
// adding into the v0 element the thread has just written.
__global__ void __launch_bounds__(kSpinThreads, 1) spin_row_kernel(SpinRowArgs a, const BitTerm *__restrict__ gterms,
                                                                  int ngen, const uint32_t *__restrict__ l21,
                                                                  const uint32_t *__restrict__ l22,
                                                                  const double *__restrict__ diag,
                                                                  const double *__restrict__ v1,
                                                                  double *__restrict__ v0,
                                                                  const double *__restrict__ coef,
                                                                  double *__restrict__ part) {
  extern __shared__ __align__(128) double srows[];  // block 0 at 0, block 1 at kSpinRow2
  double *row1 = srows + kSpinRow2 / 8;
  __shared__ XRec s_x[2][kSpinGenMax];
  __shared__ int s_nact[2];
  const double acc = coef[0], scale = coef[1];
  const int tid = threadIdx.x, lane = tid & 31;
  const uint32_t sm0 = smem_u32(srows), sm1 = sm0 + kSpinRow2;
  const char *rb = reinterpret_cast<const char *>(srows);
  const uint64_t hi_mask = ~a.lo_mask;
  double pr = 0.0;
  for (int t = blockIdx.x; t < a.ntask; t += gridDim.x) {
    const int cls = a.t_cls[t];
    const int n = a.c_n[cls], npad = (n + 31) & ~31, groups = a.c_groups[cls];
    const int64_t s0 = a.t_start[2 * t], s1r = a.t_start[2 * t + 1];
    const bool two = s1r >= 0;
    const int64_t s1 = two ? s1r : s0;
    const uint64_t hi0 = (uint64_t)a.t_ib[2 * t] << a.lo_bits;
    const uint64_t hi1 = two ? ((uint64_t)a.t_ib[2 * t + 1] << a.lo_bits) : hi0;
    __syncthreads();  // the previous blocks and term lists are no longer read
    for (int i = tid; i < n; i += kSpinThreads) {
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sm0 + 8 * i), "l"(v1 + s0 + i) : "memory");
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sm1 + 8 * i), "l"(v1 + s1 + i) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    if (tid < 16) {  // zero words after each block (one per bank pair): the empty slots read them
      srows[n + tid] = 0.0;
      row1[n + tid] = 0.0;
    }
    if (tid < 64) {  // crossing terms whose upper-half condition block w meets (warp w)
      const int w = tid >> 5;
      const uint64_t hi = w ? hi1 : hi0;
      int m = 0;
      for (int k0 = 0; k0 < ngen; k0 += 32) {
        const int k = k0 + lane;
        bool on = false;
        XRec x{};
        if (k < ngen) {
          const BitTerm t = gterms[k];
          on = (hi & t.cm) == (t.cv & hi_mask);
          if (on) {
            const uint32_t b1 = __ldg(l22 + ((hi ^ t.flip) >> a.lo_bits));
            on = b1 != 0u;
            const int xb = a.g_xbit[k];
            x.src = (int64_t)b1 - 1;
            x.xt_off = (xb >= 0) ? a.c_xt[cls] + (int64_t)xb * n : -1;
            x.c = (__popcll(hi & t.sm) & 1) ? -t.re : t.re;
            x.cm = (uint32_t)(t.cm & a.lo_mask);
            x.cv = (uint32_t)(t.cv & a.lo_mask);
            x.sm = (uint32_t)(t.sm & a.lo_mask);
            x.flo = (uint32_t)(t.flip & a.lo_mask);
          }
        }
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, on);
        if (on) s_x[w][m + __popc(bal & ((1u << lane) - 1u))] = x;
        m += __popc(bal);
      }
      if (lane == 0) s_nact[w] = m;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    const uint4 *gk = a.gat + a.c_gat[cls];
    const uint8_t *wk = a.wslots + a.c_ws[cls];
    for (int p = tid; p < npad; p += kSpinThreads) {
      const int w = p >> 5, ns = wk[w];
      const uint4 *gp = gk + ((int64_t)w * groups) * 32 + lane;
      const int pc = (p < n) ? p : n - 1;
      const double d0 = __ldg(diag + s0 + pc), d1 = __ldg(diag + s1 + pc);
      const double y0old = (acc != 0.0) ? __ldcs(v0 + s0 + pc) : 0.0;
      const double y1old = (acc != 0.0 && two) ? __ldcs(v0 + s1 + pc) : 0.0;
      double g0 = 0.0, g1 = 0.0;
      auto gather2 = [&](uint32_t r) {
        const uint32_t o0 = (r << 3) & 0x3FFF8u, o1 = (r >> 13) & 0x3FFF8u;
        const uint32_t sg0 = r << 16;
        const double *x0 = reinterpret_cast<const double *>(rb + o0);
        const double *x1 = reinterpret_cast<const double *>(rb + o1);
        g0 += rb_flip(x0[0], sg0 & 0x80000000u);
        g1 += rb_flip(x0[kSpinRow2 / 8], sg0 & 0x80000000u);
        g0 += rb_flip(x1[0], r & 0x80000000u);
        g1 += rb_flip(x1[kSpinRow2 / 8], r & 0x80000000u);
      };
      for (int g = 0; 8 * g < ns; g++) {
        const uint4 e = __ldg(gp + g * 32);
        gather2(e.x);
        if (8 * g + 2 < ns) gather2(e.y);
        if (8 * g + 4 < ns) gather2(e.z);
        if (8 * g + 6 < ns) gather2(e.w);
      }
      if (p < n) {
        const double x0 = srows[p];
        const double y0 = d0 * x0 + a.t_lo * g0;
        v0[s0 + p] = (acc == 0.0) ? scale * y0 : acc * y0old + scale * y0;
        pr += x0 * y0;
        if (two) {
          const double x1 = row1[p];
          const double y1 = d1 * x1 + a.t_lo * g1;
          v0[s1 + p] = (acc == 0.0) ? scale * y1 : acc * y1old + scale * y1;
          pr += x1 * y1;
        }
      }
    }
    // crossing terms: four of the thread's columns at a time, the block's terms one by one with
    // every load of a term issued before its first use, one update of each v0 element
    const uint32_t *un = a.unrank + a.c_uoff[cls];
    constexpr int U = 4;
    for (int w = 0; w < (two ? 2 : 1); w++) {
      const int64_t sw = w ? s1 : s0;
      const double *xw = w ? row1 : srows;
      const int nact = s_nact[w];
      if (nact == 0) continue;
      for (int p0 = tid; p0 < n; p0 += U * kSpinThreads) {
        uint32_t ia[U];
        double hx[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const int p = p0 + u * kSpinThreads;
          ia[u] = (p < n) ? __ldg(un + p) : 0u;
          hx[u] = 0.0;
        }
        for (int i = 0; i < nact; i++) {
          const XRec x = s_x[w][i];
          bool on[U];
          int64_t j[U];
#pragma unroll
          for (int u = 0; u < U; u++) {
            const int p = p0 + u * kSpinThreads;
            on[u] = (p < n) && (ia[u] & x.cm) == x.cv;
            j[u] = x.src;
            if (on[u]) {
              if (x.xt_off >= 0) {
                j[u] += __ldg(a.xt + x.xt_off + p);
              } else {
                const uint32_t a1 = __ldg(l21 + (ia[u] ^ x.flo));
                on[u] = a1 != 0u;
                j[u] += (int64_t)a1 - 2;
              }
            }
          }
#pragma unroll
          for (int u = 0; u < U; u++)
            if (on[u]) {
              const double vv = __ldg(v1 + j[u]);
              hx[u] += (__popc(ia[u] & x.sm) & 1) ? -x.c * vv : x.c * vv;
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
          const int p = p0 + u * kSpinThreads;
          if (p < n && hx[u] != 0.0) {
            v0[sw + p] += scale * hx[u];
            pr += xw[p] * hx[u];
          }
        }
      }
    }
  }
  double v[2] = {pr, 0.0};
  block_sum<2>(v);
  if (tid == 0) {
    part[2 * blockIdx.x] = v[0];
    part[2 * blockIdx.x + 1] = 0.0;
  }
}

uint64_t binom_rb(int n, int k) {
  if (k < 0 || k > n) return 0;
  uint64_t r = 1;
  for (int i = 1; i <= k; i++) r = r * (uint64_t)(n - k + i) / (uint64_t)i;
  return r;
}

}  // namespace

struct RowBlockPlan {
  RBArgs args{};
  std::vector<void *> allocs;
  int grid_row[2] = {0, 0};     // real, complex (0: the block does not fit in shared memory)
  size_t smem_row[2] = {0, 0};
  int grid_col = 0;
  const int64_t *cl_task[2] = {nullptr, nullptr};  // column-pass task offsets per class: 128 / 64 positions
  SpinRowArgs fast{};           // fast row pass (real vectors), when grid_fast > 0
  int grid_fast = 0;
  size_t smem_fast = 0;
  double *part = nullptr;       // 2 * (max(grid_row, grid_fast) + grid_col) doubles
};

void rb_plan_free(RowBlockPlan *p) {
  if (!p) return;
  for (void *q : p->allocs) cudaFree(q);
  delete p;
}

namespace {
template <typename V>
int rb_upload(RowBlockPlan *p, const std::vector<V> &h, const V **d, std::string *err) {
  void *q = nullptr;
  const size_t bytes = h.empty() ? 16 : sizeof(V) * h.size();
  if (cudaMalloc(&q, bytes) != cudaSuccess) {
    *err = "row-block plan: device allocation failed";
    return -1;
  }
  p->allocs.push_back(q);
  if (!h.empty() && cudaMemcpy(q, h.data(), sizeof(V) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    *err = "row-block plan: copy failed";
    return -1;
  }
  *d = (const V *)q;
  return 0;
}

template <typename T, bool GC>
int rb_set_smem(size_t bytes) {
  return raise_smem_limit((const void *)rb_row_kernel<T, GC>, bytes) == cudaSuccess
             ? 0
             : -1;
}
}  // namespace

int rb_plan_build(Sector *s, std::string *err) {
  s->rb = nullptr;
  const Model &m = s->model;
  const bool spin = m.calc_model == kSpin && !m.general_spin && !s->gc;
  const bool gc = s->gc && (m.calc_model == kHubbardGC || (m.calc_model == kSpinGC && !m.general_spin));
  if (!spin && !gc) return 0;
  if (!s->split.lo_ptr || s->split.ngen > kRowTermMax || s->lo_bits > 20 || s->lo_bits < 1) return 0;
  const uint64_t nh = s->sdim;
  std::vector<uint32_t> blk_ib, unrank;
  std::vector<int64_t> blk_start;
  std::vector<int> blk_n, blk_uoff, blk_key;
  int nkey = 1;
  if (gc) {
    const int n = 1 << s->lo_bits;
    for (uint64_t ib = 0; ib < nh; ib++) {
      blk_ib.push_back((uint32_t)ib);
      blk_start.push_back((int64_t)(ib << s->lo_bits));
      blk_n.push_back(n);
      blk_uoff.push_back(0);
      blk_key.push_back(0);
    }
  } else {
    // lower halves by popcount, in increasing order (the order of a block's rows)
    const int L = s->lo_bits;
    nkey = L + 1;
    std::vector<int> key_off(L + 2, 0);
    std::vector<std::vector<uint32_t>> by_pop(L + 1);
    for (uint32_t ia = 0; ia < (1u << L); ia++) by_pop[__builtin_popcount(ia)].push_back(ia);
    for (int k = 0; k <= L; k++) {
      key_off[k] = (int)unrank.size();
      unrank.insert(unrank.end(), by_pop[k].begin(), by_pop[k].end());
    }
    // check the block layout against HPhi's lists: start = list_2_2 - 1, position = list_2_1 - 2
    std::vector<uint32_t> l21(s->ihfbit), l22(nh);
    if (cudaMemcpy(l21.data(), s->d_list_2_1, sizeof(uint32_t) * s->ihfbit, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(l22.data(), s->d_list_2_2, sizeof(uint32_t) * nh, cudaMemcpyDeviceToHost) != cudaSuccess) {
      *err = "row-block plan: list copy failed";
      return -1;
    }
    int64_t row = 0;
    for (uint64_t ib = 0; ib < nh; ib++) {
      const int k = m.ne - __builtin_popcountll(ib);
      if (k < 0 || k > L) continue;
      const int n = (int)binom_rb(L, k);
      if (n == 0) continue;
      if ((int64_t)l22[ib] - 1 != row) return 0;  // not the layout this plan assumes
      blk_ib.push_back((uint32_t)ib);
      blk_start.push_back(row);
      blk_n.push_back(n);
      blk_uoff.push_back(key_off[k]);
      blk_key.push_back(k);
      row += n;
    }
    if (row != s->dim) return 0;
    for (int k = 0; k <= L; k++)
      for (size_t r = 0; r < by_pop[k].size(); r++)
        if (l21[by_pop[k][r]] != 0 && l21[by_pop[k][r]] != (uint32_t)r + 2u) return 0;
    nkey = L + 1;
  }
  const int nblk = (int)blk_ib.size();
  if (nblk == 0) return 0;
  int max_n = 0;
  for (int n : blk_n) max_n = std::max(max_n, n);
  // row pass order: largest blocks first
  std::vector<int> ord(nblk);
  for (int i = 0; i < nblk; i++) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return blk_n[a] > blk_n[b]; });
  std::vector<uint32_t> rb_ib(nblk);
  std::vector<int64_t> rb_start(nblk);
  std::vector<int> rb_n(nblk), rb_uoff(nblk);
  for (int i = 0; i < nblk; i++) {
    rb_ib[i] = blk_ib[ord[i]];
    rb_start[i] = blk_start[ord[i]];
    rb_n[i] = blk_n[ord[i]];
    rb_uoff[i] = blk_uoff[ord[i]];
  }
  // column pass: blocks grouped by class (upper-half terms keep the class), tasks class by
  // class, chunk by chunk, block by block
  std::vector<std::vector<int>> cls(nkey);
  for (int i = 0; i < nblk; i++) cls[blk_key[i]].push_back(i);
  std::vector<int64_t> cl_task4(1, 0), cl_task2(1, 0);
  std::vector<int> cl_nblk, cl_boff;
  std::vector<uint32_t> cb_ib;
  std::vector<int64_t> cb_start;
  std::vector<int> cb_n, cb_key;
  for (int k = 0; k < nkey; k++) {
    if (cls[k].empty()) continue;
    const int n = blk_n[cls[k][0]];
    cl_boff.push_back((int)cb_ib.size());
    cl_nblk.push_back((int)cls[k].size());
    for (int i : cls[k]) {
      cb_ib.push_back(blk_ib[i]);
      cb_start.push_back(blk_start[i]);
      cb_n.push_back(blk_n[i]);
      cb_key.push_back(blk_key[i]);
    }
    cl_task4.push_back(cl_task4.back() + (int64_t)((n + 127) / 128) * (int64_t)cls[k].size());
    cl_task2.push_back(cl_task2.back() + (int64_t)((n + 63) / 64) * (int64_t)cls[k].size());
  }
  RowBlockPlan *p = new RowBlockPlan();
  RBArgs &a = p->args;
  a.nblk = nblk;
  a.nclass = (int)cl_nblk.size();
  a.lo_bits = s->lo_bits;
  a.lo_mask = s->ihfbit - 1;
  a.lo_base = gc ? 0 : 2;
  auto fail = [&]() { rb_plan_free(p); return -1; };
  if (rb_upload(p, rb_ib, &a.rb_ib, err) || rb_upload(p, rb_start, &a.rb_start, err) || rb_upload(p, rb_n, &a.rb_n, err) ||
      rb_upload(p, rb_uoff, &a.rb_uoff, err) || rb_upload(p, unrank, &a.unrank, err) ||
      rb_upload(p, cl_task4, &p->cl_task[0], err) || rb_upload(p, cl_task2, &p->cl_task[1], err) ||
      rb_upload(p, cl_nblk, &a.cl_nblk, err) ||
      rb_upload(p, cl_boff, &a.cl_boff, err) || rb_upload(p, cb_ib, &a.cb_ib, err) ||
      rb_upload(p, cb_start, &a.cb_start, err) || rb_upload(p, cb_n, &a.cb_n, err) ||
      rb_upload(p, cb_key, &a.cb_key, err))
    return fail();
  // fast row pass: canonical Spin, every lower-half term real and of one magnitude
  if (!gc && s->split.ngen <= kSpinGenMax && !std::getenv("HPHI_B200_RB_SIMPLE")) {
    const uint64_t lo_mask = s->ihfbit - 1;
    const int L = s->lo_bits;
    std::vector<const BitTerm *> lo_terms;
    for (const BitTerm &t : m.offdiag)
      if (((t.cm | t.flip | t.sm) & ~lo_mask) == 0) lo_terms.push_back(&t);
    double tlo = -1.0;
    bool ok = !lo_terms.empty();
    for (const BitTerm *t : lo_terms) {
      if (t->im != 0.0 || t->re == 0.0) ok = false;
      if (tlo < 0.0) tlo = std::fabs(t->re);
      else if (std::fabs(t->re) != tlo) ok = false;
    }
    for (int n : blk_n) ok = ok && (n + 16 <= kSpinRow2 / 8);
    if (ok) {
      std::vector<int> pos_of(1u << L, 0);
      std::vector<std::vector<uint32_t>> by_pop(L + 1);
      for (uint32_t ia = 0; ia < (1u << L); ia++) {
        pos_of[ia] = (int)by_pop[__builtin_popcount(ia)].size();
        by_pop[__builtin_popcount(ia)].push_back(ia);
      }
      std::vector<int> c_n(L + 1, 0), c_groups(L + 1, 1), c_uoff(L + 1, 0), c_ws(L + 1, 0);
      std::vector<int64_t> c_gat(L + 1, 0);
      std::vector<uint4> gat_all;
      std::vector<uint8_t> ws_all;
      std::vector<char> used(L + 1, 0);
      for (int k : blk_key) used[k] = 1;
      int key_off = 0;
      for (int k = 0; k <= L && ok; k++) {
        c_uoff[k] = key_off;
        key_off += (int)by_pop[k].size();
        if (!used[k]) continue;
        const int n = (int)by_pop[k].size();
        std::vector<std::vector<uint32_t>> rows(n);
        for (int q = 0; q < n && ok; q++) {
          const uint32_t ia = by_pop[k][q];
          for (const BitTerm *t : lo_terms) {
            if ((ia & t->cm) != t->cv) continue;
            const uint32_t src = ia ^ (uint32_t)t->flip;
            if (__builtin_popcount(src) != k) { ok = false; break; }
            const bool neg = (t->re < 0.0) != ((__builtin_popcountll((uint64_t)ia & t->sm) & 1) != 0);
            rows[q].push_back((uint32_t)pos_of[src] | (neg ? 0x10000u : 0u));
          }
          if (rows[q].size() > 255) ok = false;
        }
        if (!ok) break;
        std::vector<uint32_t> g;
        std::vector<uint8_t> ws;
        int groups = 1;
        build_gather_table(rows, n, &g, &ws, &groups);
        c_n[k] = n;
        c_groups[k] = groups;
        c_gat[k] = (int64_t)gat_all.size();
        c_ws[k] = (int)ws_all.size();
        for (size_t i = 0; i + 3 < g.size(); i += 4) gat_all.push_back(make_uint4(g[i], g[i + 1], g[i + 2], g[i + 3]));
        ws_all.insert(ws_all.end(), ws.begin(), ws.end());
      }
      if (ok) {
        // tasks: pairs of blocks of one class.  Blocks whose upper halves differ only in bits
        // that crossing terms flip read each other's rows, so they are grouped (by the other
        // upper bits) and a group's tasks run together: the source blocks of the crossing terms
        // are then read while they are in L2.
        std::vector<BitTerm> gen_h0(s->split.ngen);
        if (s->split.ngen &&
            cudaMemcpy(gen_h0.data(), s->split.gen, sizeof(BitTerm) * gen_h0.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
          *err = "row-block plan: term copy failed";
          return fail();
        }
        uint64_t xhi = 0;
        for (const BitTerm &t : gen_h0) xhi |= t.flip >> L;
        std::vector<int> order_b(nblk);
        for (int i = 0; i < nblk; i++) order_b[i] = i;
        std::stable_sort(order_b.begin(), order_b.end(), [&](int x, int y) {
          const uint64_t gx = blk_ib[x] & ~xhi, gy = blk_ib[y] & ~xhi;
          if (gx != gy) return gx < gy;
          if (blk_key[x] != blk_key[y]) return blk_key[x] < blk_key[y];
          return blk_ib[x] < blk_ib[y];
        });
        std::vector<int64_t> t_start;
        std::vector<uint32_t> t_ib;
        std::vector<int> t_cls;
        for (size_t i = 0; i < order_b.size();) {
          const int b0 = order_b[i];
          const bool two = i + 1 < order_b.size() && blk_key[order_b[i + 1]] == blk_key[b0] &&
                           (blk_ib[order_b[i + 1]] & ~xhi) == (blk_ib[b0] & ~xhi);
          const int b1 = two ? order_b[i + 1] : b0;
          t_start.push_back(blk_start[b0]);
          t_start.push_back(two ? blk_start[b1] : -1);
          t_ib.push_back(blk_ib[b0]);
          t_ib.push_back(blk_ib[b1]);
          t_cls.push_back(blk_key[b0]);
          i += two ? 2 : 1;
        }
        // crossing terms: single lower-half flip bit -> per class and site position tables
        std::vector<BitTerm> gen_h(s->split.ngen);
        if (s->split.ngen &&
            cudaMemcpy(gen_h.data(), s->split.gen, sizeof(BitTerm) * gen_h.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
          *err = "row-block plan: term copy failed";
          return fail();
        }
        std::vector<int8_t> g_xbit(std::max<size_t>(1, gen_h.size()), -1);
        for (size_t q = 0; q < gen_h.size(); q++) {
          const uint64_t fl = gen_h[q].flip & lo_mask;
          if (fl && (fl & (fl - 1)) == 0) g_xbit[q] = (int8_t)__builtin_ctzll(fl);
        }
        std::vector<int64_t> c_xt(L + 1, 0);
        std::vector<uint16_t> xt;
        for (int k = 0; k <= L; k++) {
          if (!used[k]) continue;
          c_xt[k] = (int64_t)xt.size();
          for (int j = 0; j < L; j++)
            for (uint32_t ia : by_pop[k]) xt.push_back((uint16_t)pos_of[ia ^ (1u << j)]);
        }
        SpinRowArgs &f = p->fast;
        if (rb_upload(p, g_xbit, &f.g_xbit, err) || rb_upload(p, c_xt, &f.c_xt, err) || rb_upload(p, xt, &f.xt, err))
          return fail();
        f.ntask = (int)t_cls.size();
        f.t_lo = tlo;
        f.lo_bits = L;
        f.lo_mask = lo_mask;
        f.unrank = a.unrank;
        if (rb_upload(p, t_start, &f.t_start, err) || rb_upload(p, t_ib, &f.t_ib, err) ||
            rb_upload(p, t_cls, &f.t_cls, err) || rb_upload(p, c_n, &f.c_n, err) ||
            rb_upload(p, c_groups, &f.c_groups, err) || rb_upload(p, c_uoff, &f.c_uoff, err) ||
            rb_upload(p, c_gat, &f.c_gat, err) || rb_upload(p, c_ws, &f.c_ws, err) ||
            rb_upload(p, gat_all, &f.gat, err) || rb_upload(p, ws_all, &f.wslots, err))
          return fail();
        p->smem_fast = 2 * (size_t)kSpinRow2;
        if (raise_smem_limit((const void *)spin_row_kernel, p->smem_fast) == cudaSuccess)
          p->grid_fast = std::max(1, std::min(f.ntask, s->num_sms));
      }
    }
  }
  const size_t tbytes = sizeof(BitTerm) * (size_t)s->split.ngen;
  const size_t need[2] = {tbytes + sizeof(double) * (size_t)max_n, tbytes + sizeof(cplx) * (size_t)max_n};
  for (int vt = 0; vt < 2; vt++) {
    if (need[vt] > kSmemLimit) continue;
    int rc;
    const void *fn;
    if (vt == 0) {
      rc = gc ? rb_set_smem<double, true>(need[0]) : rb_set_smem<double, false>(need[0]);
      fn = gc ? (const void *)rb_row_kernel<double, true> : (const void *)rb_row_kernel<double, false>;
    } else {
      rc = gc ? rb_set_smem<cplx, true>(need[1]) : rb_set_smem<cplx, false>(need[1]);
      fn = gc ? (const void *)rb_row_kernel<cplx, true> : (const void *)rb_row_kernel<cplx, false>;
    }
    if (rc != 0) continue;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kRowThreads, need[vt]) != cudaSuccess || per_sm < 1)
      continue;
    p->smem_row[vt] = need[vt];
    p->grid_row[vt] = std::max(1, std::min(nblk, per_sm * s->num_sms));
  }
  if (p->grid_row[0] == 0 && p->grid_row[1] == 0) {
    rb_plan_free(p);
    return 0;
  }
  int col_per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&col_per_sm, gc ? (const void *)rb_col_kernel<cplx, true, 2>
                                                                : (const void *)rb_col_kernel<cplx, false, 2>,
                                                kColThreads, 0);
  p->grid_col = std::max(1, std::max(1, col_per_sm) * s->num_sms);
  const int rows_max = std::max(std::max(p->grid_row[0], p->grid_row[1]), p->grid_fast);
  if (cudaMalloc(&p->part, sizeof(double) * 2 * (size_t)(rows_max + p->grid_col)) != cudaSuccess) {
    *err = "row-block plan: device allocation failed";
    return fail();
  }
  p->allocs.push_back(p->part);
  cudaGetLastError();
  s->rb = p;
  return 0;
}

bool rb_applies(const Sector *s, VecType vt) {
  return s->rb && (s->rb->grid_row[vt == kReal64 ? 0 : 1] > 0 || (vt == kReal64 && s->rb->grid_fast > 0));
}

size_t rb_scratch_doubles(const Sector *s) {
  const RowBlockPlan *p = s->rb;
  return 2 * (size_t)(std::max(std::max(p->grid_row[0], p->grid_row[1]), p->grid_fast) + p->grid_col);
}

int rb_hv_launch_scratch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                         double *d_part) {
  RowBlockPlan *p = s->rb;
  const int iv = (vt == kReal64) ? 0 : 1;
  const bool fast = (vt == kReal64) && p->grid_fast > 0;
  const int gr = fast ? p->grid_fast : p->grid_row[iv], gcol = p->grid_col;
  const SplitView sv = split_view(s->split);
  double *pc = d_part + 2 * (size_t)gr;
  if (fast) {
    spin_row_kernel<<<gr, kSpinThreads, p->smem_fast, s->stream>>>(p->fast, s->split.gen, s->split.ngen,
                                                                   s->d_list_2_1, s->d_list_2_2, s->d_diag,
                                                                   (const double *)d_v1, (double *)d_v0, d_coef, d_part);
    rb_col_kernel<double, false, 4><<<gcol, kColThreads, 0, s->stream>>>(p->args, p->cl_task[0], sv,
                                                                         (const double *)d_v1, (double *)d_v0, d_coef, pc);
    finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(d_part, gr + gcol, d_out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error(std::string("row-block kernels: launch failed: ") + cudaGetErrorString(e));
      return -1;
    }
    return 0;
  }
#define HPHI_RB_LAUNCH(T, GC, P)                                                                                        \
  do {                                                                                                               \
    rb_row_kernel<T, GC><<<gr, kRowThreads, p->smem_row[iv], s->stream>>>(                                           \
        p->args, sv, s->split.gen, s->split.ngen, s->d_list_2_1, s->d_list_2_2, s->d_diag, (const T *)d_v1, (T *)d_v0, \
        d_coef, d_part);                                                                                             \
    rb_col_kernel<T, GC, P><<<gcol, kColThreads, 0, s->stream>>>(p->args, p->cl_task[P == 4 ? 0 : 1], sv,              \
                                                              (const T *)d_v1, (T *)d_v0, d_coef, pc);                \
  } while (0)
  if (vt == kReal64) {
    if (s->gc) HPHI_RB_LAUNCH(double, true, 4);
    else HPHI_RB_LAUNCH(double, false, 4);
  } else {
    if (s->gc) HPHI_RB_LAUNCH(cplx, true, 2);
    else HPHI_RB_LAUNCH(cplx, false, 2);
  }
#undef HPHI_RB_LAUNCH
  finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(d_part, gr + gcol, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("row-block kernels: launch failed: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

int rb_hv_launch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out) {
  return rb_hv_launch_scratch(s, vt, d_v1, d_v0, d_coef, d_out, s->rb->part);
}

}  // namespace hphi
