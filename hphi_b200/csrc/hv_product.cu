// Product-layout kernel for canonical Hubbard Hamiltonians.
//
// Applies when every off-diagonal term is a spin-conserving single hop c+_{i s} c_{j s}
// (Trans terms, src/mltplyHubbard.c:174-209, element routine CisAjt,
// src/mltplyHubbardCore.c:305-347), Nsite <= 16 and both spin counts are fixed; diagonal
// terms of any kind are allowed (src/diagonalcalc.c).
//
// Native vector order.  The sector of HPhi (Nup up and Ndown down electrons) is the set
// of pairs (u, d) of N-bit occupations with popcount Nup and Ndown.  The native order
// stores it as a dense matrix
//   pos = rank(u) * C(N, Ndown) + rank(d),
// ranks among N-bit numbers of equal popcount in increasing order, in the species-first
// fermion basis (all up modes before all down modes).  That basis differs from HPhi's
// interleaved one (bit 2i + s) by the diagonal sign
//   sigma(c) = (-1)^#{(down at i, up at j) : i < j},
// applied by the boundary permutation; in it a hop's sign only counts occupied modes of its
// own species strictly between its two sites, so it is a property of u (up hops) or d
// (down hops) alone:
//   (H v)[u, d] = D(u, d) v[u, d] + sum_{down hops} c(d) v[u, d'] + sum_{up hops} c(u) v[u', d].
//
// Kernel: persistent CTAs take whole rows u from an atomic dispenser.  The row v1[u, :]
// (C(N, Ndown) elements) is staged in shared memory; down hops are gathers inside it driven
// by an ELL table ell_dn[slot][d] (source rank, coefficient index), read coalesced across
// the lanes that own consecutive d; up hops of the row (the same for every d) are staged in
// shared memory and applied as coalesced reads of the source rows v1[u', :]; the diagonal is
// rebuilt from per-species tables plus U * popcount(u & d) (or read when it has other
// cross-species terms).  Each row's <v1|H v1> contribution is reduced in the CTA and summed
// over rows in a fixed order afterwards, so results do not depend on scheduling.
//
// Two-pass form (real vectors, down hops of one magnitude |t|; the default there).  H v is
// split into a row pass (diagonal + down hops: every row is a gather inside itself) and a
// column pass (up hops: whole source rows).  The row pass stages two rows per CTA in shared
// memory and reads them through an edge-coloured gather table: within each slot of a warp,
// the 16 lanes of a half-warp hit 16 different shared-memory bank pairs, so every 8-byte
// gather takes the minimum two wavefronts; entries are 16-bit word indices with the hop's
// sign in bit 15, eight per lane in one 16-byte load issued a column block ahead, and empty
// slots point at zero words placed one per bank.  The column pass walks
// the matrix in column chunks (all rows of chunk 0, then chunk 1, ...) so the source rows of
// the chunk being processed stay in L2 while every row gathers its ~N/2 up-hop sources; a
// warp takes one row and 128 columns, its lanes hold the row's packed hop entries and
// broadcast them by shuffles, and every source row is read as two 512-byte warp loads.
// Both passes take their work by static striding (no dispenser) and keep per-CTA partial
// sums of <v1|H v1>, so the result is reproducible.
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
#include "tma.cuh"

namespace hphi {
namespace {

constexpr int kProdThreads = 512;
constexpr int kMaxUpWidth = 128;          // up hops of one row, staged in shared memory
constexpr uint32_t kEllNone = 0xFFFFFFFFu;

struct ProdArgs {
  int N, Uc, Dc;               // sites, rows (up configurations), columns (down configurations)
  int wd, wu;                  // ELL widths
  const uint16_t *rank;        // [2^N] position of an up configuration (its rank)
  const uint16_t *pos_dn;      // [2^N] position of a down configuration
  const uint16_t *unrank_up;   // [Uc]
  const uint16_t *unrank_dn;   // [Dc]
  const uint32_t *ell_dn;      // [wd][Dc]: source rank | coefficient index << 16
  const uint32_t *ell_up;      // [Uc][wu]
  const uint8_t *cnt_dn;       // [Dc] valid entries of each ELL column
  const uint8_t *wmax_dn;      // [ceil(Dc / 32)] largest count in each aligned block of 32 columns
  const double *utab;          // [17] u0 * k for k = 0..16 (cross_mode 0)
  const double2 *cf_dn, *cf_up;
  const double *du, *dd;       // diagonal terms of one species, by rank
  const double *usite;         // on-site U per site (cross_mode 1)
  double u0;                   // uniform on-site U (cross_mode 0)
  int cross_mode;              // 0: u0 * popc(u & d); 1: per-site U; 2: read dfull
  const double *dfull;         // [Uc * Dc] diagonal in native order (cross_mode 2)
  const int *order;            // [Uc] processing order of the rows
};

template <typename T> __device__ __forceinline__ T ldg_v(const T *p);
template <> __device__ __forceinline__ double ldg_v<double>(const double *p) { return __ldg(p); }
template <> __device__ __forceinline__ cplx ldg_v<cplx>(const cplx *p) {
  const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
  return cplx{v.x, v.y};
}

__device__ __forceinline__ int next_row(int *counter) {
  __shared__ int s_row;
  __syncthreads();
  if (threadIdx.x == 0) s_row = atomicAdd(counter, 1);
  __syncthreads();
  return s_row;
}

// The last CTA to leave resets the dispenser for the next launch.
__device__ __forceinline__ void retire(int *counter) {
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(counter + 1, 1) == (int)gridDim.x - 1) {
      counter[0] = 0;
      counter[1] = 0;
      __threadfence();
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kProdThreads, 2) prod_hv_kernel(ProdArgs a, const T *__restrict__ v1,
                                                                    T *__restrict__ v0,
                                                                    const double *__restrict__ coef,
                                                                    double *__restrict__ part, int *counter) {
  extern __shared__ unsigned char smem_raw[];
  T *row = reinterpret_cast<T *>(smem_raw);
  __shared__ uint32_t s_src[kMaxUpWidth];
  __shared__ double2 s_cf[kMaxUpWidth];
  __shared__ int s_nu;
  const double acc = coef[0], scale = coef[1];
  const int Dc = a.Dc;
  for (;;) {
    const int k_row = next_row(counter);
    if (k_row >= a.Uc) break;
    const int ua = a.order[k_row];
    const T *src = v1 + (int64_t)ua * Dc;
    for (int i = threadIdx.x; i < Dc; i += blockDim.x) row[i] = src[i];
    if (threadIdx.x == 0) {
      int n = 0;
      for (; n < a.wu; n++)
        if (a.ell_up[(int64_t)ua * a.wu + n] == kEllNone) break;
      s_nu = n;
    }
    for (int s = threadIdx.x; s < a.wu; s += blockDim.x) {
      const uint32_t e = a.ell_up[(int64_t)ua * a.wu + s];
      if (e != kEllNone) {
        s_src[s] = e & 0xFFFFu;
        s_cf[s] = a.cf_up[e >> 16];
      }
    }
    __syncthreads();
    const int nu = s_nu;
    const uint32_t u = a.unrank_up[ua];
    const double du = a.du[ua];
    double pr[2] = {0.0, 0.0};
    T *dst = v0 + (int64_t)ua * Dc;
    constexpr int CPT = 2;  // columns per thread per iteration
    for (int base = 0; base < Dc; base += CPT * (int)blockDim.x) {
      int da[CPT];
      bool ok[CPT];
      T y[CPT], x[CPT];
      int cnt[CPT], wmax = 0;
#pragma unroll
      for (int c = 0; c < CPT; c++) {
        const int d0 = base + c * (int)blockDim.x + (int)threadIdx.x;
        ok[c] = d0 < Dc;
        da[c] = ok[c] ? d0 : Dc - 1;
        x[c] = row[da[c]];
        double D;
        if (a.cross_mode == 2) {
          D = __ldg(a.dfull + (int64_t)ua * Dc + da[c]);
        } else {
          D = du + __ldg(a.dd + da[c]);
          const uint32_t ud = u & (uint32_t)__ldg(a.unrank_dn + da[c]);
          if (a.cross_mode == 0) D += __ldg(a.utab + __popc(ud));
          else for (uint32_t m = ud; m; m &= m - 1) D += __ldg(a.usite + (__ffs(m) - 1));
        }
        y[c] = VT<T>::scale(D, x[c]);
        cnt[c] = __ldg(a.cnt_dn + da[c]);
        // a warp's columns are the aligned block [base + c*blockDim + 32w, ... + 32)
        wmax = max(wmax, (int)__ldg(a.wmax_dn + ((base + c * (int)blockDim.x + (int)(threadIdx.x & ~31u)) >> 5)));
      }
      for (int s = 0; s < wmax; s += 4) {
        uint32_t e[CPT][4];
#pragma unroll
        for (int c = 0; c < CPT; c++)
#pragma unroll
          for (int k = 0; k < 4; k++)
            e[c][k] = (s + k < cnt[c]) ? __ldg(a.ell_dn + (int64_t)(s + k) * Dc + da[c]) : kEllNone;
#pragma unroll
        for (int c = 0; c < CPT; c++)
#pragma unroll
          for (int k = 0; k < 4; k++)
            if (e[c][k] != kEllNone) {
              const double2 cf = __ldg(a.cf_dn + (e[c][k] >> 16));
              y[c] = VT<T>::add(y[c], VT<T>::cmul_re_im(cf.x, cf.y, row[e[c][k] & 0xFFFFu]));
            }
      }
      constexpr int kS = (sizeof(T) > 8) ? 2 : 4;  // up hops per batch (registers: complex holds twice as much)
      for (int s = 0; s < nu; s += kS) {
        T v[kS][CPT];
#pragma unroll
        for (int k = 0; k < kS; k++) {
          const T *p = v1 + (int64_t)s_src[(s + k < nu) ? s + k : s] * Dc;
#pragma unroll
          for (int c = 0; c < CPT; c++) v[k][c] = (s + k < nu) ? ldg_v<T>(p + da[c]) : VT<T>::zero();
        }
#pragma unroll
        for (int k = 0; k < kS; k++)
          if (s + k < nu) {
            const double2 cf = s_cf[s + k];
#pragma unroll
            for (int c = 0; c < CPT; c++) y[c] = VT<T>::add(y[c], VT<T>::cmul_re_im(cf.x, cf.y, v[k][c]));
          }
      }
#pragma unroll
      for (int c = 0; c < CPT; c++)
        if (ok[c]) {
          pr[0] += VT<T>::conj_mul_re(x[c], y[c]);
          pr[1] += VT<T>::conj_mul_im(x[c], y[c]);
          const T yy = VT<T>::scale(scale, y[c]);
          dst[da[c]] = (acc == 0.0) ? yy : VT<T>::add(VT<T>::scale(acc, dst[da[c]]), yy);
        }
    }
    block_sum<2>(pr);
    if (threadIdx.x == 0) {
      part[2 * (int64_t)ua] = pr[0];
      part[2 * (int64_t)ua + 1] = pr[1];
    }
  }
  retire(counter);
}

constexpr int kDownThreads = 1024;            // row pass: one CTA per SM, two rows at a time
constexpr int kRow2Bytes = 103168;            // shared-memory offset of the second row (>= (12870 + 16) * 8)
constexpr int kUpThreads = 128;               // column pass
constexpr int kUpBatch = 8;                   // source loads in flight per thread
constexpr int kUpMinBlocks = 12;               // CTAs per SM (40 registers)
constexpr int kUpChunk = 2 * kUpThreads;      // columns per column-pass task (two per thread)

struct TwoPassArgs {
  int npad;                    // Dc rounded up to a multiple of 32
  int groups;                  // slot groups of 8 stored per warp (max over warps)
  const uint4 *gat;            // [npad / 32][groups][32 lanes] 8 entries: word | sign << 15
  const uint8_t *wslots;       // [npad / 32] slots of each warp's 32 columns
  double t_dn;                 // magnitude of every down hop
  double t_up;                 // magnitude of every up hop (up_uniform)
  int up_uniform;              // usrc carries the sign in bit 31 and ucf is unused
  const int *usrc;             // [Uc][wu] up-hop source rank
  const double *ucf;           // [Uc][wu] up-hop coefficient
  const uint8_t *nus;          // [Uc] up hops of each row
  const uint32_t *usrc16;      // [Uc][wu2] two up hops per word: rank | sign << 15 (16 bits each)
  int wu2;                     // words per row of usrc16 (0: no packed table)
};

__device__ __forceinline__ double flip_sign(double x, uint32_t sg) {
  return __hiloint2double(__double2hiint(x) ^ (int)sg, __double2loint(x));
}

// Row pass: v0[u, :] = acc * v0[u, :] + scale * (D + down hops) v1[u, :] for two rows at a time;
// part[blockIdx] = sum over the CTA's rows of v1 . (D + down) v1.  The two rows are staged
// by bulk asynchronous copies completing on an mbarrier (per-thread cp.async when the rows
// are not 16-byte aligned); a bounded wait that gives up makes the CTA's partial sum NaN.
// Gathers: each 16-bit table entry (word | sign << 15) serves both rows.
__global__ void __launch_bounds__(kDownThreads, 1) prod_down_kernel(ProdArgs a, TwoPassArgs b,
                                                                   const double *__restrict__ v1,
                                                                   double *__restrict__ v0,
                                                                   const double *__restrict__ coef,
                                                                   double *__restrict__ part) {
  extern __shared__ __align__(128) double rows[];  // row 0 at 0, row 1 at kRow2Bytes; each Dc + 16 words
  __shared__ uint64_t bar;
  double *row1 = rows + kRow2Bytes / 8;
  const double acc = coef[0], scale = coef[1];
  const int Dc = a.Dc, Uc = a.Uc;
  const int tid = threadIdx.x;
  double pr = 0.0;
  // rows arrive by bulk copies when they start on 16-byte boundaries and are whole 16-byte units
  const bool bulk = (Dc % 2 == 0) && ((uintptr_t)v1 % 16 == 0);
  const uint32_t sm0 = smem_u32(rows), sm1 = sm0 + kRow2Bytes;
  if (tid == 0) mbar_init(&bar, 1);
  mbar_fence_init();
  if (tid < 16) {  // zero words after each row (one per bank pair), never overwritten by the copies
    rows[Dc + tid] = 0.0;
    row1[Dc + tid] = 0.0;
  }
  uint32_t phase = 0;
  bool ok = true;
  for (int u0 = 2 * blockIdx.x; u0 < Uc; u0 += 2 * gridDim.x) {
    const bool two = u0 + 1 < Uc;
    __syncthreads();  // the previous rows are no longer read
    const double *s0 = v1 + (int64_t)u0 * Dc;
    const double *s1 = two ? s0 + Dc : s0;
    if (bulk) {
      if (tid == 0) {
        mbar_arrive_expect_tx(&bar, (uint32_t)(2 * Dc * 8));
        bulk_g2s(rows, s0, (uint32_t)(Dc * 8), &bar);
        bulk_g2s(row1, s1, (uint32_t)(Dc * 8), &bar);
      }
    } else {
      for (int i = tid; i < Dc; i += kDownThreads) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sm0 + 8 * i), "l"(s0 + i) : "memory");
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sm1 + 8 * i), "l"(s1 + i) : "memory");
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    // the next pair's rows toward L2 while this pair is processed (a hint, no completion)
    const int un = u0 + 2 * gridDim.x;
    if (bulk && tid < 2 && un + tid < Uc) {
      const double *pf = v1 + (int64_t)(un + tid) * Dc;
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(pf), "r"((uint32_t)(Dc * 8)) : "memory");
    }
    if (bulk) {
      const bool got = mbar_wait(&bar, phase);
      phase ^= 1;
      if (__syncthreads_or(!got)) {
        ok = false;
        mbar_wait(&bar, phase ^ 1);  // copies still in flight land before the CTA leaves (bounded)
        break;
      }
    } else {
      asm volatile("cp.async.wait_all;\n" ::: "memory");
      __syncthreads();
    }
    const int ua1 = two ? u0 + 1 : u0;
    const uint32_t uc0 = a.unrank_up[u0], uc1 = a.unrank_up[ua1];
    const double du0 = a.du[u0], du1 = a.du[ua1];
    const int lane = tid & 31;
    const double tdn = b.t_dn;
    const char *rb = reinterpret_cast<const char *>(rows);
    for (int p = tid; p < b.npad; p += kDownThreads) {
      const int w = p >> 5, ns = b.wslots[w];  // the same for the warp's 32 columns
      const uint4 *gp = b.gat + ((int64_t)w * b.groups) * 32 + lane;
      // per-column diagonal parts and the old v0, loaded before the gathers
      const int pc = (p < Dc) ? p : Dc - 1;
      const double ddp = (a.cross_mode == 2) ? 0.0 : __ldg(a.dd + pc);
      const uint32_t cdp = __ldg(a.unrank_dn + pc);
      double *o0 = v0 + (int64_t)u0 * Dc + pc;
      const double y0old = (acc != 0.0) ? __ldcs(o0) : 0.0;
      const double y1old = (acc != 0.0 && two) ? __ldcs(o0 + Dc) : 0.0;
      double g0 = 0.0, g1 = 0.0;
      // two 16-bit entries: word index (15 bits) | sign << 15; the sign is applied by flipping
      // the sign bit of the gathered value; every slot at or beyond the warp's count holds a
      // zero word, so only whole entry pairs are skipped
      auto gather2 = [&](uint32_t r) {
        const uint32_t o0 = (r << 3) & 0x3FFF8u, o1 = (r >> 13) & 0x3FFF8u;
        const uint32_t s0 = r << 16;  // sign of the low entry at bit 31 (the high entry's is there already)
        const double *x0 = reinterpret_cast<const double *>(rb + o0);
        const double *x1 = reinterpret_cast<const double *>(rb + o1);
        g0 += flip_sign(x0[0], s0 & 0x80000000u);
        g1 += flip_sign(x0[kRow2Bytes / 8], s0 & 0x80000000u);
        g0 += flip_sign(x1[0], r & 0x80000000u);
        g1 += flip_sign(x1[kRow2Bytes / 8], r & 0x80000000u);
      };
      for (int g = 0; 8 * g < ns; g++) {
        const uint4 e = __ldg(gp + g * 32);
        gather2(e.x);
        if (8 * g + 2 < ns) gather2(e.y);
        if (8 * g + 4 < ns) gather2(e.z);
        if (8 * g + 6 < ns) gather2(e.w);
      }
      if (p < Dc) {
        auto diag = [&](int ua, uint32_t uc, double du) -> double {
          if (a.cross_mode == 2) return __ldg(a.dfull + (int64_t)ua * Dc + p);
          double D = du + ddp;
          const uint32_t ud = uc & cdp;
          if (a.cross_mode == 0) D += a.u0 * (double)__popc(ud);
          else for (uint32_t m = ud; m; m &= m - 1) D += __ldg(a.usite + (__ffs(m) - 1));
          return D;
        };
        const double x0 = rows[p], y0 = diag(u0, uc0, du0) * x0 + tdn * g0;
        __stcs(o0, (acc == 0.0) ? scale * y0 : acc * y0old + scale * y0);
        pr += x0 * y0;
        if (two) {
          const double x1 = row1[p], y1 = diag(ua1, uc1, du1) * x1 + tdn * g1;
          __stcs(o0 + Dc, (acc == 0.0) ? scale * y1 : acc * y1old + scale * y1);
          pr += x1 * y1;
        }
      }
    }
  }
  double v[2] = {ok ? pr : __longlong_as_double(0x7FF8000000000000ll), 0.0};
  block_sum<2>(v);
  if (tid == 0) {
    part[2 * blockIdx.x] = v[0];
    part[2 * blockIdx.x + 1] = 0.0;
  }
}

// Column pass: v0[u, chunk] += scale * sum_up c * v1[u', chunk], chunk-major tasks by static
// striding; part[blockIdx] = sum of v1 . (up hops) v1 over the CTA's tasks.  VEC2: Dc is even,
// so a thread's two columns are one aligned 16-byte load.
template <bool VEC2, bool UNIFORM>
__global__ void __launch_bounds__(kUpThreads, kUpMinBlocks) prod_up_kernel(ProdArgs a, TwoPassArgs b, const double *__restrict__ v1,
                                                             double *__restrict__ v0, const double *__restrict__ coef,
                                                             double *__restrict__ part) {
  __shared__ int s_src[kMaxUpWidth];
  __shared__ double s_cf[UNIFORM ? 1 : kMaxUpWidth];
  const double scale = coef[1];
  const int Dc = a.Dc, Uc = a.Uc, wu = a.wu;
  const int nchunk = (Dc + kUpChunk - 1) / kUpChunk;
  const int64_t ntask = (int64_t)nchunk * Uc;
  double pr = 0.0;
  for (int64_t task = blockIdx.x; task < ntask; task += gridDim.x) {
    const int c = (int)(task / Uc), u = (int)(task - (int64_t)c * Uc);
    const int nu = b.nus[u];
    __syncthreads();
    for (int k = threadIdx.x; k < nu; k += kUpThreads) {
      s_src[k] = b.usrc[(int64_t)u * wu + k];
      if (!UNIFORM) s_cf[k] = b.ucf[(int64_t)u * wu + k];
    }
    __syncthreads();
    const int d = c * kUpChunk + 2 * (int)threadIdx.x;
    if (d >= Dc) continue;
    const bool pair = VEC2 || d + 1 < Dc;
    double h0 = 0.0, h1 = 0.0;
    int k = 0;
    for (; k + kUpBatch <= nu; k += kUpBatch) {
      double w0[kUpBatch], w1[kUpBatch];
#pragma unroll
      for (int q = 0; q < kUpBatch; q++) {
        const double *sp = v1 + (int64_t)(s_src[k + q] & 0x7FFFFFFF) * Dc + d;
        if (VEC2) {
          const double2 sv = __ldg(reinterpret_cast<const double2 *>(sp));
          w0[q] = sv.x; w1[q] = sv.y;
        } else {
          w0[q] = __ldg(sp);
          w1[q] = pair ? __ldg(sp + 1) : 0.0;
        }
      }
#pragma unroll
      for (int q = 0; q < kUpBatch; q++) {
        if (UNIFORM) {
          const uint32_t sg = (uint32_t)s_src[k + q] & 0x80000000u;
          h0 += flip_sign(w0[q], sg);
          h1 += flip_sign(w1[q], sg);
        } else {
          h0 += s_cf[k + q] * w0[q];
          h1 += s_cf[k + q] * w1[q];
        }
      }
    }
    for (; k < nu; k++) {
      const double *sp = v1 + (int64_t)(s_src[k] & 0x7FFFFFFF) * Dc + d;
      if (UNIFORM) {
        const uint32_t sg = (uint32_t)s_src[k] & 0x80000000u;
        h0 += flip_sign(__ldg(sp), sg);
        if (pair) h1 += flip_sign(__ldg(sp + 1), sg);
      } else {
        h0 += s_cf[k] * __ldg(sp);
        if (pair) h1 += s_cf[k] * __ldg(sp + 1);
      }
    }
    if (UNIFORM) {
      h0 *= b.t_up;
      h1 *= b.t_up;
    }
    const double *xp = v1 + (int64_t)u * Dc + d;
    double *yp = v0 + (int64_t)u * Dc + d;
    double x0, x1 = 0.0, y0, y1 = 0.0;
    // v0 is streamed (read and written once): evict-first, so it does not push the chunk of
    // v1 that the following rows gather from out of L2
    if (VEC2) {
      const double2 xv = __ldg(reinterpret_cast<const double2 *>(xp));
      const double2 yv = __ldcs(reinterpret_cast<const double2 *>(yp));
      x0 = xv.x; x1 = xv.y; y0 = yv.x; y1 = yv.y;
    } else {
      x0 = __ldg(xp);
      y0 = __ldcs(yp);
      if (pair) { x1 = __ldg(xp + 1); y1 = __ldcs(yp + 1); }
    }
    pr += x0 * h0 + x1 * h1;
    if (VEC2) {
      __stcs(reinterpret_cast<double2 *>(yp), make_double2(y0 + scale * h0, y1 + scale * h1));
    } else {
      __stcs(yp, y0 + scale * h0);
      if (pair) __stcs(yp + 1, y1 + scale * h1);
    }
  }
  double v[2] = {pr, 0.0};
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = v[0];
    part[2 * blockIdx.x + 1] = 0.0;
  }
}

constexpr int kUpWThreads = 256;     // column pass, warp tasks: 8 warps per CTA
constexpr int kUpWMinBlocks = 3;     // CTAs per SM (at most 85 registers)
constexpr int kUpWChunk = 128;       // columns per warp task (4 per lane, two 16-byte loads)
constexpr int kUpWBatch = 4;         // up hops per batch: 8 loads of 16 bytes in flight per lane

// Column pass with warp tasks (uniform up hops, Dc even, 16-byte aligned vectors, Uc <= 32768,
// at most 64 up hops per row): v0[u, chunk] += scale * t_up * sum_up sign * v1[u', chunk].  A
// task is one row u and 128 columns (lane l: columns 2l, 2l + 1 and 64 + 2l, 65 + 2l, so each
// load instruction of the warp reads 512 contiguous bytes); tasks run chunk-major (every row of chunk 0, then chunk
// 1, ...) by static striding over the warps of a grid that is resident at once, so the 1 KB
// pieces of v1 the rows gather stay in L2.  Each lane holds two 16-bit hop entries of the row
// and the warp broadcasts them by shuffles (no shared memory, no CTA barrier).
// part[blockIdx] = sum over the CTA's tasks of v1 . (up hops) v1.
__global__ void __launch_bounds__(kUpWThreads, kUpWMinBlocks) prod_up_warp_kernel(ProdArgs a, TwoPassArgs b,
                                                                                 const double *__restrict__ v1,
                                                                                 double *__restrict__ v0,
                                                                                 const double *__restrict__ coef,
                                                                                 double *__restrict__ part) {
  const int lane = threadIdx.x & 31;
  const int warp = (int)((blockIdx.x * (unsigned)kUpWThreads + threadIdx.x) >> 5);
  const int nwarps = (int)(gridDim.x * (unsigned)kUpWThreads) >> 5;
  const int Dc = a.Dc, Uc = a.Uc;
  const int nchunk = (Dc + kUpWChunk - 1) / kUpWChunk;
  const int64_t ntask = (int64_t)nchunk * Uc;
  const double tup = b.t_up, st = coef[1] * b.t_up;
  double pr = 0.0;
  // the row's hop count and packed entries of the next task are loaded one task ahead
  int64_t task = warp;
  int nu_n = 0;
  uint32_t my_n = 0u;
  auto fetch = [&](int64_t t) {
    if (t < ntask) {
      const int un = (int)(t % Uc);
      nu_n = b.nus[un];
      my_n = (2 * lane < nu_n) ? __ldg(b.usrc16 + (int64_t)un * b.wu2 + lane) : 0u;
    }
  };
  fetch(task);
  const uint64_t rowb = (uint64_t)Dc * sizeof(double);
  for (; task < ntask; task += nwarps) {
    const int c = (int)(task / Uc), u = (int)(task - (int64_t)c * Uc);
    const int nu = nu_n;
    const uint32_t my = my_n;
    fetch(task + nwarps);
    const int d = c * kUpWChunk + 2 * lane;     // columns d, d + 1 and d + 64, d + 65
    const bool ok0 = d < Dc, ok1 = d + 64 < Dc;  // Dc is even: pairs are whole
    // lanes past the last column read a valid pair (column 0) and discard what they summed
    const char *base0 = reinterpret_cast<const char *>(v1 + (ok0 ? d : 0));
    const char *base1 = reinterpret_cast<const char *>(v1 + (ok1 ? d + 64 : 0));
    double h0 = 0.0, h1 = 0.0, h2 = 0.0, h3 = 0.0;
    auto hop = [&](uint32_t e, double2 &w0, double2 &w1) {
      const uint64_t off = (uint64_t)(e & 0x7FFFu) * rowb;
      w0 = __ldg(reinterpret_cast<const double2 *>(base0 + off));
      w1 = __ldg(reinterpret_cast<const double2 *>(base1 + off));
    };
    auto add = [&](uint32_t e, const double2 &w0, const double2 &w1) {
      const uint32_t sg = (e & 0x8000u) << 16;
      h0 += flip_sign(w0.x, sg);
      h1 += flip_sign(w0.y, sg);
      h2 += flip_sign(w1.x, sg);
      h3 += flip_sign(w1.y, sg);
    };
    int k = 0;
    for (; k + kUpWBatch <= nu; k += kUpWBatch) {
      double2 w0[kUpWBatch], w1[kUpWBatch];
      uint32_t e[kUpWBatch];
#pragma unroll
      for (int q = 0; q < kUpWBatch; q += 2) {
        const uint32_t word = __shfl_sync(0xFFFFFFFFu, my, ((k + q) >> 1) & 31);
        e[q] = word & 0xFFFFu;
        e[q + 1] = word >> 16;
      }
#pragma unroll
      for (int q = 0; q < kUpWBatch; q++) hop(e[q], w0[q], w1[q]);
#pragma unroll
      for (int q = 0; q < kUpWBatch; q++) add(e[q], w0[q], w1[q]);
    }
    for (; k < nu; k++) {
      const uint32_t word = __shfl_sync(0xFFFFFFFFu, my, (k >> 1) & 31);
      const uint32_t e = (k & 1) ? (word >> 16) : (word & 0xFFFFu);
      double2 w0, w1;
      hop(e, w0, w1);
      add(e, w0, w1);
    }
    const double *xp = v1 + (int64_t)u * Dc + d;
    double *yp = v0 + (int64_t)u * Dc + d;
    // v0 is streamed (read and written once): evict-first, so it does not push the chunk of
    // v1 that the following rows gather from out of L2
    if (ok0) {
      const double2 xv = __ldg(reinterpret_cast<const double2 *>(xp));
      const double2 yv = __ldcs(reinterpret_cast<const double2 *>(yp));
      pr += tup * (xv.x * h0 + xv.y * h1);
      __stcs(reinterpret_cast<double2 *>(yp), make_double2(yv.x + st * h0, yv.y + st * h1));
    }
    if (ok1) {
      const double2 xv = __ldg(reinterpret_cast<const double2 *>(xp + 64));
      const double2 yv = __ldcs(reinterpret_cast<const double2 *>(yp + 64));
      pr += tup * (xv.x * h2 + xv.y * h3);
      __stcs(reinterpret_cast<double2 *>(yp + 64), make_double2(yv.x + st * h2, yv.y + st * h3));
    }
  }
  double v[2] = {pr, 0.0};
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = v[0];
    part[2 * blockIdx.x + 1] = 0.0;
  }
}

__device__ __forceinline__ uint32_t compress_species(uint64_t c, int s, int N) {
  uint32_t x = 0;
  for (int i = 0; i < N; i++) x |= (uint32_t)((c >> (2 * i + s)) & 1ull) << i;
  return x;
}

// sigma(c) of the species-first basis: (-1)^#{(down at i, up at j) : i < j}.
__device__ __forceinline__ int species_parity(uint64_t c, int N) {
  int cnt = 0, downs = 0;
  for (int i = 0; i < N; i++) {
    if ((c >> (2 * i)) & 1ull) cnt += downs;
    downs += (int)((c >> (2 * i + 1)) & 1ull);
  }
  return cnt & 1;
}

// HPhi order <-> native order, per row r of HPhi's list_1; SIGN applies sigma (vectors),
// without it the values are moved as they are (functions of the configuration).
template <typename T, bool TO_NATIVE, bool SIGN>
__global__ void prod_permute_kernel(int64_t dim, int N, int Dc, const uint64_t *__restrict__ list_1,
                                    const uint16_t *__restrict__ rank, const uint16_t *__restrict__ pos_dn,
                                    const T *__restrict__ in, T *__restrict__ out) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = list_1[r];
    const int64_t pos = (int64_t)rank[compress_species(c, 0, N)] * Dc + pos_dn[compress_species(c, 1, N)];
    const double sg = (SIGN && species_parity(c, N)) ? -1.0 : 1.0;
    if (TO_NATIVE) out[pos] = VT<T>::scale(sg, in[r]);
    else out[r] = VT<T>::scale(sg, in[pos]);
  }
}

// HPhi order -> native order as a gather over the native positions: position (up rank ua, down
// position da) holds the configuration c with the up spins of unrank_up[ua] on the even bits
// and the down spins of unrank_dn[da] on the odd bits, whose HPhi row is
// list_2_1[c & lo_mask] + list_2_2[c >> lo_bits] - 3.  Writes are coalesced and only the reads
// scattered, where the row-ordered form above scatters its writes.
__device__ __forceinline__ uint64_t spread_even_bits(uint64_t x) {  // bit i -> bit 2i, x < 2^32
  x &= 0xFFFFFFFFull;
  x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
  x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
  x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}

template <typename T>
__global__ void prod_to_native_gather_kernel(int64_t n, int N, int Dc, const uint16_t *__restrict__ unrank_up,
                                             const uint16_t *__restrict__ unrank_dn, const uint32_t *__restrict__ l21,
                                             const uint32_t *__restrict__ l22, int lo_bits, uint64_t lo_mask,
                                             const T *__restrict__ in, T *__restrict__ out) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ua = p / Dc;
    const int64_t da = p - ua * Dc;
    const uint64_t c = spread_even_bits(__ldg(unrank_up + ua)) | (spread_even_bits(__ldg(unrank_dn + da)) << 1);
    const int64_t r = (int64_t)__ldg(l21 + (c & lo_mask)) + (int64_t)__ldg(l22 + (c >> lo_bits)) - 3;
    const double sg = species_parity(c, N) ? -1.0 : 1.0;
    out[p] = VT<T>::scale(sg, in[r]);
  }
}

// Diagonal observables in native order (expec_energy_flct_Hubbard, src/expec_energy_flct.c:259-330).
template <typename T>
__global__ void prod_obs_kernel(ProdArgs a, const T *__restrict__ v, double *__restrict__ part) {
  double o[6] = {0, 0, 0, 0, 0, 0};
  const int64_t n = (int64_t)a.Uc * a.Dc;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const int ua = (int)(p / a.Dc), da = (int)(p - (int64_t)ua * a.Dc);
    const uint32_t u = a.unrank_up[ua], d = a.unrank_dn[da];
    const double w = VT<T>::abs2(v[p]);
    const int up = __popc(u), dn = __popc(d);
    const double D = (double)__popc(u & d), Nn = (double)(up + dn), Sz = 0.5 * (double)(up - dn);
    o[0] += w * D; o[1] += w * D * D; o[2] += w * Nn; o[3] += w * Nn * Nn; o[4] += w * Sz; o[5] += w * Sz * Sz;
  }
  block_sum<6>(o);
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; k++) part[6 * blockIdx.x + k] = o[k];
}

uint64_t binom_p(int n, int k) {
  if (k < 0 || k > n) return 0;
  uint64_t r = 1;
  for (int i = 1; i <= k; i++) r = r * (uint64_t)(n - k + i) / (uint64_t)i;
  return r;
}

int cuda_ok(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    set_error(std::string("product kernel: ") + what + ": " + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

}  // namespace

struct ProdPlan {
  ProdArgs args{};
  std::vector<void *> allocs;
  int grid = 0;
  size_t smem[2] = {0, 0};  // real, complex
  double *part = nullptr;   // partial sums: 2 * max(Uc, grid_dn + grid_up)
  int *counter = nullptr;
  bool two_pass = false;    // real vectors take the two-pass kernels
  TwoPassArgs tp{};
  int grid_dn = 0, grid_up = 0;  // grid_up: records reserved for the column pass (either kernel)
  int grid_upw = 0;              // grid of prod_up_warp_kernel (0: not applicable)
  size_t smem_dn = 0;
};

void prod_plan_free(ProdPlan *p) {
  if (!p) return;
  for (void *q : p->allocs) cudaFree(q);
  delete p;
}

namespace {

template <typename V>
int upload(ProdPlan *p, const std::vector<V> &h, const V **d, std::string *err) {
  void *q = nullptr;
  const size_t bytes = h.empty() ? 16 : sizeof(V) * h.size();
  if (cudaMalloc(&q, bytes) != cudaSuccess) {
    *err = "product plan: device allocation failed";
    return -1;
  }
  p->allocs.push_back(q);
  if (!h.empty() && cudaMemcpy(q, h.data(), sizeof(V) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    *err = "product plan: copy failed";
    return -1;
  }
  *d = (const V *)q;
  return 0;
}

struct SpeciesHop {
  int i, j;          // created, annihilated site
  double re, im;     // operator coefficient
};

// ELL of one species' hops over its configurations (by rank): per configuration the
// applicable hops as (source rank, coefficient index 2h + sign).
void build_ell(const std::vector<SpeciesHop> &hops, const std::vector<uint16_t> &unrank,
               const std::vector<uint16_t> &rank, std::vector<std::vector<uint32_t>> *rows, int *width) {
  rows->assign(unrank.size(), {});
  *width = 0;
  for (size_t r = 0; r < unrank.size(); r++) {
    const uint32_t x = unrank[r];
    for (size_t h = 0; h < hops.size(); h++) {
      const int i = hops[h].i, j = hops[h].j;
      if (!((x >> i) & 1u) || ((x >> j) & 1u)) continue;
      const uint32_t src = x ^ (1u << i) ^ (1u << j);
      const int lo = std::min(i, j), hi = std::max(i, j);
      const uint32_t between = (uint32_t)(((1ull << hi) - 1) ^ ((1ull << (lo + 1)) - 1));
      const uint32_t sign = (uint32_t)(__builtin_popcount(x & between) & 1);
      (*rows)[r].push_back((uint32_t)rank[src] | ((2u * (uint32_t)h + sign) << 16));
    }
    *width = std::max(*width, (int)(*rows)[r].size());
  }
}

std::vector<double2> coef_table(const std::vector<SpeciesHop> &hops) {
  std::vector<double2> c(2 * hops.size() + 1);
  for (size_t h = 0; h < hops.size(); h++) {
    c[2 * h] = make_double2(hops[h].re, hops[h].im);
    c[2 * h + 1] = make_double2(-hops[h].re, -hops[h].im);
  }
  return c;
}

uint64_t spread_species(uint32_t x, int s, int N) {
  uint64_t c = 0;
  for (int i = 0; i < N; i++)
    if ((x >> i) & 1u) c |= 1ull << (2 * i + s);
  return c;
}

// Gather table of the row pass.  Column p belongs to warp p / 32 and half-warp (p / 16) % 2;
// the entries of the 16 columns of a half-warp form a bipartite multigraph between lanes and
// shared-memory bank pairs (source word mod 16).  A proper edge colouring with Delta colours
// (Delta = its largest degree; Konig's theorem, built by swapping alternating paths) gives
// slots in which every lane and every bank pair carries at most one entry.  Lanes left
// without an entry in a slot read a zero word of a bank pair that slot leaves free (words
// Dc .. Dc+15, one per bank pair).  Stored packed: per warp and group of 8 slots, each lane's
// 8 entries (16 bits: word | sign << 15) are one 16-byte load.
void build_gather(const std::vector<std::vector<uint32_t>> &rows_dn, const std::vector<SpeciesHop> &hops, int Dc,
                  int npad, std::vector<uint32_t> *gat, std::vector<uint8_t> *wslots, int *nslots, int *groups) {
  const int nwarp = npad / 32;
  auto zero_word = [&](int bank) { return (uint32_t)(Dc + (((bank - Dc) % 16) + 16) % 16); };
  std::vector<std::vector<uint32_t>> lane_slots(npad);  // per column: entry of each slot of its half
  wslots->assign(nwarp, 0);
  *nslots = 0;
  for (int w = 0; w < nwarp; w++) {
    int wmax = 0;
    for (int hw = 0; hw < 2; hw++) {
      std::vector<int> el, eb;
      std::vector<uint32_t> ev;
      for (int l = 0; l < 16; l++) {
        const int col = 32 * w + 16 * hw + l;
        if (col >= Dc) continue;
        for (uint32_t e : rows_dn[col]) {
          const uint32_t word = e & 0xFFFFu, h = (e >> 16) >> 1, sign = (e >> 16) & 1u;
          const bool neg = ((hops[h].re < 0) != (sign != 0));
          el.push_back(l);
          eb.push_back((int)(word % 16));
          ev.push_back((word * 8u) | (neg ? 0x80000000u : 0u));
        }
      }
      int ldeg[16] = {0}, bdeg[16] = {0};
      for (size_t i = 0; i < el.size(); i++) { ldeg[el[i]]++; bdeg[eb[i]]++; }
      int D = 0;
      for (int i = 0; i < 16; i++) D = std::max(D, std::max(ldeg[i], bdeg[i]));
      std::vector<int> L(16 * std::max(D, 1), -1), B(16 * std::max(D, 1), -1), colr(el.size(), -1);
      for (size_t i = 0; i < el.size(); i++) {
        const int l = el[i], bk = eb[i];
        int a = 0, c = 0;
        while (L[l * D + a] >= 0) a++;
        while (B[bk * D + c] >= 0) c++;
        if (B[bk * D + a] >= 0) {
          // alternating a/c path from bank bk; swapping it frees a at bk
          std::vector<int> path;
          int node = bk, want = a;
          bool at_bank = true;
          for (;;) {
            const int ed = at_bank ? B[node * D + want] : L[node * D + want];
            if (ed < 0) break;
            path.push_back(ed);
            node = at_bank ? el[ed] : eb[ed];
            at_bank = !at_bank;
            want = (want == a) ? c : a;
          }
          for (int ed : path) { L[el[ed] * D + colr[ed]] = -1; B[eb[ed] * D + colr[ed]] = -1; }
          for (int ed : path) colr[ed] = (colr[ed] == a) ? c : a;
          for (int ed : path) { L[el[ed] * D + colr[ed]] = ed; B[eb[ed] * D + colr[ed]] = ed; }
        }
        colr[i] = a;
        L[l * D + a] = (int)i;
        B[bk * D + a] = (int)i;
      }
      for (int l = 0; l < 16; l++) lane_slots[32 * w + 16 * hw + l].assign(D, 0u);
      for (int c = 0; c < D; c++) {
        std::vector<int> free_banks;
        for (int bk = 0; bk < 16; bk++)
          if (B[bk * D + c] < 0) free_banks.push_back(bk);
        size_t f = 0;
        for (int l = 0; l < 16; l++) {
          const int ed = L[l * D + c];
          lane_slots[32 * w + 16 * hw + l][c] = (ed >= 0) ? ev[ed] : zero_word(free_banks[f++]) * 8u;
        }
      }
      wmax = std::max(wmax, D);
    }
    (*wslots)[w] = (uint8_t)wmax;
    *nslots = std::max(*nslots, wmax);
  }
  // packed: per warp and slot group g, 32 lanes x 8 entries of 16 bits (word | sign << 15)
  *groups = std::max(1, (*nslots + 7) / 8);
  gat->assign((size_t)nwarp * *groups * 32 * 4, 0u);
  for (int p = 0; p < npad; p++) {
    const int w = p / 32, lane = p % 32, l = p % 16;
    for (int sl = 0; sl < 8 * *groups; sl++) {
      uint32_t word, neg = 0;
      if (sl < (int)lane_slots[p].size()) {
        word = (lane_slots[p][sl] & 0x7FFFFFFFu) / 8u;
        neg = lane_slots[p][sl] >> 31;
      } else {
        word = zero_word(l);
      }
      const uint32_t e16 = word | (neg << 15);
      const size_t q = (((size_t)w * *groups + sl / 8) * 32 + lane) * 4 + (sl % 8) / 2;
      (*gat)[q] |= (sl % 2) ? (e16 << 16) : e16;
    }
  }
}


// Positions of the down configurations for the row pass.  The row pass gives column p to
// lane p % 32 of warp p / 32, and an 8-byte gather of source column q hits the shared-memory
// bank pair q % 16; a half-warp's slot count is max(largest lane degree, largest bank-pair
// load) (the edge colouring of build_gather), so positions decide both.  Start from the
// configurations sorted by hop count (equal lane degrees in a half-warp), then swap positions
// (within a half-warp: a bank change; across half-warps: only between equal hop counts) when
// that does not raise the summed slot counts of the half-warps it touches.  rows[r]: sources
// of configuration r (ELL entries, source in the low 16 bits).  Returns the position of each
// configuration; deterministic (fixed seed).
std::vector<int> balance_positions(const std::vector<std::vector<uint32_t>> &rows) {
  const int n = (int)rows.size();
  constexpr int G = 16;
  std::vector<int> order(n), pos(n);
  for (int r = 0; r < n; r++) order[r] = r;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return rows[a].size() > rows[b].size(); });
  for (int p = 0; p < n; p++) pos[order[p]] = p;
  const int ng = (n + G - 1) / G;
  if (n < 4 * G) return pos;
  std::vector<std::vector<int>> src(n), rdr(n);
  for (int r = 0; r < n; r++)
    for (uint32_t e : rows[r]) {
      const int q = (int)(e & 0xFFFFu);
      src[r].push_back(q);
      rdr[q].push_back(r);
    }
  std::vector<int> at(order);  // configuration at each position
  std::vector<int> load((size_t)ng * G, 0), lmax(ng, 0), D(ng, 0);
  for (int r = 0; r < n; r++) {
    const int g = pos[r] / G;
    lmax[g] = std::max(lmax[g], (int)src[r].size());
    for (int q : src[r]) load[(size_t)g * G + pos[q] % G]++;
  }
  auto eval = [&](int g) {
    int m = lmax[g];
    for (int k = 0; k < G; k++) m = std::max(m, load[(size_t)g * G + k]);
    return m;
  };
  for (int g = 0; g < ng; g++) D[g] = eval(g);
  uint64_t rng = 0x9E3779B97F4A7C15ull;
  auto next = [&]() { rng ^= rng << 13; rng ^= rng >> 7; rng ^= rng << 17; return rng; };
  std::vector<int> touched;
  std::vector<char> mark(ng, 0);
  auto touch = [&](int g) { if (!mark[g]) { mark[g] = 1; touched.push_back(g); } };
  // adds (sgn = 1) or removes (-1) a configuration's edges: its reads (in its own half-warp)
  // and the reads of it; edges to `other` are left to the other configuration's call
  auto contrib = [&](int r, int p, int sgn, int other) {
    const int g = p / G, bk = p % G;
    for (int q : src[r])
      if (q != other) load[(size_t)g * G + pos[q] % G] += sgn;
    for (int rr : rdr[r])
      if (rr != other) { const int gg = pos[rr] / G; load[(size_t)gg * G + bk] += sgn; touch(gg); }
    touch(g);
  };
  const int64_t iters = std::min<int64_t>(200 * (int64_t)n, 4000000);
  for (int64_t it = 0; it < iters; it++) {
    const int p1 = (int)(next() % n);
    int p2;
    if (next() & 1) p2 = (p1 / G) * G + (int)(next() % G);
    else p2 = (int)(next() % n);
    if (p2 >= n || p2 == p1 || src[at[p1]].size() != src[at[p2]].size()) continue;
    const int a = at[p1], b = at[p2];
    touched.clear();
    contrib(a, p1, -1, -1);
    contrib(b, p2, -1, a);
    pos[a] = p2; pos[b] = p1; at[p1] = b; at[p2] = a;
    contrib(a, p2, +1, -1);
    contrib(b, p1, +1, a);
    long before = 0, after = 0;
    std::vector<int> nd(touched.size());
    for (size_t i = 0; i < touched.size(); i++) {
      before += D[touched[i]];
      nd[i] = eval(touched[i]);
      after += nd[i];
    }
    if (after <= before) {
      for (size_t i = 0; i < touched.size(); i++) D[touched[i]] = nd[i];
    } else {
      contrib(a, p2, -1, -1);
      contrib(b, p1, -1, a);
      pos[a] = p1; pos[b] = p2; at[p1] = a; at[p2] = b;
      contrib(a, p1, +1, -1);
      contrib(b, p2, +1, a);
    }
    for (int g : touched) mark[g] = 0;
  }
  return pos;
}

}  // namespace

void build_gather_table(const std::vector<std::vector<uint32_t>> &rows, int n, std::vector<uint32_t> *gat,
                        std::vector<uint8_t> *wslots, int *groups) {
  // entries carry their sign directly: one hop of coefficient +1, sign bit = (entry >> 16) & 1
  const std::vector<SpeciesHop> unit{SpeciesHop{0, 0, 1.0, 0.0}};
  int nslots = 0;
  build_gather(rows, unit, n, (n + 31) / 32 * 32, gat, wslots, &nslots, groups);
}

int prod_plan_build(Sector *s, std::string *err) {
  const Model &m = s->model;
  s->prod = nullptr;
  if (m.calc_model != kHubbard || s->gc || m.nsite > 16 || m.nsite < 1) return 0;
  const int N = m.nsite;
  std::vector<SpeciesHop> hops[2];
  for (const BitTerm &t : m.offdiag) {
    if (__builtin_popcountll(t.flip) != 2 || t.cm != t.flip) return 0;
    const int p = __builtin_ctzll(t.flip), q = 63 - __builtin_clzll(t.flip);
    if ((p & 1) != (q & 1)) return 0;
    if (t.cv != (1ull << p) && t.cv != (1ull << q)) return 0;
    const int created = __builtin_ctzll(t.cv), annihilated = (created == p) ? q : p;
    const double sg = (__builtin_popcountll(t.cv & t.sm) & 1) ? -1.0 : 1.0;
    hops[p & 1].push_back(SpeciesHop{created >> 1, annihilated >> 1, sg * t.re, sg * t.im});
  }
  if (hops[0].size() > 16000 || hops[1].size() > 16000) return 0;
  const int Uc = (int)binom_p(N, m.nup), Dc = (int)binom_p(N, m.ndown);
  if (Uc < 1 || Dc < 1 || Uc > 65535 || Dc > 65535 || (int64_t)Uc * Dc != s->dim) return 0;
  const size_t smem_r = sizeof(double) * (size_t)Dc, smem_c = sizeof(cplx) * (size_t)Dc;
  if (smem_c + 4096 > 227 * 1024) return 0;
  const int nx = 1 << N;
  std::vector<uint16_t> rank(nx), unrank_up, unrank_dn;
  {
    std::vector<int> fill(N + 1, 0);
    for (int x = 0; x < nx; x++) {
      const int k = __builtin_popcount(x);
      rank[x] = (uint16_t)fill[k]++;
      if (k == m.nup) unrank_up.push_back((uint16_t)x);
      if (k == m.ndown) unrank_dn.push_back((uint16_t)x);
    }
  }
  std::vector<std::vector<uint32_t>> rows_dn, rows_up;
  int wd = 0, wu = 0;
  build_ell(hops[1], unrank_dn, rank, &rows_dn, &wd);
  build_ell(hops[0], unrank_up, rank, &rows_up, &wu);
  // Two-pass kernels (real vectors): every down hop of one magnitude, real up hops, the
  // second staged row at its fixed offset.  HPHI_B200_PROD=single keeps the one-pass kernel.
  bool two_pass_ok;
  double tmag;
  {
    const char *pe = getenv("HPHI_B200_PROD");
    two_pass_ok = !(pe && std::string(pe) == "single") && !hops[1].empty() &&
                  (size_t)(Dc + 16) * 8 <= (size_t)kRow2Bytes && wd <= 255;
    tmag = hops[1].empty() ? 0.0 : std::fabs(hops[1][0].re);
    for (const SpeciesHop &h : hops[1]) two_pass_ok = two_pass_ok && h.im == 0.0 && std::fabs(h.re) == tmag && tmag > 0.0;
    for (const SpeciesHop &h : hops[0]) two_pass_ok = two_pass_ok && h.im == 0.0;
  }
  // Down configurations take the positions balanced for the row pass's gather table
  // (balance_positions); HPHI_B200_BALANCE=0 keeps rank order.  Up configurations keep
  // their rank.
  std::vector<uint16_t> pos_dn(rank);
  {
    const char *bal = getenv("HPHI_B200_BALANCE");
    if (two_pass_ok && !(bal && std::string(bal) == "0")) {
      const std::vector<int> pos = balance_positions(rows_dn);
      std::vector<uint16_t> un(Dc);
      for (int r = 0; r < Dc; r++) un[pos[r]] = unrank_dn[r];
      unrank_dn.swap(un);
      for (int p = 0; p < Dc; p++) pos_dn[unrank_dn[p]] = (uint16_t)p;
      build_ell(hops[1], unrank_dn, pos_dn, &rows_dn, &wd);
    }
  }
  if (wu > kMaxUpWidth || wd > 255) return 0;
  std::vector<uint32_t> ell_dn((size_t)std::max(wd, 1) * Dc, kEllNone), ell_up((size_t)Uc * std::max(wu, 1), kEllNone);
  std::vector<uint8_t> cnt_dn(Dc), wmax_dn((Dc + 31) / 32, 0);
  for (int r = 0; r < Dc; r++) {
    for (size_t k = 0; k < rows_dn[r].size(); k++) ell_dn[k * (size_t)Dc + r] = rows_dn[r][k];
    cnt_dn[r] = (uint8_t)rows_dn[r].size();
    wmax_dn[r >> 5] = std::max<uint8_t>(wmax_dn[r >> 5], cnt_dn[r]);
  }
  for (int r = 0; r < Uc; r++)
    for (size_t k = 0; k < rows_up[r].size(); k++) ell_up[(size_t)r * std::max(wu, 1) + k] = rows_up[r][k];
  // diagonal: per-species parts, on-site cross terms, or the full diagonal
  const uint64_t even = 0x5555555555555555ull, odd = even << 1;
  std::vector<double> du(Uc, 0.0), dd(Dc, 0.0), usite(N, 0.0);
  bool general_cross = false;
  std::vector<DiagTerm> up_t, dn_t;
  for (const DiagTerm &t : m.diag) {
    if ((t.cm & odd) == 0) up_t.push_back(t);
    else if ((t.cm & even) == 0) dn_t.push_back(t);
    else {
      const int i = __builtin_ctzll(t.cm) >> 1;
      const uint64_t site = 3ull << (2 * i);
      if (t.cm == site && t.cv == site) usite[i] += t.v;
      else general_cross = true;
    }
  }
  for (int r = 0; r < Uc; r++) {
    const uint64_t c = spread_species(unrank_up[r], 0, N);
    for (const DiagTerm &t : up_t)
      if ((c & t.cm) == t.cv) du[r] += t.v;
  }
  for (int r = 0; r < Dc; r++) {
    const uint64_t c = spread_species(unrank_dn[r], 1, N);
    for (const DiagTerm &t : dn_t)
      if ((c & t.cm) == t.cv) dd[r] += t.v;
  }
  // Row processing order.  Up hops read whole source rows; rows processed close together in
  // time share sources in L2 when the order follows the hop graph.  Default: Cuthill-McKee
  // (breadth-first from a minimum-degree row, neighbours by increasing degree);
  // HPHI_B200_ROW_ORDER=natural keeps the rank order.
  std::vector<int> order(Uc);
  {
    const char *ro = getenv("HPHI_B200_ROW_ORDER");
    if (ro && std::string(ro) == "natural") {
      for (int r = 0; r < Uc; r++) order[r] = r;
    } else {
      std::vector<char> seen(Uc, 0);
      int n = 0;
      while (n < Uc) {
        int start = -1;
        for (int r = 0; r < Uc; r++)
          if (!seen[r] && (start < 0 || rows_up[r].size() < rows_up[start].size())) start = r;
        size_t head = n;
        order[n++] = start;
        seen[start] = 1;
        while (head < (size_t)n) {
          const int r = order[head++];
          std::vector<int> nb;
          for (uint32_t e : rows_up[r]) {
            const int q = (int)(e & 0xFFFFu);
            if (!seen[q]) { seen[q] = 1; nb.push_back(q); }
          }
          std::stable_sort(nb.begin(), nb.end(), [&](int x, int y) { return rows_up[x].size() < rows_up[y].size(); });
          for (int q : nb) order[n++] = q;
        }
      }
    }
  }
  ProdPlan *p = new ProdPlan();
  ProdArgs &a = p->args;
  a.N = N;
  a.Uc = Uc;
  a.Dc = Dc;
  a.wd = wd;
  a.wu = wu;
  bool uniform = true;
  for (int i = 1; i < N; i++) uniform = uniform && (usite[i] == usite[0]);
  a.cross_mode = general_cross ? 2 : (uniform ? 0 : 1);
  a.u0 = usite[0];
  std::vector<double> utab(17);
  for (int k = 0; k <= 16; k++) utab[k] = a.u0 * (double)k;
  auto fail = [&]() { prod_plan_free(p); return -1; };
  if (upload(p, rank, &a.rank, err) || upload(p, pos_dn, &a.pos_dn, err) || upload(p, unrank_up, &a.unrank_up, err) ||
      upload(p, unrank_dn, &a.unrank_dn, err) || upload(p, ell_dn, &a.ell_dn, err) ||
      upload(p, ell_up, &a.ell_up, err) || upload(p, coef_table(hops[1]), &a.cf_dn, err) ||
      upload(p, coef_table(hops[0]), &a.cf_up, err) || upload(p, du, &a.du, err) || upload(p, dd, &a.dd, err) ||
      upload(p, usite, &a.usite, err) || upload(p, order, &a.order, err) || upload(p, cnt_dn, &a.cnt_dn, err) ||
      upload(p, wmax_dn, &a.wmax_dn, err) || upload(p, utab, &a.utab, err))
    return fail();
  if (a.cross_mode == 2) {
    void *q = nullptr;
    if (cudaMalloc(&q, sizeof(double) * (size_t)s->dim) != cudaSuccess) {
      *err = "product plan: device allocation failed";
      return fail();
    }
    p->allocs.push_back(q);
    const unsigned nb = (unsigned)std::min<int64_t>((s->dim + 255) / 256, (int64_t)s->num_sms * 16);
    prod_permute_kernel<double, true, false><<<nb, 256, 0, s->stream>>>(s->dim, N, Dc, s->d_list_1, a.rank, a.pos_dn,
                                                                        s->d_diag, (double *)q);
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
      *err = "product plan: diagonal permutation failed";
      return fail();
    }
    a.dfull = (const double *)q;
  }
  if (cudaMalloc(&p->part, sizeof(double) * 2 * (size_t)Uc) != cudaSuccess ||
      cudaMalloc(&p->counter, 2 * sizeof(int)) != cudaSuccess) {
    *err = "product plan: device allocation failed";
    return fail();
  }
  p->allocs.push_back(p->part);
  p->allocs.push_back(p->counter);
  if (cudaMemset(p->counter, 0, 2 * sizeof(int)) != cudaSuccess) {
    *err = "product plan: clear failed";
    return fail();
  }
  p->smem[0] = smem_r;
  p->smem[1] = smem_c;
  if (raise_smem_limit((const void *)prod_hv_kernel<double>, smem_r) != cudaSuccess ||
      raise_smem_limit((const void *)prod_hv_kernel<cplx>, smem_c) != cudaSuccess) {
    *err = "product plan: shared-memory attribute rejected";
    return fail();
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, prod_hv_kernel<double>, kProdThreads, smem_r);
  p->grid = std::max(1, std::min(Uc, std::max(1, per_sm) * s->num_sms));
  {
    if (two_pass_ok) {
      TwoPassArgs &b = p->tp;
      b.npad = (Dc + 31) / 32 * 32;
      b.t_dn = tmag;
      std::vector<uint32_t> gat;
      std::vector<uint8_t> wslots;
      int nslots = 0;
      build_gather(rows_dn, hops[1], Dc, b.npad, &gat, &wslots, &nslots, &b.groups);
      std::vector<uint4> gat4(gat.size() / 4);
      for (size_t i = 0; i < gat4.size(); i++) gat4[i] = make_uint4(gat[4 * i], gat[4 * i + 1], gat[4 * i + 2], gat[4 * i + 3]);
      b.t_up = hops[0].empty() ? 0.0 : std::fabs(hops[0][0].re);
      b.up_uniform = b.t_up > 0.0 ? 1 : 0;
      for (const SpeciesHop &h : hops[0]) b.up_uniform = b.up_uniform && std::fabs(h.re) == b.t_up;
      const int wuu = std::max(wu, 1);
      std::vector<int> usrc((size_t)Uc * wuu, 0);
      std::vector<double> ucf((size_t)Uc * wuu, 0.0);
      std::vector<uint8_t> nus(Uc, 0);
      for (int r = 0; r < Uc; r++) {
        for (size_t k = 0; k < rows_up[r].size(); k++) {
          const uint32_t e = rows_up[r][k], h = (e >> 16) >> 1, sign = (e >> 16) & 1u;
          const double cf = sign ? -hops[0][h].re : hops[0][h].re;
          usrc[(size_t)r * wuu + k] = (int)(e & 0xFFFFu) | ((b.up_uniform && cf < 0) ? (int)0x80000000 : 0);
          ucf[(size_t)r * wuu + k] = cf;
        }
        nus[r] = (uint8_t)rows_up[r].size();
      }
      // packed up-hop table of the warp-task column pass (uniform hops, ranks below 2^15)
      std::vector<uint32_t> usrc16;
      b.wu2 = 0;
      if (b.up_uniform && Uc <= 32768 && wu <= 64) {
        b.wu2 = std::max(1, (wu + 1) / 2);
        usrc16.assign((size_t)Uc * b.wu2, 0u);
        for (int r = 0; r < Uc; r++)
          for (int k = 0; k < (int)nus[r]; k++) {
            const uint32_t e = (uint32_t)usrc[(size_t)r * wuu + k];
            const uint32_t e16 = (e & 0x7FFFu) | ((e >> 31) << 15);
            usrc16[(size_t)r * b.wu2 + k / 2] |= (k % 2) ? (e16 << 16) : e16;
          }
      }
      if (upload(p, gat4, &b.gat, err) || upload(p, wslots, &b.wslots, err) || upload(p, usrc, &b.usrc, err) ||
          upload(p, ucf, &b.ucf, err) || upload(p, nus, &b.nus, err) || upload(p, usrc16, &b.usrc16, err))
        return fail();
      p->smem_dn = (size_t)kRow2Bytes + (size_t)(Dc + 16) * 8;
      if (raise_smem_limit((const void *)prod_down_kernel, p->smem_dn) != cudaSuccess) {
        *err = "product plan: shared-memory attribute rejected (row pass)";
        return fail();
      }
      int up_per_sm = 0, upw_per_sm = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&up_per_sm, prod_up_kernel<true, true>, kUpThreads, 0);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&upw_per_sm, prod_up_warp_kernel, kUpWThreads, 0);
      p->grid_dn = std::max(1, std::min((Uc + 1) / 2, s->num_sms));
      p->grid_upw = (b.wu2 > 0) ? std::max(1, upw_per_sm) * s->num_sms : 0;
      {
        const char *ue = getenv("HPHI_B200_UPPASS");
        if (ue && std::string(ue) == "block") p->grid_upw = 0;
      }
      p->grid_up = std::max(std::max(1, std::max(1, up_per_sm) * s->num_sms), p->grid_upw);
      p->two_pass = true;
      if (2 * (p->grid_dn + p->grid_up) > 2 * Uc) {
        cudaFree(p->part);
        p->allocs.erase(std::find(p->allocs.begin(), p->allocs.end(), (void *)p->part));
        p->part = nullptr;
        if (cudaMalloc(&p->part, sizeof(double) * 2 * (size_t)(p->grid_dn + p->grid_up)) != cudaSuccess) {
          *err = "product plan: device allocation failed";
          return fail();
        }
        p->allocs.push_back(p->part);
      }
    }
  }
  s->prod = p;
  return 0;
}

bool prod_two_pass(const Sector *s) { return s->prod && s->prod->two_pass; }

size_t prod_scratch_doubles(const Sector *s, VecType vt) {
  const ProdPlan *p = s->prod;
  // the two-pass kernels (real vectors) keep one partial sum per CTA of each pass; the
  // one-pass kernel one per row
  if (vt == kReal64 && p->two_pass) return 2 * (size_t)(p->grid_dn + p->grid_up);
  return 2 * (size_t)p->args.Uc;
}

namespace {
// Row pass then column pass; partial sums at d_part (grid_dn + grid_up records of 2).
void two_pass_launch(Sector *s, const double *v1, double *v0, const double *d_coef, double *d_out, double *d_part) {
  ProdPlan *p = s->prod;
  prod_down_kernel<<<p->grid_dn, kDownThreads, p->smem_dn, s->stream>>>(p->args, p->tp, v1, v0, d_coef, d_part);
  const bool vec2 = (p->args.Dc % 2 == 0) && ((((uintptr_t)v1) | ((uintptr_t)v0)) % 16 == 0);
  double *pu = d_part + 2 * p->grid_dn;
  if (vec2 && p->grid_upw > 0) {
    prod_up_warp_kernel<<<p->grid_upw, kUpWThreads, 0, s->stream>>>(p->args, p->tp, v1, v0, d_coef, pu);
    finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(d_part, p->grid_dn + p->grid_upw, d_out);
    return;
  }
  const int g = p->grid_up;
  if (vec2 && p->tp.up_uniform)
    prod_up_kernel<true, true><<<g, kUpThreads, 0, s->stream>>>(p->args, p->tp, v1, v0, d_coef, pu);
  else if (vec2)
    prod_up_kernel<true, false><<<g, kUpThreads, 0, s->stream>>>(p->args, p->tp, v1, v0, d_coef, pu);
  else if (p->tp.up_uniform)
    prod_up_kernel<false, true><<<g, kUpThreads, 0, s->stream>>>(p->args, p->tp, v1, v0, d_coef, pu);
  else
    prod_up_kernel<false, false><<<g, kUpThreads, 0, s->stream>>>(p->args, p->tp, v1, v0, d_coef, pu);
  finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(d_part, p->grid_dn + p->grid_up, d_out);
}
}  // namespace

int prod_hv_launch_scratch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                           double *d_part, int *d_counter) {
  ProdPlan *p = s->prod;
  if (vt == kReal64 && s->model.complex_terms) {
    set_error("H has complex coefficients: real vectors are not allowed");
    return -1;
  }
  if (vt == kReal64 && p->two_pass) {
    two_pass_launch(s, (const double *)d_v1, (double *)d_v0, d_coef, d_out, d_part);
    return cuda_ok(cudaGetLastError(), "launch");
  }
  if (cudaMemsetAsync(d_counter, 0, 2 * sizeof(int), s->stream) != cudaSuccess) {
    set_error("product kernel: clearing the row counter failed");
    return -1;
  }
  if (vt == kReal64)
    prod_hv_kernel<double><<<p->grid, kProdThreads, p->smem[0], s->stream>>>(
        p->args, (const double *)d_v1, (double *)d_v0, d_coef, d_part, d_counter);
  else
    prod_hv_kernel<cplx><<<p->grid, kProdThreads, p->smem[1], s->stream>>>(p->args, (const cplx *)d_v1,
                                                                           (cplx *)d_v0, d_coef, d_part, d_counter);
  finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(d_part, p->args.Uc, d_out);
  return cuda_ok(cudaGetLastError(), "launch");
}

int prod_hv_launch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out) {
  ProdPlan *p = s->prod;
  if (vt == kReal64 && s->model.complex_terms) {
    set_error("H has complex coefficients: real vectors are not allowed");
    return -1;
  }
  if (vt == kReal64 && p->two_pass) {
    two_pass_launch(s, (const double *)d_v1, (double *)d_v0, d_coef, d_out, p->part);
    return cuda_ok(cudaGetLastError(), "launch");
  }
  if (vt == kReal64)
    prod_hv_kernel<double><<<p->grid, kProdThreads, p->smem[0], s->stream>>>(
        p->args, (const double *)d_v1, (double *)d_v0, d_coef, p->part, p->counter);
  else
    prod_hv_kernel<cplx><<<p->grid, kProdThreads, p->smem[1], s->stream>>>(p->args, (const cplx *)d_v1,
                                                                           (cplx *)d_v0, d_coef, p->part, p->counter);
  finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(p->part, p->args.Uc, d_out);
  return cuda_ok(cudaGetLastError(), "launch");
}

int prod_permute(Sector *s, VecType vt, const void *in, void *out, bool to_native) {
  ProdPlan *p = s->prod;
  const unsigned nb = (unsigned)std::min<int64_t>((s->dim + 255) / 256, (int64_t)s->num_sms * 16);
  const int N = p->args.N, Dc = p->args.Dc;
  if (to_native && s->d_list_2_1 && s->d_list_2_2) {
    const uint64_t lo_mask = s->ihfbit - 1;
    if (vt == kReal64)
      prod_to_native_gather_kernel<double><<<nb, 256, 0, s->stream>>>(
          s->dim, N, Dc, p->args.unrank_up, p->args.unrank_dn, s->d_list_2_1, s->d_list_2_2, s->lo_bits, lo_mask,
          (const double *)in, (double *)out);
    else
      prod_to_native_gather_kernel<cplx><<<nb, 256, 0, s->stream>>>(
          s->dim, N, Dc, p->args.unrank_up, p->args.unrank_dn, s->d_list_2_1, s->d_list_2_2, s->lo_bits, lo_mask,
          (const cplx *)in, (cplx *)out);
    return cuda_ok(cudaGetLastError(), "permute");
  }
  if (vt == kReal64) {
    if (to_native)
      prod_permute_kernel<double, true, true><<<nb, 256, 0, s->stream>>>(s->dim, N, Dc, s->d_list_1, p->args.rank, p->args.pos_dn,
                                                                         (const double *)in, (double *)out);
    else
      prod_permute_kernel<double, false, true><<<nb, 256, 0, s->stream>>>(s->dim, N, Dc, s->d_list_1, p->args.rank, p->args.pos_dn,
                                                                          (const double *)in, (double *)out);
  } else {
    if (to_native)
      prod_permute_kernel<cplx, true, true><<<nb, 256, 0, s->stream>>>(s->dim, N, Dc, s->d_list_1, p->args.rank, p->args.pos_dn,
                                                                       (const cplx *)in, (cplx *)out);
    else
      prod_permute_kernel<cplx, false, true><<<nb, 256, 0, s->stream>>>(s->dim, N, Dc, s->d_list_1, p->args.rank, p->args.pos_dn,
                                                                        (const cplx *)in, (cplx *)out);
  }
  return cuda_ok(cudaGetLastError(), "permute");
}

int prod_observables(Sector *s, VecType vt, const void *v, double *d_out) {
  ProdPlan *p = s->prod;
  const int nb = s->red_blocks;
  if (vt == kReal64)
    prod_obs_kernel<double><<<nb, 256, 0, s->stream>>>(p->args, (const double *)v, s->d_red);
  else
    prod_obs_kernel<cplx><<<nb, 256, 0, s->stream>>>(p->args, (const cplx *)v, s->d_red);
  finalize_partials_kernel<6><<<1, 256, 0, s->stream>>>(s->d_red, nb, d_out);
  return cuda_ok(cudaGetLastError(), "observables");
}

}  // namespace hphi
