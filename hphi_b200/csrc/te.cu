// Time-dependent terms of the real-time evolution (CalcType 4).
//
// The reference adds the terms of time index `step` to its Hamiltonian before each
// mltply of that step: the off-diagonal ones are appended to the transfer / InterAll
// lists the term passes walk (MakeTEDTransfer / MakeTEDInterAll, src/CalcByTEM.c:237-279),
// the diagonal ones are applied after the diagonal pass (diagonalcalcForTE,
// src/diagonalcalc.c:195-245, called from src/mltply.c:49).  Here the static part of H
// runs through the general row kernel and te_terms_kernel adds the step's terms to the
// same output rows: one thread per row in gather form, the same test / flip / two-level
// lookup / parity sign as the static terms, so no output row is written twice.  The masks of
// the time-dependent rows are fixed, their values change with the time index: the terms whose
// masks lie in one half of the configuration go through a split-term plan (split.cuh) built
// once for all indices, with one coefficient table per index; the others are tested per row.
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "engine.hpp"
#include "split.cuh"

namespace hphi {
namespace {

constexpr int kThreads = 256;

constexpr int kSmemTermMax = 1024;  // 48 KiB of BitTerm

// SMEM: the step's off-diagonal terms are staged in shared memory (every row reads all of them).
template <bool GC, bool SMEM>
__global__ void __launch_bounds__(kThreads) te_terms_kernel(
    int64_t dim, const uint64_t *__restrict__ list_1, const uint32_t *__restrict__ l21,
    const uint32_t *__restrict__ l22, int lo_bits, uint64_t lo_mask, SplitView split,
    const BitTerm *__restrict__ goff, int noff, const DiagTerm *__restrict__ dg, int ndg,
    const cplx *__restrict__ v1, cplx *__restrict__ v0) {
  extern __shared__ BitTerm sterms[];
  const BitTerm *off = goff;
  if (SMEM) {
    for (int k = threadIdx.x; k < noff; k += blockDim.x) sterms[k] = goff[k];
    __syncthreads();
    off = sterms;
  }
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = GC ? (uint64_t)r : list_1[r];
    const cplx x = v1[r];
    double d = 0.0;
    for (int k = 0; k < ndg; k++)
      if ((c & dg[k].cm) == dg[k].cv) d += dg[k].v;
    double yr = d * x.x, yi = d * x.y;
    if (split.lo_ptr) {
      const cplx t = split_terms<cplx, GC>(split, c, r, lo_bits, lo_mask, l22, [&](int64_t j) { return v1[j]; },
                                           cplx{0.0, 0.0});
      yr += t.x;
      yi += t.y;
    }
    for (int k = 0; k < noff; k++) {
      const BitTerm t = off[k];
      if ((c & t.cm) != t.cv) continue;
      const uint64_t src = c ^ t.flip;
      int64_t j;
      if (GC) {
        j = (int64_t)src;
      } else {
        const uint32_t a = l21[src & lo_mask];
        const uint32_t b = l22[src >> lo_bits];
        if (a == 0u || b == 0u) continue;
        j = (int64_t)a + (int64_t)b - 3;
      }
      const bool neg = __popcll(c & t.sm) & 1;
      const double cr = neg ? -t.re : t.re, ci = neg ? -t.im : t.im;
      const cplx u = v1[j];
      yr += cr * u.x - ci * u.y;
      yi += cr * u.y + ci * u.x;
    }
    cplx o = v0[r];
    o.x += yr;
    o.y += yi;
    v0[r] = o;
  }
}

__global__ void caxpy_kernel(int64_t n, double ar, double ai, const cplx *__restrict__ x, cplx *__restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const cplx a = x[i];
    cplx b = y[i];
    b.x += ar * a.x - ai * a.y;
    b.y += ar * a.y + ai * a.x;
    y[i] = b;
  }
}

}  // namespace

int te_terms_apply(Sector *s, const SplitPlan &plan, const double *d_coef, const BitTerm *d_off, int noff,
                   const DiagTerm *d_diag, int ndiag, const void *d_v1, void *d_v0) {
  if (noff == 0 && ndiag == 0 && !plan.lo_ptr) return 0;
  SplitView sv = split_view(plan);
  sv.coef = d_coef;
  const uint64_t lo_mask = s->ihfbit - 1;
  const bool smem = noff <= kSmemTermMax;
  const size_t bytes = smem ? sizeof(BitTerm) * (size_t)noff : 0;
#define HPHI_TE_LAUNCH(GC, SM)                                                                              \
  te_terms_kernel<GC, SM><<<s->red_blocks, kThreads, bytes, s->stream>>>(                                   \
      s->dim, s->d_list_1, s->d_list_2_1, s->d_list_2_2, s->lo_bits, lo_mask, sv, d_off, noff, d_diag, ndiag, \
      (const cplx *)d_v1, (cplx *)d_v0)
  if (s->gc) {
    if (smem) HPHI_TE_LAUNCH(true, true);
    else HPHI_TE_LAUNCH(true, false);
  } else {
    if (smem) HPHI_TE_LAUNCH(false, true);
    else HPHI_TE_LAUNCH(false, false);
  }
#undef HPHI_TE_LAUNCH
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("te_terms launch failed: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

int vec_caxpy(Sector *s, double a_re, double a_im, const void *d_x, void *d_y) {
  caxpy_kernel<<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, a_re, a_im, (const cplx *)d_x, (cplx *)d_y);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("caxpy launch failed: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

}  // namespace hphi
