// Matrix-free H*v, general path: every off-diagonal term in gather form.
//
// Replaces mltply (src/mltply.c:56-132) and the term passes it dispatches to
// (mltplyHubbard / mltplyHubbardGC, src/mltplyHubbard.c:150-528; mltplyHalfSpin /
// mltplyHalfSpinGC, src/mltplySpin.c:192-703).  The reference makes one full pass over
// the vector per term and scatters v0[off(j)] += c * v1[j]; here each output row is
// owned by one thread, which walks the compiled terms once, tests the row's
// configuration against each term's pattern, and gathers the matching source element:
//   s = c ^ flip,  row(s) = list_2_1[s & (ihfbit-1)] + list_2_2[s >> lo_bits] - 3,
//   sign = (-1)^popcount(c & sign_mask)            (GetOffComp / SgnBit, src/bitcalc.c).
// Output rows are written exactly once, so there are no races and no atomics, and the
// fused <v1|H|v1> of the reference (X->Large.prdct) comes from a block reduction of
// conj(v1[r]) * (H v1)[r].
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "engine.hpp"
#include "hv_hubbard.hpp"
#include "hv_product.hpp"
#include "hv_rowblock.hpp"
#include "split.cuh"

namespace hphi {
namespace {

constexpr int kHvThreads = 256;
constexpr int kSmemTermMax = 1024;  // 48 KiB of BitTerm

template <typename T, bool GC, bool SMEM>
__global__ void __launch_bounds__(kHvThreads) hv_general_kernel(
    int64_t dim, const uint64_t *__restrict__ list_1, const uint32_t *__restrict__ l21,
    const uint32_t *__restrict__ l22, int lo_bits, uint64_t lo_mask, SplitView split,
    const BitTerm *__restrict__ gterms, int nterms, const double *__restrict__ diag, const T *__restrict__ v1,
    T *__restrict__ v0, const double *__restrict__ coef, double *__restrict__ part) {
  const double acc = coef[0], scale = coef[1];
  extern __shared__ BitTerm sterms[];
  const BitTerm *terms = gterms;
  if (SMEM) {
    for (int k = threadIdx.x; k < nterms; k += blockDim.x) sterms[k] = gterms[k];
    __syncthreads();
    terms = sterms;
  }
  double pr[2] = {0.0, 0.0};
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = GC ? (uint64_t)r : list_1[r];
    const T x = v1[r];
    T y = VT<T>::scale(diag[r], x);
    if (split.lo_ptr) y = split_terms<T, GC>(split, c, r, lo_bits, lo_mask, l22, [&](int64_t j) { return v1[j]; }, y);
    for (int k = 0; k < nterms; k++) {
      const BitTerm t = terms[k];
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
      const double sg = (__popcll(c & t.sm) & 1) ? -t.re : t.re;
      const double sgi = (__popcll(c & t.sm) & 1) ? -t.im : t.im;
      y = VT<T>::add(y, VT<T>::cmul_re_im(sg, sgi, v1[j]));
    }
    pr[0] += VT<T>::conj_mul_re(x, y);
    pr[1] += VT<T>::conj_mul_im(x, y);
    y = VT<T>::scale(scale, y);
    v0[r] = (acc == 0.0) ? y : VT<T>::add(VT<T>::scale(acc, v0[r]), y);
  }
  block_sum<2>(pr);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = pr[0];
    part[2 * blockIdx.x + 1] = pr[1];
  }
}

template <typename T, bool GC>
void launch_general(Sector *s, const T *v1, T *v0, const double *coef) {
  const int grid = s->red_blocks;
  const uint64_t lo_mask = s->ihfbit - 1;
  const SplitView sv = split_view(s->split);
  if (s->split.ngen <= kSmemTermMax) {
    const size_t smem = sizeof(BitTerm) * (size_t)s->split.ngen;
    hv_general_kernel<T, GC, true><<<grid, kHvThreads, smem, s->stream>>>(
        s->dim, s->d_list_1, s->d_list_2_1, s->d_list_2_2, s->lo_bits, lo_mask, sv, s->split.gen, s->split.ngen,
        s->d_diag, v1, v0, coef, s->d_red);
  } else {
    hv_general_kernel<T, GC, false><<<grid, kHvThreads, 0, s->stream>>>(
        s->dim, s->d_list_1, s->d_list_2_1, s->d_list_2_2, s->lo_bits, lo_mask, sv, s->split.gen, s->split.ngen,
        s->d_diag, v1, v0, coef, s->d_red);
  }
}

// B vectors at once (independent samples of one sector, vector b at v + b * stride): the
// configuration, diagonal, split-plan entries, list lookups and signs of a row are worked out
// once and applied to all B, which is where the general kernel spends its memory traffic.
// Per vector the arithmetic and its order are the general kernel's, so every output equals a
// separate launch bit for bit.  Coefficients (acc, scale) of vector b at coef + b * cstride;
// partial sums of <v1_b|H v1_b> in part[(2B) * block + 2b (+1)].
template <typename T, int B>
struct Blk {
  T v[B];
};

template <typename T, int B>
struct BlkOps {
  static __device__ __forceinline__ Blk<T, B> add(Blk<T, B> a, const Blk<T, B> &b) {
#pragma unroll
    for (int q = 0; q < B; q++) a.v[q] = VT<T>::add(a.v[q], b.v[q]);
    return a;
  }
  static __device__ __forceinline__ Blk<T, B> cmul_re_im(double re, double im, const Blk<T, B> &x) {
    Blk<T, B> r;
#pragma unroll
    for (int q = 0; q < B; q++) r.v[q] = VT<T>::cmul_re_im(re, im, x.v[q]);
    return r;
  }
};

template <typename T, bool GC, bool SMEM, int B>
__global__ void __launch_bounds__(kHvThreads) hv_block_kernel(
    int64_t dim, int64_t stride, const uint64_t *__restrict__ list_1, const uint32_t *__restrict__ l21,
    const uint32_t *__restrict__ l22, int lo_bits, uint64_t lo_mask, SplitView split,
    const BitTerm *__restrict__ gterms, int nterms, const double *__restrict__ diag, const T *__restrict__ v1,
    T *__restrict__ v0, const double *__restrict__ coef, int cstride, double *__restrict__ part) {
  extern __shared__ BitTerm sterms[];
  const BitTerm *terms = gterms;
  if (SMEM) {
    for (int k = threadIdx.x; k < nterms; k += blockDim.x) sterms[k] = gterms[k];
    __syncthreads();
    terms = sterms;
  }
  double pr[2 * B];
#pragma unroll
  for (int q = 0; q < 2 * B; q++) pr[q] = 0.0;
  auto load = [&](int64_t j) {
    Blk<T, B> z;
#pragma unroll
    for (int q = 0; q < B; q++) z.v[q] = v1[q * stride + j];
    return z;
  };
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = GC ? (uint64_t)r : list_1[r];
    const Blk<T, B> x = load(r);
    const double dg = diag[r];
    Blk<T, B> y;
#pragma unroll
    for (int q = 0; q < B; q++) y.v[q] = VT<T>::scale(dg, x.v[q]);
    if (split.lo_ptr) {
      // split_terms with the block accumulator (same entries, same order)
      const uint32_t ia = (uint32_t)(c & lo_mask);
      const uint64_t ib = c >> lo_bits;
      const int64_t base = GC ? (int64_t)(c & ~lo_mask) : (int64_t)__ldg(l22 + ib) - 3;
      const uint32_t l0 = __ldg(split.lo_ptr + ia), l1 = __ldg(split.lo_ptr + ia + 1);
      for (uint32_t e = l0; e < l1; e++) {
        const uint32_t v = __ldg(split.lo_ent + e);
        const uint32_t tgt = v & ((1u << kSplitTargetBits) - 1u);
        const uint32_t k = v >> kSplitTargetBits;
        const int64_t j = GC ? (base | (int64_t)tgt) : base + (int64_t)tgt;
        const double2 cf = __ldg(reinterpret_cast<const double2 *>(split.coef) + k);
        y = BlkOps<T, B>::add(y, BlkOps<T, B>::cmul_re_im(cf.x, cf.y, load(j)));
      }
      const uint32_t h0 = __ldg(split.hi_ptr + ib), h1 = __ldg(split.hi_ptr + ib + 1);
      for (uint32_t e = h0; e < h1; e++) {
        const HiEnt h = split.hi_ent[e];
        const int64_t j = GC ? (int64_t)((uint64_t)r ^ (uint64_t)h.delta) : r + h.delta;
        const double2 cf = __ldg(reinterpret_cast<const double2 *>(split.coef) + h.k);
        y = BlkOps<T, B>::add(y, BlkOps<T, B>::cmul_re_im(cf.x, cf.y, load(j)));
      }
    }
    for (int k = 0; k < nterms; k++) {
      const BitTerm t = terms[k];
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
      const double sg = (__popcll(c & t.sm) & 1) ? -t.re : t.re;
      const double sgi = (__popcll(c & t.sm) & 1) ? -t.im : t.im;
      y = BlkOps<T, B>::add(y, BlkOps<T, B>::cmul_re_im(sg, sgi, load(j)));
    }
#pragma unroll
    for (int q = 0; q < B; q++) {
      pr[2 * q] += VT<T>::conj_mul_re(x.v[q], y.v[q]);
      pr[2 * q + 1] += VT<T>::conj_mul_im(x.v[q], y.v[q]);
      const double acc = coef[q * cstride], scale = coef[q * cstride + 1];
      const T yq = VT<T>::scale(scale, y.v[q]);
      T *o = v0 + q * stride + r;
      *o = (acc == 0.0) ? yq : VT<T>::add(VT<T>::scale(acc, *o), yq);
    }
  }
  block_sum<2 * B>(pr);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 2 * B; q++) part[2 * B * blockIdx.x + q] = pr[q];
}

// out[q * ostride + (0, 1)] = sum over blocks of part[(2B) * block + 2q (+1)]
template <int B>
__global__ void finalize_block_partials_kernel(const double *__restrict__ part, int n, double *__restrict__ out,
                                               int ostride) {
  double v[2 * B];
#pragma unroll
  for (int k = 0; k < 2 * B; k++) v[k] = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
#pragma unroll
    for (int k = 0; k < 2 * B; k++) v[k] += part[i * 2 * B + k];
  block_sum<2 * B>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < B; q++) {
      out[q * ostride] = v[2 * q];
      out[q * ostride + 1] = v[2 * q + 1];
    }
}

template <typename T, bool GC, int B>
void launch_block(Sector *s, int64_t stride, const T *v1, T *v0, const double *coef, int cstride, double *out,
                  int ostride, double *part) {
  const int grid = s->red_blocks;
  const uint64_t lo_mask = s->ihfbit - 1;
  const SplitView sv = split_view(s->split);
  if (s->split.ngen <= kSmemTermMax) {
    const size_t smem = sizeof(BitTerm) * (size_t)s->split.ngen;
    hv_block_kernel<T, GC, true, B><<<grid, kHvThreads, smem, s->stream>>>(
        s->dim, stride, s->d_list_1, s->d_list_2_1, s->d_list_2_2, s->lo_bits, lo_mask, sv, s->split.gen,
        s->split.ngen, s->d_diag, v1, v0, coef, cstride, part);
  } else {
    hv_block_kernel<T, GC, false, B><<<grid, kHvThreads, 0, s->stream>>>(
        s->dim, stride, s->d_list_1, s->d_list_2_1, s->d_list_2_2, s->lo_bits, lo_mask, sv, s->split.gen,
        s->split.ngen, s->d_diag, v1, v0, coef, cstride, part);
  }
  finalize_block_partials_kernel<B><<<1, 256, 0, s->stream>>>(part, grid, out, ostride);
}

template <typename T, bool GC>
void launch_block_n(Sector *s, int nb, int64_t stride, const T *v1, T *v0, const double *coef, int cstride,
                    double *out, int ostride, double *part) {
  switch (nb) {
    case 1: launch_block<T, GC, 1>(s, stride, v1, v0, coef, cstride, out, ostride, part); break;
    case 2: launch_block<T, GC, 2>(s, stride, v1, v0, coef, cstride, out, ostride, part); break;
    case 3: launch_block<T, GC, 3>(s, stride, v1, v0, coef, cstride, out, ostride, part); break;
    case 4: launch_block<T, GC, 4>(s, stride, v1, v0, coef, cstride, out, ostride, part); break;
    case 5: launch_block<T, GC, 5>(s, stride, v1, v0, coef, cstride, out, ostride, part); break;
    case 6: launch_block<T, GC, 6>(s, stride, v1, v0, coef, cstride, out, ostride, part); break;
    case 7: launch_block<T, GC, 7>(s, stride, v1, v0, coef, cstride, out, ostride, part); break;
    default: launch_block<T, GC, 8>(s, stride, v1, v0, coef, cstride, out, ostride, part); break;
  }
}

}  // namespace

bool hv_block_applies(const Sector *s, VecType vt) {
  return !s->prod && !s->hub && !rb_applies(s, vt) && !(vt == kReal64 && s->model.complex_terms);
}

int hv_block_native(Sector *s, VecType vt, int nb, int64_t stride, const void *d_v1, void *d_v0,
                    const double *d_coef, int cstride, double *d_out, int ostride, double *d_part) {
  if (nb < 1 || nb > kHvBlockMax || !hv_block_applies(s, vt)) {
    set_error("hv_block_native: block products need the general kernel and 1..8 vectors");
    return -1;
  }
  if (vt == kReal64) {
    if (s->gc) launch_block_n<double, true>(s, nb, stride, (const double *)d_v1, (double *)d_v0, d_coef, cstride,
                                            d_out, ostride, d_part);
    else launch_block_n<double, false>(s, nb, stride, (const double *)d_v1, (double *)d_v0, d_coef, cstride,
                                       d_out, ostride, d_part);
  } else {
    if (s->gc) launch_block_n<cplx, true>(s, nb, stride, (const cplx *)d_v1, (cplx *)d_v0, d_coef, cstride, d_out,
                                          ostride, d_part);
    else launch_block_n<cplx, false>(s, nb, stride, (const cplx *)d_v1, (cplx *)d_v0, d_coef, cstride, d_out,
                                     ostride, d_part);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("block hv launch failed: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

int hv_launch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out) {
  if (vt == kReal64 && s->model.complex_terms) {
    set_error("H has complex coefficients: real vectors are not allowed");
    return -1;
  }
  if (rb_applies(s, vt)) return rb_hv_launch(s, vt, d_v1, d_v0, d_coef, d_out);
  if (vt == kReal64) {
    if (s->gc) launch_general<double, true>(s, (const double *)d_v1, (double *)d_v0, d_coef);
    else launch_general<double, false>(s, (const double *)d_v1, (double *)d_v0, d_coef);
  } else {
    if (s->gc) launch_general<cplx, true>(s, (const cplx *)d_v1, (cplx *)d_v0, d_coef);
    else launch_general<cplx, false>(s, (const cplx *)d_v1, (cplx *)d_v0, d_coef);
  }
  finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(s->d_red, s->red_blocks, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("hv launch failed: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

int hv_launch_scratch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                      double *d_part) {
  if (vt == kReal64 && s->model.complex_terms) {
    set_error("H has complex coefficients: real vectors are not allowed");
    return -1;
  }
  if (rb_applies(s, vt)) return rb_hv_launch_scratch(s, vt, d_v1, d_v0, d_coef, d_out, d_part);
  const int grid = s->red_blocks;
  const uint64_t lo_mask = s->ihfbit - 1;
  const bool smem_terms = s->split.ngen <= kSmemTermMax;
  const size_t smem = smem_terms ? sizeof(BitTerm) * (size_t)s->split.ngen : 0;
  const SplitView sv = split_view(s->split);
#define HPHI_GENERAL_LAUNCH(T, GC)                                                                              \
  do {                                                                                                          \
    if (smem_terms)                                                                                             \
      hv_general_kernel<T, GC, true><<<grid, kHvThreads, smem, s->stream>>>(                                    \
          s->dim, s->d_list_1, s->d_list_2_1, s->d_list_2_2, s->lo_bits, lo_mask, sv, s->split.gen,             \
          s->split.ngen, s->d_diag, (const T *)d_v1, (T *)d_v0, d_coef, d_part);                               \
    else                                                                                                        \
      hv_general_kernel<T, GC, false><<<grid, kHvThreads, 0, s->stream>>>(                                      \
          s->dim, s->d_list_1, s->d_list_2_1, s->d_list_2_2, s->lo_bits, lo_mask, sv, s->split.gen,             \
          s->split.ngen, s->d_diag, (const T *)d_v1, (T *)d_v0, d_coef, d_part);                               \
  } while (0)
  if (vt == kReal64) {
    if (s->gc) HPHI_GENERAL_LAUNCH(double, true);
    else HPHI_GENERAL_LAUNCH(double, false);
  } else {
    if (s->gc) HPHI_GENERAL_LAUNCH(cplx, true);
    else HPHI_GENERAL_LAUNCH(cplx, false);
  }
#undef HPHI_GENERAL_LAUNCH
  finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(d_part, grid, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("hv launch failed: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

size_t hv_scratch_doubles(const Sector *s, VecType vt) {
  if (s->prod) return prod_scratch_doubles(s, vt);
  if (s->hub) return hub_scratch_doubles(s);
  if (rb_applies(s, vt)) return rb_scratch_doubles(s);
  return 2 * (size_t)s->red_blocks;
}

int hv_native_scratch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                      double *d_part, int *d_counter) {
  if (s->prod) return prod_hv_launch_scratch(s, vt, d_v1, d_v0, d_coef, d_out, d_part, d_counter);
  if (s->hub) return hub_hv_launch_scratch(s, vt, d_v1, d_v0, d_coef, d_out, d_part, d_counter);
  return hv_launch_scratch(s, vt, d_v1, d_v0, d_coef, d_out, d_part);
}

bool has_native_order(const Sector *s) { return s->hub != nullptr || s->prod != nullptr; }

int hv_native(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
              bool acc_read) {
  if (s->prod) return prod_hv_launch(s, vt, d_v1, d_v0, d_coef, d_out);
  if (s->hub) return hub_hv_launch(s, vt, d_v1, d_v0, d_coef, d_out, acc_read);
  return hv_launch(s, vt, d_v1, d_v0, d_coef, d_out);
}

int to_native(Sector *s, VecType vt, const void *in, void *out) {
  if (s->prod) return prod_permute(s, vt, in, out, true);
  if (s->hub) return hub_permute(s, vt, in, out, true);
  const size_t esz = (vt == kReal64) ? sizeof(double) : sizeof(cplx);
  if (in != out && cudaMemcpyAsync(out, in, esz * (size_t)s->dim, cudaMemcpyDeviceToDevice, s->stream) != cudaSuccess) {
    set_error("to_native: copy failed");
    return -1;
  }
  return 0;
}

int from_native(Sector *s, VecType vt, const void *in, void *out) {
  if (s->prod) return prod_permute(s, vt, in, out, false);
  if (s->hub) return hub_permute(s, vt, in, out, false);
  const size_t esz = (vt == kReal64) ? sizeof(double) : sizeof(cplx);
  if (in != out && cudaMemcpyAsync(out, in, esz * (size_t)s->dim, cudaMemcpyDeviceToDevice, s->stream) != cudaSuccess) {
    set_error("from_native: copy failed");
    return -1;
  }
  return 0;
}

int native_observables(Sector *s, VecType vt, const void *v, double *d_out) {
  if (s->prod) return prod_observables(s, vt, v, d_out);
  if (s->hub) return hub_observables(s, vt, v, d_out);
  return vec_diag_observables(s, vt, v, d_out);
}

}  // namespace hphi
