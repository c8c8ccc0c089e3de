// Streaming vector kernels for the Lanczos / TPQ drivers.
//
// The reference does these as separate OpenMP loops over 1-based complex arrays
// (recurrence sweep src/Lanczos_EigenValue.c:153-160, beta src/Lanczos_EigenValue.c:170-177,
// TPQ Multiply src/Multiply.c:42-68).  Here every reduction writes one record per
// block and a single block sums the records, so results do not depend on timing.
#include <cuda_runtime.h>

#include <string>

#include "batch.hpp"
#include "device_util.cuh"
#include "engine.hpp"

namespace hphi {
namespace {

constexpr int kThreads = 256;

template <typename T>
__global__ void norm2_kernel(int64_t n, const T *__restrict__ x, double *__restrict__ part) {
  double v[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[0] += VT<T>::abs2(x[i]);
  block_sum<1>(v);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

template <typename T>
__global__ void dot_kernel(int64_t n, const T *__restrict__ x, const T *__restrict__ y, double *__restrict__ part) {
  double v[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    v[0] += VT<T>::conj_mul_re(x[i], y[i]);
    v[1] += VT<T>::conj_mul_im(x[i], y[i]);
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = v[0]; part[2 * blockIdx.x + 1] = v[1]; }
}

template <typename T>
__global__ void axpby_kernel(int64_t n, double a, const T *__restrict__ x, double b, T *__restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = VT<T>::add(VT<T>::scale(a, x[i]), VT<T>::scale(b, y[i]));
}

template <typename T>
__global__ void scale_kernel(int64_t n, double a, T *__restrict__ x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = VT<T>::scale(a, x[i]);
}

// p <- p - (alpha*sq) q and |p|^2, alpha*sq read from device memory.
template <typename T>
__global__ void lanczos_sweep_kernel(int64_t n, const double *__restrict__ coef, T *__restrict__ p,
                                     const T *__restrict__ q, double *__restrict__ part) {
  const double c = coef[0];
  double v[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T w = VT<T>::sub(p[i], VT<T>::scale(c, q[i]));
    p[i] = w;
    v[0] += VT<T>::abs2(w);
  }
  block_sum<1>(v);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// Occupation statistics of a configuration, as expec_energy_flct_Hubbard /
// _HalfSpinGC (src/expec_energy_flct.c:186-666): out = <D>, <D^2>, <N>, <N^2>, <Sz>, <Sz^2>
// with D = doubly occupied sites, Sz = (N_up - N_dn)/2 (Hubbard bit 2i+s; spin bit i = up).
// General spin (site_bits > 0): site i's digit is bits [site_bits*i, site_bits*(i+1)) and
// Sz = sum of digits - sum of S_i (expec_energy_flct_GeneralSpin[GC], src/expec_energy_flct.c:
// 501-540, 618-660).
template <typename T>
__global__ void diag_obs_kernel(int64_t n, int gc, int spin, int nsite, int site_bits, int sum2s,
                                const uint64_t *__restrict__ list_1, const T *__restrict__ x,
                                double *__restrict__ part) {
  double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const uint64_t even = 0x5555555555555555ull;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = gc ? (uint64_t)i : list_1[i];
    const double w = VT<T>::abs2(x[i]);
    double D, N, Sz;
    if (spin && site_bits > 0) {
      int dsum = 0;
      const uint64_t fm = (1ull << site_bits) - 1;
      for (int q = 0; q < nsite; q++) dsum += (int)((c >> (site_bits * q)) & fm);
      D = 0.0;
      N = (double)nsite;
      Sz = 0.5 * (double)(2 * dsum - sum2s);
    } else if (spin) {
      D = 0.0;
      N = (double)nsite;
      Sz = 0.5 * (double)(2 * __popcll(c) - nsite);
    } else {
      const int up = __popcll(c & even), dn = __popcll(c & ~even);
      D = (double)__popcll(c & (c >> 1) & even);
      N = (double)(up + dn);
      Sz = 0.5 * (double)(up - dn);
    }
    v[0] += w * D; v[1] += w * D * D;
    v[2] += w * N; v[3] += w * N * N;
    v[4] += w * Sz; v[5] += w * Sz * Sz;
  }
  block_sum<6>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 6; k++) part[6 * blockIdx.x + k] = v[k];
}

__global__ void real_from_c128_kernel(int64_t n, const cplx *__restrict__ src, double *__restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i].x;
}
__global__ void c128_from_real_kernel(int64_t n, const double *__restrict__ src, cplx *__restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = cplx{src[i], 0.0};
}

int check_launch(const char *what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

}  // namespace

int vec_norm2(Sector *s, VecType vt, const void *x, double *out) {
  if (vt == kReal64) norm2_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, (const double *)x, s->d_red);
  else norm2_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, (const cplx *)x, s->d_red);
  finalize_partials_kernel<1><<<1, 256, 0, s->stream>>>(s->d_red, s->red_blocks, out);
  return check_launch("vec_norm2");
}

int vec_dot(Sector *s, VecType vt, const void *x, const void *y, double *out) {
  if (vt == kReal64)
    dot_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, (const double *)x, (const double *)y, s->d_red);
  else
    dot_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, (const cplx *)x, (const cplx *)y, s->d_red);
  finalize_partials_kernel<2><<<1, 256, 0, s->stream>>>(s->d_red, s->red_blocks, out);
  return check_launch("vec_dot");
}

int vec_axpby(Sector *s, VecType vt, double a, const void *x, double b, void *y) {
  if (vt == kReal64)
    axpby_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, a, (const double *)x, b, (double *)y);
  else
    axpby_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, a, (const cplx *)x, b, (cplx *)y);
  return check_launch("vec_axpby");
}

int vec_scale(Sector *s, VecType vt, double a, void *x) {
  if (vt == kReal64) scale_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, a, (double *)x);
  else scale_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, a, (cplx *)x);
  return check_launch("vec_scale");
}

int vec_lanczos_sweep(Sector *s, VecType vt, const double *coef, void *p, const void *q, double *out) {
  if (vt == kReal64)
    lanczos_sweep_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, coef, (double *)p,
                                                                            (const double *)q, s->d_red);
  else
    lanczos_sweep_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, coef, (cplx *)p, (const cplx *)q,
                                                                          s->d_red);
  finalize_partials_kernel<1><<<1, 256, 0, s->stream>>>(s->d_red, s->red_blocks, out);
  return check_launch("vec_lanczos_sweep");
}

int vec_diag_observables(Sector *s, VecType vt, const void *x, double *out) {
  const Model &m = s->model;
  const int spin = m.is_spin() ? 1 : 0;
  const int gbits = m.general_spin ? m.site_bits : 0;
  int sum2s = 0;
  for (int q = 0; q < m.nsite && m.general_spin; q++) sum2s += m.locspn[q];
  if (vt == kReal64)
    diag_obs_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(
        s->dim, s->gc ? 1 : 0, spin, m.nsite, gbits, sum2s, s->d_list_1, (const double *)x, s->d_red);
  else
    diag_obs_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(
        s->dim, s->gc ? 1 : 0, spin, m.nsite, gbits, sum2s, s->d_list_1, (const cplx *)x, s->d_red);
  finalize_partials_kernel<6><<<1, 256, 0, s->stream>>>(s->d_red, s->red_blocks, out);
  return check_launch("vec_diag_observables");
}

int vec_from_host_c128(Sector *s, VecType vt, const double *h, void *d) {
  const size_t bytes = sizeof(cplx) * (size_t)s->dim;
  if (vt == kComplex128) {
    if (cudaMemcpyAsync(d, h + 2, bytes, cudaMemcpyHostToDevice, s->stream) != cudaSuccess) {
      set_error("vec_from_host_c128: copy failed");
      return -1;
    }
    return 0;
  }
  cplx *tmp = nullptr;
  if (cudaMallocAsync(&tmp, bytes, s->stream) != cudaSuccess) { set_error("vec_from_host_c128: out of memory"); return -1; }
  cudaMemcpyAsync(tmp, h + 2, bytes, cudaMemcpyHostToDevice, s->stream);
  real_from_c128_kernel<<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, tmp, (double *)d);
  cudaFreeAsync(tmp, s->stream);
  return check_launch("vec_from_host_c128");
}

int vec_to_host_c128(Sector *s, VecType vt, const void *d, double *h) {
  const size_t bytes = sizeof(cplx) * (size_t)s->dim;
  h[0] = 0.0;
  h[1] = 0.0;
  if (vt == kComplex128) {
    if (cudaMemcpyAsync(h + 2, d, bytes, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess) {
      set_error("vec_to_host_c128: copy failed");
      return -1;
    }
    cudaStreamSynchronize(s->stream);
    return 0;
  }
  cplx *tmp = nullptr;
  if (cudaMallocAsync(&tmp, bytes, s->stream) != cudaSuccess) { set_error("vec_to_host_c128: out of memory"); return -1; }
  c128_from_real_kernel<<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, (const double *)d, tmp);
  cudaMemcpyAsync(h + 2, tmp, bytes, cudaMemcpyDeviceToHost, s->stream);
  cudaFreeAsync(tmp, s->stream);
  cudaStreamSynchronize(s->stream);
  return check_launch("vec_to_host_c128");
}

}  // namespace hphi

namespace hphi {
namespace {

// Per-step scalar bookkeeping of the device-resident Lanczos recurrence.  st layout:
//   st[0..1] raw sum conj(Q)(HQ) from hv   st[2] acc   st[3] s (scale of Q)
//   st[4] sweep coefficient alpha*s       st[5] |w|^2 from the sweep
// phase 0 (after hv, step k):    alpha_k = s^2 Re(raw); coef = alpha_k * s
// phase 1 (after sweep, step k): beta_k = sqrt(|w|^2); acc = -beta_k * s; s = 1/beta_k
__global__ void lanczos_scalars_kernel(int phase, int k, double *st, double *alpha, double *beta) {
  if (threadIdx.x != 0) return;
  if (phase == 0) {
    const double s = st[3];
    const double a = s * s * st[0];
    alpha[k] = a;
    st[4] = a * s;
  } else {
    const double b = sqrt(st[5]);
    beta[k] = b;
    st[2] = -b * st[3];
    st[3] = 1.0 / b;
  }
}

// Eigenvector replay sweep (src/Lanczos_EigenVector.c:150-190): with the stored
// alpha_k, beta_k: w = p - alpha_k*sq*q; p = w; vg += c * w / beta_k.
template <typename T>
__global__ void replay_sweep_kernel(int64_t n, double a_sq, double c_over_b, T *__restrict__ p,
                                    const T *__restrict__ q, T *__restrict__ vg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T w = VT<T>::sub(p[i], VT<T>::scale(a_sq, q[i]));
    p[i] = w;
    vg[i] = VT<T>::add(vg[i], VT<T>::scale(c_over_b, w));
  }
}

// TPQ sweep (src/Multiply.c:42-68 with the normalisation deferred):
// w = (L*sv)*v - (sh/Ns)*h written into v, |w|^2 into part.
template <typename T>
__global__ void tpq_sweep_kernel(int64_t n, double cv, double ch, T *__restrict__ v, const T *__restrict__ h,
                                 double *__restrict__ part) {
  double acc[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T w = VT<T>::sub(VT<T>::scale(cv, v[i]), VT<T>::scale(ch, h[i]));
    v[i] = w;
    acc[0] += VT<T>::abs2(w);
  }
  block_sum<1>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
}

// CG sweep of the eigenvector refinement (src/CG_EigenVector.c:143-185) with the shifted
// product y = hp + shift*p formed on the fly: x += a*p; r -= a*y; |r|^2 into part.
template <typename T>
__global__ void cg_sweep_kernel(int64_t n, double a, double shift, const T *__restrict__ p,
                                const T *__restrict__ hp, T *__restrict__ x, T *__restrict__ r,
                                double *__restrict__ part) {
  double acc[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T pi = p[i];
    const T yi = VT<T>::add(hp[i], VT<T>::scale(shift, pi));
    x[i] = VT<T>::add(x[i], VT<T>::scale(a, pi));
    const T w = VT<T>::sub(r[i], VT<T>::scale(a, yi));
    r[i] = w;
    acc[0] += VT<T>::abs2(w);
  }
  block_sum<1>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
}

// Adds amp * start_value(seed, configuration, 0) to the real part of an HPhi-order vector
// (the random components of src/CG_EigenVector.c:84-99, keyed by configuration).
template <typename T>
__global__ void add_hashed_kernel(int64_t n, uint64_t seed, double amp, const uint64_t *__restrict__ list_1,
                                  T *__restrict__ x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = list_1 ? list_1[i] : (uint64_t)i;
    x[i] = VT<T>::add_re(x[i], amp * start_value(seed, c, 0));
  }
}

// x[i] = start_value(seed, configuration of row i, 0) (+ i start_value(.., 1) for complex
// vectors), HPhi's row order: the hashed start vector before normalisation.
template <typename T>
__global__ void fill_hashed_kernel(int64_t n, uint64_t seed, const uint64_t *__restrict__ list_1, T *__restrict__ x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = list_1 ? list_1[i] : (uint64_t)i;
    if constexpr (VT<T>::kComplex) x[i] = cplx{start_value(seed, c, 0), start_value(seed, c, 1)};
    else x[i] = start_value(seed, c, 0);
  }
}

}  // namespace

int vec_fill_hashed(Sector *s, VecType vt, uint64_t seed, void *x) {
  const uint64_t *l1 = s->gc ? nullptr : s->d_list_1;
  if (vt == kReal64)
    fill_hashed_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, seed, l1, (double *)x);
  else
    fill_hashed_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, seed, l1, (cplx *)x);
  return check_launch("vec_fill_hashed");
}

int lanczos_scalars(Sector *s, int phase, int k, double *st, double *alpha, double *beta) {
  lanczos_scalars_kernel<<<1, 32, 0, s->stream>>>(phase, k, st, alpha, beta);
  return check_launch("lanczos_scalars");
}

int vec_replay_sweep(Sector *s, VecType vt, double a_sq, double c_over_b, void *p, const void *q, void *vg) {
  if (vt == kReal64)
    replay_sweep_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, a_sq, c_over_b, (double *)p,
                                                                           (const double *)q, (double *)vg);
  else
    replay_sweep_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, a_sq, c_over_b, (cplx *)p,
                                                                         (const cplx *)q, (cplx *)vg);
  return check_launch("vec_replay_sweep");
}

int vec_tpq_sweep(Sector *s, VecType vt, double cv, double ch, void *v, const void *h, double *out) {
  if (vt == kReal64)
    tpq_sweep_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, cv, ch, (double *)v,
                                                                        (const double *)h, s->d_red);
  else
    tpq_sweep_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, cv, ch, (cplx *)v, (const cplx *)h,
                                                                      s->d_red);
  finalize_partials_kernel<1><<<1, 256, 0, s->stream>>>(s->d_red, s->red_blocks, out);
  return check_launch("vec_tpq_sweep");
}

}  // namespace hphi

namespace hphi {

int vec_cg_sweep(Sector *s, VecType vt, double a, double shift, const void *p, const void *hp, void *x, void *r,
                 double *out) {
  if (vt == kReal64)
    cg_sweep_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(
        s->dim, a, shift, (const double *)p, (const double *)hp, (double *)x, (double *)r, s->d_red);
  else
    cg_sweep_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, a, shift, (const cplx *)p,
                                                                     (const cplx *)hp, (cplx *)x, (cplx *)r, s->d_red);
  finalize_partials_kernel<1><<<1, 256, 0, s->stream>>>(s->d_red, s->red_blocks, out);
  return check_launch("vec_cg_sweep");
}

int vec_add_hashed(Sector *s, VecType vt, uint64_t seed, double amp, void *x) {
  const uint64_t *l1 = s->gc ? nullptr : s->d_list_1;
  if (vt == kReal64)
    add_hashed_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, seed, amp, l1, (double *)x);
  else
    add_hashed_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, seed, amp, l1, (cplx *)x);
  return check_launch("vec_add_hashed");
}

}  // namespace hphi

namespace hphi {
namespace {
__global__ void split_c128_kernel(int64_t n, const cplx *__restrict__ c, double *__restrict__ re,
                                  double *__restrict__ im) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const cplx v = c[i];
    re[i] = v.x;
    im[i] = v.y;
  }
}
__global__ void join_c128_kernel(int64_t n, const double *__restrict__ re, const double *__restrict__ im,
                                 cplx *__restrict__ c) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    c[i] = cplx{re[i], im[i]};
}
__global__ void add_c128_kernel(int64_t n, cplx *__restrict__ y, const cplx *__restrict__ x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = y[i] + x[i];
}
}  // namespace

int vec_split_c128(Sector *s, const void *c, double *re, double *im) {
  split_c128_kernel<<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, (const cplx *)c, re, im);
  return check_launch("vec_split_c128");
}

int vec_join_c128(Sector *s, const double *re, const double *im, void *c) {
  join_c128_kernel<<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, re, im, (cplx *)c);
  return check_launch("vec_join_c128");
}

int vec_add_c128(Sector *s, cudaStream_t st, int64_t n, void *y, const void *x) {
  add_c128_kernel<<<s->num_sms * 4, kThreads, 0, st>>>(n, (cplx *)y, (const cplx *)x);
  return check_launch("vec_add_c128");
}

}  // namespace hphi

