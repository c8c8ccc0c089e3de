// Green's functions <v| O_e |v> for batches of operator strings.
//
// Replaces the per-entry passes of expec_cisajs (src/expec_cisajs.c:66-641) and
// expec_cisajscktaltdc (src/expec_cisajscktaltdc.c:87-1647).  The reference makes one full
// pass over the vector for every entry, each row testing the entry's occupation pattern,
// looking up the row of the changed configuration (GetOffComp, src/bitcalc.c:195-223) and
// adding conj(v[off]) * sgn * v[j].  Here one pass serves a batch of entries: each thread
// reads its row's configuration and vector element once and evaluates every entry of the
// batch on it, accumulating in registers; the batch's masks are kernel parameters (constant
// bank operands of the unrolled entry loop); a fixed-order block reduction and a fixed-order
// sum over blocks make the result reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "device_util.cuh"
#include "engine.hpp"

namespace hphi {
namespace {

constexpr int kGreenThreads = 256;
constexpr int kGreenAcc = 16;  // doubles accumulated per thread: 16 real or 8 complex entries

template <typename T> struct GreenWidth;
template <> struct GreenWidth<double> { static constexpr int w = 1; };
template <> struct GreenWidth<cplx> { static constexpr int w = 2; };

template <typename T>
__device__ __forceinline__ void green_acc(double (&acc)[kGreenAcc], int k, double sg, const T &y, const T &x);
template <>
__device__ __forceinline__ void green_acc<double>(double (&acc)[kGreenAcc], int k, double sg, const double &y,
                                                  const double &x) {
  acc[k] += sg * (y * x);
}
template <>
__device__ __forceinline__ void green_acc<cplx>(double (&acc)[kGreenAcc], int k, double sg, const cplx &y,
                                                const cplx &x) {
  // conj(y) * x
  acc[2 * k] += sg * (y.x * x.x + y.y * x.y);
  acc[2 * k + 1] += sg * (y.x * x.y - y.y * x.x);
}

// A batch of entries passed by value: the masks sit in the kernel's parameter (constant)
// bank and enter the unrolled entry loop as instruction operands.  Unused slots hold a
// pattern no configuration matches (cm = 0, cv = 1).
template <int NB> struct GreenBatch { GreenTerm t[NB]; };

// One batch over all rows (grid-stride, one row per thread); per-block sums of the kGreenAcc
// accumulators go to part[blockIdx.x * kGreenAcc ...].
// C: the configuration word, uint32_t when every configuration fits in 32 bits (halves the
// mask, flip and parity work), else uint64_t.
template <typename C> __device__ __forceinline__ int parity_of(C x);
template <> __device__ __forceinline__ int parity_of<uint32_t>(uint32_t x) { return __popc(x) & 1; }
template <> __device__ __forceinline__ int parity_of<uint64_t>(uint64_t x) { return __popcll(x) & 1; }

template <typename T, bool GC, typename C>
__global__ void __launch_bounds__(kGreenThreads) green_kernel(int64_t dim, const uint64_t *__restrict__ list_1,
                                                              const uint32_t *__restrict__ l21,
                                                              const uint32_t *__restrict__ l22, int lo_bits,
                                                              uint64_t lo_mask,
                                                              const GreenBatch<kGreenAcc / GreenWidth<T>::w> batch,
                                                              const T *__restrict__ v, double *__restrict__ part) {
  constexpr int NB = kGreenAcc / GreenWidth<T>::w;
  double acc[kGreenAcc];
#pragma unroll
  for (int q = 0; q < kGreenAcc; q++) acc[q] = 0.0;
  const C lmask = (C)lo_mask;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
    const C c = GC ? (C)r : (C)__ldg(list_1 + r);
    const T x = v[r];
#pragma unroll
    for (int k = 0; k < NB; k++) {
      const GreenTerm &t = batch.t[k];
      bool hit = (c & (C)t.cm) == (C)t.cv;
      int64_t j = r;
      if (hit && t.flip) {
        const C tg = c ^ (C)t.flip;
        if (GC) {
          j = (int64_t)tg;
        } else {
          const uint32_t a = __ldg(l21 + (tg & lmask));
          const uint32_t b = __ldg(l22 + (tg >> lo_bits));
          hit = a != 0u && b != 0u;
          j = (int64_t)a + (int64_t)b - 3;
        }
      }
      if (hit) {
        const double sg = parity_of<C>(c & (C)t.sm) ? -t.coef : t.coef;
        green_acc<T>(acc, k, sg, (j == r) ? x : v[j], x);
      }
    }
  }
  block_sum<kGreenAcc>(acc);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < kGreenAcc; q++) part[(size_t)blockIdx.x * kGreenAcc + q] = acc[q];
}

template <typename T>
int green_batches(Sector *s, const T *d_v, const std::vector<GreenTerm> &nz, double *d_terms_out) {
  constexpr int NB = kGreenAcc / GreenWidth<T>::w;
  const int grid = s->red_blocks;
  const int nbatch = (int)((nz.size() + NB - 1) / NB);
  double *d_part = nullptr;
  if (cudaMalloc(&d_part, sizeof(double) * (size_t)grid * kGreenAcc) != cudaSuccess) {
    set_error("Green's functions: device allocation failed");
    return -1;
  }
  int rc = 0;
  const uint64_t lo_mask = s->ihfbit - 1;
  for (int b = 0; b < nbatch && rc == 0; b++) {
    const int nb = std::min<int>(NB, (int)nz.size() - b * NB);
    GreenBatch<NB> batch;
    for (int k = 0; k < NB; k++) batch.t[k] = k < nb ? nz[(size_t)b * NB + k] : GreenTerm{0, 1, 0, 0, 0.0, 0.0};
#define HPHI_GREEN_LAUNCH(GCV, CW)                                                                          \
  green_kernel<T, GCV, CW><<<grid, kGreenThreads, 0, s->stream>>>(s->dim, s->d_list_1, s->d_list_2_1,       \
                                                                  s->d_list_2_2, s->lo_bits, lo_mask, batch, \
                                                                  d_v, d_part)
    const bool narrow = s->model.nbits <= 32;
    if (s->gc) {
      if (narrow) HPHI_GREEN_LAUNCH(true, uint32_t);
      else HPHI_GREEN_LAUNCH(true, uint64_t);
    } else {
      if (narrow) HPHI_GREEN_LAUNCH(false, uint32_t);
      else HPHI_GREEN_LAUNCH(false, uint64_t);
    }
#undef HPHI_GREEN_LAUNCH
    finalize_partials_kernel<kGreenAcc><<<1, 256, 0, s->stream>>>(d_part, grid, d_terms_out + (size_t)b * kGreenAcc);
    if (cudaGetLastError() != cudaSuccess) rc = -1;
  }
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) rc = -1;
  cudaFree(d_part);
  if (rc != 0) set_error("Green's function kernels failed");
  return rc;
}

__global__ void imag_check_kernel(int64_t n, const cplx *__restrict__ v, double *__restrict__ re,
                                  int *__restrict__ complex_flag) {
  bool nz = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const cplx z = v[i];
    re[i] = z.x;
    nz = nz || z.y != 0.0;
  }
  if (__any_sync(0xffffffffu, nz) && (threadIdx.x & 31) == 0) *complex_flag = 1;
}

}  // namespace

int green_stage_host_vector(Sector *s, const double *h_v_1based, void **d_vec, VecType *vt) {
  const int64_t n = s->dim;
  cplx *dc = nullptr;
  double *dr = nullptr;
  int *flag = nullptr;
  if (cudaMalloc(&dc, sizeof(cplx) * (size_t)n) != cudaSuccess || cudaMalloc(&dr, sizeof(double) * (size_t)n) != cudaSuccess ||
      cudaMalloc(&flag, sizeof(int)) != cudaSuccess) {
    cudaFree(dc);
    cudaFree(dr);
    set_error("Green's functions: device allocation failed");
    return -1;
  }
  int h_flag = 0;
  bool ok = cudaMemsetAsync(flag, 0, sizeof(int), s->stream) == cudaSuccess &&
            cudaMemcpyAsync(dc, h_v_1based + 2, sizeof(cplx) * (size_t)n, cudaMemcpyHostToDevice, s->stream) == cudaSuccess;
  if (ok) {
    imag_check_kernel<<<s->red_blocks, 256, 0, s->stream>>>(n, dc, dr, flag);
    ok = cudaGetLastError() == cudaSuccess &&
         cudaMemcpyAsync(&h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream) == cudaSuccess &&
         cudaStreamSynchronize(s->stream) == cudaSuccess;
  }
  cudaFree(flag);
  if (!ok) {
    cudaFree(dc);
    cudaFree(dr);
    set_error("Green's functions: staging the vector failed");
    return -1;
  }
  if (h_flag) {  // complex: keep the complex copy
    cudaFree(dr);
    *d_vec = dc;
    *vt = kComplex128;
  } else {       // real: the real parts, gathered by the same pass
    cudaFree(dc);
    *d_vec = dr;
    *vt = kReal64;
  }
  return 0;
}

int green_expect(Sector *s, VecType vt, const void *d_v, const std::vector<GreenTerm> &terms,
                 std::vector<double> *out) {
  out->assign(2 * terms.size(), 0.0);
  std::vector<GreenTerm> nz;
  std::vector<int> where;
  for (size_t e = 0; e < terms.size(); e++)
    if (terms[e].coef != 0.0) {
      nz.push_back(terms[e]);
      where.push_back((int)e);
    }
  if (nz.empty()) return 0;
  if (cudaSetDevice(s->device) != cudaSuccess) {
    set_error("cudaSetDevice failed");
    return -1;
  }
  const int w = vt == kReal64 ? 1 : 2;
  const int NB = kGreenAcc / w;
  const size_t nbatch = (nz.size() + NB - 1) / NB;
  double *d_out = nullptr;
  if (cudaMalloc(&d_out, sizeof(double) * nbatch * kGreenAcc) != cudaSuccess) {
    set_error("Green's functions: device allocation failed");
    return -1;
  }
  const int rc = vt == kReal64 ? green_batches<double>(s, (const double *)d_v, nz, d_out)
                               : green_batches<cplx>(s, (const cplx *)d_v, nz, d_out);
  std::vector<double> h(nbatch * kGreenAcc);
  const bool ok = rc == 0 && cudaMemcpy(h.data(), d_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost) == cudaSuccess;
  cudaFree(d_out);
  if (!ok) {
    if (rc == 0) set_error("Green's functions: copy failed");
    return -1;
  }
  for (size_t q = 0; q < nz.size(); q++) {
    const size_t b = q / NB, k = q % NB;
    const double *rec = h.data() + b * kGreenAcc;
    (*out)[2 * where[q]] = rec[w * k];
    (*out)[2 * where[q] + 1] = w == 2 ? rec[w * k + 1] : 0.0;
  }
  return 0;
}

}  // namespace hphi
