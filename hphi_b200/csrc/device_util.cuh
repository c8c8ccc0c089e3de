// Small device helpers shared by the kernels: real/complex arithmetic on double and
// a deterministic block reduction.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

#include "engine.hpp"

namespace hphi {

// Raises the dynamic shared-memory limit of kernel fn on the current device to at least bytes
// (never lowers it: plans of several open sectors share one kernel, and a later sector with
// smaller blocks must not invalidate an earlier one's launches).  Returns the CUDA status.
inline cudaError_t raise_smem_limit(const void *fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, size_t> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  size_t &cur = done[{dev, fn}];
  if (bytes <= cur) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

__host__ __device__ __forceinline__ cplx cmk(double x, double y) { return cplx{x, y}; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return cplx{a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return cplx{a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ cplx operator*(double a, cplx b) { return cplx{a * b.x, a * b.y}; }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return cplx{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}

// Scalar traits: T is double (real vectors) or cplx (complex128 vectors).
template <typename T> struct VT;
template <> struct VT<double> {
  static constexpr bool kComplex = false;
  static __device__ __forceinline__ double zero() { return 0.0; }
  // coefficient (re, im) times x; real vectors carry real coefficients only
  static __device__ __forceinline__ double cmul_re_im(double re, double, double x) { return re * x; }
  static __device__ __forceinline__ double conj_mul_re(double a, double b) { return a * b; }
  static __device__ __forceinline__ double conj_mul_im(double, double) { return 0.0; }
  static __device__ __forceinline__ double abs2(double a) { return a * a; }
  static __device__ __forceinline__ double scale(double a, double x) { return a * x; }
  static __device__ __forceinline__ double add(double a, double b) { return a + b; }
  static __device__ __forceinline__ double sub(double a, double b) { return a - b; }
  static __device__ __forceinline__ double add_re(double x, double a) { return x + a; }
};
template <> struct VT<cplx> {
  static constexpr bool kComplex = true;
  static __device__ __forceinline__ cplx zero() { return cplx{0.0, 0.0}; }
  static __device__ __forceinline__ cplx cmul_re_im(double re, double im, cplx x) {
    return cplx{re * x.x - im * x.y, re * x.y + im * x.x};
  }
  // conj(a) * b
  static __device__ __forceinline__ double conj_mul_re(cplx a, cplx b) { return a.x * b.x + a.y * b.y; }
  static __device__ __forceinline__ double conj_mul_im(cplx a, cplx b) { return a.x * b.y - a.y * b.x; }
  static __device__ __forceinline__ double abs2(cplx a) { return a.x * a.x + a.y * a.y; }
  static __device__ __forceinline__ cplx scale(double a, cplx x) { return cplx{a * x.x, a * x.y}; }
  static __device__ __forceinline__ cplx add(cplx a, cplx b) { return a + b; }
  static __device__ __forceinline__ cplx sub(cplx a, cplx b) { return a - b; }
  static __device__ __forceinline__ cplx add_re(cplx x, double a) { return cplx{x.x + a, x.y}; }
};

// Sum of NV doubles over the block; thread 0 gets the result.  Fixed order, so
// results are reproducible for a fixed launch shape.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double red_smem[32][NV];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) red_smem[wid][k] = v[k];
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      v[k] = (lane < nw) ? red_smem[lane][k] : 0.0;
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
  }
  __syncthreads();
}

// Sums `n` partial records of NV doubles (stride NV) into out[0..NV).  One block.
template <int NV>
__global__ void finalize_partials_kernel(const double *__restrict__ part, int n, double *__restrict__ out) {
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] += part[i * NV + k];
  block_sum<NV>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) out[k] = v[k];
}

}  // namespace hphi
