// extern "C" entry points (include/hphi_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cerrno>
#include <cstring>
#include <sys/stat.h>
#include <string>
#include <vector>

#include "../../include/hphi_b200.h"
#include "driver.hpp"
#include "engine.hpp"
#include "hv_product.hpp"
#include "refrand.hpp"
#include "model.hpp"
#include "stdface.hpp"

namespace hphi {
namespace {
thread_local std::string g_err;
}
void set_error(const std::string &msg) { g_err = msg; }
const char *get_error() { return g_err.c_str(); }
}  // namespace hphi

struct hphi_handle {
  hphi::Sector *sector = nullptr;
  hphi::LanczosResult last_lanczos;
  double *d_scal = nullptr;  // coefficient / result slots for hphi_mltply*
  void *d_stage0 = nullptr;  // device staging vectors of hphi_mltply (allocated on first use)
  void *d_stage1 = nullptr;
  void *d_perm0 = nullptr;   // native-order scratch of the HPhi-order device entry points
  void *d_perm1 = nullptr;
  cudaStream_t copy_up = nullptr;    // hphi_mltply: v0 upload, overlapping the H v1 compute
  cudaStream_t copy_back = nullptr;  // hphi_mltply: v0 download
  std::vector<cudaEvent_t> ev;       // hphi_mltply: per chunk uploaded / updated, plus v1 consumed
};

namespace hphi {
// The sector behind a handle (nullptr for an invalid handle); for entry points in other files.
Sector *handle_sector(hphi_handle *h) { return (h && h->sector) ? h->sector : nullptr; }
}  // namespace hphi

using namespace hphi;

namespace {
#define CHECK_HANDLE(h)                     \
  do {                                         \
    if (!(h) || !(h)->sector) {                \
      set_error("invalid handle");             \
      return -1;                               \
    }                                          \
    cudaGetLastError();                        \
  } while (0)

int cuda_fail(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return 0;
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return -1;
}
}  // namespace

extern "C" {

const char *hphi_version(void) { return "hphi_b200 0.1 (sm_100a)"; }

const char *hphi_last_error(void) { return get_error(); }

int hphi_open_expert(const char *namelist_def, int device, hphi_handle **out) {
  if (!namelist_def || !out) { set_error("null argument"); return -1; }
  *out = nullptr;
  Model m;
  std::string err;
  if (read_expert(namelist_def, &m, &err) != 0) { set_error(err); return -1; }
  int ndev = 0;
  cudaGetLastError();
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device available");
    return -1;
  }
  if (device < 0 || device >= ndev) { set_error("device index out of range"); return -1; }
  Sector *s = nullptr;
  if (sector_build(m, device, &s, &err) != 0) {
    set_error(err);
    sector_free(s);
    return -1;
  }
  hphi_handle *h = new hphi_handle();
  h->sector = s;
  if (cuda_fail(cudaMalloc(&h->d_scal, sizeof(double) * 8), "alloc")) { hphi_close(h); return -1; }
  *out = h;
  return 0;
}

int hphi_stdface(const char *stan_in, const char *out_dir) {
  if (!stan_in || !out_dir) { set_error("null argument"); return -1; }
  std::string err;
  if (stdface::generate(stan_in, out_dir, &err) != 0) { set_error(err); return -1; }
  return 0;
}

int hphi_inspect_terms(const char *namelist_def, uint64_t *masks, double *coefs, int cap_off, uint64_t *dmasks,
                       double *dcoefs, int cap_diag, int64_t *counts) {
  if (!namelist_def || !counts) { set_error("null argument"); return -1; }
  Model m;
  std::string err;
  if (read_expert(namelist_def, &m, &err) != 0) { set_error(err); return -1; }
  counts[0] = (int64_t)m.offdiag.size();
  counts[1] = (int64_t)m.diag.size();
  for (int k = 0; k < (int)m.offdiag.size() && k < cap_off; k++) {
    const BitTerm &t = m.offdiag[k];
    if (masks) { masks[4 * k] = t.cm; masks[4 * k + 1] = t.cv; masks[4 * k + 2] = t.flip; masks[4 * k + 3] = t.sm; }
    if (coefs) { coefs[2 * k] = t.re; coefs[2 * k + 1] = t.im; }
  }
  for (int k = 0; k < (int)m.diag.size() && k < cap_diag; k++) {
    if (dmasks) { dmasks[2 * k] = m.diag[k].cm; dmasks[2 * k + 1] = m.diag[k].cv; }
    if (dcoefs) dcoefs[k] = m.diag[k].v;
  }
  return 0;
}

int hphi_inspect_green(const char *namelist_def, int body, int *rows, int cap) {
  if (!namelist_def || (body != 1 && body != 2 && body != 3 && body != 4 && body != 6)) {
    set_error("bad argument");
    return -1;
  }
  Model m;
  std::string err;
  if (read_expert(namelist_def, &m, &err) != 0) { set_error(err); return -1; }
  const std::vector<std::vector<int>> &multi = body == 3 ? m.green_three : body == 4 ? m.green_four : m.green_six;
  const int n = body == 1 ? (int)m.green_one.size() : body == 2 ? (int)m.green_two.size() : (int)multi.size();
  const int w = 4 * (body == 1 ? 1 : body == 2 ? 2 : body);
  for (int e = 0; rows && e < n && e < cap; e++)
    for (int q = 0; q < w; q++)
      rows[w * e + q] = body == 1 ? m.green_one[e][q] : body == 2 ? m.green_two[e][q] : multi[e][q];
  return n;
}

void hphi_close(hphi_handle *h) {
  if (!h) return;
  if (h->sector) {
    cudaSetDevice(h->sector->device);
    cudaFree(h->d_scal);
    cudaFree(h->d_stage0);
    cudaFree(h->d_stage1);
    cudaFree(h->d_perm0);
    cudaFree(h->d_perm1);
    if (h->copy_up) cudaStreamDestroy(h->copy_up);
    if (h->copy_back) cudaStreamDestroy(h->copy_back);
    for (cudaEvent_t e : h->ev)
      if (e) cudaEventDestroy(e);
    sector_free(h->sector);
  }
  delete h;
}

int hphi_info(const hphi_handle *h, int64_t *info, int n) {
  CHECK_HANDLE(h);
  const Sector &s = *h->sector;
  int64_t v[HPHI_INFO_COUNT];
  v[HPHI_INFO_DIM] = s.dim;
  v[HPHI_INFO_NSITE] = s.model.nsite;
  v[HPHI_INFO_CALC_MODEL] = s.model.calc_model;
  v[HPHI_INFO_CALC_TYPE] = s.model.calc_type;
  v[HPHI_INFO_SIZE_LIST_2_1] = s.size_list_2_1;
  v[HPHI_INFO_SIZE_LIST_2_2] = s.size_list_2_2;
  v[HPHI_INFO_IS_GC] = s.model.is_gc() ? 1 : 0;
  v[HPHI_INFO_VEC_TYPE] = default_vec_type(s);
  v[HPHI_INFO_N_OFFDIAG] = s.nterms;
  v[HPHI_INFO_N_DIAG] = s.ndterms;
  v[HPHI_INFO_LANCZOS_MAX] = s.model.lanczos_max;
  v[HPHI_INFO_NUM_AVE] = s.model.num_ave;
  v[HPHI_INFO_NATIVE_ORDER] = has_native_order(&s) ? 1 : 0;
  v[HPHI_INFO_EXCT] = s.model.k_exct;
  v[HPHI_INFO_KERNEL] = s.prod ? (prod_two_pass(&s) ? 3 : 2) : (s.hub ? 1 : (s.rb ? 4 : 0));
  v[HPHI_INFO_N_GREEN_ONE] = (int64_t)s.model.green_one.size();
  v[HPHI_INFO_N_GREEN_TWO] = (int64_t)s.model.green_two.size();
  for (int i = 0; i < n && i < HPHI_INFO_COUNT; i++) info[i] = v[i];
  return 0;
}

int hphi_sz(const hphi_handle *h, uint64_t *list_1, uint64_t *list_2_1, uint64_t *list_2_2) {
  CHECK_HANDLE(h);
  const Sector &s = *h->sector;
  // HubbardGC and SpinGC (any spin) have no lists: the row is the configuration index
  if (s.model.calc_model == kHubbardGC || s.model.calc_model == kSpinGC) {
    set_error("grand-canonical models have no sector lists");
    return -1;
  }
  if (s.model.general_spin) {  // HPhi's mixed-radix lists, kept on the host
    if (list_1) {
      list_1[0] = 0;
      std::memcpy(list_1 + 1, s.gs_list_1.data() + 1, sizeof(uint64_t) * s.dim);
    }
    if (list_2_1) std::memcpy(list_2_1, s.gs_list_2_1.data(), sizeof(uint64_t) * s.size_list_2_1);
    if (list_2_2) std::memcpy(list_2_2, s.gs_list_2_2.data(), sizeof(uint64_t) * s.size_list_2_2);
    return 0;
  }
  cudaSetDevice(s.device);
  if (list_1) {
    list_1[0] = 0;
    if (cuda_fail(cudaMemcpy(list_1 + 1, s.d_list_1, sizeof(uint64_t) * s.dim, cudaMemcpyDeviceToHost), "copy list_1"))
      return -1;
  }
  if (list_2_1 || list_2_2) {
    std::vector<uint32_t> tmp(std::max<uint64_t>(s.ihfbit, s.sdim));
    if (list_2_1) {
      if (cuda_fail(cudaMemcpy(tmp.data(), s.d_list_2_1, sizeof(uint32_t) * s.ihfbit, cudaMemcpyDeviceToHost), "copy"))
        return -1;
      for (int64_t i = 0; i < s.size_list_2_1; i++) list_2_1[i] = (uint64_t)i < s.ihfbit ? tmp[i] : 0;
    }
    if (list_2_2) {
      if (cuda_fail(cudaMemcpy(tmp.data(), s.d_list_2_2, sizeof(uint32_t) * s.sdim, cudaMemcpyDeviceToHost), "copy"))
        return -1;
      for (int64_t i = 0; i < s.size_list_2_2; i++) list_2_2[i] = (uint64_t)i < s.sdim ? tmp[i] : 0;
    }
  }
  return 0;
}

int hphi_diagonalcalc(const hphi_handle *h, double *list_diagonal) {
  CHECK_HANDLE(h);
  const Sector &s = *h->sector;
  cudaSetDevice(s.device);
  list_diagonal[0] = 0.0;
  return cuda_fail(cudaMemcpy(list_diagonal + 1, s.d_diag, sizeof(double) * s.dim, cudaMemcpyDeviceToHost),
                   "copy list_Diagonal");
}

int hphi_mltply_device(hphi_handle *h, int vec_type, void *d_v0, const void *d_v1, double acc, double scale,
                       double *prdct) {
  CHECK_HANDLE(h);
  Sector *s = h->sector;
  if (vec_type != HPHI_REAL64 && vec_type != HPHI_COMPLEX128) { set_error("bad vec_type"); return -1; }
  const VecType vt = (VecType)vec_type;
  cudaSetDevice(s->device);
  const double coef[2] = {acc, scale};
  if (cuda_fail(cudaMemcpyAsync(h->d_scal, coef, sizeof(coef), cudaMemcpyHostToDevice, s->stream), "coef")) return -1;
  if (!has_native_order(s)) {
    if (hv_launch(s, vt, d_v1, d_v0, h->d_scal, h->d_scal + 2) != 0) return -1;
  } else {
    // HPhi order in and out: permute to the native order around the native kernel
    const size_t bytes = sizeof(cplx) * (size_t)s->dim;
    if (!h->d_perm0) {
      if (cuda_fail(cudaMalloc(&h->d_perm0, bytes), "alloc scratch")) return -1;
      if (cuda_fail(cudaMalloc(&h->d_perm1, bytes), "alloc scratch")) {
        cudaFree(h->d_perm0);
        h->d_perm0 = nullptr;
        return -1;
      }
    }
    if (to_native(s, vt, d_v1, h->d_perm1) != 0) return -1;
    if (acc != 0.0 && to_native(s, vt, d_v0, h->d_perm0) != 0) return -1;
    if (hv_native(s, vt, h->d_perm1, h->d_perm0, h->d_scal, h->d_scal + 2) != 0) return -1;
    if (from_native(s, vt, h->d_perm0, d_v0) != 0) return -1;
  }
  double out[2];
  if (cuda_fail(cudaMemcpyAsync(out, h->d_scal + 2, sizeof(out), cudaMemcpyDeviceToHost, s->stream), "prdct")) return -1;
  if (cuda_fail(cudaStreamSynchronize(s->stream), "sync")) return -1;
  if (prdct) { prdct[0] = out[0]; prdct[1] = out[1]; }
  return 0;
}

int hphi_to_native(hphi_handle *h, int vec_type, const void *d_hphi, void *d_native) {
  CHECK_HANDLE(h);
  if (vec_type != HPHI_REAL64 && vec_type != HPHI_COMPLEX128) { set_error("bad vec_type"); return -1; }
  if (d_hphi == d_native && has_native_order(h->sector)) { set_error("in-place permutation is not supported"); return -1; }
  cudaSetDevice(h->sector->device);
  if (to_native(h->sector, (VecType)vec_type, d_hphi, d_native) != 0) return -1;
  return cuda_fail(cudaStreamSynchronize(h->sector->stream), "sync");
}

int hphi_from_native(hphi_handle *h, int vec_type, const void *d_native, void *d_hphi) {
  CHECK_HANDLE(h);
  if (vec_type != HPHI_REAL64 && vec_type != HPHI_COMPLEX128) { set_error("bad vec_type"); return -1; }
  if (d_hphi == d_native && has_native_order(h->sector)) { set_error("in-place permutation is not supported"); return -1; }
  cudaSetDevice(h->sector->device);
  if (from_native(h->sector, (VecType)vec_type, d_native, d_hphi) != 0) return -1;
  return cuda_fail(cudaStreamSynchronize(h->sector->stream), "sync");
}

int hphi_mltply(hphi_handle *h, double *v0, const double *v1, double *prdct) {
  // HPhi's mltply on host vectors.  Stream st: upload v1, H v1 on the device (a real H takes
  // the real kernels on the real and imaginary parts), then chunk by chunk v0 += H v1.  Once
  // v1 has been read, v0 uploads chunk by chunk into v1's buffer on copy_up (overlapping the
  // H v1 compute), and each updated chunk downloads on copy_back while the next one uploads.
  CHECK_HANDLE(h);
  Sector *s = h->sector;
  cudaSetDevice(s->device);
  const int64_t dim = s->dim;
  const size_t bytes = sizeof(cplx) * (size_t)dim;
  constexpr int64_t kChunk = 4 << 20;  // complex elements per chunk (64 MB)
  const int nchunk = (int)((dim + kChunk - 1) / kChunk);
  if (!h->d_stage0) {
    void *a = nullptr, *b = nullptr;
    if (cuda_fail(cudaMalloc(&a, bytes), "alloc") || cuda_fail(cudaMalloc(&b, bytes), "alloc") ||
        cuda_fail(cudaStreamCreateWithFlags(&h->copy_up, cudaStreamNonBlocking), "stream") ||
        cuda_fail(cudaStreamCreateWithFlags(&h->copy_back, cudaStreamNonBlocking), "stream")) {
      cudaFree(a); cudaFree(b);
      return -1;
    }
    h->d_stage0 = a; h->d_stage1 = b;
  }
  if (!h->d_perm0) {
    if (cuda_fail(cudaMalloc(&h->d_perm0, bytes), "alloc scratch")) return -1;
    if (cuda_fail(cudaMalloc(&h->d_perm1, bytes), "alloc scratch")) {
      cudaFree(h->d_perm0);
      h->d_perm0 = nullptr;
      return -1;
    }
  }
  while ((int)h->ev.size() < 2 * nchunk + 1) {
    cudaEvent_t e;
    if (cuda_fail(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event")) return -1;
    h->ev.push_back(e);
  }
  cudaEvent_t v1_done = h->ev[2 * nchunk];
  cudaStream_t st = s->stream;
  // v1 (elements 1 .. dim of the 1-based array)
  if (cuda_fail(cudaMemcpyAsync(h->d_stage1, v1 + 2, bytes, cudaMemcpyHostToDevice, st), "copy v1")) return -1;
  double out[4] = {0, 0, 0, 0};
  const double c01[2] = {0.0, 1.0};
  if (cuda_fail(cudaMemcpyAsync(h->d_scal, c01, sizeof(c01), cudaMemcpyHostToDevice, st), "coef")) return -1;
  const bool nat = has_native_order(s);
  const bool real_h = !s->model.complex_terms;
  double *re = (double *)h->d_perm0, *im = re + dim, *hre = (double *)h->d_perm1, *him = hre + dim;
  // read v1 into the compute buffers, then free its buffer for v0
  if (real_h) {
    const void *src = h->d_stage1;
    if (nat) {
      if (to_native(s, kComplex128, h->d_stage1, h->d_stage0) != 0) return -1;
      src = h->d_stage0;
    }
    if (vec_split_c128(s, src, re, im) != 0) return -1;
  } else if (nat) {
    if (to_native(s, kComplex128, h->d_stage1, h->d_perm1) != 0) return -1;
  } else if (cuda_fail(cudaMemcpyAsync(h->d_perm1, h->d_stage1, bytes, cudaMemcpyDeviceToDevice, st), "copy")) {
    return -1;
  }
  if (cuda_fail(cudaEventRecord(v1_done, st), "event") || cuda_fail(cudaStreamWaitEvent(h->copy_up, v1_done, 0), "wait"))
    return -1;
  cplx *v0d = (cplx *)h->d_stage1;
  for (int k = 0; k < nchunk; k++) {
    const int64_t c0 = (int64_t)k * kChunk, n = std::min<int64_t>(kChunk, dim - c0);
    if (cuda_fail(cudaMemcpyAsync(v0d + c0, v0 + 2 * (1 + c0), sizeof(cplx) * n, cudaMemcpyHostToDevice, h->copy_up),
                  "copy v0") ||
        cuda_fail(cudaEventRecord(h->ev[k], h->copy_up), "event"))
      return -1;
  }
  // H v1 into d_stage0 (HPhi order)
  if (real_h) {
    if ((nat ? hv_native(s, kReal64, re, hre, h->d_scal, h->d_scal + 2)
             : hv_launch(s, kReal64, re, hre, h->d_scal, h->d_scal + 2)) != 0)
      return -1;
    if ((nat ? hv_native(s, kReal64, im, him, h->d_scal, h->d_scal + 4)
             : hv_launch(s, kReal64, im, him, h->d_scal, h->d_scal + 4)) != 0)
      return -1;
    if (nat) {
      if (vec_join_c128(s, hre, him, h->d_perm0) != 0 || from_native(s, kComplex128, h->d_perm0, h->d_stage0) != 0)
        return -1;
    } else if (vec_join_c128(s, hre, him, h->d_stage0) != 0) {
      return -1;
    }
  } else {
    if ((nat ? hv_native(s, kComplex128, h->d_perm1, h->d_perm0, h->d_scal, h->d_scal + 2)
             : hv_launch(s, kComplex128, h->d_perm1, h->d_perm0, h->d_scal, h->d_scal + 2)) != 0)
      return -1;
    if (nat ? from_native(s, kComplex128, h->d_perm0, h->d_stage0) != 0
            : cuda_fail(cudaMemcpyAsync(h->d_stage0, h->d_perm0, bytes, cudaMemcpyDeviceToDevice, st), "copy"))
      return -1;
  }
  if (cuda_fail(cudaMemcpyAsync(out, h->d_scal + 2, sizeof(out), cudaMemcpyDeviceToHost, st), "prdct")) return -1;
  // v0 += H v1 per chunk, downloaded as it is done
  const cplx *hv = (const cplx *)h->d_stage0;
  for (int k = 0; k < nchunk; k++) {
    const int64_t c0 = (int64_t)k * kChunk, n = std::min<int64_t>(kChunk, dim - c0);
    if (cuda_fail(cudaStreamWaitEvent(st, h->ev[k], 0), "wait") || vec_add_c128(s, st, n, v0d + c0, hv + c0) != 0 ||
        cuda_fail(cudaEventRecord(h->ev[nchunk + k], st), "event") ||
        cuda_fail(cudaStreamWaitEvent(h->copy_back, h->ev[nchunk + k], 0), "wait") ||
        cuda_fail(cudaMemcpyAsync(v0 + 2 * (1 + c0), v0d + c0, sizeof(cplx) * n, cudaMemcpyDeviceToHost, h->copy_back),
                  "copy back"))
      return -1;
  }
  if (cuda_fail(cudaStreamSynchronize(h->copy_back), "sync") || cuda_fail(cudaStreamSynchronize(st), "sync") ||
      cuda_fail(cudaStreamSynchronize(h->copy_up), "sync"))
    return -1;
  if (prdct) {
    if (real_h) {
      prdct[0] = out[0] + out[2];  // <a|Ha> + <b|Hb>; a real symmetric H has no imaginary part
      prdct[1] = 0.0;
    } else {
      prdct[0] = out[0];
      prdct[1] = out[1];
    }
  }
  return 0;
}

int hphi_mltply_device_async(hphi_handle *h, int vec_type, void *d_v0, const void *d_v1, const double *d_coef,
                             double *d_prdct) {
  CHECK_HANDLE(h);
  Sector *s = h->sector;
  if (vec_type != HPHI_REAL64 && vec_type != HPHI_COMPLEX128) { set_error("bad vec_type"); return -1; }
  cudaSetDevice(s->device);
  return hv_native(s, (VecType)vec_type, d_v1, d_v0, d_coef, d_prdct);
}

void *hphi_stream(hphi_handle *h) { return (h && h->sector) ? (void *)h->sector->stream : nullptr; }

int hphi_synchronize(hphi_handle *h) {
  CHECK_HANDLE(h);
  cudaSetDevice(h->sector->device);
  return cuda_fail(cudaStreamSynchronize(h->sector->stream), "synchronize");
}

int hphi_lanczos_steps(hphi_handle *h, int steps, uint64_t seed, double *energies, int nev) {
  CHECK_HANDLE(h);
  if (steps < 2) { set_error("hphi_lanczos_steps: steps must be >= 2"); return -1; }
  Sector *s = h->sector;
  const VecType vt = default_vec_type(*s);
  LanczosOptions opt;
  opt.fixed_steps = steps;
  opt.hashed_start = true;
  opt.hashed_seed = seed;
  LanczosResult &r = h->last_lanczos;
  r = LanczosResult();
  if (lanczos_run(s, vt, nullptr, opt, &r) != 0) return -1;
  for (int q = 0; energies && q < nev; q++)
    energies[q] = (q < r.steps) ? tridiag_eigenvalue(r.alpha.data(), r.beta.data(), r.steps, q) : 0.0;
  return 0;
}

namespace {
// OpenMP thread count whose random start vectors HPhi would draw: HPHI_B200_REF_THREADS,
// else OMP_NUM_THREADS, else 1.
int reference_threads() {
  for (const char *k : {"HPHI_B200_REF_THREADS", "OMP_NUM_THREADS"}) {
    const char *v = getenv(k);
    if (v && atoi(v) > 0) return atoi(v);
  }
  return 1;
}
}  // namespace

int hphi_lanczos(hphi_handle *h, const double *v_init, const char *output_dir, double *result, int nresult) {
  CHECK_HANDLE(h);
  Sector *s = h->sector;
  const VecType vt = default_vec_type(*s);
  const int iev = s->model.input_eigenvec;
  if (iev == 1 || iev == 2) {
    // InputEigenVec: the stored eigenvector (in output_dir) instead of a Lanczos run
    LanczosResult &r = h->last_lanczos;
    r = LanczosResult();
    if (lanczos_input_vector(s, vt, output_dir ? output_dir : "", iev, &r) != 0) return -1;
    if (result && nresult > 0) {
      double v[17] = {1.0, 0, 0, 0, 0, 0, 0, r.energy, r.var, r.doublon, r.sz, 0, 0, 0, 0, 0, 0};
      for (int i = 0; i < nresult && i < 17; i++) result[i] = v[i];
    }
    return output_dir ? write_lanczos_outputs(*s, r, output_dir) : 0;
  }
  std::vector<double> start;
  if (!v_init) {
    if (!single_element_start(*s, &start))
      reference_random_start(s->dim, kRefLanczos, s->model.initial_iv, 0, s->model.initial_vec_type,
                             reference_threads(), 1, &start);
    v_init = start.data();
  }
  LanczosOptions opt;
  opt.eigenvector = (s->model.calc_eigenvec != -1);
  opt.copy_eigenvector = opt.eigenvector;
  // ReStart (src/Lanczos_EigenValue.c:80-101, 287-297): 1 writes the restart files, 3 reads
  // them, 2 does both; they live in output_dir
  LanczosRestart resume;
  const int rmode = s->model.restart;
  if (output_dir && (rmode == 2 || rmode == 3)) {
    if (read_lanczos_restart(*s, output_dir, &resume) != 0) return -1;
    opt.resume = &resume;
  }
  opt.restart_out = output_dir && (rmode == 1 || rmode == 2);
  LanczosResult &r = h->last_lanczos;
  r = LanczosResult();
  const int rc = lanczos_run(s, vt, v_init, opt, &r);
  if (rc == 0 && r.has_restart && write_lanczos_restart(*s, r.restart, output_dir) != 0) return -1;
  if (result && nresult > 0) {
    double v[17] = {r.converged ? 1.0 : 0.0, (double)r.steps, r.e_target, 0, 0, 0, 0, r.energy, r.var, r.doublon, r.sz,
                    r.check_diff, r.check_var, (double)r.cg_rounds, (double)r.cg_iterations, r.cg_diff, r.cg_var};
    for (int q = 0; q < 4 && q < (int)r.energies.size(); q++) v[3 + q] = r.energies[q];
    for (int i = 0; i < nresult && i < 17; i++) result[i] = v[i];
  }
  if (rc != 0) {
    // HPhi writes its step lines while it iterates, so a run that stops unconverged leaves
    // them behind (src/Lanczos_EigenValue.c:200-258, then exitMPI(-3) in src/HPhiMain.c:294-297)
    if (output_dir && !r.converged && !r.lines.empty()) {
      const std::string msg = hphi_last_error();
      write_lanczos_outputs(*s, r, output_dir);
      set_error(msg);
    }
    return -1;
  }
  if (output_dir && write_lanczos_outputs(*s, r, output_dir) != 0) return -1;
  return 0;
}

int hphi_lanczos_tridiagonal(hphi_handle *h, double *alpha, double *beta, int cap, int *steps) {
  CHECK_HANDLE(h);
  const LanczosResult &r = h->last_lanczos;
  if (steps) *steps = r.steps;
  for (int i = 0; i < cap && i < (int)r.alpha.size(); i++) {
    if (alpha) alpha[i] = r.alpha[i];
    if (beta) beta[i] = r.beta[i];
  }
  return 0;
}

int hphi_lanczos_eigenvector(hphi_handle *h, double *v) {
  CHECK_HANDLE(h);
  const auto &e = h->last_lanczos.eigenvector;
  if (e.empty()) { set_error("no eigenvector: run hphi_lanczos with CalcEigenVec != -1 first"); return -1; }
  std::memcpy(v, e.data(), sizeof(double) * e.size());
  return 0;
}

int hphi_tpq(hphi_handle *h, const double *v_init, const char *output_dir, double *result, int nresult) {
  CHECK_HANDLE(h);
  Sector *s = h->sector;
  const VecType vt = default_vec_type(*s);
  const std::string out = output_dir ? output_dir : "output";
  const int64_t stride = 2 * (s->dim + 1);
  TpqResult r;
  const int restart = s->model.restart;  // RESTART_OUT 1, RESTART_INOUT 2, RESTART_IN 3
  TpqOptions opt;
  opt.keep_vector = restart == 1 || restart == 2;
  auto tmpvec = [&](int rand_i) {
    char vname[256];
    snprintf(vname, sizeof(vname), "tmpvec_set%d_rank_%d.dat", rand_i, 0);
    return out + "/" + vname;
  };
  auto save = [&](int rand_i, const TpqResult &rr) -> int {
    // tmpvec_set%d_rank_%d.dat after the loop (src/CalcByTPQ.c:275-290)
    FILE *fo = fopen(tmpvec(rand_i).c_str(), "wb");
    if (!fo) {
      set_error("cannot write " + tmpvec(rand_i));
      return -1;
    }
    const int stp = rr.final_step;
    const long dim = (long)s->dim;
    fwrite(&stp, sizeof(int), 1, fo);
    fwrite(&dim, sizeof(long), 1, fo);
    fwrite(rr.final_vector.data(), sizeof(double), rr.final_vector.size(), fo);
    fclose(fo);
    return 0;
  };
  // The samples of the reference's loop (src/CalcByTPQ.c:76) run in blocks of up to
  // kHvBlockMax in lockstep, sharing each H application (one block H*V), where the sector's
  // H*v is the general kernel; a sample continued from a stored state runs alone.
  // HPHI_B200_TPQ_BLOCK: 0 runs the samples one after another, N in 2..8 caps the block size
  // (default 8).
  const char *blk_env = std::getenv("HPHI_B200_TPQ_BLOCK");
  int block_cap = kHvBlockMax;
  if (blk_env && *blk_env) block_cap = std::max(0, std::min(kHvBlockMax, std::atoi(blk_env)));
  const bool block_ok = hv_block_applies(s, vt) && block_cap > 1;
  const int block_max = block_ok ? block_cap : 1;
  std::vector<std::vector<double>> starts;
  std::vector<int> pending;
  auto run_pending = [&]() -> int {
    if (pending.empty()) return 0;
    std::vector<const double *> hv;
    for (size_t b = 0; b < pending.size(); b++) hv.push_back(starts[b].empty() ? v_init + stride * pending[b] : starts[b].data());
    std::vector<TpqResult> rr;
    if (tpq_run_samples(s, vt, hv, pending, out, &rr, opt, block_ok && pending.size() > 1) != 0) return -1;
    for (size_t b = 0; b < pending.size(); b++)
      if (opt.keep_vector && save(pending[b], rr[b]) != 0) return -1;
    r = std::move(rr.back());
    pending.clear();
    starts.clear();
    return 0;
  };
  for (int rand_i = 0; rand_i < s->model.num_ave; rand_i++) {
    const std::string vpath = tmpvec(rand_i);
    FILE *fin = (restart == 2 || restart == 3) ? fopen(vpath.c_str(), "rb") : nullptr;
    if (fin) {
      // stored state: int step, long dim, complex128[dim+1] (src/CalcByTPQ.c:86-104)
      int stp = 0;
      long dim = 0;
      std::vector<double> start(stride, 0.0);
      const bool ok = fread(&stp, sizeof(int), 1, fin) == 1 && fread(&dim, sizeof(long), 1, fin) == 1 &&
                      dim == (long)s->dim && fread(start.data(), sizeof(double), stride, fin) == (size_t)stride;
      fclose(fin);
      if (!ok) {
        set_error("Error: A file of Inputvector is incorrect.");
        return -1;
      }
      if (run_pending() != 0) return -1;
      TpqOptions o = opt;
      o.resume_step = stp;
      if (tpq_run(s, vt, start.data(), rand_i, out, &r, o) != 0) return -1;
      if (opt.keep_vector && save(rand_i, r) != 0) return -1;
      continue;
    }
    pending.push_back(rand_i);
    starts.emplace_back();
    if (!v_init) {
      // a missing stored state starts the sample normally, as the reference announces
      // (src/CalcByTPQ.c:93-96; it then reads from the missing file, here it does not)
      reference_random_start(s->dim, kRefTPQ, s->model.initial_iv, rand_i, s->model.initial_vec_type,
                             reference_threads(), 1, &starts.back());
    }
    if ((int)pending.size() == block_max && run_pending() != 0) return -1;
  }
  if (run_pending() != 0) return -1;
  if (result)
    for (int i = 0; i < nresult && i < (int)r.energy.size(); i++) result[i] = r.energy[i];
  return 0;
}

int hphi_lobpcg(hphi_handle *h, const double *v_init, const char *output_dir, double *result, int nresult) {
  CHECK_HANDLE(h);
  Sector *s = h->sector;
  VecType vt = default_vec_type(*s);
  const int k = std::max(1, s->model.k_exct);
  std::vector<double> start;
  const int restart = s->model.restart;  // RESTART_OUT 1, RESTART_INOUT 2, RESTART_IN 3
  const std::string out = output_dir ? output_dir : "";
  const int64_t stride = 2 * (s->dim + 1);
  auto tmpvec = [&](int ie) {
    char name[64];
    snprintf(name, sizeof(name), "tmpvec_set%d_rank_%d.dat", ie, 0);
    return out.empty() ? std::string(name) : out + "/" + name;
  };
  if ((restart == 2 || restart == 3) && output_dir) {
    // Initialize_wave (A): the stored vectors of every state, else the usual start
    // (src/CalcByLOBPCG.c:175-212)
    std::vector<double> stored((size_t)stride * k, 0.0);
    bool all = true;
    for (int ie = 0; ie < k && all; ie++) {
      FILE *f = fopen(tmpvec(ie).c_str(), "rb");
      if (!f) { all = false; break; }
      int itr = 0;
      unsigned long dim = 0;
      const bool ok = fread(&itr, sizeof(int), 1, f) == 1 && fread(&dim, sizeof(dim), 1, f) == 1 &&
                      dim == (unsigned long)s->dim &&
                      fread(stored.data() + (size_t)stride * ie, sizeof(double), stride, f) == (size_t)stride;
      fclose(f);
      if (!ok) { set_error("Error: Invalid restart file."); return -1; }
      stored[(size_t)stride * ie] = stored[(size_t)stride * ie + 1] = 0.0;
    }
    if (all && !v_init) {
      start.swap(stored);
      v_init = start.data();
    }
  }
  bool from_input = false;
  if (s->model.input_eigenvec != 0 && !v_init) {
    // InputEigenVec: the states stored in <head>_eigenvec_%d_rank_0.dat (src/CalcByLOBPCG.c:688-716)
    start.assign((size_t)stride * k, 0.0);
    for (int ie = 0; ie < k; ie++) {
      char name[256];
      snprintf(name, sizeof(name), "%s_eigenvec_%d_rank_%d.dat", s->model.data_head.c_str(), ie, 0);
      const std::string path = out.empty() ? std::string(name) : out + "/" + name;
      FILE *f = fopen(path.c_str(), "rb");
      if (!f) { set_error("Error: Inputvector file is not found."); return -1; }
      int itr = 0;
      long dim = 0;
      const bool ok = fread(&itr, sizeof(int), 1, f) == 1 && fread(&dim, sizeof(long), 1, f) == 1 &&
                      dim == (long)s->dim &&
                      fread(start.data() + (size_t)stride * ie, sizeof(double), stride, f) == (size_t)stride;
      fclose(f);
      if (!ok) { set_error("Error: Invalid Inputvector file."); return -1; }
      start[(size_t)stride * ie] = start[(size_t)stride * ie + 1] = 0.0;
    }
    v_init = start.data();
    from_input = true;
    for (size_t q = 1; q < start.size() && vt == kReal64; q += 2)
      if (start[q] != 0.0) vt = kComplex128;  // complex stored states keep their phases
  }
  if (!v_init) {
    if (!lobpcg_single_element_start(*s, &start))
      reference_random_start(s->dim, kRefLOBPCG, s->model.initial_iv, 0, s->model.initial_vec_type,
                             reference_threads(), k, &start);
    v_init = start.data();
  }
  LobpcgResult r;
  r.phys_only = from_input;
  const bool restart_out = (restart == 1 || restart == 2) && output_dir;
  // OutputEigenVec files and the restart vectors need the states on the host
  r.copy_vectors = (s->model.output_eigenvec != 0 && output_dir) || restart_out;
  const int rc = lobpcg_run(s, vt, v_init, &r);
  if (restart_out && !r.eigenvectors.empty()) {
    // Output_restart (src/CalcByLOBPCG.c:295-319, called at :600-606): the current vectors
    if (!out.empty() && mkdir(out.c_str(), 0755) != 0 && errno != EEXIST) {
      set_error("cannot create output directory " + out);
      return -1;
    }
    for (int ie = 0; ie < k; ie++) {
      FILE *f = fopen(tmpvec(ie).c_str(), "wb");
      if (!f) { set_error("cannot write " + tmpvec(ie)); return -1; }
      const int itr = r.itr;
      const long dim = (long)s->dim;
      fwrite(&itr, sizeof(int), 1, f);
      fwrite(&dim, sizeof(long), 1, f);
      fwrite(r.eigenvectors.data() + (size_t)stride * ie, sizeof(double), stride, f);
      fclose(f);
    }
    if (!r.converged) {
      // an unconverged run in restart mode ends here without error (LOBPCG_Main returns 1,
      // CalcByLOBPCG returns TRUE, :650-656): the step file only
      if (write_lobpcg_outputs(*s, r, out) != 0) return -1;
      if (result && nresult > 0) {
        result[0] = 0.0;
        if (nresult > 1) result[1] = (double)r.steps;
        if (nresult > 2) result[2] = r.residual;
      }
      return 0;
    }
  }
  if (result && nresult > 0) {
    std::vector<double> v = {r.converged ? 1.0 : 0.0, (double)r.steps, r.residual};
    for (int i = 0; i < k; i++) {
      v.push_back(r.energy.size() > (size_t)i ? r.energy[i] : 0.0);
      v.push_back(r.var.size() > (size_t)i ? r.var[i] : 0.0);
      v.push_back(r.doublon.size() > (size_t)i ? r.doublon[i] : 0.0);
      v.push_back(r.sz.size() > (size_t)i ? r.sz[i] : 0.0);
    }
    for (int i = 0; i < nresult && i < (int)v.size(); i++) result[i] = v[i];
  }
  if (output_dir) {
    const std::string err = get_error();
    if (write_lobpcg_outputs(*s, r, output_dir) != 0) return -1;
    if (rc != 0) set_error(err);
  }
  return rc;
}

int hphi_tem(hphi_handle *h, const double *v_init, const char *output_dir, double *result, int nresult) {
  CHECK_HANDLE(h);
  Sector *s = h->sector;
  const Model &m = s->model;
  const std::string out = output_dir ? output_dir : "output";
  const int64_t stride = 2 * (s->dim + 1);
  std::vector<double> start;
  int step_initial = 0;
  if (!v_init) {
    // the input state <SpectrumVec>_rank_0.dat in the output folder (src/CalcByTEM.c:74-103)
    if (!m.input_eigenvec) {
      set_error("Error: A file of Inputvector is not inputted.");
      return -1;
    }
    const std::string path = out + "/" + m.spectrum_vec + "_rank_0.dat";
    FILE *fin = m.spectrum_vec.empty() ? nullptr : fopen(path.c_str(), "rb");
    if (!fin) {
      set_error("Error: A file of Inputvector does not exist.");
      return -1;
    }
    int stp = 0;
    long dim = 0;
    start.assign(stride, 0.0);
    const bool ok = fread(&stp, sizeof(int), 1, fin) == 1 && fread(&dim, sizeof(long), 1, fin) == 1 &&
                    dim == (long)s->dim && fread(start.data(), sizeof(double), stride, fin) == (size_t)stride;
    fclose(fin);
    if (!ok) {
      set_error("Error: A file of Inputvector is incorrect.");
      return -1;
    }
    // ReStart 2 / 3 continues from the file's step (RESTART_NOT / RESTART_OUT start at 0)
    if (m.restart == 2 || m.restart == 3) step_initial = stp;
    if (step_initial < 0) {
      set_error("Error: A file of Inputvector is incorrect.");
      return -1;
    }
    v_init = start.data();
  }
  TeResult r;
  if (te_run(s, v_init, step_initial, out, &r) != 0) return -1;
  if (result)
    for (int i = 0; i < nresult && i < (int)r.energy.size(); i++) result[i] = r.energy[i];
  return 0;
}

int hphi_spectrum(hphi_handle *h, const double *h_vec, const char *output_dir, double *result, int nresult) {
  CHECK_HANDLE(h);
  Sector *s = h->sector;
  const Model &m = s->model;
  const std::string out = output_dir ? output_dir : "output";
  // CalcType 0 is the reference's Lanczos spectrum; for CalcType 3 it solves the same
  // Green's function by shifted BiCG (src/CalcSpectrum.c, CalcSpectrumByBiCG), which the
  // Lanczos continued fraction here reproduces to the printed digits.  TPQ and full
  // diagonalisation spectra are other quantities.
  if (m.calc_type != kLanczos && m.calc_type != kCG) {
    set_error("spectrum: CalcType 0 (Lanczos) or 3 (CG) only");
    return -1;
  }
  std::vector<double> vec;
  if (!h_vec) {
    // the input vector <SpectrumVec>_rank_0.dat in the output folder (src/CalcSpectrum.c:153-182)
    const std::string path = out + "/" + m.spectrum_vec + "_rank_0.dat";
    FILE *fin = m.spectrum_vec.empty() ? nullptr : fopen(path.c_str(), "rb");
    if (!fin) {
      set_error("Error: A file of Input vector does not exist.");
      return -1;
    }
    const int64_t stride = 2 * (s->dim + 1);
    int stp = 0;
    long dim = 0;
    vec.assign(stride, 0.0);
    const bool ok = fread(&stp, sizeof(int), 1, fin) == 1 && fread(&dim, sizeof(long), 1, fin) == 1 &&
                    dim == (long)s->dim && fread(vec.data(), sizeof(double), stride, fin) == (size_t)stride;
    fclose(fin);
    if (!ok) {
      set_error("Error: A file of Input vector is incorrect.");
      return -1;
    }
    h_vec = vec.data();
  }
  SpectrumResult r;
  if (spectrum_run(s, h_vec, out, &r) != 0) return -1;
  for (int i = 0; result && i < nresult && i < (int)r.omega.size(); i++) {
    result[4 * i] = r.omega[i].real();
    result[4 * i + 1] = r.omega[i].imag();
    result[4 * i + 2] = r.green[i].real();
    result[4 * i + 3] = r.green[i].imag();
  }
  return 0;
}

int hphi_run(hphi_handle *h, const char *output_dir) {
  CHECK_HANDLE(h);
  const std::string out = output_dir ? output_dir : "output";
  if (h->sector->model.calc_spec == 1) return hphi_spectrum(h, nullptr, out.c_str(), nullptr, 0);
  switch (h->sector->model.calc_type) {
    case kLanczos: return hphi_lanczos(h, nullptr, out.c_str(), nullptr, 0);
    case kTPQ:
    case kcTPQ: return hphi_tpq(h, nullptr, out.c_str(), nullptr, 0);
    case kCG: return hphi_lobpcg(h, nullptr, out.c_str(), nullptr, 0);
    case kTimeEvolution: return hphi_tem(h, nullptr, out.c_str(), nullptr, 0);
    default:
      set_error("CalcType not supported by this engine (Lanczos = 0, TPQ = 1, LOBPCG = 3, time evolution = 4 "
                "and cTPQ = 5 are)");
      return -1;
  }
}

int hphi_reference_start(int64_t dim, int kind, int initial_iv, int sample, int vec_type, int threads, int count,
                         double *v) {
  if (dim < 1 || kind < 0 || kind > 2 || !v) {
    set_error("hphi_reference_start: bad arguments");
    return -1;
  }
  std::vector<double> out;
  reference_random_start(dim, (RefStartKind)kind, initial_iv, sample, vec_type, threads, count, &out);
  std::memcpy(v, out.data(), sizeof(double) * out.size());
  return 0;
}

// Green's functions of host vector `vec` (HPhi layout); a vector with no imaginary part runs
// through the real kernels (checked on the device after one upload).
static int green_host(hphi_handle *h, int body, int n, const int *rows, const double *vec, std::vector<double> *out,
                      std::vector<char> *trail) {
  Sector *s = h->sector;
  std::vector<GreenTerm> terms;
  std::string err;
  if (compile_green(s->model, body, rows, n, &terms, trail, &err) != 0) {
    set_error(err);
    return -1;
  }
  cudaSetDevice(s->device);
  void *d = nullptr;
  VecType vt = kComplex128;
  if (green_stage_host_vector(s, vec, &d, &vt) != 0) return -1;
  const int rc = green_expect(s, vt, d, terms, out);
  cudaStreamSynchronize(s->stream);
  cudaFree(d);
  return rc;
}

int hphi_expec_green(hphi_handle *h, int body, int n, const int *rows, const double *vec, double *out) {
  CHECK_HANDLE(h);
  if ((body != 1 && body != 2 && body != 3 && body != 4 && body != 6) || n < 0 || (n > 0 && (!rows || !vec || !out))) {
    set_error("hphi_expec_green: bad arguments");
    return -1;
  }
  if (n == 0) return 0;
  std::vector<double> g;
  std::vector<char> trail;
  if (green_host(h, body, n, rows, vec, &g, &trail) != 0) return -1;
  std::memcpy(out, g.data(), sizeof(double) * g.size());
  return 0;
}

int hphi_expec_green_device(hphi_handle *h, int body, int n, const int *rows, int vec_type, const void *d_vec,
                            double *out) {
  CHECK_HANDLE(h);
  if ((body != 1 && body != 2 && body != 3 && body != 4 && body != 6) || n < 0 ||
      (vec_type != kReal64 && vec_type != kComplex128) ||
      (n > 0 && (!rows || !d_vec || !out))) {
    set_error("hphi_expec_green_device: bad arguments");
    return -1;
  }
  if (n == 0) return 0;
  Sector *s = h->sector;
  std::vector<GreenTerm> terms;
  std::vector<char> trail;
  std::string err;
  if (compile_green(s->model, body, rows, n, &terms, &trail, &err) != 0) {
    set_error(err);
    return -1;
  }
  std::vector<double> g;
  if (green_expect(s, (VecType)vec_type, d_vec, terms, &g) != 0) return -1;
  std::memcpy(out, g.data(), sizeof(double) * g.size());
  return 0;
}

static int expec_model_green(hphi_handle *h, int body, const double *vec, double *out, const char *path) {
  CHECK_HANDLE(h);
  const Model &m = h->sector->model;
  const int n = body == 1 ? (int)m.green_one.size() : (int)m.green_two.size();
  if (n == 0) return 0;  // the reference returns without a file (src/expec_cisajs.c:80)
  if (!vec) { set_error("null vector"); return -1; }
  GreenValues g;
  std::vector<char> trail;
  if (green_host(h, body, n, body == 1 ? m.green_one[0].data() : m.green_two[0].data(), vec,
                 body == 1 ? &g.one : &g.two, body == 1 ? &trail : &g.trail_two) != 0)
    return -1;
  if (out) std::memcpy(out, (body == 1 ? g.one : g.two).data(), sizeof(double) * 2 * (size_t)n);
  if (path && write_green_file(m, g, body, path) != 0) return -1;
  return 0;
}

int hphi_expec_cisajs(hphi_handle *h, const double *vec, double *out, const char *path) {
  return expec_model_green(h, 1, vec, out, path);
}

int hphi_expec_cisajscktaltdc(hphi_handle *h, const double *vec, double *out, const char *path) {
  return expec_model_green(h, 2, vec, out, path);
}

}  // extern "C"
