// H*v entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the time they need an H*v: a solver running
// under a memory budget owned by another component (a framework's caching allocator
// that must account for every byte on the device), or a latency-critical loop that
// cannot afford cudaMalloc's implicit device-wide synchronisation.  For them
// hphi_mltply_device_noalloc runs the same H*v as hphi_mltply_device_async, but the
// kernel's scratch (launch coefficients, the block counters of the Hubbard kernel and the
// per-block partial sums of <v1|H|v1>) lives in one file-scope device array below instead
// of buffers allocated for the handle.  The caller passes the input and output vectors.
//
// The array has a fixed size (kScratchDoubles doubles = 128 KiB) and exists on every
// GPU that loads this library, until the process exits.  Calls share it: two calls whose
// work overlaps on the GPU (different streams, different threads, or different handles on
// the same device) race on it, so callers must order them.  Each call waits for its
// stream before it returns (it reads <v1|H|v1> back to the host).  The first call on a
// device looks up the array's device address (cudaGetSymbolAddress, which may load the
// module); make that first call before any stream capture.  The partial sums it needs are
// 2 per CTA of the two passes for real vectors on the product-layout Hubbard kernels
// (a few thousand), 2 per row of the up-spin matrix for its complex one-pass kernel, 2 per
// block otherwise; a sector that needs more than the array holds is refused.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/hphi_b200.h"
#include "engine.hpp"

namespace hphi {
Sector *handle_sector(hphi_handle *h);

namespace {

constexpr size_t kScratchDoubles = 16384;     // 128 KiB per device
constexpr size_t kCoefSlot = 0;               // [0, 2): acc, scale
constexpr size_t kResultSlot = 2;             // [2, 4): sum conj(v1) H v1
constexpr size_t kCounterSlot = 4;            // [4, 5): two int block counters
constexpr size_t kPartialSlot = 8;            // [8, ...): per-block partial sums
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_scratch[kScratchDoubles];

std::mutex g_mutex;
double *g_scratch_ptr[kMaxDevices] = {};

// Device address of g_scratch on `device` (which must be current); looked up once per device.
int scratch_address(int device, double **out) {
  if (device < 0 || device >= kMaxDevices) {
    set_error("hphi_mltply_device_noalloc: device index out of range");
    return -1;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_ptr[device]) {
    double *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error(std::string("hphi_mltply_device_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return -1;
    }
    g_scratch_ptr[device] = p;
  }
  *out = g_scratch_ptr[device];
  return 0;
}

}  // namespace
}  // namespace hphi

using namespace hphi;

extern "C" int hphi_mltply_device_noalloc(hphi_handle *h, int vec_type, void *d_v0, const void *d_v1, double acc,
                                          double scale, double *prdct) {
  Sector *s = handle_sector(h);
  if (!s) {
    set_error("invalid handle");
    return -1;
  }
  cudaGetLastError();
  if (vec_type != HPHI_REAL64 && vec_type != HPHI_COMPLEX128) {
    set_error("bad vec_type");
    return -1;
  }
  if (cudaSetDevice(s->device) != cudaSuccess) {
    set_error("hphi_mltply_device_noalloc: cudaSetDevice failed");
    return -1;
  }
  const size_t need = hv_scratch_doubles(s, (VecType)vec_type);
  if (need > kScratchDoubles - kPartialSlot) {
    set_error("hphi_mltply_device_noalloc: this sector needs " + std::to_string(need) +
              " partial sums, more than the fixed scratch of " + std::to_string(kScratchDoubles - kPartialSlot));
    return -1;
  }
  double *scr = nullptr;
  if (scratch_address(s->device, &scr) != 0) return -1;
  const double coef[2] = {acc, scale};
  if (cudaMemcpyAsync(scr + kCoefSlot, coef, sizeof(coef), cudaMemcpyHostToDevice, s->stream) != cudaSuccess) {
    set_error("hphi_mltply_device_noalloc: coefficient copy failed");
    return -1;
  }
  int *counters = reinterpret_cast<int *>(scr + kCounterSlot);
  if (hv_native_scratch(s, (VecType)vec_type, d_v1, d_v0, scr + kCoefSlot, scr + kResultSlot, scr + kPartialSlot,
                        counters) != 0)
    return -1;
  double out[2];
  if (cudaMemcpyAsync(out, scr + kResultSlot, sizeof(out), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess) {
    set_error("hphi_mltply_device_noalloc: result copy failed");
    return -1;
  }
  if (prdct) {
    prdct[0] = out[0];
    prdct[1] = out[1];
  }
  return 0;
}
