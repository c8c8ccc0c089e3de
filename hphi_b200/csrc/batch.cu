// Batched Lanczos engine and request server (batch.hpp).
//
// Work unit: a tile of consecutive rows of one instance.  Every phase kernel is launched
// with a persistent grid whose CTAs draw tiles from a global counter (largest instances
// first), so instances of very different sizes share the GPU without a launch each.
// Per tile the CTA writes its partial sums; the CTA that completes an instance's last tile
// (counted with an atomic per instance) sums that instance's partials in tile order and
// updates its scalars, so no extra reduction launch and no host round trip is needed.
// Row work is the gather form of the general H*v kernel (hv.cu): each thread owns output
// rows, tests the row's configuration against the compiled terms and gathers the sources
// through list_2_1 / list_2_2 (GetOffComp, src/bitcalc.c:195-223).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hphi_b200.h"
#include "batch.hpp"
#include "device_util.cuh"
#include "driver.hpp"
#include "split.cuh"

namespace hphi {
namespace {

// Launch kinds and per-instance modes.
enum Kind : int { kSetup = 0, kStep = 1, kRefineKind = 2, kTuneKind = 3 };
enum Mode : int { kIdle = 0, kInit = 1, kForward = 2, kReplayInit = 3, kReplay = 4, kRefine = 5 };
constexpr int kSmemTermCap = 1000;        // terms staged in shared memory (48,000 B)
constexpr int kMaxTilesPerInstance = 16384;
constexpr int kStSlots = 16;              // per-instance device scalars
constexpr int kGraphSteps = 16;

// st slots: [0,1] <Q|HQ> raw, [2] acc, [3] s, [4] alpha*s, [5] |P|^2, [6] |start|^2,
// [8,9] <x|Hx>, [10] |x|^2, [11] Rayleigh quotient, [12] |Hx - E x|^2.
struct BInst {
  const uint64_t *list_1;
  const uint32_t *l21, *l22;
  const double *diag;
  const BitTerm *terms;         // generic-path terms (the split plan holds the others)
  SplitView split;
  int64_t dim;
  uint64_t lo_mask;
  uint64_t seed;
  int nterms, lo_bits, gc, cplx;
  int tile_begin, tile_end;
  void *vec0, *vec1, *vstart;   // storage precision
  void *vg, *w;                 // FP64 (rebuilt eigenvector and H times it)
  double *st, *alpha, *beta, *coef;
  int *kstep, *done;
  int kmax;                     // step limit of the current mode
  int mode;
};

struct BTile {
  int64_t row0;
  int inst;
  int nrows;
};

struct BArgs {
  const BInst *inst;
  const BTile *tiles;
  int ntiles;
  int smem_terms;
  double *part;
  int *counter;
};

// ---------------------------------------------------------------- storage traits
template <typename S, bool C> struct Stor;
template <> struct Stor<double, false> {
  using M = double;
  using A = double;
  static __device__ __forceinline__ A ldg(const M *p, int64_t i) { return __ldg(p + i); }
  static __device__ __forceinline__ A ld(const M *p, int64_t i) { return p[i]; }
  static __device__ __forceinline__ M pack(A v) { return v; }
  static __device__ __forceinline__ A unpack(M v) { return v; }
};
template <> struct Stor<float, false> {
  using M = float;
  using A = double;
  static __device__ __forceinline__ A ldg(const M *p, int64_t i) { return (double)__ldg(p + i); }
  static __device__ __forceinline__ A ld(const M *p, int64_t i) { return (double)p[i]; }
  static __device__ __forceinline__ M pack(A v) { return (float)v; }
  static __device__ __forceinline__ A unpack(M v) { return (double)v; }
};
template <> struct Stor<double, true> {
  using M = double2;
  using A = cplx;
  static __device__ __forceinline__ A ldg(const M *p, int64_t i) { const double2 v = __ldg(p + i); return cplx{v.x, v.y}; }
  static __device__ __forceinline__ A ld(const M *p, int64_t i) { const double2 v = p[i]; return cplx{v.x, v.y}; }
  static __device__ __forceinline__ M pack(A v) { return make_double2(v.x, v.y); }
  static __device__ __forceinline__ A unpack(M v) { return cplx{v.x, v.y}; }
};
template <> struct Stor<float, true> {
  using M = float2;
  using A = cplx;
  static __device__ __forceinline__ A ldg(const M *p, int64_t i) { const float2 v = __ldg(p + i); return cplx{v.x, v.y}; }
  static __device__ __forceinline__ A ld(const M *p, int64_t i) { const float2 v = p[i]; return cplx{v.x, v.y}; }
  static __device__ __forceinline__ M pack(A v) { return make_float2((float)v.x, (float)v.y); }
  static __device__ __forceinline__ A unpack(M v) { return cplx{(double)v.x, (double)v.y}; }
};

// ---------------------------------------------------------------- tile plumbing
__device__ __forceinline__ int next_tile(int *counter) {
  __shared__ int s_tile;
  __syncthreads();
  if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1);
  __syncthreads();
  return s_tile;
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

// Whether instance I works in a launch of this kind (the same answer in every thread and
// for every tile of I within one launch: kstep changes only after I's last tile).
__device__ __forceinline__ bool takes_part(int kind, const BInst &I) {
  const int m = I.mode;
  if (kind == kTuneKind) return true;
  if (kind == kSetup) return m == kInit || m == kReplayInit;
  if (kind == kStep) return (m == kForward || m == kReplay) && *I.kstep < I.kmax;
  return m == kRefine;
}

// Publishes the tile's partial sums; true (in every thread) in the CTA that completed the
// instance's last tile.
__device__ __forceinline__ bool finish_tile(const BArgs &A, const BInst &I, int t, double (&pr)[3]) {
  __shared__ int s_last;
  block_sum<3>(pr);
  if (threadIdx.x == 0) {
    double *p = A.part + 3 * (size_t)t;
    p[0] = pr[0];
    p[1] = pr[1];
    p[2] = pr[2];
    __threadfence();
    const int prev = atomicAdd(I.done, 1);
    s_last = (prev == I.tile_end - I.tile_begin - 1);
  }
  __syncthreads();
  return s_last != 0;
}

// Sum of the instance's tile partials in tile order (thread 0 gets it).
__device__ __forceinline__ void reduce_instance(const BArgs &A, const BInst &I, double (&q)[3]) {
  __threadfence();
  q[0] = q[1] = q[2] = 0.0;
  for (int u = I.tile_begin + threadIdx.x; u < I.tile_end; u += blockDim.x) {
    q[0] += __ldcg(A.part + 3 * (size_t)u);
    q[1] += __ldcg(A.part + 3 * (size_t)u + 1);
    q[2] += __ldcg(A.part + 3 * (size_t)u + 2);
  }
  block_sum<3>(q);
}

// ---------------------------------------------------------------- H*v rows
template <typename S, bool C, bool GC>
__device__ __forceinline__ void hv_rows(const BInst &I, const BitTerm *terms, int64_t r0, int nrows,
                                        const void *v1v, void *v0v, double acc, double scale, double (&pr)[3]) {
  using St = Stor<S, C>;
  using A = typename St::A;
  const typename St::M *__restrict__ v1 = (const typename St::M *)v1v;
  typename St::M *__restrict__ v0 = (typename St::M *)v0v;
  const uint64_t *__restrict__ list_1 = I.list_1;
  const uint32_t *__restrict__ l21 = I.l21;
  const uint32_t *__restrict__ l22 = I.l22;
  const double *__restrict__ diag = I.diag;
  const int nterms = I.nterms, lo_bits = I.lo_bits;
  const uint64_t lo_mask = I.lo_mask;
  for (int j = threadIdx.x; j < nrows; j += blockDim.x) {
    const int64_t r = r0 + j;
    const uint64_t c = GC ? (uint64_t)r : __ldg(list_1 + r);
    const A x = St::ldg(v1, r);
    A y = VT<A>::scale(__ldg(diag + r), x);
    if (I.split.lo_ptr)
      y = split_terms<A, GC>(I.split, c, r, lo_bits, lo_mask, l22, [&](int64_t jj) { return St::ldg(v1, jj); }, y);
    for (int k = 0; k < nterms; k++) {
      const BitTerm t = terms[k];
      if ((c & t.cm) != t.cv) continue;
      const uint64_t src = c ^ t.flip;
      int64_t jj;
      if (GC) {
        jj = (int64_t)src;
      } else {
        const uint32_t a = __ldg(l21 + (src & lo_mask));
        const uint32_t b = __ldg(l22 + (src >> lo_bits));
        if (a == 0u || b == 0u) continue;
        jj = (int64_t)a + (int64_t)b - 3;
      }
      const bool neg = __popcll(c & t.sm) & 1;
      y = VT<A>::add(y, VT<A>::cmul_re_im(neg ? -t.re : t.re, neg ? -t.im : t.im, St::ldg(v1, jj)));
    }
    pr[0] += VT<A>::conj_mul_re(x, y);
    pr[1] += VT<A>::conj_mul_im(x, y);
    pr[2] += VT<A>::abs2(x);
    y = VT<A>::scale(scale, y);
    if (acc == 0.0) v0[r] = St::pack(y);
    else v0[r] = St::pack(VT<A>::add(VT<A>::scale(acc, St::ld(v0, r)), y));
  }
}

template <typename S>
__device__ __forceinline__ void hv_dispatch(const BInst &I, const BitTerm *terms, int64_t r0, int n, const void *v1,
                                            void *v0, double acc, double scale, double (&pr)[3]) {
  if (I.cplx) {
    if (I.gc) hv_rows<S, true, true>(I, terms, r0, n, v1, v0, acc, scale, pr);
    else hv_rows<S, true, false>(I, terms, r0, n, v1, v0, acc, scale, pr);
  } else {
    if (I.gc) hv_rows<S, false, true>(I, terms, r0, n, v1, v0, acc, scale, pr);
    else hv_rows<S, false, false>(I, terms, r0, n, v1, v0, acc, scale, pr);
  }
}

// hv phase.  kStep: forward or replay instances on the storage vectors (S = storage type);
// kRefineKind: H times the rebuilt FP64 vector (launched with S = double); kTuneKind:
// every instance, no scalar update.
template <typename S>
__global__ void batch_hv_kernel(BArgs A, int parity, int kind) {
  extern __shared__ BitTerm sterms[];
  int loaded = -1;
  for (;;) {
    const int t = next_tile(A.counter);
    if (t >= A.ntiles) break;
    const BTile tile = A.tiles[t];
    const BInst &I = A.inst[tile.inst];
    if (!takes_part(kind, I)) continue;
    const BitTerm *terms = I.terms;
    if (I.nterms <= A.smem_terms) {
      if (loaded != tile.inst) {
        __syncthreads();
        for (int k = threadIdx.x; k < I.nterms; k += blockDim.x) sterms[k] = I.terms[k];
        __syncthreads();
        loaded = tile.inst;
      }
      terms = sterms;
    }
    const void *v1;
    void *v0;
    double acc, scale;
    if (kind == kRefineKind) {
      v1 = I.vg;
      v0 = I.w;
      acc = 0.0;
      scale = 1.0;
    } else {
      v1 = parity ? I.vec1 : I.vec0;
      v0 = parity ? I.vec0 : I.vec1;
      acc = I.st[2];
      scale = I.st[3];
    }
    double pr[3] = {0.0, 0.0, 0.0};
    hv_dispatch<S>(I, terms, tile.row0, tile.nrows, v1, v0, acc, scale, pr);
    if (kind == kTuneKind) continue;
    if (finish_tile(A, I, t, pr)) {
      double q[3];
      reduce_instance(A, I, q);
      if (threadIdx.x == 0) {
        double *st = I.st;
        *I.done = 0;
        const int k = *I.kstep + 1;
        if (kind == kRefineKind) {
          st[8] = q[0];
          st[9] = q[1];
          st[10] = q[2];
          st[11] = q[0] / q[2];
        } else if (I.mode == kForward) {
          st[0] = q[0];
          st[1] = q[1];
          const double s = st[3];
          const double a = s * s * q[0];
          I.alpha[k] = a;
          st[4] = a * s;
        } else {  // kReplay: the stored alpha gives the same sweep coefficient
          st[4] = I.alpha[k] * st[3];
        }
      }
    }
  }
  retire(A.counter);
}

// ---------------------------------------------------------------- vector sweeps
template <typename S, bool C>
__device__ __forceinline__ void sweep_rows(const BInst &I, int64_t r0, int nrows, int parity, int kind, double a,
                                           double cv, double E, double (&pr)[3]) {
  using St = Stor<S, C>;
  using D = Stor<double, C>;  // FP64 vectors (vg, w)
  using A = typename St::A;
  typename St::M *p = (typename St::M *)(parity ? I.vec0 : I.vec1);
  const typename St::M *q = (const typename St::M *)(parity ? I.vec1 : I.vec0);
  const int mode = I.mode;
  for (int j = threadIdx.x; j < nrows; j += blockDim.x) {
    const int64_t r = r0 + j;
    if (kind == kStep) {
      const A qv = St::ld(q, r);
      const A w = St::unpack(St::pack(VT<A>::sub(St::ld(p, r), VT<A>::scale(a, qv))));
      p[r] = St::pack(w);
      pr[0] += VT<A>::abs2(w);
      if (mode == kReplay) {
        typename D::M *vg = (typename D::M *)I.vg;
        vg[r] = D::pack(VT<A>::add(D::ld(vg, r), VT<A>::scale(cv, qv)));
      }
    } else if (kind == kSetup) {
      if (mode == kInit) {
        const uint64_t c = I.gc ? (uint64_t)r : I.list_1[r];
        A v;
        if constexpr (C) v = cplx{start_value(I.seed, c, 0), start_value(I.seed, c, 1)};
        else v = start_value(I.seed, c, 0);
        const typename St::M m = St::pack(v);
        ((typename St::M *)I.vec0)[r] = m;
        ((typename St::M *)I.vstart)[r] = m;
        pr[0] += VT<A>::abs2(St::unpack(m));
      } else {  // kReplayInit
        ((typename St::M *)I.vec0)[r] = ((const typename St::M *)I.vstart)[r];
        typename D::M *vg = (typename D::M *)I.vg;
        vg[r] = D::pack(VT<A>::zero());
      }
    } else {  // kRefineKind: residual of the rebuilt vector
      const typename D::M *w = (const typename D::M *)I.w;
      const typename D::M *x = (const typename D::M *)I.vg;
      const A d = VT<A>::sub(D::ld(w, r), VT<A>::scale(E, D::ld(x, r)));
      pr[0] += VT<A>::abs2(d);
    }
  }
}

template <typename S>
__global__ void batch_sweep_kernel(BArgs A, int parity, int kind) {
  for (;;) {
    const int t = next_tile(A.counter);
    if (t >= A.ntiles) break;
    const BTile tile = A.tiles[t];
    const BInst &I = A.inst[tile.inst];
    if (!takes_part(kind, I)) continue;
    const int k = *I.kstep + 1;
    const double a = I.st[4];
    const double cv = (kind == kStep && I.mode == kReplay) ? I.coef[k] * I.st[3] : 0.0;
    const double E = (kind == kRefineKind) ? I.st[11] : 0.0;
    double pr[3] = {0.0, 0.0, 0.0};
    if (I.cplx) sweep_rows<S, true>(I, tile.row0, tile.nrows, parity, kind, a, cv, E, pr);
    else sweep_rows<S, false>(I, tile.row0, tile.nrows, parity, kind, a, cv, E, pr);
    if (finish_tile(A, I, t, pr)) {
      double q[3];
      reduce_instance(A, I, q);
      if (threadIdx.x == 0) {
        double *st = I.st;
        *I.done = 0;
        if (kind == kStep) {
          const double b = (I.mode == kForward) ? sqrt(q[0]) : I.beta[k];
          if (I.mode == kForward) I.beta[k] = b;
          st[5] = q[0];
          st[2] = -b * st[3];
          st[3] = 1.0 / b;
          *I.kstep = k;
        } else if (kind == kSetup) {
          if (I.mode == kInit) st[6] = q[0];
          st[2] = 0.0;
          st[3] = 1.0 / sqrt(st[6]);
          *I.kstep = 0;
        } else {
          st[12] = q[0];
        }
      }
    }
  }
  retire(A.counter);
}

// ---------------------------------------------------------------- host side
int cuda_ok(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    set_error(std::string("batch: ") + what + ": " + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}
#define BRET(x) do { if ((x) != 0) return -1; } while (0)

std::mutex g_tune_mutex;
std::map<std::string, BatchTuning> g_tune_cache;

struct Slot {
  bool used = false;
  Sector *s = nullptr;
  bool owned = false;       // sector freed with the slot (server members)
  BInst inst{};
  void *vecs = nullptr;     // vec0, vec1, vstart
  void *fp64 = nullptr;     // vg, w
  double *scal = nullptr;   // st, alpha, beta, coef, then kstep / done
  int cap = 0;              // alpha / beta capacity (steps)
  int host_k = 0;           // steps of the current mode known to be enqueued
};

}  // namespace

struct Batch {
  Precision prec = kFP64;
  int device = 0, num_sms = 0;
  cudaStream_t stream = nullptr;
  std::vector<Slot> slots;
  BInst *d_inst = nullptr;
  size_t inst_cap = 0;
  BTile *d_tiles = nullptr;
  size_t tile_cap = 0;
  int ntiles = 0;
  double *d_part = nullptr;
  int *d_counter = nullptr;
  int smem_terms = 0;
  bool plan_dirty = true;
  int plan_version = 0;
  BatchTuning tune;
  bool tuned = false;
  cudaGraphExec_t graph = nullptr;
  int graph_version = -1;
};

namespace {

size_t storage_elem(Precision prec, bool cplx) { return (prec == kFP32 ? 4 : 8) * (cplx ? 2 : 1); }

void release_graph(Batch *b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graph_version = -1;
}

int alloc_scalars(Slot &sl, int cap) {
  if (sl.scal && sl.cap >= cap) return 0;
  if (sl.scal) cudaFree(sl.scal);
  sl.scal = nullptr;
  const size_t stride = (size_t)cap + 2;
  const size_t ndbl = kStSlots + 3 * stride + 1;
  BRET(cuda_ok(cudaMalloc(&sl.scal, sizeof(double) * ndbl), "alloc scalars"));
  BRET(cuda_ok(cudaMemset(sl.scal, 0, sizeof(double) * ndbl), "clear scalars"));
  sl.cap = cap;
  BInst &I = sl.inst;
  I.st = sl.scal;
  I.alpha = sl.scal + kStSlots;
  I.beta = I.alpha + stride;
  I.coef = I.beta + stride;
  I.kstep = (int *)(I.coef + stride);
  I.done = I.kstep + 1;
  return 0;
}

int alloc_fp64(Slot &sl) {
  if (sl.fp64) return 0;
  const size_t bytes = (size_t)(sl.inst.cplx ? 16 : 8) * (size_t)sl.inst.dim;
  BRET(cuda_ok(cudaMalloc(&sl.fp64, 2 * bytes), "alloc FP64 vectors"));
  sl.inst.vg = sl.fp64;
  sl.inst.w = (char *)sl.fp64 + bytes;
  return 0;
}

void free_slot(Slot &sl) {
  if (sl.vecs) cudaFree(sl.vecs);
  if (sl.fp64) cudaFree(sl.fp64);
  if (sl.scal) cudaFree(sl.scal);
  if (sl.owned) sector_free(sl.s);
  sl = Slot();
}

int engine_add(Batch *b, Sector *s, bool owned, uint64_t seed, int cap, int *slot_out) {
  if (s->device != b->device) {
    set_error("batch: every instance must be open on the batch's device");
    return -1;
  }
  int idx = -1;
  for (size_t i = 0; i < b->slots.size(); i++)
    if (!b->slots[i].used) { idx = (int)i; break; }
  if (idx < 0) {
    idx = (int)b->slots.size();
    b->slots.emplace_back();
  }
  Slot &sl = b->slots[idx];
  sl = Slot();
  BInst &I = sl.inst;
  I.list_1 = s->d_list_1;
  I.l21 = s->d_list_2_1;
  I.l22 = s->d_list_2_2;
  I.diag = s->d_diag;
  I.terms = s->split.gen;
  I.split = split_view(s->split);
  I.dim = s->dim;
  I.lo_mask = s->ihfbit - 1;
  I.nterms = s->split.ngen;
  I.lo_bits = s->lo_bits;
  I.gc = s->gc ? 1 : 0;
  I.cplx = (default_vec_type(*s) == kComplex128) ? 1 : 0;
  I.seed = seed;
  I.mode = kIdle;
  const size_t bytes = storage_elem(b->prec, I.cplx) * (size_t)I.dim;
  if (cuda_ok(cudaMalloc(&sl.vecs, 3 * bytes), "alloc vectors")) { sl = Slot(); return -1; }
  I.vec0 = sl.vecs;
  I.vec1 = (char *)sl.vecs + bytes;
  I.vstart = (char *)sl.vecs + 2 * bytes;
  if (alloc_scalars(sl, cap)) { cudaFree(sl.vecs); sl = Slot(); return -1; }
  sl.used = true;
  sl.s = s;
  sl.owned = owned;
  b->plan_dirty = true;
  *slot_out = idx;
  return 0;
}

void engine_remove(Batch *b, int idx) {
  free_slot(b->slots[idx]);
  b->plan_dirty = true;
}

int rows_per_tile(const BatchTuning &t) { return t.threads * t.rows_per_thread; }

// Tiles of every member, largest first; an instance's tiles depend only on its dimension
// and the tile size (at most kMaxTilesPerInstance per instance: bigger ones get longer
// tiles), so its partial sums and results do not depend on the other members.
int upload_plan(Batch *b, const BatchTuning &t) {
  std::vector<int> order;
  for (size_t i = 0; i < b->slots.size(); i++)
    if (b->slots[i].used) order.push_back((int)i);
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return b->slots[x].inst.dim > b->slots[y].inst.dim; });
  std::vector<BTile> tiles;
  const int64_t base = rows_per_tile(t);
  int smem_terms = 0;
  for (int i : order) {
    BInst &I = b->slots[i].inst;
    int64_t rows = base;
    const int64_t nt = (I.dim + base - 1) / base;
    if (nt > kMaxTilesPerInstance) rows = base * ((nt + kMaxTilesPerInstance - 1) / kMaxTilesPerInstance);
    I.tile_begin = (int)tiles.size();
    for (int64_t r0 = 0; r0 < I.dim; r0 += rows) tiles.push_back(BTile{r0, i, (int)std::min<int64_t>(rows, I.dim - r0)});
    I.tile_end = (int)tiles.size();
    if (I.nterms <= kSmemTermCap) smem_terms = std::max(smem_terms, I.nterms);
  }
  if (tiles.size() > b->tile_cap || b->slots.size() > b->inst_cap) release_graph(b);
  if (tiles.size() > b->tile_cap) {
    if (b->d_tiles) cudaFree(b->d_tiles);
    if (b->d_part) cudaFree(b->d_part);
    b->d_tiles = nullptr;
    b->d_part = nullptr;
    b->tile_cap = std::max<size_t>(tiles.size(), 2 * b->tile_cap);
    BRET(cuda_ok(cudaMalloc(&b->d_tiles, sizeof(BTile) * b->tile_cap), "alloc tiles"));
    BRET(cuda_ok(cudaMalloc(&b->d_part, 3 * sizeof(double) * b->tile_cap), "alloc partials"));
  }
  if (b->slots.size() > b->inst_cap) {
    if (b->d_inst) cudaFree(b->d_inst);
    b->d_inst = nullptr;
    b->inst_cap = std::max<size_t>(b->slots.size(), 2 * b->inst_cap);
    BRET(cuda_ok(cudaMalloc(&b->d_inst, sizeof(BInst) * b->inst_cap), "alloc instances"));
  }
  b->ntiles = (int)tiles.size();
  b->smem_terms = smem_terms;
  if (!tiles.empty())
    BRET(cuda_ok(cudaMemcpyAsync(b->d_tiles, tiles.data(), sizeof(BTile) * tiles.size(), cudaMemcpyHostToDevice,
                                 b->stream), "upload tiles"));
  b->plan_dirty = false;
  b->plan_version++;
  return 0;
}

// Descriptors (modes, step limits, pointers) to the device; re-plans first if members changed.
int upload(Batch *b) {
  if (b->plan_dirty) BRET(upload_plan(b, b->tune));
  std::vector<BInst> h(b->slots.size());
  for (size_t i = 0; i < b->slots.size(); i++) {
    h[i] = b->slots[i].inst;
    if (!b->slots[i].used) h[i].mode = kIdle;
  }
  if (!h.empty())
    BRET(cuda_ok(cudaMemcpyAsync(b->d_inst, h.data(), sizeof(BInst) * h.size(), cudaMemcpyHostToDevice, b->stream),
                 "upload instances"));
  return 0;
}

BArgs args_of(const Batch *b) {
  BArgs a;
  a.inst = b->d_inst;
  a.tiles = b->d_tiles;
  a.ntiles = b->ntiles;
  a.smem_terms = b->smem_terms;
  a.part = b->d_part;
  a.counter = b->d_counter;
  return a;
}

int grid_of(const Batch *b, const BatchTuning &t) { return std::max(1, std::min(b->ntiles, t.ctas_per_sm * b->num_sms)); }

template <typename S>
void launch_hv(Batch *b, const BatchTuning &t, int parity, int kind) {
  if (b->ntiles == 0) return;
  batch_hv_kernel<S><<<grid_of(b, t), t.threads, sizeof(BitTerm) * b->smem_terms, b->stream>>>(args_of(b), parity,
                                                                                                 kind);
}
template <typename S>
void launch_sweep(Batch *b, const BatchTuning &t, int parity, int kind) {
  if (b->ntiles == 0) return;
  batch_sweep_kernel<S><<<grid_of(b, t), t.threads, 0, b->stream>>>(args_of(b), parity, kind);
}

void step_pair(Batch *b, int parity) {
  if (b->prec == kFP32) {
    launch_hv<float>(b, b->tune, parity, kStep);
    launch_sweep<float>(b, b->tune, parity, kStep);
  } else {
    launch_hv<double>(b, b->tune, parity, kStep);
    launch_sweep<double>(b, b->tune, parity, kStep);
  }
}

int engine_setup(Batch *b) {
  if (b->prec == kFP32) launch_sweep<float>(b, b->tune, 0, kSetup);
  else launch_sweep<double>(b, b->tune, 0, kSetup);
  return cuda_ok(cudaGetLastError(), "setup launch");
}

int engine_refine(Batch *b) {
  launch_hv<double>(b, b->tune, 0, kRefineKind);
  launch_sweep<double>(b, b->tune, 0, kRefineKind);
  return cuda_ok(cudaGetLastError(), "refine launch");
}

// `count` recurrence steps of every forward / replay member, starting at parity 0 (every
// member's step count is even at iteration boundaries: counts are even or end a mode).
// With use_graph, blocks of kGraphSteps steps replay one captured graph.
int engine_steps(Batch *b, int count, bool use_graph) {
  int done = 0;
  if (use_graph && count >= kGraphSteps) {
    if (b->graph_version != b->plan_version) {
      release_graph(b);
      cudaGraph_t graph = nullptr;
      BRET(cuda_ok(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture"));
      for (int k = 0; k < kGraphSteps; k++) step_pair(b, k & 1);
      BRET(cuda_ok(cudaStreamEndCapture(b->stream, &graph), "end capture"));
      const cudaError_t ie = cudaGraphInstantiate(&b->graph, graph, 0);
      cudaGraphDestroy(graph);
      BRET(cuda_ok(ie, "instantiate graph"));
      b->graph_version = b->plan_version;
    }
    for (; done + kGraphSteps <= count; done += kGraphSteps)
      BRET(cuda_ok(cudaGraphLaunch(b->graph, b->stream), "graph launch"));
  }
  for (; done < count; done++) step_pair(b, done & 1);
  return cuda_ok(cudaGetLastError(), "step launch");
}

std::string signature(const Batch *b) {
  std::string s = std::to_string((int)b->prec) + ":" + std::to_string(b->device);
  for (const Slot &sl : b->slots)
    if (sl.used)
      s += "|" + std::to_string(sl.inst.dim) + "," + std::to_string(sl.inst.nterms) + "," +
           std::to_string(sl.inst.cplx) + "," + std::to_string(sl.inst.gc);
  return s;
}

int engine_create(int device, Precision prec, Batch **out) {
  *out = nullptr;
  Batch *b = new Batch();
  b->prec = prec;
  b->device = device;
  auto fail = [&]() { batch_free(b); return -1; };
  if (cuda_ok(cudaSetDevice(device), "set device") ||
      cuda_ok(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream") ||
      cuda_ok(cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device), "SM count") ||
      cuda_ok(cudaMalloc(&b->d_counter, 2 * sizeof(int)), "alloc counter") ||
      cuda_ok(cudaMemset(b->d_counter, 0, 2 * sizeof(int)), "clear counter"))
    return fail();
  const int smem = (int)(sizeof(BitTerm) * kSmemTermCap);
  cudaFuncSetAttribute(batch_hv_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(batch_hv_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  *out = b;
  return 0;
}

int read_slot(Batch *b, int idx, size_t ndbl, std::vector<double> *out) {
  out->resize(ndbl);
  return cuda_ok(cudaMemcpyAsync(out->data(), b->slots[idx].scal, sizeof(double) * ndbl, cudaMemcpyDeviceToHost,
                                 b->stream), "read scalars");
}

// Steps used and lowest eigenvalue of a slot's tridiagonal matrix after `k` steps.
void tridiag_of(const std::vector<double> &scal, int cap, int k, int64_t dim, int *m_out, double *e_out) {
  const size_t stride = (size_t)cap + 2;
  const double *al = scal.data() + kStSlots + 1;
  const double *be = scal.data() + kStSlots + stride + 1;
  int m = (int)std::min<int64_t>(k, dim);
  for (int j = 0; j < m; j++)
    if (!(std::fabs(be[j]) >= 1e-14)) { m = j + 1; break; }
  *m_out = m;
  *e_out = tridiag_eigenvalue(al, be, m, 0);
}

// Replay length and coefficients of the ground state.  Without reorthogonalisation the
// recurrence keeps going after the ground state has converged and produces ghost copies of
// it; a Ritz vector of the full T_m then mixes the copies and loses accuracy.  So the vector
// is taken from T_mc, mc the first step (checked every 4) whose Ritz residual estimate
// beta_k |s_k| (s_k the last component of the lowest eigenvector of T_k) is below
// 1e-7 max(1, |E_k|), as the reference's driver stops at convergence before building its
// eigenvector.  The dropped tail of that Ritz vector has norm below replay_tol, which moves
// the Rayleigh quotient by about replay_tol^2 times the spectral width.
int replay_plan(const std::vector<double> &scal, int cap, int m, double replay_tol, std::vector<double> *coef) {
  const size_t stride = (size_t)cap + 2;
  const double *al = scal.data() + kStSlots + 1;
  const double *be = scal.data() + kStSlots + stride + 1;
  std::vector<double> c;
  int mc = m;
  for (int k = 8; k < m; k += 4) {
    const double ek = tridiag_eigenvalue(al, be, k, 0);
    tridiag_eigenvector(al, be, k, ek, &c);
    if (std::fabs(be[k - 1] * c[k - 1]) <= 1e-7 * std::max(1.0, std::fabs(ek))) {
      mc = k;
      break;
    }
  }
  m = mc;
  tridiag_eigenvector(al, be, m, tridiag_eigenvalue(al, be, m, 0), &c);
  const double tol2 = replay_tol * replay_tol;
  int K = m;
  double tail = 0.0;
  while (K > 1 && tail + c[K - 1] * c[K - 1] < tol2) { tail += c[K - 1] * c[K - 1]; K--; }
  coef->assign(stride, 0.0);
  for (int k = 0; k < K; k++) (*coef)[k + 1] = c[k];
  return K;
}

}  // namespace

// ================================================================ fixed batch API
int batch_size(const Batch *b) {
  int n = 0;
  if (b)
    for (const Slot &sl : b->slots) n += sl.used ? 1 : 0;
  return n;
}

const BatchTuning &batch_tuning(const Batch *b) { return b->tune; }

int batch_create(const std::vector<Sector *> &sectors, Precision prec, Batch **out) {
  *out = nullptr;
  if (sectors.empty()) {
    set_error("batch: no instances");
    return -1;
  }
  for (Sector *s : sectors)
    if (!s || s->device != sectors[0]->device) {
      set_error("batch: every instance must be open on the same device");
      return -1;
    }
  Batch *b = nullptr;
  BRET(engine_create(sectors[0]->device, prec, &b));
  for (Sector *s : sectors) {
    int idx;
    if (engine_add(b, s, false, 0, 16, &idx)) {
      batch_free(b);
      return -1;
    }
  }
  if (upload(b)) {
    batch_free(b);
    return -1;
  }
  *out = b;
  return 0;
}

void batch_free(Batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  release_graph(b);
  for (Slot &sl : b->slots)
    if (sl.used) free_slot(sl);
  cudaFree(b->d_inst);
  cudaFree(b->d_tiles);
  cudaFree(b->d_part);
  cudaFree(b->d_counter);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int batch_autotune(Batch *b, bool force) {
  BRET(cuda_ok(cudaSetDevice(b->device), "set device"));
  const std::string key = signature(b);
  if (!force) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      b->tune = it->second;
      b->tuned = true;
      b->plan_dirty = true;
      return upload(b);
    }
  }
  // trial launches run every member with its current scalars; they only overwrite the
  // storage vectors, which the next start-vector setup rewrites
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  BatchTuning best;
  best.hv_ms = 1e30f;
  // candidate launch shapes, the usual winners first: the search stops once it has spent
  // kTuneBudgetS seconds (after at least three shapes), so a single very large instance is
  // not timed 36 x 4 times while a batch of small instances still tries every shape
  constexpr double kTuneBudgetS = 2.0;
  std::vector<std::array<int, 3>> cand;  // threads, rows per thread, CTAs per SM
  for (int rp : {1, 2})
    for (int th : {256, 128, 512})
      for (int cs : {8, 16, 4, 2})
        if (th * cs <= 2048) cand.push_back({th, rp, cs});
  for (int rp : {4, 8})
    for (int th : {256, 128, 512})
      for (int cs : {8, 16, 4, 2})
        if (th * cs <= 2048) cand.push_back({th, rp, cs});
  const BatchTuning saved = b->tune;
  int rc = 0;
  const auto t_start = std::chrono::steady_clock::now();
  int tried = 0;
  for (const auto &cnd : cand) {
    const double spent = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    if (rc || (tried >= 3 && spent > kTuneBudgetS)) break;
    tried++;
    BatchTuning t;
    t.threads = cnd[0];
    t.rows_per_thread = cnd[1];
    t.ctas_per_sm = cnd[2];
    b->tune = t;
    b->plan_dirty = true;
    if ((rc = upload(b))) break;
    auto trial = [&]() {
      if (b->prec == kFP32) launch_hv<float>(b, t, 0, kTuneKind);
      else launch_hv<double>(b, t, 0, kTuneKind);
    };
    trial();
    cudaEventRecord(e0, b->stream);
    for (int r = 0; r < 3; r++) trial();
    cudaEventRecord(e1, b->stream);
    if ((rc = cuda_ok(cudaEventSynchronize(e1), "tune sync"))) break;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= 3.0f;
    if (ms < best.hv_ms) {
      best = t;
      best.hv_ms = ms;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    b->tune = saved;
    return -1;
  }
  b->tune = best;
  b->tuned = true;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = best;
  }
  b->plan_dirty = true;
  return upload(b);
}

int batch_lanczos(Batch *b, int steps, uint64_t seed, bool use_graph, bool refine, double replay_tol,
                  BatchResult *res) {
  if (steps < 1) {
    set_error("batch: steps must be >= 1");
    return -1;
  }
  BRET(cuda_ok(cudaSetDevice(b->device), "set device"));
  if (!b->tuned) BRET(batch_autotune(b, false));
  std::vector<int> members;
  for (size_t i = 0; i < b->slots.size(); i++)
    if (b->slots[i].used) members.push_back((int)i);
  const int n = (int)members.size();
  for (int j = 0; j < n; j++) {
    Slot &sl = b->slots[members[j]];
    BRET(alloc_scalars(sl, steps));
    BRET(cuda_ok(cudaMemsetAsync(sl.scal, 0, sizeof(double) * (kStSlots + 3 * ((size_t)sl.cap + 2) + 1), b->stream),
                 "clear scalars"));
    if (refine) BRET(alloc_fp64(sl));
    sl.inst.seed = seed + 1000003ull * (uint64_t)j;
    sl.inst.mode = kInit;
    sl.inst.kmax = steps;
  }
  cudaEvent_t ev[5];
  for (auto &e : ev) cudaEventCreate(&e);
  struct EvGuard {
    cudaEvent_t *e;
    ~EvGuard() { for (int k = 0; k < 5; k++) cudaEventDestroy(e[k]); }
  } guard{ev};

  // forward recurrence
  BRET(upload(b));
  cudaEventRecord(ev[0], b->stream);
  BRET(engine_setup(b));
  for (int i : members) b->slots[i].inst.mode = kForward;
  BRET(upload(b));
  BRET(engine_steps(b, steps, use_graph));
  cudaEventRecord(ev[1], b->stream);
  std::vector<std::vector<double>> scal(n);
  for (int j = 0; j < n; j++) {
    const Slot &sl = b->slots[members[j]];
    BRET(read_slot(b, members[j], kStSlots + 3 * ((size_t)sl.cap + 2), &scal[j]));
  }
  BRET(cuda_ok(cudaStreamSynchronize(b->stream), "forward sync"));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ev[0], ev[1]);
  res->forward_ms = ms;
  res->e_lanczos.assign(n, 0.0);
  res->steps.assign(n, 0);
  res->e_refined.assign(n, 0.0);
  res->residual.assign(n, 0.0);
  res->replay_steps.assign(n, 0);
  res->tuning = b->tune;
  int kmax_all = 0;
  for (int j = 0; j < n; j++) {
    Slot &sl = b->slots[members[j]];
    tridiag_of(scal[j], sl.cap, steps, sl.inst.dim, &res->steps[j], &res->e_lanczos[j]);
    sl.inst.mode = kIdle;
    if (refine) {
      std::vector<double> coef;
      const int K = replay_plan(scal[j], sl.cap, res->steps[j], replay_tol, &coef);
      BRET(cuda_ok(cudaMemcpyAsync(sl.inst.coef, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice,
                                   b->stream), "upload coefficients"));
      sl.inst.mode = kReplayInit;
      sl.inst.kmax = K;
      res->replay_steps[j] = K;
      kmax_all = std::max(kmax_all, K);
    }
  }
  if (!refine) return upload(b);
  BRET(upload(b));
  cudaEventRecord(ev[2], b->stream);
  BRET(engine_setup(b));
  for (int i : members) b->slots[i].inst.mode = kReplay;
  BRET(upload(b));
  BRET(engine_steps(b, kmax_all, use_graph));
  cudaEventRecord(ev[3], b->stream);
  for (int i : members) b->slots[i].inst.mode = kRefine;
  BRET(upload(b));
  BRET(engine_refine(b));
  cudaEventRecord(ev[4], b->stream);
  for (int j = 0; j < n; j++) BRET(read_slot(b, members[j], kStSlots, &scal[j]));
  BRET(cuda_ok(cudaStreamSynchronize(b->stream), "refine sync"));
  cudaEventElapsedTime(&ms, ev[2], ev[3]);
  res->replay_ms = ms;
  cudaEventElapsedTime(&ms, ev[3], ev[4]);
  res->refine_ms = ms;
  for (int j = 0; j < n; j++) {
    res->e_refined[j] = scal[j][11];
    res->residual[j] = std::sqrt(scal[j][12] / scal[j][10]);
    b->slots[members[j]].inst.mode = kIdle;
  }
  return upload(b);
}

// ================================================================ request server
namespace {

struct Request {
  int64_t id = -1;
  Model model;
  uint64_t seed = 0;
  int64_t dim = 0;
  int64_t footprint = 0;
  double t_arrival = 0.0, t_admit = 0.0;
  int slot = -1;
  double e_lanczos = 0.0;
  int steps = 0;
  double e_prev = 0.0;
  bool have_prev = false;
  int status = 0;
};

}  // namespace

struct Server {
  Batch *eng = nullptr;
  Precision prec = kFP64;
  int device = 0;
  int64_t budget = 0, used = 0;
  int max_active = 0, K = 16;
  double replay_tol = 1e-9;
  int64_t next_id = 1;
  std::deque<Request> queue;
  std::vector<Request> active;
  std::deque<ServeResult> finished;
};

double server_clock() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

namespace {

// Device bytes a request holds while active: lists, diagonal, tables, vectors, scalars.
int64_t footprint_of(const Model &m, int64_t dim, Precision prec) {
  const bool cplx = m.complex_terms || m.initial_vec_type != 1;
  const int64_t lists = m.rows_are_configs() ? 0 : 8 * dim + 4 * ((1ll << ((m.nbits + 1) / 2)) + (1ll << (m.nbits / 2)));
  const int64_t vecs = 3 * (int64_t)storage_elem(prec, cplx) * dim + (prec == kFP32 ? 2 * (cplx ? 16 : 8) * dim : 0);
  return lists + 8 * dim + vecs + (int64_t)sizeof(BitTerm) * (int64_t)m.offdiag.size() + (1 << 20);
}

void finish(Server *sv, Request &r, int status, double energy, double residual, const std::string &err) {
  ServeResult out;
  out.id = r.id;
  out.status = status;
  out.energy = energy;
  out.e_lanczos = r.e_lanczos;
  out.residual = residual;
  out.steps = r.steps;
  out.dim = r.dim;
  out.t_wait = r.t_admit - r.t_arrival;
  out.t_latency = server_clock() - r.t_arrival;
  out.error = err;
  sv->finished.push_back(out);
  if (r.slot >= 0) {
    engine_remove(sv->eng, r.slot);
    sv->used -= r.footprint;
    r.slot = -1;
  }
}

}  // namespace

int server_create(int device, Precision prec, int64_t hbm_budget, int max_active, int steps_per_iteration,
                  Server **out) {
  *out = nullptr;
  if (max_active < 1 || steps_per_iteration < 2 || (steps_per_iteration & 1)) {
    set_error("server: max_active >= 1 and an even steps_per_iteration >= 2 are required");
    return -1;
  }
  Server *sv = new Server();
  sv->prec = prec;
  sv->device = device;
  sv->max_active = max_active;
  sv->K = steps_per_iteration;
  if (engine_create(device, prec, &sv->eng)) {
    delete sv;
    return -1;
  }
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  sv->budget = hbm_budget > 0 ? hbm_budget : (int64_t)(0.8 * (double)free_b);
  sv->eng->tuned = true;  // fixed launch shape: results do not depend on the other members
  *out = sv;
  return 0;
}

int server_submit(Server *sv, const std::string &namelist, uint64_t seed, double arrival, int64_t *id) {
  Request r;
  std::string err;
  if (read_expert(namelist, &r.model, &err) != 0) {
    set_error("server: " + err);
    return -1;
  }
  if (r.model.calc_type != kLanczos) {
    set_error("server: only CalcType 0 (Lanczos) requests are served");
    return -1;
  }
  r.id = sv->next_id++;
  r.seed = seed;
  r.dim = sector_dim(r.model);
  r.footprint = footprint_of(r.model, r.dim, sv->prec);
  r.t_arrival = arrival >= 0.0 ? arrival : server_clock();
  if (id) *id = r.id;
  sv->queue.push_back(std::move(r));
  return 0;
}

int server_step(Server *sv, int64_t counts[3]) {
  Batch *b = sv->eng;
  BRET(cuda_ok(cudaSetDevice(sv->device), "set device"));
  // ---- admission: slots and HBM budget, first come first served
  while (!sv->queue.empty() && (int)sv->active.size() < sv->max_active) {
    Request &r = sv->queue.front();
    if (sv->used + r.footprint > sv->budget) {
      if (!sv->active.empty()) break;
      Request x = std::move(r);
      sv->queue.pop_front();
      x.t_admit = server_clock();
      finish(sv, x, -1, 0.0, 0.0, "request needs more device memory than the server budget");
      continue;
    }
    Request x = std::move(r);
    sv->queue.pop_front();
    x.t_admit = server_clock();
    Sector *s = nullptr;
    std::string err;
    if (sector_build(x.model, sv->device, &s, &err, false) != 0) {
      sector_free(s);
      finish(sv, x, -1, 0.0, 0.0, err);
      continue;
    }
    const int cap = std::max(2, std::min<int>(x.model.lanczos_max, (int)std::min<int64_t>(x.dim, 1 << 20)));
    if (engine_add(b, s, true, x.seed, cap, &x.slot) != 0) {
      sector_free(s);
      finish(sv, x, -1, 0.0, 0.0, get_error());
      continue;
    }
    sv->used += x.footprint;
    if (sv->prec == kFP32 && alloc_fp64(b->slots[x.slot]) != 0) {
      finish(sv, x, -1, 0.0, 0.0, get_error());
      continue;
    }
    b->slots[x.slot].inst.mode = kInit;
    b->slots[x.slot].inst.kmax = cap;
    b->slots[x.slot].host_k = 0;
    sv->active.push_back(std::move(x));
  }
  if (!sv->active.empty()) {
    // ---- start vectors of new members, replay starts
    bool setup = false;
    for (Request &r : sv->active) {
      const int m = b->slots[r.slot].inst.mode;
      setup = setup || m == kInit || m == kReplayInit;
    }
    BRET(upload(b));
    if (setup) {
      BRET(engine_setup(b));
      for (Request &r : sv->active) {
        BInst &I = b->slots[r.slot].inst;
        if (I.mode == kInit) I.mode = kForward;
        else if (I.mode == kReplayInit) I.mode = kReplay;
      }
      BRET(upload(b));
    }
    // ---- one iteration of K steps for every forward / replay member
    BRET(engine_steps(b, sv->K, false));
    bool refine = false;
    for (Request &r : sv->active) {
      Slot &sl = b->slots[r.slot];
      if (sl.inst.mode == kForward || sl.inst.mode == kReplay) sl.host_k = std::min(sl.host_k + sv->K, sl.inst.kmax);
      if (sl.inst.mode == kReplay && sl.host_k >= sl.inst.kmax) {
        sl.inst.mode = kRefine;
        refine = true;
      }
    }
    if (refine) {
      BRET(upload(b));
      BRET(engine_refine(b));
    }
    std::vector<std::vector<double>> scal(sv->active.size());
    for (size_t j = 0; j < sv->active.size(); j++) {
      const Slot &sl = b->slots[sv->active[j].slot];
      const size_t ndbl = (sl.inst.mode == kForward) ? kStSlots + 3 * ((size_t)sl.cap + 2) : kStSlots;
      BRET(read_slot(b, sv->active[j].slot, ndbl, &scal[j]));
    }
    BRET(cuda_ok(cudaStreamSynchronize(b->stream), "iteration sync"));
    // ---- convergence (HPhi's test at iteration boundaries), replay plans, results
    std::vector<Request> keep;
    for (size_t j = 0; j < sv->active.size(); j++) {
      Request &r = sv->active[j];
      Slot &sl = b->slots[r.slot];
      if (sl.inst.mode == kForward) {
        const Model &m = r.model;
        const int k = sl.host_k;
        int mstep;
        double e0;
        tridiag_of(scal[j], sl.cap, k, sl.inst.dim, &mstep, &e0);
        const size_t stride = (size_t)sl.cap + 2;
        const double *al = scal[j].data() + kStSlots + 1;
        const double *be = scal[j].data() + kStSlots + stride + 1;
        const int tgt = std::max(0, std::min(m.lanczos_target, mstep - 1));
        const double et = tridiag_eigenvalue(al, be, mstep, tgt);
        const double eps = std::pow(10.0, -m.lanczos_eps);
        const bool breakdown = mstep < std::min<int64_t>(k, sl.inst.dim) || mstep >= sl.inst.dim;
        const bool conv = r.have_prev && std::fabs((et - r.e_prev) / et) < eps;
        r.e_prev = et;
        r.have_prev = true;
        const bool at_max = k >= sl.inst.kmax;
        if (conv || breakdown || at_max) {
          r.steps = mstep;
          r.e_lanczos = e0;
          r.status = (conv || breakdown) ? 0 : 1;
          if (sv->prec == kFP32) {
            std::vector<double> coef;
            const int Kr = replay_plan(scal[j], sl.cap, mstep, sv->replay_tol, &coef);
            BRET(cuda_ok(cudaMemcpyAsync(sl.inst.coef, coef.data(), sizeof(double) * coef.size(),
                                         cudaMemcpyHostToDevice, b->stream), "upload coefficients"));
            sl.inst.mode = kReplayInit;
            sl.inst.kmax = Kr;
            sl.host_k = 0;
          } else {
            finish(sv, r, r.status, e0, 0.0, "");
            continue;
          }
        }
      } else if (sl.inst.mode == kRefine) {
        const double *s = scal[j].data();
        finish(sv, r, r.status, s[11], std::sqrt(s[12] / s[10]), "");
        continue;
      }
      keep.push_back(std::move(r));
    }
    sv->active.swap(keep);
  }
  if (counts) {
    counts[0] = (int64_t)sv->active.size();
    counts[1] = (int64_t)sv->queue.size();
    counts[2] = (int64_t)sv->finished.size();
  }
  return 0;
}

bool server_poll(Server *sv, ServeResult *out) {
  if (sv->finished.empty()) return false;
  *out = sv->finished.front();
  sv->finished.pop_front();
  return true;
}

void server_free(Server *sv) {
  if (!sv) return;
  batch_free(sv->eng);
  delete sv;
}

}  // namespace hphi

// ---------------------------------------------------------------- C-ABI
using namespace hphi;

namespace hphi {
Sector *handle_sector(hphi_handle *h);
}

struct hphi_batch {
  Batch *b = nullptr;
};
struct hphi_server {
  Server *s = nullptr;
};

extern "C" {

int hphi_batch_create(hphi_handle *const *handles, int n, int precision, hphi_batch **out) {
  if (!handles || !out || n < 1) {
    set_error("hphi_batch_create: null argument or empty batch");
    return -1;
  }
  *out = nullptr;
  if (precision != HPHI_FP64 && precision != HPHI_FP32) {
    set_error("hphi_batch_create: precision must be HPHI_FP64 or HPHI_FP32");
    return -1;
  }
  cudaGetLastError();
  std::vector<Sector *> secs;
  for (int i = 0; i < n; i++) {
    Sector *s = handle_sector(handles[i]);
    if (!s) {
      set_error("hphi_batch_create: invalid handle at position " + std::to_string(i));
      return -1;
    }
    secs.push_back(s);
  }
  Batch *b = nullptr;
  if (batch_create(secs, (Precision)precision, &b) != 0) return -1;
  *out = new hphi_batch();
  (*out)->b = b;
  return 0;
}

int hphi_batch_lanczos(hphi_batch *hb, int steps, uint64_t seed, int flags, double replay_tol, double *result,
                       double *timing) {
  if (!hb || !hb->b) {
    set_error("invalid batch");
    return -1;
  }
  cudaGetLastError();
  BatchResult r;
  if (batch_lanczos(hb->b, steps, seed, (flags & HPHI_BATCH_GRAPH) != 0, (flags & HPHI_BATCH_REFINE) != 0,
                    replay_tol > 0.0 ? replay_tol : 1e-9, &r) != 0)
    return -1;
  const int n = (int)r.e_lanczos.size();
  if (result)
    for (int i = 0; i < n; i++) {
      double *o = result + (size_t)HPHI_BATCH_RESULT_FIELDS * i;
      o[0] = r.e_lanczos[i];
      o[1] = r.e_refined[i];
      o[2] = r.residual[i];
      o[3] = r.steps[i];
      o[4] = r.replay_steps[i];
    }
  if (timing) {
    timing[0] = r.forward_ms;
    timing[1] = r.replay_ms;
    timing[2] = r.refine_ms;
    timing[3] = r.tuning.hv_ms;
  }
  return 0;
}

int hphi_batch_tuning(hphi_batch *hb, int retune, int *shape) {
  if (!hb || !hb->b) {
    set_error("invalid batch");
    return -1;
  }
  cudaGetLastError();
  if (retune || !hb->b->tuned)
    if (batch_autotune(hb->b, retune != 0) != 0) return -1;
  if (shape) {
    shape[0] = hb->b->tune.threads;
    shape[1] = hb->b->tune.rows_per_thread;
    shape[2] = hb->b->tune.ctas_per_sm;
  }
  return 0;
}

void hphi_batch_free(hphi_batch *hb) {
  if (!hb) return;
  batch_free(hb->b);
  delete hb;
}

int hphi_server_create(int device, int precision, int64_t hbm_budget, int max_active, int steps_per_iteration,
                       hphi_server **out) {
  if (!out) {
    set_error("hphi_server_create: null argument");
    return -1;
  }
  *out = nullptr;
  if (precision != HPHI_FP64 && precision != HPHI_FP32) {
    set_error("hphi_server_create: precision must be HPHI_FP64 or HPHI_FP32");
    return -1;
  }
  int ndev = 0;
  cudaGetLastError();
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    set_error("hphi_server_create: no such CUDA device");
    return -1;
  }
  Server *s = nullptr;
  if (server_create(device, (Precision)precision, hbm_budget, max_active, steps_per_iteration, &s) != 0) return -1;
  *out = new hphi_server();
  (*out)->s = s;
  return 0;
}

int hphi_server_submit(hphi_server *hs, const char *namelist_def, uint64_t seed, double arrival, int64_t *request_id) {
  if (!hs || !hs->s || !namelist_def) {
    set_error("hphi_server_submit: invalid server or null input");
    return -1;
  }
  return server_submit(hs->s, namelist_def, seed, arrival, request_id);
}

int hphi_server_step(hphi_server *hs, int64_t *counts) {
  if (!hs || !hs->s) {
    set_error("invalid server");
    return -1;
  }
  cudaGetLastError();
  int64_t c[3];
  if (server_step(hs->s, c) != 0) return -1;
  if (counts)
    for (int i = 0; i < 3; i++) counts[i] = c[i];
  return 0;
}

int hphi_server_poll(hphi_server *hs, int64_t *request_id, double *result) {
  if (!hs || !hs->s) {
    set_error("invalid server");
    return -1;
  }
  ServeResult r;
  if (!server_poll(hs->s, &r)) return 0;
  if (request_id) *request_id = r.id;
  if (result) {
    result[0] = r.status;
    result[1] = r.energy;
    result[2] = r.e_lanczos;
    result[3] = r.residual;
    result[4] = r.steps;
    result[5] = (double)r.dim;
    result[6] = r.t_wait;
    result[7] = r.t_latency;
  }
  if (r.status < 0) set_error(r.error);
  return 1;
}

double hphi_server_clock(void) { return server_clock(); }

void hphi_server_free(hphi_server *hs) {
  if (!hs) return;
  server_free(hs->s);
  delete hs;
}

}  // extern "C"
