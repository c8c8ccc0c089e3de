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
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "device_util.cuh"
#include "engine.hpp"
#include "hv_product.hpp"

namespace hphi {
namespace {

constexpr int kProdThreads = 512;
constexpr int kMaxUpWidth = 128;          // up hops of one row, staged in shared memory
constexpr uint32_t kEllNone = 0xFFFFFFFFu;

struct ProdArgs {
  int N, Uc, Dc;               // sites, rows (up configurations), columns (down configurations)
  int wd, wu;                  // ELL widths
  const uint16_t *rank;        // [2^N]
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
                                    const uint16_t *__restrict__ rank, const T *__restrict__ in, T *__restrict__ out) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = list_1[r];
    const int64_t pos = (int64_t)rank[compress_species(c, 0, N)] * Dc + rank[compress_species(c, 1, N)];
    const double sg = (SIGN && species_parity(c, N)) ? -1.0 : 1.0;
    if (TO_NATIVE) out[pos] = VT<T>::scale(sg, in[r]);
    else out[r] = VT<T>::scale(sg, in[pos]);
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
  double *part = nullptr;   // 2 * Uc row partial sums
  int *counter = nullptr;
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

}  // namespace

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
  if (upload(p, rank, &a.rank, err) || upload(p, unrank_up, &a.unrank_up, err) ||
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
    prod_permute_kernel<double, true, false><<<nb, 256, 0, s->stream>>>(s->dim, N, Dc, s->d_list_1, a.rank,
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
  if (cudaFuncSetAttribute(prod_hv_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_r) !=
          cudaSuccess ||
      cudaFuncSetAttribute(prod_hv_kernel<cplx>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_c) !=
          cudaSuccess) {
    *err = "product plan: shared-memory attribute rejected";
    return fail();
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, prod_hv_kernel<double>, kProdThreads, smem_r);
  p->grid = std::max(1, std::min(Uc, std::max(1, per_sm) * s->num_sms));
  s->prod = p;
  return 0;
}

size_t prod_scratch_doubles(const Sector *s) { return 2 * (size_t)s->prod->args.Uc; }

int prod_hv_launch_scratch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                           double *d_part, int *d_counter) {
  ProdPlan *p = s->prod;
  if (vt == kReal64 && s->model.complex_terms) {
    set_error("H has complex coefficients: real vectors are not allowed");
    return -1;
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
  if (vt == kReal64) {
    if (to_native)
      prod_permute_kernel<double, true, true><<<nb, 256, 0, s->stream>>>(s->dim, N, Dc, s->d_list_1, p->args.rank,
                                                                         (const double *)in, (double *)out);
    else
      prod_permute_kernel<double, false, true><<<nb, 256, 0, s->stream>>>(s->dim, N, Dc, s->d_list_1, p->args.rank,
                                                                          (const double *)in, (double *)out);
  } else {
    if (to_native)
      prod_permute_kernel<cplx, true, true><<<nb, 256, 0, s->stream>>>(s->dim, N, Dc, s->d_list_1, p->args.rank,
                                                                       (const cplx *)in, (cplx *)out);
    else
      prod_permute_kernel<cplx, false, true><<<nb, 256, 0, s->stream>>>(s->dim, N, Dc, s->d_list_1, p->args.rank,
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
