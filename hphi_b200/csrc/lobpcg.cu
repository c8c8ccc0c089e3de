// Block LOBPCG driver (CalcType 3) over the device sector.
//
// Follows LOBPCG_Main / CalcByLOBPCG (src/CalcByLOBPCG.c:328-632, 636-776): k = exct
// vectors x with H x, search directions w (residuals) and p; each step
//   w_i = H x_i - e_i x_i,  |w|max < eps  -> converged, eps = 10^(-LanczosEps/2) * max(1, |e|max)
//   (steps > 1) optional point-Jacobi preconditioning with the adaptive shift
//   (calc_preshift, :129-148), then w_i /= |w_i|
//   W = H w; subspace matrices Hsub = B^+ (H B), O = B^+ B over B = (w, x, p)
//   Lowdin-orthogonalised generalized eigenproblem (diag_ovrp, :43-123): overlap
//   eigenvalues <= 1e-10 drop their directions
//   e_i = (<x_i|H x_i> + mu_i) / 2; x, H x, p, H p from the lowest k subspace vectors;
//   x and p normalised.
// Vectors live on the device in the engine's native order; the block dot products and
// block linear combinations are single passes over all vectors involved.  The small
// subspace problem is solved on the host with a Jacobi method for Hermitian matrices.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "device_util.cuh"
#include "driver.hpp"
#include "engine.hpp"

namespace hphi {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxPairs = 8;   // dot products per pass
constexpr int kMaxIn = 12;     // inputs of one linear combination (3 * exct)
constexpr int kMaxOut = 4;     // outputs of one linear combination

using zc = std::complex<double>;

struct DotPairs {
  const void *a[kMaxPairs];
  const void *b[kMaxPairs];
  int n;
};

// part[blk][2i..2i+1] = sum over the block's rows of conj(a_i) b_i
template <typename T>
__global__ void multi_dot_kernel(int64_t dim, DotPairs P, double *__restrict__ part) {
  double acc[2 * kMaxPairs];
#pragma unroll
  for (int i = 0; i < 2 * kMaxPairs; i++) acc[i] = 0.0;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int i = 0; i < kMaxPairs; i++) {
      if (i < P.n) {
        const T x = ((const T *)P.a[i])[r];
        const T y = ((const T *)P.b[i])[r];
        acc[2 * i] += VT<T>::conj_mul_re(x, y);
        acc[2 * i + 1] += VT<T>::conj_mul_im(x, y);
      }
    }
  }
  block_sum<2 * kMaxPairs>(acc);
  if (threadIdx.x == 0)
    for (int i = 0; i < 2 * kMaxPairs; i++) part[(size_t)blockIdx.x * 2 * kMaxPairs + i] = acc[i];
}

struct LinComb {
  const void *in[kMaxIn];
  void *out[kMaxOut];
  int nin, nout;
  int accumulate;  // add to the outputs (a later chunk of inputs)
};

// out_o[r] (+)= sum_j coef[j][o] in_j[r] (coef complex, row-major nin x nout; real vectors
// use the real parts).  Outputs never alias inputs.  Larger combinations run as chunks of at
// most kMaxIn inputs and kMaxOut outputs.
template <typename T>
__global__ void lincomb_kernel(int64_t dim, LinComb L, const double *__restrict__ coef) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
    T v[kMaxIn];
#pragma unroll
    for (int j = 0; j < kMaxIn; j++)
      if (j < L.nin) v[j] = ((const T *)L.in[j])[r];
#pragma unroll
    for (int o = 0; o < kMaxOut; o++) {
      if (o < L.nout) {
        T y = L.accumulate ? ((const T *)L.out[o])[r] : VT<T>::zero();
#pragma unroll
        for (int j = 0; j < kMaxIn; j++)
          if (j < L.nin) {
            const double *c = coef + 2 * (j * L.nout + o);
            y = VT<T>::add(y, VT<T>::cmul_re_im(c[0], c[1], v[j]));
          }
        ((T *)L.out[o])[r] = y;
      }
    }
  }
}

// Point-Jacobi preconditioner of src/CalcByLOBPCG.c:420-429: w /= (diag - shift) where
// |diag - shift| > eps.
template <typename T>
__global__ void precondition_kernel(int64_t dim, const double *__restrict__ diag, double shift, double eps,
                                    T *__restrict__ w) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x) {
    const double p = diag[r] - shift;
    if (fabs(p) > eps) w[r] = VT<T>::scale(1.0 / p, w[r]);
  }
}

__global__ void fill_kernel(int64_t dim, double v, double *__restrict__ x) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x)
    x[r] = v;
}

__global__ void mul_kernel(int64_t dim, const double *__restrict__ a, double *__restrict__ x) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim; r += (int64_t)gridDim.x * blockDim.x)
    x[r] *= a[r];
}

int cuda_ok(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    set_error(std::string("lobpcg: ") + what + ": " + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}
#define LRET(x) do { if ((x) != 0) return -1; } while (0)

struct DevMem {
  void *p = nullptr;
  ~DevMem() { if (p) cudaFree(p); }
};

// ---------------------------------------------------------------- host linear algebra
// Eigen-decomposition of the Hermitian n x n matrix A (column-major, a[r + c*n]) by cyclic
// Jacobi rotations; eigenvalues ascending in w, eigenvectors in the columns of z.
void hermitian_eigen(int n, std::vector<zc> a, std::vector<double> *w, std::vector<zc> *z) {
  std::vector<zc> v(n * n, 0.0);
  for (int i = 0; i < n; i++) v[i + i * n] = 1.0;
  auto A = [&](int r, int c) -> zc & { return a[r + c * n]; };
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, tot = 0.0;
    for (int c = 0; c < n; c++)
      for (int r = 0; r < n; r++) {
        tot += std::norm(A(r, c));
        if (r != c) off += std::norm(A(r, c));
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        const zc apq = A(p, q);
        const double mag = std::abs(apq);
        if (mag == 0.0) continue;
        // phase making the (p, q) element real and positive; exact for real input
        const zc ph = (apq.imag() == 0.0) ? zc(apq.real() > 0 ? 1.0 : -1.0, 0.0) : apq / mag;
        const double app = A(p, p).real(), aqq = A(q, q).real();
        const double tau = (aqq - app) / (2.0 * mag);
        const double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
        // V = diag(1, conj(ph)) * [[c, s], [-s, c]] on (p, q)
        const zc vpp = c, vpq = s, vqp = -s * std::conj(ph), vqq = c * std::conj(ph);
        for (int k = 0; k < n; k++) {  // columns: A <- A V
          const zc akp = A(k, p), akq = A(k, q);
          A(k, p) = akp * vpp + akq * vqp;
          A(k, q) = akp * vpq + akq * vqq;
        }
        for (int k = 0; k < n; k++) {  // rows: A <- V^+ A
          const zc apk = A(p, k), aqk = A(q, k);
          A(p, k) = std::conj(vpp) * apk + std::conj(vqp) * aqk;
          A(q, k) = std::conj(vpq) * apk + std::conj(vqq) * aqk;
        }
        A(p, q) = 0.0;
        A(q, p) = 0.0;
        for (int k = 0; k < n; k++) {
          const zc zkp = v[k + p * n], zkq = v[k + q * n];
          v[k + p * n] = zkp * vpp + zkq * vqp;
          v[k + q * n] = zkp * vpq + zkq * vqq;
        }
      }
  }
  std::vector<int> idx(n);
  for (int i = 0; i < n; i++) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return A(x, x).real() < A(y, y).real(); });
  w->assign(n, 0.0);
  z->assign(n * n, 0.0);
  for (int j = 0; j < n; j++) {
    (*w)[j] = A(idx[j], idx[j]).real();
    for (int r = 0; r < n; r++) (*z)[r + j * n] = v[r + idx[j] * n];
  }
}

// Generalized problem H v = mu O v with Lowdin's orthogonalisation (diag_ovrp,
// src/CalcByLOBPCG.c:43-123): returns the kept dimension n2; vec (n x n2, column-major)
// and mu (n2) ascending.
int lowdin_eigen(int n, const std::vector<zc> &h, const std::vector<zc> &o, std::vector<zc> *vec,
                 std::vector<double> *mu) {
  std::vector<double> oe;
  std::vector<zc> ov;
  hermitian_eigen(n, o, &oe, &ov);
  std::vector<zc> S;  // n x n2
  int n2 = 0;
  for (int i = 0; i < n; i++)
    if (oe[i] > 1.0e-10) {
      const double f = 1.0 / std::sqrt(oe[i]);
      for (int r = 0; r < n; r++) S.push_back(ov[r + i * n] * f);
      n2++;
    }
  // H' = S^+ H S (n2 x n2)
  std::vector<zc> HS(n * n2, 0.0), Hp(n2 * n2, 0.0);
  for (int c = 0; c < n2; c++)
    for (int r = 0; r < n; r++) {
      zc acc = 0.0;
      for (int k = 0; k < n; k++) acc += h[r + k * n] * S[k + c * n];
      HS[r + c * n] = acc;
    }
  for (int c = 0; c < n2; c++)
    for (int r = 0; r < n2; r++) {
      zc acc = 0.0;
      for (int k = 0; k < n; k++) acc += std::conj(S[k + r * n]) * HS[k + c * n];
      Hp[r + c * n2] = acc;
    }
  std::vector<zc> phi;
  hermitian_eigen(n2, Hp, mu, &phi);
  vec->assign(n * n2, 0.0);
  for (int c = 0; c < n2; c++)
    for (int r = 0; r < n; r++) {
      zc acc = 0.0;
      for (int k = 0; k < n2; k++) acc += S[r + k * n] * phi[k + c * n2];
      (*vec)[r + c * n] = acc;
    }
  return n2;
}

// Adaptive shift of the preconditioner (calc_preshift, src/CalcByLOBPCG.c:129-148).
double preshift_of(double eig, double res, double eps) {
  if (res >= 1.0) return 0.0;
  const double k = std::trunc(std::log10(std::fabs(eig)));
  const double i = (eps > res) ? std::ceil(std::log10(eps)) : std::ceil(std::log10(res));
  const double p = std::pow(10.0, k + i);
  return std::trunc(eig / p) * p;
}

struct Ops {
  Sector *s;
  VecType vt;
  double *part;      // 2 * kMaxPairs * red_blocks
  double *d_out;     // 2 * kMaxPairs
  double *d_coef;    // 2 * kMaxIn * kMaxOut

  // out[i] = sum conj(a[i]) b[i] for any number of pairs
  int dots(const std::vector<const void *> &a, const std::vector<const void *> &b, std::vector<zc> *out) {
    out->assign(a.size(), 0.0);
    for (size_t base = 0; base < a.size(); base += kMaxPairs) {
      DotPairs P{};
      P.n = (int)std::min<size_t>(kMaxPairs, a.size() - base);
      for (int i = 0; i < P.n; i++) {
        P.a[i] = a[base + i];
        P.b[i] = b[base + i];
      }
      if (vt == kReal64) multi_dot_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, P, part);
      else multi_dot_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, P, part);
      finalize_partials_kernel<2 * kMaxPairs><<<1, 256, 0, s->stream>>>(part, s->red_blocks, d_out);
      double h[2 * kMaxPairs];
      LRET(cuda_ok(cudaMemcpyAsync(h, d_out, sizeof(h), cudaMemcpyDeviceToHost, s->stream), "read dots"));
      LRET(cuda_ok(cudaStreamSynchronize(s->stream), "dots"));
      for (int i = 0; i < P.n; i++) (*out)[base + i] = zc(h[2 * i], vt == kReal64 ? 0.0 : h[2 * i + 1]);
    }
    return 0;
  }

  // out[o] = sum_j c[j][o] in[j], in chunks of kMaxOut outputs x kMaxIn inputs (later input
  // chunks accumulate into the outputs)
  int lincomb(const std::vector<const void *> &in, const std::vector<void *> &out, const std::vector<zc> &c) {
    const int nin = (int)in.size(), nout = (int)out.size();
    for (int o0 = 0; o0 < nout; o0 += kMaxOut)
      for (int j0 = 0; j0 < nin; j0 += kMaxIn) {
        LinComb L{};
        L.nin = std::min(kMaxIn, nin - j0);
        L.nout = std::min(kMaxOut, nout - o0);
        L.accumulate = j0 > 0;
        std::vector<double> hc(2 * L.nin * L.nout);
        for (int j = 0; j < L.nin; j++)
          for (int o = 0; o < L.nout; o++) {
            const zc cc = c[(j0 + j) * nout + (o0 + o)];
            hc[2 * (j * L.nout + o)] = cc.real();
            hc[2 * (j * L.nout + o) + 1] = cc.imag();
          }
        for (int j = 0; j < L.nin; j++) L.in[j] = in[j0 + j];
        for (int o = 0; o < L.nout; o++) L.out[o] = out[o0 + o];
        LRET(cuda_ok(cudaMemcpyAsync(d_coef, hc.data(), sizeof(double) * hc.size(), cudaMemcpyHostToDevice,
                                     s->stream), "coefficients"));
        if (vt == kReal64) lincomb_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, L, d_coef);
        else lincomb_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(s->dim, L, d_coef);
        LRET(cuda_ok(cudaGetLastError(), "lincomb launch"));
        // the coefficient buffer is reused by the next call: wait for this one
        LRET(cuda_ok(cudaStreamSynchronize(s->stream), "lincomb"));
      }
    return 0;
  }

  // H v into out (out = H v, acc = 0)
  int hv(const void *v, void *out) {
    const double c[2] = {0.0, 1.0};
    LRET(cuda_ok(cudaMemcpyAsync(d_coef, c, sizeof(c), cudaMemcpyHostToDevice, s->stream), "coef"));
    LRET(hv_native(s, vt, v, out, d_coef, d_out));
    return cuda_ok(cudaStreamSynchronize(s->stream), "hv");
  }

  int scale(void *x, double a) { return vec_scale(s, vt, a, x); }
};

int ensure_dir(const std::string &dir) {
  if (dir.empty()) return 0;
  struct stat st;
  if (stat(dir.c_str(), &st) == 0) return 0;
  if (mkdir(dir.c_str(), 0755) != 0) {
    set_error("cannot create output directory " + dir);
    return -1;
  }
  return 0;
}

}  // namespace

// Initial vectors of Initialize_wave (src/CalcByLOBPCG.c:153-293) for the deterministic
// single-element mode: x_ie has one non-zero element at iv + 1 (1-based) with
// iv = (dim/2 + initial_iv + ie) % dim + 1 (no element when iv == dim).
bool lobpcg_single_element_start(const Sector &s, std::vector<double> *v) {
  const Model &m = s.model;
  if (m.is_gc() || m.general_spin || m.initial_iv <= 0) return false;
  const uint64_t dim = (uint64_t)s.dim;
  const int k = std::max(1, m.k_exct);
  v->assign((size_t)k * 2 * (dim + 1), 0.0);
  for (int ie = 0; ie < k; ie++) {
    const uint64_t iv = (dim / 2 + (uint64_t)m.initial_iv + (uint64_t)ie) % dim + 1;
    if (iv >= dim) continue;
    double *x = v->data() + (size_t)ie * 2 * (dim + 1);
    if (m.initial_vec_type == 0) {
      x[2 * (iv + 1)] = 1.0 / std::sqrt(2.0);
      x[2 * (iv + 1) + 1] = 1.0 / std::sqrt(2.0);
    } else {
      x[2 * (iv + 1)] = 1.0;
    }
  }
  return true;
}

int lobpcg_run(Sector *s, VecType vt, const double *h_init, LobpcgResult *res) {
  const Model &m = s->model;
  const int k = std::max(1, m.k_exct);
  const int64_t dim = s->dim;
  if (dim < 3 * k) {
    set_error("lobpcg: sector dimension smaller than the LOBPCG subspace (3 * exct)");
    return -1;
  }
  LRET(cuda_ok(cudaSetDevice(s->device), "set device"));
  const size_t esz = (vt == kReal64) ? sizeof(double) : sizeof(cplx);
  const size_t vbytes = esz * (size_t)dim;
  // blocks: 0 w, 1 x, 2 p (search space), 3..5 H times them, 6..9 updated x, Hx, p, Hp
  DevMem VEC, AUX, DIAG, HOST_TMP;
  LRET(cuda_ok(cudaMalloc(&VEC.p, vbytes * 10 * k), "alloc vectors"));
  LRET(cuda_ok(cudaMemsetAsync(VEC.p, 0, vbytes * 10 * k, s->stream), "clear vectors"));
  auto vec = [&](int blk, int i) -> void * { return (char *)VEC.p + ((size_t)blk * k + i) * vbytes; };
  LRET(cuda_ok(cudaMalloc(&AUX.p, sizeof(double) * (2 * kMaxPairs * (size_t)s->red_blocks + 2 * kMaxPairs +
                                                    2 * kMaxIn * kMaxOut + 8)), "alloc scratch"));
  Ops ops{s, vt, (double *)AUX.p, (double *)AUX.p + 2 * kMaxPairs * s->red_blocks,
          (double *)AUX.p + 2 * kMaxPairs * s->red_blocks + 2 * kMaxPairs};
  // diagonal in the native order for the preconditioner.  The native order may carry a
  // per-configuration sign s(c) = +-1 (fermion reordering); the diagonal is a function of
  // the configuration, so undo it: to_native(diag) * to_native(1) = s^2 diag = diag.
  LRET(cuda_ok(cudaMalloc(&DIAG.p, sizeof(double) * dim), "alloc diagonal"));
  LRET(cuda_ok(cudaMalloc(&HOST_TMP.p, vbytes), "alloc staging"));
  LRET(to_native(s, kReal64, s->d_diag, DIAG.p));
  if (has_native_order(s)) {
    DevMem ONES;
    LRET(cuda_ok(cudaMalloc(&ONES.p, sizeof(double) * dim), "alloc signs"));
    fill_kernel<<<s->red_blocks, kThreads, 0, s->stream>>>(dim, 1.0, (double *)HOST_TMP.p);
    LRET(to_native(s, kReal64, HOST_TMP.p, ONES.p));
    mul_kernel<<<s->red_blocks, kThreads, 0, s->stream>>>(dim, (const double *)ONES.p, (double *)DIAG.p);
    LRET(cuda_ok(cudaGetLastError(), "diagonal signs"));
    LRET(cuda_ok(cudaStreamSynchronize(s->stream), "diagonal signs"));
  }
  // start vectors (HPhi layout, normalised here) -> native order
  for (int i = 0; i < k; i++) {
    LRET(vec_from_host_c128(s, vt, h_init + (size_t)i * 2 * (dim + 1), HOST_TMP.p));
    LRET(to_native(s, vt, HOST_TMP.p, vec(1, i)));
  }
  std::vector<zc> d;
  {
    std::vector<const void *> a, b;
    for (int i = 0; i < k; i++) { a.push_back(vec(1, i)); b.push_back(vec(1, i)); }
    LRET(ops.dots(a, b, &d));
    for (int i = 0; i < k; i++) {
      if (d[i].real() <= 0.0) {
        set_error("lobpcg: zero start vector");
        return -1;
      }
      LRET(ops.scale(vec(1, i), 1.0 / std::sqrt(d[i].real())));
    }
  }
  for (int i = 0; i < k; i++) LRET(ops.hv(vec(1, i), vec(4, i)));
  std::vector<double> eig(k);
  {
    std::vector<const void *> a, b;
    for (int i = 0; i < k; i++) { a.push_back(vec(1, i)); b.push_back(vec(4, i)); }
    LRET(ops.dots(a, b, &d));
    for (int i = 0; i < k; i++) eig[i] = d[i].real();
  }
  const int n = 3 * k;
  const double pos_shift = m.large_value * m.nsite;
  res->lines.clear();
  res->lines.push_back("    Step   Residual-2-norm     Threshold      Energy\n");
  res->converged = false;
  int stp;
  char line[512];
  for (stp = 1; !res->phys_only && stp <= m.lanczos_max; stp++) {
    double eabs = 0.0;
    for (int i = 0; i < k; i++) eabs = std::max(eabs, std::fabs(eig[i]));
    double eps = std::pow(10.0, -0.5 * m.lanczos_eps);
    if (eabs > 1.0) eps *= eabs;
    double dmax = 0.0;
    for (int i = 0; i < k; i++) {
      // w = H x - e x
      LRET(ops.lincomb({vec(4, i), vec(1, i)}, {vec(0, i)}, {zc(1.0), zc(-eig[i])}));
      std::vector<zc> nn;
      LRET(ops.dots({vec(0, i)}, {vec(0, i)}, &nn));
      double dn = std::sqrt(nn[0].real());
      dmax = std::max(dmax, dn);
      if (stp != 1) {
        if (m.pre_cg == 1) {
          const double shift = preshift_of(eig[i] + pos_shift, dn, eps) - pos_shift;
          if (vt == kReal64)
            precondition_kernel<double><<<s->red_blocks, kThreads, 0, s->stream>>>(dim, (const double *)DIAG.p, shift,
                                                                                  eps, (double *)vec(0, i));
          else
            precondition_kernel<cplx><<<s->red_blocks, kThreads, 0, s->stream>>>(dim, (const double *)DIAG.p, shift,
                                                                                eps, (cplx *)vec(0, i));
          LRET(cuda_ok(cudaGetLastError(), "precondition"));
        }
        LRET(ops.dots({vec(0, i)}, {vec(0, i)}, &nn));
        dn = std::sqrt(nn[0].real());
        LRET(ops.scale(vec(0, i), 1.0 / dn));
      }
    }
    int len = snprintf(line, sizeof(line), "%9d %15.5e %15.5e      ", stp, dmax, eps);
    for (int i = 0; i < k && len < (int)sizeof(line) - 20; i++) len += snprintf(line + len, sizeof(line) - len, " %15.5e", eig[i]);
    snprintf(line + len, sizeof(line) - len, "\n");
    res->lines.push_back(line);
    res->residual = dmax;
    if (dmax < eps) {
      res->converged = true;
      break;
    }
    for (int i = 0; i < k; i++) LRET(ops.hv(vec(0, i), vec(3, i)));
    // subspace matrices over B = (w_0..w_k-1, x_0.., p_0..): Hsub(r, c) = <B_r|H B_c>
    std::vector<const void *> ba, bh, bb;
    std::vector<zc> hs(n * n), ov(n * n);
    {
      std::vector<const void *> a1, b1, a2, b2;
      for (int c = 0; c < n; c++)
        for (int r = 0; r < n; r++) {
          const int rb = r / k, ri = r % k, cb = c / k, ci = c % k;
          a1.push_back(vec(rb, ri));
          b1.push_back(vec(3 + cb, ci));
          a2.push_back(vec(rb, ri));
          b2.push_back(vec(cb, ci));
        }
      std::vector<zc> h1, o1;
      LRET(ops.dots(a1, b1, &h1));
      LRET(ops.dots(a2, b2, &o1));
      for (int q = 0; q < n * n; q++) { hs[q] = h1[q]; ov[q] = o1[q]; }
    }
    for (int i = 0; i < k; i++) eig[i] = hs[(k + i) + (k + i) * n].real();
    std::vector<zc> V;
    std::vector<double> mu;
    const int n2 = lowdin_eigen(n, hs, ov, &V, &mu);
    if (n2 < k) {
      set_error("lobpcg: subspace collapsed (overlap rank below exct)");
      return -1;
    }
    for (int i = 0; i < k; i++) eig[i] = 0.5 * (eig[i] + mu[i]);
    // x' = B V[:, i], (Hx)' = HB V[:, i], p' = (w, p) parts, (Hp)' likewise
    std::vector<const void *> inB, inH;
    for (int b = 0; b < 3; b++)
      for (int i = 0; i < k; i++) { inB.push_back(vec(b, i)); inH.push_back(vec(3 + b, i)); }
    std::vector<zc> cx(n * k), cp(n * k);
    for (int j = 0; j < n; j++)
      for (int i = 0; i < k; i++) {
        cx[j * k + i] = V[j + i * n];
        cp[j * k + i] = (j / k == 1) ? zc(0.0) : V[j + i * n];
      }
    std::vector<void *> ox, ohx, op, ohp;
    for (int i = 0; i < k; i++) {
      ox.push_back(vec(6, i)); ohx.push_back(vec(7, i)); op.push_back(vec(8, i)); ohp.push_back(vec(9, i));
    }
    LRET(ops.lincomb(inB, ox, cx));
    LRET(ops.lincomb(inH, ohx, cx));
    LRET(ops.lincomb(inB, op, cp));
    LRET(ops.lincomb(inH, ohp, cp));
    for (int i = 0; i < k; i++) {
      std::vector<zc> nx, np;
      LRET(ops.dots({vec(6, i)}, {vec(6, i)}, &nx));
      LRET(ops.dots({vec(8, i)}, {vec(8, i)}, &np));
      const double fx = 1.0 / std::sqrt(nx[0].real()), fp = 1.0 / std::sqrt(np[0].real());
      LRET(ops.scale(vec(6, i), fx));
      LRET(ops.scale(vec(7, i), fx));
      LRET(ops.scale(vec(8, i), fp));
      LRET(ops.scale(vec(9, i), fp));
      LRET(cuda_ok(cudaMemcpyAsync(vec(1, i), vec(6, i), vbytes, cudaMemcpyDeviceToDevice, s->stream), "copy x"));
      LRET(cuda_ok(cudaMemcpyAsync(vec(4, i), vec(7, i), vbytes, cudaMemcpyDeviceToDevice, s->stream), "copy Hx"));
      LRET(cuda_ok(cudaMemcpyAsync(vec(2, i), vec(8, i), vbytes, cudaMemcpyDeviceToDevice, s->stream), "copy p"));
      LRET(cuda_ok(cudaMemcpyAsync(vec(5, i), vec(9, i), vbytes, cudaMemcpyDeviceToDevice, s->stream), "copy Hp"));
    }
  }
  res->steps = std::min(stp, m.lanczos_max);
  res->itr = stp;
  if (res->phys_only) {
    // CalcByLOBPCG with InputEigenVec (src/CalcByLOBPCG.c:688-722): phys() of the read vectors
    res->steps = res->itr = 0;
    res->converged = true;
    res->lines.clear();
  }
  res->eig = eig;
  // phys() / expec_energy_flct for each x: energy, <Hx|Hx>, doublon, Sz
  res->energy.assign(k, 0.0);
  res->var.assign(k, 0.0);
  res->doublon.assign(k, 0.0);
  res->sz.assign(k, 0.0);
  res->eigenvectors.clear();
  res->green.clear();
  double *obs = ops.d_out;
  for (int i = 0; i < k; i++) {
    LRET(ops.hv(vec(1, i), vec(6, i)));
    std::vector<zc> e, h2;
    LRET(ops.dots({vec(1, i)}, {vec(6, i)}, &e));
    LRET(ops.dots({vec(6, i)}, {vec(6, i)}, &h2));
    LRET(native_observables(s, vt, vec(1, i), obs));
    double o[6];
    LRET(cuda_ok(cudaMemcpyAsync(o, obs, sizeof(o), cudaMemcpyDeviceToHost, s->stream), "read observables"));
    LRET(cuda_ok(cudaStreamSynchronize(s->stream), "observables"));
    res->energy[i] = e[0].real();
    res->var[i] = h2[0].real();
    res->doublon[i] = o[0];
    res->sz[i] = o[4];
    if (!m.green_one.empty() || !m.green_two.empty() || !m.green_three.empty() || !m.green_four.empty() ||
        !m.green_six.empty()) {
      // expec_cisajs / expec_cisajscktaltdc of each vector (phys, src/phys.c:100-110)
      LRET(from_native(s, vt, vec(1, i), HOST_TMP.p));
      res->green.emplace_back();
      LRET(model_green(s, vt, HOST_TMP.p, 1.0, &res->green.back()));
    }
    if (res->copy_vectors) {
      std::vector<double> hv(2 * (dim + 1), 0.0);
      LRET(from_native(s, vt, vec(1, i), HOST_TMP.p));
      LRET(vec_to_host_c128(s, vt, HOST_TMP.p, hv.data()));
      res->eigenvectors.insert(res->eigenvectors.end(), hv.begin(), hv.end());
    }
  }
  if (!res->converged) {
    set_error("LOBPCG is not converged in this process.");
    return -1;
  }
  return 0;
}

int write_lobpcg_outputs(const Sector &s, const LobpcgResult &r, const std::string &outdir) {
  LRET(ensure_dir(outdir));
  const Model &m = s.model;
  const std::string sep = outdir.empty() ? "" : "/";
  const std::string step_file = outdir + sep + m.data_head + "_Lanczos_Step.dat";
  FILE *f = nullptr;
  if (!r.phys_only) {
    f = fopen(step_file.c_str(), "w");
    if (!f) {
      set_error("cannot write " + step_file);
      return -1;
    }
    for (const auto &l : r.lines) fputs(l.c_str(), f);
    fclose(f);
  }
  if (!r.converged) return 0;
  const std::string ef = outdir + sep + m.data_head + "_energy.dat";
  f = fopen(ef.c_str(), "w");
  if (!f) {
    set_error("cannot write " + ef);
    return -1;
  }
  for (size_t i = 0; i < r.energy.size(); i++) {
    fprintf(f, "State %ld\n", (long)i);
    fprintf(f, "  Energy  %.16lf \n", r.energy[i]);
    fprintf(f, "  Doublon  %.16lf \n", r.doublon[i]);
    fprintf(f, "  Sz  %.16lf \n", r.sz[i]);
    fprintf(f, "\n");
  }
  fclose(f);
  if (m.output_eigenvec && !r.eigenvectors.empty()) {
    // zvo_eigenvec_%d_rank_%d.dat per state: int itr, long dim, complex128[dim+1]
    // (src/CalcByLOBPCG.c:754-771)
    const size_t per = 2 * (size_t)(s.dim + 1);
    for (size_t i = 0; i * per < r.eigenvectors.size(); i++) {
      char name[256];
      snprintf(name, sizeof(name), "%s_eigenvec_%d_rank_%d.dat", m.data_head.c_str(), (int)i, 0);
      const std::string vf = outdir + sep + name;
      FILE *fv = fopen(vf.c_str(), "wb");
      if (!fv) {
        set_error("cannot write " + vf);
        return -1;
      }
      const int itr = r.itr;
      const long dim = (long)s.dim;
      fwrite(&itr, sizeof(int), 1, fv);
      fwrite(&dim, sizeof(long), 1, fv);
      fwrite(r.eigenvectors.data() + i * per, sizeof(double), per, fv);
      fclose(fv);
    }
  }
  for (size_t i = 0; i < r.green.size(); i++) {
    // FullDiag/CG file names (src/global.c:85-86) with the vector's index
    char suffix[64];
    snprintf(suffix, sizeof(suffix), "_eigen%d", (int)i);
    LRET(write_green_files(m, r.green[i], outdir, suffix));
  }
  return 0;
}

}  // namespace hphi
