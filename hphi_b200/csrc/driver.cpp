// Lanczos and TPQ drivers (host C++ over the device kernels) and HPhi-format output.
//
// Lanczos follows Lanczos_EigenValue (src/Lanczos_EigenValue.c:50-310): two-vector
// recurrence without reorthogonalisation, eigenvalues of the stp x stp tridiagonal
// matrix every step, stop when |(E_target - E_before)/E_target| < 10^-LanczosEps or
// beta < 1e-14, E_target = E[LanczosTarget] (0-based).  The eigenvector pass replays
// the recurrence (Lanczos_EigenVector, src/Lanczos_EigenVector.c:46-208) and energy /
// variance follow expec_energy_flct (src/expec_energy_flct.c:34-179).  TPQ follows
// CalcByTPQ / FirstMultiply / Multiply (src/CalcByTPQ.c:52-294, src/FirstMultiply.c:41-85,
// src/Multiply.c:42-68).
//
// Device recurrence per Lanczos step (q_k = s*Q, P holds q_{k-1} scaled):
//   hv:     P <- acc*P + s*H Q  (acc = -beta_{k-1} s_{k-1}),  raw = <Q|HQ>
//   scalar: alpha_k = s^2 raw
//   sweep:  P <- P - alpha_k s Q,  |P|^2
//   scalar: beta_k = |P|; swap(P, Q); s = 1/beta_k
// Scalars stay on the device; the host reads alpha/beta every few steps to run the
// reference's convergence test step by step.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <sys/stat.h>
#include <vector>

#include "batch.hpp"
#include "driver.hpp"
#include "engine.hpp"

namespace hphi {

// ---------------------------------------------------------------- tridiagonal
// Number of eigenvalues of the symmetric tridiagonal (a[0..n), b[0..n-1)) below x
// (Sturm sequence of the LDL^T factorisation of T - x).
static int sturm_count(const double *a, const double *b, int n, double x) {
  int cnt = 0;
  double d = a[0] - x;
  const double tiny = 1e-300;
  if (d < 0) cnt++;
  for (int i = 1; i < n; i++) {
    if (std::fabs(d) < tiny) d = (d < 0) ? -tiny : tiny;
    d = a[i] - x - b[i - 1] * b[i - 1] / d;
    if (d < 0) cnt++;
  }
  return cnt;
}

// k-th smallest eigenvalue (0-based) by bisection to full double precision.
double tridiag_eigenvalue(const double *a, const double *b, int n, int k) {
  double lo = a[0], hi = a[0];
  for (int i = 0; i < n; i++) {
    const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i < n - 1 ? std::fabs(b[i]) : 0.0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  const double span = std::max(std::fabs(lo), std::fabs(hi));
  lo -= 1e-12 * span + 1e-300;
  hi += 1e-12 * span + 1e-300;
  for (int it = 0; it < 200; it++) {
    const double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    if (sturm_count(a, b, n, mid) > k) hi = mid;
    else lo = mid;
  }
  return 0.5 * (lo + hi);
}

// Eigenvector of the tridiagonal matrix for eigenvalue lam by inverse iteration
// (Gaussian elimination with partial pivoting on T - lam), normalised, with the
// sign fixed so that the largest component is positive.
void tridiag_eigenvector(const double *a, const double *b, int n, double lam, std::vector<double> *out) {
  std::vector<double> x(n, 1.0);
  if (n == 1) { out->assign(1, 1.0); return; }
  const double eps = 1e-14 * (std::fabs(lam) + 1.0);
  // Banded LU with partial pivoting: rows have up to 3 non-zeros after pivoting.
  std::vector<double> d(n), du(n), du2(n), dl(n);
  std::vector<int> piv(n);
  for (int it = 0; it < 3; it++) {
    for (int i = 0; i < n; i++) { d[i] = a[i] - lam; du[i] = (i < n - 1) ? b[i] : 0.0; dl[i] = (i < n - 1) ? b[i] : 0.0; du2[i] = 0.0; }
    std::vector<double> rhs = x;
    for (int i = 0; i < n - 1; i++) {
      if (std::fabs(d[i]) >= std::fabs(dl[i])) {
        piv[i] = 0;
        if (std::fabs(d[i]) < eps) d[i] = eps;
        const double f = dl[i] / d[i];
        d[i + 1] -= f * du[i];
        rhs[i + 1] -= f * rhs[i];
        dl[i] = f;
      } else {
        piv[i] = 1;
        const double f = d[i] / dl[i];
        d[i] = dl[i];
        const double t = d[i + 1];
        d[i + 1] = du[i] - f * t;
        du2[i] = (i < n - 2) ? du[i + 1] : 0.0;
        if (i < n - 2) du[i + 1] = -f * du2[i];
        du[i] = t;
        std::swap(rhs[i], rhs[i + 1]);
        rhs[i + 1] -= f * rhs[i];
        dl[i] = f;
      }
    }
    if (std::fabs(d[n - 1]) < eps) d[n - 1] = eps;
    // back substitution
    x[n - 1] = rhs[n - 1] / d[n - 1];
    if (n >= 2) x[n - 2] = (rhs[n - 2] - du[n - 2] * x[n - 1]) / d[n - 2];
    for (int i = n - 3; i >= 0; i--) x[i] = (rhs[i] - du[i] * x[i + 1] - du2[i] * x[i + 2]) / d[i];
    double nrm = 0.0;
    for (double v : x) nrm += v * v;
    nrm = std::sqrt(nrm);
    for (double &v : x) v /= nrm;
  }
  int imax = 0;
  for (int i = 1; i < n; i++)
    if (std::fabs(x[i]) > std::fabs(x[imax])) imax = i;
  if (x[imax] < 0)
    for (double &v : x) v = -v;
  *out = x;
}

namespace {

// ---------------------------------------------------------------- helpers
struct DevBuf {
  void *p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
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

std::string join(const std::string &dir, const std::string &name) {
  if (dir.empty()) return name;
  return dir + "/" + name;
}

int cuda_ok(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

#define RET(x) do { if ((x) != 0) return -1; } while (0)

}  // namespace

VecType default_vec_type(const Sector &s) {
  if (s.model.complex_terms) return kComplex128;
  return (s.model.initial_vec_type == 1) ? kReal64 : kComplex128;
}

// Initial vector of SetInitialVector (src/Lanczos_EigenValue.c:499-611) for the
// deterministic single-element mode (initial_iv > 0 on canonical models), in HPhi's
// 1-based complex128 layout.  Returns false when the reference would use a random vector.
bool single_element_start(const Sector &s, std::vector<double> *v) {
  const Model &m = s.model;
  // random for grand-canonical and general-spin models (src/CalcByLanczos.c:66-93)
  if (m.is_gc() || m.general_spin || m.initial_iv <= 0) return false;
  const uint64_t dim = (uint64_t)s.dim;
  const uint64_t iv = (dim / 2 + (uint64_t)m.initial_iv) % dim + 1;
  v->assign(2 * (dim + 1), 0.0);
  if (iv < dim) {
    if (m.initial_vec_type == 0) {
      (*v)[2 * (iv + 1)] = 1.0 / std::sqrt(2.0);
      (*v)[2 * (iv + 1) + 1] = 1.0 / std::sqrt(2.0);
    } else {
      (*v)[2 * (iv + 1)] = 1.0;
    }
  }
  return true;
}

// Seeded uniform start in [-1, 1) (complex: both parts), normalised; 1-based complex128.
void random_start(const Sector &s, uint64_t seed, bool complex_vec, std::vector<double> *v) {
  const uint64_t dim = (uint64_t)s.dim;
  v->assign(2 * (dim + 1), 0.0);
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
  auto next = [&]() {
    z += 0x9E3779B97F4A7C15ull;
    uint64_t x = z;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x ^= x >> 31;
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
  };
  double nrm = 0.0;
  for (uint64_t i = 1; i <= dim; i++) {
    const double re = 2.0 * (next() - 0.5);
    const double im = complex_vec ? 2.0 * (next() - 0.5) : 0.0;
    (*v)[2 * i] = re;
    (*v)[2 * i + 1] = im;
    nrm += re * re + im * im;
  }
  nrm = std::sqrt(nrm);
  for (uint64_t i = 1; i <= dim; i++) { (*v)[2 * i] /= nrm; (*v)[2 * i + 1] /= nrm; }
}

// ------------------------------------------------------- CG eigenvector refinement
namespace {
constexpr double kEpsEnergy = 1e-12;  // eps_Energy (src/readdef.c:2703,2707)
constexpr double kEpsCG = 1e-8;       // eps and eps_CG (src/readdef.c:2701-2706)

// Inverse iteration with conjugate-gradient solves of (H - Eig + eps_CG) x = b
// (src/CG_EigenVector.c:30-255).  vg holds the normalised Lanczos vector on entry and the
// refined, normalised vector on return (native order).  b gets vg plus random components
// of amplitude 1e-3 (the reference draws them from per-thread dSFMT streams seeded
// 123432 + |iv| + thread; here they are start_value(seed, configuration), so the result
// does not depend on thread counts or the vector order), normalised.  Each round runs CG
// from x = 0 until |r| < eps |b| (at most 500 iterations), normalises x and stops when
// ||<x|b>| - 1| < eps, else restarts from b = x (at most 51 rounds).  The CG scalars are
// real: for a Hermitian H, <p|(H - Eig) p> has no imaginary part.
int cg_eigenvector(Sector *s, VecType vt, double eig, uint64_t seed, void *vg, void *b, void *r, void *p, void *hp,
                   double *st, LanczosResult *res) {
  const int64_t dim = s->dim;
  const size_t esz = (vt == kReal64) ? sizeof(double) : sizeof(cplx);
  const double shift = -eig + kEpsCG;
  auto read = [&](const double *d, double *h, int n) -> int {
    RET(cuda_ok(cudaMemcpyAsync(h, d, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream), "read"));
    return cuda_ok(cudaStreamSynchronize(s->stream), "sync");
  };
  auto copy = [&](void *dst, const void *src) {
    return cuda_ok(cudaMemcpyAsync(dst, src, esz * dim, cudaMemcpyDeviceToDevice, s->stream), "copy");
  };
  // b = vg + random components, in HPhi order so the components follow the configurations
  RET(from_native(s, vt, vg, hp));
  RET(vec_add_hashed(s, vt, seed, 0.002, hp));
  RET(to_native(s, vt, hp, b));
  double h[2];
  RET(vec_norm2(s, vt, b, st + 20));
  RET(read(st + 20, h, 1));
  RET(vec_scale(s, vt, 1.0 / std::sqrt(h[0]), b));
  const double coef[2] = {0.0, 1.0};  // hp = H p
  RET(cuda_ok(cudaMemcpyAsync(st + 22, coef, sizeof(coef), cudaMemcpyHostToDevice, s->stream), "coef"));
  res->cg_rounds = 0;
  res->cg_iterations = 0;
  for (int round = 0; round <= 50; round++) {
    res->cg_rounds = round + 1;
    RET(vec_norm2(s, vt, b, st + 20));
    RET(read(st + 20, h, 1));
    const double bnorm = h[0];
    RET(copy(r, b));
    RET(copy(p, b));
    RET(cuda_ok(cudaMemsetAsync(vg, 0, esz * dim, s->stream), "zero x"));
    double rnorm = bnorm;  // |r|^2 of the current residual
    for (int itr = 1; itr <= 500; itr++) {
      RET(hv_native(s, vt, p, hp, st + 22, st + 24, false));
      RET(vec_dot(s, vt, p, hp, st + 26));
      RET(vec_norm2(s, vt, p, st + 28));
      double d[3];
      RET(read(st + 26, d, 3));
      const double yp = d[0] + shift * d[2];  // <p|(H - Eig + eps_CG) p>
      const double alpha = rnorm / yp;
      RET(vec_cg_sweep(s, vt, alpha, shift, p, hp, vg, r, st + 20));
      RET(read(st + 20, h, 1));
      const double rnorm2 = h[0];
      RET(vec_axpby(s, vt, 1.0, r, rnorm2 / rnorm, p));  // p = r + beta p
      rnorm = rnorm2;
      res->cg_iterations++;
      if (std::sqrt(rnorm2) < kEpsCG * std::sqrt(bnorm)) break;
    }
    RET(vec_norm2(s, vt, vg, st + 20));
    RET(read(st + 20, h, 1));
    RET(vec_scale(s, vt, 1.0 / std::sqrt(h[0]), vg));
    RET(vec_dot(s, vt, vg, b, st + 20));
    RET(read(st + 20, h, 2));
    if (std::fabs(std::hypot(h[0], h[1]) - 1.0) < kEpsCG) break;
    RET(copy(b, vg));
  }
  return 0;
}
}  // namespace

// ------------------------------------------------------------------- Lanczos
int model_green(Sector *s, VecType vt, const void *d_hphi, double scale, GreenValues *g) {
  const Model &m = s->model;
  std::string err;
  std::vector<GreenTerm> terms;
  std::vector<char> trail;
  *g = GreenValues();
  if (!m.green_one.empty()) {
    if (compile_green(m, 1, m.green_one[0].data(), (int)m.green_one.size(), &terms, &trail, &err) != 0) {
      set_error(err);
      return -1;
    }
    RET(green_expect(s, vt, d_hphi, terms, &g->one));
  }
  if (!m.green_two.empty()) {
    if (compile_green(m, 2, m.green_two[0].data(), (int)m.green_two.size(), &terms, &g->trail_two, &err) != 0) {
      set_error(err);
      return -1;
    }
    RET(green_expect(s, vt, d_hphi, terms, &g->two));
  }
  const std::vector<std::vector<int>> *multi[3] = {&m.green_three, &m.green_four, &m.green_six};
  const int body[3] = {3, 4, 6};
  for (int q = 0; q < 3; q++) {
    if (multi[q]->empty()) continue;
    std::vector<int> flat;
    for (const auto &r : *multi[q]) flat.insert(flat.end(), r.begin(), r.end());
    if (compile_green(m, body[q], flat.data(), (int)multi[q]->size(), &terms, &g->multi_short[q], &err) != 0) {
      set_error(err);
      return -1;
    }
    RET(green_expect(s, vt, d_hphi, terms, &g->multi[q]));
  }
  for (double &x : g->one) x *= scale;
  for (double &x : g->two) x *= scale;
  for (auto &v : g->multi)
    for (double &x : v) x *= scale;
  return 0;
}

int write_green_file(const Model &m, const GreenValues &g, int kind, const std::string &path) {
  FILE *f = fopen(path.c_str(), "w");
  if (!f) { set_error("cannot write " + path); return -1; }
  if (kind == 1) {
    for (size_t e = 0; e < m.green_one.size() && 2 * e + 1 < g.one.size(); e++) {
      const auto &r = m.green_one[e];
      fprintf(f, " %4ld %4ld %4ld %4ld %.10lf %.10lf\n", (long)r[0], (long)r[1], (long)r[2], (long)r[3],
              g.one[2 * e], g.one[2 * e + 1]);
    }
  } else if (kind == 2) {
    for (size_t e = 0; e < m.green_two.size() && 2 * e + 1 < g.two.size(); e++) {
      const auto &r = m.green_two[e];
      fprintf(f, " %4ld %4ld %4ld %4ld %4ld %4ld %4ld %4ld %.10lf %.10lf%s\n", (long)r[0], (long)r[1], (long)r[2],
              (long)r[3], (long)r[4], (long)r[5], (long)r[6], (long)r[7], g.two[2 * e], g.two[2 * e + 1],
              g.trail_two[e] ? " " : "");
    }
  } else if (m.calc_model == kSpinGC && !m.general_spin) {
    // expec_Threebody / Fourbody / Sixbody_SpinGCHalf lines (src/expec_cisajscktaltdc.c:1064,
    // 1256, 1402): an extra space before indices 12 and 16 of the four- and six-body rows;
    // other models leave the file empty (:1092-1107)
    const int q = kind == 3 ? 0 : kind == 4 ? 1 : 2;
    const std::vector<std::vector<int>> &rows = kind == 3 ? m.green_three : kind == 4 ? m.green_four : m.green_six;
    for (size_t e = 0; e < rows.size() && 2 * e + 1 < g.multi[q].size(); e++) {
      const int n = g.multi_short[q][e] ? 8 : (int)rows[e].size();
      for (int i = 0; i < n; i++) fprintf(f, "%s %4ld", (kind != 3 && !g.multi_short[q][e] && (i == 12 || (kind == 6 && i == 16))) ? " " : "", (long)rows[e][i]);
      fprintf(f, " %.10lf %.10lf \n", g.multi[q][2 * e], g.multi[q][2 * e + 1]);
    }
  }
  fclose(f);
  return 0;
}

int write_green_files(const Model &m, const GreenValues &g, const std::string &dir, const std::string &suffix) {
  const std::string h = m.data_head;
  if (!m.green_one.empty()) RET(write_green_file(m, g, 1, join(dir, h + "_cisajs" + suffix + ".dat")));
  if (!m.green_two.empty() || !m.green_three.empty() || !m.green_four.empty() || !m.green_six.empty())
    RET(write_green_file(m, g, 2, join(dir, h + "_cisajscktalt" + suffix + ".dat")));
  if (!m.green_three.empty()) RET(write_green_file(m, g, 3, join(dir, h + "_ThreeBody" + suffix + ".dat")));
  if (!m.green_four.empty()) RET(write_green_file(m, g, 4, join(dir, h + "_FourBody" + suffix + ".dat")));
  if (!m.green_six.empty()) RET(write_green_file(m, g, 6, join(dir, h + "_SixBody" + suffix + ".dat")));
  return 0;
}

int lanczos_run(Sector *s, VecType vt, const double *h_init, const LanczosOptions &opt, LanczosResult *res) {
  const Model &m = s->model;
  const int64_t dim = s->dim;
  const size_t esz = (vt == kReal64) ? sizeof(double) : sizeof(cplx);
  RET(cuda_ok(cudaSetDevice(s->device), "cudaSetDevice"));
  DevBuf P, Q, V0, ST, AL, BE;
  RET(cuda_ok(cudaMalloc(&P.p, esz * dim), "alloc P"));
  RET(cuda_ok(cudaMalloc(&Q.p, esz * dim), "alloc Q"));
  RET(cuda_ok(cudaMalloc(&ST.p, sizeof(double) * 32), "alloc scalars"));  // slots used: [0, 29)
  const bool fixed = opt.fixed_steps > 0;
  const LanczosRestart *rs = opt.resume;
  const int n0 = rs ? rs->steps : 0;  // steps already done (restart)
  res->resumed = (rs != nullptr);
  int max_steps = fixed ? opt.fixed_steps : n0 + m.lanczos_max;
  if ((int64_t)max_steps > dim) max_steps = (int)dim;
  if (rs && (n0 < 1 || n0 >= max_steps)) {
    set_error("Lanczos restart: the stored step count leaves no step to run");
    return -1;
  }
  if (!fixed && dim < m.lanczos_target) max_steps = (int)dim;
  RET(cuda_ok(cudaMalloc(&AL.p, sizeof(double) * (max_steps + 2)), "alloc alpha"));
  RET(cuda_ok(cudaMalloc(&BE.p, sizeof(double) * (max_steps + 2)), "alloc beta"));
  // start vector: HPhi order on the host (or hashed on the device) -> native order on the device
  if (opt.hashed_start) {
    RET(vec_fill_hashed(s, vt, opt.hashed_seed, P.p));
    RET(vec_norm2(s, vt, P.p, s->d_scal));
    double n2 = 0.0;
    RET(cuda_ok(cudaMemcpyAsync(&n2, s->d_scal, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "norm"));
    RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
    if (!(n2 > 0.0)) {
      set_error("hashed start vector has zero norm");
      return -1;
    }
    RET(vec_scale(s, vt, 1.0 / std::sqrt(n2), P.p));
  } else if (opt.device_start) {
    RET(cuda_ok(cudaMemcpyAsync(P.p, opt.device_start, esz * dim, cudaMemcpyDeviceToDevice, s->stream), "start"));
  } else {
    RET(vec_from_host_c128(s, vt, h_init, P.p));
  }
  RET(to_native(s, vt, P.p, Q.p));
  const bool want_vec = opt.eigenvector;
  if (want_vec) {
    RET(cuda_ok(cudaMalloc(&V0.p, esz * dim), "alloc V0"));
    RET(cuda_ok(cudaMemcpyAsync(V0.p, Q.p, esz * dim, cudaMemcpyDeviceToDevice, s->stream), "copy V0"));
  }
  double *st = (double *)ST.p;
  std::vector<double> alpha(max_steps + 2, 0.0), beta(max_steps + 2, 0.0);
  if (rs) {
    // HPhi's next step takes v1' = (v0 - alpha_n v1) / beta_n: here Q = v0 - alpha_n v1 with
    // scale 1/beta_n and P = v1 with acc = -beta_n (src/Lanczos_EigenValue.c:80-101, 153-160)
    DevBuf T;
    RET(cuda_ok(cudaMalloc(&T.p, esz * dim), "alloc restart"));
    RET(vec_from_host_c128(s, vt, rs->v1.data(), T.p));
    RET(to_native(s, vt, T.p, P.p));
    RET(vec_from_host_c128(s, vt, rs->v0.data(), T.p));
    RET(to_native(s, vt, T.p, Q.p));
    RET(vec_axpby(s, vt, -rs->alpha[n0], P.p, 1.0, Q.p));
    for (int i = 1; i <= n0; i++) { alpha[i] = rs->alpha[i]; beta[i] = rs->beta[i]; }
    RET(cuda_ok(cudaMemcpyAsync(AL.p, alpha.data(), sizeof(double) * (n0 + 1), cudaMemcpyHostToDevice, s->stream), "alpha"));
    RET(cuda_ok(cudaMemcpyAsync(BE.p, beta.data(), sizeof(double) * (n0 + 1), cudaMemcpyHostToDevice, s->stream), "beta"));
    const double rs_st[6] = {0.0, 0.0, -rs->beta[n0], 1.0 / rs->beta[n0], 0.0, 0.0};
    RET(cuda_ok(cudaMemcpyAsync(st, rs_st, sizeof(rs_st), cudaMemcpyHostToDevice, s->stream), "restart scalars"));
    RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
  } else {
    const double init_st[6] = {0.0, 0.0, 0.0, 1.0, 0.0, 0.0};  // acc = 0, s = 1
    RET(cuda_ok(cudaMemcpyAsync(st, init_st, sizeof(init_st), cudaMemcpyHostToDevice, s->stream), "init scalars"));
    RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
  }
  void *pp = P.p, *qq = Q.p;
  auto do_step = [&](int k) -> int {
    RET(hv_native(s, vt, qq, pp, st + 2, st + 0));
    RET(lanczos_scalars(s, 0, k, st, (double *)AL.p, (double *)BE.p));
    RET(vec_lanczos_sweep(s, vt, st + 4, pp, qq, st + 5));
    RET(lanczos_scalars(s, 1, k, st, (double *)AL.p, (double *)BE.p));
    std::swap(pp, qq);
    return 0;
  };

  const int target = m.lanczos_target;
  const double eps = std::pow(10.0, -m.lanczos_eps);
  res->lines.clear();
  res->converged = false;
  res->steps = 0;
  // restart output needs the device state of the exact last step: check every step
  const int batch = opt.restart_out ? 1 : (opt.batch > 0 ? opt.batch : (fixed ? 32 : (dim >= (1 << 20) ? 1 : 16)));
  int done = n0;            // steps executed on the device
  int checked = rs ? n0 : 1;  // steps examined on the host
  double ebefor = 0.0;
  std::vector<double> E(5, 0.0);
  const double ns = (double)m.nsite;
  char line[512];
  if (dim == 1) {
    RET(do_step(1));
    RET(cuda_ok(cudaMemcpy(alpha.data(), AL.p, sizeof(double) * 2, cudaMemcpyDeviceToHost), "read alpha"));
    res->converged = true;
    res->steps = 1;
    res->energies.assign(1, alpha[1]);
    res->e_target = alpha[1];
  }
  while (dim > 1 && !res->converged && checked < max_steps) {
    const int upto = std::min(max_steps, done + batch);
    if (done == 0) { RET(do_step(1)); done = 1; }
    while (done < upto) { done++; RET(do_step(done)); }
    RET(cuda_ok(cudaMemcpyAsync(alpha.data(), AL.p, sizeof(double) * (done + 1), cudaMemcpyDeviceToHost, s->stream), "read alpha"));
    RET(cuda_ok(cudaMemcpyAsync(beta.data(), BE.p, sizeof(double) * (done + 1), cudaMemcpyDeviceToHost, s->stream), "read beta"));
    RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
    for (int stp = checked + 1; stp <= done; stp++) {
      checked = stp;
      const double *a = alpha.data() + 1;
      const double *b = beta.data() + 1;
      if (fixed) {  // no step lines, no convergence test: stop at max_steps or on a breakdown
        if (std::fabs(beta[stp]) < 1e-14 || stp == max_steps) {
          res->converged = true;
          res->steps = stp;
          res->e_target = tridiag_eigenvalue(a, b, stp, std::min(target, stp - 1));
          break;
        }
        continue;
      }
      if (stp == 2) {
        E[1] = tridiag_eigenvalue(a, b, 2, 0);
        E[2] = tridiag_eigenvalue(a, b, 2, 1);
        res->lines.push_back(std::string("LanczosStep  E[1] E[2] E[3] E[4] Target:E[") + std::to_string(target + 1) +
                             "] E_Max/Nsite\n");
        if (target < 2) {
          const double et = (target == 0) ? E[1] : E[2];
          ebefor = et;
          snprintf(line, sizeof(line), "stp = %d %.10lf %.10lf xxxxxxxxxx xxxxxxxxx %.10lf xxxxxxxxx \n", stp, E[1],
                   E[2], et);
        } else {
          snprintf(line, sizeof(line), "stp = %d %.10lf %.10lf xxxxxxxxxx xxxxxxxxx xxxxxxxxx xxxxxxxxx \n", stp, E[1],
                   E[2]);
        }
        res->lines.push_back(line);
      }
      if (stp > 2) {
        for (int q = 0; q < 4; q++) E[q + 1] = (q < stp) ? tridiag_eigenvalue(a, b, stp, q) : 0.0;
        E[0] = tridiag_eigenvalue(a, b, stp, stp - 1);
        double et = 0.0;
        if (stp > target) {
          et = tridiag_eigenvalue(a, b, stp, target);
          snprintf(line, sizeof(line), "stp=%d %.10lf %.10lf %.10lf %.10lf %.10lf %.10lf\n", stp, E[1], E[2], E[3],
                   E[4], et, E[0] / ns);
        } else {
          snprintf(line, sizeof(line), "stp=%d %.10lf %.10lf %.10lf %.10lf xxxxxxxxx %.10lf\n", stp, E[1], E[2], E[3],
                   E[4], E[0] / ns);
        }
        res->lines.push_back(line);
        if (stp > target) {
          if (std::fabs((et - ebefor) / et) < eps || std::fabs(beta[stp]) < 1e-14) {
            res->converged = true;
            res->steps = stp;
            res->e_target = et;
            break;
          }
          ebefor = et;
        }
      }
    }
  }
  if (!res->converged) {
    res->steps = checked;
  }
  if (opt.restart_out && dim > 1) {
    // HPhi's v0 and v1 after the last step k (src/Lanczos_EigenValue.c:287-291): v1 = q_k =
    // P / beta_{k-1} (P holds q_k unscaled; beta_0 = 1, or the stored beta_n when resumed),
    // v0 = H q_k - beta_{k-1} q_{k-1} = Q + alpha_k v1.  The files record (exit step - 1)
    // coefficients: the converged step, or one past the last step when none converged.
    const int k = checked;
    LanczosRestart &R = res->restart;
    R.dnorm = rs ? rs->dnorm : 0.0;
    R.steps = res->converged ? k - 1 : k;
    R.vec_steps = R.steps;
    R.alpha.assign(alpha.begin(), alpha.begin() + R.steps + 1);
    R.beta.assign(beta.begin(), beta.begin() + R.steps + 1);
    const double bprev = (k >= 2) ? beta[k - 1] : 1.0;
    DevBuf A, B;
    RET(cuda_ok(cudaMalloc(&A.p, esz * dim), "alloc restart"));
    RET(cuda_ok(cudaMalloc(&B.p, esz * dim), "alloc restart"));
    RET(cuda_ok(cudaMemcpyAsync(A.p, pp, esz * dim, cudaMemcpyDeviceToDevice, s->stream), "copy"));
    RET(vec_scale(s, vt, 1.0 / bprev, A.p));                 // v1 (native)
    RET(cuda_ok(cudaMemcpyAsync(B.p, qq, esz * dim, cudaMemcpyDeviceToDevice, s->stream), "copy"));
    RET(vec_axpby(s, vt, alpha[k], A.p, 1.0, B.p));          // v0 (native)
    R.v0.assign(2 * (dim + 1), 0.0);
    R.v1.assign(2 * (dim + 1), 0.0);
    RET(from_native(s, vt, B.p, pp));
    RET(vec_to_host_c128(s, vt, pp, R.v0.data()));
    RET(from_native(s, vt, A.p, pp));
    RET(vec_to_host_c128(s, vt, pp, R.v1.data()));
    // HPhi's loop variable ends at the converged step or one past the last step, and it
    // skips the files when that is two steps past the run's start
    const int exit_stp = res->converged ? k : k + 1;
    res->has_restart = (exit_stp != (rs ? n0 : 1) + 2);
  }
  const int itr = res->steps;
  res->alpha.assign(alpha.begin() + 1, alpha.begin() + 1 + itr);
  res->beta.assign(beta.begin() + 1, beta.begin() + 1 + itr);
  res->energies.clear();
  const int nev = std::min(itr, std::max(m.nvec, m.lanczos_target + 1));
  for (int q = 0; q < nev && q < itr; q++) res->energies.push_back(tridiag_eigenvalue(res->alpha.data(), res->beta.data(), itr, q));
  if (!res->converged) {
    if (opt.restart_out) return 0;  // restart mode: the files carry the run on
    set_error("Lanczos Eigenvalue is not converged in this process.");
    return -1;
  }
  if (!want_vec) return 0;

  // ---- eigenvector: vg = sum_k c_k q_k with c the k_exct-th tridiagonal eigenvector
  const int kx = m.k_exct - 1;
  const double lam = tridiag_eigenvalue(res->alpha.data(), res->beta.data(), itr, kx);
  res->e_tridiag = lam;
  std::vector<double> c;
  tridiag_eigenvector(res->alpha.data(), res->beta.data(), itr, lam, &c);
  DevBuf VG;
  RET(cuda_ok(cudaMalloc(&VG.p, esz * dim), "alloc VG"));
  pp = P.p; qq = Q.p;
  RET(cuda_ok(cudaMemcpyAsync(qq, V0.p, esz * dim, cudaMemcpyDeviceToDevice, s->stream), "copy"));
  RET(cuda_ok(cudaMemcpyAsync(VG.p, V0.p, esz * dim, cudaMemcpyDeviceToDevice, s->stream), "copy"));
  RET(vec_scale(s, vt, c[0], VG.p));
  double sq = 1.0, acc = 0.0;
  for (int k = 1; k < itr; k++) {
    const double coef[2] = {acc, sq};
    RET(cuda_ok(cudaMemcpyAsync(st + 8, coef, sizeof(coef), cudaMemcpyHostToDevice, s->stream), "coef"));
    RET(hv_native(s, vt, qq, pp, st + 8, st + 10));
    const double ak = res->alpha[k - 1], bk = res->beta[k - 1];
    RET(vec_replay_sweep(s, vt, ak * sq, c[k] / bk, pp, qq, VG.p));
    RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
    acc = -bk * sq;
    sq = 1.0 / bk;
    std::swap(pp, qq);
  }
  double nrm2 = 0.0;
  RET(vec_norm2(s, vt, VG.p, st + 12));
  RET(cuda_ok(cudaMemcpyAsync(&nrm2, st + 12, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "read"));
  RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
  RET(vec_scale(s, vt, 1.0 / std::sqrt(nrm2), VG.p));
  // expec_energy_flct: H vg -> E = <vg|H vg>, var = <H vg|H vg>
  auto expec = [&]() -> int {
    const double coef1[2] = {0.0, 1.0};
    RET(cuda_ok(cudaMemcpyAsync(st + 8, coef1, sizeof(coef1), cudaMemcpyHostToDevice, s->stream), "coef"));
    RET(hv_native(s, vt, VG.p, pp, st + 8, st + 10));
    RET(vec_norm2(s, vt, pp, st + 12));
    RET(native_observables(s, vt, VG.p, st + 13));
    double sc[10];
    RET(cuda_ok(cudaMemcpyAsync(sc, st + 10, sizeof(double) * 9, cudaMemcpyDeviceToHost, s->stream), "read"));
    RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
    res->energy = sc[0];
    res->var = sc[2];
    res->doublon = sc[3];
    res->sz = sc[7];
    return 0;
  };
  RET(expec());
  // accuracy check (src/CalcByLanczos.c:120-128), eps_Energy = 1e-12 (src/readdef.c:2701-2707)
  auto rel_var = [&]() { return std::fabs(res->var - res->energy * res->energy) / std::fabs(res->var); };
  auto rel_diff = [&]() { return std::fabs(lam - res->energy) / std::fabs(lam); };
  res->check_var = rel_var();
  res->check_diff = rel_diff();
  if (!(res->check_diff < kEpsEnergy && res->check_var < kEpsEnergy) && m.calc_eigenvec == 0) {
    DevBuf B, HP;
    RET(cuda_ok(cudaMalloc(&B.p, esz * dim), "alloc CG b"));
    RET(cuda_ok(cudaMalloc(&HP.p, esz * dim), "alloc CG hp"));
    // V0 (the start vector) is no longer needed: it holds the CG search direction
    RET(cg_eigenvector(s, vt, lam, (uint64_t)(123432 + std::abs((long)m.initial_iv)), VG.p, B.p, pp, V0.p, HP.p, st, res));
    RET(expec());
    res->cg_ran = true;
    res->cg_var = rel_var();
    res->cg_diff = rel_diff();
  }
  // expec_cisajs / expec_cisajscktaltdc of the eigenvector (src/CalcByLanczos.c:229-240)
  if (!m.green_one.empty() || !m.green_two.empty() || !m.green_three.empty() || !m.green_four.empty() ||
      !m.green_six.empty()) {
    RET(from_native(s, vt, VG.p, pp));
    RET(model_green(s, vt, pp, 1.0, &res->green));
  }
  res->eigenvector.assign(2 * (dim + 1), 0.0);
  if (opt.copy_eigenvector) {
    RET(from_native(s, vt, VG.p, pp));
    RET(vec_to_host_c128(s, vt, pp, res->eigenvector.data()));
  } else {
    res->eigenvector.clear();
  }
  return 0;
}

int lanczos_input_vector(Sector *s, VecType vt, const std::string &outdir, int mode, LanczosResult *res) {
  const Model &m = s->model;
  const int64_t dim = s->dim;
  char name[256];
  snprintf(name, sizeof(name), "%s_eigenvec_%d_rank_%d.dat", m.data_head.c_str(), std::max(1, m.k_exct) - 1, 0);
  const std::string path = join(outdir, name);
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) { set_error("Error: A file of Inputvector does not exist."); return -1; }
  int itr = 0;
  long fdim = 0;
  std::vector<double> h(2 * (size_t)(dim + 1), 0.0);
  const bool ok = fread(&itr, sizeof(int), 1, f) == 1 && fread(&fdim, sizeof(long), 1, f) == 1 && fdim == (long)dim &&
                  fread(h.data(), sizeof(double), h.size(), f) == h.size();
  fclose(f);
  if (!ok) { set_error("Error: A file of Inputvector is incorrect."); return -1; }
  h[0] = h[1] = 0.0;
  for (int64_t i = 1; i <= dim && vt == kReal64; i++)
    if (h[2 * i + 1] != 0.0) vt = kComplex128;  // a complex stored vector keeps its phases
  const size_t esz = (vt == kReal64) ? sizeof(double) : sizeof(cplx);
  RET(cuda_ok(cudaSetDevice(s->device), "cudaSetDevice"));
  DevBuf A, B, C, ST;
  RET(cuda_ok(cudaMalloc(&A.p, esz * dim), "alloc"));
  RET(cuda_ok(cudaMalloc(&B.p, esz * dim), "alloc"));
  RET(cuda_ok(cudaMalloc(&ST.p, sizeof(double) * 32), "alloc scalars"));
  double *st = (double *)ST.p;
  RET(vec_from_host_c128(s, vt, h.data(), A.p));
  RET(to_native(s, vt, A.p, B.p));
  if (mode == 2) {
    // v0 = H v1 (v0 starts at zero), v1 = v0 / |v0| (src/CalcByLanczos.c:208-223)
    RET(cuda_ok(cudaMalloc(&C.p, esz * dim), "alloc"));
    const double coef[2] = {0.0, 1.0};
    RET(cuda_ok(cudaMemcpyAsync(st, coef, sizeof(coef), cudaMemcpyHostToDevice, s->stream), "coef"));
    RET(hv_native(s, vt, B.p, C.p, st, st + 2, false));
    RET(vec_norm2(s, vt, C.p, st + 4));
    double n2 = 0.0;
    RET(cuda_ok(cudaMemcpyAsync(&n2, st + 4, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "read"));
    RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
    RET(vec_scale(s, vt, 1.0 / std::sqrt(n2), C.p));
    std::swap(B.p, C.p);
    RET(from_native(s, vt, B.p, A.p));
  }
  RET(model_green(s, vt, A.p, 1.0, &res->green));
  RET(native_observables(s, vt, B.p, st + 8));  // expec_totalSz
  double ob[6];
  RET(cuda_ok(cudaMemcpyAsync(ob, st + 8, sizeof(ob), cudaMemcpyDeviceToHost, s->stream), "read"));
  RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
  res->sz = ob[4];
  res->energy = res->doublon = 0.0;
  res->converged = true;
  res->from_input = true;
  res->steps = 0;
  res->eigenvector.assign(2 * (dim + 1), 0.0);
  RET(vec_to_host_c128(s, vt, A.p, res->eigenvector.data()));
  return cuda_ok(cudaStreamSynchronize(s->stream), "sync");
}

// OutputTMComponents / OutputLanczosVector (src/Lanczos_EigenValue.c:457-500, 697-720).
int write_lanczos_restart(const Sector &s, const LanczosRestart &r, const std::string &outdir) {
  RET(ensure_dir(outdir));
  const std::string head = s.model.data_head;
  const std::string tm = join(outdir, head + "_TMComponents.dat");
  FILE *f = fopen(tm.c_str(), "w");
  if (!f) { set_error("cannot write " + tm); return -1; }
  fprintf(f, "%d \n", r.steps);
  fprintf(f, "%.10lf \n", r.dnorm);
  for (int i = 1; i <= r.steps; i++) fprintf(f, "%.10lf %.10lf \n", r.alpha[i], r.beta[i]);
  fclose(f);
  const std::string vf = join(outdir, head + "_recalcvec_rank_0.dat");
  f = fopen(vf.c_str(), "wb");
  if (!f) { set_error("cannot write " + vf); return -1; }
  const unsigned long stp = (unsigned long)r.vec_steps;
  const long dim = (long)s.dim;
  fwrite(&stp, sizeof(stp), 1, f);
  fwrite(&dim, sizeof(dim), 1, f);
  fwrite(r.v0.data(), sizeof(double), r.v0.size(), f);
  fwrite(r.v1.data(), sizeof(double), r.v1.size(), f);
  fclose(f);
  return 0;
}

// ReadInitialVector / ReadTMComponents (src/Lanczos_EigenValue.c:428-455, 624-695): the
// coefficients come back with the 10 decimals they were printed with.
int read_lanczos_restart(const Sector &s, const std::string &outdir, LanczosRestart *r) {
  const std::string head = s.model.data_head;
  const std::string vf = join(outdir, head + "_recalcvec_rank_0.dat");
  FILE *f = fopen(vf.c_str(), "rb");
  if (!f) { set_error("Lanczos restart: cannot open " + vf); return -1; }
  unsigned long stp = 0;
  long dim = 0;
  const size_t n = 2 * (size_t)(s.dim + 1);
  r->v0.assign(n, 0.0);
  r->v1.assign(n, 0.0);
  const bool ok = fread(&stp, sizeof(stp), 1, f) == 1 && fread(&dim, sizeof(dim), 1, f) == 1 && dim == (long)s.dim &&
                  fread(r->v0.data(), sizeof(double), n, f) == n && fread(r->v1.data(), sizeof(double), n, f) == n;
  fclose(f);
  if (!ok) { set_error("Lanczos restart: " + vf + " does not hold vectors of this sector"); return -1; }
  const std::string tm = join(outdir, head + "_TMComponents.dat");
  f = fopen(tm.c_str(), "r");
  if (!f) { set_error("Lanczos restart: cannot open " + tm); return -1; }
  long steps = 0;
  char buf[256];
  if (!fgets(buf, sizeof(buf), f) || sscanf(buf, "%ld", &steps) != 1 || !fgets(buf, sizeof(buf), f) ||
      sscanf(buf, "%lf", &r->dnorm) != 1) {
    fclose(f);
    set_error("Lanczos restart: malformed " + tm);
    return -1;
  }
  r->alpha.assign(1, 0.0);
  r->beta.assign(1, 0.0);
  double a, b;
  while (fgets(buf, sizeof(buf), f))
    if (sscanf(buf, "%lf %lf", &a, &b) == 2) { r->alpha.push_back(a); r->beta.push_back(b); }
  fclose(f);
  if ((long)r->alpha.size() - 1 != steps || (unsigned long)steps != stp) {
    set_error("Lanczos restart: input files for vector and TMcomponents are incorrect");
    return -1;
  }
  r->steps = (int)steps;
  r->vec_steps = (int)stp;
  return 0;
}

int write_lanczos_outputs(const Sector &s, const LanczosResult &r, const std::string &outdir) {
  RET(ensure_dir(outdir));
  const Model &m = s.model;
  FILE *f = nullptr;
  if (!r.from_input) {
    const std::string step_file = join(outdir, m.data_head + "_Lanczos_Step.dat");
    // a continued run appends to the step file (src/Lanczos_EigenValue.c:200-222)
    f = fopen(step_file.c_str(), r.resumed ? "a" : "w");
    if (!f) { set_error("cannot write " + step_file); return -1; }
    for (const auto &l : r.lines) fputs(l.c_str(), f);
    fclose(f);
    if (m.calc_eigenvec == -1 || !r.converged) return 0;
  }
  const std::string ef = join(outdir, m.data_head + "_energy.dat");
  f = fopen(ef.c_str(), "w");
  if (!f) { set_error("cannot write " + ef); return -1; }
  fprintf(f, "Energy  %.16lf \n", r.energy);
  fprintf(f, "Doublon  %.16lf \n", r.doublon);
  fprintf(f, "Sz  %.16lf \n", r.sz);
  fclose(f);
  RET(write_green_files(m, r.green, outdir, ""));
  if (m.output_eigenvec && !r.eigenvector.empty()) {
    // zvo_eigenvec_%d_rank_%d.dat: int step, long dim, complex128[dim+1] (src/CalcByLanczos.c:262-273)
    char name[256];
    snprintf(name, sizeof(name), "%s_eigenvec_%d_rank_%d.dat", m.data_head.c_str(), m.k_exct - 1, 0);
    const std::string vf = join(outdir, name);
    f = fopen(vf.c_str(), "wb");
    if (!f) { set_error("cannot write " + vf); return -1; }
    const int itr = r.steps;
    const long dim = (long)s.dim;
    fwrite(&itr, sizeof(int), 1, f);
    fwrite(&dim, sizeof(long), 1, f);
    fwrite(r.eigenvector.data(), sizeof(double), r.eigenvector.size(), f);
    fclose(f);
  }
  return 0;
}

// ------------------------------------------------------------------------ TPQ
int tpq_run(Sector *s, VecType vt, const double *h_init, int rand_i, const std::string &outdir, TpqResult *res,
            const TpqOptions &opt) {
  std::vector<TpqResult> r(1);
  const int rc = tpq_run_samples(s, vt, {h_init}, {rand_i}, outdir, &r, opt, false);
  *res = std::move(r[0]);
  return rc;
}

int tpq_run_samples(Sector *s, VecType vt, const std::vector<const double *> &h_init, const std::vector<int> &rand_i,
                    const std::string &outdir, std::vector<TpqResult> *res, const TpqOptions &opt, bool block) {
  // Samples run in lockstep: every H application of a step is one block H*V over all of them
  // (hv_block_native) when `block`, else one launch per sample; everything else is per sample.
  const Model &m = s->model;
  const int nb = (int)h_init.size();
  const int64_t dim = s->dim;
  const size_t esz = (vt == kReal64) ? sizeof(double) : sizeof(cplx);
  const double Ns = (double)m.nsite;
  const double L = m.large_value;
  if (nb < 1 || (int)rand_i.size() != nb || (block && (nb > kHvBlockMax || !hv_block_applies(s, vt))) ||
      (nb > 1 && opt.resume_step > 0)) {
    set_error("tpq_run_samples: bad sample block");
    return -1;
  }
  res->assign(nb, TpqResult());
  RET(cuda_ok(cudaSetDevice(s->device), "cudaSetDevice"));
  constexpr int kSlots = 32;  // per-sample scalar slots (coefficients, sums)
  DevBuf V, H, ST, PART;
  RET(cuda_ok(cudaMalloc(&V.p, esz * dim * nb), "alloc V"));
  RET(cuda_ok(cudaMalloc(&H.p, esz * dim * nb), "alloc H"));
  RET(cuda_ok(cudaMalloc(&ST.p, sizeof(double) * kSlots * nb), "alloc scalars"));
  if (block) RET(cuda_ok(cudaMalloc(&PART.p, sizeof(double) * 2 * nb * (size_t)s->red_blocks), "alloc partials"));
  auto vec = [&](void *base, int b) { return (void *)((char *)base + esz * dim * b); };
  auto slot = [&](int b) { return (double *)ST.p + kSlots * b; };
  // h_init[b] is the un-normalised start vector of sample b; its norm is global_1st_norm.
  for (int b = 0; b < nb; b++) {
    RET(vec_from_host_c128(s, vt, h_init[b], vec(H.p, b)));
    RET(to_native(s, vt, vec(H.p, b), vec(V.p, b)));
    RET(vec_norm2(s, vt, vec(V.p, b), slot(b)));
  }
  std::vector<double> host(kSlots * nb);
  auto read_slots = [&]() -> int {
    RET(cuda_ok(cudaMemcpyAsync(host.data(), ST.p, sizeof(double) * kSlots * nb, cudaMemcpyDeviceToHost, s->stream),
                "read"));
    return cuda_ok(cudaStreamSynchronize(s->stream), "sync");
  };
  RET(read_slots());
  const bool resumed = opt.resume_step > 0;
  // global_1st_norm is only set by MakeIniVec, so a continued run prints 0 (its initial value)
  std::vector<double> first_norm(nb), sv(nb);  // V_b holds the current vector times 1/sv[b]
  for (int b = 0; b < nb; b++) {
    first_norm[b] = resumed ? 0.0 : std::sqrt(host[kSlots * b]);
    sv[b] = 1.0 / std::sqrt(host[kSlots * b]);
  }
  RET(ensure_dir(outdir));
  std::vector<FILE *> fss(nb, nullptr), fnorm(nb, nullptr), fflct(nb, nullptr);
  struct Closer {
    std::vector<FILE *> *f[3];
    ~Closer() {
      for (auto *v : f)
        for (FILE *x : *v)
          if (x) fclose(x);
    }
  } closer{{&fss, &fnorm, &fflct}};
  const char *mode = resumed ? "a" : "w";  // a continued run appends (src/CalcByTPQ.c:118-136)
  for (int b = 0; b < nb; b++) {
    char name[256];
    snprintf(name, sizeof(name), "SS_rand%d.dat", rand_i[b]);
    fss[b] = fopen(join(outdir, name).c_str(), mode);
    snprintf(name, sizeof(name), "Norm_rand%d.dat", rand_i[b]);
    fnorm[b] = fopen(join(outdir, name).c_str(), mode);
    snprintf(name, sizeof(name), "Flct_rand%d.dat", rand_i[b]);
    fflct[b] = fopen(join(outdir, name).c_str(), mode);
    if (!fss[b] || !fnorm[b] || !fflct[b]) {
      set_error("cannot write TPQ output files in " + outdir);
      return -1;
    }
    if (!resumed) {
      fprintf(fss[b], " # inv_tmp, energy, phys_var, phys_doublon, phys_num, step_i\n");
      fprintf(fnorm[b], " # inv_temp, global_norm, global_1st_norm, step_i \n");
      fprintf(fflct[b], " # inv_temp, N, N^2, D, D^2, Sz, Sz^2, step_i \n");
    }
  }
  // H applied to every sample: dst_b = acc_b dst_b + scale_b H src_b with (acc, scale) in slot
  // c0 and <src_b|H src_b> into slot c0 + 2 of each sample
  auto apply_h = [&](void *src, void *dst, int c0) -> int {
    if (block)
      return hv_block_native(s, vt, nb, dim, src, dst, slot(0) + c0, kSlots, slot(0) + c0 + 2, kSlots,
                             (double *)PART.p);
    for (int b = 0; b < nb; b++) RET(hv_native(s, vt, vec(src, b), vec(dst, b), slot(b) + c0, slot(b) + c0 + 2, false));
    return 0;
  };
  // expec_energy_flct on every sample's current vector sv*V: observables, H = H*(sv V), E, var.
  std::vector<std::array<double, 6>> ob(nb);
  std::vector<double> E(nb, 0.0), var(nb, 0.0);
  auto expec = [&]() -> int {
    for (int b = 0; b < nb; b++) {
      RET(native_observables(s, vt, vec(V.p, b), slot(b) + 16));
      const double coef[2] = {0.0, sv[b]};
      RET(cuda_ok(cudaMemcpyAsync(slot(b) + 4, coef, sizeof(coef), cudaMemcpyHostToDevice, s->stream), "coef"));
    }
    RET(apply_h(V.p, H.p, 4));
    for (int b = 0; b < nb; b++) RET(vec_norm2(s, vt, vec(H.p, b), slot(b) + 8));
    RET(read_slots());
    for (int b = 0; b < nb; b++) {
      const double *h = host.data() + kSlots * b;
      const double w2 = sv[b] * sv[b];
      for (int k = 0; k < 6; k++) ob[b][k] = h[16 + k] * w2;
      E[b] = h[6] * sv[b] * sv[b];
      var[b] = h[8];
    }
    return 0;
  };
  auto write_lines = [&](int b, double inv_temp, double gnorm, int step, bool flct) {
    fprintf(fss[b], "%.16lf  %.16lf %.16lf %.16lf %.16lf %d\n", inv_temp, E[b], var[b], ob[b][0], ob[b][2], step);
    fprintf(fnorm[b], "%.16lf %.16lf %.16lf %d\n", inv_temp, gnorm, first_norm[b], step);
    if (flct)
      fprintf(fflct[b], "%.16lf %.16lf %.16lf %.16lf %.16lf %.16lf %.16lf %d\n", inv_temp, ob[b][2], ob[b][3],
              ob[b][0], ob[b][1], ob[b][4], ob[b][5], step);
  };
  std::vector<double> gnorm(nb, 0.0), inv_temp(nb, 0.0);
  auto multiply = [&]() -> int {
    // v = L*v - H v / Ns with v = sv V: V <- (L sv) V - (1/Ns) H, then normalise lazily.
    for (int b = 0; b < nb; b++) RET(vec_tpq_sweep(s, vt, L * sv[b], 1.0 / Ns, vec(V.p, b), vec(H.p, b), slot(b) + 10));
    RET(read_slots());
    for (int b = 0; b < nb; b++) {
      gnorm[b] = std::sqrt(host[kSlots * b + 10]);
      sv[b] = 1.0 / gnorm[b];
    }
    return 0;
  };
  // Green's functions of the normalised state sv*V at step 0 and at every ExpecInterval-th
  // step from 2 on (src/CalcByTPQ.c:170-179, 261-271), files %s_cisajs_set%dstep%d.dat
  const bool green = !m.green_one.empty() || !m.green_two.empty() || !m.green_three.empty() ||
                     !m.green_four.empty() || !m.green_six.empty();
  DevBuf GV;
  if (green) RET(cuda_ok(cudaMalloc(&GV.p, esz * dim), "alloc Green's function staging"));
  auto green_step = [&](int step) -> int {
    for (int b = 0; b < nb; b++) {
      RET(from_native(s, vt, vec(V.p, b), GV.p));
      GreenValues g;
      RET(model_green(s, vt, GV.p, sv[b] * sv[b], &g));
      char suffix[64];
      snprintf(suffix, sizeof(suffix), "_set%dstep%d", rand_i[b], step);
      RET(write_green_files(m, g, outdir, suffix));
    }
    return 0;
  };
  // canonical TPQ (CalcType 5, CalcByCanonicalTPQ src/CalcByCanonicalTPQ.c:52-287): the step
  // is v <- exp(-dtau H / 2) v / |.|, dtau = 1/LargeValue, by a Taylor sum of ExpandCoef terms
  // (MultiplyForCanonicalTPQ src/Multiply.c:162-203), and the inverse temperature grows by dtau
  const bool canonical = m.calc_type == kcTPQ;
  const int expand = m.expand_coef > 0 ? m.expand_coef : 10;
  const double dtau = 1.0 / L;
  DevBuf CA, CT, CU;
  if (canonical) {
    RET(cuda_ok(cudaMalloc(&CA.p, esz * dim * nb), "alloc cTPQ sum"));
    RET(cuda_ok(cudaMalloc(&CT.p, esz * dim * nb), "alloc cTPQ term"));
    RET(cuda_ok(cudaMalloc(&CU.p, esz * dim * nb), "alloc cTPQ term"));
  }
  auto ctpq_multiply = [&]() -> int {
    // x = sv V and h = H x (expec left H x in H): sum = x + a h + sum_c a^c/c! H^c x;
    // scalar slots [26, 31) (expec and the observables use [0, 22))
    const double a = -0.5 * dtau;
    RET(cuda_ok(cudaMemcpyAsync(CA.p, V.p, esz * dim * nb, cudaMemcpyDeviceToDevice, s->stream), "copy"));
    for (int b = 0; b < nb; b++) {
      RET(vec_scale(s, vt, sv[b], vec(CA.p, b)));
      RET(vec_axpby(s, vt, a, vec(H.p, b), 1.0, vec(CA.p, b)));
    }
    RET(cuda_ok(cudaMemcpyAsync(CT.p, H.p, esz * dim * nb, cudaMemcpyDeviceToDevice, s->stream), "copy"));
    double coeff = a;
    const double c01[2] = {0.0, 1.0};
    for (int b = 0; b < nb; b++)
      RET(cuda_ok(cudaMemcpyAsync(slot(b) + 26, c01, sizeof(c01), cudaMemcpyHostToDevice, s->stream), "coef"));
    for (int c = 2; c <= expand; c++) {
      coeff *= a / (double)c;
      RET(apply_h(CT.p, CU.p, 26));
      for (int b = 0; b < nb; b++) RET(vec_axpby(s, vt, coeff, vec(CU.p, b), 1.0, vec(CA.p, b)));
      std::swap(CT.p, CU.p);
    }
    for (int b = 0; b < nb; b++) RET(vec_norm2(s, vt, vec(CA.p, b), slot(b) + 30));
    RET(read_slots());
    for (int b = 0; b < nb; b++) {
      gnorm[b] = std::sqrt(host[kSlots * b + 30]);
      sv[b] = 1.0 / gnorm[b];
    }
    std::swap(V.p, CA.p);
    return 0;
  };
  auto record = [&](int b) {
    (*res)[b].energy.push_back(E[b]);
    (*res)[b].inv_temp.push_back(inv_temp[b]);
  };
  if (canonical && m.expand_coef <= 0) printf("In cTPQ calc., the default value of ExpandCoef (=10) is used. \n");
  int step = 2;
  if (resumed) {
    // expec_energy_flct on the stored state, then the loop from its step (src/CalcByTPQ.c:107-113);
    // a continued cTPQ run resumes its inverse temperature at (step - 1) dtau (the reference
    // leaves it unset on this path)
    RET(expec());
    step = opt.resume_step;
    if (canonical) inv_temp[0] = (step - 1) * dtau;
  } else if (canonical) {
    // step 0: the normalised start vector, its Green's functions, expec (with the Flct line)
    RET(expec());
    if (green) RET(green_step(0));
    for (int b = 0; b < nb; b++) {
      write_lines(b, 0.0, first_norm[b], 0, true);
      record(b);
    }
    step = 1;
  } else {
    // FirstMultiply: expec on the start vector, then v = (L - H/Ns) v normalised.
    RET(expec());
    if (green) RET(green_step(0));
    RET(multiply());
    for (int b = 0; b < nb; b++) {
      write_lines(b, 0.0, first_norm[b], 0, false);
      record(b);
    }
    RET(expec());
    for (int b = 0; b < nb; b++) {
      inv_temp[b] = (2.0 / Ns) / (L - E[b] / Ns);
      write_lines(b, inv_temp[b], gnorm[b], 1, true);
      record(b);
    }
  }
  for (; step < m.lanczos_max; step++) {
    if (canonical) {
      RET(ctpq_multiply());
      RET(expec());
      for (int b = 0; b < nb; b++) inv_temp[b] += dtau;
    } else {
      RET(multiply());
      RET(expec());
      for (int b = 0; b < nb; b++) inv_temp[b] = (2.0 * step / Ns) / (L - E[b] / Ns);
    }
    for (int b = 0; b < nb; b++) {
      write_lines(b, inv_temp[b], gnorm[b], step, true);
      record(b);
    }
    if (green && m.expec_interval > 0 && step % m.expec_interval == 0) RET(green_step(step));
  }
  for (int b = 0; b < nb; b++) {
    (*res)[b].final_step = step;
    if (opt.keep_vector) {
      // the normalised state sv*V in HPhi's order
      RET(from_native(s, vt, vec(V.p, b), vec(H.p, b)));
      (*res)[b].final_vector.assign(2 * (dim + 1), 0.0);
      RET(vec_to_host_c128(s, vt, vec(H.p, b), (*res)[b].final_vector.data()));
      RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
      for (double &x : (*res)[b].final_vector) x *= sv[b];
    }
  }
  return 0;
}

int te_run(Sector *s, const double *h_init, int step_initial, const std::string &outdir, TeResult *res) {
  const Model &m = s->model;
  const int64_t dim = s->dim;
  const VecType vt = kComplex128;
  const size_t esz = sizeof(cplx);
  if ((int)m.te_time.size() < m.lanczos_max) {
    set_error("Error: NTETimeSteps must be larger than Lanczos_max.");
    return -1;
  }
  if (m.output_eigenvec && m.output_interval <= 0) {
    set_error("OutputEigenVec in time evolution needs a positive OutputInterval");
    return -1;
  }
  RET(cuda_ok(cudaSetDevice(s->device), "cudaSetDevice"));
  // The off-diagonal terms of all time indices by their masks (the union), one split-term plan
  // for the union, and per index its coefficient table and its generic terms (back to back);
  // the diagonal terms of each index back to back.
  std::vector<BitTerm> uni;
  std::map<std::tuple<uint64_t, uint64_t, uint64_t, uint64_t>, int> where;
  const size_t nidx = m.te_time.size();
  std::vector<std::vector<std::pair<int, BitTerm>>> by_idx(nidx);
  for (size_t k = 0; k < nidx; k++)
    for (const BitTerm &t : m.te_offdiag[k]) {
      const auto key = std::make_tuple(t.cm, t.cv, t.flip, t.sm);
      auto it = where.find(key);
      if (it == where.end()) {
        it = where.emplace(key, (int)uni.size()).first;
        uni.push_back(t);
      }
      by_idx[k].push_back({it->second, t});
    }
  SplitPlan plan;
  struct PlanFree {
    SplitPlan *p;
    ~PlanFree() { split_plan_free(p); }
  } plan_free{&plan};
  std::vector<int> tab, gen_ids;
  {
    std::string err;
    if (!uni.empty() && split_plan_for_terms(s, uni, &plan, &tab, &gen_ids, &err) != 0) {
      set_error("time-evolution term plan: " + err);
      return -1;
    }
  }
  std::vector<int> tab_pos(uni.size(), -1), gen_pos(uni.size(), -1);
  for (size_t i = 0; i < tab.size(); i++) tab_pos[tab[i]] = (int)i;
  for (size_t i = 0; i < gen_ids.size(); i++) gen_pos[gen_ids[i]] = (int)i;
  const size_t ncoef = 4 * tab.size() + 2;
  std::vector<double> coefs(nidx * ncoef, 0.0);
  std::vector<BitTerm> off;
  std::vector<DiagTerm> dg;
  std::vector<size_t> off_at, dg_at;
  for (size_t k = 0; k < nidx; k++) {
    off_at.push_back(off.size());
    dg_at.push_back(dg.size());
    for (const auto &e : by_idx[k]) {
      if (tab_pos[e.first] >= 0) {
        double *c = &coefs[k * ncoef + 4 * tab_pos[e.first]];
        c[0] = e.second.re; c[1] = e.second.im; c[2] = -e.second.re; c[3] = -e.second.im;
      } else {
        off.push_back(e.second);
      }
    }
    dg.insert(dg.end(), m.te_diag[k].begin(), m.te_diag[k].end());
  }
  off_at.push_back(off.size());
  dg_at.push_back(dg.size());
  DevBuf OFF, DG, CO, P, HP, ACC, U, ST;
  if (plan.lo_ptr) {
    RET(cuda_ok(cudaMalloc(&CO.p, sizeof(double) * coefs.size()), "alloc coefficient tables"));
    RET(cuda_ok(cudaMemcpyAsync(CO.p, coefs.data(), sizeof(double) * coefs.size(), cudaMemcpyHostToDevice,
                                s->stream), "upload coefficient tables"));
  }
  if (!off.empty()) {
    RET(cuda_ok(cudaMalloc(&OFF.p, sizeof(BitTerm) * off.size()), "alloc terms"));
    RET(cuda_ok(cudaMemcpyAsync(OFF.p, off.data(), sizeof(BitTerm) * off.size(), cudaMemcpyHostToDevice, s->stream),
                "upload terms"));
  }
  if (!dg.empty()) {
    RET(cuda_ok(cudaMalloc(&DG.p, sizeof(DiagTerm) * dg.size()), "alloc terms"));
    RET(cuda_ok(cudaMemcpyAsync(DG.p, dg.data(), sizeof(DiagTerm) * dg.size(), cudaMemcpyHostToDevice, s->stream),
                "upload terms"));
  }
  for (DevBuf *b : {&P, &HP, &ACC, &U}) RET(cuda_ok(cudaMalloc(&b->p, esz * dim), "alloc vector"));
  RET(cuda_ok(cudaMalloc(&ST.p, sizeof(double) * 32), "alloc scalars"));
  double *st = (double *)ST.p;
  const double c01[2] = {0.0, 1.0};
  RET(cuda_ok(cudaMemcpyAsync(st, c01, sizeof(c01), cudaMemcpyHostToDevice, s->stream), "coef"));
  // y = H(step) x: the static part (general row kernel) plus the step's terms
  auto apply_h = [&](int step, const void *x, void *y) -> int {
    RET(hv_launch(s, vt, x, y, st, st + 2));
    return te_terms_apply(s, plan, (const double *)CO.p + (plan.lo_ptr ? step * ncoef : 0),
                          (const BitTerm *)OFF.p + off_at[step], (int)(off_at[step + 1] - off_at[step]),
                          (const DiagTerm *)DG.p + dg_at[step], (int)(dg_at[step + 1] - dg_at[step]), x, y);
  };
  RET(vec_from_host_c128(s, vt, h_init, P.p));
  // the reference's v0 (H psi of the previous step) is zero before the first step
  RET(cuda_ok(cudaMemsetAsync(HP.p, 0, esz * dim, s->stream), "zero"));
  RET(ensure_dir(outdir));
  const std::string ss_file = join(outdir, "SS.dat"), norm_file = join(outdir, "Norm.dat"),
                    flct_file = join(outdir, "Flct.dat");
  FILE *fss = fopen(ss_file.c_str(), "w"), *fnorm = fopen(norm_file.c_str(), "w"), *fflct = fopen(flct_file.c_str(), "w");
  if (!fss || !fnorm || !fflct) {
    if (fss) fclose(fss);
    if (fnorm) fclose(fnorm);
    if (fflct) fclose(fflct);
    set_error("cannot write time-evolution output files in " + outdir);
    return -1;
  }
  struct Closer {
    FILE *a, *b, *c;
    ~Closer() { fclose(a); fclose(b); fclose(c); }
  } closer{fss, fnorm, fflct};
  fprintf(fss, " # time, energy, phys_var, phys_doublon, phys_num, step_i\n");
  fprintf(fnorm, " # time, norm, step_i \n");
  fprintf(fflct, " # time, N, N^2, D, D^2, Sz, Sz^2, step_i \n");
  const bool green = !m.green_one.empty() || !m.green_two.empty() || !m.green_three.empty() ||
                     !m.green_four.empty() || !m.green_six.empty();
  std::vector<double> host;
  auto write_state = [&](int step, int label) -> int {
    // <head>_eigenvec_<label>_rank_0.dat: int step, long dim, complex128[dim + 1]
    host.assign(2 * (dim + 1), 0.0);
    RET(vec_to_host_c128(s, vt, P.p, host.data()));
    char name[256];
    snprintf(name, sizeof(name), "%s_eigenvec_%d_rank_%d.dat", m.data_head.c_str(), label, 0);
    FILE *f = fopen(join(outdir, name).c_str(), "wb");
    if (!f) { set_error(std::string("cannot write ") + name); return -1; }
    const long ld = (long)dim;
    fwrite(&step, sizeof(int), 1, f);
    fwrite(&ld, sizeof(long), 1, f);
    fwrite(host.data(), sizeof(double), host.size(), f);
    fclose(f);
    return 0;
  };
  res->time.clear();
  res->energy.clear();
  res->norm.clear();
  const std::complex<double> mi(0.0, -1.0);
  int step = step_initial;
  for (; step < m.lanczos_max; step++) {
    const double time = m.te_time[step];
    const double dt = step == 0 ? 0.0 : m.te_time[step] - m.te_time[step - 1];
    // MultiplyForTEM: psi <- (psi - i dt H' psi + sum_{k=2}^{ExpandCoef} (-i dt)^k / k! H^k psi) / |.|
    // where H' psi is the previous step's H psi; a step with dt < 1e-14 keeps psi
    if (dt >= 1e-14) {
      RET(cuda_ok(cudaMemcpyAsync(ACC.p, P.p, esz * dim, cudaMemcpyDeviceToDevice, s->stream), "copy"));
      std::complex<double> coef = mi * dt;
      RET(vec_caxpy(s, coef.real(), coef.imag(), HP.p, ACC.p));
      void *t = HP.p, *u = U.p;
      for (int k = 2; k <= m.expand_coef; k++) {
        coef *= mi * dt / (double)k;
        RET(apply_h(step, t, u));
        RET(vec_caxpy(s, coef.real(), coef.imag(), u, ACC.p));
        std::swap(t, u);
      }
      std::swap(P.p, ACC.p);
    }
    RET(vec_norm2(s, vt, P.p, st + 4));
    double n2 = 0.0;
    RET(cuda_ok(cudaMemcpyAsync(&n2, st + 4, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "read"));
    RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
    const double gnorm = std::sqrt(n2);
    RET(vec_scale(s, vt, 1.0 / gnorm, P.p));
    // expec_energy_flct: observables of psi, H psi with this step's terms, E, var
    RET(vec_diag_observables(s, vt, P.p, st + 16));
    RET(apply_h(step, P.p, HP.p));
    RET(vec_dot(s, vt, P.p, HP.p, st + 6));
    RET(vec_norm2(s, vt, HP.p, st + 8));
    double sc[4], ob[6];
    RET(cuda_ok(cudaMemcpyAsync(sc, st + 6, sizeof(sc), cudaMemcpyDeviceToHost, s->stream), "read"));
    RET(cuda_ok(cudaMemcpyAsync(ob, st + 16, sizeof(ob), cudaMemcpyDeviceToHost, s->stream), "read"));
    RET(cuda_ok(cudaStreamSynchronize(s->stream), "sync"));
    const double E = sc[0], var = sc[2];
    fprintf(fss, "%.16lf  %.16lf %.16lf %.16lf %.16lf %d\n", time, E, var, ob[0], ob[2], step);
    fprintf(fnorm, "%.16lf %.16lf %d\n", time, gnorm, step);
    fprintf(fflct, "%.16lf %.16lf %.16lf %.16lf %.16lf %.16lf %.16lf %d\n", time, ob[2], ob[3], ob[0], ob[1], ob[4],
            ob[5], step);
    fflush(fss);
    fflush(fnorm);
    fflush(fflct);
    res->time.push_back(time);
    res->energy.push_back(E);
    res->norm.push_back(gnorm);
    if (green && m.expec_interval > 0 && step % m.expec_interval == 0) {
      GreenValues g;
      RET(model_green(s, vt, P.p, 1.0, &g));
      char suffix[64];
      snprintf(suffix, sizeof(suffix), "_step%d", step);
      RET(write_green_files(m, g, outdir, suffix));
    }
    if (m.output_eigenvec && step % m.output_interval == 0) RET(write_state(step, step));
  }
  res->final_step = step;
  if (m.output_eigenvec) RET(write_state(step, 0));
  return 0;
}

}  // namespace hphi
