// Dynamical Green's function by the Lanczos method (CalcSpec 1):
// replaces CalcSpectrum (src/CalcSpectrum.c:90-312) with CalcSpectrumByLanczos
// (src/CalcSpectrumByLanczos.c:43-219) for an input vector, single or pair excitation
// operators and the Lanczos tridiagonal components.
//
//   1. The input vector <SpectrumVec>_rank_0.dat (a state of the original sector) is read and
//      the excitation operators are applied: v_ex = sum_k A_k v (GetExcitedState, :315-345),
//      in gather form on the excited sector's rows (a configuration c' gets
//      coef * sign * v[row of c' ^ flip in the original sector] per operator that applies),
//      one thread per row, so no two threads write one element.
//   2. dnorm = |v_ex|; a vector of norm < 1e-15 gives a zero spectrum (:184-195).
//   3. The Lanczos recurrence from v_ex / dnorm for Lanczos_max steps, capped at the sector's
//      dimension and stopped when beta < 1e-14 (Lanczos_GetTridiagonalMatrixComponents,
//      src/Lanczos_EigenValue.c:324-414), runs on the excited sector's H*v kernels.
//   4. G(omega) = dnorm^2 / (omega - a_1 - b_1^2 / (omega - a_2 - ...)) on the frequency grid,
//      evaluated as the reference does (GetSpectrumByTridiagonalMatrixComponents,
//      src/CalcSpectrumByLanczos.c:169-219: the same recursion, the same eps_Energy guard and
//      stopping rule, a_{L+1} = 0 past the computed components).
//   5. <head>_TMComponents.dat and <head>_DynamicalGreen.dat in the reference's formats
//      (OutputTMComponents, src/Lanczos_EigenValue.c:697-720; OutputSpectrum,
//      src/CalcSpectrum.c:49-73), <head>_excitedvec_rank_0.dat when OutputExVec is set.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <string>
#include <vector>

#include "device_util.cuh"
#include "driver.hpp"
#include "engine.hpp"

namespace hphi {
namespace {

constexpr int kExThreads = 256;

// v_ex[r] = sum over the operators of coef * (-1)^popcount(c & sm) * v[row_org(c ^ flip)],
// c the configuration of excited row r (row = configuration for grand-canonical sectors).
__global__ void excite_kernel(int64_t dim_ex, int gc, const uint64_t *__restrict__ list_1_ex,
                              const uint32_t *__restrict__ l21_org, const uint32_t *__restrict__ l22_org,
                              int lo_bits, uint64_t lo_mask, const BitTerm *__restrict__ ops, int nops,
                              const cplx *__restrict__ v_org, cplx *__restrict__ v_ex) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < dim_ex; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = gc ? (uint64_t)r : list_1_ex[r];
    cplx y{0.0, 0.0};
    for (int k = 0; k < nops; k++) {
      const BitTerm t = ops[k];
      if ((c & t.cm) != t.cv) continue;
      const uint64_t s = c ^ t.flip;
      int64_t j;
      if (gc) {
        j = (int64_t)s;
      } else {
        const uint32_t a = l21_org[s & lo_mask], b = l22_org[s >> lo_bits];
        if (a == 0u || b == 0u) continue;
        j = (int64_t)a + (int64_t)b - 3;
      }
      const bool neg = __popcll(c & t.sm) & 1;
      y = y + VT<cplx>::cmul_re_im(neg ? -t.re : t.re, neg ? -t.im : t.im, v_org[j]);
    }
    v_ex[r] = y;
  }
}

struct Dev {
  void *p = nullptr;
  ~Dev() { if (p) cudaFree(p); }
};

int ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    set_error(std::string("spectrum: ") + what + ": " + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

// GetSpectrumByTridiagonalMatrixComponents (src/CalcSpectrumByLanczos.c:169-219) with 1-based
// a, b of L components; the caller multiplies by dnorm once more, as CalcSpectrumByLanczos
// does (:143-151).
std::complex<double> continued_fraction(const std::vector<double> &a, const std::vector<double> &b, int L,
                                        double dnorm, std::complex<double> w) {
  const double eps_energy = 1e-12, eps = 1e-8;  // SetConvergenceFactor, src/readdef.c:2695-2708
  auto A = [&](int i) { return (i <= L) ? a[i] : 0.0; };  // components past L: zero (calloc)
  const std::complex<double> b0 = w - A(1);
  if (L == 1) {
    std::complex<double> d = b0;
    if (std::abs(d) < eps_energy) d = eps_energy;
    return dnorm / d;
  }
  std::complex<double> bn = w - A(2);
  std::complex<double> an = -b[1] * b[1];
  std::complex<double> dn = 1.0 / bn;
  std::complex<double> dh = an * dn;
  std::complex<double> h = b0 + dh;
  for (int stp = 2; stp <= L; stp++) {
    bn = w - A(stp + 1);
    an = -b[stp] * b[stp];
    dn = bn + an * dn;
    if (std::abs(dn) < eps_energy) dn = eps_energy;
    dn = 1.0 / dn;
    dh = (bn * dn - 1.0) * dh;
    h += dh;
    if (std::abs(dh / h) < std::abs(b0) * eps) break;
  }
  return dnorm / h;
}

// SetOmega (src/CalcSpectrum.c:353-436) for a Lanczos run: OmegaMin = E1 and OmegaMax =
// Nsite times the fifth value of the last line of <head>_Lanczos_Step.dat (the target energy
// column, as the reference's sscanf reads it) when modpara leaves them unset.
int set_omega(const Model &m, const std::string &outdir, std::complex<double> *wmax, std::complex<double> *wmin) {
  *wmax = {m.omega_max[0], m.omega_max[1]};
  *wmin = {m.omega_min[0], m.omega_min[1]};
  if (m.omega_max_set && m.omega_min_set) return 0;
  const std::string path = outdir + "/" + m.data_head + "_Lanczos_Step.dat";
  FILE *f = fopen(path.c_str(), "r");
  if (!f) {
    set_error("Error: xx_Lanczos_Step.dat does not exist.");
    return -1;
  }
  char line[512];
  std::vector<std::string> lines;
  while (fgets(line, sizeof(line), f)) lines.push_back(line);
  fclose(f);
  int istp = 0;
  double e[5];
  int got = (lines.size() >= 3) ? sscanf(lines.back().c_str(), "stp=%d %lf %lf %lf %lf %lf", &istp, &e[0], &e[1], &e[2],
                                         &e[3], &e[4])
                                : 0;
  if (got < 2 || istp < 4) {
    set_error("Error: Lanczos step must be greater than 4 for using spectrum calculation.");
    return -1;
  }
  if (!m.omega_max_set) {
    if (got < 6) {
      set_error("spectrum: the last line of the Lanczos step file has no target energy for OmegaMax");
      return -1;
    }
    *wmax = e[4] * (double)m.nsite;
  }
  if (!m.omega_min_set) *wmin = e[0];
  return 0;
}

}  // namespace

int spectrum_run(Sector *org, const double *h_vec, const std::string &outdir, SpectrumResult *res) {
  const Model &m = org->model;
  if (m.excitation.empty() && m.n_single_ex == 0 && m.n_pair_ex == 0) {
    set_error("Error: Any excitation operators are not defined.");
    return -1;
  }
  std::complex<double> wmax, wmin;
  if (set_omega(m, outdir, &wmax, &wmin) != 0) return -1;
  std::complex<double> worg{m.omega_org[0], m.omega_org[1]};
  if (!m.omega_org_set) worg = std::complex<double>(0.0, 1.0) * (wmax - wmin) / (double)m.n_omega;
  const int nw = m.n_omega;
  if (nw < 1) {
    set_error("spectrum: NOmega must be positive");
    return -1;
  }
  // the excited sector (MakeExcitedList, src/CalcSpectrum.c:438-634)
  Sector *ex = org;
  Sector *owned = nullptr;
  if (!m.is_gc() && (m.ex_nup != m.nup || m.ex_ndown != m.ndown || m.ex_ne != m.ne)) {
    Model mx = m;
    mx.nup = m.ex_nup;
    mx.ndown = m.ex_ndown;
    mx.ne = m.ex_ne;
    mx.total_2sz = m.ex_2sz;
    if (mx.nup < 0 || mx.ndown < 0 || mx.nup > m.nsite || mx.ndown > m.nsite) {
      set_error("spectrum: the excited state leaves every sector");
      return -1;
    }
    std::string err;
    if (sector_build(mx, org->device, &owned, &err) != 0) {
      sector_free(owned);
      set_error("spectrum: excited sector: " + err);
      return -1;
    }
    ex = owned;
  }
  struct Guard {
    Sector *s;
    ~Guard() { if (s) sector_free(s); }
  } guard{owned};
  const int64_t dim0 = org->dim, dim1 = ex->dim;
  Dev V0, V1, OPS;
  if (ck(cudaSetDevice(org->device), "device") || ck(cudaMalloc(&V0.p, sizeof(cplx) * dim0), "alloc") ||
      ck(cudaMalloc(&V1.p, sizeof(cplx) * dim1), "alloc") ||
      ck(cudaMalloc(&OPS.p, sizeof(BitTerm) * m.excitation.size() + 16), "alloc"))
    return -1;
  if (vec_from_host_c128(org, kComplex128, h_vec, V0.p) != 0) return -1;
  if (ck(cudaMemcpyAsync(OPS.p, m.excitation.data(), sizeof(BitTerm) * m.excitation.size(), cudaMemcpyHostToDevice,
                         org->stream),
         "copy operators"))
    return -1;
  // the excited sector's kernels run on its own stream: order them after the upload
  if (ck(cudaStreamSynchronize(org->stream), "sync")) return -1;
  const unsigned nb = (unsigned)std::min<int64_t>((dim1 + kExThreads - 1) / kExThreads, (int64_t)ex->num_sms * 16);
  excite_kernel<<<nb, kExThreads, 0, ex->stream>>>(dim1, ex->gc ? 1 : 0, ex->d_list_1, org->d_list_2_1, org->d_list_2_2,
                                                   org->lo_bits, org->ihfbit - 1, (const BitTerm *)OPS.p,
                                                   (int)m.excitation.size(), (const cplx *)V0.p, (cplx *)V1.p);
  if (ck(cudaGetLastError(), "excitation kernel")) return -1;
  if (vec_norm2(ex, kComplex128, V1.p, ex->d_scal) != 0) return -1;
  double n2 = 0.0;
  if (ck(cudaMemcpyAsync(&n2, ex->d_scal, sizeof(double), cudaMemcpyDeviceToHost, ex->stream), "norm") ||
      ck(cudaStreamSynchronize(ex->stream), "sync"))
    return -1;
  const double dnorm = std::sqrt(n2);
  res->dnorm = dnorm;
  res->omega.assign(nw, 0.0);
  res->green.assign(nw, 0.0);
  const std::complex<double> wmax_o = wmax + worg, wmin_o = wmin + worg;
  for (int i = 0; i < nw; i++) res->omega[i] = (wmax_o - wmin_o) / (double)nw * (double)i + wmin_o;
  if (m.output_exvec == 1 && dnorm >= 1e-15) {
    std::vector<double> h(2 * (dim1 + 1), 0.0);
    if (vec_to_host_c128(ex, kComplex128, V1.p, h.data()) != 0) return -1;
    char name[512];
    snprintf(name, sizeof(name), "%s/%s_excitedvec_rank_%d.dat", outdir.c_str(), m.data_head.c_str(), 0);
    FILE *f = fopen(name, "w");
    if (!f) { set_error(std::string("cannot write ") + name); return -1; }
    fprintf(f, "%ld\n", (long)dim1);
    for (int64_t i = 1; i <= dim1; i++) fprintf(f, "%.10lf, %.10lf\n", h[2 * i], h[2 * i + 1]);
    fclose(f);
  }
  res->steps = 0;
  if (dnorm >= 1e-15) {
    if (vec_scale(ex, kComplex128, 1.0 / dnorm, V1.p) != 0) return -1;
    LanczosOptions opt;
    opt.fixed_steps = std::max(1, (int)std::min<int64_t>(m.lanczos_max, dim1));
    opt.device_start = V1.p;
    LanczosResult lr;
    if (lanczos_run(ex, kComplex128, nullptr, opt, &lr) != 0) return -1;
    const int L = lr.steps;
    res->steps = L;
    res->alpha.assign(L + 2, 0.0);
    res->beta.assign(L + 2, 0.0);
    for (int i = 1; i <= L; i++) {
      res->alpha[i] = lr.alpha[i - 1];
      res->beta[i] = lr.beta[i - 1];
    }
    for (int i = 0; i < nw; i++) res->green[i] = dnorm * continued_fraction(res->alpha, res->beta, L, dnorm, res->omega[i]);
    char name[512];
    snprintf(name, sizeof(name), "%s/%s_TMComponents.dat", outdir.c_str(), m.data_head.c_str());
    FILE *f = fopen(name, "w");
    if (!f) { set_error(std::string("cannot write ") + name); return -1; }
    fprintf(f, "%d \n", L);
    fprintf(f, "%.10lf \n", dnorm);
    for (int i = 1; i <= L; i++) fprintf(f, "%.10lf %.10lf \n", res->alpha[i], res->beta[i]);
    fclose(f);
  }
  char name[512];
  snprintf(name, sizeof(name), "%s/%s_DynamicalGreen.dat", outdir.c_str(), m.data_head.c_str());
  FILE *f = fopen(name, "w");
  if (!f) { set_error(std::string("cannot write ") + name); return -1; }
  for (int i = 0; i < nw; i++) {
    const std::complex<double> w = res->omega[i] - worg;
    fprintf(f, "%.10lf %.10lf %.10lf %.10lf \n", w.real(), w.imag(), res->green[i].real(), res->green[i].imag());
  }
  fclose(f);
  return 0;
}

}  // namespace hphi
