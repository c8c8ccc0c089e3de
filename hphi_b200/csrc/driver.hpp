// Lanczos / TPQ drivers over a device Sector.
#pragma once
#include <complex>
#include <string>
#include <vector>

#include "engine.hpp"

namespace hphi {

// Lanczos restart data in HPhi's files (src/Lanczos_EigenValue.c:419-500, 620-720):
// zvo_TMComponents.dat holds the step count, dnorm and alpha_i, beta_i printed with 10
// decimals; zvo_recalcvec_rank_0.dat the step, dim and HPhi's v0 and v1 (1-based complex128)
// of the last step: v1 = q_n, v0 = H q_n - beta_{n-1} q_{n-1}.
struct LanczosRestart {
  int steps = 0;                     // alpha / beta entries
  int vec_steps = 0;                 // step recorded with the vectors
  double dnorm = 0.0;
  std::vector<double> alpha, beta;   // [1 .. steps] (index 0 unused)
  std::vector<double> v0, v1;        // 2 * (dim + 1) doubles each
};

struct LanczosOptions {
  bool eigenvector = false;       // replay the recurrence for the k_exct-th eigenvector
  bool copy_eigenvector = false;  // copy it back to the host (HPhi layout)
  int batch = 0;                  // steps between host convergence checks (0: automatic)
  int fixed_steps = 0;            // > 0: exactly this many steps, convergence test off
  bool restart_out = false;       // fill LanczosResult::restart (ReStart 1 / 2); then a run
                                  // that does not converge is not an error
  const LanczosRestart *resume = nullptr;  // continue from these (ReStart 2 / 3)
  bool hashed_start = false;      // start from the hashed vector of hashed_seed, made on the
  uint64_t hashed_seed = 0;       // device (h_init is not read)
  const void *device_start = nullptr;  // start from this normalised device vector in HPhi's order
};

// Green's function values of the model's OneBodyG / TwoBodyG rows (expec_cisajs,
// src/expec_cisajs.c:66-641; expec_cisajscktaltdc, src/expec_cisajscktaltdc.c:87-1647):
// (re, im) per row, with the reference's line endings of the two-body rows.
struct GreenValues {
  std::vector<double> one, two;
  std::vector<char> trail_two;
  std::vector<double> multi[3];       // three-, four- and six-body rows
  std::vector<char> multi_short[3];   // rows the reference prints with 8 indices
};

// The model's Green's functions of the vector d_hphi (device, HPhi row order), multiplied
// by `scale`; nothing when the model requests none.
int model_green(Sector *s, VecType vt, const void *d_hphi, double scale, GreenValues *g);
// One Green's function file (kind 1, 2, 3, 4, 6) in the reference's format at `path`.
int write_green_file(const Model &m, const GreenValues &g, int kind, const std::string &path);
// Every requested Green's function file in dir: <head>_cisajs<suffix>.dat,
// <head>_cisajscktalt<suffix>.dat, <head>_ThreeBody<suffix>.dat, ... (src/global.c:43-89;
// suffix "" for Lanczos, "_set%dstep%d" for TPQ, "_eigen%d" for LOBPCG).  A file whose rows
// were not requested is not written (src/expec_cisajs.c:80, src/expec_cisajscktaltdc.c:102),
// except that the two-body file exists whenever any of the two-, three-, four- or six-body
// lists is requested (src/expec_cisajscktaltdc.c:102-180).
int write_green_files(const Model &m, const GreenValues &g, const std::string &dir, const std::string &suffix);

struct LanczosResult {
  bool converged = false;
  int steps = 0;                     // X->Large.itr
  double e_target = 0.0;             // X->Phys.Target_energy
  double e_tridiag = 0.0;            // eigenvalue used for the eigenvector (Target_CG_energy)
  std::vector<double> alpha, beta;   // alpha[0..steps), beta[0..steps)
  std::vector<double> energies;      // lowest eigenvalues of the final tridiagonal matrix
  std::vector<std::string> lines;    // zvo_Lanczos_Step.dat
  bool resumed = false;              // continued from restart files (step lines are appended)
  bool has_restart = false;          // restart files to write (restart_out)
  LanczosRestart restart;
  double energy = 0.0, var = 0.0, doublon = 0.0, sz = 0.0;
  // accuracy check of the Lanczos vector (src/CalcByLanczos.c:120-121) and, when it fails
  // with CalcEigenVec 0, the CG refinement (src/CG_EigenVector.c): relative variance and
  // energy difference before / after, inverse-iteration rounds and total CG iterations
  double check_var = 0.0, check_diff = 0.0, cg_var = 0.0, cg_diff = 0.0;
  bool cg_ran = false;
  int cg_rounds = 0, cg_iterations = 0;
  std::vector<double> eigenvector;   // 1-based complex128 (HPhi layout) when requested
  GreenValues green;                 // of the eigenvector (src/CalcByLanczos.c:229-240)
  bool from_input = false;           // InputEigenVec: no Lanczos run, no step file
};

// CalcByLanczos with InputEigenVec 1 or 2 (src/CalcByLanczos.c:160-225): the vector stored in
// <outdir>/<head>_eigenvec_<exct-1>_rank_0.dat replaces the Lanczos run (mode 2 takes
// H v / |H v|); its Green's functions and Sz follow.  Energy and Doublon are not computed
// on this path (they print as 0, as in the reference).
int lanczos_input_vector(Sector *s, VecType vt, const std::string &outdir, int mode, LanczosResult *res);

struct LobpcgResult {
  bool converged = false;
  bool copy_vectors = false;         // copy the eigenvectors back (HPhi layout, exct blocks)
  bool phys_only = false;            // InputEigenVec: the start block is the result (no iteration, no step file)
  int steps = 0;                     // steps run (at most Lanczos_max)
  int itr = 0;                       // X->Large.itr: the loop counter (Lanczos_max + 1 when unconverged)
  double residual = 0.0;             // largest residual 2-norm of the last step
  std::vector<double> eig;           // LOBPCG eigenvalue estimates of the last step
  std::vector<double> energy, var, doublon, sz;  // phys() of each converged vector
  std::vector<std::string> lines;    // zvo_Lanczos_Step.dat
  std::vector<double> eigenvectors;  // exct x (dim + 1) complex128 when copy_vectors
  std::vector<GreenValues> green;    // of each vector (phys, src/phys.c:100-110)
};

struct TpqResult {
  std::vector<double> inv_temp, energy;
  int final_step = 0;                // step_i after the loop (the restart file's step)
  std::vector<double> final_vector;  // the last state (HPhi layout) when TpqOptions::keep_vector
};

// TPQ restart (ReStart, src/CalcByTPQ.c:86-110, 275-290): resume_step > 0 continues from a
// stored state (h_init) at that step, appending to the sample's files; keep_vector returns
// the last state for tmpvec_set%d_rank_%d.dat.
struct TpqOptions {
  int resume_step = 0;
  bool keep_vector = false;
};

// Real-time evolution (CalcType 4, CalcByTEM src/CalcByTEM.c:52-234): per step the state
// is advanced by the Taylor sum of exp(-i dt H) (MultiplyForTEM src/Multiply.c:79-139),
// normalised, and measured (SS.dat, Norm.dat, Flct.dat, Green's function files every
// ExpecInterval steps, eigenvector files every OutputInterval steps with OutputEigenVec).
struct TeResult {
  std::vector<double> time, energy, norm;
  int final_step = 0;
};

// Dynamical Green's function (spectrum.cu): the frequencies (omega, OmegaOrg included), the
// Green's function on them, the excited state's norm and the Lanczos components a[1..steps],
// b[1..steps].
struct SpectrumResult {
  std::vector<std::complex<double>> omega, green;
  double dnorm = 0.0;
  int steps = 0;
  std::vector<double> alpha, beta;
};
// CalcSpectrum with CalcSpec 1 and the Lanczos method for the input vector h_vec (HPhi's
// 1-based complex128 layout, org's sector); writes the output files to outdir.
int spectrum_run(Sector *org, const double *h_vec, const std::string &outdir, SpectrumResult *res);

// k-th smallest eigenvalue (0-based) of the symmetric tridiagonal matrix with diagonal
// a[0..n) and off-diagonal b[0..n-1), by Sturm bisection; its eigenvector by inverse iteration.
double tridiag_eigenvalue(const double *a, const double *b, int n, int k);
void tridiag_eigenvector(const double *a, const double *b, int n, double lam, std::vector<double> *out);

VecType default_vec_type(const Sector &s);
bool single_element_start(const Sector &s, std::vector<double> *v);
void random_start(const Sector &s, uint64_t seed, bool complex_vec, std::vector<double> *v);

// h_init: normalised start vector in HPhi's 1-based complex128 layout (not read when
// opt.hashed_start is set).
int lanczos_run(Sector *s, VecType vt, const double *h_init, const LanczosOptions &opt, LanczosResult *res);
int write_lanczos_outputs(const Sector &s, const LanczosResult &r, const std::string &outdir);
int write_lanczos_restart(const Sector &s, const LanczosRestart &r, const std::string &outdir);
int read_lanczos_restart(const Sector &s, const std::string &outdir, LanczosRestart *r);
// h_init: start vector (any norm) of sample rand_i; writes SS/Norm/Flct_rand<rand_i>.dat.
int tpq_run(Sector *s, VecType vt, const double *h_init, int rand_i, const std::string &outdir, TpqResult *res,
            const TpqOptions &opt = TpqOptions());
// Several TPQ samples in lockstep (rand_i[b] from start h_init[b]), with every H application
// of a step one block H*V over the samples when `block` (hv_block_applies, at most
// kHvBlockMax samples), else one launch per sample.  Output files and results per sample are
// those of tpq_run; resume_step > 0 takes a single sample.
int tpq_run_samples(Sector *s, VecType vt, const std::vector<const double *> &h_init, const std::vector<int> &rand_i,
                    const std::string &outdir, std::vector<TpqResult> *res, const TpqOptions &opt, bool block);
// h_init: the input state (SpectrumVec file contents, HPhi's 1-based complex128 layout);
// step_initial: the first time index (the file's step on a ReStart 2 / 3 run, else 0).
int te_run(Sector *s, const double *h_init, int step_initial, const std::string &outdir, TeResult *res);
// Block LOBPCG for the exct lowest states (CalcType 3).  h_init: exct start vectors in
// HPhi's 1-based complex128 layout, back to back (any norm).
bool lobpcg_single_element_start(const Sector &s, std::vector<double> *v);
int lobpcg_run(Sector *s, VecType vt, const double *h_init, LobpcgResult *res);
int write_lobpcg_outputs(const Sector &s, const LobpcgResult &r, const std::string &outdir);

}  // namespace hphi
