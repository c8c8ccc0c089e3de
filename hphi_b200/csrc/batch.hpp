// Batched Lanczos: many independent sectors advanced together by one persistent kernel
// per phase, with FP64 or FP32 vector storage, and the request server built on it.
//
// The reference solves one Hamiltonian per process (CalcByLanczos,
// src/CalcByLanczos.c:55-276, over Lanczos_EigenValue, src/Lanczos_EigenValue.c:50-310);
// this engine runs the same two-vector recurrence for every instance at once:
//   hv phase:    P_i <- acc_i P_i + s_i H_i Q_i,   alpha_i,k = s_i^2 <Q_i|H_i Q_i>
//   sweep phase: P_i <- P_i - alpha_i,k s_i Q_i,   beta_i,k = |P_i|,  s_i <- 1/beta_i,k
// Each phase is one launch over a table of row tiles of all member instances; the CTA
// that finishes an instance's last tile reduces its partial sums (in tile order, so the
// result does not depend on scheduling or on the other members) and updates that
// instance's scalars on the device.  Every instance carries its own mode (start vector,
// forward recurrence, replay, FP64 refinement), so instances at different stages share
// the same launches; members can join and leave between launches.
//
// FP32 storage keeps P, Q and the start vector in float (float2 for complex) and computes
// every row sum, dot product and update in FP64 registers; the ground state is rebuilt by
// replaying the recurrence into an FP64 vector (as Lanczos_EigenVector,
// src/Lanczos_EigenVector.c:46-208), and a final FP64 H*v gives its Rayleigh quotient and
// the residual |H x - E x| / |x|.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "engine.hpp"

namespace hphi {

enum Precision : int { kFP64 = 0, kFP32 = 1 };

// Launch shape of the persistent kernels.  threads * rows_per_thread fixes how an instance
// is cut into tiles, and with it the summation order of its dot products.
struct BatchTuning {
  int threads = 256;         // CTA size
  int rows_per_thread = 8;   // a tile is threads * rows_per_thread consecutive rows
  int ctas_per_sm = 8;       // persistent grid = ctas_per_sm * SMs (capped by the tile count)
  float hv_ms = 0.0f;        // measured time of one hv phase with this shape
};

struct BatchResult {
  std::vector<double> e_lanczos;   // lowest eigenvalue of each instance's tridiagonal matrix
  std::vector<int> steps;          // Lanczos steps used (fewer than asked after a breakdown)
  std::vector<double> e_refined;   // FP64 Rayleigh quotient of the rebuilt ground state
  std::vector<double> residual;    // |H x - E x| / |x| of that vector, in FP64
  std::vector<int> replay_steps;   // steps replayed to rebuild it
  double forward_ms = 0.0, replay_ms = 0.0, refine_ms = 0.0;
  BatchTuning tuning;
};

struct Batch;

// ---- fixed batch: the caller's sectors (must outlive the batch), all on one device.
int batch_create(const std::vector<Sector *> &sectors, Precision prec, Batch **out);
// `steps` Lanczos steps for every instance from the hashed start vector (start_value) of
// seed + 1000003 * i; with `refine`, rebuild each ground state and refine it in FP64,
// replaying until the rest of the Ritz vector has norm below replay_tol.  use_graph
// captures the iterations in CUDA graphs.
int batch_lanczos(Batch *b, int steps, uint64_t seed, bool use_graph, bool refine, double replay_tol,
                  BatchResult *res);
// Chooses the launch shape by timing candidate shapes on the current members (cached per
// member signature); batch_lanczos calls it on first use.
int batch_autotune(Batch *b, bool force);
const BatchTuning &batch_tuning(const Batch *b);
void batch_free(Batch *b);
int batch_size(const Batch *b);

// ---- request server (continuous batching over the same engine).
struct Server;
struct ServeResult {
  int64_t id = -1;
  int status = 0;                  // 0 converged, 1 stopped at Lanczos_max, -1 failed
  double energy = 0.0;             // refined energy (FP32 storage) or the Lanczos eigenvalue
  double e_lanczos = 0.0, residual = 0.0;
  int steps = 0;
  int64_t dim = 0;
  double t_wait = 0.0, t_latency = 0.0;  // seconds from arrival to admission / to completion
  std::string error;
};
int server_create(int device, Precision prec, int64_t hbm_budget, int max_active, int steps_per_iteration,
                  Server **out);
// Parses the expert-mode input on the host and queues it; arrival < 0 means now (seconds on
// server_clock()).
int server_submit(Server *s, const std::string &namelist, uint64_t seed, double arrival, int64_t *id);
// Admits queued requests that fit (slots and HBM budget), advances every member by one
// iteration, retires finished ones.  counts: active, queued, finished-not-polled.
int server_step(Server *s, int64_t counts[3]);
bool server_poll(Server *s, ServeResult *out);
double server_clock();
void server_free(Server *s);

// Start-vector element of configuration `config` for `seed`: uniform in [-0.5, 0.5),
// part 0 real, part 1 imaginary.  Keyed by configuration, so any vector order gives the
// same vector.
__host__ __device__ inline double start_value(uint64_t seed, uint64_t config, int part) {
  uint64_t x = seed * 0x9E3779B97F4A7C15ull + (config * 2 + (uint64_t)part + 1) * 0xD1B54A32D192ED03ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (double)(x >> 11) * (1.0 / 9007199254740992.0) - 0.5;
}

}  // namespace hphi
