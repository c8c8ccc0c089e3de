// The reference's random start vectors, reproduced on the host.
//
// HPhi draws its random start vectors from dSFMT (double-precision SIMD-oriented Fast
// Mersenne Twister, Saito & Matsumoto; the MEXP = 19937 parameter set, vendored as
// src/dSFMT.c with src/include/dSFMT-params19937.h).  Each OpenMP thread seeds its own
// generator and fills its share of the rows under `#pragma omp for` (static schedule), so
// the vector depends on the thread count; given that count these functions give the same
// vector.
//   Lanczos  SetInitialVector   src/Lanczos_EigenValue.c:556-610  seed 123432 + |iv| + thread
//   TPQ      MakeIniVec         src/MakeIniVec.c:41-117           seed 123432 + (sample+1)|iv| + thread
//   LOBPCG   Initialize_wave    src/CalcByLOBPCG.c:252-290        seed 123432 + |iv| + thread, k vectors
#pragma once

#include <cstdint>
#include <vector>

namespace hphi {

// dSFMT with the MEXP = 19937 parameters: genrand_close_open() returns uniform doubles in [0, 1).
class Dsfmt19937 {
 public:
  explicit Dsfmt19937(uint32_t seed);
  double genrand_close_open();

 private:
  static constexpr int kN = 191;  // (19937 - 128) / 104 + 1 128-bit words
  void next_block();
  uint64_t st_[2 * (kN + 1)];     // kN words of state + the "lung" word
  int idx_;
};

enum RefStartKind { kRefLanczos = 0, kRefTPQ = 1, kRefLOBPCG = 2 };

// Rows [begin, end) (0-based) that OpenMP's static schedule gives thread t of `threads`
// for a loop over n rows.
void omp_static_chunk(int64_t n, int threads, int t, int64_t *begin, int64_t *end);

// The reference's normalised random start vector(s) in HPhi's 1-based complex128 layout:
// `count` vectors of dim + 1 complex numbers each (count = k_exct for LOBPCG, else 1).
// vec_type: HPhi's InitialVecType (0 complex, 1 real; -1 Gaussian complex for TPQ).
void reference_random_start(int64_t dim, RefStartKind kind, int initial_iv, int sample, int vec_type, int threads,
                            int count, std::vector<double> *out);

}  // namespace hphi
