// The reference's random start vectors (see refrand.hpp).
//
// dSFMT-19937 restated from the published algorithm (Saito & Matsumoto, "SIMD-oriented
// Fast Mersenne Twister", double-precision variant) with the parameter set the reference
// builds (src/include/dSFMT-params19937.h): a 192-word state of 128-bit words, 191 of them
// holding IEEE doubles in [1, 2) and one "lung" word; every block of 382 outputs comes from
// the recursion over the 191 words (src/dSFMT.c:154-174 recursion, :510-525 block).
#include "refrand.hpp"

#include <cmath>
#include <cstdlib>
#include <cstring>

namespace hphi {
namespace {
constexpr int kPos1 = 117, kSl1 = 19, kSr = 12;
constexpr uint64_t kMsk1 = 0x000ffafffffffb3full, kMsk2 = 0x000ffdfffc90fffdull;
constexpr uint64_t kFix1 = 0x90014964b32f4329ull, kFix2 = 0x3b8d12ac548a7c7aull;
constexpr uint64_t kPcv1 = 0x3d84e1ac0dc82880ull, kPcv2 = 0x0000000000000001ull;
constexpr uint64_t kLowMask = 0x000FFFFFFFFFFFFFull, kHighConst = 0x3FF0000000000000ull;
}  // namespace

Dsfmt19937::Dsfmt19937(uint32_t seed) {
  // 32-bit linear-congruential fill of the whole state (dsfmt_chk_init_gen_rand,
  // src/dSFMT.c:625-645), read as little-endian 64-bit words
  constexpr int n32 = (kN + 1) * 4;
  uint32_t w[n32];
  w[0] = seed;
  for (int i = 1; i < n32; i++) w[i] = 1812433253u * (w[i - 1] ^ (w[i - 1] >> 30)) + (uint32_t)i;
  for (int j = 0; j < 2 * (kN + 1); j++) st_[j] = (uint64_t)w[2 * j] | ((uint64_t)w[2 * j + 1] << 32);
  // the 191 working words become doubles in [1, 2) (initial_mask, src/dSFMT.c:429-437)
  for (int j = 0; j < 2 * kN; j++) st_[j] = (st_[j] & kLowMask) | kHighConst;
  // period certification of the lung word (src/dSFMT.c:443-482; PCV2 is odd)
  uint64_t inner = ((st_[2 * kN] ^ kFix1) & kPcv1) ^ ((st_[2 * kN + 1] ^ kFix2) & kPcv2);
  for (int sh = 32; sh > 0; sh >>= 1) inner ^= inner >> sh;
  if ((inner & 1) != 1) st_[2 * kN + 1] ^= 1;
  idx_ = 2 * kN;
}

void Dsfmt19937::next_block() {
  uint64_t l0 = st_[2 * kN], l1 = st_[2 * kN + 1];
  for (int i = 0; i < kN; i++) {
    const int b = (i + kPos1 < kN) ? i + kPos1 : i + kPos1 - kN;  // already updated past the wrap
    const uint64_t t0 = st_[2 * i], t1 = st_[2 * i + 1];
    const uint64_t n0 = (t0 << kSl1) ^ (l1 >> 32) ^ (l1 << 32) ^ st_[2 * b];
    const uint64_t n1 = (t1 << kSl1) ^ (l0 >> 32) ^ (l0 << 32) ^ st_[2 * b + 1];
    l0 = n0;
    l1 = n1;
    st_[2 * i] = (l0 >> kSr) ^ (l0 & kMsk1) ^ t0;
    st_[2 * i + 1] = (l1 >> kSr) ^ (l1 & kMsk2) ^ t1;
  }
  st_[2 * kN] = l0;
  st_[2 * kN + 1] = l1;
}

double Dsfmt19937::genrand_close_open() {
  if (idx_ >= 2 * kN) {
    next_block();
    idx_ = 0;
  }
  double r;
  std::memcpy(&r, &st_[idx_++], sizeof(double));  // a double in [1, 2)
  return r - 1.0;
}

void omp_static_chunk(int64_t n, int threads, int t, int64_t *begin, int64_t *end) {
  int64_t q = n / threads, r = n % threads;
  if (t < r) {
    q++;
    r = 0;
  }
  *begin = q * t + r;
  *end = *begin + q;
}

void reference_random_start(int64_t dim, RefStartKind kind, int initial_iv, int sample, int vec_type, int threads,
                            int count, std::vector<double> *out) {
  if (threads < 1) threads = 1;
  if (count < 1) count = 1;
  const uint64_t aiv = (uint64_t)(initial_iv < 0 ? -(long long)initial_iv : (long long)initial_iv);
  const int64_t stride = 2 * (dim + 1);
  out->assign((size_t)(stride * count), 0.0);
  for (int t = 0; t < threads; t++) {
    const uint64_t seed = (kind == kRefTPQ) ? 123432ull + (uint64_t)(sample + 1) * aiv + (uint64_t)t
                                            : 123432ull + aiv + (uint64_t)t;
    Dsfmt19937 g((uint32_t)seed);
    int64_t b, e;
    omp_static_chunk(dim, threads, t, &b, &e);
    for (int k = 0; k < count; k++) {
      double *v = out->data() + stride * k;
      for (int64_t i = b; i < e; i++) {
        double re, im = 0.0;
        if (vec_type == 0) {
          // 2(u - 1/2) + 2(u' - 1/2) i: the reference's build draws the imaginary part first
          im = 2.0 * (g.genrand_close_open() - 0.5);
          re = 2.0 * (g.genrand_close_open() - 0.5);
        } else if (vec_type == -1 && kind == kRefTPQ) {
          // Box-Muller pair (src/MakeIniVec.c:84-93)
          const double x = g.genrand_close_open(), y = g.genrand_close_open();
          const double rr = std::sqrt(-2.0 * std::log(x));
          re = rr * std::cos(2.0 * M_PI * y);
          im = rr * std::sin(2.0 * M_PI * y);
        } else {
          re = 2.0 * (g.genrand_close_open() - 0.5);
        }
        v[2 * (i + 1)] = re;
        v[2 * (i + 1) + 1] = im;
      }
    }
  }
  // normalisation (TPQ keeps the raw vector: its norm is the first TPQ norm); partial sums
  // per thread chunk, added in thread order
  if (kind == kRefTPQ) return;
  for (int k = 0; k < count; k++) {
    double *v = out->data() + stride * k;
    double nrm = 0.0;
    for (int t = 0; t < threads; t++) {
      int64_t b, e;
      omp_static_chunk(dim, threads, t, &b, &e);
      double part = 0.0;
      for (int64_t i = b; i < e; i++) part += v[2 * (i + 1)] * v[2 * (i + 1)] + v[2 * (i + 1) + 1] * v[2 * (i + 1) + 1];
      nrm += part;
    }
    nrm = std::sqrt(nrm);
    for (int64_t i = 1; i <= dim; i++) {
      v[2 * i] /= nrm;
      v[2 * i + 1] /= nrm;
    }
  }
}

}  // namespace hphi
