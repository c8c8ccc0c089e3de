// Split-term gather for the general H*v row kernels.
//
// HPhi keeps a configuration c as an upper half ib = c >> lo_bits and a lower half
// ia = c & (ihfbit - 1), and its row is list_2_1[ia] + list_2_2[ib] - 3 (GetOffComp,
// src/bitcalc.c:195-223).  A term whose condition, flip and sign masks all lie in the lower
// half applies, lands and signs the same way for every row with the same ia; one whose
// masks all lie in the upper half, the same way for every row with the same ib, and it
// keeps ia, so its source row is the output row shifted by
// list_2_2[ib ^ flip] - list_2_2[ib] (grand-canonical models: xor by the flip).  The plan
// stores, per lower half, the applicable lower-half terms as (list_2_1 of the source half,
// signed coefficient) and, per upper half, the applicable upper-half terms as (row shift,
// signed coefficient), so a row walks only the terms that act on it; the remaining terms
// take the generic test-and-lookup path.
#pragma once
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "engine.hpp"

namespace hphi {

// Lower-half entry: bits [0, 20) source value (list_2_1 of the source lower half, or the
// source lower half itself for grand-canonical models), bits [20, 32) coefficient index.
constexpr int kSplitTargetBits = 20;

struct SplitView {
  const uint32_t *lo_ptr;   // [2^lo_bits + 1] or nullptr (no plan)
  const uint32_t *lo_ent;
  const uint32_t *hi_ptr;   // [2^hi_bits + 1]
  const HiEnt *hi_ent;
  const double *coef;       // (re, im) per coefficient index, sign included
};

__host__ inline SplitView split_view(const SplitPlan &p) {
  return SplitView{p.lo_ptr, p.lo_ent, p.hi_ptr, p.hi_ent, p.coef};
}

// Adds the lower- and upper-half terms of row r (configuration c) to y.  load(j) returns
// the source element of row j as A.
template <typename A, bool GC, typename Load>
__device__ __forceinline__ A split_terms(const SplitView &P, uint64_t c, int64_t r, int lo_bits, uint64_t lo_mask,
                                         const uint32_t *__restrict__ l22, Load load, A y) {
  const uint32_t ia = (uint32_t)(c & lo_mask);
  const uint64_t ib = c >> lo_bits;
  const int64_t base = GC ? (int64_t)(c & ~lo_mask) : (int64_t)__ldg(l22 + ib) - 3;
  const uint32_t l0 = __ldg(P.lo_ptr + ia), l1 = __ldg(P.lo_ptr + ia + 1);
  for (uint32_t e = l0; e < l1; e++) {
    const uint32_t v = __ldg(P.lo_ent + e);
    const uint32_t tgt = v & ((1u << kSplitTargetBits) - 1u);
    const uint32_t k = v >> kSplitTargetBits;
    const int64_t j = GC ? (base | (int64_t)tgt) : base + (int64_t)tgt;
    const double2 cf = __ldg(reinterpret_cast<const double2 *>(P.coef) + k);
    y = VT<A>::add(y, VT<A>::cmul_re_im(cf.x, cf.y, load(j)));
  }
  const uint32_t h0 = __ldg(P.hi_ptr + ib), h1 = __ldg(P.hi_ptr + ib + 1);
  for (uint32_t e = h0; e < h1; e++) {
    const HiEnt h = P.hi_ent[e];
    const int64_t j = GC ? (int64_t)((uint64_t)r ^ (uint64_t)h.delta) : r + h.delta;
    const double2 cf = __ldg(reinterpret_cast<const double2 *>(P.coef) + h.k);
    y = VT<A>::add(y, VT<A>::cmul_re_im(cf.x, cf.y, load(j)));
  }
  return y;
}

}  // namespace hphi
