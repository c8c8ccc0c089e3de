// Row-block kernels for spin models (hv_rowblock.cu).
#pragma once
#include <string>

#include "engine.hpp"

namespace hphi {

struct RowBlockPlan;
// Builds the plan when the model qualifies (leaves s->rb null otherwise); needs the
// split-term plan.
int rb_plan_build(Sector *s, std::string *err);
void rb_plan_free(RowBlockPlan *p);
// True when vectors of type vt take the row-block kernels (the block fits in shared memory).
bool rb_applies(const Sector *s, VecType vt);
// H*v in HPhi's order (as hv_launch); the _scratch form takes rb_scratch_doubles(s) doubles
// of partial sums from the caller.
int rb_hv_launch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out);
int rb_hv_launch_scratch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                         double *d_part);
size_t rb_scratch_doubles(const Sector *s);

}  // namespace hphi
