// Product-layout kernel for canonical Hubbard models (hv_product.cu).
#pragma once
#include <string>

#include "engine.hpp"

namespace hphi {

struct ProdPlan;
// Builds the plan when the model qualifies (leaves s->prod null otherwise).
int prod_plan_build(Sector *s, std::string *err);
void prod_plan_free(ProdPlan *p);
// Native-order H*v (see engine.hpp hv_native).
int prod_hv_launch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out);
// Same with caller-provided row partial sums (prod_scratch_doubles) and row counter (2 ints).
int prod_hv_launch_scratch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                           double *d_part, int *d_counter);
size_t prod_scratch_doubles(const Sector *s, VecType vt);
// True when real vectors take the two-pass kernels (row pass + column pass).
bool prod_two_pass(const Sector *s);
int prod_permute(Sector *s, VecType vt, const void *in, void *out, bool to_native);
int prod_observables(Sector *s, VecType vt, const void *v, double *d_out);

}  // namespace hphi
