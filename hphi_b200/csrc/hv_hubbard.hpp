// Block kernel for canonical Hubbard models (hv_hubbard.cu).
#pragma once
#include <string>

#include "engine.hpp"

namespace hphi {

struct HubPlan;
// Builds the plan when the model qualifies (leaves s->hub null otherwise).
int hub_plan_build(Sector *s, std::string *err);
void hub_plan_free(HubPlan *p);
// Native-order H*v (see engine.hpp hv_native); acc_read = coefficient of v0 may be non-zero.
int hub_hv_launch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                  bool acc_read);
int hub_permute(Sector *s, VecType vt, const void *in, void *out, bool to_native);
// Same as hub_hv_launch with caller-provided partial sums and block counters (2 ints).
int hub_hv_launch_scratch(Sector *s, VecType vt, const void *d_v1, void *d_v0, const double *d_coef, double *d_out,
                          double *d_part, int *d_counter);
size_t hub_scratch_doubles(const Sector *s);
int hub_observables(Sector *s, VecType vt, const void *v, double *d_out);

}  // namespace hphi
