// Product-layout kernel for canonical Hubbard models (hv_product.cu).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

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
// Edge-coloured gather table of the row pass for n columns (positions): rows[p] lists the
// sources of column p as (source position | negative << 16).  gat: per warp of 32 columns and
// group of 8 slots, 32 lanes x 4 words of two 16-bit entries (position | sign << 15);
// wslots: slots per warp; groups: slot groups per warp in the table.  Empty slots read one of
// the zero words n .. n + 15 (one per shared-memory bank pair).
void build_gather_table(const std::vector<std::vector<uint32_t>> &rows, int n, std::vector<uint32_t> *gat,
                        std::vector<uint8_t> *wslots, int *groups);

}  // namespace hphi
