// Standard-mode input: stan.in -> expert-mode .def files.
#pragma once

#include <string>

namespace hphi {
namespace stdface {

// Reads the keyword file `stan_in` and writes namelist.def and the .def files it lists into
// `out_dir` (which must exist).  Returns 0, or -1 with a message in *err.
int generate(const std::string &stan_in, const std::string &out_dir, std::string *err);

}  // namespace stdface
}  // namespace hphi
