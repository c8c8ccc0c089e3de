// Command-line front end with HPhi's expert-mode interface: `HPhi_b200 -e namelist.def`
// runs the input on CUDA device 0 (or $HPHI_DEVICE) and writes HPhi's output files
// into ./output (src/HPhiMain.c:178-358 for the modes this engine supports).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/hphi_b200.h"

int main(int argc, char **argv) {
  if (argc < 3 || std::strcmp(argv[1], "-e") != 0) {
    std::fprintf(stderr, "usage: %s -e namelist.def\n", argv[0]);
    return 1;
  }
  const char *dev = std::getenv("HPHI_DEVICE");
  hphi_handle *h = nullptr;
  if (hphi_open_expert(argv[2], dev ? std::atoi(dev) : 0, &h) != 0) {
    std::fprintf(stderr, "error: %s\n", hphi_last_error());
    return 1;
  }
  const int rc = hphi_run(h, "output");
  if (rc != 0) std::fprintf(stderr, "error: %s\n", hphi_last_error());
  hphi_close(h);
  return rc == 0 ? 0 : 1;
}
