// Command-line front end with HPhi's interface (src/HPhiMain.c:178-358 for the modes this
// engine supports):
//   HPhi_b200 -e namelist.def   runs an expert-mode input;
//   HPhi_b200 -s stan.in        writes the expert-mode files of a standard-mode input into the
//                               current directory and runs them;
//   HPhi_b200 -sdry stan.in     only writes those files.
// Runs on CUDA device 0 (or $HPHI_DEVICE) and writes HPhi's output files into ./output.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/hphi_b200.h"

int main(int argc, char **argv) {
  const bool expert = argc >= 3 && std::strcmp(argv[1], "-e") == 0;
  const bool standard = argc >= 3 && std::strcmp(argv[1], "-s") == 0;
  const bool dry = argc >= 3 && std::strcmp(argv[1], "-sdry") == 0;
  if (!expert && !standard && !dry) {
    std::fprintf(stderr, "usage: %s -e namelist.def | -s stan.in | -sdry stan.in\n", argv[0]);
    return 1;
  }
  const char *namelist = argv[2];
  if (standard || dry) {
    if (hphi_stdface(argv[2], ".") != 0) {
      std::fprintf(stderr, "error: %s\n", hphi_last_error());
      return 1;
    }
    if (dry) return 0;
    namelist = "namelist.def";
  }
  const char *dev = std::getenv("HPHI_DEVICE");
  hphi_handle *h = nullptr;
  if (hphi_open_expert(namelist, dev ? std::atoi(dev) : 0, &h) != 0) {
    std::fprintf(stderr, "error: %s\n", hphi_last_error());
    return 1;
  }
  const int rc = hphi_run(h, "output");
  if (rc != 0) std::fprintf(stderr, "error: %s\n", hphi_last_error());
  hphi_close(h);
  return rc == 0 ? 0 : 1;
}
