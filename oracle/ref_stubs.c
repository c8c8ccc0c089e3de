/*
 * Stubs that let the reference HPhi link without its absent parts (test infrastructure).
 *  - StdFace_main: the StdFace git submodule (src/StdFace/) is not present, so standard
 *    mode cannot run; expert mode (HPhi -e namelist.def) is unaffected.
 *  - CalcSpectrumByBiCG: needs the Fortran komega library (no gfortran here); spectra
 *    are outside the hot path.
 */
#include <stdio.h>
#include <stdlib.h>
#include <complex.h>

struct EDMainCalStruct;

void StdFace_main(char *fname) {
  (void)fname;
  fprintf(stderr, "StdFace is not available in this build; use expert mode (-e namelist.def)\n");
  exit(1);
}

int CalcSpectrumByBiCG(struct EDMainCalStruct *X, double complex *a, double complex *b,
                       double complex *c, int n, double complex *d, double complex *e) {
  (void)X; (void)a; (void)b; (void)c; (void)n; (void)d; (void)e;
  fprintf(stderr, "komega (shifted BiCG) is not available in this build\n");
  return -1;
}
