/*
 * Drop-in check of the C-ABI (test infrastructure): the unmodified reference HPhi with its
 * mltply (src/mltply.c:56) replaced at link time (-Wl,--wrap=mltply) by hphi_mltply from
 * libhphi_b200.so, the patch the integration notes give a maintainer.  Everything else --
 * CalcByLanczos (src/CalcByLanczos.c:55), the Lanczos recurrence and its convergence test,
 * the eigenvector replay, expec_energy_flct, the output files -- is the reference's own code,
 * so its output equals the plain reference's when hphi_mltply is a faithful mltply.
 *
 *   HPHI_B200_NAMELIST   namelist the engine's handle is opened from (default namelist.def,
 *                        the file the reference itself reads with -e namelist.def)
 *   HPHI_B200_DEVICE     CUDA device (default 0)
 *
 * Time evolution keeps the reference's own mltply (its time-dependent terms are set by
 * CalcByTEM through globals the C-ABI does not see).
 */
#include <complex.h>
#include <stdio.h>
#include <stdlib.h>

#include "struct.h"
#include "global.h"
#include "bitcalc.h"
#include "mltplyCommon.h"
#include "hphi_b200.h"

int __real_mltply(struct BindStruct *X, double complex *tmp_v0, double complex *tmp_v1);

static hphi_handle *g_b200 = NULL;

int __wrap_mltply(struct BindStruct *X, double complex *tmp_v0, double complex *tmp_v1) {
  if (X->Def.iCalcType == TimeEvolution) return __real_mltply(X, tmp_v0, tmp_v1);
  if (!g_b200) {
    const char *nl = getenv("HPHI_B200_NAMELIST");
    const char *dev = getenv("HPHI_B200_DEVICE");
    if (hphi_open_expert(nl && nl[0] ? nl : "namelist.def", dev ? atoi(dev) : 0, &g_b200) != 0) {
      fprintf(stderr, "hphi_b200: %s\n", hphi_last_error());
      return -1;
    }
  }
  /* the fields mltply leaves in X->Large for its callers (src/mltply.c:66-96) */
  long unsigned int irght = 0, ilft = 0, ihfbit = 0;
  const long unsigned int i_max = X->Check.idim_max;
  if (i_max != 0) {
    if (X->Def.iFlgGeneralSpin == FALSE) {
      if (GetSplitBitByModel(X->Def.Nsite, X->Def.iCalcModel, &irght, &ilft, &ihfbit) != 0) return -1;
    } else if (X->Def.iCalcModel == Spin) {
      if (GetSplitBitForGeneralSpin(X->Def.Nsite, &ihfbit, X->Def.SiteToBit) != 0) return -1;
    }
  }
  X->Large.i_max = i_max;
  X->Large.irght = irght;
  X->Large.ilft = ilft;
  X->Large.ihfbit = ihfbit;
  X->Large.mode = M_MLTPLY;
  double pr[2];
  if (hphi_mltply(g_b200, (double *)tmp_v0, (const double *)tmp_v1, pr) != 0) {
    fprintf(stderr, "hphi_b200: %s\n", hphi_last_error());
    return -1;
  }
  X->Large.prdct = pr[0] + I * pr[1];
  return 0;
}
