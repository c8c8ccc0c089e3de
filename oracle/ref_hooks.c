/*
 * Link-time hooks around the reference HPhi executable (test infrastructure).
 *
 * This file is linked into oracle/_ref/HPhi_ref together with the unmodified
 * reference sources (-Wl,--wrap=mltply -Wl,--wrap=sz -Wl,--wrap=diagonalcalc
 * -Wl,--wrap=expec_cisajs).
 * It never changes what the reference computes; it only records it:
 *
 *   HPHI_DUMP_DIR=<dir>      enables the dumps below (nothing is written otherwise)
 *   HPHI_DUMP_CALL=<k>       which mltply call to dump (0 = the first one, -1 = none)
 *   HPHI_DUMP_LISTS=0        skip the lists.bin / diag.bin dumps (timing runs)
 *
 *   <dir>/lists.bin   after sz():           int64 idim, n21, n22, then list_1[0..idim],
 *                                            list_2_1[0..n21), list_2_2[0..n22) as uint64
 *   <dir>/diag.bin    after diagonalcalc(): int64 idim, then list_Diagonal[0..idim] (f64)
 *   <dir>/hv.bin      around mltply call k: int64 idim, v1[0..idim], v0_before[0..idim],
 *                                            v0_after[0..idim] (complex128), prdct (complex128)
 *   <dir>/mltply_times.txt at exit:          number of mltply calls and their wall times (s)
 *   <dir>/green_times.txt at exit:           number of expec_cisajs calls and their wall times (s)
 *
 * Reference interfaces wrapped:
 *   int mltply(struct BindStruct*, double complex*, double complex*)   src/mltply.c:56
 *   int sz(struct BindStruct*, long unsigned int*, ...)                 src/sz.c:62
 *   int diagonalcalc(struct BindStruct*)                                src/diagonalcalc.c:84
 *   int expec_cisajs(struct BindStruct*, double complex*)               src/expec_cisajs.c:66
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <complex.h>
#include "struct.h"
#include "global.h"

int __real_mltply(struct BindStruct *X, double complex *v0_, double complex *v1_);
int __real_sz(struct BindStruct *X, long unsigned int *a, long unsigned int *b, long unsigned int *c);
int __real_diagonalcalc(struct BindStruct *X);
int __real_expec_cisajs(struct BindStruct *X, double complex *vec);

static long g_ncall = 0;
static double *g_times = NULL;
static long g_cap = 0;
static int g_atexit = 0;

static const char *dump_dir(void) {
  const char *d = getenv("HPHI_DUMP_DIR");
  return (d && d[0]) ? d : NULL;
}

static FILE *open_dump(const char *name) {
  char path[4096];
  const char *d = dump_dir();
  if (!d) return NULL;
  snprintf(path, sizeof(path), "%s/%s", d, name);
  return fopen(path, "wb");
}

static int dump_lists(void) {
  const char *d = getenv("HPHI_DUMP_LISTS");
  return !(d && d[0] == '0');
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static long g_ngreen = 0;
static double g_green_times[64];

static void write_times(void) {
  char path[4096];
  const char *d = dump_dir();
  if (!d) return;
  snprintf(path, sizeof(path), "%s/mltply_times.txt", d);
  FILE *f = fopen(path, "w");
  if (!f) return;
  fprintf(f, "%ld\n", g_ncall);
  for (long i = 0; i < g_ncall && i < g_cap; i++) fprintf(f, "%.9e\n", g_times[i]);
  fclose(f);
  if (g_ngreen == 0) return;
  snprintf(path, sizeof(path), "%s/green_times.txt", d);
  f = fopen(path, "w");
  if (!f) return;
  fprintf(f, "%ld\n", g_ngreen);
  for (long i = 0; i < g_ngreen && i < 64; i++) fprintf(f, "%.9e\n", g_green_times[i]);
  fclose(f);
}

int __wrap_expec_cisajs(struct BindStruct *X, double complex *vec) {
  double t0 = now_s();
  int r = __real_expec_cisajs(X, vec);
  double t1 = now_s();
  if (g_ngreen < 64) g_green_times[g_ngreen] = t1 - t0;
  g_ngreen++;
  if (!g_atexit) { atexit(write_times); g_atexit = 1; }
  return r;
}

int __wrap_sz(struct BindStruct *X, long unsigned int *a, long unsigned int *b, long unsigned int *c) {
  int r = __real_sz(X, a, b, c);
  /* grand-canonical models have no lists (GetlistSize, src/xsetmem.c:284-318) */
  FILE *f = (a && b && c && dump_lists()) ? open_dump("lists.bin") : NULL;
  if (f) {
    long long idim = (long long)X->Check.idim_max;
    long long n21 = X->Large.SizeOflist_2_1, n22 = X->Large.SizeOflist_2_2;
    fwrite(&idim, 8, 1, f); fwrite(&n21, 8, 1, f); fwrite(&n22, 8, 1, f);
    fwrite(a, 8, (size_t)idim + 1, f);
    fwrite(b, 8, (size_t)n21, f);
    fwrite(c, 8, (size_t)n22, f);
    fclose(f);
  }
  return r;
}

int __wrap_diagonalcalc(struct BindStruct *X) {
  int r = __real_diagonalcalc(X);
  FILE *f = dump_lists() ? open_dump("diag.bin") : NULL;
  if (f) {
    long long idim = (long long)X->Check.idim_max;
    fwrite(&idim, 8, 1, f);
    fwrite(list_Diagonal, 8, (size_t)idim + 1, f);
    fclose(f);
  }
  return r;
}

int __wrap_mltply(struct BindStruct *X, double complex *v0_, double complex *v1_) {
  const char *k = getenv("HPHI_DUMP_CALL");
  long want = k ? atol(k) : 0;
  long long idim = (long long)X->Check.idim_max;
  FILE *f = NULL;
  if (g_ncall == want) f = open_dump("hv.bin");
  if (f) {
    fwrite(&idim, 8, 1, f);
    fwrite(v1_, 16, (size_t)idim + 1, f);
    fwrite(v0_, 16, (size_t)idim + 1, f);
  }
  double t0 = now_s();
  int r = __real_mltply(X, v0_, v1_);
  double t1 = now_s();
  if (f) {
    double complex p = X->Large.prdct;
    fwrite(v0_, 16, (size_t)idim + 1, f);
    fwrite(&p, 16, 1, f);
    fclose(f);
  }
  if (g_ncall >= g_cap) {
    g_cap = g_cap ? 2 * g_cap : 1024;
    g_times = (double *)realloc(g_times, sizeof(double) * (size_t)g_cap);
  }
  g_times[g_ncall] = t1 - t0;
  g_ncall++;
  if (!g_atexit) { atexit(write_times); g_atexit = 1; }
  return r;
}
