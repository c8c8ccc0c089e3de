/*
 * hphi_b200 - C-ABI of the B200 engine for HPhi's H*v / Lanczos / TPQ path.
 *
 * Plain C types only.  Complex vectors on the host use HPhi's layout: an array of
 * (dim + 1) complex128 values stored as interleaved (re, im) doubles, element 0 unused
 * (src/include/global.h:34-50, src/xsetmem.c:178-193); this is layout-compatible with
 * C99 `double complex v[dim + 1]`.  Device vectors are 0-based arrays of dim elements
 * of the given element type.
 *
 * Every entry point returns 0 on success and -1 on failure; hphi_last_error() then
 * returns a message (per thread).  Nothing here calls exit().
 */
#ifndef HPHI_B200_H
#define HPHI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hphi_handle hphi_handle;

/* Element types of device vectors. */
#define HPHI_REAL64 0      /* double */
#define HPHI_COMPLEX128 1  /* interleaved (re, im) doubles */

/* Indices into the info array of hphi_info(). */
#define HPHI_INFO_DIM 0          /* idim_max (src/check.c:51-209) */
#define HPHI_INFO_NSITE 1
#define HPHI_INFO_CALC_MODEL 2   /* CalcModel; 6 = Hubbard with Ncond only (HubbardNConserved) */
#define HPHI_INFO_CALC_TYPE 3
#define HPHI_INFO_SIZE_LIST_2_1 4 /* X->Large.SizeOflist_2_1 (src/xsetmem.c:284-318) */
#define HPHI_INFO_SIZE_LIST_2_2 5 /* X->Large.SizeOflist_2_2 */
#define HPHI_INFO_IS_GC 6
#define HPHI_INFO_VEC_TYPE 7     /* element type the drivers use for this input */
#define HPHI_INFO_N_OFFDIAG 8    /* compiled off-diagonal terms */
#define HPHI_INFO_N_DIAG 9       /* compiled diagonal projector terms */
#define HPHI_INFO_LANCZOS_MAX 10
#define HPHI_INFO_NUM_AVE 11
#define HPHI_INFO_NATIVE_ORDER 12 /* 1 if the engine's native vector order differs from HPhi's */
#define HPHI_INFO_EXCT 13         /* exct: states of LOBPCG / the Lanczos eigenvector index */
#define HPHI_INFO_KERNEL 14       /* native H*v kernel: 0 general, 1 Hubbard block plan, 2 Hubbard product layout, 3 product layout two-pass (real vectors), 4 spin row-block passes */
#define HPHI_INFO_N_GREEN_ONE 15  /* OneBodyG rows read (NCisAjt) */
#define HPHI_INFO_N_GREEN_TWO 16  /* TwoBodyG rows read (NCisAjtCkuAlvDC) */
#define HPHI_INFO_COUNT 17

/* Library version string. */
const char *hphi_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char *hphi_last_error(void);

/*
 * Reads an expert-mode input (namelist.def and the files it names) and builds the
 * sector and diagonal on CUDA device `device`.
 * Replaces: ReadDefFileNInt + ReadDefFileIdxPara (src/readdef.c:463, 1006), check
 * (src/check.c:51), setmem_large (src/xsetmem.c:153), sz (src/sz.c:62) and
 * diagonalcalc (src/diagonalcalc.c:84), as called from main (src/HPhiMain.c:223-288).
 */
int hphi_open_expert(const char *namelist_def, int device, hphi_handle **out);

/*
 * Standard mode: reads the keyword file stan_in (lattice = chain / ladder / square /
 * triangular / honeycomb / kagome; model = Hubbard / Spin / Kondo and their GC forms;
 * method = Lanczos / CG / TPQ / cTPQ / FullDiag / Time-Evolution with quench or laser pumps;
 * CalcSpec with SpectrumType SzSz / S+S- / Density / Up / Down; their parameters) and writes
 * namelist.def and the expert-mode files it lists into out_dir, which then open with
 * hphi_open_expert.  Host only.
 * Replaces: StdFace_main (called at src/HPhiMain.c:212-214 for `HPhi -s` / `HPhi -sdry`).
 */
int hphi_stdface(const char *stan_in, const char *out_dir);

/*
 * Reads an expert-mode input on the host only (no device needed) and exports the
 * compiled Hamiltonian: counts[0] = off-diagonal terms, counts[1] = diagonal terms.
 * Off-diagonal term k (gather form, for an output configuration t): applies iff
 * (t & masks[4k]) == masks[4k+1]; source s = t ^ masks[4k+2]; value
 * (coefs[2k] + i coefs[2k+1]) * (-1)^popcount(t & masks[4k+3]) * v[row(s)].
 * Diagonal term k adds dcoefs[k] iff (c & dmasks[2k]) == dmasks[2k+1].
 * Arrays may be NULL (counts only); at most cap_off / cap_diag terms are written.
 * Inspection aid with no counterpart in the reference (its terms live in
 * struct DefineList, include/struct.h:43-300).
 */
int hphi_inspect_terms(const char *namelist_def, uint64_t *masks, double *coefs, int cap_off, uint64_t *dmasks,
                       double *dcoefs, int cap_diag, int64_t *counts);

/* Frees the handle and its device memory. */
void hphi_close(hphi_handle *h);

/* Fills info[0 .. min(n, HPHI_INFO_COUNT)) with the HPHI_INFO_* values. */
int hphi_info(const hphi_handle *h, int64_t *info, int n);

/*
 * Copies the sector tables in HPhi's layout: list_1[0 .. dim] (element 0 unused),
 * list_2_1[0 .. SizeOflist_2_1), list_2_2[0 .. SizeOflist_2_2), as filled by
 * sz() (src/sz.c:62-832).  Any pointer may be NULL.  Fails for grand-canonical models,
 * which have no lists.
 */
int hphi_sz(const hphi_handle *h, uint64_t *list_1, uint64_t *list_2_1, uint64_t *list_2_2);

/* Copies list_Diagonal[0 .. dim] (element 0 unused) as diagonalcalc computes it
 * (src/diagonalcalc.c:84-187). */
int hphi_diagonalcalc(const hphi_handle *h, double *list_diagonal);

/*
 * v0 += H v1 on host vectors in HPhi's layout, and *prdct = <v1|H|v1> (complex, 2 doubles).
 * Replaces: int mltply(struct BindStruct *X, double complex *v0, double complex *v1)
 * (src/mltply.c:56-132), whose X->Large.prdct is returned in prdct.
 */
int hphi_mltply(hphi_handle *h, double *v0, const double *v1, double *prdct);

/*
 * Device form of mltply: d_v0 = acc * d_v0 + scale * (H d_v1) on 0-based device vectors
 * of element type vec_type (acc == 0 never reads d_v0), and prdct (host, 2 doubles) =
 * sum conj(d_v1) (H d_v1).  Runs on the handle's stream and waits for it.
 * Replaces: mltply (src/mltply.c:56-132) for callers that keep vectors on the device.
 */
int hphi_mltply_device(hphi_handle *h, int vec_type, void *d_v0, const void *d_v1, double acc, double scale,
                       double *prdct);

/*
 * Asynchronous device form for callers that launch back to back, on vectors in the
 * engine's NATIVE order (see hphi_to_native): d_v0 = acc * d_v0 + scale * (H d_v1)
 * with (acc, scale) = d_coef[0..1] read on the device, and d_prdct[0..1] =
 * sum conj(d_v1) (H d_v1), all device pointers; enqueued on the handle's stream
 * (hphi_stream) without waiting.  acc == 0 never reads d_v0.
 * Replaces: mltply (src/mltply.c:56-132) inside device-resident solver loops.
 */
int hphi_mltply_device_async(hphi_handle *h, int vec_type, void *d_v0, const void *d_v1, const double *d_coef,
                             double *d_prdct);

/*
 * Dynamical Green's function by the Lanczos method: CalcSpectrum with CalcSpec 1
 * (src/CalcSpectrum.c:90-312) and CalcSpectrumByLanczos (src/CalcSpectrumByLanczos.c:43-163).
 * The excitation operators of the input (SingleExcitation / PairExcitation) act on h_vec
 * (HPhi-layout complex128, 2*(dim+1) doubles; NULL: <SpectrumVec>_rank_0.dat in output_dir),
 * the Lanczos tridiagonal components of the normalised excited state are computed on its
 * sector and G(omega) = |A v|^2 / (omega - a_1 - b_1^2 / (omega - a_2 - ...)) is evaluated on the
 * modpara frequency grid (OmegaMax, OmegaMin, OmegaIm / OmegaOrg, NOmega; without OmegaMax /
 * OmegaMin, from <head>_Lanczos_Step.dat as the reference's SetOmega does).  Writes
 * <head>_DynamicalGreen.dat, <head>_TMComponents.dat and, with OutputExVec 1,
 * <head>_excitedvec_rank_0.dat.  result (optional): per frequency Re omega, Im omega (OmegaOrg
 * included), Re G, Im G, for the first nresult frequencies.
 */
int hphi_spectrum(hphi_handle *h, const double *h_vec, const char *output_dir, double *result, int nresult);

/*
 * The H*v of hphi_mltply_device_async for callers that may not allocate device memory
 * when they call it: code whose device memory belongs to another allocator's budget, or a
 * latency-bound loop that cannot take cudaMalloc's device-wide synchronisation.  Same
 * vectors (native order, d_v0 = acc * d_v0 + scale * (H d_v1), acc == 0 never reads d_v0),
 * but the coefficients, the block counters and the partial sums of prdct live in one fixed
 * static device array of 128 KiB that every GPU loading the library keeps until exit; no
 * cudaMalloc or cudaFree is called.  prdct (host, 2 doubles) = sum conj(d_v1) (H d_v1);
 * the call waits for the handle's stream.  A sector whose kernel needs more partial sums
 * than the array holds is refused with an error (-1).  Every call shares the array: calls
 * that overlap on the GPU (other threads, streams or handles on the same device) race.
 * The first call on a device looks up the array's address; make it before any stream
 * capture.  No counterpart in the reference (HPhi allocates its work vectors itself).
 */
int hphi_mltply_device_noalloc(hphi_handle *h, int vec_type, void *d_v0, const void *d_v1, double acc,
                               double scale, double *prdct);

/*
 * Native vector order.  For canonical Hubbard inputs the engine stores each block of
 * HPhi's sector (rows sharing the upper half of the configuration, src/sz.c:993-1094)
 * as an (up, down) product matrix; otherwise the native order is HPhi's order.  These
 * permute 0-based device vectors between the two orders (d_in != d_out); they copy
 * when the orders coincide.  No counterpart in the reference (HPhi has one order).
 */
int hphi_to_native(hphi_handle *h, int vec_type, const void *d_hphi, void *d_native);
int hphi_from_native(hphi_handle *h, int vec_type, const void *d_native, void *d_hphi);

/* The CUDA stream (cudaStream_t) the handle launches on, and a blocking wait on it. */
void *hphi_stream(hphi_handle *h);
int hphi_synchronize(hphi_handle *h);

/*
 * Lanczos ground state (and, with CalcEigenVec != -1, the eigenvector, its energy and
 * variance).  v_init: normalised start vector in HPhi's layout, or NULL for the
 * reference's own start (single element for initial_iv > 0 on canonical models, else a
 * seeded random vector).  Writes zvo_Lanczos_Step.dat (and zvo_energy.dat with the
 * eigenvector) into output_dir when it is not NULL.  result (may be NULL) receives
 *   [0] converged (1/0)  [1] steps  [2] E_target  [3] E[1]  [4] E[2]  [5] E[3]  [6] E[4]
 *   [7] energy <v|H|v>   [8] <Hv|Hv>  [9] doublon  [10] Sz
 *   [11] diff_ene and [12] var of the accuracy check of the Lanczos vector
 *   [13] CG rounds (0: the check passed or CalcEigenVec is 1)  [14] CG iterations
 *   [15] diff_ene and [16] var after the CG refinement
 * With CalcEigenVec 0 and a failed accuracy check (relative variance or energy difference
 * not below 1e-12) the vector is refined by inverse iteration with CG solves before the
 * energy, doublon and Sz are taken.
 * Replaces: CalcByLanczos (src/CalcByLanczos.c:55-276) with Lanczos_EigenValue
 * (src/Lanczos_EigenValue.c:50), Lanczos_EigenVector (src/Lanczos_EigenVector.c:46) and
 * CG_EigenVector (src/CG_EigenVector.c:30).
 */
int hphi_lanczos(hphi_handle *h, const double *v_init, const char *output_dir, double *result, int nresult);

/*
 * Tridiagonal coefficients of the last hphi_lanczos run: alpha[0 .. n) and beta[0 .. n)
 * with n = min(cap, steps); *steps receives the step count.  These are the reference's
 * alpha[1 .. itr] and beta[1 .. itr] (src/Lanczos_EigenValue.c:113-176).
 */
int hphi_lanczos_tridiagonal(hphi_handle *h, double *alpha, double *beta, int cap, int *steps);

/*
 * Lanczos eigenvector copy-out: after hphi_lanczos with CalcEigenVec != -1, copies the
 * eigenvector (HPhi layout, dim + 1 complex128) into v.
 */
int hphi_lanczos_eigenvector(hphi_handle *h, double *v);

/*
 * mTPQ: NumAve samples of Lanczos_max steps each.  v_init: NumAve start vectors in HPhi's
 * layout, back to back ((dim + 1) complex128 each; any norm), or NULL for seeded random
 * starts.  Writes SS_rand%d.dat, Norm_rand%d.dat, Flct_rand%d.dat into output_dir.
 * result (may be NULL) receives the energies of the last sample, one per step
 * (nresult values at most).
 * Replaces: CalcByTPQ (src/CalcByTPQ.c:52-294), FirstMultiply (src/FirstMultiply.c:41),
 * Multiply (src/Multiply.c:42), expec_energy_flct (src/expec_energy_flct.c:34).
 */
int hphi_tpq(hphi_handle *h, const double *v_init, const char *output_dir, double *result, int nresult);

/*
 * Real-time evolution (CalcType 4) under H(t) = H + the TEOneBody / TETwoBody terms of each
 * time index.  Per step: psi <- sum_{k<=ExpandCoef} (-i dt H)^k / k! psi, normalised (the
 * first-order term uses the previous step's H psi; ExpandCoef 0 keeps first order only), then
 * E, var and the diagonal observables of psi.  v_init: the start state in HPhi's layout
 * ((dim + 1) complex128), or NULL to read <SpectrumVec>_rank_0.dat from output_dir (needs
 * InputEigenVec; ReStart 2 / 3 continue from the file's step).  Writes SS.dat, Norm.dat,
 * Flct.dat, <head>_cisajs_step%d.dat (every ExpecInterval steps) and, with OutputEigenVec,
 * <head>_eigenvec_%d_rank_0.dat (every OutputInterval steps and at the end, as index 0).
 * result (may be NULL) receives the energy of each step (nresult values at most).
 * Replaces: CalcByTEM (src/CalcByTEM.c:52-234), MultiplyForTEM (src/Multiply.c:79-139),
 * MakeTEDTransfer / MakeTEDInterAll (src/CalcByTEM.c:237-279), diagonalcalcForTE
 * (src/diagonalcalc.c:195-245).
 */
int hphi_tem(hphi_handle *h, const double *v_init, const char *output_dir, double *result, int nresult);

/*
 * Block LOBPCG for the exct lowest states (CalcType 3, "CG"; preconditioned when PreCG = 1).
 * v_init: exct start vectors in HPhi's layout, back to back (any norm), or NULL for the
 * reference's single-element starts (initial_iv > 0 on canonical models) or its random
 * ones (see hphi_reference_start).  Writes zvo_Lanczos_Step.dat and, when converged,
 * zvo_energy.dat into output_dir (NULL: no files).  result (may be NULL, nresult values at
 * most): [0] converged (1/0), [1] steps, [2] last residual 2-norm, then per state
 * [3 + 4i] energy, [4 + 4i] <Hx|Hx>, [5 + 4i] doublon, [6 + 4i] Sz.  Any exct up to dim / 3.
 * Replaces: CalcByLOBPCG / LOBPCG_Main (src/CalcByLOBPCG.c:328-776) with phys (src/phys.c:48).
 */
int hphi_lobpcg(hphi_handle *h, const double *v_init, const char *output_dir, double *result, int nresult);

/*
 * The whole expert-mode run of `HPhi -e namelist.def` for CalcType 0 (Lanczos),
 * 1 (TPQ) and 3 (LOBPCG), writing HPhi's output files into output_dir ("output" when NULL).
 * Replaces: main (src/HPhiMain.c:178-358) for those modes.
 */
int hphi_run(hphi_handle *h, const char *output_dir);

/*
 * Fixed-length Lanczos through the same driver as hphi_lanczos: exactly `steps` steps
 * (fewer only on a breakdown, beta < 1e-14) with the convergence test off, from the
 * hashed start vector of `seed` (element of configuration c: uniform in [-0.5, 0.5)
 * keyed by (seed, c), imaginary part too for complex vectors; the same vector
 * hphi_batch_lanczos uses).  energies[0 .. nev) receives the lowest eigenvalues of the
 * tridiagonal matrix.  This is CalcByLanczos (src/CalcByLanczos.c:55-276) with
 * Lanczos_max = steps and the LanczosEps test of src/Lanczos_EigenValue.c:262-275 off.
 */
int hphi_lanczos_steps(hphi_handle *h, int steps, uint64_t seed, double *energies, int nev);

/*
 * Batched Lanczos over many open Hamiltonians (same device).  No counterpart in the
 * reference, which solves one Hamiltonian per run; each instance follows the recurrence
 * of Lanczos_EigenValue (src/Lanczos_EigenValue.c:50-310).  precision HPHI_FP32 stores
 * the Lanczos vectors in float (FP64 sums, dots and scalars); with HPHI_BATCH_REFINE the
 * ground state of every instance is rebuilt in FP64 by replaying the recurrence
 * (as Lanczos_EigenVector, src/Lanczos_EigenVector.c:46-208) and its FP64 Rayleigh
 * quotient and residual are reported.  The handles must stay open while the batch lives.
 */
typedef struct hphi_batch hphi_batch;
#define HPHI_FP64 0
#define HPHI_FP32 1
#define HPHI_BATCH_GRAPH 1   /* capture the iterations in CUDA graphs */
#define HPHI_BATCH_REFINE 2  /* rebuild the ground state and refine its energy in FP64 */
#define HPHI_BATCH_RESULT_FIELDS 5
int hphi_batch_create(hphi_handle *const *handles, int n, int precision, hphi_batch **out);
/*
 * `steps` Lanczos steps for every instance from the hashed start vector of seed + 1000003*i
 * (instance i).  With HPHI_BATCH_REFINE the replay stops where the rest of the Ritz vector
 * has norm below replay_tol (<= 0: 1e-9).  result (n x HPHI_BATCH_RESULT_FIELDS, may be
 * NULL): [0] lowest eigenvalue of the tridiagonal matrix, [1] refined energy, [2] residual
 * |Hx - Ex|/|x|, [3] steps used, [4] steps replayed ([1]-[2],[4] zero without
 * HPHI_BATCH_REFINE).  timing (4, may be NULL): forward, replay and refinement
 * milliseconds, and the tuned hv-phase milliseconds.
 */
int hphi_batch_lanczos(hphi_batch *b, int steps, uint64_t seed, int flags, double replay_tol, double *result,
                       double *timing);
/* Launch shape (threads, rows per thread, CTAs per SM) chosen by the autotuner; retune != 0
 * times the candidates again. */
int hphi_batch_tuning(hphi_batch *b, int retune, int *shape);
void hphi_batch_free(hphi_batch *b);

/*
 * Request server: continuous batching of Lanczos ground-state requests (expert-mode
 * inputs of any model and sector size, CalcType 0) on one device.  No counterpart in the
 * reference; each request follows Lanczos_EigenValue (src/Lanczos_EigenValue.c:50-310)
 * with its own Lanczos_max, LanczosEps and LanczosTarget, tested every
 * steps_per_iteration steps.  Requests are admitted first come first served while a slot
 * (max_active) and the HBM budget (bytes; <= 0: 80% of the free memory) allow; every
 * admitted request keeps its sector and Lanczos state on the device and advances in the
 * same launches as the others; finished ones free their memory at once.  With HPHI_FP32
 * each ground state is rebuilt and refined in FP64 as in hphi_batch_lanczos.  An
 * instance's arithmetic does not depend on the other members, so a request gives the
 * same result alone and in a mix.
 */
typedef struct hphi_server hphi_server;
#define HPHI_SERVE_RESULT_FIELDS 8
int hphi_server_create(int device, int precision, int64_t hbm_budget, int max_active, int steps_per_iteration,
                       hphi_server **out);
/* Queues a request (the input is parsed now); arrival is its arrival time on
 * hphi_server_clock() (< 0: now), from which its latency is counted. */
int hphi_server_submit(hphi_server *s, const char *namelist_def, uint64_t seed, double arrival,
                       int64_t *request_id);
/* Admits, runs one iteration, retires finished requests.  counts (3, may be NULL):
 * active, queued, finished but not yet polled. */
int hphi_server_step(hphi_server *s, int64_t *counts);
/*
 * Pops one finished request: returns 1 and fills result (HPHI_SERVE_RESULT_FIELDS):
 * [0] status (0 converged, 1 stopped at Lanczos_max, -1 failed: message in
 * hphi_last_error), [1] energy (FP64-refined with HPHI_FP32), [2] lowest tridiagonal
 * eigenvalue, [3] residual of the refined vector (0 for HPHI_FP64), [4] Lanczos steps,
 * [5] dimension, [6] seconds waiting for admission, [7] seconds from arrival to result.
 * Returns 0 when nothing has finished.
 */
int hphi_server_poll(hphi_server *s, int64_t *request_id, double *result);
/* Seconds on the server's monotonic clock. */
double hphi_server_clock(void);
void hphi_server_free(hphi_server *s);

/*
 * The reference's random start vector(s) for a sector of `dim` rows, as HPhi draws them
 * with `threads` OpenMP threads (each thread seeds its own dSFMT-19937 generator and fills
 * its static-schedule share of the rows): kind 0 Lanczos (SetInitialVector,
 * src/Lanczos_EigenValue.c:552-610; normalised), 1 TPQ sample `sample` (MakeIniVec,
 * src/MakeIniVec.c:41-117; not normalised, its norm is the first TPQ norm), 2 LOBPCG
 * (Initialize_wave, src/CalcByLOBPCG.c:252-290; `count` normalised vectors).  vec_type is
 * InitialVecType (0 complex, 1 real, -1 Gaussian complex for TPQ).  v receives
 * count * (dim + 1) complex128 in HPhi's layout.  Host only.  hphi_lanczos, hphi_tpq and
 * hphi_lobpcg use these vectors when called without one (HPHI_B200_REF_THREADS, else
 * OMP_NUM_THREADS, else 1 thread).
 */
int hphi_reference_start(int64_t dim, int kind, int initial_iv, int sample, int vec_type, int threads, int count,
                         double *v);

/*
 * Green's functions <v| O |v> of the rows `rows` on the host vector vec (HPhi's layout,
 * complex128[dim+1], element 0 unused): body 1 rows are OneBodyG rows (i, s1, j, s2),
 * O = c+_{i s1} c_{j s2}; body 2 rows are TwoBodyG rows (i, s1, j, s2, k, s3, l, s4),
 * O = c+_{i s1} c_{j s2} c+_{k s3} c_{l s4} (spin models: |s><s'| on a site); body 3, 4, 6
 * rows are ThreeBodyG / FourBodyG / SixBodyG rows of 3, 4, 6 such pairs (4 integers each,
 * spin-1/2 SpinGC only, zero otherwise), with the reference's rules for each model.  out
 * receives (re, im) per row.
 * Replaces the entry loops of expec_cisajs (src/expec_cisajs.c:66-641) and
 * expec_cisajscktaltdc (src/expec_cisajscktaltdc.c:87-1647), one batch of rows per pass.
 */
int hphi_expec_green(hphi_handle *h, int body, int n, const int *rows, const double *vec, double *out);
/* The same on a device vector in HPhi's row order (d_vec[r] for row r + 1; vec_type 0 real
 * float64, 1 complex128), on the handle's stream; returns when out is filled. */
int hphi_expec_green_device(hphi_handle *h, int body, int n, const int *rows, int vec_type, const void *d_vec,
                            double *out);

/*
 * expec_cisajs (src/expec_cisajs.c:66) and expec_cisajscktaltdc (src/expec_cisajscktaltdc.c:87)
 * for the rows of the input's OneBodyG / TwoBodyG files: out receives (re, im) per row
 * (HPHI_INFO_N_GREEN_ONE / _TWO rows; may be NULL), and when path is not NULL the file is
 * written there in the reference's format (zvo_cisajs.dat, zvo_cisajscktalt.dat).
 */
int hphi_expec_cisajs(hphi_handle *h, const double *vec, double *out, const char *path);
int hphi_expec_cisajscktaltdc(hphi_handle *h, const double *vec, double *out, const char *path);

/*
 * Reads an expert-mode input on the host only and copies its OneBodyG (body 1, 4 ints per
 * row), TwoBodyG (body 2, 8 ints per row) or ThreeBodyG / FourBodyG / SixBodyG (body 3, 4,
 * 6: 12, 16, 24 ints per row) rows as the reader keeps them (a canonical Spin
 * model drops one-body rows with i != j, src/readdef.c:1455-1460).  Returns the row count
 * (at most cap rows are written; rows may be NULL), or -1 with a message for an input the
 * reference rejects (spin two-body rows need i == j and k == l, src/readdef.c:1497-1503).
 */
int hphi_inspect_green(const char *namelist_def, int body, int *rows, int cap);

#ifdef __cplusplus
}
#endif

#endif /* HPHI_B200_H */
