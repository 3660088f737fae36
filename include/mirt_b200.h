/*
 * mirt_b200.h -- C ABI of the B200 (sm_100a) implementation of MIRT's
 * table-based NUFFT interpolation (JeffFessler/mirt, nufft/table/).
 *
 * Three layers, all plain C types:
 *
 *  1. Drop-ins for the eight mex gateways.  Same arguments, in the same order,
 *     as the MATLAB calls
 *        fm = interpD_table_mex(ck, h1..hD, J, L, tm, [order, flips])
 *        ck = interpD_table_adj_mex(fm, h1..hD, J, L, tm, K, [order, flips])
 *     with each mxArray passed as its data pointers (split real/imag FP64,
 *     column-major) and its dimensions.  An optional argument that the MATLAB
 *     call omits is passed as a NULL pointer.  The caller allocates the output
 *     (the gateway's mxCreateDoubleMatrix(..., mxCOMPLEX)) and passes its two
 *     data pointers.  Calls are synchronous; inputs are read-only.  Device
 *     arithmetic is FP32 with FP64 table-index selection, so the output agrees
 *     with the reference's FP64 kernels to FP32 rounding (relative L2 ~1e-7).
 *
 *  2. A device-resident interpolation plan: tables and trajectory are
 *     uploaded and bin-sorted once, then forward / adjoint run on float2
 *     (complex64) device buffers with the column (coil) index innermost.
 *
 *  3. A device-resident NUFFT (nufft.m / nufft_adj.m with 'table' and
 *     'minmax:kb'): tables and scaling factors built here in FP64, the
 *     oversampled FFT by cuFFT, deapodisation and phase fused around it.
 *
 * Every function returns MIRT_OK (0) or an error code; mirt_last_error()
 * gives the message of the last failure on the calling thread.  Argument
 * errors carry the reference gateway's own diagnostic, e.g.
 * "interp2_table_mex failed: h1 size problem".
 */
#ifndef MIRT_B200_H
#define MIRT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MIRT_OK 0
#define MIRT_ERR_ARG 1    /* invalid argument (reference: Fail() / mexFail()) */
#define MIRT_ERR_CUDA 2   /* CUDA runtime error, or no CUDA device */
#define MIRT_ERR_ALLOC 3  /* device allocation failed */
#define MIRT_ERR_FFT 4    /* cuFFT error */

/* Message of the last failing call on this thread ("" if none). */
const char *mirt_last_error(void);

/* Library version, major * 10000 + minor * 100 + patch. */
int mirt_version(void);

/* ------------------------------------------------------------------------
 * 1. mex gateway drop-ins
 *
 * Common conventions:
 *   *_re / *_im   data of a complex double mxArray (mxGetPr / mxGetPi).
 *                 An `_im` of NULL means a real mxArray: for a table this
 *                 selects the real-table kernels; for ck / fm it is the
 *                 reference's "mxIsComplexDouble" failure.
 *   *_rows/_cols  mxGetM / mxGetN of the array.
 *   J, L, K       int32 arrays with their element counts (mxGetM*mxGetN).
 *   order, flips  int32 arrays with element counts, or NULL when omitted.
 *   tm            real double [M, D], column-major.
 * ---------------------------------------------------------------------- */

/* fm = interp1_table_mex(ck, h, J, L, tm, [order, flips])
 * replaces nufft/table/interp1_table_mex.c:21-121 (gateway :126-149) and the
 * kernels of nufft/table/interp1_table1_for.c:19,70,126.
 * ck [K1, N] (ck_rows = K1, ck_cols = N); fm [M, N]. */
int mirt_interp1_table_mex(
	const double *ck_re, const double *ck_im, int64_t ck_rows, int64_t ck_cols,
	const double *h_re, const double *h_im, int64_t h_rows, int64_t h_cols,
	const int32_t *J, int64_t J_numel,
	const int32_t *L, int64_t L_numel,
	const double *tm, int64_t tm_rows, int64_t tm_cols,
	const int32_t *order, int64_t order_numel,
	const int32_t *flips, int64_t flips_numel,
	double *fm_re, double *fm_im);

/* fm = interp2_table_mex(ck, h1, h2, J, L, tm, [order, flips])
 * replaces nufft/table/interp2_table_mex.c:14-128 (gateway :132-154) and the
 * kernels of nufft/table/interp2_table1_for.c:24,106,198.
 * ck has dimensions ck_dims[0..ck_ndim-1] = [K1 K2 N] (N = 1 if absent). */
int mirt_interp2_table_mex(
	const double *ck_re, const double *ck_im, const int64_t *ck_dims, int32_t ck_ndim,
	const double *h1_re, const double *h1_im, int64_t h1_rows, int64_t h1_cols,
	const double *h2_re, const double *h2_im, int64_t h2_rows, int64_t h2_cols,
	const int32_t *J, int64_t J_numel,
	const int32_t *L, int64_t L_numel,
	const double *tm, int64_t tm_rows, int64_t tm_cols,
	const int32_t *order, int64_t order_numel,
	const int32_t *flips, int64_t flips_numel,
	double *fm_re, double *fm_im);

/* fm = interp3_table_mex(ck, h1, h2, h3, J, L, tm, [order, flips])
 * replaces nufft/table/interp3_table_mex.c:14-146 (gateway :150-175) and the
 * kernels of nufft/table/interp3_table1_for.c:24,134,258.
 * ck dimensions [K1 K2 K3 N].  The reference gateway rejects N > 1
 * ("N=1 done only", :85-86); this drop-in accepts any N. */
int mirt_interp3_table_mex(
	const double *ck_re, const double *ck_im, const int64_t *ck_dims, int32_t ck_ndim,
	const double *h1_re, const double *h1_im, int64_t h1_rows, int64_t h1_cols,
	const double *h2_re, const double *h2_im, int64_t h2_rows, int64_t h2_cols,
	const double *h3_re, const double *h3_im, int64_t h3_rows, int64_t h3_cols,
	const int32_t *J, int64_t J_numel,
	const int32_t *L, int64_t L_numel,
	const double *tm, int64_t tm_rows, int64_t tm_cols,
	const int32_t *order, int64_t order_numel,
	const int32_t *flips, int64_t flips_numel,
	double *fm_re, double *fm_im);

/* ck = interp1_table_adj_mex(fm, h, J, L, tm, K, [order, flips])
 * replaces nufft/table/interp1_table_adj_mex.c:21-126 (gateway :131-154) and
 * nufft/table/interp1_table1_adj.c:20,69,123.  fm [M, N]; ck [K1, N]. */
int mirt_interp1_table_adj_mex(
	const double *fm_re, const double *fm_im, int64_t fm_rows, int64_t fm_cols,
	const double *h_re, const double *h_im, int64_t h_rows, int64_t h_cols,
	const int32_t *J, int64_t J_numel,
	const int32_t *L, int64_t L_numel,
	const double *tm, int64_t tm_rows, int64_t tm_cols,
	const int32_t *K, int64_t K_numel,
	const int32_t *order, int64_t order_numel,
	const int32_t *flips, int64_t flips_numel,
	double *ck_re, double *ck_im);

/* ck = interp2_table_adj_mex(fm, h1, h2, J, L, tm, K, [order, flips])
 * replaces nufft/table/interp2_table_adj_mex.c:17-131 (gateway :135-159) and
 * nufft/table/interp2_table1_adj.c:24,102,190.  ck [K1*K2, N]. */
int mirt_interp2_table_adj_mex(
	const double *fm_re, const double *fm_im, int64_t fm_rows, int64_t fm_cols,
	const double *h1_re, const double *h1_im, int64_t h1_rows, int64_t h1_cols,
	const double *h2_re, const double *h2_im, int64_t h2_rows, int64_t h2_cols,
	const int32_t *J, int64_t J_numel,
	const int32_t *L, int64_t L_numel,
	const double *tm, int64_t tm_rows, int64_t tm_cols,
	const int32_t *K, int64_t K_numel,
	const int32_t *order, int64_t order_numel,
	const int32_t *flips, int64_t flips_numel,
	double *ck_re, double *ck_im);

/* ck = interp3_table_adj_mex(fm, h1, h2, h3, J, L, tm, K, [order, flips])
 * replaces nufft/table/interp3_table_adj_mex.c:17-149 (gateway :153-179) and
 * nufft/table/interp3_table1_adj.c:24,127,243.  ck [K1*K2*K3, N]. */
int mirt_interp3_table_adj_mex(
	const double *fm_re, const double *fm_im, int64_t fm_rows, int64_t fm_cols,
	const double *h1_re, const double *h1_im, int64_t h1_rows, int64_t h1_cols,
	const double *h2_re, const double *h2_im, int64_t h2_rows, int64_t h2_cols,
	const double *h3_re, const double *h3_im, int64_t h3_rows, int64_t h3_cols,
	const int32_t *J, int64_t J_numel,
	const int32_t *L, int64_t L_numel,
	const double *tm, int64_t tm_rows, int64_t tm_cols,
	const int32_t *K, int64_t K_numel,
	const int32_t *order, int64_t order_numel,
	const int32_t *flips, int64_t flips_numel,
	double *ck_re, double *ck_im);

/* fm = interp4_table_mex(ck, h1, h2, h3, h4, J, L, tm, [order, flips])
 * replaces nufft/table/interp4_table_mex.c:12-163 (gateway :167-184) and the
 * kernels of nufft/table/interp4_table1_for.c:30,168,325.
 * ck dimensions [K1 K2 K3 K4 N].  The reference gateway rejects N > 1
 * ("N=1 done only", :97-98); this drop-in accepts any N.  Its failure text
 * is the reference gateway's own, "interp3_table_mex failed" (:182).
 * K1..K3 must be >= J1..J3 (the GPU kernels wrap a tap once); K4 is free. */
int mirt_interp4_table_mex(
	const double *ck_re, const double *ck_im, const int64_t *ck_dims, int32_t ck_ndim,
	const double *h1_re, const double *h1_im, int64_t h1_rows, int64_t h1_cols,
	const double *h2_re, const double *h2_im, int64_t h2_rows, int64_t h2_cols,
	const double *h3_re, const double *h3_im, int64_t h3_rows, int64_t h3_cols,
	const double *h4_re, const double *h4_im, int64_t h4_rows, int64_t h4_cols,
	const int32_t *J, int64_t J_numel,
	const int32_t *L, int64_t L_numel,
	const double *tm, int64_t tm_rows, int64_t tm_cols,
	const int32_t *order, int64_t order_numel,
	const int32_t *flips, int64_t flips_numel,
	double *fm_re, double *fm_im);

/* ck = interp4_table_adj_mex(fm, h1, h2, h3, h4, J, L, tm, K, [order, flips])
 * replaces nufft/table/interp4_table_adj_mex.c:12-166 (gateway :170-189) and
 * nufft/table/interp4_table1_adj.c:31,160,306.  ck [K1*K2*K3*K4, N]. */
int mirt_interp4_table_adj_mex(
	const double *fm_re, const double *fm_im, int64_t fm_rows, int64_t fm_cols,
	const double *h1_re, const double *h1_im, int64_t h1_rows, int64_t h1_cols,
	const double *h2_re, const double *h2_im, int64_t h2_rows, int64_t h2_cols,
	const double *h3_re, const double *h3_im, int64_t h3_rows, int64_t h3_cols,
	const double *h4_re, const double *h4_im, int64_t h4_rows, int64_t h4_cols,
	const int32_t *J, int64_t J_numel,
	const int32_t *L, int64_t L_numel,
	const double *tm, int64_t tm_rows, int64_t tm_cols,
	const int32_t *K, int64_t K_numel,
	const int32_t *order, int64_t order_numel,
	const int32_t *flips, int64_t flips_numel,
	double *ck_re, double *ck_im);

/* ------------------------------------------------------------------------
 * 2. device-resident interpolation plan (no reference counterpart: the
 *    reference re-reads its tables and tm on every mex call)
 *
 * A plan covers `nslice` trajectories of slice_moff[s+1]-slice_moff[s]
 * samples each, sharing geometry, tables and the column count `ncol`.
 * Device layouts (float2 = complex64):
 *   grid    ck[s][k][c]  k = k1 + K1*(k2 + K2*k3), c < ncol
 *   samples fm[m][c]     m over all slices (slice s owns [moff[s], moff[s+1]))
 * ---------------------------------------------------------------------- */
typedef struct mirt_interp_plan mirt_interp_plan;

/* D = 1..4.  tm: host FP64 [Mtot, D] column-major (t = omega / (2 pi / K)).
 * h_re[d] / h_im[d]: host FP64 tables of length J[d]*L[d]+1; h_im == NULL or
 * h_im[0] == NULL selects real tables.  slice_moff: nslice+1 offsets
 * (NULL when nslice == 1).  phase_re/phase_im: optional host FP64 per-sample
 * factor applied after the gather and conjugated before the spread (NULL for
 * none).  stream: cudaStream_t used for the set-up work (NULL = default).
 * J[d] <= K[d] in the first three dimensions.  A 4D plan runs as a 3D plan
 * over the nslice * K4 hyperplanes of its grids, each sample once per
 * 4th-dimension tap (Mtot * J4 < 2^31), the tap's coefficient as that
 * sample's phase; the launch setters and the autotuner act on that 3D plan. */
int mirt_interp_plan_create(mirt_interp_plan **plan, int32_t D,
	const int32_t *K, const int32_t *J, const int32_t *L,
	const double *const *h_re, const double *const *h_im, int32_t order,
	const double *tm, int64_t Mtot, const int64_t *slice_moff, int32_t nslice,
	int32_t ncol, const double *phase_re, const double *phase_im, void *stream);

/* fm = interp(ck) on device buffers, asynchronous on `stream`. */
int mirt_interp_plan_forward(mirt_interp_plan *plan, const void *ck, void *fm, void *stream);

/* ck = interp_adj(fm) on device buffers; overwrites all of ck. */
int mirt_interp_plan_adjoint(mirt_interp_plan *plan, const void *fm, void *ck, void *stream);

/* Autotune: time candidate spread tile shapes (multiples of the sort bins),
 * warps per spread CTA (each owning a band of rows / planes), spare tile
 * columns, the split size of dense tiles and the task order, and the gather
 * CTA size, on this plan's trajectory; keep the fastest.  Allocates a scratch
 * grid and sample buffer for the duration of the call.  Results stay
 * bitwise deterministic for any choice. */
int mirt_interp_plan_autotune(mirt_interp_plan *plan, void *stream);

/* Current launch configuration: up to 23 values
 * {T1, T2, T3, spread threads, spread heavy-first order, coil lanes,
 *  gather threads, (unused), gather CTAs, B1, B2, B3, split chunk,
 *  spread tasks, spare tile columns, partial-tile reductions,
 *  spread shared-tile atomics, ownership spread, row-sweep segments (0: off,
 *  -1: balanced team list), row-sweep rows per band, TMA gather,
 *  row-sweep dense-bin patches, staged row sweep mode}. */
int mirt_interp_plan_config(mirt_interp_plan *plan, int32_t *out, int32_t n);

/* Adjoint accumulation order.  deterministic = 1 (the default): every
 * shared-memory accumulator of a spread tile has one owner warp and samples
 * are added in a fixed order, so the adjoint is bitwise reproducible.
 * deterministic = 0: all warps of a tile take whole samples and add with
 * shared-memory atomics (more warps per tile, no band tests; the same FP32
 * arithmetic, summed in a run-dependent order); the autotuner then also
 * tries this variant.  No reference counterpart (the reference is serial). */
int mirt_interp_plan_set_deterministic(mirt_interp_plan *plan, int32_t deterministic);

/* Ownership spread (2D, J = 6): the tile holding a sample's first tap adds
 * all 36 taps into a shared tile padded by J - 1 points; tiles run in four
 * launches by the parities of their indices (no two padded tiles of one
 * launch overlap) and add their padded tiles into the cleared grid.
 * Deterministic.  Needs tiles of >= 5 points and an even number of tiles
 * (the last >= 5 points) per dimension; else MIRT_ERR_ARG.  The autotuner
 * tries it where it applies.  No reference counterpart. */
int mirt_interp_plan_set_ownership(mirt_interp_plan *plan, int32_t own, void *stream);

/* Row-sweep spread (2D, J = 6, K >= 6 per dimension): lanes of one coil
 * chunk own a band of `rows` grid rows (1, 2 or 4) and one of `segments`
 * segments of their columns, and sweep the bin columns of the rows + 5 bin
 * rows whose samples reach the band, with six grid columns of accumulators
 * per row in registers; each grid point is written once, summed in a fixed
 * order that does not depend on rows or segments (deterministic), with no
 * tiles, shared memory or reduction launches.  segments: 1..K1 uniform
 * segments per row (more segments, more parallel teams, five warm-up columns
 * each); -1 a balanced team list built from the sort's bins (rows cut into
 * segments of about equal visit counts, about 64k teams: the default for
 * 32-coil plans); 0 returns to the tiled spread.  Teams are taken by the
 * kernel's warps from a work queue, heaviest first.  3D plans (J = 6, K >= 6
 * per dimension, coil chunks of 8, 16 or 32): the line sweep, in which a
 * warp owns a block of 2 x 2, 2 x 1 or one grid lines along k1 (lanes = coils
 * x lines) and `segments` (1..K1) uniform segments of their columns, and
 * sweeps the bin columns of the bin lines around the block with six columns
 * of accumulators per line in registers (rows unused; the default there,
 * two segments).  MIRT_ERR_ARG where it does not apply.  The autotuner tries
 * it where it applies.  No reference counterpart. */
int mirt_interp_plan_set_sweep(mirt_interp_plan *plan, int32_t segments, int32_t rows);

/* Dense bins of the sweeps: bins holding at least 16 samples (the k-space
 * centre of radial and kooshball trajectories) are summed, before the sweep,
 * into patches of J^D taps x C (in chunks of 64 samples, added in a fixed
 * order), and the sweep adds a bin's patch where it meets the bin instead of
 * its samples, so that no warp runs through thousands of samples of one bin.
 * 3D line sweeps always do; for the 2D row sweep on = 1 turns it on (one-row
 * bands only; the default where dense bins exist) and 0 off.  The sums per
 * grid point stay in a fixed order (deterministic), with the bins' samples
 * summed first.  MIRT_ERR_ARG if the plan has no dense bins.  No reference
 * counterpart. */
int mirt_interp_plan_set_dense(mirt_interp_plan *plan, int32_t on);

/* The 2D row sweep with 32-coil lanes, staged per bin column: the warp lists
 * the samples of the column's bin rows, copies their tap records and sample
 * rows into shared memory (cp.async) and sums them from there, the sums in the
 * order of the unstaged sweep (the same bits).  mode 0: unstaged; 1: staged,
 * after the pass that copies the samples into plan order; 2: staged, reading
 * the caller's samples through the sort permutation (no ordering pass).  Not
 * with dense-bin patches (set_dense 0 where both would apply); the autotuner
 * times 1 and 2 beside the unstaged sweep.  MIRT_ERR_ARG for other modes or
 * when the plan's lanes are not 32 coils wide.  No reference counterpart. */
int mirt_interp_plan_set_staged(mirt_interp_plan *plan, int32_t mode);

/* Gather over TMA-staged tiles and records (2D, J = 6, an even C >= 32,
 * K >= 13; 3D below; the default there, and the autotuner times it against the plain
 * gather): the gather order groups samples by 8 x 8 blocks of first taps; for
 * each work item (up to 96 samples of one block) a CTA loads the block's
 * 13 x 13 x 32-coil grid tile (cp.async.bulk.tensor) and the item's tap
 * coefficients and first taps (1-D bulk copies) into shared memory, two
 * stages deep, and reads all taps and records from there; blocks whose taps
 * wrap past K read the grid directly.  Same arithmetic and summation order
 * as the plain gather: identical results.  tma = 1: tiles of 32 coils (a warp
 * per sample, two CTAs per SM); 2: tiles of 16 coils (a half-warp per sample,
 * three CTAs per SM); 0 selects the plain gather.  3D plans (J = 6, an even
 * C >= 8, K >= 9): tma = 1 stages 9 x 9 x 9 x 8-coil tiles of 4 x 4 x 4
 * blocks of first taps (items of up to 32 samples, a quarter-warp per
 * sample); mode 2 is 2D only.  The autotuner times the forms that apply.
 * MIRT_ERR_ARG for other modes and where the plan has no TMA blocks.  No
 * reference counterpart. */
int mirt_interp_plan_set_gather(mirt_interp_plan *plan, int32_t tma);

/* Fault flag of the plan's bounded in-kernel waits (TMA stage arrivals):
 * synchronises the device, stores 1 in *fault if a wait ran out since the
 * last call, else 0, and clears it.  After a 1, treat the plan as poisoned:
 * the CTA whose wait ran out returned without computing its samples, and a
 * copy that was only late may still have landed in shared memory after that
 * CTA left, so no output of that launch, nor of kernels that ran beside it on
 * the same GPU, can be trusted.  Destroy the plan and build a new one.
 * No reference counterpart. */
int mirt_interp_plan_fault(mirt_interp_plan *plan, int32_t *fault);

/* Test hook of the bounded waits behind mirt_interp_plan_fault: with on = 1,
 * the TMA gather arms each stage's barrier for bytes that no copy delivers and
 * issues no copy at all, with a short wait limit, so every wait runs out with
 * nothing in flight; the launch computes no sample and sets the fault flag.
 * on = 0 restores the normal gather.  MIRT_ERR_ARG if the plan's gather is not
 * the TMA one.  No reference counterpart. */
int mirt_interp_plan_set_fault_test(mirt_interp_plan *plan, int32_t on);

/* Fix the spread's tiling instead of autotuning it: tile extents T[0..D-1]
 * (multiples of the sort bins B of mirt_interp_plan_config, at most the grid
 * extent rounded up to a bin), CTA size `threads` (a multiple of 32, each
 * warp owns a band of the tile) and `padc` spare columns per tile row side in
 * shared memory (0, or J1 - 1 = 5 for the J = 6 kernels in 2D/3D: the row
 * update then needs no bounds tests).  Results are identical to rounding for
 * every choice.  MIRT_ERR_ARG for out-of-range values (no reference
 * counterpart: tuning of this implementation). */
int mirt_interp_plan_set_spread(mirt_interp_plan *plan, const int32_t *T, int32_t threads,
                                int32_t padc, void *stream);

int mirt_interp_plan_destroy(mirt_interp_plan *plan);

/* ------------------------------------------------------------------------
 * 3. device-resident NUFFT with min-max:KB tables
 *    forward = nufft/nufft.m:128-165, adjoint = nufft/nufft_adj.m:32-80,
 *    set-up = nufft/nufft_init.m:93-95 -> nufft/nufft_table_init.m:38-134
 *
 * om: host FP64 [Mtot, D] column-major, radians.  n_shift: D values.
 * Device layouts:  image x[s][n][c] (n = n1 + N1*(n2 + N2*n3)),
 *                  samples X[m][c].
 * ---------------------------------------------------------------------- */
typedef struct mirt_nufft mirt_nufft;

int mirt_nufft_create(mirt_nufft **out, int32_t D, const int32_t *Nd, const int32_t *Kd,
	const int32_t *Jd, const int32_t *Ld, const double *n_shift,
	const double *om, int64_t Mtot, const int64_t *slice_moff, int32_t nslice,
	int32_t ncol, void *stream);

int mirt_nufft_forward(mirt_nufft *p, const void *x, void *X, void *stream);
int mirt_nufft_adjoint(mirt_nufft *p, const void *X, void *x, void *stream);

/* Same, from and to HOST complex64 buffers (interleaved re/im float pairs in
 * the device layouts above); copies in and out are part of the call, which
 * returns when the result is in host memory. */
int mirt_nufft_forward_host(mirt_nufft *p, const float *x, float *X, void *stream);
int mirt_nufft_adjoint_host(mirt_nufft *p, const float *X, float *x, void *stream);

/* The interpolation plan inside a NUFFT (for direct gather/spread calls). */
mirt_interp_plan *mirt_nufft_interp_plan(mirt_nufft *p);

/* mirt_interp_plan_autotune on the NUFFT's interpolation plan. */
int mirt_nufft_autotune(mirt_nufft *p, void *stream);

/* How the NUFFT runs: up to 3 values {1 if the oversampled FFT runs as the
 * library's fused passes over the interpolation grid (power-of-two K from
 * 64 to 1024 in every dimension), 0 if through cuFFT with coil-layout
 * transposes; library kernel launches of one forward; of one adjoint} (cuFFT's
 * own launches not counted).  No reference counterpart. */
int mirt_nufft_config(mirt_nufft *p, int32_t *out, int32_t n);

int mirt_nufft_destroy(mirt_nufft *p);

/* nufft_init's other interpolators in table mode (host FP64), for
 * nufft_init(om, Nd, Jd, Kd, n_shift, 'table', L, ktype, ...): the 1D table
 * of nufft/nufft_table_init.m:100-116 (J*L+1 complex values split into
 * h_re / h_im: nufft_init's sparse interpolator read by the 'fast'
 * construction, the last entry 0) and the 1D factors whose outer product is
 * st.sn (nufft/nufft_init.m:210-230, conjugated as its st.sn(:) * tmp'
 * does).  ktype:
 *   MIRT_KTYPE_KB_MINMAX    'kaiser' (alpha = 2.34 J, m = 0)
 *   MIRT_KTYPE_KB_USER      'kaiser', alpha, m (kb_alf, integer kb_m)
 *   MIRT_KTYPE_MINMAX_KB    'minmax:kb' (the tables of mirt_nufft_create)
 *   MIRT_KTYPE_MINMAX_TUNED 'minmax:tuned'
 *   MIRT_KTYPE_MINMAX_USER  'minmax:user' (alpha[0 .. nalpha-1], beta)
 *   MIRT_KTYPE_MINMAX_UNIF  'uniform' (alpha = 1, beta = 0)
 *   MIRT_KTYPE_LINEAR       'linear' (scale 1 / nufft_interp_zn(0, ...))
 * A NUFFT with these is mirt_newfft_create with phasing 'complex', mode
 * 'table0' and the tables and st.sn given (nufft.m / nufft_adj.m apply only
 * the n_shift phase around the same gather). */
int mirt_nufft_ktype_table(int32_t ktype, int32_t N, int32_t J, int32_t K, int32_t L,
	double kb_alf, int32_t kb_m, const double *alpha, int32_t nalpha, double beta,
	double *h_re, double *h_im);
int mirt_nufft_ktype_scale(int32_t ktype, int32_t N, int32_t J, int32_t K, double kb_alf,
	int32_t kb_m, const double *alpha, int32_t nalpha, double beta,
	double *sn_re, double *sn_im);

/* ------------------------------------------------------------------------
 * 3a. newfft in table mode: st = newfft(om, Nd, 'Jd', Jd, 'Kd', Kd,
 *     'n_shift', n_shift, 'mode', 'table0' | 'table1', 'oversample', Ld,
 *     'phasing', 'real' | 'complex', ...)
 *     set-up    nufft/newfft.m:146-176, nufft/private/newfft_table_init.m:40-52,130-137
 *     forward   st.fft  = nufft/private/newfft_approx_for.m:15-63
 *     adjoint   st.adj  = nufft/private/newfft_approx_adj.m:30-82
 *
 * The caller gives the tables h{d} (J_d L_d + 1 values each; h_im NULL or
 * h_im[0] NULL for real tables), the interpolation order (0 or 1; 1 only
 * with real tables, as the table mex files require), the scaling factors
 * st.sn [prod Nd] (sn_im may be NULL) and Nmid (NULL: no phases, as
 * phasing 'complex').  The plan applies, inside its existing passes:
 *   phase_before[k] = prod_d exp(i 2 pi k_d Nmid_d / K_d)   (nufft/newfft.m:511-520)
 *       on the grid after the FFT (conjugate before the inverse FFT), and
 *   phase_after[m] = exp(i om_m . (n_shift - Nmid))           (nufft/newfft.m:522-527)
 *       on the samples after interpolation (conjugate before spreading).
 * Everything else (layouts, forward/adjoint/host/autotune/capture/destroy)
 * is that of mirt_nufft above.
 * ---------------------------------------------------------------------- */
int mirt_newfft_create(mirt_nufft **out, int32_t D, const int32_t *Nd, const int32_t *Kd,
	const int32_t *Jd, const int32_t *Ld, const double *const *h_re,
	const double *const *h_im, int32_t order, const double *sn_re, const double *sn_im,
	const double *nmid, const double *n_shift, const double *om, int64_t Mtot,
	const int64_t *slice_moff, int32_t nslice, int32_t ncol, void *stream);

/* newfft's default interpolator, ktype 'kb:minmax' with phasing 'real'
 * (host FP64):
 *   table: J*L+1 real values, the KB kernel (alpha = 2.34 J, kb_m = 0)
 *          at t = -J/2 + i/L  (nufft/private/newfft_table_init.m:140-184,
 *          nufft/kaiser_bessel.m:106-117)
 *   scale: N real values 1 / KB-FT((n - nmid) / K)  (nufft/newfft.m:352-356,
 *          nufft/kaiser_bessel_ft.m); st.sn is their outer product and
 *          nmid = floor(N/2) for phasing 'real' (nufft/newfft.m:146-151). */
int mirt_newfft_kb_table(int32_t J, int32_t L, double *h);
int mirt_newfft_kb_scale(int32_t N, int32_t J, int32_t K, double nmid, double *sn);

/* newfft's table interpolators by ktype (phasing 'real'; host FP64):
 *   MIRT_KTYPE_KB_MINMAX  'kb:minmax' (as mirt_newfft_kb_table / _kb_scale)
 *   MIRT_KTYPE_KB_BEATTY  'kb:beatty': the KB kernel (kb_m = 0) of shape
 *                         alpha = pi sqrt(J^2 / r^2 (r - 1/2)^2 - 0.8), r = K/N
 *                         (nufft/newfft.m:275-283), scale 1 / KB-FT((n - nmid) / K)
 *   MIRT_KTYPE_DIRIC      'diric': N'/K diric(t, N', K) with N' = 2 floor((K+1)/2) - 1
 *                         (nufft/newfft.m:256-266, nufft/nufft_diric.m), scale 1;
 *                         exact only when J = K, as the reference warns
 *   MIRT_KTYPE_MINMAX_KB  'minmax:kb': the min-max interpolator with KB-fitted
 *                         scaling (nufft/newfft.m:315-320, 384-395), the fit at
 *                         Nmid = floor(N/2), no phase; scale the real part of
 *                         nufft_scale1 at nmid (N <= K)
 *   MIRT_KTYPE_MINMAX_UNIF  'minmax:unif': the min-max interpolator with
 *                         uniform scaling, alpha = 1, beta = 0
 *                         (nufft/newfft.m:337-341); scale 1 (N <= K)
 *   MIRT_KTYPE_MINMAX_TUNED 'minmax:tuned': the min-max interpolator with the
 *                         tuned coefficients of nufft_best_alpha(J, 0, K/N)
 *                         (nufft/newfft.m:322-327, nufft/nufft_best_alpha.m):
 *                         K = 2N needs J in 2..10; other K/N take alpha = 1,
 *                         beta = 0.5 as the reference does (N <= K)
 *   MIRT_KTYPE_LINEAR     'linear': the triangle 1 - |t|/(J/2) on |t| < J/2
 *                         (nufft/newfft.m:268-273); scale newfft_scale_tri
 *                         (nufft/newfft.m:535-550) at this dimension's nmid
 * table: J*L+1 values at t = -J/2 + i/L; scale: N values (st.sn is their outer
 * product over dimensions).  MIRT_ERR_ARG for unknown ktypes, for
 * 'kb:beatty' where its shape is not real and for 'minmax:tuned' where the
 * reference has no coefficients. */
#define MIRT_KTYPE_KB_MINMAX 0
#define MIRT_KTYPE_KB_BEATTY 1
#define MIRT_KTYPE_DIRIC 2
#define MIRT_KTYPE_MINMAX_KB 3
#define MIRT_KTYPE_MINMAX_UNIF 4
#define MIRT_KTYPE_MINMAX_TUNED 5
#define MIRT_KTYPE_LINEAR 6
int mirt_newfft_ktype_table(int32_t ktype, int32_t N, int32_t J, int32_t K, int32_t L, double *h);
int mirt_newfft_ktype_scale(int32_t ktype, int32_t N, int32_t J, int32_t K, double nmid,
	double *sn);

/* newfft's interpolators with caller parameters (phasing 'real'; host FP64):
 *   'kb:user' (nufft/newfft.m:300-313): the KB kernel of shape alpha and
 *       integer order m in 0..32, f^m I_m(alpha f) / I_m(alpha), f = sqrt(1 -
 *       (t/(J/2))^2) (nufft/kaiser_bessel.m:106-117; alpha and m printed with
 *       %g into the kernel as the reference's inline kernel does); scale
 *       1 / KB-FT((n - nmid) / K, J, alpha, m) (nufft/kaiser_bessel_ft.m:70-73)
 *   'minmax:user' (nufft/newfft.m:329-335): the min-max interpolator for the
 *       real Fourier coefficients alpha[0 .. nalpha-1] and beta of its scaling
 *       factors (nufft/private/nufft_T.m, nufft_r.m); scale the real part of
 *       nufft_scale1 (N <= K)
 * One dimension per call, as the reference's st.kb_alf(id) / st.alpha{id}. */
int mirt_newfft_kb_user_table(int32_t J, int32_t L, double alpha, int32_t m, double *h);
int mirt_newfft_kb_user_scale(int32_t N, int32_t J, int32_t K, double nmid, double alpha,
	int32_t m, double *sn);
int mirt_newfft_minmax_user_table(int32_t N, int32_t J, int32_t K, int32_t L,
	const double *alpha, int32_t nalpha, double beta, double *h);
int mirt_newfft_minmax_user_scale(int32_t N, int32_t K, double nmid, const double *alpha,
	int32_t nalpha, double beta, double *sn);

/* newfft's tables with phasing 'complex' (host FP64, J*L+1 complex values
 * split into h_re / h_im) for every ktype above, MIRT_KTYPE_KB_USER (kb_alf,
 * kb_m) and MIRT_KTYPE_MINMAX_USER (alpha[0 .. nalpha-1], beta); the other
 * ktypes ignore those arguments.  The sparse interpolator's entries
 * conj(exp(i gam (N-1)/2 (t - k)) c) (nufft/newfft.m:405-411, 446) read by
 * the 'fast' construction (nufft/private/newfft_table_init.m:160-169: the
 * last entry repeats the first; 'diric' without the odd-N trick of phasing
 * 'real'), or for 'kb:*' by the 'ratio' construction (:173-184: a fake
 * problem N' = J, K' = J K / N and the phase exp(i pi t (1/K - 1/K'))).
 * 'minmax:kb' fits its alphas at Nmid = (N-1)/2.  Scaling factors: the
 * functions above with nmid = (N-1)/2. */
#define MIRT_KTYPE_KB_USER 7
#define MIRT_KTYPE_MINMAX_USER 8
int mirt_newfft_table_complex(int32_t ktype, int32_t N, int32_t J, int32_t K, int32_t L,
	double kb_alf, int32_t kb_m, const double *alpha, int32_t nalpha, double beta,
	double *h_re, double *h_im);

/* Capture one batched step of the plan -- forward x -> X when x is given,
 * then adjoint X -> xa when xa is given -- into a CUDA graph (on an internal
 * capture stream) and return it instantiated; mirt_graph_launch replays it
 * on `stream` with the same buffers.  The plan's calls allocate nothing per
 * call, so the whole step (deapodise/pad, FFTs, transposes, gather, spread,
 * crop) is one graph launch.  The plan and buffers must outlive the graph. */
typedef struct mirt_graph mirt_graph;
int mirt_nufft_capture(mirt_nufft *p, const void *x, void *X, void *xa, mirt_graph **out);
int mirt_graph_launch(mirt_graph *g, void *stream);
int mirt_graph_destroy(mirt_graph *g);

/* ------------------------------------------------------------------------
 * 3b. density compensation on a single-column NUFFT plan (ncol = 1)
 *
 * mirt_dcf_pipe replaces ir_mri_dcf_pipe_do (mri/ir_mri_density_comp.m:
 * 203-281): from w = 1 (init_ones = 1) or the caller's w, repeat
 * goal = real(P P' w), w = w ./ goal (P = the plan's table interpolator with
 * its phase shift) until max |goal - 1| <= thresh, with at most niter + 1
 * updates as in the reference loop; then scale so that sum(real(G' w)) =
 * prod(N ./ fov) per slice (fov: D values, NULL for 1).  Every slice of a
 * batched plan is its own problem and stops on its own residual.  A
 * non-positive goal fails with "pipe bug", as the reference does.  The
 * reference's `unitv` and `isave` options are not provided.
 *   w       device FP64 [Mtot], sample order of the plan (in / out)
 *   iters   host int32 [nslice] or NULL: updates done per slice
 *   resid   host FP64 [nslice] or NULL: last max |goal - 1| per slice
 * Interpolation in FP32; weights, ratio update, residual and scale in FP64.
 * Returns after the result is in w.
 *
 * mirt_dcf_jackson replaces ir_mri_dcf_jackson (:160-180) for table plans:
 * w = 1 ./ real(P (P' 1)). */
int mirt_dcf_pipe(mirt_nufft *p, double *w, int32_t init_ones, int32_t niter, double thresh,
	const double *fov, int32_t *iters, double *resid, void *stream);
int mirt_dcf_jackson(mirt_nufft *p, double *w, void *stream);

/* The final step of mirt_dcf_pipe on its own: scale w (device FP64 [Mtot])
 * so that sum(real(G' w)) = prod(N ./ fov) per slice (fov: D values or NULL
 * for 1), as mri/ir_mri_density_comp.m:258-261 does; for weights from
 * elsewhere (e.g. the learned regressor below).  Synchronous. */
int mirt_dcf_scale(mirt_nufft *p, double *w, const double *fov, void *stream);

/* ------------------------------------------------------------------------
 * 3d. batched CG-SENSE on a 2D NUFFT plan (one problem per slice, ncol = coils)
 *
 * A = Asense(G, sens) (systems/Asense.m:53-56), R = C'C of Reg1's quadratic
 * first-order penalty with its defaults (penalty/Reg1.m, offsets
 * [1 nx nx+1 nx-1] of penalty/penalty_offsets.m, 'tight' edges and
 * w = beta / |offset| of penalty/Rweights.m), beta per problem.
 *   sens  device complex64 [S][N2][N1][C] (copied)
 *   x     device complex64 [S][N2][N1];  y: device complex64 [Mtot][C]
 * forward y = A x, adjoint x = A' y, reg rx = R x (all asynchronous).
 * mirt_sense_cg runs `niter` iterations of wls/qpwls_pcg1.m:94-189 (precon 1,
 * Fletcher-Reeves, real step, FP64 inner products per problem) from the x
 * given, in place, with data weights W (device FP32 [Mtot], all coils) or
 * NULL for W = 1.  With xref (device, layout of x) and nrmse (host FP64
 * [(niter + 1) * S]), nrmse[it * S + s] = ||x_it - xref|| / ||xref|| of
 * problem s; ms (host FP32 [niter] or NULL) gets the device time from the
 * start of the call to the end of each iteration.  Returns after the last
 * iteration.  S <= 1024. */
typedef struct mirt_sense mirt_sense;
int mirt_sense_create(mirt_sense **out, mirt_nufft *G, const void *sens, const double *beta,
	void *stream);
int mirt_sense_forward(mirt_sense *op, const void *x, void *y, void *stream);
int mirt_sense_adjoint(mirt_sense *op, const void *y, void *x, void *stream);
int mirt_sense_reg(mirt_sense *op, const void *x, void *rx, void *stream);
int mirt_sense_cg(mirt_sense *op, void *x, const void *y, const float *W, int32_t niter,
	const void *xref, double *nrmse, float *ms, void *stream);
/* Attach the Toeplitz Gram operator of the plan's NUFFT (no data weights;
 * see mirt_toeplitz_create) and the circulant preconditioner built from it
 * (spectrum 1 / max(lam Re H + r, 1e-3 max), lam the problem's mean coil
 * power, r the spectrum of the Reg1 penalty).  om: the plan's host FP64
 * [Mtot, 2] column-major trajectory.  Synchronous. */
int mirt_sense_toeplitz(mirt_sense *op, const double *om, void *stream);

/* The circulant preconditioner from density-compensation weights (the learned
 * DCF, or any): the spectrum of G' diag(w^2) G -- the inverse sampling density
 * where the trajectory samples -- floored at 1e-3 of its maximum per problem,
 * so that the preconditioner stays Hermitian positive definite and the
 * minimiser is unchanged, and blended with the unweighted spectrum of
 * mirt_sense_toeplitz: P = blend Pw / mean(Pw) + (1 - blend) P1 / mean(P1)
 * per problem (blend 0: the unweighted preconditioner again).  Replaces the
 * attached preconditioner; MIRT_PCG_CIRCULANT then uses it.  om: the plan's
 * host FP64 trajectory; w: device FP64 [Mtot] in the plan's sample order.
 * MIRT_ERR_ARG without mirt_sense_toeplitz or with blend outside [0, 1].
 * Synchronous.  No reference counterpart. */
int mirt_sense_precon_dcf(mirt_sense *op, const double *om, const double *w, double blend,
	void *stream);

/* mirt_sense_cg with options (flags, OR of):
 *   MIRT_PCG_CIRCULANT  precondition with the attached circulant
 *                       preconditioner (qpwls_pcg1's `precon`)
 *   MIRT_PCG_TOEPLITZ   iterate on the normal equations with the attached
 *                       Toeplitz Gram operator, b = A'y, as
 *                       wls/qpwls_pcg2.m does (W must be NULL)
 * Both need mirt_sense_toeplitz first. */
#define MIRT_PCG_CIRCULANT 1
#define MIRT_PCG_TOEPLITZ 2
int mirt_sense_pcg(mirt_sense *op, void *x, const void *y, const float *W, int32_t niter,
	int32_t flags, const void *xref, double *nrmse, float *ms, void *stream);

/* Warm start for mirt_sense_cg: x = a A'(W y) per problem, the density-
 * compensated conjugate-phase image (the initial estimate of
 * example/mri_example.m:125 and :148) with a = Re<A x, y> / ||A x||^2, the
 * least-squares scale.  W: device FP32 [Mtot] weights (a density
 * compensation) or NULL.  Synchronous. */
int mirt_sense_warm_start(mirt_sense *op, void *x, const void *y, const float *W, void *stream);
int mirt_sense_destroy(mirt_sense *op);

/* ------------------------------------------------------------------------
 * 3e. Toeplitz Gram operator T = G'WG of a batched 2D NUFFT
 *     (systems/Gnufft_gram.m; kernel as Gnufft_gram_init2, :183-198)
 *
 * Built from two adjoint NUFFTs of the weights (FP32 tables and FFTs, one
 * slice per problem), embedded in a 2N1 x 2N2 circulant per slice and made
 * Hermitian (systems/private/dsft_gram_hermitify.m).  om: host FP64 [M, 2]
 * column-major; w: device FP64 [M] or NULL for W = 1; ncol: columns per
 * image for apply.  apply: y = T x for x, y device complex64
 * [S][N2][N1][ncol] (asynchronous). */
typedef struct mirt_toeplitz mirt_toeplitz;
int mirt_toeplitz_create(mirt_toeplitz **out, const double *om, int64_t M,
	const int64_t *slice_moff, int32_t nslice, const int32_t *Nd, const int32_t *Kd,
	const int32_t *Jd, const int32_t *Ld, const double *w, int32_t ncol, void *stream);
int mirt_toeplitz_apply(mirt_toeplitz *T, const void *x, void *y, void *stream);
int mirt_toeplitz_destroy(mirt_toeplitz *T);

/* ------------------------------------------------------------------------
 * 3c. learned density compensation (no counterpart in the reference)
 *
 * Features of each 2D sample (MIRT_DCF_NFEAT floats, row per sample, sample
 * order of om): |omega| / pi, atan2(omega_2, omega_1) / pi, and log1p of the
 * counts of other samples of the same trajectory (slice) at distance
 * [b/8, (b+1)/8) grid cells, b < 16, of the oversampled grid
 * (t = omega / (2 pi / K), no periodic wrap).  Counts are exact (FP64
 * distances).  om: device FP64 [M, 2] column-major; feat: device FP32.
 * Synchronous. */
#define MIRT_DCF_NFEAT 18
int mirt_dcf_features(const double *om, int64_t M, const int64_t *slice_moff, int32_t nslice,
	const int32_t *K, float *feat, void *stream);

/* Regressor 18 -> 64 -> 64 -> 64 -> 1 (ReLU) with BF16 weights and FP32
 * accumulation.  Parameters: one FP32 vector of MIRT_MLP_NPARAM values,
 * W1[64][18] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64] b4 (row =
 * output unit); the kernels use their BF16 rounding.
 *   create   copies the initial parameters (host) to the device
 *   params   copies the FP32 master parameters back to the host
 *   grad     gradient (host, MIRT_MLP_NPARAM) and loss of the mean squared
 *            error over the n rows of x (device [n][18]) against y (device [n])
 *   train    `steps` Adam steps (lr, beta 0.9 / 0.999, eps 1e-8) on batches of
 *            `batch` rows drawn by a counter-based hash of (seed, step, row);
 *            loss_hist (host, `steps` floats, or NULL) gets each step's loss
 *   infer    yhat = network output (device FP32 [n], or NULL) and / or
 *            w = exp(sigma * yhat + mu) (device FP64 [n], or NULL); async.
 *            On the tensor cores (mma.sync m16n8k16 BF16, FP32 accumulation;
 *            each FP32 activation enters as three BF16 terms, so the result
 *            keeps FP32 accuracy: ~3e-8 relative to FP64 on random weights)
 *   set_tensor_cores  0: inference on the FP32 pipes instead (the training
 *            kernels' forward), 1 (the default): on the tensor cores */
#define MIRT_MLP_NPARAM 9601
typedef struct mirt_mlp mirt_mlp;
int mirt_mlp_create(mirt_mlp **out, const float *params);
int mirt_mlp_params(mirt_mlp *m, float *params);
int mirt_mlp_grad(mirt_mlp *m, const float *x, const float *y, int64_t n, float *grad,
	float *loss, void *stream);
int mirt_mlp_train(mirt_mlp *m, const float *x, const float *y, int64_t n, int32_t batch,
	int32_t steps, float lr, uint64_t seed, float *loss_hist, void *stream);
int mirt_mlp_infer(mirt_mlp *m, const float *x, int64_t n, float mu, float sigma, float *yhat,
	double *w, void *stream);
int mirt_mlp_set_tensor_cores(mirt_mlp *m, int32_t on);
int mirt_mlp_destroy(mirt_mlp *m);

/* ------------------------------------------------------------------------
 * 4. forward gather for callers that cannot allocate device memory (no
 *    counterpart in the reference, whose mex files run on the host)
 *
 * Code that runs during CUDA-graph stream capture, hosts whose device memory
 * belongs to their own pool, and real-time loops that must not stall on an
 * allocation cannot call cudaMalloc.  This entry point runs the table gather
 * fm = interp(ck) on the caller's device buffers and allocates nothing: its
 * scratch (per-sample tap coefficients and first taps) is a fixed array of
 * MIRT_NOALLOC_SCRATCH_BYTES inside the library, held by every GPU that loads
 * the library until the process exits.  M is limited to
 * floor((MIRT_NOALLOC_SCRATCH_BYTES - 256) / (8 * (J1 + ... + JD) + 16))
 * samples (299,590 for J = 6 in 2D, 209,713 for J = 6 in 3D); larger M is
 * rejected with MIRT_ERR_ARG.  The first call on a device looks up the array's
 * device address and keeps it for the life of the process, so make that first
 * call before any stream capture; resetting a device (cudaDeviceReset) while
 * the library is loaded is not supported, since the kept address would then
 * be stale.  All calls share
 * the array, which keeps the last call's contents (every call rewrites what it
 * reads, so nothing needs clearing): calls that overlap on the GPU, on any
 * streams, race.
 *   tab[d]   device FP32 tables, float2 (complex, real_tab = 0) or float
 *            (real_tab = 1), J[d]*L[d]+1 entries
 *   tm       device FP64 [M, D] column-major, t = omega / (2 pi / K)
 *   ck       device float2 grid [K_D]...[K_1][ncol] (column innermost)
 *   fm       device float2 samples [M][ncol]
 * Asynchronous on `stream`. */
#define MIRT_NOALLOC_SCRATCH_BYTES (32u << 20)
int mirt_interp_gather_noalloc(int32_t D, const int32_t *K, const int32_t *J,
	const int32_t *L, const void *const *tab, int32_t real_tab, int32_t order,
	const double *tm, int64_t M, int32_t ncol, const void *ck, void *fm, void *stream);

/* Host FP64 builders used by mirt_nufft_create, exported for callers that
 * build their own plans (st.h{d} and the 1D factors of st.sn):
 *   table: length J*L+1 complex, nufft/nufft_table_init.m:111-134
 *   scale: length N complex,  nufft/nufft_scale.m:54-75 with
 *          nufft/nufft_alpha_kb_fit.m (st.sn = outer product of conj()). */
int mirt_minmax_kb_table(int32_t N, int32_t J, int32_t K, int32_t L,
	double *h_re, double *h_im);
int mirt_minmax_kb_scale(int32_t N, int32_t J, int32_t K,
	double *sn_re, double *sn_im);

#ifdef __cplusplus
}
#endif

#endif /* MIRT_B200_H */
