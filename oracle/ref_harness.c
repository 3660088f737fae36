/*
 * oracle/ref_harness.c -- drives the reference's own, unmodified table
 * interpolation kernels (nufft/table/interp{1,2,3,4}_table1_{for,adj}.c, built
 * from the reference sources into oracle/_ref/libmirt_ref.so) with the mex
 * gateways' column semantics.
 *
 * TEST INFRASTRUCTURE AND CPU BASELINE ONLY: used by tests/ as the bit-level
 * FP64 pin of the oracle restatement, and by bench.py's CPU-baseline leg.
 *
 * The gateways run the kernel once per column (coil) serially:
 *   nufft/table/interp2_table_mex.c:87-95 (complex h), :110-121 (real h)
 *   nufft/table/interp2_table_adj_mex.c:90-98, :113-124
 *   nufft/table/interp1_table_mex.c, interp3_table_mex.c, interp4_table_mex.c (same pattern)
 * ref_interp_cols() keeps that per-column call and, when nthreads > 1, hands
 * whole columns to POSIX threads; the kernels themselves are unchanged.
 */
#include <stddef.h>
#include <pthread.h>
#include <unistd.h>

/* reference kernel prototypes (nufft/table/def,table{1,2,3}.h, built
 * without Provide_flip as the reference's own build does) */
void interp1_table0_complex_per(const double *, const double *, int,
	const double *, const double *, int, int, const double *, int, double *, double *);
void interp1_table0_real_per(const double *, const double *, int,
	const double *, int, int, const double *, int, double *, double *);
void interp1_table1_real_per(const double *, const double *, int,
	const double *, int, int, const double *, int, double *, double *);
void interp1_table0_complex_per_adj(double *, double *, int,
	const double *, const double *, int, int, const double *, int, const double *, const double *);
void interp1_table0_real_per_adj(double *, double *, int,
	const double *, int, int, const double *, int, const double *, const double *);
void interp1_table1_real_per_adj(double *, double *, int,
	const double *, int, int, const double *, int, const double *, const double *);

void interp2_table0_complex_per(const double *, const double *, int, int,
	const double *, const double *, const double *, const double *,
	int, int, int, int, const double *, int, double *, double *);
void interp2_table0_real_per(const double *, const double *, int, int,
	const double *, const double *, int, int, int, int, const double *, int, double *, double *);
void interp2_table1_real_per(const double *, const double *, int, int,
	const double *, const double *, int, int, int, int, const double *, int, double *, double *);
void interp2_table0_complex_per_adj(double *, double *, int, int,
	const double *, const double *, const double *, const double *,
	int, int, int, int, const double *, int, const double *, const double *);
void interp2_table0_real_per_adj(double *, double *, int, int,
	const double *, const double *, int, int, int, int, const double *, int, const double *, const double *);
void interp2_table1_real_per_adj(double *, double *, int, int,
	const double *, const double *, int, int, int, int, const double *, int, const double *, const double *);

void interp3_table0_complex_per(const double *, const double *, int, int, int,
	const double *, const double *, const double *, const double *, const double *, const double *,
	int, int, int, int, int, int, const double *, int, double *, double *);
void interp3_table0_real_per(const double *, const double *, int, int, int,
	const double *, const double *, const double *,
	int, int, int, int, int, int, const double *, int, double *, double *);
void interp3_table1_real_per(const double *, const double *, int, int, int,
	const double *, const double *, const double *,
	int, int, int, int, int, int, const double *, int, double *, double *);
void interp3_table0_complex_per_adj(double *, double *, int, int, int,
	const double *, const double *, const double *, const double *, const double *, const double *,
	int, int, int, int, int, int, const double *, int, const double *, const double *);
void interp3_table0_real_per_adj(double *, double *, int, int, int,
	const double *, const double *, const double *,
	int, int, int, int, int, int, const double *, int, const double *, const double *);
void interp3_table1_real_per_adj(double *, double *, int, int, int,
	const double *, const double *, const double *,
	int, int, int, int, int, int, const double *, int, const double *, const double *);

void interp4_table0_complex_per(const double *, const double *, int, int, int, int,
	const double *, const double *, const double *, const double *, const double *, const double *,
	const double *, const double *,
	int, int, int, int, int, int, int, int, const double *, int, double *, double *);
void interp4_table0_real_per(const double *, const double *, int, int, int, int,
	const double *, const double *, const double *, const double *,
	int, int, int, int, int, int, int, int, const double *, int, double *, double *);
void interp4_table1_real_per(const double *, const double *, int, int, int, int,
	const double *, const double *, const double *, const double *,
	int, int, int, int, int, int, int, int, const double *, int, double *, double *);
void interp4_table0_complex_per_adj(double *, double *, int, int, int, int,
	const double *, const double *, const double *, const double *, const double *, const double *,
	const double *, const double *,
	int, int, int, int, int, int, int, int, const double *, int, const double *, const double *);
void interp4_table0_real_per_adj(double *, double *, int, int, int, int,
	const double *, const double *, const double *, const double *,
	int, int, int, int, int, int, int, int, const double *, int, const double *, const double *);
void interp4_table1_real_per_adj(double *, double *, int, int, int, int,
	const double *, const double *, const double *, const double *,
	int, int, int, int, int, int, int, int, const double *, int, const double *, const double *);

/* One column through the reference kernel that the gateway would pick.
 * Returns 0, or -1 for an unsupported (D, order, complex) combination. */
static int one_col(int adj, int D, const int *K, const double *const *hr,
	const double *const *hi, const int *J, const int *L, int order,
	const double *tm, int M,
	double *r_ck, double *i_ck, double *r_fm, double *i_fm)
{
	const int cx = (hi != NULL && hi[0] != NULL);
	if (cx && order != 0) return -1;
	if (order != 0 && order != 1) return -1;
	if (D == 1) {
		if (!adj) {
			if (cx) interp1_table0_complex_per(r_ck, i_ck, K[0], hr[0], hi[0], J[0], L[0], tm, M, r_fm, i_fm);
			else if (order == 0) interp1_table0_real_per(r_ck, i_ck, K[0], hr[0], J[0], L[0], tm, M, r_fm, i_fm);
			else interp1_table1_real_per(r_ck, i_ck, K[0], hr[0], J[0], L[0], tm, M, r_fm, i_fm);
		} else {
			if (cx) interp1_table0_complex_per_adj(r_ck, i_ck, K[0], hr[0], hi[0], J[0], L[0], tm, M, r_fm, i_fm);
			else if (order == 0) interp1_table0_real_per_adj(r_ck, i_ck, K[0], hr[0], J[0], L[0], tm, M, r_fm, i_fm);
			else interp1_table1_real_per_adj(r_ck, i_ck, K[0], hr[0], J[0], L[0], tm, M, r_fm, i_fm);
		}
	} else if (D == 2) {
		if (!adj) {
			if (cx) interp2_table0_complex_per(r_ck, i_ck, K[0], K[1], hr[0], hi[0], hr[1], hi[1],
				J[0], J[1], L[0], L[1], tm, M, r_fm, i_fm);
			else if (order == 0) interp2_table0_real_per(r_ck, i_ck, K[0], K[1], hr[0], hr[1],
				J[0], J[1], L[0], L[1], tm, M, r_fm, i_fm);
			else interp2_table1_real_per(r_ck, i_ck, K[0], K[1], hr[0], hr[1],
				J[0], J[1], L[0], L[1], tm, M, r_fm, i_fm);
		} else {
			if (cx) interp2_table0_complex_per_adj(r_ck, i_ck, K[0], K[1], hr[0], hi[0], hr[1], hi[1],
				J[0], J[1], L[0], L[1], tm, M, r_fm, i_fm);
			else if (order == 0) interp2_table0_real_per_adj(r_ck, i_ck, K[0], K[1], hr[0], hr[1],
				J[0], J[1], L[0], L[1], tm, M, r_fm, i_fm);
			else interp2_table1_real_per_adj(r_ck, i_ck, K[0], K[1], hr[0], hr[1],
				J[0], J[1], L[0], L[1], tm, M, r_fm, i_fm);
		}
	} else if (D == 3) {
		if (!adj) {
			if (cx) interp3_table0_complex_per(r_ck, i_ck, K[0], K[1], K[2],
				hr[0], hi[0], hr[1], hi[1], hr[2], hi[2],
				J[0], J[1], J[2], L[0], L[1], L[2], tm, M, r_fm, i_fm);
			else if (order == 0) interp3_table0_real_per(r_ck, i_ck, K[0], K[1], K[2],
				hr[0], hr[1], hr[2], J[0], J[1], J[2], L[0], L[1], L[2], tm, M, r_fm, i_fm);
			else interp3_table1_real_per(r_ck, i_ck, K[0], K[1], K[2],
				hr[0], hr[1], hr[2], J[0], J[1], J[2], L[0], L[1], L[2], tm, M, r_fm, i_fm);
		} else {
			if (cx) interp3_table0_complex_per_adj(r_ck, i_ck, K[0], K[1], K[2],
				hr[0], hi[0], hr[1], hi[1], hr[2], hi[2],
				J[0], J[1], J[2], L[0], L[1], L[2], tm, M, r_fm, i_fm);
			else if (order == 0) interp3_table0_real_per_adj(r_ck, i_ck, K[0], K[1], K[2],
				hr[0], hr[1], hr[2], J[0], J[1], J[2], L[0], L[1], L[2], tm, M, r_fm, i_fm);
			else interp3_table1_real_per_adj(r_ck, i_ck, K[0], K[1], K[2],
				hr[0], hr[1], hr[2], J[0], J[1], J[2], L[0], L[1], L[2], tm, M, r_fm, i_fm);
		}
	} else if (D == 4) {
		/* nufft/table/interp4_table_mex.c:117-160, interp4_table_adj_mex.c:120-160 */
		if (!adj) {
			if (cx) interp4_table0_complex_per(r_ck, i_ck, K[0], K[1], K[2], K[3],
				hr[0], hi[0], hr[1], hi[1], hr[2], hi[2], hr[3], hi[3],
				J[0], J[1], J[2], J[3], L[0], L[1], L[2], L[3], tm, M, r_fm, i_fm);
			else if (order == 0) interp4_table0_real_per(r_ck, i_ck, K[0], K[1], K[2], K[3],
				hr[0], hr[1], hr[2], hr[3],
				J[0], J[1], J[2], J[3], L[0], L[1], L[2], L[3], tm, M, r_fm, i_fm);
			else interp4_table1_real_per(r_ck, i_ck, K[0], K[1], K[2], K[3],
				hr[0], hr[1], hr[2], hr[3],
				J[0], J[1], J[2], J[3], L[0], L[1], L[2], L[3], tm, M, r_fm, i_fm);
		} else {
			if (cx) interp4_table0_complex_per_adj(r_ck, i_ck, K[0], K[1], K[2], K[3],
				hr[0], hi[0], hr[1], hi[1], hr[2], hi[2], hr[3], hi[3],
				J[0], J[1], J[2], J[3], L[0], L[1], L[2], L[3], tm, M, r_fm, i_fm);
			else if (order == 0) interp4_table0_real_per_adj(r_ck, i_ck, K[0], K[1], K[2], K[3],
				hr[0], hr[1], hr[2], hr[3],
				J[0], J[1], J[2], J[3], L[0], L[1], L[2], L[3], tm, M, r_fm, i_fm);
			else interp4_table1_real_per_adj(r_ck, i_ck, K[0], K[1], K[2], K[3],
				hr[0], hr[1], hr[2], hr[3],
				J[0], J[1], J[2], J[3], L[0], L[1], L[2], L[3], tm, M, r_fm, i_fm);
		}
	} else {
		return -1;
	}
	return 0;
}

typedef struct {
	int adj, D, order, M, N, nthreads, tid, bad;
	const int *K, *J, *L;
	const double *const *hr;
	const double *const *hi;
	const double *tm;
	long nk;
	double *r_ck, *i_ck, *r_fm, *i_fm;
} job_t;

static void *run_cols(void *arg)
{
	job_t *j = (job_t *)arg;
	for (int n = j->tid; n < j->N; n += j->nthreads)
		j->bad |= one_col(j->adj, j->D, j->K, j->hr, j->hi, j->J, j->L, j->order,
			j->tm, j->M, j->r_ck + n * j->nk, j->i_ck + n * j->nk,
			j->r_fm + (long)n * j->M, j->i_fm + (long)n * j->M);
	return NULL;
}

/*
 * N columns: ck is [prod(K), N] and fm is [M, N], split real/imag, column-major.
 * adj = 0: fm = interp(ck); adj = 1: ck = interp_adj(fm).
 * nthreads <= 1 reproduces the gateway's serial loop exactly; otherwise
 * column n goes to thread n % nthreads.
 */
int ref_interp_cols(int adj, int D, const int *K, const double *const *hr,
	const double *const *hi, const int *J, const int *L, int order,
	const double *tm, int M, int N,
	double *r_ck, double *i_ck, double *r_fm, double *i_fm, int nthreads)
{
	long nk = 1;
	for (int d = 0; d < D; d++) nk *= K[d];
	if (nthreads > N) nthreads = N;
	if (nthreads < 1) nthreads = 1;
	enum { TMAX = 256 };
	if (nthreads > TMAX) nthreads = TMAX;
	job_t jobs[TMAX];
	pthread_t th[TMAX];
	for (int t = 0; t < nthreads; t++) {
		job_t j = { adj, D, order, M, N, nthreads, t, 0, K, J, L, hr, hi, tm, nk,
			r_ck, i_ck, r_fm, i_fm };
		jobs[t] = j;
	}
	if (nthreads == 1) {
		run_cols(&jobs[0]);
		return jobs[0].bad ? -1 : 0;
	}
	for (int t = 0; t < nthreads; t++)
		pthread_create(&th[t], NULL, run_cols, &jobs[t]);
	int bad = 0;
	for (int t = 0; t < nthreads; t++) {
		pthread_join(th[t], NULL);
		bad |= jobs[t].bad;
	}
	return bad ? -1 : 0;
}

int ref_max_threads(void)
{
	return (int)sysconf(_SC_NPROCESSORS_ONLN);
}
