/*
 * oracle/interp_table.c -- CPU restatement of MIRT's table-based periodic
 * NUFFT interpolation (forward gather and adjoint scatter), FP64.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * kernels in mirt_b200/csrc; nothing in the product links or calls it.
 *
 * One generic routine covers D = 1..4, complex or real tables, and table
 * order 0 (nearest entry) or 1 (linear interpolation between entries).  The
 * per-tap arithmetic and the nesting of the partial sums follow the reference
 * kernels so that results agree bit for bit with them:
 *   forward  nufft/table/interp1_table1_for.c:19-64,70-120,126-180
 *            nufft/table/interp2_table1_for.c:24-99,106-191,198-287
 *            nufft/table/interp3_table1_for.c:24-130,134-252,258-380
 *            nufft/table/interp4_table1_for.c:30,168,325
 *   adjoint  nufft/table/interp1_table1_adj.c:20-64,69-118,123-177
 *            nufft/table/interp2_table1_adj.c:24-95,102-183,190-275
 *            nufft/table/interp3_table1_adj.c:24-121,127-237,243-361
 *            nufft/table/interp4_table1_adj.c:31,160,306
 * Shared definitions: mymod / iround, nufft/table/def,table2.h:7-8.
 *
 * Index selection (per sample m, dimension d, tap j = 0..J-1):
 *   koff = 1 + floor(t - J/2)          (t = tm[m + d*M], column-major [M,D])
 *   k    = koff + j
 *   p    = (t - k) * L                 (FP64, no fused multiply-add)
 *   order 0: n = floor(p + 0.5), coef = h[nc + n]
 *   order 1: n = floor(p), a = p - n, coef = (1-a) h[nc+n] + a h[nc+n+1]
 *   nc   = floor(J*L/2)                (table centre)
 *   grid index uses k mod K in [0, K), K1 fastest (MATLAB column-major).
 * Forward:  f_m = sum_jD h_D ( ... sum_j2 h_2 ( sum_j1 h_1 c[k] ) )
 * Adjoint:  c[k] += conj(h_1) conj(h_2) ... conj(h_D) f_m, with the
 *           conjugated product formed from the outermost dimension inward.
 */
#include <math.h>
#include <string.h>
#include <stdlib.h>

#define ORACLE_DMAX 4

typedef struct {
	int D, order, is_complex;
	int K[ORACLE_DMAX], J[ORACLE_DMAX], L[ORACLE_DMAX];
	const double *hr[ORACLE_DMAX]; /* centred table pointers */
	const double *hi[ORACLE_DMAX];
} spec_t;

/* coefficient of one tap: table lookup (order 0) or linear interp (order 1) */
static void tap_coef(const spec_t *s, int d, double t, int k, double *cr, double *ci)
{
	const double p = (t - (double)k) * (double)s->L[d];
	if (s->order == 0) {
		const int n = (int)floor(p + 0.5);
		*cr = s->hr[d][n];
		*ci = s->is_complex ? s->hi[d][n] : 0.0;
	} else {
		const int n = (int)floor(p);
		const double a = p - n;
		const double h0 = s->hr[d][n];
		/* the reference reads h[n+1] even when a == 0 at the table end;
		 * the product is zero there, so skip the read */
		const double h1 = (a != 0.0) ? s->hr[d][n + 1] : 0.0;
		*cr = (1 - a) * h0 + a * h1;
		*ci = 0.0;
	}
}

static int wrap(int k, int K)
{
	return (int)(k - K * floor(k / (double)K));
}

/* recursive forward partial sum over dimensions d, d-1, ..., 0 */
static void fwd_level(const spec_t *s, int d, const double *t, const int *koff,
	const double *r_ck, const double *i_ck, long base, long stride,
	double *out_r, double *out_i)
{
	double sr = 0, si = 0;
	int k = koff[d];
	for (int j = 0; j < s->J[d]; j++, k++) {
		double cr, ci;
		tap_coef(s, d, t[d], k, &cr, &ci);
		const long kk = base + (long)wrap(k, s->K[d]) * stride;
		double vr, vi;
		if (d == 0) {
			vr = r_ck[kk];
			vi = i_ck[kk];
		} else {
			fwd_level(s, d - 1, t, koff, r_ck, i_ck, kk, stride / s->K[d - 1], &vr, &vi);
		}
		if (s->is_complex) {
			sr += cr * vr - ci * vi;
			si += cr * vi + ci * vr;
		} else {
			sr += cr * vr;
			si += cr * vi;
		}
	}
	*out_r = sr;
	*out_i = si;
}

/* recursive adjoint scatter: v = conj(h_d) * v_in pushed to level d-1 */
static void adj_level(const spec_t *s, int d, const double *t, const int *koff,
	double *r_ck, double *i_ck, long base, long stride, double vr, double vi)
{
	int k = koff[d];
	for (int j = 0; j < s->J[d]; j++, k++) {
		double cr, ci;
		tap_coef(s, d, t[d], k, &cr, &ci);
		const long kk = base + (long)wrap(k, s->K[d]) * stride;
		double wr, wi;
		if (s->is_complex) {
			wr = cr * vr + ci * vi;
			wi = cr * vi - ci * vr;
		} else {
			wr = cr * vr;
			wi = cr * vi;
		}
		if (d == 0) {
			r_ck[kk] += wr;
			i_ck[kk] += wi;
		} else {
			adj_level(s, d - 1, t, koff, r_ck, i_ck, kk, stride / s->K[d - 1], wr, wi);
		}
	}
}

static int setup(spec_t *s, int D, const int *K, const double *const *hr,
	const double *const *hi, const int *J, const int *L, int order)
{
	if (D < 1 || D > ORACLE_DMAX) return -1;
	memset(s, 0, sizeof(*s));
	s->D = D;
	s->order = order;
	s->is_complex = (hi != NULL && hi[0] != NULL);
	if (s->is_complex && order != 0) return -2;
	for (int d = 0; d < D; d++) {
		const int nc = (int)floor(J[d] * L[d] / 2.);
		s->K[d] = K[d];
		s->J[d] = J[d];
		s->L[d] = L[d];
		s->hr[d] = hr[d] + nc;
		s->hi[d] = s->is_complex ? hi[d] + nc : NULL;
	}
	return 0;
}

static long grid_size(const spec_t *s)
{
	long n = 1;
	for (int d = 0; d < s->D; d++) n *= s->K[d];
	return n;
}

/* one column: f[m] for m = 0..M-1 */
int oracle_interp_for(int D, const int *K, const double *const *hr,
	const double *const *hi, const int *J, const int *L, int order,
	const double *tm, int M, const double *r_ck, const double *i_ck,
	double *r_fm, double *i_fm)
{
	spec_t s;
	int rc = setup(&s, D, K, hr, hi, J, L, order);
	if (rc) return rc;
	const long top_stride = grid_size(&s) / s.K[D - 1];
	for (int m = 0; m < M; m++) {
		double t[ORACLE_DMAX];
		int koff[ORACLE_DMAX];
		for (int d = 0; d < D; d++) {
			t[d] = tm[m + (long)d * M];
			koff[d] = 1 + (int)floor(t[d] - s.J[d] / 2.);
		}
		fwd_level(&s, D - 1, t, koff, r_ck, i_ck, 0, top_stride, &r_fm[m], &i_fm[m]);
	}
	return 0;
}

/* one column: c = sum over samples; output zeroed first */
int oracle_interp_adj(int D, const int *K, const double *const *hr,
	const double *const *hi, const int *J, const int *L, int order,
	const double *tm, int M, const double *r_fm, const double *i_fm,
	double *r_ck, double *i_ck)
{
	spec_t s;
	int rc = setup(&s, D, K, hr, hi, J, L, order);
	if (rc) return rc;
	const long n = grid_size(&s);
	memset(r_ck, 0, n * sizeof(double));
	memset(i_ck, 0, n * sizeof(double));
	const long top_stride = n / s.K[D - 1];
	for (int m = 0; m < M; m++) {
		double t[ORACLE_DMAX];
		int koff[ORACLE_DMAX];
		for (int d = 0; d < D; d++) {
			t[d] = tm[m + (long)d * M];
			koff[d] = 1 + (int)floor(t[d] - s.J[d] / 2.);
		}
		adj_level(&s, D - 1, t, koff, r_ck, i_ck, 0, top_stride, r_fm[m], i_fm[m]);
	}
	return 0;
}
