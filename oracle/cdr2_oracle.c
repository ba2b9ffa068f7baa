/*
 * cdr2_oracle.c -- CPU restatement of Cedar's serial 2D BoxMG path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the CUDA
 * kernels of cedar_b200.  Only tests, the smoke check and the CPU-baseline
 * leg of the benchmark may load it; the product path never calls it.
 *
 * Every routine restates one reference routine, cited by file:line of the
 * reference project (cedar-framework/cedar).  Arrays use the reference's
 * layout: Fortran order, one ghost ring, i fastest, one contiguous plane per
 * stencil direction.  Indices inside the routines are the reference's 1-based
 * Fortran indices so each statement can be read against the source.
 * Compile with -ffp-contract=off so no fused multiply-add changes rounding
 * (the reference's Fortran is built for baseline x86-64, which has no FMA).
 *
 * The LAPACK routines the reference calls (DPTTRF/DPTTRS, DPBTRF/DPBTRS) are
 * restated from the published reference-LAPACK algorithms (LAPACK 3.x,
 * version unpinned by the reference: CMakeLists.txt:57-58):
 *   DPTTRF  L*D*L^T of an SPD tridiagonal, e(i) <- e(i)/d(i),
 *           d(i+1) <- d(i+1) - e(i)*e_old(i);
 *   DPTTS2  forward L, then b(i) <- b(i)/d(i) - b(i+1)*e(i);
 *   DPBTF2  unblocked upper band Cholesky (DPBTRF takes it when KD < 32);
 *   DTBSV   upper band triangular solves used by DPBTRS.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <unistd.h>

#include "cdr2_oracle.h"

/* stencil plane numbers, src/2d/ftn/BMG_stencils_f90.h:30 */
enum { KO = 1, KW = 2, KS = 3, KSW = 4, KNW = 5 };
/* interpolation planes, src/2d/ftn/BMG_stencils_f90.h:37 */
enum { LL = 1, LR = 2, LA = 3, LB = 4, LSW = 5, LNW = 6, LNE = 7, LSE = 8 };
/* include/cedar/2d/ftn/BMG_parameters_c.h:240-244 */
enum { BMG_DOWN = 0, BMG_UP = 1 };

static inline size_t ix2(long i, long j, long ii) { return (size_t)(j - 1) * ii + (i - 1); }
static inline size_t ix3(long i, long j, long k, long ii, long jj)
{
	return ((size_t)(k - 1) * jj + (j - 1)) * ii + (i - 1);
}

/* ------------------------------------------------------------------ */
/* Host threads                                                        */
/* ------------------------------------------------------------------ */
/* The cycle kernels split independent rows, or lines of one colour, over the
 * host's cores.  Every element receives the same operations whatever the
 * split, so no result depends on the thread count.  ORACLE_THREADS (else
 * OMP_NUM_THREADS, else the online CPUs) sets the count; grids under 2^18
 * points stay on the calling thread. */
typedef void (*o_task_fn)(void *ctx, int t);
struct o_chunk {
	o_task_fn fn;
	void *ctx;
	int t0, t1;
};

static void *o_chunk_run(void *p)
{
	struct o_chunk *c = (struct o_chunk *)p;
	for (int t = c->t0; t < c->t1; ++t) c->fn(c->ctx, t);
	return NULL;
}

static int o_threads_set = 0;

/* Thread count for the following calls (0: back to the environment's). */
void o_set_threads(int n) { o_threads_set = n < 0 ? 0 : n > 64 ? 64 : n; }

int o_num_threads(void)
{
	static int n = 0;
	if (o_threads_set) return o_threads_set;
	if (!n) {
		const char *e = getenv("ORACLE_THREADS");
		if (!e) e = getenv("OMP_NUM_THREADS");
		long v = e ? atol(e) : sysconf(_SC_NPROCESSORS_ONLN);
		n = v < 1 ? 1 : v > 64 ? 64 : (int)v;
	}
	return n;
}

/* tasks 0..ntasks-1 of fn, over the threads when the grid has `points` points */
static void o_parallel(int ntasks, long points, o_task_fn fn, void *ctx)
{
	int T = o_num_threads();
	if (T > ntasks) T = ntasks;
	if (T <= 1 || points < (1L << 18)) {
		for (int t = 0; t < ntasks; ++t) fn(ctx, t);
		return;
	}
	pthread_t th[64];
	int ok[64];
	struct o_chunk ch[64];
	for (int k = 0; k < T; ++k) {
		ch[k].fn = fn;
		ch[k].ctx = ctx;
		ch[k].t0 = (int)((long)ntasks * k / T);
		ch[k].t1 = (int)((long)ntasks * (k + 1) / T);
	}
	for (int k = 1; k < T; ++k) ok[k] = pthread_create(&th[k], NULL, o_chunk_run, &ch[k]) == 0;
	o_chunk_run(&ch[0]);
	for (int k = 1; k < T; ++k) {
		if (ok[k]) pthread_join(th[k], NULL);
		else o_chunk_run(&ch[k]);
	}
}

/* ------------------------------------------------------------------ */
/* LAPACK restatements                                                 */
/* ------------------------------------------------------------------ */

/* DPTTRF: factor SPD tridiagonal (d: n diagonal, e: n-1 off-diagonal). */
int o_dpttrf(int n, double *d, double *e)
{
	if (n <= 0) return 0;
	for (int i = 0; i < n - 1; ++i) {
		if (d[i] <= 0.0) return i + 1;
		double ei = e[i];
		e[i] = ei / d[i];
		d[i + 1] = d[i + 1] - e[i] * ei;
	}
	if (d[n - 1] <= 0.0) return n;
	return 0;
}

/* DPTTRS (one right-hand side) through DPTTS2. */
void o_dpttrs(int n, const double *d, const double *e, double *b)
{
	if (n <= 1) {
		if (n == 1) b[0] = (1.0 / d[0]) * b[0];
		return;
	}
	for (int i = 1; i < n; ++i)
		b[i] = b[i] - b[i - 1] * e[i - 1];
	b[n - 1] = b[n - 1] / d[n - 1];
	for (int i = n - 2; i >= 0; --i)
		b[i] = b[i] / d[i] - b[i + 1] * e[i];
}

/* DPBTRF('U') for KD < 32, i.e. DPBTF2.  ab(ldab, n) column-major. */
int o_dpbtrf_u(int n, int kd, double *ab, int ldab)
{
#define AB(r, c) ab[(size_t)((c) - 1) * ldab + ((r) - 1)]
	int kld = ldab - 1 > 1 ? ldab - 1 : 1;
	for (int j = 1; j <= n; ++j) {
		double ajj = AB(kd + 1, j);
		if (ajj <= 0.0) return j;
		ajj = sqrt(ajj);
		AB(kd + 1, j) = ajj;
		int kn = kd < n - j ? kd : n - j;
		if (kn > 0) {
			/* DSCAL(kn, 1/ajj, AB(kd, j+1), kld) */
			double rcp = 1.0 / ajj;
			double *x = &AB(kd, j + 1);
			for (int p = 0; p < kn; ++p) x[(size_t)p * kld] = rcp * x[(size_t)p * kld];
			/* DSYR('U', kn, -1, x, kld, AB(kd+1, j+1), kld) */
			double *a = &AB(kd + 1, j + 1);
			for (int q = 0; q < kn; ++q) {
				double xq = x[(size_t)q * kld];
				if (xq != 0.0) {
					double temp = -1.0 * xq;
					for (int p = 0; p <= q; ++p)
						a[(size_t)p + (size_t)q * kld] = a[(size_t)p + (size_t)q * kld] + x[(size_t)p * kld] * temp;
				}
			}
		}
	}
	return 0;
#undef AB
}

/* DPBTRS('U', n, kd, 1 rhs): DTBSV upper-transpose then upper-no-transpose. */
void o_dpbtrs_u(int n, int kd, const double *ab, int ldab, double *x)
{
#define AB(r, c) ab[(size_t)((c) - 1) * ldab + ((r) - 1)]
#define X(i) x[(i) - 1]
	int kplus1 = kd + 1;
	for (int j = 1; j <= n; ++j) {
		double temp = X(j);
		int l = kplus1 - j;
		int i0 = j - kd > 1 ? j - kd : 1;
		for (int i = i0; i <= j - 1; ++i)
			temp = temp - AB(l + i, j) * X(i);
		temp = temp / AB(kplus1, j);
		X(j) = temp;
	}
	for (int j = n; j >= 1; --j) {
		if (X(j) != 0.0) {
			int l = kplus1 - j;
			X(j) = X(j) / AB(kplus1, j);
			double temp = X(j);
			int i1 = j - kd > 1 ? j - kd : 1;
			for (int i = j - 1; i >= i1; --i)
				X(i) = X(i) - temp * AB(l + i, j);
		}
	}
#undef AB
#undef X
}

/* ------------------------------------------------------------------ */
/* 2D kernels (non-periodic boundary branch)                           */
/* ------------------------------------------------------------------ */

struct o2_resid_ctx {
	const double *so, *qf, *q;
	double *res;
	int II, JJ, ifd;
};

static void o2_residual_row(void *vc, int t)
{
	const struct o2_resid_ctx *c = (const struct o2_resid_ctx *)vc;
	const double *so = c->so, *qf = c->qf, *q = c->q;
	double *res = c->res;
	const int II = c->II, JJ = c->JJ, I1 = II - 1, J = t + 2;
#define SO(i, j, k) so[ix3(i, j, k, II, JJ)]
#define Q(i, j) q[ix2(i, j, II)]
#define QF(i, j) qf[ix2(i, j, II)]
#define RES(i, j) res[ix2(i, j, II)]
	if (c->ifd != 1) {
		for (int I = 2; I <= I1; ++I)
			RES(I, J) = QF(I, J)
			          + SO(I, J, KW) * Q(I - 1, J)
			          + SO(I + 1, J, KW) * Q(I + 1, J)
			          + SO(I, J, KS) * Q(I, J - 1)
			          + SO(I, J + 1, KS) * Q(I, J + 1)
			          + SO(I, J, KSW) * Q(I - 1, J - 1)
			          + SO(I + 1, J, KNW) * Q(I + 1, J - 1)
			          + SO(I, J + 1, KNW) * Q(I - 1, J + 1)
			          + SO(I + 1, J + 1, KSW) * Q(I + 1, J + 1)
			          - SO(I, J, KO) * Q(I, J);
	} else {
		for (int I = 2; I <= I1; ++I)
			RES(I, J) = QF(I, J)
			          + SO(I, J, KW) * Q(I - 1, J)
			          + SO(I + 1, J, KW) * Q(I + 1, J)
			          + SO(I, J, KS) * Q(I, J - 1)
			          + SO(I, J + 1, KS) * Q(I, J + 1)
			          - SO(I, J, KO) * Q(I, J);
	}
#undef SO
#undef Q
#undef QF
#undef RES
}

/* BMG2_SymStd_residual, src/2d/ftn/BMG2_SymStd_residual.f90:85-119 (rows in any order) */
void o2_residual(const double *so, const double *qf, const double *q, double *res,
                 int II, int JJ, int ifd)
{
	struct o2_resid_ctx c = {so, qf, q, res, II, JJ, ifd};
	o_parallel(JJ - 2, (long)II * JJ, o2_residual_row, &c);
}

/* BMG2_SymStd_SETUP_recip, src/2d/ftn/BMG2_SymStd_SETUP_recip.f90:63-67 (MSOR = 2) */
void o2_setup_recip(const double *so, double *sor, int II, int JJ)
{
	for (int j = 2; j <= JJ - 1; ++j)
		for (int i = 2; i <= II - 1; ++i)
			sor[ix3(i, j, 2, II, JJ)] = 1.0 / so[ix3(i, j, KO, II, JJ)];
}

struct o2_gs_ctx {
	const double *so, *qf, *sor;
	double *q;
	int II, JJ, lstart, lend, lstride, beg;
};

/* 9-point: row J = beg + 2t of the row colour, both point colours in order */
static void o2_gs9_row(void *vc, int t)
{
	const struct o2_gs_ctx *c = (const struct o2_gs_ctx *)vc;
	const double *so = c->so, *qf = c->qf, *sor = c->sor;
	double *q = c->q;
	const int II = c->II, JJ = c->JJ, I1 = II - 1, J = c->beg + 2 * t;
#define SO(i, j, k) so[ix3(i, j, k, II, JJ)]
#define Q(i, j) q[ix2(i, j, II)]
#define QF(i, j) qf[ix2(i, j, II)]
#define SOR(i, j) sor[ix3(i, j, 2, II, JJ)]
	for (int IBEG = c->lstart; c->lstride > 0 ? IBEG <= c->lend : IBEG >= c->lend; IBEG += c->lstride) {
		int IEND = 2 * ((I1 - IBEG) / 2) + IBEG;
		for (int I = IBEG; I <= IEND; I += 2)
			Q(I, J) = (QF(I, J)
			           + SO(I, J, KW) * Q(I - 1, J)
			           + SO(I + 1, J, KW) * Q(I + 1, J)
			           + SO(I, J, KS) * Q(I, J - 1)
			           + SO(I, J + 1, KS) * Q(I, J + 1)
			           + SO(I, J, KSW) * Q(I - 1, J - 1)
			           + SO(I + 1, J, KNW) * Q(I + 1, J - 1)
			           + SO(I, J + 1, KNW) * Q(I - 1, J + 1)
			           + SO(I + 1, J + 1, KSW) * Q(I + 1, J + 1)) * SOR(I, J);
	}
}

/* 5-point: the colour-JO points of row J = t + 2 */
static void o2_gs5_row(void *vc, int t)
{
	const struct o2_gs_ctx *c = (const struct o2_gs_ctx *)vc;
	const double *so = c->so, *qf = c->qf, *sor = c->sor;
	double *q = c->q;
	const int II = c->II, JJ = c->JJ, I1 = II - 1, J = t + 2;
	int IBEG = (J + c->beg) % 2 + 2;
	int IEND = 2 * ((I1 - IBEG) / 2) + IBEG;
	for (int I = IBEG; I <= IEND; I += 2)
		Q(I, J) = (QF(I, J)
		           + SO(I, J, KW) * Q(I - 1, J)
		           + SO(I + 1, J, KW) * Q(I + 1, J)
		           + SO(I, J, KS) * Q(I, J - 1)
		           + SO(I, J + 1, KS) * Q(I, J + 1)) * SOR(I, J);
#undef SO
#undef Q
#undef QF
#undef SOR
}

/* BMG2_SymStd_relax_GS, src/2d/ftn/BMG2_SymStd_relax_GS.f90:68-137.  Rows of
 * one row colour (9-point) or the points of one colour (5-point) read only
 * the other colour: any order of them gives the same values. */
void o2_relax_gs(const double *so, const double *qf, double *q, const double *sor,
                 int II, int JJ, int ifd, int updown)
{
	int J1 = JJ - 1;
	struct o2_gs_ctx c = {so, qf, sor, q, II, JJ, 0, 0, 0, 0};
	if (updown == BMG_DOWN) { c.lstart = 2; c.lend = 3; c.lstride = 1; }
	else { c.lstart = 3; c.lend = 2; c.lstride = -1; }
	if (ifd != 1) {
		for (int JBEG = c.lstart; c.lstride > 0 ? JBEG <= c.lend : JBEG >= c.lend; JBEG += c.lstride) {
			int JEND = 2 * ((J1 - JBEG) / 2) + JBEG;
			c.beg = JBEG;
			o_parallel((JEND - JBEG) / 2 + 1, (long)II * JJ, o2_gs9_row, &c);
		}
	} else {
		for (int JO = c.lstart; c.lstride > 0 ? JO <= c.lend : JO >= c.lend; JO += c.lstride) {
			c.beg = JO;
			o_parallel(JJ - 2, (long)II * JJ, o2_gs5_row, &c);
		}
	}
}

/* BMG2_SymStd_SETUP_lines_x, src/2d/ftn/BMG2_SymStd_SETUP_lines_x.f90:68-87.
 * sor(Nx,Ny,2): plane 1 = D of L*D*L^T, plane 2 = multipliers (from i=3). */
int o2_setup_lines_x(const double *so, double *sor, int Nx, int Ny)
{
	int info = 0;
	for (int j = 2; j <= Ny - 1; ++j)
		for (int i = 2; i <= Nx - 1; ++i) {
			sor[ix3(i, j, 2, Nx, Ny)] = -so[ix3(i, j, KW, Nx, Ny)];
			sor[ix3(i, j, 1, Nx, Ny)] = so[ix3(i, j, KO, Nx, Ny)];
		}
	for (int j = 2; j <= Ny - 1; ++j) {
		int r = o_dpttrf(Nx - 2, &sor[ix3(2, j, 1, Nx, Ny)], &sor[ix3(3, j, 2, Nx, Ny)]);
		if (r && !info) info = r;
	}
	return info;
}

/* BMG2_SymStd_SETUP_lines_y, src/2d/ftn/BMG2_SymStd_SETUP_lines_y.f90:69-88.
 * sor is stored transposed: (Ny,Nx,2). */
int o2_setup_lines_y(const double *so, double *sor, int Nx, int Ny)
{
	int info = 0;
	for (int i = 2; i <= Nx - 1; ++i)
		for (int j = 2; j <= Ny - 1; ++j) {
			sor[ix3(j, i, 2, Ny, Nx)] = -so[ix3(i, j, KS, Nx, Ny)];
			sor[ix3(j, i, 1, Ny, Nx)] = so[ix3(i, j, KO, Nx, Ny)];
		}
	for (int i = 2; i <= Nx - 1; ++i) {
		int r = o_dpttrf(Ny - 2, &sor[ix3(2, i, 1, Ny, Nx)], &sor[ix3(3, i, 2, Ny, Nx)]);
		if (r && !info) info = r;
	}
	return info;
}

struct o2_lines_ctx {
	const double *so, *qf, *sor;
	double *q;
	int II, JJ, ifd, beg;
};

/* x-line J = beg + 2t: right-hand side into Q(., J), then DPTTRS */
static void o2_xline(void *vc, int t)
{
	const struct o2_lines_ctx *c = (const struct o2_lines_ctx *)vc;
	const double *so = c->so, *qf = c->qf, *sor = c->sor;
	double *q = c->q;
	const int II = c->II, JJ = c->JJ, I1 = II - 1, J = c->beg + 2 * t;
#define SO(i, j, k) so[ix3(i, j, k, II, JJ)]
#define Q(i, j) q[ix2(i, j, II)]
#define QF(i, j) qf[ix2(i, j, II)]
	if (c->ifd != 1) {
		for (int I = 2; I <= I1; ++I)
			Q(I, J) = QF(I, J) + SO(I, J, KS) * Q(I, J - 1) + SO(I, J + 1, KS) * Q(I, J + 1)
			        + SO(I, J, KSW) * Q(I - 1, J - 1) + SO(I + 1, J, KNW) * Q(I + 1, J - 1)
			        + SO(I, J + 1, KNW) * Q(I - 1, J + 1) + SO(I + 1, J + 1, KSW) * Q(I + 1, J + 1);
	} else {
		for (int I = 2; I <= I1; ++I)
			Q(I, J) = QF(I, J) + SO(I, J, KS) * Q(I, J - 1) + SO(I, J + 1, KS) * Q(I, J + 1);
	}
	o_dpttrs(I1 - 1, &sor[ix3(2, J, 1, II, JJ)], &sor[ix3(3, J, 2, II, JJ)], &Q(2, J));
#undef SO
#undef Q
#undef QF
}

/* BMG2_SymStd_relax_lines_x, src/2d/ftn/BMG2_SymStd_relax_lines_x.f90:74-131.
 * The reference forms all right-hand sides of a colour, then solves; lines of
 * one colour read only the other colour, so line by line gives the same. */
void o2_relax_lines_x(const double *so, const double *qf, double *q, const double *sor,
                      int II, int JJ, int ifd, int updown)
{
	int J1 = JJ - 1;
	int jstart, jend, jstride;
	if (updown == BMG_DOWN) { jstart = 3; jend = 2; jstride = -1; }
	else { jstart = 2; jend = 3; jstride = 1; }
	struct o2_lines_ctx c = {so, qf, sor, q, II, JJ, ifd, 0};
	for (int JBEG = jstart; jstride > 0 ? JBEG <= jend : JBEG >= jend; JBEG += jstride) {
		int JEND = 2 * ((J1 - JBEG) / 2) + JBEG;
		c.beg = JBEG;
		o_parallel((JEND - JBEG) / 2 + 1, (long)II * JJ, o2_xline, &c);
	}
}

/* y-line I = beg + 2t: right-hand side into a line buffer, DPTTRS, copy back */
static void o2_yline(void *vc, int t)
{
	const struct o2_lines_ctx *c = (const struct o2_lines_ctx *)vc;
	const double *so = c->so, *qf = c->qf, *sor = c->sor;
	double *q = c->q;
	const int II = c->II, JJ = c->JJ, J1 = JJ - 1, I = c->beg + 2 * t;
	double *B = (double *)malloc(sizeof(double) * (size_t)JJ);
#define SO(i, j, k) so[ix3(i, j, k, II, JJ)]
#define Q(i, j) q[ix2(i, j, II)]
#define QF(i, j) qf[ix2(i, j, II)]
	for (int J = 2; J <= J1; ++J) {
		if (c->ifd != 1)
			B[J - 1] = QF(I, J) + SO(I, J, KW) * Q(I - 1, J) + SO(I + 1, J, KW) * Q(I + 1, J)
			         + SO(I, J, KSW) * Q(I - 1, J - 1) + SO(I + 1, J, KNW) * Q(I + 1, J - 1)
			         + SO(I, J + 1, KNW) * Q(I - 1, J + 1) + SO(I + 1, J + 1, KSW) * Q(I + 1, J + 1);
		else
			B[J - 1] = QF(I, J) + SO(I, J, KW) * Q(I - 1, J) + SO(I + 1, J, KW) * Q(I + 1, J);
	}
	o_dpttrs(J1 - 1, &sor[ix3(2, I, 1, JJ, II)], &sor[ix3(3, I, 2, JJ, II)], &B[1]);
	for (int J = 2; J <= J1; ++J) Q(I, J) = B[J - 1];
	free(B);
#undef SO
#undef Q
#undef QF
}

/* BMG2_SymStd_relax_lines_y, src/2d/ftn/BMG2_SymStd_relax_lines_y.f90:74-129.
 * The 5-point branch forms every line's right-hand side in Q first; the
 * result is the same as forming each line's B before its solve. */
void o2_relax_lines_y(const double *so, const double *qf, double *q, const double *sor,
                      int II, int JJ, int ifd, int updown)
{
	int I1 = II - 1;
	int istart, iend, istride;
	if (updown == BMG_DOWN) { istart = 3; iend = 2; istride = -1; }
	else { istart = 2; iend = 3; istride = 1; }
	struct o2_lines_ctx c = {so, qf, sor, q, II, JJ, ifd, 0};
	for (int IBEG = istart; istride > 0 ? IBEG <= iend : IBEG >= iend; IBEG += istride) {
		int IEND = 2 * ((I1 - IBEG) / 2) + IBEG;
		c.beg = IBEG;
		o_parallel((IEND - IBEG) / 2 + 1, (long)II * JJ, o2_yline, &c);
	}
}

struct o2_restrict_ctx {
	const double *ci, *q;
	double *qc;
	int Nx, Nxc, Nyc;
};

static void o2_restrict_row(void *vc, int t)
{
	const struct o2_restrict_ctx *c = (const struct o2_restrict_ctx *)vc;
	const double *ci = c->ci, *q = c->q;
	double *qc = c->qc;
	const int Nx = c->Nx, Nxc = c->Nxc, Nyc = c->Nyc, jc = t + 2, j = 2 * jc - 2;
#define CI(i, j, k) ci[ix3(i, j, k, Nxc, Nyc)]
#define Q(i, j) q[ix2(i, j, Nx)]
#define QC(i, j) qc[ix2(i, j, Nxc)]
	for (int ic = 2; ic <= Nxc - 1; ++ic) {
		const int i = 2 * ic - 2;
		QC(ic, jc) = CI(ic, jc, LNE) * Q(i - 1, j - 1)
		           + CI(ic, jc, LA) * Q(i, j - 1)
		           + CI(ic + 1, jc, LNW) * Q(i + 1, j - 1)
		           + CI(ic, jc, LR) * Q(i - 1, j)
		           + Q(i, j)
		           + CI(ic + 1, jc, LL) * Q(i + 1, j)
		           + CI(ic, jc + 1, LSE) * Q(i - 1, j + 1)
		           + CI(ic, jc + 1, LB) * Q(i, j + 1)
		           + CI(ic + 1, jc + 1, LSW) * Q(i + 1, j + 1);
	}
#undef CI
#undef Q
#undef QC
}

/* BMG2_SymStd_restrict, src/2d/ftn/BMG2_SymStd_restrict.f90:72-92 */
void o2_restrict(const double *ci, const double *q, double *qc,
                 int Nx, int Ny, int Nxc, int Nyc)
{
	struct o2_restrict_ctx c = {ci, q, qc, Nx, Nxc, Nyc};
	o_parallel(Nyc - 2, (long)Nx * Ny, o2_restrict_row, &c);
}

struct o2_interp_ctx {
	double *q, *res;
	const double *qc, *so_ko, *ci;
	int IIC, JJC, IIF, JJF;
};

#define CI(i, j, k) ci[ix3(i, j, k, IIC, JJC)]
#define Q(i, j) q[ix2(i, j, IIF)]
#define QC(i, j) qc[ix2(i, j, IIC)]
#define RES(i, j) res[ix2(i, j, IIF)]
#define SOKO(i, j) so_ko[ix2(i, j, IIF)]
#define O2_INTERP_UNPACK                                                      \
	const struct o2_interp_ctx *c = (const struct o2_interp_ctx *)vc;        \
	double *q = c->q, *res = c->res;                                          \
	const double *qc = c->qc, *so_ko = c->so_ko, *ci = c->ci;                 \
	const int IIC = c->IIC, JJC = c->JJC, IIF = c->IIF;                       \
	(void)so_ko; (void)ci; (void)qc; (void)JJC

/* RES <- RES/c on fine row J = t + 2 */
static void o2_interp_div_row(void *vc, int t)
{
	O2_INTERP_UNPACK;
	const int J = t + 2;
	for (int I = 2; I <= IIF - 1; ++I) RES(I, J) = RES(I, J) / SOKO(I, J);
}

/* coarse row JC = t + 3: fine rows 2JC-2 and 2JC-3 */
static void o2_interp_row(void *vc, int t)
{
	O2_INTERP_UNPACK;
	const int IICF1 = (IIF - 2) / 2 + 2, JC = t + 3, J = 2 * JC - 2;
	int I = 2;
	Q(2, J) = Q(2, J) + QC(2, JC);
	double AQ = CI(2, JC, LA) * QC(2, JC) + CI(2, JC, LB) * QC(2, JC - 1);
	Q(2, J - 1) = Q(2, J - 1) + AQ + RES(2, J - 1);
	for (int IC = 3; IC <= IICF1; ++IC) {
		I += 2;
		Q(I, J) = Q(I, J) + QC(IC, JC);
		double A = CI(IC, JC, LR) * QC(IC, JC) + CI(IC, JC, LL) * QC(IC - 1, JC);
		Q(I - 1, J) = Q(I - 1, J) + A + RES(I - 1, J);
		AQ = CI(IC, JC, LA) * QC(IC, JC) + CI(IC, JC, LB) * QC(IC, JC - 1);
		Q(I, J - 1) = Q(I, J - 1) + AQ + RES(I, J - 1);
		A = CI(IC, JC, LSW) * QC(IC - 1, JC - 1) + CI(IC, JC, LNW) * QC(IC - 1, JC)
		  + CI(IC, JC, LNE) * QC(IC, JC) + CI(IC, JC, LSE) * QC(IC, JC - 1);
		Q(I - 1, J - 1) = Q(I - 1, J - 1) + A + RES(I - 1, J - 1);
	}
}

/* BMG2_SymStd_interp_add, src/2d/ftn/BMG2_SymStd_interp_add.f90:89-137.
 * so_ko points at the fine operator's KO plane; res is divided in place.
 * Coarse row JC writes only fine rows 2JC-2 and 2JC-3, so rows may run in
 * any order. */
void o2_interp_add(double *q, const double *qc, double *res, const double *so_ko,
                   const double *ci, int IIC, int JJC, int IIF, int JJF)
{
	struct o2_interp_ctx c = {q, res, qc, so_ko, ci, IIC, JJC, IIF, JJF};
	o_parallel(JJF - 2, (long)IIF * JJF, o2_interp_div_row, &c);
	int IICF = (IIF - 2) / 2 + 3, JJCF = (JJF - 2) / 2 + 3;
	int IICF1 = IICF - 1, JJCF1 = JJCF - 1;
	int J = 2, I = 2;
	Q(2, J) = Q(2, J) + QC(2, 2);
	for (int IC = 3; IC <= IICF1; ++IC) {
		I += 2;
		Q(I, J) = Q(I, J) + QC(IC, 2);
		double A = CI(IC, 2, LR) * QC(IC, 2) + CI(IC, 2, LL) * QC(IC - 1, 2);
		Q(I - 1, J) = Q(I - 1, J) + A + RES(I - 1, J);
	}
	if (JJCF1 >= 3) o_parallel(JJCF1 - 2, (long)IIF * JJF, o2_interp_row, &c);
}
#undef CI
#undef Q
#undef QC
#undef RES
#undef SOKO
#undef O2_INTERP_UNPACK

/* BMG2_SymStd_SETUP_interp_OI, src/2d/ftn/BMG2_SymStd_SETUP_interp_OI.f90:85-257
 * (non-periodic).  emach = D1MACH(3) = 2^-53 (src/2d/ftn/util.f90:58-66). */
void o2_setup_interp(const double *so, double *ci, int IIF, int JJF, int IIC, int JJC, int ifd)
{
#define SO(i, j, k) so[ix3(i, j, k, IIF, JJF)]
#define CI(i, j, k) ci[ix3(i, j, k, IIC, JJC)]
	const double emach = ldexp(1.0, -53);
	int IIC1 = IIC - 1, JJC1 = JJC - 1;
	int IICF = (IIF - 2) / 2 + 3, JJCF = (JJF - 2) / 2 + 3;
	int IICF1 = IICF - 1, JJCF1 = JJCF - 1;
	double A, B, EP, SUM, S;
	int I, J;
	if (ifd != 1) {
		J = 0;
		for (int JC = 2; JC <= JJC1; ++JC) {
			J += 2;
			I = 2;
			for (int IC = 3; IC <= IICF1; ++IC) {
				I += 2;
				A = SO(I, J, KW) + SO(I, J, KNW) + SO(I, J + 1, KSW);
				B = SO(I - 1, J, KW) + SO(I - 1, J, KSW) + SO(I - 1, J + 1, KNW);
				EP = fmin(fabs(A / SO(I - 1, J, KO)), fabs(B / SO(I - 1, J, KO)));
				SUM = A + B + SO(I - 1, J, KS) + SO(I - 1, J + 1, KS);
				SUM = A + B + (SO(I - 1, J, KO) - SUM) * fmax(SO(I - 1, J, KO) - (1.0 + EP) * SUM, 0.0)
				      / (fabs(SO(I - 1, J, KO) - (1.0 + EP) * SUM) + emach);
				SUM = 1.0 / SUM;
				CI(IC, JC, LR) = A * SUM;
				CI(IC, JC, LL) = B * SUM;
			}
		}
		J = 2;
		for (int JC = 3; JC <= JJCF1; ++JC) {
			J += 2;
			I = 0;
			for (int IC = 2; IC <= IIC1; ++IC) {
				I += 2;
				A = SO(I, J, KS) + SO(I, J, KNW) + SO(I + 1, J, KSW);
				B = SO(I, J - 1, KS) + SO(I, J - 1, KSW) + SO(I + 1, J - 1, KNW);
				EP = fmin(fabs(A / SO(I, J - 1, KO)), fabs(B / SO(I, J - 1, KO)));
				SUM = A + B + SO(I, J - 1, KW) + SO(I + 1, J - 1, KW);
				SUM = A + B + (SO(I, J - 1, KO) - SUM) * fmax(SO(I, J - 1, KO) - (1.0 + EP) * SUM, 0.0)
				      / (fabs(SO(I, J - 1, KO) - (1.0 + EP) * SUM) + emach);
				SUM = 1.0 / SUM;
				CI(IC, JC, LA) = A * SUM;
				CI(IC, JC, LB) = B * SUM;
			}
		}
		J = 2;
		for (int JC = 3; JC <= JJCF1; ++JC) {
			J += 2;
			I = 2;
			for (int IC = 3; IC <= IICF1; ++IC) {
				I += 2;
				SUM = SO(I - 1, J - 1, KW) + SO(I - 1, J, KNW) + SO(I - 1, J, KS)
				    + SO(I, J, KSW) + SO(I, J - 1, KW) + SO(I, J - 1, KNW)
				    + SO(I - 1, J - 1, KS) + SO(I - 1, J - 1, KSW);
				double o = SO(I - 1, J - 1, KO);
				EP = fmin(fmin(fabs((SO(I - 1, J - 1, KSW) + SO(I - 1, J - 1, KW) + SO(I - 1, J, KNW)) / o),
				               fabs((SO(I - 1, J, KNW) + SO(I - 1, J, KS) + SO(I, J, KSW)) / o)),
				          fmin(fabs((SO(I, J, KSW) + SO(I, J - 1, KW) + SO(I, J - 1, KNW)) / o),
				               fabs((SO(I, J - 1, KNW) + SO(I - 1, J - 1, KS) + SO(I - 1, J - 1, KSW)) / o)));
				SUM = SUM + (o - SUM) * fmax(o - (1.0 + EP) * SUM, 0.0) / (fabs(o - (1.0 + EP) * SUM) + emach);
				S = 1.0 / SUM;
				CI(IC, JC, LSW) = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LL)
				                   + SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LB) + SO(I - 1, J - 1, KSW)) * S;
				CI(IC, JC, LSE) = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LR)
				                   + SO(I, J - 1, KW) * CI(IC, JC, LB) + SO(I, J - 1, KNW)) * S;
				CI(IC, JC, LNW) = (SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LA)
				                   + SO(I - 1, J, KS) * CI(IC, JC, LL) + SO(I - 1, J, KNW)) * S;
				CI(IC, JC, LNE) = (SO(I - 1, J, KS) * CI(IC, JC, LR)
				                   + SO(I, J - 1, KW) * CI(IC, JC, LA) + SO(I, J, KSW)) * S;
			}
		}
	} else {
		J = 0;
		for (int JC = 2; JC <= JJC1; ++JC) {
			J += 2;
			I = 2;
			for (int IC = 3; IC <= IICF1; ++IC) {
				I += 2;
				A = SO(I, J, KW);
				B = SO(I - 1, J, KW);
				EP = fmin(fabs(A / SO(I - 1, J, KO)), fabs(B / SO(I - 1, J, KO)));
				SUM = A + B + SO(I - 1, J, KS) + SO(I - 1, J + 1, KS);
				SUM = A + B + (SO(I - 1, J, KO) - SUM) * fmax(SO(I - 1, J, KO) - (1.0 + EP) * SUM, 0.0)
				      / (fabs(SO(I - 1, J, KO) - (1.0 + EP) * SUM) + emach);
				SUM = 1.0 / SUM;
				CI(IC, JC, LR) = A * SUM;
				CI(IC, JC, LL) = B * SUM;
			}
		}
		J = 2;
		for (int JC = 3; JC <= JJCF1; ++JC) {
			J += 2;
			I = 0;
			for (int IC = 2; IC <= IIC1; ++IC) {
				I += 2;
				A = SO(I, J, KS);
				B = SO(I, J - 1, KS);
				EP = fmin(fabs(A / SO(I, J - 1, KO)), fabs(B / SO(I, J - 1, KO)));
				SUM = A + B + SO(I, J - 1, KW) + SO(I + 1, J - 1, KW);
				SUM = A + B + (SO(I, J - 1, KO) - SUM) * fmax(SO(I, J - 1, KO) - (1.0 + EP) * SUM, 0.0)
				      / (fabs(SO(I, J - 1, KO) - (1.0 + EP) * SUM) + emach);
				SUM = 1.0 / SUM;
				CI(IC, JC, LA) = A * SUM;
				CI(IC, JC, LB) = B * SUM;
			}
		}
		J = 2;
		for (int JC = 3; JC <= JJCF1; ++JC) {
			J += 2;
			I = 2;
			for (int IC = 3; IC <= IICF1; ++IC) {
				I += 2;
				SUM = SO(I - 1, J - 1, KW) + SO(I - 1, J, KS) + SO(I, J - 1, KW) + SO(I - 1, J - 1, KS);
				double o = SO(I - 1, J - 1, KO);
				EP = fmin(fmin(fabs(SO(I - 1, J - 1, KW) / o), fabs(SO(I - 1, J, KS) / o)),
				          fmin(fabs(SO(I, J - 1, KW) / o), fabs(SO(I - 1, J - 1, KS) / o)));
				SUM = SUM + (o - SUM) * fmax(o - (1.0 + EP) * SUM, 0.0) / (fabs(o - (1.0 + EP) * SUM) + emach);
				S = 1.0 / SUM;
				CI(IC, JC, LSW) = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LL) + SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LB)) * S;
				CI(IC, JC, LSE) = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LR) + SO(I, J - 1, KW) * CI(IC, JC, LB)) * S;
				CI(IC, JC, LNW) = (SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LA) + SO(I - 1, J, KS) * CI(IC, JC, LL)) * S;
				CI(IC, JC, LNE) = (SO(I - 1, J, KS) * CI(IC, JC, LR) + SO(I, J - 1, KW) * CI(IC, JC, LA)) * S;
			}
		}
	}
#undef SO
#undef CI
}

/* BMG2_SymStd_SETUP_ITLI_ex, src/2d/ftn/BMG2_SymStd_SETUP_ITLI_ex.f90:94-214 (9-point fine
 * operator) and :252-331 (5-point fine operator).  SOC gets 5 planes. */
void o2_setup_galerkin(const double *so, double *soc, const double *ci,
                       int IIF, int JJF, int IIC, int JJC, int ifd)
{
#define SO(i, j, k) so[ix3(i, j, k, IIF, JJF)]
#define CI(i, j, k) ci[ix3(i, j, k, IIC, JJC)]
#define SOC(i, j, k) soc[ix3(i, j, k, IIC, JJC)]
	int IIC1 = IIC - 1, JJC1 = JJC - 1;
	double CE, CEA, CENW, CFNW, CN, CNE, CNW, CO, COA, CONW, COSW, CS, CSA, CSE, CSEA, CSENW, CSNW,
	       CSWA, CSSW, CSW, CSWSW, CW, CWA, CWSW;
	int I, J;
	(void)JJF;
	if (ifd != 1) {
		J = 0;
		for (int JC = 2; JC <= JJC1; ++JC) {
			J += 2;
			I = 0;
			for (int IC = 2; IC <= IIC1; ++IC) {
				I += 2;
				CO = SO(I, J + 1, KNW) * CI(IC, JC + 1, LSW) + SO(I, J, KW) * CI(IC, JC, LL)
				   + SO(I, J, KSW) * CI(IC, JC, LNW);
				CS = SO(I, J - 1, KW) * CI(IC, JC, LNW) + SO(I, J, KNW) * CI(IC, JC, LL);
				CSW = -SO(I - 1, J - 1, KO) * CI(IC, JC, LNW) + SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LA)
				    + SO(I - 1, J, KNW) + SO(I - 1, J, KS) * CI(IC, JC, LL);
				CW = -SO(I - 1, J, KO) * CI(IC, JC, LL) + SO(I - 1, J, KS) * CI(IC, JC, LNW)
				   + SO(I - 1, J, KSW) * CI(IC - 1, JC, LA) + SO(I - 1, J, KW)
				   + SO(I - 1, J + 1, KNW) * CI(IC - 1, JC + 1, LB) + SO(I - 1, J + 1, KS) * CI(IC, JC + 1, LSW);
				CNW = -SO(I - 1, J + 1, KO) * CI(IC, JC + 1, LSW) + SO(I - 1, J + 1, KS) * CI(IC, JC, LL)
				    + SO(I - 1, J + 1, KSW) + SO(I - 1, J + 1, KW) * CI(IC - 1, JC + 1, LB);
				CN = SO(I, J + 1, KSW) * CI(IC, JC, LL) + SO(I, J + 1, KW) * CI(IC, JC + 1, LSW);
				SOC(IC, JC, KW) = CO + CI(IC, JC, LA) * CS + CI(IC, JC, LNE) * CSW + CI(IC, JC, LR) * CW
				                + CI(IC, JC + 1, LSE) * CNW + CI(IC, JC + 1, LB) * CN;
				COSW = SO(I, J, KSW) * CI(IC, JC, LSW);
				CSSW = SO(I, J - 1, KSW) * CI(IC, JC - 1, LL) + SO(I, J - 1, KW) * CI(IC, JC, LSW);
				CSWSW = -SO(I - 1, J - 1, KO) * CI(IC, JC, LSW) + SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LL)
				      + SO(I - 1, J - 1, KSW) + SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LB);
				CWSW = SO(I - 1, J, KS) * CI(IC, JC, LSW) + SO(I - 1, J, KSW) * CI(IC - 1, JC, LB);
				SOC(IC, JC, KSW) = COSW + CI(IC, JC, LA) * CSSW + CI(IC, JC, LNE) * CSWSW + CI(IC, JC, LR) * CWSW;
				COA = SO(I, J, KSW) * CI(IC, JC, LSE) + SO(I, J, KS) * CI(IC, JC, LB)
				    + SO(I + 1, J, KNW) * CI(IC + 1, JC, LSW);
				CEA = SO(I + 1, J, KS) * CI(IC + 1, JC, LSW) + SO(I + 1, J, KSW) * CI(IC, JC, LB);
				CSEA = -SO(I + 1, J - 1, KO) * CI(IC + 1, JC, LSW) + SO(I + 1, J - 1, KS) * CI(IC + 1, JC - 1, LL)
				     + SO(I + 1, J - 1, KSW) + SO(I + 1, J - 1, KW) * CI(IC, JC, LB);
				CSA = -SO(I, J - 1, KO) * CI(IC, JC, LB) + SO(I + 1, J - 1, KW) * CI(IC + 1, JC, LSW)
				    + SO(I + 1, J - 1, KNW) * CI(IC + 1, JC - 1, LL) + SO(I, J - 1, KS)
				    + SO(I, J - 1, KSW) * CI(IC, JC - 1, LR) + SO(I, J - 1, KW) * CI(IC, JC, LSE);
				CSWA = -SO(I - 1, J - 1, KO) * CI(IC, JC, LSE) + SO(I, J - 1, KW) * CI(IC, JC, LB)
				     + SO(I, J - 1, KNW) + SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LR);
				CWA = SO(I, J, KNW) * CI(IC, JC, LB) + SO(I - 1, J, KS) * CI(IC, JC, LSE);
				SOC(IC, JC, KS) = COA + CI(IC + 1, JC, LL) * CEA + CI(IC + 1, JC, LNW) * CSEA
				                + CI(IC, JC, LA) * CSA + CI(IC, JC, LNE) * CSWA + CI(IC, JC, LR) * CWA;
				CONW = SO(I - 1, J, KNW) * CI(IC, JC, LSE);
				CENW = SO(I, J, KNW) * CI(IC, JC, LB) + SO(I - 1, J, KS) * CI(IC, JC, LSE);
				CSENW = -SO(I - 1, J - 1, KO) * CI(IC, JC, LSE) + SO(I, J - 1, KW) * CI(IC, JC, LB)
				      + SO(I, J - 1, KNW) + SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LR);
				CFNW = SO(I - 1, J - 1, KW) * CI(IC, JC, LSE) + SO(I - 1, J - 1, KNW) * CI(IC, JC - 1, LR);
				SOC(IC, JC, KNW) = CONW + CI(IC, JC, LL) * CENW + CI(IC, JC, LNW) * CSENW + CI(IC - 1, JC, LA) * CFNW;
			}
		}
		J = 0;
		for (int JC = 2; JC <= JJC1; ++JC) {
			J += 2;
			I = 0;
			for (int IC = 2; IC <= IIC1; ++IC) {
				I += 2;
				CO = SO(I, J, KW) * CI(IC, JC, LR) + SO(I, J + 1, KNW) * CI(IC, JC + 1, LSE)
				   + SO(I, J + 1, KS) * CI(IC, JC + 1, LB) + SO(I + 1, J + 1, KSW) * CI(IC + 1, JC + 1, LSW)
				   + SO(I + 1, J, KW) * CI(IC + 1, JC, LL) + SO(I + 1, J, KNW) * CI(IC + 1, JC, LNW)
				   + SO(I, J, KS) * CI(IC, JC, LA) + SO(I, J, KSW) * CI(IC, JC, LNE) - SO(I, J, KO);
				CW = -SO(I - 1, J, KO) * CI(IC, JC, LR) + SO(I - 1, J + 1, KS) * CI(IC, JC + 1, LSE)
				   + SO(I, J + 1, KSW) * CI(IC, JC + 1, LB) + SO(I, J, KW) + SO(I, J, KNW) * CI(IC, JC, LA)
				   + SO(I - 1, J, KS) * CI(IC, JC, LNE);
				CNW = -SO(I - 1, J + 1, KO) * CI(IC, JC + 1, LSE) + SO(I, J + 1, KW) * CI(IC, JC + 1, LB)
				    + SO(I, J + 1, KNW) + SO(I - 1, J + 1, KS) * CI(IC, JC, LR);
				CN = -SO(I, J + 1, KO) * CI(IC, JC + 1, LB) + SO(I + 1, J + 1, KNW) * CI(IC + 1, JC, LL)
				   + SO(I, J + 1, KS) + SO(I, J + 1, KSW) * CI(IC, JC, LR) + SO(I, J + 1, KW) * CI(IC, JC + 1, LSE)
				   + SO(I + 1, J + 1, KW) * CI(IC + 1, JC + 1, LSW);
				CNE = -SO(I + 1, J + 1, KO) * CI(IC + 1, JC + 1, LSW) + SO(I + 1, J + 1, KS) * CI(IC + 1, JC, LL)
				    + SO(I + 1, J + 1, KSW) + SO(I + 1, J + 1, KW) * CI(IC, JC + 1, LB);
				CE = -SO(I + 1, J, KO) * CI(IC + 1, JC, LL) + SO(I + 1, J, KS) * CI(IC + 1, JC, LNW)
				   + SO(I + 1, J, KSW) * CI(IC, JC, LA) + SO(I + 1, J, KW) + SO(I + 1, J + 1, KNW) * CI(IC, JC + 1, LB)
				   + SO(I + 1, J + 1, KS) * CI(IC + 1, JC + 1, LSW);
				CSE = -SO(I + 1, J - 1, KO) * CI(IC + 1, JC, LNW) + SO(I + 1, J - 1, KW) * CI(IC, JC, LA)
				    + SO(I + 1, J, KNW) + SO(I + 1, J, KS) * CI(IC + 1, JC, LL);
				CS = -SO(I, J - 1, KO) * CI(IC, JC, LA) + SO(I, J - 1, KW) * CI(IC, JC, LNE)
				   + SO(I, J, KNW) * CI(IC, JC, LR) + SO(I, J, KS) + SO(I + 1, J, KSW) * CI(IC + 1, JC, LL)
				   + SO(I + 1, J - 1, KW) * CI(IC + 1, JC, LNW);
				CSW = -SO(I - 1, J - 1, KO) * CI(IC, JC, LNE) + SO(I - 1, J, KS) * CI(IC, JC, LR)
				    + SO(I, J, KSW) + SO(I, J - 1, KW) * CI(IC, JC, LA);
				SOC(IC, JC, KO) = -CI(IC, JC + 1, LSE) * CNW - CI(IC, JC + 1, LB) * CN
				                - CI(IC + 1, JC + 1, LSW) * CNE - CI(IC, JC, LR) * CW - CO
				                - CI(IC + 1, JC, LL) * CE - CI(IC, JC, LNE) * CSW
				                - CI(IC, JC, LA) * CS - CI(IC + 1, JC, LNW) * CSE;
			}
		}
	} else {
		J = 0;
		for (int JC = 2; JC <= JJC1; ++JC) {
			J += 2;
			I = 0;
			for (int IC = 2; IC <= IIC1; ++IC) {
				I += 2;
				CO = SO(I, J, KW) * CI(IC, JC, LL);
				CS = SO(I, J - 1, KW) * CI(IC, JC, LNW);
				CSW = -SO(I - 1, J - 1, KO) * CI(IC, JC, LNW) + SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LA)
				    + SO(I - 1, J, KS) * CI(IC, JC, LL);
				CW = -SO(I - 1, J, KO) * CI(IC, JC, LL) + SO(I - 1, J, KS) * CI(IC, JC, LNW) + SO(I - 1, J, KW)
				   + SO(I - 1, J + 1, KS) * CI(IC, JC + 1, LSW);
				CNW = -SO(I - 1, J + 1, KO) * CI(IC, JC + 1, LSW) + SO(I - 1, J + 1, KS) * CI(IC, JC, LL)
				    + SO(I - 1, J + 1, KW) * CI(IC - 1, JC + 1, LB);
				CN = SO(I, J + 1, KW) * CI(IC, JC + 1, LSW);
				SOC(IC, JC, KW) = CO + CI(IC, JC, LA) * CS + CI(IC, JC, LNE) * CSW + CI(IC, JC, LR) * CW
				                + CI(IC, JC + 1, LSE) * CNW + CI(IC, JC + 1, LB) * CN;
				CSSW = SO(I, J - 1, KW) * CI(IC, JC, LSW);
				CSWSW = -SO(I - 1, J - 1, KO) * CI(IC, JC, LSW) + SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LL)
				      + SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LB);
				CWSW = SO(I - 1, J, KS) * CI(IC, JC, LSW);
				SOC(IC, JC, KSW) = CI(IC, JC, LA) * CSSW + CI(IC, JC, LNE) * CSWSW + CI(IC, JC, LR) * CWSW;
				COA = SO(I, J, KS) * CI(IC, JC, LB);
				CEA = SO(I + 1, J, KS) * CI(IC + 1, JC, LSW);
				CSEA = -SO(I + 1, J - 1, KO) * CI(IC + 1, JC, LSW) + SO(I + 1, J - 1, KS) * CI(IC + 1, JC - 1, LL)
				     + SO(I + 1, J - 1, KW) * CI(IC, JC, LB);
				CSA = -SO(I, J - 1, KO) * CI(IC, JC, LB) + SO(I + 1, J - 1, KW) * CI(IC + 1, JC, LSW)
				    + SO(I, J - 1, KS) + SO(I, J - 1, KW) * CI(IC, JC, LSE);
				CSWA = -SO(I - 1, J - 1, KO) * CI(IC, JC, LSE) + SO(I, J - 1, KW) * CI(IC, JC, LB)
				     + SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LR);
				CWA = SO(I - 1, J, KS) * CI(IC, JC, LSE);
				SOC(IC, JC, KS) = COA + CI(IC + 1, JC, LL) * CEA + CI(IC + 1, JC, LNW) * CSEA
				                + CI(IC, JC, LA) * CSA + CI(IC, JC, LNE) * CSWA + CI(IC, JC, LR) * CWA;
				CENW = SO(I - 1, J, KS) * CI(IC, JC, LSE);
				CSENW = -SO(I - 1, J - 1, KO) * CI(IC, JC, LSE) + SO(I, J - 1, KW) * CI(IC, JC, LB)
				      + SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LR);
				CSNW = SO(I - 1, J - 1, KW) * CI(IC, JC, LSE);
				SOC(IC, JC, KNW) = CI(IC, JC, LL) * CENW + CI(IC, JC, LNW) * CSENW + CI(IC - 1, JC, LA) * CSNW;
				CO = SO(I, J, KW) * CI(IC, JC, LR) + SO(I, J + 1, KS) * CI(IC, JC + 1, LB)
				   + SO(I + 1, J, KW) * CI(IC + 1, JC, LL) + SO(I, J, KS) * CI(IC, JC, LA) - SO(I, J, KO);
				CW = -SO(I - 1, J, KO) * CI(IC, JC, LR) + SO(I - 1, J + 1, KS) * CI(IC, JC + 1, LSE)
				   + SO(I, J, KW) + SO(I - 1, J, KS) * CI(IC, JC, LNE);
				CNW = -SO(I - 1, J + 1, KO) * CI(IC, JC + 1, LSE) + SO(I, J + 1, KW) * CI(IC, JC + 1, LB)
				    + SO(I - 1, J + 1, KS) * CI(IC, JC, LR);
				CN = -SO(I, J + 1, KO) * CI(IC, JC + 1, LB) + SO(I, J + 1, KS)
				   + SO(I, J + 1, KW) * CI(IC, JC + 1, LSE) + SO(I + 1, J + 1, KW) * CI(IC + 1, JC + 1, LSW);
				CNE = -SO(I + 1, J + 1, KO) * CI(IC + 1, JC + 1, LSW) + SO(I + 1, J + 1, KS) * CI(IC + 1, JC, LL)
				    + SO(I + 1, J + 1, KW) * CI(IC, JC + 1, LB);
				CE = -SO(I + 1, J, KO) * CI(IC + 1, JC, LL) + SO(I + 1, J, KS) * CI(IC + 1, JC, LNW)
				   + SO(I + 1, J, KW) + SO(I + 1, J + 1, KS) * CI(IC + 1, JC + 1, LSW);
				CSE = -SO(I + 1, J - 1, KO) * CI(IC + 1, JC, LNW) + SO(I + 1, J - 1, KW) * CI(IC, JC, LA)
				    + SO(I + 1, J, KS) * CI(IC + 1, JC, LL);
				CS = -SO(I, J - 1, KO) * CI(IC, JC, LA) + SO(I, J - 1, KW) * CI(IC, JC, LNE) + SO(I, J, KS)
				   + SO(I + 1, J - 1, KW) * CI(IC + 1, JC, LNW);
				CSW = -SO(I - 1, J - 1, KO) * CI(IC, JC, LNE) + SO(I - 1, J, KS) * CI(IC, JC, LR)
				    + SO(I, J - 1, KW) * CI(IC, JC, LA);
				SOC(IC, JC, KO) = -CI(IC, JC + 1, LSE) * CNW - CI(IC, JC + 1, LB) * CN
				                - CI(IC + 1, JC + 1, LSW) * CNE - CI(IC, JC, LR) * CW - CO
				                - CI(IC + 1, JC, LL) * CE - CI(IC, JC, LNE) * CSW
				                - CI(IC, JC, LA) * CS - CI(IC + 1, JC, LNW) * CSE;
			}
		}
	}
#undef SO
#undef CI
#undef SOC
}

/* BMG2_SymStd_SETUP_cg_LU, src/2d/ftn/BMG2_SymStd_SETUP_cg_LU.f90:92-118 (NStncl=5)
 * and :229-255 (NStncl=3), definite non-periodic; DPBTRF('U', N, KD=II-1). */
int o2_setup_cg(const double *so, int II, int JJ, int nstncl, double *abd, int nabd1)
{
#define SO(i, j, k) so[ix3(i, j, k, II, JJ)]
#define ABD(r, c) abd[(size_t)((c) - 1) * nabd1 + ((r) - 1)]
	int I1 = II - 1, J1 = JJ - 1, I2 = I1 - 1;
	int N = I2 * (J1 - 1);
	int KK = 0;
	for (int J = 2; J <= J1; ++J)
		for (int I = 2; I <= I1; ++I) {
			KK++;
			ABD(II, KK) = SO(I, J, KO);
			ABD(I1, KK) = -SO(I, J, KW);
			ABD(3, KK) = nstncl == 5 ? -SO(I + 1, J, KNW) : 0.0;
			ABD(2, KK) = -SO(I, J, KS);
			ABD(1, KK) = nstncl == 5 ? -SO(I, J, KSW) : 0.0;
		}
	return o_dpbtrf_u(N, I1, abd, nabd1);
#undef SO
#undef ABD
}

/* BMG2_SymStd_SOLVE_cg, src/2d/ftn/BMG2_SymStd_SOLVE_cg.f90:93-123 (non-periodic) */
void o2_solve_cg(double *q, const double *qf, int II, int JJ, const double *abd, double *bbd, int nabd1)
{
	int I1 = II - 1, J1 = JJ - 1;
	int KK = 0;
	for (int J = 2; J <= J1; ++J)
		for (int I = 2; I <= I1; ++I)
			bbd[KK++] = qf[ix2(I, J, II)];
	o_dpbtrs_u(KK, I1, abd, nabd1, bbd);
	KK = 0;
	for (int J = 2; J <= J1; ++J)
		for (int I = 2; I <= I1; ++I)
			q[ix2(I, J, II)] = bbd[KK++];
}

/* grid_func::lp_norm<2>, include/cedar/2d/grid_func.h:43-54 */
double o2_l2norm(const double *r, int II, int JJ)
{
	double result = 0;
	for (int j = 2; j <= JJ - 1; ++j)
		for (int i = 2; i <= II - 1; ++i)
			result += pow(r[ix2(i, j, II)], 2);
	return pow(result, 1. / 2);
}

/* grid_func::inf_norm (signed value of largest magnitude), src/2d/grid_func.cc:132-148 */
double o2_inf_norm(const double *r, int II, int JJ)
{
	double cmax = 0;
	for (int j = 2; j <= JJ - 1; ++j)
		for (int i = 2; i <= II - 1; ++i)
			if (fabs(cmax) < fabs(r[ix2(i, j, II)])) cmax = r[ix2(i, j, II)];
	return cmax;
}

/* ------------------------------------------------------------------ */
/* Multilevel driver                                                   */
/* ------------------------------------------------------------------ */

struct o2_level {
	int nx, ny, ii, jj, nstncl;
	double *so, *x, *b, *res, *sor0, *sor1, *ci;
};

struct o2_solver {
	o2_settings s;
	int nlev;
	struct o2_level *lv;
	double *abd, *bbd;
	int nabd1, nabd2;
	int cg_info;
	int setup_info;
};

static double *zalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

/* cdr2::solver::compute_num_levels, include/cedar/2d/solver.h:63-79 */
int o2_num_levels(int nx, int ny, int min_coarse)
{
	float nxc, nyc;
	int ng = 0;
	do {
		ng++;
		nxc = (float)((nx - 1) / (1 << ng) + 1);
		nyc = (float)((ny - 1) / (1 << ng) + 1);
	} while ((nxc < nyc ? nxc : nyc) >= min_coarse);
	return ng;
}

static void alloc_level(struct o2_level *L, int nx, int ny, int nstncl)
{
	L->nx = nx; L->ny = ny; L->ii = nx + 2; L->jj = ny + 2; L->nstncl = nstncl;
	size_t n = (size_t)L->ii * L->jj;
	L->so = zalloc(n * nstncl);
	L->x = zalloc(n); L->b = zalloc(n); L->res = zalloc(n);
	L->sor0 = zalloc(n * 2); L->sor1 = zalloc(n * 2);
	L->ci = zalloc(n * 8);
}

/* multilevel::setup_relax_helper (setup part), include/cedar/multilevel.h:134-158 */
static int setup_relax(o2_solver *h, struct o2_level *L)
{
	int info = 0;
	switch (h->s.relax) {
	case O2_RELAX_POINT: o2_setup_recip(L->so, L->sor0, L->ii, L->jj); break;
	case O2_RELAX_LINE_X: info = o2_setup_lines_x(L->so, L->sor0, L->ii, L->jj); break;
	case O2_RELAX_LINE_Y: info = o2_setup_lines_y(L->so, L->sor0, L->ii, L->jj); break;
	case O2_RELAX_LINE_XY:
		info = o2_setup_lines_x(L->so, L->sor0, L->ii, L->jj);
		if (!info) info = o2_setup_lines_y(L->so, L->sor1, L->ii, L->jj);
		break;
	}
	return info;
}

/* multilevel::setup_relax_helper smoother closures, include/cedar/multilevel.h:160-222 */
static void smooth(o2_solver *h, struct o2_level *L, int updown)
{
	int ifd = L->nstncl == 3 ? 1 : 0;
	int n = updown == BMG_DOWN ? h->s.nrelax_pre : h->s.nrelax_post;
	for (int it = 0; it < n; ++it) {
		switch (h->s.relax) {
		case O2_RELAX_POINT:
			if (h->s.bc) o2_relax_gs_per(L->so, L->b, L->x, L->sor0, L->ii, L->jj, ifd, updown, h->s.bc);
			else o2_relax_gs(L->so, L->b, L->x, L->sor0, L->ii, L->jj, ifd, updown);
			break;
		case O2_RELAX_LINE_X: o2_relax_lines_x(L->so, L->b, L->x, L->sor0, L->ii, L->jj, ifd, updown); break;
		case O2_RELAX_LINE_Y: o2_relax_lines_y(L->so, L->b, L->x, L->sor0, L->ii, L->jj, ifd, updown); break;
		case O2_RELAX_LINE_XY:
			if (updown == BMG_DOWN) {
				o2_relax_lines_x(L->so, L->b, L->x, L->sor0, L->ii, L->jj, ifd, updown);
				o2_relax_lines_y(L->so, L->b, L->x, L->sor1, L->ii, L->jj, ifd, updown);
			} else {
				o2_relax_lines_y(L->so, L->b, L->x, L->sor1, L->ii, L->jj, ifd, updown);
				o2_relax_lines_x(L->so, L->b, L->x, L->sor0, L->ii, L->jj, ifd, updown);
			}
			break;
		}
	}
}

/* multilevel::setup, include/cedar/multilevel.h:243-265; cdr2::solver::setup_space,
 * include/cedar/2d/solver.h:81-123; multilevel::setup_cg_solve :95-103. */
o2_solver *o2_create(const o2_settings *s, const double *so_fine, int nstncl, int nx, int ny)
{
	o2_solver *h = (o2_solver *)calloc(1, sizeof(o2_solver));
	h->s = *s;
	int nl = o2_num_levels(nx, ny, s->min_coarse);
	if (s->num_levels > 0 && s->num_levels <= nl) nl = s->num_levels;
	h->nlev = nl;
	h->lv = (struct o2_level *)calloc(nl, sizeof(struct o2_level));
	alloc_level(&h->lv[0], nx, ny, nstncl);
	memcpy(h->lv[0].so, so_fine, sizeof(double) * (size_t)(nx + 2) * (ny + 2) * nstncl);
	for (int l = 1; l < nl; ++l) {
		int pnx = h->lv[l - 1].nx, pny = h->lv[l - 1].ny;
		int cnx = (int)((pnx - 1) / 2. + 1), cny = (int)((pny - 1) / 2. + 1);
		alloc_level(&h->lv[l], cnx, cny, 5);
	}
	for (int l = 0; l < nl - 1; ++l) {
		struct o2_level *F = &h->lv[l], *C = &h->lv[l + 1];
		int ifd = F->nstncl == 3 ? 1 : 0;
		if (h->s.bc) {
			o2_setup_interp_per(F->so, C->ci, F->ii, F->jj, C->ii, C->jj, ifd, h->s.bc);
			o2_setup_galerkin_per(F->so, C->so, C->ci, F->ii, F->jj, C->ii, C->jj, ifd, h->s.bc);
		} else {
			o2_setup_interp(F->so, C->ci, F->ii, F->jj, C->ii, C->jj, ifd);
			o2_setup_galerkin(F->so, C->so, C->ci, F->ii, F->jj, C->ii, C->jj, ifd);
		}
		int r = setup_relax(h, F);
		if (r && !h->setup_info) h->setup_info = r;
	}
	struct o2_level *Cg = &h->lv[nl - 1];
	/* periodic: a dense N x N factor (include/cedar/2d/solver.h:118-121) */
	h->nabd1 = h->s.bc ? Cg->nx * Cg->ny : Cg->nx + 2;
	h->nabd2 = Cg->nx * Cg->ny;
	h->abd = zalloc((size_t)h->nabd1 * h->nabd2);
	h->bbd = zalloc((size_t)h->nabd2);
	if (h->s.bc) h->cg_info = o2_setup_cg_per(Cg->so, Cg->ii, Cg->jj, Cg->nstncl, h->abd, h->s.bc);
	else h->cg_info = o2_setup_cg(Cg->so, Cg->ii, Cg->jj, Cg->nstncl, h->abd, h->nabd1);
	if (h->s.bc && h->s.relax != O2_RELAX_POINT && !h->setup_info) h->setup_info = -1;
	return h;
}

void o2_destroy(o2_solver *h)
{
	if (!h) return;
	for (int l = 0; l < h->nlev; ++l) {
		struct o2_level *L = &h->lv[l];
		free(L->so); free(L->x); free(L->b); free(L->res);
		free(L->sor0); free(L->sor1); free(L->ci);
	}
	free(h->lv); free(h->abd); free(h->bbd); free(h);
}

static void coarse_solve(o2_solver *h, struct o2_level *C, double *x, const double *b)
{
	if (h->s.bc) o2_solve_cg_per(x, b, C->ii, C->jj, h->abd, h->bbd, h->s.bc);
	else o2_solve_cg(x, b, C->ii, C->jj, h->abd, h->bbd, h->nabd1);
}

static void restrict_bc(o2_solver *h, struct o2_level *L, struct o2_level *C, const double *q)
{
	if (h->s.bc) o2_restrict_per(C->ci, (double *)q, C->b, L->ii, L->jj, C->ii, C->jj, h->s.bc);
	else o2_restrict(C->ci, q, C->b, L->ii, L->jj, C->ii, C->jj);
}

static void interp_bc(o2_solver *h, struct o2_level *L, struct o2_level *C, double *x)
{
	if (h->s.bc) o2_interp_add_per(x, C->x, L->res, L->so, C->ci, C->ii, C->jj, L->ii, L->jj, h->s.bc);
	else o2_interp_add(x, C->x, L->res, L->so, C->ci, C->ii, C->jj, L->ii, L->jj);
}

/* cycle::vcycle::ncycle_helper, include/cedar/cycle/vcycle.h:57-115 (n = 1) */
static void ncycle(o2_solver *h, int l, double *x, const double *b)
{
	struct o2_level *L = &h->lv[l], *C = &h->lv[l + 1];
	double *sx = L->x, *sb = L->b;
	L->x = x; L->b = (double *)b;
	smooth(h, L, BMG_DOWN);
	o2_residual(L->so, L->b, L->x, L->res, L->ii, L->jj, L->nstncl == 3 ? 1 : 0);
	restrict_bc(h, L, C, L->res);
	memset(C->x, 0, sizeof(double) * (size_t)C->ii * C->jj);
	if (l + 1 == h->nlev - 1)
		coarse_solve(h, C, C->x, C->b);
	else
		ncycle(h, l + 1, C->x, C->b);
	interp_bc(h, L, C, L->x);
	smooth(h, L, BMG_UP);
	L->x = sx; L->b = sb;
}

void o2_vcycle(o2_solver *h, double *x, const double *b)
{
	if (h->nlev == 1) {
		coarse_solve(h, &h->lv[0], x, b);
	} else {
		ncycle(h, 0, x, b);
	}
}

/* cycle::fcycle::fmg_cycle / fmg_cycle_helper, include/cedar/cycle/fcycle.h:49-83:
 * b restricted to the next level, the F-cycle there, then x = P x_c (x and the
 * level's residual zeroed first, so interp_add adds no residual term) and a
 * V-cycle from that x.  The incoming x is not used. */
static void fcycle(o2_solver *h, int l, double *x, const double *b)
{
	struct o2_level *L = &h->lv[l];
	if (l == h->nlev - 1) {
		coarse_solve(h, L, x, b);
		return;
	}
	struct o2_level *C = &h->lv[l + 1];
	restrict_bc(h, L, C, b);
	fcycle(h, l + 1, C->x, C->b);
	memset(x, 0, sizeof(double) * (size_t)L->ii * L->jj);
	memset(L->res, 0, sizeof(double) * (size_t)L->ii * L->jj);
	interp_bc(h, L, C, x);
	ncycle(h, l, x, b);
}

/* cycle->run of multilevel::solve: the V- or the F-cycle (multilevel.h:68-78) */
void o2_cycle(o2_solver *h, double *x, const double *b)
{
	if (h->s.cycle == 1 && h->nlev > 1) fcycle(h, 0, x, b);
	else o2_vcycle(h, x, b);
}

/* multilevel::solve, include/cedar/multilevel.h:278-298.  Returns the number of
 * cycles run; hist[i] = relative l2 residual after cycle i. */
int o2_solve(o2_solver *h, const double *b, double *x, double *hist, int maxhist)
{
	struct o2_level *L = &h->lv[0];
	int ifd = L->nstncl == 3 ? 1 : 0;
	o2_residual(L->so, b, x, L->res, L->ii, L->jj, ifd);
	double res0 = o2_l2norm(L->res, L->ii, L->jj);
	int it;
	for (it = 0; it < h->s.maxiter; ++it) {
		o2_cycle(h, x, b);
		o2_residual(L->so, b, x, L->res, L->ii, L->jj, ifd);
		double rel = o2_l2norm(L->res, L->ii, L->jj) / res0;
		if (hist && it < maxhist) hist[it] = rel;
		if (rel < h->s.tol) { ++it; break; }
	}
	return it;
}

/* ------------------------------------------------------------------ */
/* Flexible CG around the cycle                                        */
/* ------------------------------------------------------------------ */
/* Notay's FCG(1) preconditioned by one cycle of the solver: the CPU
 * counterpart of the GPU solver's flexible-CG outer iteration (the reference
 * has none; its solve repeats the cycle).  Recurrences, as on the GPU:
 *   beta = -(z . q_prev) / (p_prev . q_prev) (0 first), p = z + beta p_prev,
 *   q = A p, alpha = (p . r) / (p . q), x += alpha p,
 *   r = b - A x every `replace`-th iteration and to confirm convergence,
 *   r -= alpha q in between.
 * Vector work is split by rows over the host threads; each dot product sums
 * per-row partials in row order (no result depends on the thread count). */
struct o2_vec_ctx {
	int op, II;
	double a;
	double *x, *y;
	const double *u, *v;
	double *part; /* per-row partial sums (dot products) */
};

static void o2_vec_row(void *vc, int t)
{
	const struct o2_vec_ctx *c = (const struct o2_vec_ctx *)vc;
	const size_t k0 = (size_t)(t + 1) * c->II + 1, k1 = k0 + c->II - 2;
	double s = 0.0;
	switch (c->op) {
	case 0: /* part = sum u*v */
		for (size_t k = k0; k < k1; ++k) s += c->u[k] * c->v[k];
		c->part[t] = s;
		break;
	case 1: /* x = u + a*x */
		for (size_t k = k0; k < k1; ++k) c->x[k] = c->u[k] + c->a * c->x[k];
		break;
	case 2: /* x += a*u */
		for (size_t k = k0; k < k1; ++k) c->x[k] += c->a * c->u[k];
		break;
	case 3: /* x = -u */
		for (size_t k = k0; k < k1; ++k) c->x[k] = -c->u[k];
		break;
	}
}

static double o2_vec(int op, int II, int JJ, double a, double *x, const double *u, const double *v, double *part)
{
	struct o2_vec_ctx c = {op, II, a, x, NULL, u, v, part};
	o_parallel(JJ - 2, (long)II * JJ, o2_vec_row, &c);
	double s = 0.0;
	if (op == 0)
		for (int t = 0; t < JJ - 2; ++t) s += part[t];
	return s;
}

int o2_solve_fcg(o2_solver *h, const double *b, double *x, int replace, double *hist, int maxhist)
{
	struct o2_level *L = &h->lv[0];
	const int II = L->ii, JJ = L->jj, ifd = L->nstncl == 3 ? 1 : 0;
	const size_t n = (size_t)II * JJ;
	double *r = zalloc(n), *z = zalloc(n), *p = zalloc(n), *q = zalloc(n), *t = zalloc(n), *zero = zalloc(n);
	double *part = zalloc((size_t)JJ);
	const int m = replace > 1 ? replace : 1;
	o2_residual(L->so, b, x, r, II, JJ, ifd);
	const double res0 = sqrt(o2_vec(0, II, JJ, 0.0, NULL, r, r, part));
	double pq = 1.0;
	int it = 0, first = 1;
	while (res0 > 0 && it < h->s.maxiter) {
		memset(z, 0, sizeof(double) * n);
		o2_cycle(h, z, r);
		const double beta = first ? 0.0 : -o2_vec(0, II, JJ, 0.0, NULL, z, q, part) / pq;
		o2_vec(1, II, JJ, beta, p, z, NULL, part);           /* p = z + beta p */
		o2_residual(L->so, zero, p, t, II, JJ, ifd);         /* t = -A p */
		o2_vec(3, II, JJ, 0.0, q, t, NULL, part);            /* q = A p */
		pq = o2_vec(0, II, JJ, 0.0, NULL, p, q, part);
		const double alpha = o2_vec(0, II, JJ, 0.0, NULL, p, r, part) / pq;
		o2_vec(2, II, JJ, alpha, x, p, NULL, part);          /* x += alpha p */
		const int formed = (it + 1) % m == 0;
		if (formed) o2_residual(L->so, b, x, r, II, JJ, ifd);
		else o2_vec(2, II, JJ, -alpha, r, q, NULL, part);    /* r -= alpha q */
		first = 0;
		double rel = sqrt(o2_vec(0, II, JJ, 0.0, NULL, r, r, part)) / res0;
		++it;
		if (rel < h->s.tol && !formed) {
			/* an updated residual met the tolerance: form b - A x and go on from it */
			o2_residual(L->so, b, x, r, II, JJ, ifd);
			rel = sqrt(o2_vec(0, II, JJ, 0.0, NULL, r, r, part)) / res0;
		}
		if (hist && it - 1 < maxhist) hist[it - 1] = rel;
		if (!(rel == rel) || rel < h->s.tol) break;
	}
	free(r); free(z); free(p); free(q); free(t); free(zero); free(part);
	return it;
}

int o2_nlevels(const o2_solver *h) { return h->nlev; }
int o2_info(const o2_solver *h, int which) { return which == 0 ? h->setup_info : h->cg_info; }

void o2_level_dims(const o2_solver *h, int l, int *dims)
{
	dims[0] = h->lv[l].nx; dims[1] = h->lv[l].ny; dims[2] = h->lv[l].nstncl;
}

double *o2_level_array(o2_solver *h, int l, int which)
{
	struct o2_level *L = &h->lv[l];
	switch (which) {
	case O2_ARR_SO: return L->so;
	case O2_ARR_X: return L->x;
	case O2_ARR_B: return L->b;
	case O2_ARR_RES: return L->res;
	case O2_ARR_SOR0: return L->sor0;
	case O2_ARR_SOR1: return L->sor1;
	case O2_ARR_CI: return L->ci;
	case O2_ARR_ABD: return h->abd;
	default: return NULL;
	}
}

void o2_abd_dims(const o2_solver *h, int *dims) { dims[0] = h->nabd1; dims[1] = h->nabd2; }
