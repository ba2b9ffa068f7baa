/*
 * cdr2_periodic.c -- CPU restatement of the periodic branches of Cedar's
 * serial 2D BoxMG kernels (definite periodic boundary conditions).
 *
 * TEST INFRASTRUCTURE ONLY: the parity oracle the GPU path is checked
 * against.  Nothing in the product links or calls it.
 *
 * Boundary-condition codes (BMG_get_bc, src/2d/ftn/BMG_get_bc.f90:11-22;
 * values src/2d/ftn/BMG_parameters_f90.h:345-352): per_mask bit 0 (x) ->
 * BMG_BCs_def_per_x = 2, bit 1 (y) -> def_per_y = 1, both -> def_per_xy = 3;
 * 0 is the definite non-periodic case, handled by cdr2_oracle.c.  A periodic
 * direction keeps copies of the opposite interior line in its ghost lines:
 * every kernel below restates the reference's updates of those copies.
 * Indices are the Fortran ones (1-based, ghosts at 1 and II/JJ).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "cdr2_oracle.h"

enum { KO = 1, KW = 2, KS = 3, KSW = 4, KNW = 5 };
/* the oracle's plane numbers (cdr2_oracle.c; include/cedar/2d/prolong_op.h:14) */
enum { LL = 1, LR = 2, LA = 3, LB = 4, LSW = 5, LNW = 6, LNE = 7, LSE = 8 };
enum { PER_X = 2, PER_Y = 1, PER_XY = 3 };
static const int BMG_DOWN = 0;

static inline size_t ix2(long i, long j, long ii) { return (size_t)(j - 1) * ii + (i - 1); }
static inline size_t ix3(long i, long j, long k, long ii, long jj)
{
	return ((size_t)(k - 1) * jj + (j - 1)) * ii + (i - 1);
}
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int perx(int ipn) { return ipn == PER_X || ipn == PER_XY; }
static inline int pery(int ipn) { return ipn == PER_Y || ipn == PER_XY; }

int o2_bc_code(int per_mask)
{
	static const int map[4] = {0, PER_X, PER_Y, PER_XY};
	return per_mask >= 0 && per_mask < 4 ? map[per_mask] : 0;
}

/* ------------------------------------------------------------------ GS */
/* BMG2_SymStd_relax_GS, periodic branch (src/2d/ftn/BMG2_SymStd_relax_GS.f90:139-226):
 * the colour sweeps of the definite branch; after each row's points of a
 * colour its x-ghosts are refreshed, after the whole sweep the y-ghost rows. */
void o2_relax_gs_per(const double *so, const double *qf, double *q, const double *sor, int II, int JJ, int ifd,
                     int updown, int ipn)
{
#define SO(i, j, k) so[ix3(i, j, k, II, JJ)]
#define Q(i, j) q[ix2(i, j, II)]
#define QF(i, j) qf[ix2(i, j, II)]
#define SOR(i, j) sor[ix3(i, j, 2, II, JJ)]
	const int I1 = II - 1, J1 = JJ - 1;
	int LSTART, LEND, LSTRIDE;
	if (updown == BMG_DOWN) { LSTART = 2; LEND = 3; LSTRIDE = 1; }
	else { LSTART = 3; LEND = 2; LSTRIDE = -1; }
	if (ifd != 1) {
		for (int JBEG = LSTART; LSTRIDE > 0 ? JBEG <= LEND : JBEG >= LEND; JBEG += LSTRIDE) {
			const int JEND = 2 * ((J1 - JBEG) / 2) + JBEG;
			for (int J = JBEG; J <= JEND; J += 2)
				for (int IBEG = LSTART; LSTRIDE > 0 ? IBEG <= LEND : IBEG >= LEND; IBEG += LSTRIDE) {
					const int IEND = 2 * ((I1 - IBEG) / 2) + IBEG;
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
					if (perx(ipn)) {
						Q(1, J) = Q(I1, J);
						Q(II, J) = Q(2, J);
					}
				}
		}
	} else {
		for (int JO = LSTART; LSTRIDE > 0 ? JO <= LEND : JO >= LEND; JO += LSTRIDE)
			for (int J = 2; J <= J1; ++J) {
				const int IBEG = (J + JO) % 2 + 2;
				const int IEND = 2 * ((I1 - IBEG) / 2) + IBEG;
				for (int I = IBEG; I <= IEND; I += 2)
					Q(I, J) = (QF(I, J)
					           + SO(I, J, KW) * Q(I - 1, J)
					           + SO(I + 1, J, KW) * Q(I + 1, J)
					           + SO(I, J, KS) * Q(I, J - 1)
					           + SO(I, J + 1, KS) * Q(I, J + 1)) * SOR(I, J);
				if (perx(ipn)) {
					Q(1, J) = Q(I1, J);
					Q(II, J) = Q(2, J);
				}
			}
	}
	if (pery(ipn))
		for (int I = 1; I <= II; ++I) {
			Q(I, 1) = Q(I, J1);
			Q(I, JJ) = Q(I, 2);
		}
#undef SO
#undef Q
#undef QF
#undef SOR
}

/* -------------------------------------------------------- restriction */
/* BMG2_SymStd_restrict, periodic branch (src/2d/ftn/BMG2_SymStd_restrict.f90:94-130):
 * the fine vector's ghosts are refreshed (in place) where the coarse grid
 * has the "even" size Nx/2 + 1, then the definite restriction. */
void o2_restrict_per(const double *ci, double *q, double *qc, int Nx, int Ny, int Nxc, int Nyc, int ipn)
{
#define Q(i, j) q[ix2(i, j, Nx)]
	if (pery(ipn) && Ny / 2 + 1 == Nyc)
		for (int I = 1; I <= Nx; ++I) {
			Q(I, 1) = Q(I, Ny - 1);
			Q(I, Ny) = Q(I, 2);
		}
	if (perx(ipn) && Nx / 2 + 1 == Nxc)
		for (int J = 1; J <= Ny; ++J) {
			Q(1, J) = Q(Nx - 1, J);
			Q(Nx, J) = Q(2, J);
		}
#undef Q
	o2_restrict(ci, q, qc, Nx, Ny, Nxc, Nyc);
}

/* ---------------------------------------------------- interpolate-add */
/* BMG2_SymStd_interp_add, periodic branch (src/2d/ftn/BMG2_SymStd_interp_add.f90:139-156):
 * the definite interpolation, then the fine ghosts (y rows, then x columns). */
void o2_interp_add_per(double *q, const double *qc, double *res, const double *so_ko, const double *ci, int IIC,
                       int JJC, int IIF, int JJF, int ipn)
{
	o2_interp_add(q, qc, res, so_ko, ci, IIC, JJC, IIF, JJF);
#define Q(i, j) q[ix2(i, j, IIF)]
	const int IIF1 = IIF - 1, JJF1 = JJF - 1;
	if (pery(ipn))
		for (int I = 1; I <= IIF; ++I) {
			Q(I, 1) = Q(I, JJF1);
			Q(I, JJF) = Q(I, 2);
		}
	if (perx(ipn))
		for (int J = 1; J <= JJF; ++J) {
			Q(1, J) = Q(IIF1, J);
			Q(IIF, J) = Q(2, J);
		}
#undef Q
}

/* ------------------------------------------------------------ Galerkin */
/* BMG2_SymStd_SETUP_ITLI_ex, periodic ends (src/2d/ftn/BMG2_SymStd_SETUP_ITLI_ex.f90:216-247,
 * 333-363): the definite product, then the coarse operator's ghost lines. */
void o2_setup_galerkin_per(const double *so, double *soc, const double *ci, int IIF, int JJF, int IIC, int JJC,
                           int ifd, int ipn)
{
	o2_setup_galerkin(so, soc, ci, IIF, JJF, IIC, JJC, ifd);
#define SOC(i, j, k) soc[ix3(i, j, k, IIC, JJC)]
	const int IIC1 = IIC - 1, JJC1 = JJC - 1;
	static const int order_hi[5] = {KS, KW, KNW, KSW, KO};
	static const int order_lo[5] = {KO, KW, KS, KSW, KNW};
	if (pery(ipn))
		for (int IC = 1; IC <= IIC; ++IC) {
			for (int q = 0; q < 5; ++q) SOC(IC, JJC, order_hi[q]) = SOC(IC, 2, order_hi[q]);
			for (int q = 0; q < 5; ++q) SOC(IC, 1, order_lo[q]) = SOC(IC, JJC1, order_lo[q]);
		}
	if (perx(ipn))
		for (int JC = 1; JC <= JJC; ++JC) {
			static const int xo_hi[5] = {KW, KS, KNW, KSW, KO};
			static const int xo_lo[5] = {KW, KS, KSW, KNW, KO};
			for (int q = 0; q < 5; ++q) SOC(IIC, JC, xo_hi[q]) = SOC(2, JC, xo_hi[q]);
			for (int q = 0; q < 5; ++q) SOC(1, JC, xo_lo[q]) = SOC(IIC1, JC, xo_lo[q]);
		}
#undef SOC
}

/* ------------------------------------------------- operator-induced P */
/* BMG2_SymStd_SETUP_interp_OI, periodic branch
 * (src/2d/ftn/BMG2_SymStd_SETUP_interp_OI.f90:259-612).  Coarse columns
 * IBEGC..IENDC walk fine columns I through the wrap
 * I = MAX(MOD(I+2, IIFC), MIN(I+2, 3)) (the same for rows), the extra strips
 * fill the coarse ghost lines the corner weights read. */
void o2_setup_interp_per(const double *so, double *ci, int IIF, int JJF, int IIC, int JJC, int ifd, int ipn)
{
#define SO(i, j, k) so[ix3(i, j, k, IIF, JJF)]
#define CI(i, j, k) ci[ix3(i, j, k, IIC, JJC)]
	const double emach = ldexp(1.0, -53);
	const int IIC1 = IIC - 1, JJC1 = JJC - 1;
	const int IIF1 = IIF - 1, IIF2 = IIF - 2, JJF1 = JJF - 1, JJF2 = JJF - 2;
	const int IICF = (IIF - 2) / 2 + 3, JJCF = (JJF - 2) / 2 + 3;
	const int IICF1 = IICF - 1, JJCF1 = JJCF - 1;
	const int IIFC = 2 * (IICF - 2) + 2, JJFC = 2 * (JJCF - 2) + 2;
	int IBEG = 2, IBEGC = 3, IBEG_x = 2, IEND_x = IIF2, IENDC = IICF1, JENDC = JJCF1;
	if (perx(ipn)) {
		IBEG = 0;
		IBEGC = 2;
		if (IIC == IICF) {
			IENDC = IICF;
			IBEG_x = 3;
			IEND_x = IIF1;
		}
	}
	int JBEG = 2, JBEGC = 3, JBEG_y = 2, JEND_y = JJF2;
	if (pery(ipn)) {
		JBEG = 0;
		JBEGC = 2;
		if (JJC == JJCF) {
			JENDC = JJCF;
			JBEG_y = 3;
			JEND_y = JJF1;
		}
	}
#define WRAPI(I) ((I) = imax(((I) + 2) % IIFC, imin((I) + 2, 3)))
#define WRAPJ(J) ((J) = imax(((J) + 2) % JJFC, imin((J) + 2, 3)))
	double A, B, EP, SUM, S;
	/* x-edge weights at (IC, JC) from fine point (I-1, J) */
#define XEDGE(IC, JC, I, J)                                                                                   \
	do {                                                                                                      \
		if (ifd != 1) {                                                                                       \
			A = SO(I, J, KW) + SO(I, J, KNW) + SO(I, J + 1, KSW);                                            \
			B = SO(I - 1, J, KW) + SO(I - 1, J, KSW) + SO(I - 1, J + 1, KNW);                                \
		} else {                                                                                              \
			A = SO(I, J, KW);                                                                                 \
			B = SO(I - 1, J, KW);                                                                             \
		}                                                                                                     \
		EP = fmin(fabs(A / SO(I - 1, J, KO)), fabs(B / SO(I - 1, J, KO)));                                   \
		SUM = A + B + SO(I - 1, J, KS) + SO(I - 1, J + 1, KS);                                               \
		SUM = A + B + (SO(I - 1, J, KO) - SUM) * fmax(SO(I - 1, J, KO) - (1.0 + EP) * SUM, 0.0) /            \
		                  (fabs(SO(I - 1, J, KO) - (1.0 + EP) * SUM) + emach);                                 \
		SUM = 1.0 / SUM;                                                                                      \
		CI(IC, JC, LR) = A * SUM;                                                                             \
		CI(IC, JC, LL) = B * SUM;                                                                             \
	} while (0)
	/* y-edge weights at (IC, JC) from fine point (I, J-1) */
#define YEDGE(IC, JC, I, J)                                                                                   \
	do {                                                                                                      \
		if (ifd != 1) {                                                                                       \
			A = SO(I, J, KS) + SO(I, J, KNW) + SO(I + 1, J, KSW);                                            \
			B = SO(I, J - 1, KS) + SO(I, J - 1, KSW) + SO(I + 1, J - 1, KNW);                                \
		} else {                                                                                              \
			A = SO(I, J, KS);                                                                                 \
			B = SO(I, J - 1, KS);                                                                             \
		}                                                                                                     \
		SUM = A + B + SO(I, J - 1, KW) + SO(I + 1, J - 1, KW);                                               \
		EP = fmin(fabs(A / SO(I, J - 1, KO)), fabs(B / SO(I, J - 1, KO)));                                   \
		SUM = A + B + (SO(I, J - 1, KO) - SUM) * fmax(SO(I, J - 1, KO) - (1.0 + EP) * SUM, 0.0) /            \
		                  (fabs(SO(I, J - 1, KO) - (1.0 + EP) * SUM) + emach);                                 \
		SUM = 1.0 / SUM;                                                                                      \
		CI(IC, JC, LA) = A * SUM;                                                                             \
		CI(IC, JC, LB) = B * SUM;                                                                             \
	} while (0)
	int I, J;
	J = 0;
	for (int JC = 2; JC <= JJC1; ++JC) {
		J += 2;
		I = IBEG;
		for (int IC = IBEGC; IC <= IENDC; ++IC) {
			WRAPI(I);
			XEDGE(IC, JC, I, J);
		}
	}
	if (pery(ipn)) {
		I = IBEG;
		J = JBEG_y;
		for (int IC = IBEGC; IC <= IENDC; ++IC) {
			WRAPI(I);
			XEDGE(IC, JJC, I, J);
		}
		I = IBEG;
		J = JEND_y;
		for (int IC = IBEGC; IC <= IENDC; ++IC) {
			WRAPI(I);
			XEDGE(IC, 1, I, J);
		}
	}
	J = JBEG;
	for (int JC = JBEGC; JC <= JENDC; ++JC) {
		WRAPJ(J);
		I = 0;
		for (int IC = 2; IC <= IIC1; ++IC) {
			I += 2;
			YEDGE(IC, JC, I, J);
		}
	}
	if (perx(ipn)) {
		I = IBEG_x;
		J = JBEG;
		for (int JC = JBEGC; JC <= JENDC; ++JC) {
			WRAPJ(J);
			YEDGE(IIC, JC, I, J);
		}
		I = IEND_x;
		J = JBEG;
		for (int JC = JBEGC; JC <= JENDC; ++JC) {
			WRAPJ(J);
			YEDGE(1, JC, I, J);
		}
	}
	J = JBEG;
	for (int JC = JBEGC; JC <= JENDC; ++JC) {
		WRAPJ(J);
		I = IBEG;
		for (int IC = IBEGC; IC <= IENDC; ++IC) {
			WRAPI(I);
			if (ifd != 1) {
				SUM = SO(I - 1, J - 1, KW) + SO(I - 1, J, KNW) + SO(I - 1, J, KS) + SO(I, J, KSW) + SO(I, J - 1, KW) +
				      SO(I, J - 1, KNW) + SO(I - 1, J - 1, KS) + SO(I - 1, J - 1, KSW);
				EP = fmin(fmin(fabs((SO(I - 1, J - 1, KSW) + SO(I - 1, J - 1, KW) + SO(I - 1, J, KNW)) /
				                    SO(I - 1, J - 1, KO)),
				               fabs((SO(I - 1, J, KNW) + SO(I - 1, J, KS) + SO(I, J, KSW)) / SO(I - 1, J - 1, KO))),
				          fmin(fabs((SO(I, J, KSW) + SO(I, J - 1, KW) + SO(I, J - 1, KNW)) / SO(I - 1, J - 1, KO)),
				               fabs((SO(I, J - 1, KNW) + SO(I - 1, J - 1, KS) + SO(I - 1, J - 1, KSW)) /
				                    SO(I - 1, J - 1, KO))));
			} else {
				SUM = SO(I - 1, J - 1, KW) + SO(I - 1, J, KS) + SO(I, J - 1, KW) + SO(I - 1, J - 1, KS);
				EP = fmin(fmin(fabs(SO(I - 1, J - 1, KW) / SO(I - 1, J - 1, KO)),
				               fabs(SO(I - 1, J, KS) / SO(I - 1, J - 1, KO))),
				          fmin(fabs(SO(I, J - 1, KW) / SO(I - 1, J - 1, KO)),
				               fabs(SO(I - 1, J - 1, KS) / SO(I - 1, J - 1, KO))));
			}
			SUM = SUM + (SO(I - 1, J - 1, KO) - SUM) * fmax(SO(I - 1, J - 1, KO) - (1.0 + EP) * SUM, 0.0) /
			                (fabs(SO(I - 1, J - 1, KO) - (1.0 + EP) * SUM) + emach);
			S = 1.0 / SUM;
			if (ifd != 1) {
				CI(IC, JC, LSW) = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LL) + SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LB) +
				                   SO(I - 1, J - 1, KSW)) * S;
				CI(IC, JC, LSE) = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LR) + SO(I, J - 1, KW) * CI(IC, JC, LB) +
				                   SO(I, J - 1, KNW)) * S;
				CI(IC, JC, LNW) = (SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LA) + SO(I - 1, J, KS) * CI(IC, JC, LL) +
				                   SO(I - 1, J, KNW)) * S;
				CI(IC, JC, LNE) = (SO(I - 1, J, KS) * CI(IC, JC, LR) + SO(I, J - 1, KW) * CI(IC, JC, LA) +
				                   SO(I, J, KSW)) * S;
			} else {
				CI(IC, JC, LSW) = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LL) + SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LB)) * S;
				CI(IC, JC, LSE) = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, LR) + SO(I, J - 1, KW) * CI(IC, JC, LB)) * S;
				CI(IC, JC, LNW) = (SO(I - 1, J - 1, KW) * CI(IC - 1, JC, LA) + SO(I - 1, J, KS) * CI(IC, JC, LL)) * S;
				CI(IC, JC, LNE) = (SO(I - 1, J, KS) * CI(IC, JC, LR) + SO(I, J - 1, KW) * CI(IC, JC, LA)) * S;
			}
		}
	}
#undef XEDGE
#undef YEDGE
#undef WRAPI
#undef WRAPJ
#undef SO
#undef CI
}

/* ------------------------------------------------ coarsest-grid solve */
/* Upper Cholesky of a dense SPD matrix in column-major storage (leading
 * dimension lda): the unblocked LAPACK algorithm (DPOTF2; each column's
 * pivot from a sequential dot product, the row to its right updated by a
 * transposed matrix-vector product and scaled by the pivot's reciprocal).
 * Returns the failing column (1-based) or 0. */
int o_dpotf2_u(int n, double *a, int lda)
{
#define A(i, j) a[(size_t)((j) - 1) * lda + ((i) - 1)]
	for (int j = 1; j <= n; ++j) {
		double dot = 0.0;
		for (int i = 1; i < j; ++i) dot += A(i, j) * A(i, j);
		double ajj = A(j, j) - dot;
		if (ajj <= 0.0 || ajj != ajj) {
			A(j, j) = ajj;
			return j;
		}
		ajj = sqrt(ajj);
		A(j, j) = ajj;
		if (j < n) {
			for (int k = j + 1; k <= n; ++k) {
				double temp = 0.0;
				for (int i = 1; i < j; ++i) temp += A(i, k) * A(i, j);
				A(j, k) = A(j, k) + -1.0 * temp;
			}
			const double r = 1.0 / ajj;
			for (int k = j + 1; k <= n; ++k) A(j, k) = r * A(j, k);
		}
	}
	return 0;
#undef A
}

/* DPOTRS('U'): U^T y = b, then U x = y (the two triangular solves of DTRSM
 * for one right-hand side, in its loop order). */
void o_dpotrs_u(int n, const double *a, int lda, double *b)
{
#define A(i, j) a[(size_t)((j) - 1) * lda + ((i) - 1)]
	for (int i = 1; i <= n; ++i) {
		double temp = b[i - 1];
		for (int k = 1; k < i; ++k) temp = temp - A(k, i) * b[k - 1];
		b[i - 1] = temp / A(i, i);
	}
	for (int k = n; k >= 1; --k)
		if (b[k - 1] != 0.0) {
			b[k - 1] = b[k - 1] / A(k, k);
			for (int i = 1; i < k; ++i) b[i - 1] = b[i - 1] - b[k - 1] * A(i, k);
		}
#undef A
}

/* BMG2_SymStd_SETUP_cg_LU, periodic branches (src/2d/ftn/BMG2_SymStd_SETUP_cg_LU.f90:120-227
 * nine-point, :256-343 five-point): the coarsest operator as a dense N x N
 * upper triangle (N = (II-2)(JJ-2), ABD(NABD1 = N, N)) with the wrap-around
 * couplings, factored by DPOTRF.  Returns the failing column or 0. */
int o2_setup_cg_per(const double *so, int II, int JJ, int nstncl, double *abd, int ipn)
{
#define SO(i, j, k) so[ix3(i, j, k, II, JJ)]
	const int I1 = II - 1, J1 = JJ - 1, I2 = I1 - 1, N = I2 * (J1 - 1);
#define ABD(i, j) abd[(size_t)((j) - 1) * N + ((i) - 1)]
	memset(abd, 0, sizeof(double) * (size_t)N * N);
	const int nine = nstncl == 5;
	int KK = 1;
	ABD(1, 1) = SO(2, 2, KO);
	for (int I = 3; I <= I1; ++I) {
		KK = KK + 1;
		ABD(KK, KK) = SO(I, 2, KO);
		ABD(KK - 1, KK) = -SO(I, 2, KW);
	}
	if (perx(ipn)) ABD(KK - I2 + 1, KK) = -SO(II, 2, KW);
	for (int J = 3; J <= J1; ++J) {
		if (perx(ipn)) ABD(KK, KK + 1) = nine ? -SO(2, J, KSW) : 0.0;
		for (int I = 2; I <= I1; ++I) {
			KK = KK + 1;
			ABD(KK, KK) = SO(I, J, KO);
			if (I != 2) {
				ABD(KK - 1, KK) = -SO(I, J, KW);
				ABD(KK - I2 - 1, KK) = nine ? -SO(I, J, KSW) : 0.0;
			}
			ABD(KK - I2 + 1, KK) = nine ? -SO(I + 1, J, KNW) : 0.0;
			ABD(KK - I2, KK) = -SO(I, J, KS);
		}
		if (perx(ipn)) {
			ABD(KK - I2 + 1, KK) = -SO(II, J, KW);
			ABD(KK - 2 * I2 + 1, KK) = nine ? -SO(II, J, KNW) : 0.0;
		}
	}
	if (pery(ipn)) {
		KK = KK - I2;
		const int J2 = (J1 - 2) * I2;
		KK = KK + 1;
		ABD(KK - J2, KK) = -SO(2, JJ, KS);
		ABD(KK - J2 + 1, KK) = nine ? -SO(3, JJ, KSW) : 0.0;
		if (ipn == PER_XY) ABD(I2, KK) = nine ? -SO(2, JJ, KNW) : 0.0;
		for (int I = 3; I <= I1; ++I) {
			KK = KK + 1;
			ABD(KK - J2, KK) = -SO(I, JJ, KS);
			ABD(KK - J2 - 1, KK) = nine ? -SO(I, JJ, KNW) : 0.0;
			ABD(KK - J2 + 1, KK) = nine ? -SO(I + 1, JJ, KSW) : 0.0;
		}
		ABD(KK - J2 + 1, KK) = 0.0;
		if (ipn == PER_XY) ABD(1, KK) = nine ? -SO(II, JJ, KSW) : 0.0;
		if (perx(ipn)) ABD(KK - 2 * I2 + 1, KK) = nine ? -SO(II, J1, KNW) : 0.0;
	}
#undef ABD
#undef SO
	return o_dpotf2_u(N, abd, N);
}

/* BMG2_SymStd_SOLVE_cg, periodic branch (src/2d/ftn/BMG2_SymStd_SOLVE_cg.f90:88-163):
 * DPOTRS with the dense factor, the mean-zero shift (JPN != 0), the ghosts. */
void o2_solve_cg_per(double *q, const double *qf, int II, int JJ, const double *abd, double *bbd, int ipn)
{
#define Q(i, j) q[ix2(i, j, II)]
#define QF(i, j) qf[ix2(i, j, II)]
	const int I1 = II - 1, J1 = JJ - 1, I2 = I1 - 1, N = I2 * (J1 - 1);
	int KK = 0;
	for (int J = 2; J <= J1; ++J)
		for (int I = 2; I <= I1; ++I) bbd[KK++] = QF(I, J);
	o_dpotrs_u(N, abd, N, bbd);
	KK = 0;
	for (int J = 2; J <= J1; ++J)
		for (int I = 2; I <= I1; ++I) Q(I, J) = bbd[KK++];
	double CINT = 0.0, QINT = 0.0;
	for (int J = 2; J <= J1; ++J)
		for (int I = 2; I <= I1; ++I) {
			QINT = QINT + Q(I, J);
			CINT = CINT + 1;
		}
	const double C = -QINT / CINT;
	for (int J = 2; J <= J1; ++J)
		for (int I = 2; I <= I1; ++I) Q(I, J) = Q(I, J) + C;
	if (pery(ipn))
		for (int I = 2; I <= I1; ++I) {
			Q(I, JJ) = Q(I, 2);
			Q(I, 1) = Q(I, J1);
		}
	if (perx(ipn))
		for (int J = 2; J <= J1; ++J) {
			Q(II, J) = Q(2, J);
			Q(1, J) = Q(I1, J);
		}
	if (ipn == PER_XY) {
		Q(1, 1) = Q(I1, J1);
		Q(II, 1) = Q(2, J1);
		Q(1, JJ) = Q(I1, 2);
		Q(II, JJ) = Q(2, 2);
	}
#undef Q
#undef QF
}
