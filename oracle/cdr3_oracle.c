/*
 * cdr3_oracle.c -- CPU restatement of Cedar's serial 3D BoxMG path
 * (27-point and seven-point fine operators, point and plane relaxation).
 *
 * TEST INFRASTRUCTURE ONLY: the parity oracle for the 3D CUDA kernels.
 *
 * Layout as the reference: Fortran order (i fastest), one ghost layer, one
 * plane per stencil direction; indices in the routines are the reference's
 * 1-based Fortran indices.  Stencil planes (src/3d/ftn/BMG_stencils_f90.h):
 * kp=1 kpw=2 kps=3 kb=4 kpsw=5 kpnw=6 kbw=7 kbnw=8 kbn=9 kbne=10 kbe=11
 * kbse=12 kbs=13 kbsw=14; interpolation planes lxyl=1 .. ltse=26.
 *
 * The Galerkin coarse operator is formed as P^T A P from the interpolation
 * that BMG3_SymStd_interp_add applies (the reference's expanded
 * BMG3_SymStd_SETUP_ITLI27_ex formulas are that same product; its 2D
 * counterpart is restated term by term in cdr2_oracle.c and agrees with the
 * direct product to rounding).  A seven-point fine operator (seven_pt: planes
 * p, pw, ps, b) has its own residual, red-black Gauss-Seidel, interpolation
 * and plane-relaxation branches; its Galerkin product (which the reference
 * expands separately in BMG3_SymStd_SETUP_ITLI07_ex) is the same P^T A P with
 * the missing couplings zero.  Periodic and indefinite branches are not
 * restated.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "cdr2_oracle.h"
#include "cdr3_oracle.h"

enum { KP = 1, KPW, KPS, KB, KPSW, KPNW, KBW, KBNW, KBN, KBNE, KBE, KBSE, KBS, KBSW };
enum { LXYL = 1, LXYR, LXYA, LXYB, LXZA, LXZB, LXYNE, LXYSE, LXYSW, LXYNW, LXZSW, LXZNW, LXZNE, LXZSE,
       LYZSW, LYZNW, LYZNE, LYZSE, LBSW, LBNW, LBNE, LBSE, LTSW, LTNW, LTNE, LTSE };

static inline size_t ix3(long i, long j, long k, long ii, long jj) { return ((size_t)(k - 1) * jj + (j - 1)) * ii + (i - 1); }
static inline size_t ix4(long i, long j, long k, long p, long ii, long jj, long kk)
{
	return (((size_t)(p - 1) * kk + (k - 1)) * jj + (j - 1)) * ii + (i - 1);
}

int o_dpbtrf_u(int n, int kd, double *ab, int ldab);
void o_dpbtrs_u(int n, int kd, const double *ab, int ldab, double *x);

#define SO(i, j, k, p) so[ix4(i, j, k, p, II, JJ, KK)]
#define Q(i, j, k) q[ix3(i, j, k, II, JJ)]
#define QF(i, j, k) qf[ix3(i, j, k, II, JJ)]

/* the 26 neighbour terms of BMG3_SymStd_residual.f90:76-101, in its order */
#define NB27(i, j, k)                                                                                        \
	(SO(i, j, k, KPW) * Q(i - 1, j, k) + SO(i, j + 1, k, KPNW) * Q(i - 1, j + 1, k)                          \
	 + SO(i, j + 1, k, KPS) * Q(i, j + 1, k) + SO(i + 1, j + 1, k, KPSW) * Q(i + 1, j + 1, k)                \
	 + SO(i + 1, j, k, KPW) * Q(i + 1, j, k) + SO(i + 1, j, k, KPNW) * Q(i + 1, j - 1, k)                    \
	 + SO(i, j, k, KPS) * Q(i, j - 1, k) + SO(i, j, k, KPSW) * Q(i - 1, j - 1, k)                            \
	 + SO(i, j, k, KB) * Q(i, j, k - 1) + SO(i, j, k, KBW) * Q(i - 1, j, k - 1)                              \
	 + SO(i, j + 1, k, KBNW) * Q(i - 1, j + 1, k - 1) + SO(i, j + 1, k, KBN) * Q(i, j + 1, k - 1)            \
	 + SO(i + 1, j + 1, k, KBNE) * Q(i + 1, j + 1, k - 1) + SO(i + 1, j, k, KBE) * Q(i + 1, j, k - 1)        \
	 + SO(i + 1, j, k, KBSE) * Q(i + 1, j - 1, k - 1) + SO(i, j, k, KBS) * Q(i, j - 1, k - 1)                \
	 + SO(i, j, k, KBSW) * Q(i - 1, j - 1, k - 1) + SO(i, j, k + 1, KB) * Q(i, j, k + 1)                     \
	 + SO(i, j, k + 1, KBE) * Q(i - 1, j, k + 1) + SO(i, j + 1, k + 1, KBSE) * Q(i - 1, j + 1, k + 1)        \
	 + SO(i, j + 1, k + 1, KBS) * Q(i, j + 1, k + 1) + SO(i + 1, j + 1, k + 1, KBSW) * Q(i + 1, j + 1, k + 1) \
	 + SO(i + 1, j, k + 1, KBW) * Q(i + 1, j, k + 1) + SO(i + 1, j, k + 1, KBNW) * Q(i + 1, j - 1, k + 1)    \
	 + SO(i, j, k + 1, KBN) * Q(i, j - 1, k + 1) + SO(i, j, k + 1, KBNE) * Q(i - 1, j - 1, k + 1))

/* BMG3_SymStd_residual, src/3d/ftn/BMG3_SymStd_residual.f90:67-121 (27-point branch) */
void o3_residual(const double *so, const double *qf, const double *q, double *res, int II, int JJ, int KK)
{
	for (int k = 2; k <= KK - 1; ++k)
		for (int j = 2; j <= JJ - 1; ++j)
			for (int i = 2; i <= II - 1; ++i) {
				double nb = QF(i, j, k) + SO(i, j, k, KPW) * Q(i - 1, j, k);
				/* same left-to-right order as the Fortran expression */
				nb = nb + SO(i, j + 1, k, KPNW) * Q(i - 1, j + 1, k) + SO(i, j + 1, k, KPS) * Q(i, j + 1, k)
				     + SO(i + 1, j + 1, k, KPSW) * Q(i + 1, j + 1, k) + SO(i + 1, j, k, KPW) * Q(i + 1, j, k)
				     + SO(i + 1, j, k, KPNW) * Q(i + 1, j - 1, k) + SO(i, j, k, KPS) * Q(i, j - 1, k)
				     + SO(i, j, k, KPSW) * Q(i - 1, j - 1, k) + SO(i, j, k, KB) * Q(i, j, k - 1)
				     + SO(i, j, k, KBW) * Q(i - 1, j, k - 1) + SO(i, j + 1, k, KBNW) * Q(i - 1, j + 1, k - 1)
				     + SO(i, j + 1, k, KBN) * Q(i, j + 1, k - 1) + SO(i + 1, j + 1, k, KBNE) * Q(i + 1, j + 1, k - 1)
				     + SO(i + 1, j, k, KBE) * Q(i + 1, j, k - 1) + SO(i + 1, j, k, KBSE) * Q(i + 1, j - 1, k - 1)
				     + SO(i, j, k, KBS) * Q(i, j - 1, k - 1) + SO(i, j, k, KBSW) * Q(i - 1, j - 1, k - 1)
				     + SO(i, j, k + 1, KB) * Q(i, j, k + 1) + SO(i, j, k + 1, KBE) * Q(i - 1, j, k + 1)
				     + SO(i, j + 1, k + 1, KBSE) * Q(i - 1, j + 1, k + 1) + SO(i, j + 1, k + 1, KBS) * Q(i, j + 1, k + 1)
				     + SO(i + 1, j + 1, k + 1, KBSW) * Q(i + 1, j + 1, k + 1) + SO(i + 1, j, k + 1, KBW) * Q(i + 1, j, k + 1)
				     + SO(i + 1, j, k + 1, KBNW) * Q(i + 1, j - 1, k + 1) + SO(i, j, k + 1, KBN) * Q(i, j - 1, k + 1)
				     + SO(i, j, k + 1, KBNE) * Q(i - 1, j - 1, k + 1);
				res[ix3(i, j, k, II, JJ)] = nb - SO(i, j, k, KP) * Q(i, j, k);
			}
}

/* BMG3_SymStd_SETUP_recip, src/3d/ftn/BMG3_SymStd_SETUP_recip.f90:63-69 */
void o3_setup_recip(const double *so, double *sor, int II, int JJ, int KK)
{
	for (int k = 2; k <= KK - 1; ++k)
		for (int j = 2; j <= JJ - 1; ++j)
			for (int i = 2; i <= II - 1; ++i) sor[ix3(i, j, k, II, JJ)] = 1.0 / SO(i, j, k, KP);
}

/* BMG3_SymStd_relax_GS, src/3d/ftn/BMG3_SymStd_relax_GS.f90:80-138 (27-point, 8 colours):
 * colour pts has parities (i, j, k) = bits of pts-1; UP runs 1..8, DOWN 8..1. */
void o3_relax_gs(const double *so, const double *qf, double *q, const double *sor, int II, int JJ, int KK, int updown)
{
	int pstart = updown == 1 ? 1 : 8, pend = updown == 1 ? 8 : 1, pstride = updown == 1 ? 1 : -1;
	for (int pts = pstart; pstride > 0 ? pts <= pend : pts >= pend; pts += pstride)
		for (int k = 2 + ((pts - 1) / 4) % 2; k <= KK - 1; k += 2)
			for (int j = 2 + ((pts - 1) / 2) % 2; j <= JJ - 1; j += 2)
				for (int i = 2 + (pts - 1) % 2; i <= II - 1; i += 2) {
					double acc = QF(i, j, k) + SO(i, j, k, KPW) * Q(i - 1, j, k);
					acc = acc + SO(i, j + 1, k, KPNW) * Q(i - 1, j + 1, k) + SO(i, j + 1, k, KPS) * Q(i, j + 1, k)
					      + SO(i + 1, j + 1, k, KPSW) * Q(i + 1, j + 1, k) + SO(i + 1, j, k, KPW) * Q(i + 1, j, k)
					      + SO(i + 1, j, k, KPNW) * Q(i + 1, j - 1, k) + SO(i, j, k, KPS) * Q(i, j - 1, k)
					      + SO(i, j, k, KPSW) * Q(i - 1, j - 1, k) + SO(i, j, k, KB) * Q(i, j, k - 1)
					      + SO(i, j, k, KBW) * Q(i - 1, j, k - 1) + SO(i, j + 1, k, KBNW) * Q(i - 1, j + 1, k - 1)
					      + SO(i, j + 1, k, KBN) * Q(i, j + 1, k - 1) + SO(i + 1, j + 1, k, KBNE) * Q(i + 1, j + 1, k - 1)
					      + SO(i + 1, j, k, KBE) * Q(i + 1, j, k - 1) + SO(i + 1, j, k, KBSE) * Q(i + 1, j - 1, k - 1)
					      + SO(i, j, k, KBS) * Q(i, j - 1, k - 1) + SO(i, j, k, KBSW) * Q(i - 1, j - 1, k - 1)
					      + SO(i, j, k + 1, KB) * Q(i, j, k + 1) + SO(i, j, k + 1, KBE) * Q(i - 1, j, k + 1)
					      + SO(i, j + 1, k + 1, KBSE) * Q(i - 1, j + 1, k + 1) + SO(i, j + 1, k + 1, KBS) * Q(i, j + 1, k + 1)
					      + SO(i + 1, j + 1, k + 1, KBSW) * Q(i + 1, j + 1, k + 1) + SO(i + 1, j, k + 1, KBW) * Q(i + 1, j, k + 1)
					      + SO(i + 1, j, k + 1, KBNW) * Q(i + 1, j - 1, k + 1) + SO(i, j, k + 1, KBN) * Q(i, j - 1, k + 1)
					      + SO(i, j, k + 1, KBNE) * Q(i - 1, j - 1, k + 1);
					Q(i, j, k) = acc * sor[ix3(i, j, k, II, JJ)];
				}
}
#undef Q
#undef QF

/* BMG3_SymStd_restrict, src/3d/ftn/BMG3_SymStd_restrict.f90:114-154 */
void o3_restrict(const double *ci, const double *q, double *qc, int Nx, int Ny, int Nz, int Nxc, int Nyc, int Nzc)
{
#define CI(i, j, k, l) ci[ix4(i, j, k, l, Nxc, Nyc, Nzc)]
#define Q(i, j, k) q[ix3(i, j, k, Nx, Ny)]
	(void)Nz;
	int k = 0;
	for (int kc = 2; kc <= Nzc - 1; ++kc) {
		k += 2;
		int j = 0;
		for (int jc = 2; jc <= Nyc - 1; ++jc) {
			j += 2;
			int i = 0;
			for (int ic = 2; ic <= Nxc - 1; ++ic) {
				i += 2;
				qc[ix3(ic, jc, kc, Nxc, Nyc)] =
				    CI(ic, jc, kc, LXYNE) * Q(i - 1, j - 1, k) + CI(ic, jc, kc, LXYA) * Q(i, j - 1, k)
				    + CI(ic + 1, jc, kc, LXYNW) * Q(i + 1, j - 1, k) + CI(ic, jc, kc, LXYR) * Q(i - 1, j, k) + Q(i, j, k)
				    + CI(ic + 1, jc, kc, LXYL) * Q(i + 1, j, k) + CI(ic, jc + 1, kc, LXYSE) * Q(i - 1, j + 1, k)
				    + CI(ic, jc + 1, kc, LXYB) * Q(i, j + 1, k) + CI(ic + 1, jc + 1, kc, LXYSW) * Q(i + 1, j + 1, k)
				    + CI(ic, jc, kc, LTNE) * Q(i - 1, j - 1, k - 1) + CI(ic, jc, kc, LYZNW) * Q(i, j - 1, k - 1)
				    + CI(ic + 1, jc, kc, LTNW) * Q(i + 1, j - 1, k - 1) + CI(ic, jc, kc, LXZNE) * Q(i - 1, j, k - 1)
				    + CI(ic, jc, kc, LXZA) * Q(i, j, k - 1) + CI(ic + 1, jc, kc, LXZNW) * Q(i + 1, j, k - 1)
				    + CI(ic, jc + 1, kc, LTSE) * Q(i - 1, j + 1, k - 1) + CI(ic, jc + 1, kc, LYZNE) * Q(i, j + 1, k - 1)
				    + CI(ic + 1, jc + 1, kc, LTSW) * Q(i + 1, j + 1, k - 1) + CI(ic, jc, kc + 1, LBNE) * Q(i - 1, j - 1, k + 1)
				    + CI(ic, jc, kc + 1, LYZSW) * Q(i, j - 1, k + 1) + CI(ic + 1, jc, kc + 1, LBNW) * Q(i + 1, j - 1, k + 1)
				    + CI(ic, jc, kc + 1, LXZSE) * Q(i - 1, j, k + 1) + CI(ic, jc, kc + 1, LXZB) * Q(i, j, k + 1)
				    + CI(ic + 1, jc, kc + 1, LXZSW) * Q(i + 1, j, k + 1) + CI(ic, jc + 1, kc + 1, LBSE) * Q(i - 1, j + 1, k + 1)
				    + CI(ic, jc + 1, kc + 1, LYZSE) * Q(i, j + 1, k + 1) + CI(ic + 1, jc + 1, kc + 1, LBSW) * Q(i + 1, j + 1, k + 1);
			}
		}
	}
#undef CI
#undef Q
}

/* BMG3_SymStd_interp_add, src/3d/ftn/BMG3_SymStd_interp_add.f90:88-239 (non-periodic);
 * so_kp is the fine operator's kp plane; res is divided in place. */
void o3_interp_add(double *q, const double *qc, double *res, const double *so_kp, const double *ci, int iic, int jjc,
                   int kkc, int iif, int jjf, int kkf)
{
#define CI(i, j, k, l) ci[ix4(i, j, k, l, iic, jjc, kkc)]
#define Q(i, j, k) q[ix3(i, j, k, iif, jjf)]
#define QC(i, j, k) qc[ix3(i, j, k, iic, jjc)]
#define RES(i, j, k) res[ix3(i, j, k, iif, jjf)]
	int iic1 = iic - 1, jjc1 = jjc - 1, kkc1 = kkc - 1;
	int iicf1 = (iif - 2) / 2 + 2, jjcf1 = (jjf - 2) / 2 + 2, kkcf1 = (kkf - 2) / 2 + 2;
	for (int k = 2; k <= kkf - 1; ++k)
		for (int j = 2; j <= jjf - 1; ++j)
			for (int i = 2; i <= iif - 1; ++i) RES(i, j, k) = RES(i, j, k) / so_kp[ix3(i, j, k, iif, jjf)];
	int k = 0;
	for (int kc = 2; kc <= kkc1; ++kc) {
		k += 2;
		int j = 2, i = 2;
		Q(2, 2, k) = Q(2, 2, k) + QC(2, 2, kc);
		for (int ic = 3; ic <= iicf1; ++ic) {
			i += 2;
			Q(i, 2, k) = Q(i, 2, k) + QC(ic, 2, kc);
			double a = CI(ic, 2, kc, LXYR) * QC(ic, 2, kc) + CI(ic, 2, kc, LXYL) * QC(ic - 1, 2, kc);
			Q(i - 1, j, k) = Q(i - 1, j, k) + a + RES(i - 1, j, k);
		}
		for (int jc = 3; jc <= jjcf1; ++jc) {
			j += 2;
			i = 2;
			Q(2, j, k) = Q(2, j, k) + QC(2, jc, kc);
			double aq = CI(2, jc, kc, LXYA) * QC(2, jc, kc) + CI(2, jc, kc, LXYB) * QC(2, jc - 1, kc);
			Q(2, j - 1, k) = Q(2, j - 1, k) + aq + RES(2, j - 1, k);
			for (int ic = 3; ic <= iicf1; ++ic) {
				i += 2;
				Q(i, j, k) = Q(i, j, k) + QC(ic, jc, kc);
				double a = CI(ic, jc, kc, LXYR) * QC(ic, jc, kc) + CI(ic, jc, kc, LXYL) * QC(ic - 1, jc, kc);
				Q(i - 1, j, k) = Q(i - 1, j, k) + a + RES(i - 1, j, k);
				aq = CI(ic, jc, kc, LXYA) * QC(ic, jc, kc) + CI(ic, jc, kc, LXYB) * QC(ic, jc - 1, kc);
				Q(i, j - 1, k) = Q(i, j - 1, k) + aq + RES(i, j - 1, k);
				a = CI(ic, jc, kc, LXYSW) * QC(ic - 1, jc - 1, kc) + CI(ic, jc, kc, LXYNW) * QC(ic - 1, jc, kc)
				    + CI(ic, jc, kc, LXYNE) * QC(ic, jc, kc) + CI(ic, jc, kc, LXYSE) * QC(ic, jc - 1, kc);
				Q(i - 1, j - 1, k) = Q(i - 1, j - 1, k) + a + RES(i - 1, j - 1, k);
			}
		}
	}
	k = 1;
	for (int kc = 3; kc <= kkcf1; ++kc) {
		k += 2;
		int j = 2, jc = 2, i = 0;
		for (int ic = 2; ic <= iic1; ++ic) {
			i += 2;
			Q(i, j, k) = Q(i, j, k) + CI(ic, jc, kc, LXZA) * QC(ic, jc, kc) + CI(ic, jc, kc, LXZB) * QC(ic, jc, kc - 1)
			             + RES(i, j, k);
		}
		j = 2;
		for (jc = 3; jc <= jjcf1; ++jc) {
			j += 2;
			i = 0;
			for (int ic = 2; ic <= iic1; ++ic) {
				i += 2;
				Q(i, j, k) = Q(i, j, k) + CI(ic, jc, kc, LXZA) * QC(ic, jc, kc) + CI(ic, jc, kc, LXZB) * QC(ic, jc, kc - 1)
				             + RES(i, j, k);
				Q(i, j - 1, k) = Q(i, j - 1, k) + CI(ic, jc, kc, LYZNW) * QC(ic, jc, kc) + CI(ic, jc, kc, LYZNE) * QC(ic, jc - 1, kc)
				                 + CI(ic, jc, kc, LYZSW) * QC(ic, jc, kc - 1) + CI(ic, jc, kc, LYZSE) * QC(ic, jc - 1, kc - 1)
				                 + RES(i, j - 1, k);
			}
		}
	}
	k = 1;
	for (int kc = 3; kc <= kkcf1; ++kc) {
		k += 2;
		int j = 2, jc = 2, i = 1;
		for (int ic = 3; ic <= iicf1; ++ic) {
			i += 2;
			Q(i, j, k) = Q(i, j, k) + CI(ic, jc, kc, LXZNW) * QC(ic - 1, jc, kc) + CI(ic, jc, kc, LXZNE) * QC(ic, jc, kc)
			             + CI(ic, jc, kc, LXZSW) * QC(ic - 1, jc, kc - 1) + CI(ic, jc, kc, LXZSE) * QC(ic, jc, kc - 1)
			             + RES(i, j, k);
		}
		j = 2;
		for (jc = 3; jc <= jjcf1; ++jc) {
			j += 2;
			i = 1;
			for (int ic = 3; ic <= iicf1; ++ic) {
				i += 2;
				Q(i, j, k) = Q(i, j, k) + CI(ic, jc, kc, LXZNW) * QC(ic - 1, jc, kc) + CI(ic, jc, kc, LXZNE) * QC(ic, jc, kc)
				             + CI(ic, jc, kc, LXZSW) * QC(ic - 1, jc, kc - 1) + CI(ic, jc, kc, LXZSE) * QC(ic, jc, kc - 1)
				             + RES(i, j, k);
				Q(i, j - 1, k) = Q(i, j - 1, k) + CI(ic, jc, kc, LTNW) * QC(ic - 1, jc, kc) + CI(ic, jc, kc, LTNE) * QC(ic, jc, kc)
				                 + CI(ic, jc, kc, LTSW) * QC(ic - 1, jc - 1, kc) + CI(ic, jc, kc, LTSE) * QC(ic, jc - 1, kc)
				                 + CI(ic, jc, kc, LBNW) * QC(ic - 1, jc, kc - 1) + CI(ic, jc, kc, LBNE) * QC(ic, jc, kc - 1)
				                 + CI(ic, jc, kc, LBSW) * QC(ic - 1, jc - 1, kc - 1) + CI(ic, jc, kc, LBSE) * QC(ic, jc - 1, kc - 1)
				                 + RES(i, j - 1, k);
			}
		}
	}
	(void)jjc1;
#undef CI
#undef Q
#undef QC
#undef RES
}

static double dmin2(double a, double b) { return a < b ? a : b; }

/* BMG3_SymStd_SETUP_interp_OI, src/3d/ftn/BMG3_SymStd_SETUP_interp_OI.f90:121-537
 * (non-periodic, 27-point fine operator).  emach = D1MACH(3) = 2^-53. */
void o3_setup_interp(const double *so, double *ci, int iif, int jjf, int kkf, int iic, int jjc, int kkc)
{
	const int II = iif, JJ = jjf, KK = kkf;
#define CI(i, j, k, l) ci[ix4(i, j, k, l, iic, jjc, kkc)]
	const double emach = ldexp(1.0, -53);
	int iic1 = iic - 1, jjc1 = jjc - 1, kkc1 = kkc - 1;
	int iicf1 = (iif - 2) / 2 + 2, jjcf1 = (jjf - 2) / 2 + 2, kkcf1 = (kkf - 2) / 2 + 2;
	double a, b, c, ep, dnw, dn, dne, dw, de, dsw, ds, dse, dp, sum;
	int i, j, k;
	/* fine points on CF k-planes on fine-only y-lines (x-edges): lxyl, lxyr */
	k = 0;
	for (int kc = 2; kc <= kkc1; ++kc) {
		k += 2;
		j = 0;
		for (int jc = 2; jc <= jjc1; ++jc) {
			j += 2;
			i = 2;
			for (int ic = 3; ic <= iicf1; ++ic) {
				i += 2;
				a = SO(i - 1, j + 1, k, KPNW) + SO(i - 1, j, k, KPW) + SO(i - 1, j, k, KPSW) + SO(i - 1, j + 1, k, KBNW)
				    + SO(i - 1, j, k, KBW) + SO(i - 1, j, k, KBSW) + SO(i - 1, j + 1, k + 1, KBSE) + SO(i - 1, j, k + 1, KBE)
				    + SO(i - 1, j, k + 1, KBNE);
				b = SO(i, j + 1, k, KPSW) + SO(i, j, k, KPW) + SO(i, j, k, KPNW) + SO(i, j + 1, k, KBNE) + SO(i, j, k, KBE)
				    + SO(i, j, k, KBSE) + SO(i, j + 1, k + 1, KBSW) + SO(i, j, k + 1, KBW) + SO(i, j, k + 1, KBNW);
				c = a + b + SO(i - 1, j, k, KPS) + SO(i - 1, j + 1, k, KPS) + SO(i - 1, j + 1, k, KBN) + SO(i - 1, j, k, KB)
				    + SO(i - 1, j, k, KBS) + SO(i - 1, j + 1, k + 1, KBS) + SO(i - 1, j, k + 1, KB) + SO(i - 1, j, k + 1, KBN);
				ep = dmin2(fabs(a / SO(i - 1, j, k, KP)), fabs(b / SO(i - 1, j, k, KP)));
				c = a + b + (SO(i - 1, j, k, KP) - c) * fmax(SO(i - 1, j, k, KP) - (1.0 + ep) * c, 0.0)
				            / (fabs(SO(i - 1, j, k, KP) - (1.0 + ep) * c) + emach);
				CI(ic, jc, kc, LXYL) = a / c;
				CI(ic, jc, kc, LXYR) = b / c;
			}
		}
	}
	/* CF k-planes on fine-only x-lines (y-edges): lxya, lxyb */
	k = 0;
	for (int kc = 2; kc <= kkc1; ++kc) {
		k += 2;
		j = 2;
		for (int jc = 3; jc <= jjcf1; ++jc) {
			j += 2;
			i = 0;
			for (int ic = 2; ic <= iic1; ++ic) {
				i += 2;
				a = SO(i, j, k, KPNW) + SO(i, j, k, KPS) + SO(i + 1, j, k, KPSW) + SO(i, j, k, KBNW) + SO(i, j, k, KBN)
				    + SO(i + 1, j, k, KBNE) + SO(i, j, k + 1, KBSE) + SO(i, j, k + 1, KBS) + SO(i + 1, j, k + 1, KBSW);
				b = SO(i, j - 1, k, KPSW) + SO(i, j - 1, k, KPS) + SO(i + 1, j - 1, k, KPNW) + SO(i, j - 1, k, KBSW)
				    + SO(i, j - 1, k, KBS) + SO(i + 1, j - 1, k, KBSE) + SO(i, j - 1, k + 1, KBNE) + SO(i, j - 1, k + 1, KBN)
				    + SO(i + 1, j - 1, k + 1, KBNW);
				ep = dmin2(fabs(a / SO(i, j - 1, k, KP)), fabs(b / SO(i, j - 1, k, KP)));
				c = a + b + SO(i, j - 1, k, KPW) + SO(i + 1, j - 1, k, KPW) + SO(i, j - 1, k, KBW) + SO(i, j - 1, k, KB)
				    + SO(i + 1, j - 1, k, KBE) + SO(i, j - 1, k + 1, KBE) + SO(i, j - 1, k + 1, KB) + SO(i + 1, j - 1, k + 1, KBW);
				c = a + b + (SO(i, j - 1, k, KP) - c) * fmax(SO(i, j - 1, k, KP) - (1.0 + ep) * c, 0.0)
				            / (fabs(SO(i, j - 1, k, KP) - (1.0 + ep) * c) + emach);
				CI(ic, jc, kc, LXYA) = a / c;
				CI(ic, jc, kc, LXYB) = b / c;
			}
		}
	}
	/* CF j-planes on fine-only x-lines (z-edges): lxza, lxzb */
	k = 2;
	for (int kc = 3; kc <= kkcf1; ++kc) {
		k += 2;
		j = 0;
		for (int jc = 2; jc <= jjc1; ++jc) {
			j += 2;
			i = 0;
			for (int ic = 2; ic <= iic1; ++ic) {
				i += 2;
				a = SO(i, j + 1, k, KBSE) + SO(i, j + 1, k, KBS) + SO(i + 1, j + 1, k, KBSW) + SO(i, j, k, KBE) + SO(i, j, k, KB)
				    + SO(i + 1, j, k, KBW) + SO(i, j, k, KBNE) + SO(i, j, k, KBN) + SO(i + 1, j, k, KBNW);
				b = SO(i, j + 1, k - 1, KBNW) + SO(i, j + 1, k - 1, KBN) + SO(i + 1, j + 1, k - 1, KBNE) + SO(i, j, k - 1, KBW)
				    + SO(i, j, k - 1, KB) + SO(i + 1, j, k - 1, KBE) + SO(i, j, k - 1, KBSW) + SO(i, j, k - 1, KBS)
				    + SO(i + 1, j, k - 1, KBSE);
				c = a + b + SO(i, j, k - 1, KPW) + SO(i + 1, j, k - 1, KPW) + SO(i, j + 1, k - 1, KPNW) + SO(i, j + 1, k - 1, KPS)
				    + SO(i + 1, j + 1, k - 1, KPSW) + SO(i, j, k - 1, KPSW) + SO(i, j, k - 1, KPS) + SO(i + 1, j, k - 1, KPNW);
				ep = dmin2(fabs(a / SO(i, j, k - 1, KP)), fabs(b / SO(i, j, k - 1, KP)));
				c = a + b + (SO(i, j, k - 1, KP) - c) * fmax(SO(i, j, k - 1, KP) - (1.0 + ep) * c, 0.0)
				            / (fabs(SO(i, j, k - 1, KP) - (1.0 + ep) * c) + emach);
				CI(ic, jc, kc, LXZA) = a / c;
				CI(ic, jc, kc, LXZB) = b / c;
			}
		}
	}
	/* CF k-planes on fine-only x- and y-lines (xy faces) */
	k = 0;
	for (int kc = 2; kc <= kkc1; ++kc) {
		k += 2;
		j = 2;
		for (int jc = 3; jc <= jjcf1; ++jc) {
			j += 2;
			i = 2;
			for (int ic = 3; ic <= iicf1; ++ic) {
				i += 2;
				dnw = SO(i - 1, j, k, KPNW) + SO(i - 1, j, k, KBNW) + SO(i - 1, j, k + 1, KBSE);
				dn = SO(i - 1, j, k, KPS) + SO(i - 1, j, k, KBN) + SO(i - 1, j, k + 1, KBS);
				dne = SO(i, j, k, KPSW) + SO(i, j, k, KBNE) + SO(i, j, k + 1, KBSW);
				dw = SO(i - 1, j - 1, k, KPW) + SO(i - 1, j - 1, k, KBW) + SO(i - 1, j - 1, k + 1, KBE);
				de = SO(i, j - 1, k, KPW) + SO(i, j - 1, k, KBE) + SO(i, j - 1, k + 1, KBW);
				dsw = SO(i - 1, j - 1, k, KPSW) + SO(i - 1, j - 1, k, KBSW) + SO(i - 1, j - 1, k + 1, KBNE);
				ds = SO(i - 1, j - 1, k, KPS) + SO(i - 1, j - 1, k, KBS) + SO(i - 1, j - 1, k + 1, KBN);
				dse = SO(i, j - 1, k, KPNW) + SO(i, j - 1, k, KBSE) + SO(i, j - 1, k + 1, KBNW);
				double o = SO(i - 1, j - 1, k, KP);
				ep = dmin2(dmin2(dmin2(fabs((dsw + dw + dnw) / o), fabs((dnw + dn + dne) / o)), fabs((dne + de + dse) / o)),
				           fabs((dse + ds + dsw) / o));
				dp = dw + dnw + dn + dne + de + dse + ds + dsw;
				sum = o - SO(i - 1, j - 1, k, KB) - SO(i - 1, j - 1, k + 1, KB);
				dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
				dp = 1.0 / dp;
				CI(ic, jc, kc, LXYNW) = dp * (dnw + CI(ic - 1, jc, kc, LXYA) * dw + CI(ic, jc, kc, LXYL) * dn);
				CI(ic, jc, kc, LXYNE) = dp * (dne + CI(ic, jc, kc, LXYR) * dn + CI(ic, jc, kc, LXYA) * de);
				CI(ic, jc, kc, LXYSE) = dp * (dse + CI(ic, jc, kc, LXYB) * de + CI(ic, jc - 1, kc, LXYR) * ds);
				CI(ic, jc, kc, LXYSW) = dp * (dsw + CI(ic, jc - 1, kc, LXYL) * ds + CI(ic - 1, jc, kc, LXYB) * dw);
			}
		}
	}
	/* CF j-planes on fine-only x- and z-lines (xz faces) */
	k = 2;
	for (int kc = 3; kc <= kkcf1; ++kc) {
		k += 2;
		j = 0;
		for (int jc = 2; jc <= jjc1; ++jc) {
			j += 2;
			i = 2;
			for (int ic = 3; ic <= iicf1; ++ic) {
				i += 2;
				dnw = SO(i - 1, j + 1, k, KBSE) + SO(i - 1, j, k, KBE) + SO(i - 1, j, k, KBNE);
				dn = SO(i - 1, j + 1, k, KBS) + SO(i - 1, j, k, KB) + SO(i - 1, j, k, KBN);
				dne = SO(i, j + 1, k, KBSW) + SO(i, j, k, KBW) + SO(i, j, k, KBNW);
				dw = SO(i - 1, j + 1, k - 1, KPNW) + SO(i - 1, j, k - 1, KPW) + SO(i - 1, j, k - 1, KPSW);
				de = SO(i, j + 1, k - 1, KPSW) + SO(i, j, k - 1, KPW) + SO(i, j, k - 1, KPNW);
				dsw = SO(i - 1, j + 1, k - 1, KBNW) + SO(i - 1, j, k - 1, KBW) + SO(i - 1, j, k - 1, KBSW);
				ds = SO(i - 1, j + 1, k - 1, KBN) + SO(i - 1, j, k - 1, KB) + SO(i - 1, j, k - 1, KBS);
				dse = SO(i, j + 1, k - 1, KBNE) + SO(i, j, k - 1, KBE) + SO(i, j, k - 1, KBSE);
				double o = SO(i - 1, j, k - 1, KP);
				ep = dmin2(dmin2(dmin2(fabs((dsw + dw + dnw) / o), fabs((dnw + dn + dne) / o)), fabs((dne + de + dse) / o)),
				           fabs((dse + ds + dsw) / o));
				dp = dw + dnw + dn + dne + de + dse + ds + dsw;
				sum = o - SO(i - 1, j + 1, k - 1, KPS) - SO(i - 1, j, k - 1, KPS);
				dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
				dp = 1.0 / dp;
				CI(ic, jc, kc, LXZNW) = dp * (dnw + CI(ic - 1, jc, kc, LXZA) * dw + CI(ic, jc, kc, LXYL) * dn);
				CI(ic, jc, kc, LXZNE) = dp * (dne + CI(ic, jc, kc, LXYR) * dn + CI(ic, jc, kc, LXZA) * de);
				CI(ic, jc, kc, LXZSE) = dp * (dse + CI(ic, jc, kc, LXZB) * de + CI(ic, jc, kc - 1, LXYR) * ds);
				CI(ic, jc, kc, LXZSW) = dp * (dsw + CI(ic, jc, kc - 1, LXYL) * ds + CI(ic - 1, jc, kc, LXZB) * dw);
			}
		}
	}
	/* CF i-planes on fine-only y- and z-lines (yz faces) */
	k = 2;
	for (int kc = 3; kc <= kkcf1; ++kc) {
		k += 2;
		j = 2;
		for (int jc = 3; jc <= jjcf1; ++jc) {
			j += 2;
			i = 0;
			for (int ic = 2; ic <= iic1; ++ic) {
				i += 2;
				dnw = SO(i, j, k, KBSE) + SO(i, j, k, KBS) + SO(i + 1, j, k, KBSW);
				dn = SO(i, j - 1, k, KBE) + SO(i, j - 1, k, KB) + SO(i + 1, j - 1, k, KBW);
				dne = SO(i, j - 1, k, KBNE) + SO(i, j - 1, k, KBN) + SO(i + 1, j - 1, k, KBNW);
				dw = SO(i, j, k - 1, KPNW) + SO(i, j, k - 1, KPS) + SO(i + 1, j, k - 1, KPSW);
				de = SO(i, j - 1, k - 1, KPSW) + SO(i, j - 1, k - 1, KPS) + SO(i + 1, j - 1, k - 1, KPNW);
				dsw = SO(i, j, k - 1, KBNW) + SO(i, j, k - 1, KBN) + SO(i + 1, j, k - 1, KBNE);
				ds = SO(i, j - 1, k - 1, KBW) + SO(i, j - 1, k - 1, KB) + SO(i + 1, j - 1, k - 1, KBE);
				dse = SO(i, j - 1, k - 1, KBSW) + SO(i, j - 1, k - 1, KBS) + SO(i + 1, j - 1, k - 1, KBSE);
				double o = SO(i, j - 1, k - 1, KP);
				ep = dmin2(dmin2(dmin2(fabs((dsw + dw + dnw) / o), fabs((dnw + dn + dne) / o)), fabs((dne + de + dse) / o)),
				           fabs((dse + ds + dsw) / o));
				dp = dw + dnw + dn + dne + de + dse + ds + dsw;
				sum = o - SO(i, j - 1, k - 1, KPW) - SO(i + 1, j - 1, k - 1, KPW);
				dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
				dp = 1.0 / dp;
				CI(ic, jc, kc, LYZNW) = dp * (dnw + CI(ic, jc, kc, LXZA) * dw + CI(ic, jc, kc, LXYA) * dn);
				CI(ic, jc, kc, LYZNE) = dp * (dne + CI(ic, jc, kc, LXYB) * dn + CI(ic, jc - 1, kc, LXZA) * de);
				CI(ic, jc, kc, LYZSE) = dp * (dse + CI(ic, jc - 1, kc, LXZB) * de + CI(ic, jc, kc - 1, LXYB) * ds);
				CI(ic, jc, kc, LYZSW) = dp * (dsw + CI(ic, jc, kc - 1, LXYA) * ds + CI(ic, jc, kc, LXZB) * dw);
			}
		}
	}
	/* fine points on fine-only x-, y- and z-lines (interior) */
	k = 2;
	for (int kc = 3; kc <= kkcf1; ++kc) {
		k += 2;
		j = 2;
		for (int jc = 3; jc <= jjcf1; ++jc) {
			j += 2;
			i = 2;
			for (int ic = 3; ic <= iicf1; ++ic) {
				i += 2;
				double yp = SO(i - 1, j - 1, k - 1, KPW) + SO(i - 1, j, k - 1, KPNW) + SO(i - 1, j, k - 1, KPS)
				            + SO(i, j, k - 1, KPSW) + SO(i, j - 1, k - 1, KPW) + SO(i, j - 1, k - 1, KPNW)
				            + SO(i - 1, j - 1, k - 1, KPS) + SO(i - 1, j - 1, k - 1, KPSW) + SO(i - 1, j - 1, k - 1, KB)
				            + SO(i - 1, j - 1, k - 1, KBW) + SO(i - 1, j, k - 1, KBNW) + SO(i - 1, j, k - 1, KBN)
				            + SO(i, j, k - 1, KBNE) + SO(i, j - 1, k - 1, KBE) + SO(i, j - 1, k - 1, KBSE)
				            + SO(i - 1, j - 1, k - 1, KBS) + SO(i - 1, j - 1, k - 1, KBSW) + SO(i - 1, j - 1, k, KB)
				            + SO(i - 1, j - 1, k, KBE) + SO(i - 1, j, k, KBSE) + SO(i - 1, j, k, KBS) + SO(i, j, k, KBSW)
				            + SO(i, j - 1, k, KBW) + SO(i, j - 1, k, KBNW) + SO(i - 1, j - 1, k, KBN) + SO(i - 1, j - 1, k, KBNE);
				double o = SO(i - 1, j - 1, k - 1, KP);
				double m1 = fabs(SO(i - 1, j - 1, k - 1, KPW) + SO(i - 1, j, k - 1, KPNW) + SO(i - 1, j, k, KBSE)
				                 + SO(i - 1, j - 1, k, KBE) + SO(i - 1, j - 1, k, KBNE) + SO(i - 1, j - 1, k - 1, KPSW)
				                 + SO(i - 1, j - 1, k - 1, KBSW) + SO(i - 1, j - 1, k - 1, KBW) + SO(i - 1, j, k - 1, KBNW))
				            / o;
				double m2 = fabs(SO(i, j - 1, k - 1, KPW) + SO(i, j, k - 1, KPSW) + SO(i, j, k, KBSW) + SO(i, j - 1, k, KBW)
				                 + SO(i, j - 1, k, KBNW) + SO(i, j - 1, k - 1, KPNW) + SO(i, j - 1, k - 1, KBSE)
				                 + SO(i, j - 1, k - 1, KBE) + SO(i, j, k - 1, KBNE))
				            / o;
				double m3 = fabs(SO(i - 1, j, k - 1, KPS) + SO(i - 1, j, k - 1, KPNW) + SO(i - 1, j, k, KBSE) + SO(i - 1, j, k, KBS)
				                 + SO(i, j, k, KBSW) + SO(i, j, k - 1, KPSW) + SO(i, j, k - 1, KBNE) + SO(i - 1, j, k - 1, KBN)
				                 + SO(i - 1, j, k - 1, KBNW));
				double m4 = fabs(SO(i - 1, j - 1, k - 1, KPS) + SO(i - 1, j - 1, k - 1, KPSW) + SO(i - 1, j - 1, k, KBNE)
				                 + SO(i - 1, j - 1, k, KBN) + SO(i, j - 1, k, KBNW) + SO(i, j - 1, k - 1, KPNW)
				                 + SO(i, j - 1, k - 1, KBSE) + SO(i - 1, j - 1, k - 1, KBS) + SO(i, j - 1, k - 1, KBSE))
				            / o;
				/* the reference's third MIN argument is not divided by so(kp) */
				double ypw = dmin2(dmin2(dmin2(m1, m2), m3), m4);
				double m5 = fabs(SO(i - 1, j - 1, k - 1, KB) + SO(i - 1, j - 1, k - 1, KBW) + SO(i - 1, j, k - 1, KBNW)
				                 + SO(i - 1, j, k - 1, KBN) + SO(i, j, k - 1, KBNE) + SO(i, j - 1, k - 1, KBE)
				                 + SO(i, j - 1, k - 1, KBSE) + SO(i - 1, j - 1, k - 1, KBS) + SO(i - 1, j - 1, k - 1, KBSW));
				double m6 = fabs(SO(i - 1, j - 1, k, KB) + SO(i - 1, j - 1, k, KBE) + SO(i - 1, j, k, KBSE) + SO(i - 1, j, k, KBS)
				                 + SO(i, j, k, KBSW) + SO(i, j - 1, k, KBW) + SO(i, j - 1, k, KBNW) + SO(i - 1, j - 1, k, KBN)
				                 + SO(i - 1, j - 1, k, KBNE))
				            / o;
				/* and neither is its fifth */
				ypw = dmin2(dmin2(ypw, m5), m6);
				yp = yp + (o - yp) * fmax(o - (1.0 + ypw) * yp, 0.0) / (fabs(o - (1.0 + ypw) * yp) + emach);
				yp = 1.0 / yp;
				CI(ic, jc, kc, LTNW) = yp * (SO(i - 1, j, k, KBSE) + CI(ic - 1, jc, kc, LYZNW) * SO(i - 1, j - 1, k - 1, KPW)
				                             + CI(ic - 1, jc, kc, LXZA) * SO(i - 1, j, k - 1, KPNW) + CI(ic, jc, kc, LXZNW) * SO(i - 1, j, k - 1, KPS)
				                             + CI(ic - 1, jc, kc, LXYA) * SO(i - 1, j - 1, k, KBE) + CI(ic, jc, kc, LXYL) * SO(i - 1, j, k, KBS)
				                             + CI(ic, jc, kc, LXYNW) * SO(i - 1, j - 1, k, KB));
				CI(ic, jc, kc, LTNE) = yp * (SO(i, j, k, KBSW) + CI(ic, jc, kc, LXZNE) * SO(i - 1, j, k - 1, KPS)
				                             + CI(ic, jc, kc, LXZA) * SO(i, j, k - 1, KPSW) + CI(ic, jc, kc, LYZNW) * SO(i, j - 1, k - 1, KPW)
				                             + CI(ic, jc, kc, LXYR) * SO(i - 1, j, k, KBS) + CI(ic, jc, kc, LXYA) * SO(i, j - 1, k, KBW)
				                             + CI(ic, jc, kc, LXYNE) * SO(i - 1, j - 1, k, KB));
				CI(ic, jc, kc, LBNW) = yp * (SO(i - 1, j, k - 1, KBNW) + CI(ic - 1, jc, kc - 1, LXYA) * SO(i - 1, j - 1, k - 1, KBW)
				                             + CI(ic, jc, kc - 1, LXYL) * SO(i - 1, j, k - 1, KBN) + CI(ic, jc, kc - 1, LXYNW) * SO(i - 1, j - 1, k - 1, KB)
				                             + CI(ic - 1, jc, kc, LYZSW) * SO(i - 1, j - 1, k - 1, KPW) + CI(ic - 1, jc, kc, LXZB) * SO(i - 1, j, k - 1, KPNW)
				                             + CI(ic, jc, kc, LXZSW) * SO(i - 1, j, k - 1, KPS));
				CI(ic, jc, kc, LBNE) = yp * (SO(i, j, k - 1, KBNE) + CI(ic, jc, kc - 1, LXYNE) * SO(i - 1, j - 1, k - 1, KB)
				                             + CI(ic, jc, kc - 1, LXYR) * SO(i - 1, j, k - 1, KBN) + CI(ic, jc, kc - 1, LXYA) * SO(i, j - 1, k - 1, KBE)
				                             + CI(ic, jc, kc, LXZSE) * SO(i - 1, j, k - 1, KPS) + CI(ic, jc, kc, LXZB) * SO(i, j, k - 1, KPSW)
				                             + CI(ic, jc, kc, LYZSW) * SO(i, j - 1, k - 1, KPW));
				CI(ic, jc, kc, LBSW) = yp * (SO(i - 1, j - 1, k - 1, KBSW) + CI(ic - 1, jc, kc - 1, LXYB) * SO(i - 1, j - 1, k - 1, KBW)
				                             + CI(ic, jc, kc - 1, LXYSW) * SO(i - 1, j - 1, k - 1, KB) + CI(ic, jc - 1, kc - 1, LXYL) * SO(i - 1, j - 1, k - 1, KBS)
				                             + CI(ic - 1, jc, kc, LYZSE) * SO(i - 1, j - 1, k - 1, KPW) + CI(ic, jc - 1, kc, LXZSW) * SO(i - 1, j - 1, k - 1, KPS)
				                             + CI(ic - 1, jc - 1, kc, LXZB) * SO(i - 1, j - 1, k - 1, KPSW));
				CI(ic, jc, kc, LTSW) = yp * (SO(i - 1, j - 1, k, KBNE) + CI(ic - 1, jc, kc, LXYB) * SO(i - 1, j - 1, k, KBE)
				                             + CI(ic, jc, kc, LXYSW) * SO(i - 1, j - 1, k, KB) + CI(ic, jc - 1, kc, LXYL) * SO(i - 1, j - 1, k, KBN)
				                             + CI(ic - 1, jc, kc, LYZNE) * SO(i - 1, j - 1, k - 1, KPW) + CI(ic, jc - 1, kc, LXZNW) * SO(i - 1, j - 1, k - 1, KPS)
				                             + CI(ic - 1, jc - 1, kc, LXZA) * SO(i - 1, j - 1, k - 1, KPSW));
				CI(ic, jc, kc, LTSE) = yp * (SO(i, j - 1, k, KBNW) + CI(ic, jc - 1, kc, LXYR) * SO(i - 1, j - 1, k, KBN)
				                             + CI(ic, jc, kc, LXYSE) * SO(i - 1, j - 1, k, KB) + CI(ic, jc, kc, LXYB) * SO(i, j - 1, k, KBW)
				                             + CI(ic, jc - 1, kc, LXZNE) * SO(i - 1, j - 1, k - 1, KPS) + CI(ic, jc, kc, LYZNE) * SO(i, j - 1, k - 1, KPW)
				                             + CI(ic, jc - 1, kc, LXZA) * SO(i, j - 1, k - 1, KPNW));
				CI(ic, jc, kc, LBSE) = yp * (SO(i, j - 1, k - 1, KBSE) + CI(ic, jc - 1, kc - 1, LXYR) * SO(i - 1, j - 1, k - 1, KBS)
				                             + CI(ic, jc, kc - 1, LXYSE) * SO(i - 1, j - 1, k - 1, KB) + CI(ic, jc, kc - 1, LXYB) * SO(i, j - 1, k - 1, KBE)
				                             + CI(ic, jc - 1, kc, LXZSE) * SO(i - 1, j - 1, k - 1, KPS) + CI(ic, jc, kc, LYZSE) * SO(i, j - 1, k - 1, KPW)
				                             + CI(ic, jc - 1, kc, LXZB) * SO(i, j - 1, k - 1, KPNW));
			}
		}
	}
#undef CI
}

/* ------------------------------------------------ 7-point fine operators */
/* BMG3_SymStd_residual.f90:104-119 (seven-point branch; planes p, pw, ps, b) */
void o3_residual7(const double *so, const double *qf, const double *q, double *res, int II, int JJ, int KK)
{
#define Q(i, j, k) q[ix3(i, j, k, II, JJ)]
	for (int k = 2; k <= KK - 1; ++k)
		for (int j = 2; j <= JJ - 1; ++j)
			for (int i = 2; i <= II - 1; ++i)
				res[ix3(i, j, k, II, JJ)] = qf[ix3(i, j, k, II, JJ)] + SO(i, j, k, KPW) * Q(i - 1, j, k)
				                            + SO(i, j + 1, k, KPS) * Q(i, j + 1, k) + SO(i + 1, j, k, KPW) * Q(i + 1, j, k)
				                            + SO(i, j, k, KPS) * Q(i, j - 1, k) + SO(i, j, k, KB) * Q(i, j, k - 1)
				                            + SO(i, j, k + 1, KB) * Q(i, j, k + 1) - SO(i, j, k, KP) * Q(i, j, k);
}

/* BMG3_SymStd_relax_GS.f90:141-180 (seven-point): two colours, a point of colour
 * pts has i+j+k+pts even; UP (and the non-symmetric sweep) runs 0 then 1, DOWN 1 then 0 */
void o3_relax_gs7(const double *so, const double *qf, double *q, const double *sor, int II, int JJ, int KK, int updown)
{
	const int p0 = updown == 1 ? 0 : 1, p1 = updown == 1 ? 1 : 0, pst = updown == 1 ? 1 : -1;
	for (int pts = p0; pst > 0 ? pts <= p1 : pts >= p1; pts += pst)
		for (int k = 2; k <= KK - 1; ++k)
			for (int j = 2; j <= JJ - 1; ++j) {
				const int ibeg = (j + k + pts) % 2 + 2;
				for (int i = ibeg; i <= II - 1; i += 2)
					Q(i, j, k) = (qf[ix3(i, j, k, II, JJ)] + SO(i, j, k, KPW) * Q(i - 1, j, k)
					              + SO(i, j + 1, k, KPS) * Q(i, j + 1, k) + SO(i + 1, j, k, KPW) * Q(i + 1, j, k)
					              + SO(i, j, k, KPS) * Q(i, j - 1, k) + SO(i, j, k, KB) * Q(i, j, k - 1)
					              + SO(i, j, k + 1, KB) * Q(i, j, k + 1))
					             * sor[ix3(i, j, k, II, JJ)];
			}
#undef Q
}

/* BMG3_SymStd_SETUP_interp_OI.f90:543-807, the seven-point branch (used when the
 * fine level is the finest and its operator seven-point).  Quirk kept: the
 * x-edge ep takes abs(b)/so(kp) rather than abs(b/so(kp)). */
void o3_setup_interp7(const double *so, double *ci, int iif, int jjf, int kkf, int iic, int jjc, int kkc)
{
	const int II = iif, JJ = jjf, KK = kkf;
#define CI(i, j, k, l) ci[ix4(i, j, k, l, iic, jjc, kkc)]
	const double emach = ldexp(1.0, -53);
	const int iic1 = iic - 1, jjc1 = jjc - 1, kkc1 = kkc - 1;
	const int iicf1 = (iif - 2) / 2 + 2, jjcf1 = (jjf - 2) / 2 + 2, kkcf1 = (kkf - 2) / 2 + 2;
	double a, b, c, ep, dn, dw, de, ds, dp, sum;
	for (int kc = 2; kc <= kkc1; ++kc)
		for (int jc = 2; jc <= jjc1; ++jc)
			for (int ic = 3; ic <= iicf1; ++ic) {
				const int i = 2 * ic - 2, j = 2 * jc - 2, k = 2 * kc - 2;
				a = SO(i - 1, j, k, KPW);
				b = SO(i, j, k, KPW);
				ep = dmin2(fabs(a / SO(i - 1, j, k, KP)), fabs(b) / SO(i - 1, j, k, KP));
				c = a + b + SO(i - 1, j, k, KPS) + SO(i - 1, j + 1, k, KPS) + SO(i - 1, j, k, KB) + SO(i - 1, j, k + 1, KB);
				c = a + b + (SO(i - 1, j, k, KP) - c) * fmax(SO(i - 1, j, k, KP) - (1.0 + ep) * c, 0.0)
				            / (fabs(SO(i - 1, j, k, KP) - (1.0 + ep) * c) + emach);
				CI(ic, jc, kc, LXYL) = a / c;
				CI(ic, jc, kc, LXYR) = b / c;
			}
	for (int kc = 2; kc <= kkc1; ++kc)
		for (int jc = 3; jc <= jjcf1; ++jc)
			for (int ic = 2; ic <= iic1; ++ic) {
				const int i = 2 * ic - 2, j = 2 * jc - 2, k = 2 * kc - 2;
				a = SO(i, j, k, KPS);
				b = SO(i, j - 1, k, KPS);
				c = a + b + SO(i, j - 1, k, KPW) + SO(i + 1, j - 1, k, KPW) + SO(i, j - 1, k, KB) + SO(i, j - 1, k + 1, KB);
				ep = dmin2(fabs(a / SO(i, j - 1, k, KP)), fabs(b / SO(i, j - 1, k, KP)));
				c = a + b + (SO(i, j - 1, k, KP) - c) * fmax(SO(i, j - 1, k, KP) - (1.0 + ep) * c, 0.0)
				            / (fabs(SO(i, j - 1, k, KP) - (1.0 + ep) * c) + emach);
				CI(ic, jc, kc, LXYA) = a / c;
				CI(ic, jc, kc, LXYB) = b / c;
			}
	for (int kc = 3; kc <= kkcf1; ++kc)
		for (int jc = 2; jc <= jjc1; ++jc)
			for (int ic = 2; ic <= iic1; ++ic) {
				const int i = 2 * ic - 2, j = 2 * jc - 2, k = 2 * kc - 2;
				a = SO(i, j, k, KB);
				b = SO(i, j, k - 1, KB);
				c = a + b + SO(i, j, k - 1, KPW) + SO(i + 1, j, k - 1, KPW) + SO(i, j + 1, k - 1, KPS) + SO(i, j, k - 1, KPS);
				ep = dmin2(fabs(a / SO(i, j, k - 1, KP)), fabs(b / SO(i, j, k - 1, KP)));
				c = a + b + (SO(i, j, k - 1, KP) - c) * fmax(SO(i, j, k - 1, KP) - (1.0 + ep) * c, 0.0)
				            / (fabs(SO(i, j, k - 1, KP) - (1.0 + ep) * c) + emach);
				CI(ic, jc, kc, LXZA) = a / c;
				CI(ic, jc, kc, LXZB) = b / c;
			}
	/* xy faces */
	for (int ic = 3; ic <= iicf1; ++ic)
		for (int jc = 3; jc <= jjcf1; ++jc)
			for (int kc = 2; kc <= kkc1; ++kc) {
				const int i = 2 * ic - 2, j = 2 * jc - 2, k = 2 * kc - 2;
				const double o = SO(i - 1, j - 1, k, KP);
				dn = SO(i - 1, j, k, KPS);
				dw = SO(i - 1, j - 1, k, KPW);
				de = SO(i, j - 1, k, KPW);
				ds = SO(i - 1, j - 1, k, KPS);
				dp = dw + dn + de + ds;
				sum = o - SO(i - 1, j - 1, k, KB) - SO(i - 1, j - 1, k + 1, KB);
				ep = dmin2(dmin2(dmin2(fabs(dw / o), fabs(dn / o)), fabs(de / o)), fabs(ds / o));
				dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
				dp = 1.0 / dp;
				CI(ic, jc, kc, LXYNW) = dp * (CI(ic - 1, jc, kc, LXYA) * dw + CI(ic, jc, kc, LXYL) * dn);
				CI(ic, jc, kc, LXYNE) = dp * (CI(ic, jc, kc, LXYR) * dn + CI(ic, jc, kc, LXYA) * de);
				CI(ic, jc, kc, LXYSE) = dp * (CI(ic, jc, kc, LXYB) * de + CI(ic, jc - 1, kc, LXYR) * ds);
				CI(ic, jc, kc, LXYSW) = dp * (CI(ic, jc - 1, kc, LXYL) * ds + CI(ic - 1, jc, kc, LXYB) * dw);
			}
	/* xz faces */
	for (int kc = 3; kc <= kkcf1; ++kc)
		for (int jc = 2; jc <= jjc1; ++jc)
			for (int ic = 3; ic <= iicf1; ++ic) {
				const int i = 2 * ic - 2, j = 2 * jc - 2, k = 2 * kc - 2;
				const double o = SO(i - 1, j, k - 1, KP);
				dn = SO(i - 1, j, k, KB);
				dw = SO(i - 1, j, k - 1, KPW);
				de = SO(i, j, k - 1, KPW);
				ds = SO(i - 1, j, k - 1, KB);
				dp = dw + dn + de + ds;
				sum = o - SO(i - 1, j + 1, k - 1, KPS) - SO(i - 1, j, k - 1, KPS);
				ep = dmin2(dmin2(dmin2(fabs(dw / o), fabs(dn / o)), fabs(de / o)), fabs(ds / o));
				dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
				dp = 1.0 / dp;
				CI(ic, jc, kc, LXZNW) = dp * (CI(ic - 1, jc, kc, LXZA) * dw + CI(ic, jc, kc, LXYL) * dn);
				CI(ic, jc, kc, LXZNE) = dp * (CI(ic, jc, kc, LXYR) * dn + CI(ic, jc, kc, LXZA) * de);
				CI(ic, jc, kc, LXZSE) = dp * (CI(ic, jc, kc, LXZB) * de + CI(ic, jc, kc - 1, LXYR) * ds);
				CI(ic, jc, kc, LXZSW) = dp * (CI(ic, jc, kc - 1, LXYL) * ds + CI(ic - 1, jc, kc, LXZB) * dw);
			}
	/* yz faces */
	for (int kc = 3; kc <= kkcf1; ++kc)
		for (int jc = 3; jc <= jjcf1; ++jc)
			for (int ic = 2; ic <= iic1; ++ic) {
				const int i = 2 * ic - 2, j = 2 * jc - 2, k = 2 * kc - 2;
				const double o = SO(i, j - 1, k - 1, KP);
				dn = SO(i, j - 1, k, KB);
				dw = SO(i, j, k - 1, KPS);
				de = SO(i, j - 1, k - 1, KPS);
				ds = SO(i, j - 1, k - 1, KB);
				dp = dw + dn + de + ds;
				sum = o - SO(i, j - 1, k - 1, KPW) - SO(i + 1, j - 1, k - 1, KPW);
				ep = dmin2(dmin2(dmin2(fabs(dw / o), fabs(dn / o)), fabs(de / o)), fabs(ds / o));
				dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
				dp = 1.0 / dp;
				CI(ic, jc, kc, LYZNW) = dp * (CI(ic, jc, kc, LXZA) * dw + CI(ic, jc, kc, LXYA) * dn);
				CI(ic, jc, kc, LYZNE) = dp * (CI(ic, jc, kc, LXYB) * dn + CI(ic, jc - 1, kc, LXZA) * de);
				CI(ic, jc, kc, LYZSE) = dp * (CI(ic, jc - 1, kc, LXZB) * de + CI(ic, jc, kc - 1, LXYB) * ds);
				CI(ic, jc, kc, LYZSW) = dp * (CI(ic, jc, kc - 1, LXYA) * ds + CI(ic, jc, kc, LXZB) * dw);
			}
	/* interior points */
	for (int kc = 3; kc <= kkcf1; ++kc)
		for (int jc = 3; jc <= jjcf1; ++jc)
			for (int ic = 3; ic <= iicf1; ++ic) {
				const int i = 2 * ic - 2, j = 2 * jc - 2, k = 2 * kc - 2;
				const double o = SO(i - 1, j - 1, k - 1, KP);
				dp = SO(i - 1, j - 1, k - 1, KPW) + SO(i - 1, j, k - 1, KPS) + SO(i, j - 1, k - 1, KPW)
				     + SO(i - 1, j - 1, k - 1, KPS) + SO(i - 1, j - 1, k - 1, KB) + SO(i - 1, j - 1, k, KB);
				ep = dmin2(dmin2(dmin2(dmin2(dmin2(fabs(SO(i - 1, j - 1, k - 1, KPW) / o), fabs(SO(i - 1, j, k - 1, KPS) / o)),
				                             fabs(SO(i, j - 1, k - 1, KPW) / o)),
				                       fabs(SO(i - 1, j - 1, k - 1, KPS) / o)),
				                 fabs(SO(i - 1, j - 1, k - 1, KB) / o)),
				           fabs(SO(i - 1, j - 1, k, KB) / o));
				dp = (o - dp) * fmax(o - (1.0 + ep) * dp, 0.0) / (fabs(o - (1.0 + ep) * dp) + emach) + dp;
				dp = 1.0 / dp;
				CI(ic, jc, kc, LTNW) = dp * (CI(ic - 1, jc, kc, LYZNW) * SO(i - 1, j - 1, k - 1, KPW)
				                             + CI(ic, jc, kc, LXZNW) * SO(i - 1, j, k - 1, KPS)
				                             + CI(ic, jc, kc, LXYNW) * SO(i - 1, j - 1, k, KB));
				CI(ic, jc, kc, LTNE) = dp * (CI(ic, jc, kc, LXZNE) * SO(i - 1, j, k - 1, KPS)
				                             + CI(ic, jc, kc, LYZNW) * SO(i, j - 1, k - 1, KPW)
				                             + CI(ic, jc, kc, LXYNE) * SO(i - 1, j - 1, k, KB));
				CI(ic, jc, kc, LBNW) = dp * (CI(ic, jc, kc - 1, LXYNW) * SO(i - 1, j - 1, k - 1, KB)
				                             + CI(ic - 1, jc, kc, LYZSW) * SO(i - 1, j - 1, k - 1, KPW)
				                             + CI(ic, jc, kc, LXZSW) * SO(i - 1, j, k - 1, KPS));
				CI(ic, jc, kc, LBNE) = dp * (CI(ic, jc, kc - 1, LXYNE) * SO(i - 1, j - 1, k - 1, KB)
				                             + CI(ic, jc, kc, LXZSE) * SO(i - 1, j, k - 1, KPS)
				                             + CI(ic, jc, kc, LYZSW) * SO(i, j - 1, k - 1, KPW));
				CI(ic, jc, kc, LBSW) = dp * (CI(ic, jc, kc - 1, LXYSW) * SO(i - 1, j - 1, k - 1, KB)
				                             + CI(ic - 1, jc, kc, LYZSE) * SO(i - 1, j - 1, k - 1, KPW)
				                             + CI(ic, jc - 1, kc, LXZSW) * SO(i - 1, j - 1, k - 1, KPS));
				CI(ic, jc, kc, LTSW) = dp * (CI(ic, jc, kc, LXYSW) * SO(i - 1, j - 1, k, KB)
				                             + CI(ic - 1, jc, kc, LYZNE) * SO(i - 1, j - 1, k - 1, KPW)
				                             + CI(ic, jc - 1, kc, LXZNW) * SO(i - 1, j - 1, k - 1, KPS));
				CI(ic, jc, kc, LTSE) = dp * (CI(ic, jc, kc, LXYSE) * SO(i - 1, j - 1, k, KB)
				                             + CI(ic, jc - 1, kc, LXZNE) * SO(i - 1, j - 1, k - 1, KPS)
				                             + CI(ic, jc, kc, LYZNE) * SO(i, j - 1, k - 1, KPW));
				CI(ic, jc, kc, LBSE) = dp * (CI(ic, jc, kc - 1, LXYSE) * SO(i - 1, j - 1, k - 1, KB)
				                             + CI(ic, jc - 1, kc, LXZSE) * SO(i - 1, j - 1, k - 1, KPS)
				                             + CI(ic, jc, kc, LYZSE) * SO(i, j - 1, k - 1, KPW));
			}
#undef CI
}

/* ---------------------------------------------------------------- Galerkin */
/* A[(i,j,k), (i,j,k)+(di,dj,dk)] from the lower-half 14-plane storage (the
 * coefficient that multiplies that neighbour in BMG3_SymStd_residual.f90:76-101,
 * negated). */
static double a3(const double *so, int II, int JJ, int KK, int i, int j, int k, int di, int dj, int dk)
{
	if (di == 0 && dj == 0 && dk == 0) return SO(i, j, k, KP);
	double c = 0.0;
	switch ((dk + 1) * 9 + (dj + 1) * 3 + (di + 1)) {
	/* dk = 0 */
	case 9 + 3 + 0: c = SO(i, j, k, KPW); break;              /* (-1, 0, 0) */
	case 9 + 6 + 0: c = SO(i, j + 1, k, KPNW); break;         /* (-1,+1, 0) */
	case 9 + 6 + 1: c = SO(i, j + 1, k, KPS); break;          /* ( 0,+1, 0) */
	case 9 + 6 + 2: c = SO(i + 1, j + 1, k, KPSW); break;     /* (+1,+1, 0) */
	case 9 + 3 + 2: c = SO(i + 1, j, k, KPW); break;          /* (+1, 0, 0) */
	case 9 + 0 + 2: c = SO(i + 1, j, k, KPNW); break;         /* (+1,-1, 0) */
	case 9 + 0 + 1: c = SO(i, j, k, KPS); break;              /* ( 0,-1, 0) */
	case 9 + 0 + 0: c = SO(i, j, k, KPSW); break;             /* (-1,-1, 0) */
	/* dk = -1 */
	case 0 + 3 + 1: c = SO(i, j, k, KB); break;
	case 0 + 3 + 0: c = SO(i, j, k, KBW); break;
	case 0 + 6 + 0: c = SO(i, j + 1, k, KBNW); break;
	case 0 + 6 + 1: c = SO(i, j + 1, k, KBN); break;
	case 0 + 6 + 2: c = SO(i + 1, j + 1, k, KBNE); break;
	case 0 + 3 + 2: c = SO(i + 1, j, k, KBE); break;
	case 0 + 0 + 2: c = SO(i + 1, j, k, KBSE); break;
	case 0 + 0 + 1: c = SO(i, j, k, KBS); break;
	case 0 + 0 + 0: c = SO(i, j, k, KBSW); break;
	/* dk = +1 */
	case 18 + 3 + 1: c = SO(i, j, k + 1, KB); break;
	case 18 + 3 + 0: c = SO(i, j, k + 1, KBE); break;
	case 18 + 6 + 0: c = SO(i, j + 1, k + 1, KBSE); break;
	case 18 + 6 + 1: c = SO(i, j + 1, k + 1, KBS); break;
	case 18 + 6 + 2: c = SO(i + 1, j + 1, k + 1, KBSW); break;
	case 18 + 3 + 2: c = SO(i + 1, j, k + 1, KBW); break;
	case 18 + 0 + 2: c = SO(i + 1, j, k + 1, KBNW); break;
	case 18 + 0 + 1: c = SO(i, j, k + 1, KBN); break;
	case 18 + 0 + 0: c = SO(i, j, k + 1, KBNE); break;
	}
	return -c;
}

/* weight of coarse point (ic,jc,kc) at fine point F + (dx,dy,dz), F its fine
 * position, as BMG3_SymStd_interp_add applies it (interp_add.f90:108-239) */
static double p3(const double *ci, int iic, int jjc, int kkc, int ic, int jc, int kc, int dx, int dy, int dz)
{
#define CI(i, j, k, l) ci[ix4(i, j, k, l, iic, jjc, kkc)]
	if (dz == 0) {
		if (dx == 0 && dy == 0) return 1.0;
		if (dy == 0) return dx < 0 ? CI(ic, jc, kc, LXYR) : CI(ic + 1, jc, kc, LXYL);
		if (dx == 0) return dy < 0 ? CI(ic, jc, kc, LXYA) : CI(ic, jc + 1, kc, LXYB);
		if (dy < 0) return dx < 0 ? CI(ic, jc, kc, LXYNE) : CI(ic + 1, jc, kc, LXYNW);
		return dx < 0 ? CI(ic, jc + 1, kc, LXYSE) : CI(ic + 1, jc + 1, kc, LXYSW);
	}
	const int ko = dz < 0 ? 0 : 1; /* owner offset in z */
	if (dx == 0 && dy == 0) return dz < 0 ? CI(ic, jc, kc, LXZA) : CI(ic, jc, kc + 1, LXZB);
	if (dx == 0) { /* yz faces */
		if (dy < 0) return dz < 0 ? CI(ic, jc, kc, LYZNW) : CI(ic, jc, kc + 1, LYZSW);
		return dz < 0 ? CI(ic, jc + 1, kc, LYZNE) : CI(ic, jc + 1, kc + 1, LYZSE);
	}
	if (dy == 0) { /* xz faces */
		if (dx < 0) return dz < 0 ? CI(ic, jc, kc, LXZNE) : CI(ic, jc, kc + 1, LXZSE);
		return dz < 0 ? CI(ic + 1, jc, kc, LXZNW) : CI(ic + 1, jc, kc + 1, LXZSW);
	}
	/* interior points */
	const int io = dx < 0 ? 0 : 1, jo = dy < 0 ? 0 : 1;
	int l;
	if (dz < 0) l = dy < 0 ? (dx < 0 ? LTNE : LTNW) : (dx < 0 ? LTSE : LTSW);
	else l = dy < 0 ? (dx < 0 ? LBNE : LBNW) : (dx < 0 ? LBSE : LBSW);
	return CI(ic + io, jc + jo, kc + ko, l);
#undef CI
}

/* sum over f1 in supp(c1), f2 in supp(c2) of P(f1,c1) A(f1,f2) P(f2,c2) */
static double rap3(const double *so, int II, int JJ, int KK, const double *ci, int iic, int jjc, int kkc, int i1, int j1,
                   int k1, int i2, int j2, int k2)
{
	const int F1x = 2 * i1 - 2, F1y = 2 * j1 - 2, F1z = 2 * k1 - 2;
	double tot = 0.0;
	for (int dz1 = -1; dz1 <= 1; ++dz1)
		for (int dy1 = -1; dy1 <= 1; ++dy1)
			for (int dx1 = -1; dx1 <= 1; ++dx1) {
				const int fx = F1x + dx1, fy = F1y + dy1, fz = F1z + dz1;
				if (fx < 2 || fx > II - 1 || fy < 2 || fy > JJ - 1 || fz < 2 || fz > KK - 1) continue;
				double inner = 0.0;
				for (int ddz = -1; ddz <= 1; ++ddz)
					for (int ddy = -1; ddy <= 1; ++ddy)
						for (int ddx = -1; ddx <= 1; ++ddx) {
							const int ex = dx1 + ddx - 2 * (i2 - i1), ey = dy1 + ddy - 2 * (j2 - j1), ez = dz1 + ddz - 2 * (k2 - k1);
							if (ex < -1 || ex > 1 || ey < -1 || ey > 1 || ez < -1 || ez > 1) continue;
							inner += a3(so, II, JJ, KK, fx, fy, fz, ddx, ddy, ddz) * p3(ci, iic, jjc, kkc, i2, j2, k2, ex, ey, ez);
						}
				tot += p3(ci, iic, jjc, kkc, i1, j1, k1, dx1, dy1, dz1) * inner;
			}
	return tot;
}

/* Galerkin coarse operator (14 planes), the product BMG3_SymStd_SETUP_ITLI27_ex expands */
void o3_galerkin(const double *so, double *soc, const double *ci, int II, int JJ, int KK, int iic, int jjc, int kkc)
{
#define SOC(i, j, k, p) soc[ix4(i, j, k, p, iic, jjc, kkc)]
	for (int kc = 2; kc <= kkc - 1; ++kc)
		for (int jc = 2; jc <= jjc - 1; ++jc)
			for (int ic = 2; ic <= iic - 1; ++ic) {
#define R(a, b, c, d, e, f) rap3(so, II, JJ, KK, ci, iic, jjc, kkc, a, b, c, d, e, f)
				SOC(ic, jc, kc, KP) = R(ic, jc, kc, ic, jc, kc);
				SOC(ic, jc, kc, KPW) = -R(ic, jc, kc, ic - 1, jc, kc);
				SOC(ic, jc, kc, KPS) = -R(ic, jc, kc, ic, jc - 1, kc);
				SOC(ic, jc, kc, KB) = -R(ic, jc, kc, ic, jc, kc - 1);
				SOC(ic, jc, kc, KPSW) = -R(ic, jc, kc, ic - 1, jc - 1, kc);
				SOC(ic, jc, kc, KPNW) = -R(ic, jc - 1, kc, ic - 1, jc, kc);
				SOC(ic, jc, kc, KBW) = -R(ic, jc, kc, ic - 1, jc, kc - 1);
				SOC(ic, jc, kc, KBNW) = -R(ic, jc - 1, kc, ic - 1, jc, kc - 1);
				SOC(ic, jc, kc, KBN) = -R(ic, jc - 1, kc, ic, jc, kc - 1);
				SOC(ic, jc, kc, KBNE) = -R(ic - 1, jc - 1, kc, ic, jc, kc - 1);
				SOC(ic, jc, kc, KBE) = -R(ic - 1, jc, kc, ic, jc, kc - 1);
				SOC(ic, jc, kc, KBSE) = -R(ic - 1, jc, kc, ic, jc - 1, kc - 1);
				SOC(ic, jc, kc, KBS) = -R(ic, jc, kc, ic, jc - 1, kc - 1);
				SOC(ic, jc, kc, KBSW) = -R(ic, jc, kc, ic - 1, jc - 1, kc - 1);
#undef R
			}
#undef SOC
}

/* BMG3_SymStd_SETUP_cg_LU, src/3d/ftn/BMG3_SymStd_SETUP_cg_LU.f90:93-193 (14 planes,
 * definite non-periodic) with DPBTRF('U', N, IBW); IBW = (II-2)*(JJ-1)+1. */
int o3_setup_cg(const double *so, int II, int JJ, int KK, double *abd, int nabd1)
{
#define ABD(r, c) abd[(size_t)((c) - 1) * nabd1 + ((r) - 1)]
	int i1 = II - 1, j1 = JJ - 1, k1 = KK - 1, i2 = i1 - 1;
	int ibw = i2 * j1 + 1;
	int kl = 0;
	for (int k = 2; k <= k1; ++k)
		for (int j = 2; j <= j1; ++j)
			for (int i = 2; i <= i1; ++i) {
				kl++;
				ABD(ibw + 1, kl) = SO(i, j, k, KP);
				ABD(ibw, kl) = -SO(i, j, k, KPW);
				ABD(ibw - i1 + 3, kl) = -SO(i + 1, j, k, KPNW);
				ABD(ibw - i1 + 2, kl) = -SO(i, j, k, KPS);
				ABD(ibw - i1 + 1, kl) = -SO(i, j, k, KPSW);
				ABD(ibw - (j1 - 2) * i2 + 2, kl) = -SO(i + 1, j + 1, k, KBNE);
				ABD(ibw - (j1 - 2) * i2 + 1, kl) = -SO(i, j + 1, k, KBN);
				ABD(ibw - (j1 - 2) * i2, kl) = -SO(i, j + 1, k, KBNW);
				ABD(ibw - (j1 - 1) * i2 + 2, kl) = -SO(i + 1, j, k, KBE);
				ABD(ibw - (j1 - 1) * i2 + 1, kl) = -SO(i, j, k, KB);
				ABD(ibw - (j1 - 1) * i2, kl) = -SO(i, j, k, KBW);
				ABD(3, kl) = -SO(i + 1, j, k, KBSE);
				ABD(2, kl) = -SO(i, j, k, KBS);
				ABD(1, kl) = -SO(i, j, k, KBSW);
			}
	return o_dpbtrf_u(kl, ibw, abd, nabd1);
#undef ABD
}
#undef SO

/* BMG3_SymStd_SOLVE_cg, src/3d/ftn/BMG3_SymStd_SOLVE_cg.f90:105-131 */
void o3_solve_cg(double *q, const double *qf, int II, int JJ, int KK, const double *abd, double *bbd, int nabd1)
{
	int kl = 0;
	for (int k = 2; k <= KK - 1; ++k)
		for (int j = 2; j <= JJ - 1; ++j)
			for (int i = 2; i <= II - 1; ++i) bbd[kl++] = qf[ix3(i, j, k, II, JJ)];
	o_dpbtrs_u(kl, (II - 2) * (JJ - 1) + 1, abd, nabd1, bbd);
	kl = 0;
	for (int k = 2; k <= KK - 1; ++k)
		for (int j = 2; j <= JJ - 1; ++j)
			for (int i = 2; i <= II - 1; ++i) q[ix3(i, j, k, II, JJ)] = bbd[kl++];
}

double o3_l2norm(const double *r, int II, int JJ, int KK)
{
	double result = 0;
	for (int k = 2; k <= KK - 1; ++k)
		for (int j = 2; j <= JJ - 1; ++j)
			for (int i = 2; i <= II - 1; ++i) result += pow(r[ix3(i, j, k, II, JJ)], 2);
	return pow(result, 1. / 2);
}

/* ------------------------------------------------------------ driver */
/* plane relaxation of one direction on one level: one 2D solver per plane
 * (planes<rdir>::setup_impl, include/cedar/3d/relax_planes.h:171-222) */
struct o3_planes {
	int n, n1, n2;          /* planes, and the plane grid */
	o2_solver **s;
	double **so2;           /* each plane's 2D operator (5 planes, kept for inspection) */
	double *x2, *b2;        /* work grid functions of the plane grid */
};
struct o3_level {
	int nx, ny, nz, ii, jj, kk;
	int ns;                 /* 14 (27-point) or 4 (7-point fine operator, stored in 14 planes) */
	double *so, *x, *b, *res, *sor, *ci;
	struct o3_planes pl[3];
};
struct o3_solver {
	o3_settings s;
	int nlev;
	struct o3_level *lv;
	double *abd, *bbd;
	int nabd1, cg_info;
};

static double *zal(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

/* ------------------------------------------------------- plane relaxation */
/* Index helpers in the reference's C++ (0-based, ghost-inclusive) indices. */
#define X3(a, i, j, k) (a)[ix3((i) + 1, (j) + 1, (k) + 1, II, JJ)]
#define S3(p, i, j, k) so[ix4((i) + 1, (j) + 1, (k) + 1, p, II, JJ, KK)]
#define X2(a, i, j) (a)[(size_t)(j) * (n1 + 2) + (i)]
#define S2(p, i, j) so2[((size_t)(p) * (n2 + 2) + (j)) * (n1 + 2) + (i)]

/* copy_coeff for xxvii_pt -> nine_pt, include/cedar/3d/relax_planes.h:110-149
 * (2D planes c, w, s, sw, nw = 0..4); ghost rows included */
static void copy_coeff(const double *so, int II, int JJ, int KK, int dir, int ipl, double *so2, int n1, int n2)
{
	if (dir == O3_XY) {
		for (int j = 0; j < n2 + 2; ++j)
			for (int i = 0; i < n1 + 2; ++i) {
				S2(0, i, j) = S3(KP, i, j, ipl);
				S2(1, i, j) = S3(KPW, i, j, ipl);
				S2(2, i, j) = S3(KPS, i, j, ipl);
				S2(3, i, j) = S3(KPSW, i, j, ipl);
				S2(4, i, j) = S3(KPNW, i, j, ipl);
			}
	} else if (dir == O3_XZ) {
		for (int k = 1; k <= n2; ++k) /* so3.range(2): interior k only */
			for (int i = 0; i < n1 + 2; ++i) {
				S2(0, i, k) = S3(KP, i, ipl, k);
				S2(1, i, k) = S3(KPW, i, ipl, k);
				S2(2, i, k) = S3(KB, i, ipl, k);
				S2(3, i, k) = S3(KBW, i, ipl, k);
				S2(4, i, k) = S3(KBE, i, ipl, k);
			}
	} else {
		for (int k = 0; k < n2 + 2; ++k)
			for (int j = 0; j < n1 + 2; ++j) {
				S2(0, j, k) = S3(KP, ipl, j, k);
				S2(1, j, k) = S3(KPS, ipl, j, k);
				S2(2, j, k) = S3(KB, ipl, j, k);
				S2(3, j, k) = S3(KBS, ipl, j, k);
				S2(4, j, k) = S3(KBN, ipl, j, k);
			}
	}
}

/* copy32 / copy23, src/3d/relax_planes.cc:185-238 (ghost-inclusive) */
static void copy32(const double *x, int II, int JJ, int dir, int ipl, double *x2, int n1, int n2)
{
	for (int b = 0; b < n2 + 2; ++b)
		for (int a = 0; a < n1 + 2; ++a)
			X2(x2, a, b) = dir == O3_XY ? X3(x, a, b, ipl) : dir == O3_XZ ? X3(x, a, ipl, b) : X3(x, ipl, a, b);
}
static void copy23(const double *x2, double *x, int II, int JJ, int dir, int ipl, int n1, int n2)
{
	for (int b = 0; b < n2 + 2; ++b)
		for (int a = 0; a < n1 + 2; ++a) {
			if (dir == O3_XY) X3(x, a, b, ipl) = X2(x2, a, b);
			else if (dir == O3_XZ) X3(x, a, ipl, b) = X2(x2, a, b);
			else X3(x, ipl, a, b) = X2(x2, a, b);
		}
}

/* copy_rhs for xxvii_pt, src/3d/relax_planes.cc:43-72 (xy), :95-127 (xz), :146-178 (yz);
 * interior of the plane only, in the reference's operand order */
static void copy_rhs(const double *so, const double *x, const double *b, int II, int JJ, int KK, int dir, int ipl,
                     double *b2, int n1, int n2)
{
	for (int q = 1; q <= n2; ++q)
		for (int p = 1; p <= n1; ++p) {
			double v;
			if (dir == O3_XY) {
				const int i = p, j = q, k = ipl;
				v = X3(b, i, j, k) + S3(KB, i, j, k) * X3(x, i, j, k - 1) + S3(KBW, i, j, k) * X3(x, i - 1, j, k - 1)
				    + S3(KBNW, i, j + 1, k) * X3(x, i - 1, j + 1, k - 1) + S3(KBN, i, j + 1, k) * X3(x, i, j + 1, k - 1)
				    + S3(KBNE, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k - 1) + S3(KBE, i + 1, j, k) * X3(x, i + 1, j, k - 1)
				    + S3(KBSE, i + 1, j, k) * X3(x, i + 1, j - 1, k - 1) + S3(KBS, i, j, k) * X3(x, i, j - 1, k - 1)
				    + S3(KBSW, i, j, k) * X3(x, i - 1, j - 1, k - 1) + S3(KBE, i, j, k + 1) * X3(x, i - 1, j, k + 1)
				    + S3(KBSE, i, j + 1, k + 1) * X3(x, i - 1, j + 1, k + 1) + S3(KBS, i, j + 1, k + 1) * X3(x, i, j + 1, k + 1)
				    + S3(KBSW, i + 1, j + 1, k + 1) * X3(x, i + 1, j + 1, k + 1) + S3(KBW, i + 1, j, k + 1) * X3(x, i + 1, j, k + 1)
				    + S3(KB, i, j, k + 1) * X3(x, i, j, k + 1) + S3(KBNW, i + 1, j, k + 1) * X3(x, i + 1, j - 1, k + 1)
				    + S3(KBN, i, j, k + 1) * X3(x, i, j - 1, k + 1) + S3(KBNE, i, j, k + 1) * X3(x, i - 1, j - 1, k + 1);
			} else if (dir == O3_XZ) {
				const int i = p, k = q, j = ipl;
				v = X3(b, i, j, k) + S3(KPNW, i, j + 1, k) * X3(x, i - 1, j + 1, k) + S3(KPS, i, j + 1, k) * X3(x, i, j + 1, k)
				    + S3(KPSW, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k) + S3(KBNW, i, j + 1, k) * X3(x, i - 1, j + 1, k - 1)
				    + S3(KBN, i, j + 1, k) * X3(x, i, j + 1, k - 1) + S3(KBNE, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k - 1)
				    + S3(KBSE, i, j + 1, k + 1) * X3(x, i - 1, j + 1, k + 1) + S3(KBS, i, j + 1, k + 1) * X3(x, i, j + 1, k + 1)
				    + S3(KBSW, i + 1, j + 1, k + 1) * X3(x, i + 1, j + 1, k + 1) + S3(KPSW, i, j, k) * X3(x, i - 1, j - 1, k)
				    + S3(KPS, i, j, k) * X3(x, i, j - 1, k) + S3(KPNW, i + 1, j, k) * X3(x, i + 1, j - 1, k)
				    + S3(KBSW, i, j, k) * X3(x, i - 1, j - 1, k - 1) + S3(KBS, i, j, k) * X3(x, i, j - 1, k - 1)
				    + S3(KBSE, i + 1, j, k) * X3(x, i + 1, j - 1, k - 1) + S3(KBNE, i, j, k + 1) * X3(x, i - 1, j - 1, k + 1)
				    + S3(KBN, i, j, k + 1) * X3(x, i, j - 1, k + 1) + S3(KBNW, i + 1, j, k + 1) * X3(x, i + 1, j - 1, k + 1);
			} else {
				const int j = p, k = q, i = ipl;
				v = X3(b, i, j, k) + S3(KPNW, i, j + 1, k) * X3(x, i - 1, j + 1, k) + S3(KPW, i, j, k) * X3(x, i - 1, j, k)
				    + S3(KPSW, i, j, k) * X3(x, i - 1, j - 1, k) + S3(KBNW, i, j + 1, k) * X3(x, i - 1, j + 1, k - 1)
				    + S3(KBW, i, j, k) * X3(x, i - 1, j, k - 1) + S3(KBSW, i, j, k) * X3(x, i - 1, j - 1, k - 1)
				    + S3(KBSE, i, j + 1, k + 1) * X3(x, i - 1, j + 1, k + 1) + S3(KBE, i, j, k + 1) * X3(x, i - 1, j, k + 1)
				    + S3(KBNE, i, j, k + 1) * X3(x, i - 1, j - 1, k + 1) + S3(KPSW, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k)
				    + S3(KPW, i + 1, j, k) * X3(x, i + 1, j, k) + S3(KPNW, i + 1, j, k) * X3(x, i + 1, j - 1, k)
				    + S3(KBNE, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k - 1) + S3(KBE, i + 1, j, k) * X3(x, i + 1, j, k - 1)
				    + S3(KBSE, i + 1, j, k) * X3(x, i + 1, j - 1, k - 1) + S3(KBSW, i + 1, j + 1, k + 1) * X3(x, i + 1, j + 1, k + 1)
				    + S3(KBW, i + 1, j, k + 1) * X3(x, i + 1, j, k + 1) + S3(KBNW, i + 1, j, k + 1) * X3(x, i + 1, j - 1, k + 1);
			}
			X2(b2, p, q) = v;
		}
}
/* copy_coeff for seven_pt -> five_pt (include/cedar/3d/relax_planes.h:73-107):
 * c, w, s from xy: p, pw, ps; xz: p, pw, b (interior k only); yz: p, ps, b */
static void copy_coeff7(const double *so, int II, int JJ, int KK, int dir, int ipl, double *so2, int n1, int n2)
{
	for (int b = 0; b < n2 + 2; ++b) {
		if (dir == O3_XZ && (b < 1 || b > n2)) continue;
		for (int a = 0; a < n1 + 2; ++a) {
			if (dir == O3_XY) {
				S2(0, a, b) = S3(KP, a, b, ipl); S2(1, a, b) = S3(KPW, a, b, ipl); S2(2, a, b) = S3(KPS, a, b, ipl);
			} else if (dir == O3_XZ) {
				S2(0, a, b) = S3(KP, a, ipl, b); S2(1, a, b) = S3(KPW, a, ipl, b); S2(2, a, b) = S3(KB, a, ipl, b);
			} else {
				S2(0, a, b) = S3(KP, ipl, a, b); S2(1, a, b) = S3(KPS, ipl, a, b); S2(2, a, b) = S3(KB, ipl, a, b);
			}
		}
	}
}

/* copy_rhs for seven_pt (src/3d/relax_planes.cc:25-38 xy, :77-90 xz, :130-143 yz) */
static void copy_rhs7(const double *so, const double *x, const double *b, int II, int JJ, int KK, int dir, int ipl,
                      double *b2, int n1, int n2)
{
	for (int q = 1; q <= n2; ++q)
		for (int p = 1; p <= n1; ++p) {
			double v;
			if (dir == O3_XY)
				v = X3(b, p, q, ipl) + S3(KB, p, q, ipl) * X3(x, p, q, ipl - 1) + S3(KB, p, q, ipl + 1) * X3(x, p, q, ipl + 1);
			else if (dir == O3_XZ)
				v = X3(b, p, ipl, q) + S3(KPS, p, ipl, q) * X3(x, p, ipl - 1, q) + S3(KPS, p, ipl + 1, q) * X3(x, p, ipl + 1, q);
			else
				v = X3(b, ipl, p, q) + S3(KPW, ipl, p, q) * X3(x, ipl - 1, p, q) + S3(KPW, ipl + 1, p, q) * X3(x, ipl + 1, p, q);
			X2(b2, p, q) = v;
		}
}
#undef X3
#undef S3
#undef X2
#undef S2

/* the plane solvers' settings: kernel_params plane_config default,
 * src/kernel_params.cc:83-89 (line-xy, max-iter 1; other keys at their defaults) */
static void plane_settings(o2_settings *s2)
{
	s2->relax = O2_RELAX_LINE_XY;
	s2->nrelax_pre = 2;
	s2->nrelax_post = 1;
	s2->num_levels = -1;
	s2->maxiter = 1;
	s2->tol = 1e-8;
	s2->min_coarse = 3;
	s2->cycle = 0;
	s2->bc = 0;
}

static void planes_setup(struct o3_level *L, int dir)
{
	struct o3_planes *P = &L->pl[dir];
	P->n = dir == O3_XY ? L->nz : dir == O3_XZ ? L->ny : L->nx;
	P->n1 = dir == O3_YZ ? L->ny : L->nx;
	P->n2 = dir == O3_XY ? L->ny : L->nz;
	const size_t g2 = (size_t)(P->n1 + 2) * (P->n2 + 2);
	P->s = (o2_solver **)calloc(P->n, sizeof(o2_solver *));
	P->so2 = (double **)calloc(P->n, sizeof(double *));
	P->x2 = (double *)calloc(g2, sizeof(double));
	P->b2 = (double *)calloc(g2, sizeof(double));
	o2_settings s2;
	plane_settings(&s2);
	const int ns2 = L->ns == 4 ? 3 : 5;  /* five_pt planes for a seven-point level */
	for (int ipl = 1; ipl <= P->n; ++ipl) {
		double *so2 = (double *)calloc(g2 * 5, sizeof(double));
		if (ns2 == 3) copy_coeff7(L->so, L->ii, L->jj, L->kk, dir, ipl, so2, P->n1, P->n2);
		else copy_coeff(L->so, L->ii, L->jj, L->kk, dir, ipl, so2, P->n1, P->n2);
		P->so2[ipl - 1] = so2;
		P->s[ipl - 1] = o2_create(&s2, so2, ns2, P->n1, P->n2);
	}
}

static void planes_free(struct o3_level *L)
{
	for (int d = 0; d < 3; ++d) {
		struct o3_planes *P = &L->pl[d];
		for (int i = 0; i < P->n && P->s; ++i) {
			o2_destroy(P->s[i]);
			free(P->so2[i]);
		}
		free(P->s); free(P->so2); free(P->x2); free(P->b2);
		memset(P, 0, sizeof(*P));
	}
}

/* relax_planes, include/cedar/3d/relax_planes.h:35-70: red-black over planes
 * (DOWN: odd planes first), each plane one 2D V-cycle (solve with max-iter 1;
 * its residual norms do not touch x) on b + off-plane couplings */
static void relax_planes_level(struct o3_level *L, int dir, double *x, const double *b, int updown)
{
	struct o3_planes *P = &L->pl[dir];
	const int beg0 = updown == 0 ? 1 : 2, beg1 = updown == 0 ? 2 : 1;
	for (int c = 0; c < 2; ++c) {
		const int beg = c == 0 ? beg0 : beg1;
		for (int ipl = beg; ipl <= P->n; ipl += 2) {
			copy32(x, L->ii, L->jj, dir, ipl, P->x2, P->n1, P->n2);
			if (L->ns == 4) copy_rhs7(L->so, x, b, L->ii, L->jj, L->kk, dir, ipl, P->b2, P->n1, P->n2);
			else copy_rhs(L->so, x, b, L->ii, L->jj, L->kk, dir, ipl, P->b2, P->n1, P->n2);
			o2_vcycle(P->s[ipl - 1], P->x2, P->b2);
			copy23(P->x2, x, L->ii, L->jj, dir, ipl, P->n1, P->n2);
		}
	}
}

/* cdr3::solver::compute_num_levels, include/cedar/3d/solver.h:59-77 */
int o3_num_levels(int nx, int ny, int nz, int min_coarse)
{
	float a, b, c;
	int ng = 0;
	do {
		ng++;
		a = (float)((nx - 1) / (1 << ng) + 1);
		b = (float)((ny - 1) / (1 << ng) + 1);
		c = (float)((nz - 1) / (1 << ng) + 1);
	} while (fminf(fminf(a, b), c) >= min_coarse);
	return ng;
}

/* so_fine: nstncl = 14 (xxvii_pt) or 4 (seven_pt: p, pw, ps, b) planes */
o3_solver *o3_create(const o3_settings *s, const double *so_fine, int nstncl, int nx, int ny, int nz)
{
	o3_solver *h = (o3_solver *)calloc(1, sizeof(o3_solver));
	h->s = *s;
	int nl = o3_num_levels(nx, ny, nz, s->min_coarse);
	if (s->num_levels > 0 && s->num_levels <= nl) nl = s->num_levels;
	h->nlev = nl;
	h->lv = (struct o3_level *)calloc(nl, sizeof(struct o3_level));
	for (int l = 0; l < nl; ++l) {
		struct o3_level *L = &h->lv[l];
		if (l == 0) { L->nx = nx; L->ny = ny; L->nz = nz; }
		else {
			L->nx = (int)((h->lv[l - 1].nx - 1) / 2. + 1);
			L->ny = (int)((h->lv[l - 1].ny - 1) / 2. + 1);
			L->nz = (int)((h->lv[l - 1].nz - 1) / 2. + 1);
		}
		L->ii = L->nx + 2; L->jj = L->ny + 2; L->kk = L->nz + 2;
		L->ns = l == 0 ? nstncl : 14;
		size_t n = (size_t)L->ii * L->jj * L->kk;
		L->so = zal(n * 14); L->x = zal(n); L->b = zal(n); L->res = zal(n); L->sor = zal(n); L->ci = zal(n * 26);
	}
	memcpy(h->lv[0].so, so_fine, sizeof(double) * (size_t)(nx + 2) * (ny + 2) * (nz + 2) * nstncl);
	for (int l = 0; l + 1 < nl; ++l) {
		struct o3_level *F = &h->lv[l], *C = &h->lv[l + 1];
		if (F->ns == 4) o3_setup_interp7(F->so, C->ci, F->ii, F->jj, F->kk, C->ii, C->jj, C->kk);
		else o3_setup_interp(F->so, C->ci, F->ii, F->jj, F->kk, C->ii, C->jj, C->kk);
		o3_galerkin(F->so, C->so, C->ci, F->ii, F->jj, F->kk, C->ii, C->jj, C->kk);
		o3_setup_recip(F->so, F->sor, F->ii, F->jj, F->kk);
	}
	/* plane smoothers on every level but the coarsest (multilevel.h:147-159) */
	for (int l = 0; l + 1 < nl; ++l) {
		struct o3_level *F = &h->lv[l];
		if (s->relax == O3_RELAX_PLANE_XYZ || s->relax == O3_RELAX_PLANE_XY) planes_setup(F, O3_XY);
		if (s->relax == O3_RELAX_PLANE_XYZ || s->relax == O3_RELAX_PLANE_XZ) planes_setup(F, O3_XZ);
		if (s->relax == O3_RELAX_PLANE_XYZ || s->relax == O3_RELAX_PLANE_YZ) planes_setup(F, O3_YZ);
	}
	struct o3_level *Cg = &h->lv[nl - 1];
	h->nabd1 = Cg->nx * (Cg->ny + 1) + 2;
	int nn = Cg->nx * Cg->ny * Cg->nz;
	h->abd = zal((size_t)h->nabd1 * nn);
	h->bbd = zal(nn);
	h->cg_info = o3_setup_cg(Cg->so, Cg->ii, Cg->jj, Cg->kk, h->abd, h->nabd1);
	return h;
}

void o3_destroy(o3_solver *h)
{
	if (!h) return;
	for (int l = 0; l < h->nlev; ++l) {
		struct o3_level *L = &h->lv[l];
		planes_free(L);
		free(L->so); free(L->x); free(L->b); free(L->res); free(L->sor); free(L->ci);
	}
	free(h->lv); free(h->abd); free(h->bbd); free(h);
}

static void resid3(struct o3_level *L, const double *b, const double *x)
{
	if (L->ns == 4) o3_residual7(L->so, b, x, L->res, L->ii, L->jj, L->kk);
	else o3_residual(L->so, b, x, L->res, L->ii, L->jj, L->kk);
}

/* multilevel::setup_relax_helper closures, include/cedar/multilevel.h:160-222:
 * plane-xyz runs xy, yz, xz going down and xz, yz, xy going up */
static void smooth3(o3_solver *h, struct o3_level *L, int updown)
{
	int n = updown == 0 ? h->s.nrelax_pre : h->s.nrelax_post;
	for (int it = 0; it < n; ++it) {
		switch (h->s.relax) {
		case O3_RELAX_PLANE_XY: relax_planes_level(L, O3_XY, L->x, L->b, updown); break;
		case O3_RELAX_PLANE_XZ: relax_planes_level(L, O3_XZ, L->x, L->b, updown); break;
		case O3_RELAX_PLANE_YZ: relax_planes_level(L, O3_YZ, L->x, L->b, updown); break;
		case O3_RELAX_PLANE_XYZ:
			if (updown == 0) {
				relax_planes_level(L, O3_XY, L->x, L->b, updown);
				relax_planes_level(L, O3_YZ, L->x, L->b, updown);
				relax_planes_level(L, O3_XZ, L->x, L->b, updown);
			} else {
				relax_planes_level(L, O3_XZ, L->x, L->b, updown);
				relax_planes_level(L, O3_YZ, L->x, L->b, updown);
				relax_planes_level(L, O3_XY, L->x, L->b, updown);
			}
			break;
		default:
			if (L->ns == 4) o3_relax_gs7(L->so, L->b, L->x, L->sor, L->ii, L->jj, L->kk, updown);
			else o3_relax_gs(L->so, L->b, L->x, L->sor, L->ii, L->jj, L->kk, updown);
		}
	}
}

static void ncycle3(o3_solver *h, int l, double *x, const double *b)
{
	struct o3_level *L = &h->lv[l], *C = &h->lv[l + 1];
	double *sx = L->x, *sb = L->b;
	L->x = x; L->b = (double *)b;
	smooth3(h, L, 0);
	resid3(L, L->b, L->x);
	o3_restrict(C->ci, L->res, C->b, L->ii, L->jj, L->kk, C->ii, C->jj, C->kk);
	memset(C->x, 0, sizeof(double) * (size_t)C->ii * C->jj * C->kk);
	if (l + 1 == h->nlev - 1) o3_solve_cg(C->x, C->b, C->ii, C->jj, C->kk, h->abd, h->bbd, h->nabd1);
	else ncycle3(h, l + 1, C->x, C->b);
	o3_interp_add(L->x, C->x, L->res, L->so, C->ci, C->ii, C->jj, C->kk, L->ii, L->jj, L->kk);
	smooth3(h, L, 1);
	L->x = sx; L->b = sb;
}

void o3_vcycle(o3_solver *h, double *x, const double *b)
{
	if (h->nlev == 1) {
		struct o3_level *L = &h->lv[0];
		o3_solve_cg(x, b, L->ii, L->jj, L->kk, h->abd, h->bbd, h->nabd1);
	} else {
		ncycle3(h, 0, x, b);
	}
}

/* cycle::fcycle::fmg_cycle / fmg_cycle_helper (include/cedar/cycle/fcycle.h:49-83):
 * restrict b, recurse (the coarsest level solved directly), then x = P x_c with a
 * zero residual term and one V-cycle on this level */
static void fcycle3(o3_solver *h, int l, double *x, const double *b)
{
	struct o3_level *L = &h->lv[l];
	if (l == h->nlev - 1) {
		o3_solve_cg(x, b, L->ii, L->jj, L->kk, h->abd, h->bbd, h->nabd1);
		return;
	}
	struct o3_level *C = &h->lv[l + 1];
	const size_t n = (size_t)L->ii * L->jj * L->kk;
	o3_restrict(C->ci, b, C->b, L->ii, L->jj, L->kk, C->ii, C->jj, C->kk);
	fcycle3(h, l + 1, C->x, C->b);
	memset(x, 0, sizeof(double) * n);
	memset(L->res, 0, sizeof(double) * n);
	o3_interp_add(x, C->x, L->res, L->so, C->ci, C->ii, C->jj, C->kk, L->ii, L->jj, L->kk);
	ncycle3(h, l, x, b);
}

void o3_cycle(o3_solver *h, double *x, const double *b)
{
	if (h->s.cycle == 1 && h->nlev > 1) fcycle3(h, 0, x, b);
	else o3_vcycle(h, x, b);
}

int o3_solve(o3_solver *h, const double *b, double *x, double *hist, int maxhist)
{
	struct o3_level *L = &h->lv[0];
	resid3(L, b, x);
	double res0 = o3_l2norm(L->res, L->ii, L->jj, L->kk);
	int it;
	for (it = 0; it < h->s.maxiter; ++it) {
		o3_cycle(h, x, b);
		resid3(L, b, x);
		double rel = o3_l2norm(L->res, L->ii, L->jj, L->kk) / res0;
		if (hist && it < maxhist) hist[it] = rel;
		if (rel < h->s.tol) { ++it; break; }
	}
	return it;
}

int o3_nlevels(const o3_solver *h) { return h->nlev; }
int o3_cg_info(const o3_solver *h) { return h->cg_info; }
void o3_level_dims(const o3_solver *h, int l, int *d) { d[0] = h->lv[l].nx; d[1] = h->lv[l].ny; d[2] = h->lv[l].nz; }
double *o3_level_array(o3_solver *h, int l, int which)
{
	struct o3_level *L = &h->lv[l];
	switch (which) {
	case 0: return L->so;
	case 1: return L->x;
	case 2: return L->b;
	case 3: return L->res;
	case 4: return L->sor;
	case 6: return L->ci;
	default: return NULL;
	}
}

void o3_relax_planes(o3_solver *h, int l, int dir, double *x, const double *b, int updown)
{
	relax_planes_level(&h->lv[l], dir, x, b, updown);
}

const double *o3_plane_op(o3_solver *h, int l, int dir, int ipl, int *n1, int *n2)
{
	struct o3_planes *P = &h->lv[l].pl[dir];
	if (!P->s || ipl < 1 || ipl > P->n) return NULL;
	*n1 = P->n1;
	*n2 = P->n2;
	return P->so2[ipl - 1];
}
