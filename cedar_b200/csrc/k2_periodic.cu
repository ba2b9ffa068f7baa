// k2_periodic.cu -- periodic boundary conditions of the 2D BoxMG kernels.
//
// Cedar maps grid.periodic to a boundary-condition code (BMG_get_bc,
// src/2d/ftn/BMG_get_bc.f90:11-22): per_mask bit 0 (x) -> BMG_BCs_def_per_x,
// bit 1 (y) -> def_per_y, both -> def_per_xy.  A periodic direction keeps, in
// each ghost line, a copy of the opposite interior line, and every kernel
// restates the reference's updates of those copies:
//   - ghost_copy_2d: the copies themselves (Gauss-Seidel, restriction,
//     interpolation, Galerkin operator);
//   - setup_interp_per_2d: the periodic branch of the operator-induced
//     interpolation (src/2d/ftn/BMG2_SymStd_SETUP_interp_OI.f90:259-612);
//   - setup_cg_per_2d / solve_cg_per_2d: the coarsest operator as a dense
//     matrix with the wrap-around couplings, its Cholesky factor and solve
//     with the mean-zero shift (SETUP_cg_LU.f90:120-227, 256-343 with DPOTRF;
//     SOLVE_cg.f90:88-163 with DPOTRS).
// Arithmetic keeps the reference's operand order (no FMA contraction in this
// library), so every array has the bits of the serial restatement.
#include "k2_point.cuh"
#include "kernels2d.cuh"

namespace cdrgpu {

// ------------------------------------------------------------- ghost copies
// A ghost line of a periodic direction takes the opposite interior line:
// x: column 0 <- nx, column nx+1 <- 1; y: row 0 <- ny, row ny+1 <- 1.
// xmode 1 copies the x ghosts of interior rows (those of parity jpar when
// jpar >= 0), xmode 2 of every row; ymode 1 copies the y ghost rows over
// their full width.  With both, the corners take the interior corner point,
// which is what the reference's two loops in sequence leave there (the x and
// y copies commute).  No cell read is written in the same launch.
template <typename T>
__global__ void k_ghost(T *__restrict__ q, Dims2 d, int planes, int xmode, int ymode, int jpar)
{
	const int nxg = d.nx + 2, nrow = 2 * nxg;
	int t = blockIdx.x * blockDim.x + threadIdx.x, i, j;
	if (t < nrow) {
		j = t < nxg ? 0 : d.ny + 1;
		i = t < nxg ? t : t - nxg;
	} else if (t < nrow + 2 * d.ny) {
		t -= nrow;
		i = t < d.ny ? 0 : d.nx + 1;
		j = 1 + (t < d.ny ? t : t - d.ny);
	} else {
		return;
	}
	const bool gx = i == 0 || i == d.nx + 1, gy = j == 0 || j == d.ny + 1;
	bool wx = false;
	if (xmode && gx) wx = xmode == 2 || (!gy && (jpar < 0 || (j & 1) == jpar));
	const bool wy = ymode && gy;
	if (!wx && !wy) return;
	const int si = wx ? (i == 0 ? d.nx : 1) : i;
	const int sj = wy ? (j == 0 ? d.ny : 1) : j;
	const size_t ps = d.plane();
	for (int p = 0; p < planes; ++p) q[p * ps + d.at(i, j)] = q[p * ps + d.at(si, sj)];
}

template <typename T>
int ghost_copy_2d(T *q, Dims2 d, int planes, int xmode, int ymode, int jpar, cudaStream_t st)
{
	if (!xmode && !ymode) return CDR_OK;
	if (xmode == 1 && ymode) {  // the corner sources would race; no caller needs it
		set_error(CDR_ERR_ARG, "ghost_copy_2d: interior-row x copies and y copies in one launch");
		return CDR_ERR_ARG;
	}
	const int n = 2 * (d.nx + 2) + 2 * d.ny;
	k_ghost<T><<<ceil_div(n, 256), 256, 0, st>>>(q, d, planes, xmode, ymode, jpar);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int ghost_copy_2d<double>(double *, Dims2, int, int, int, int, cudaStream_t);
template int ghost_copy_2d<float>(float *, Dims2, int, int, int, int, cudaStream_t);

// ---------------------------------------- operator-induced interpolation
// Fortran indices below (1-based, ghosts at 1 and II/JJ), as in the reference.
// Coarse column IC reads fine column I = 2(IC-1), except that the reference
// walks I by I <- MAX(MOD(I+2, IIFC), MIN(I+2, 3)), which wraps to 3 once
// I + 2 reaches IIFC (only at the coarse ghost column of an odd periodic
// grid).  wrap_index gives the walk's value at IC; the host checks it
// against the walk itself before the launch.
struct PerOI {
	int IIC, JJC, IBEGC, IENDC, JBEGC, JENDC, IIFC, JJFC, IBEG_x, IEND_x, JBEG_y, JEND_y, perx, pery;
};

__host__ __device__ inline int wrap_index(int v, int P) { return v < P ? v : (v == P ? 3 : v - P + 3); }

static PerOI per_oi_geometry(Dims2 f, Dims2 c, int per)
{
	PerOI g;
	const int IIF = f.nx + 2, JJF = f.ny + 2;
	g.IIC = c.nx + 2;
	g.JJC = c.ny + 2;
	const int IICF = (IIF - 2) / 2 + 3, JJCF = (JJF - 2) / 2 + 3;
	g.IIFC = 2 * (IICF - 2) + 2;
	g.JJFC = 2 * (JJCF - 2) + 2;
	g.perx = per & 1;
	g.pery = (per >> 1) & 1;
	g.IBEGC = 3;
	g.IENDC = IICF - 1;
	g.IBEG_x = 2;
	g.IEND_x = IIF - 2;
	if (g.perx) {
		g.IBEGC = 2;
		if (g.IIC == IICF) {
			g.IENDC = IICF;
			g.IBEG_x = 3;
			g.IEND_x = IIF - 1;
		}
	}
	g.JBEGC = 3;
	g.JENDC = JJCF - 1;
	g.JBEG_y = 2;
	g.JEND_y = JJF - 2;
	if (g.pery) {
		g.JBEGC = 2;
		if (g.JJC == JJCF) {
			g.JENDC = JJCF;
			g.JBEG_y = 3;
			g.JEND_y = JJF - 1;
		}
	}
	return g;
}

// the reference's walk from its start value, compared with wrap_index
static bool walk_matches(int beg, int begc, int endc, int P)
{
	int I = beg;
	for (int IC = begc; IC <= endc; ++IC) {
		const int a = (I + 2) % P, b = I + 2 < 3 ? I + 2 : 3;
		I = a > b ? a : b;
		if (I != wrap_index(2 * (IC - 1), P)) return false;
	}
	return true;
}

constexpr double kEmach = 1.1102230246251565e-16;  // D1MACH(3) = 2^-53

template <int NS>
struct OISten {
	const double *so;
	size_t ps;
	int fp;
	__device__ double operator()(int I, int J, int K) const { return so[K * ps + (size_t)(J - 1) * fp + (I - 1)]; }
};
enum : int { KO = 0, KW = 1, KS = 2, KSW = 3, KNW = 4 };

// x-edge weights (LR, LL) at coarse (IC, JC) from fine point (I-1, J)
template <int NS>
__device__ void oi_xedge(const OISten<NS> &SO, double *ci, size_t cps, const Dims2 &c, int IC, int JC, int I, int J)
{
	double A, B;
	if (NS == 5) {
		A = SO(I, J, KW) + SO(I, J, KNW) + SO(I, J + 1, KSW);
		B = SO(I - 1, J, KW) + SO(I - 1, J, KSW) + SO(I - 1, J + 1, KNW);
	} else {
		A = SO(I, J, KW);
		B = SO(I - 1, J, KW);
	}
	const double o = SO(I - 1, J, KO);
	const double EP = fmin(fabs(A / o), fabs(B / o));
	double SUM = A + B + SO(I - 1, J, KS) + SO(I - 1, J + 1, KS);
	SUM = A + B + (o - SUM) * fmax(o - (1.0 + EP) * SUM, 0.0) / (fabs(o - (1.0 + EP) * SUM) + kEmach);
	SUM = 1.0 / SUM;
	const size_t kc = c.at(IC - 1, JC - 1);
	ci[IR * cps + kc] = A * SUM;
	ci[IL * cps + kc] = B * SUM;
}

// y-edge weights (LA, LB) at coarse (IC, JC) from fine point (I, J-1)
template <int NS>
__device__ void oi_yedge(const OISten<NS> &SO, double *ci, size_t cps, const Dims2 &c, int IC, int JC, int I, int J)
{
	double A, B;
	if (NS == 5) {
		A = SO(I, J, KS) + SO(I, J, KNW) + SO(I + 1, J, KSW);
		B = SO(I, J - 1, KS) + SO(I, J - 1, KSW) + SO(I + 1, J - 1, KNW);
	} else {
		A = SO(I, J, KS);
		B = SO(I, J - 1, KS);
	}
	const double o = SO(I, J - 1, KO);
	double SUM = A + B + SO(I, J - 1, KW) + SO(I + 1, J - 1, KW);
	const double EP = fmin(fabs(A / o), fabs(B / o));
	SUM = A + B + (o - SUM) * fmax(o - (1.0 + EP) * SUM, 0.0) / (fabs(o - (1.0 + EP) * SUM) + kEmach);
	SUM = 1.0 / SUM;
	const size_t kc = c.at(IC - 1, JC - 1);
	ci[IA * cps + kc] = A * SUM;
	ci[IB * cps + kc] = B * SUM;
}

// Phase 1: every edge weight of the periodic branch -- the x-edge loop over
// interior coarse rows and its two y strips (coarse ghost rows), the y-edge
// loop over interior coarse columns and its two x strips.  Each (IC, JC,
// plane) is written once.
template <int NS>
__global__ void k_oi_per_edges(const double *__restrict__ so, double *__restrict__ ci, Dims2 f, Dims2 c, PerOI g)
{
	const int IC = blockIdx.x * TX + threadIdx.x + 1, JC = blockIdx.y * TY + threadIdx.y + 1;
	if (IC > g.IIC || JC > g.JJC) return;
	const OISten<NS> SO{so, f.plane(), f.pitch};
	const size_t cps = c.plane();
	if (IC >= g.IBEGC && IC <= g.IENDC) {
		int J = -1;
		if (JC >= 2 && JC <= g.JJC - 1) J = 2 * (JC - 1);
		else if (g.pery && JC == g.JJC) J = g.JBEG_y;
		else if (g.pery && JC == 1) J = g.JEND_y;
		if (J >= 0) oi_xedge<NS>(SO, ci, cps, c, IC, JC, wrap_index(2 * (IC - 1), g.IIFC), J);
	}
	if (JC >= g.JBEGC && JC <= g.JENDC) {
		int I = -1;
		if (IC >= 2 && IC <= g.IIC - 1) I = 2 * (IC - 1);
		else if (g.perx && IC == g.IIC) I = g.IBEG_x;
		else if (g.perx && IC == 1) I = g.IEND_x;
		if (I >= 0) oi_yedge<NS>(SO, ci, cps, c, IC, JC, I, wrap_index(2 * (JC - 1), g.JJFC));
	}
}

// Phase 2: the corner weights, which read the edge weights of phase 1.
template <int NS>
__global__ void k_oi_per_corners(const double *__restrict__ so, double *__restrict__ ci, Dims2 f, Dims2 c, PerOI g)
{
	const int IC = blockIdx.x * TX + threadIdx.x + g.IBEGC, JC = blockIdx.y * TY + threadIdx.y + g.JBEGC;
	if (IC > g.IENDC || JC > g.JENDC) return;
	const OISten<NS> SO{so, f.plane(), f.pitch};
	const size_t cps = c.plane();
	const int I = wrap_index(2 * (IC - 1), g.IIFC), J = wrap_index(2 * (JC - 1), g.JJFC);
	auto CI = [&](int ic, int jc, int k) { return ci[k * cps + c.at(ic - 1, jc - 1)]; };
	const double o = SO(I - 1, J - 1, KO);
	double SUM, EP;
	if (NS == 5) {
		SUM = SO(I - 1, J - 1, KW) + SO(I - 1, J, KNW) + SO(I - 1, J, KS) + SO(I, J, KSW) + SO(I, J - 1, KW) +
		      SO(I, J - 1, KNW) + SO(I - 1, J - 1, KS) + SO(I - 1, J - 1, KSW);
		EP = fmin(fmin(fabs((SO(I - 1, J - 1, KSW) + SO(I - 1, J - 1, KW) + SO(I - 1, J, KNW)) / o),
		               fabs((SO(I - 1, J, KNW) + SO(I - 1, J, KS) + SO(I, J, KSW)) / o)),
		          fmin(fabs((SO(I, J, KSW) + SO(I, J - 1, KW) + SO(I, J - 1, KNW)) / o),
		               fabs((SO(I, J - 1, KNW) + SO(I - 1, J - 1, KS) + SO(I - 1, J - 1, KSW)) / o)));
	} else {
		SUM = SO(I - 1, J - 1, KW) + SO(I - 1, J, KS) + SO(I, J - 1, KW) + SO(I - 1, J - 1, KS);
		EP = fmin(fmin(fabs(SO(I - 1, J - 1, KW) / o), fabs(SO(I - 1, J, KS) / o)),
		          fmin(fabs(SO(I, J - 1, KW) / o), fabs(SO(I - 1, J - 1, KS) / o)));
	}
	SUM = SUM + (o - SUM) * fmax(o - (1.0 + EP) * SUM, 0.0) / (fabs(o - (1.0 + EP) * SUM) + kEmach);
	const double S = 1.0 / SUM;
	const size_t kc = c.at(IC - 1, JC - 1);
	if (NS == 5) {
		ci[ISW * cps + kc] = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, IL) + SO(I - 1, J - 1, KW) * CI(IC - 1, JC, IB) +
		                      SO(I - 1, J - 1, KSW)) * S;
		ci[ISE * cps + kc] = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, IR) + SO(I, J - 1, KW) * CI(IC, JC, IB) +
		                      SO(I, J - 1, KNW)) * S;
		ci[INW * cps + kc] = (SO(I - 1, J - 1, KW) * CI(IC - 1, JC, IA) + SO(I - 1, J, KS) * CI(IC, JC, IL) +
		                      SO(I - 1, J, KNW)) * S;
		ci[INE * cps + kc] = (SO(I - 1, J, KS) * CI(IC, JC, IR) + SO(I, J - 1, KW) * CI(IC, JC, IA) +
		                      SO(I, J, KSW)) * S;
	} else {
		ci[ISW * cps + kc] = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, IL) + SO(I - 1, J - 1, KW) * CI(IC - 1, JC, IB)) * S;
		ci[ISE * cps + kc] = (SO(I - 1, J - 1, KS) * CI(IC, JC - 1, IR) + SO(I, J - 1, KW) * CI(IC, JC, IB)) * S;
		ci[INW * cps + kc] = (SO(I - 1, J - 1, KW) * CI(IC - 1, JC, IA) + SO(I - 1, J, KS) * CI(IC, JC, IL)) * S;
		ci[INE * cps + kc] = (SO(I - 1, J, KS) * CI(IC, JC, IR) + SO(I, J - 1, KW) * CI(IC, JC, IA)) * S;
	}
}

int setup_interp_per_2d(const double *so, int nstencil, double *ci, Dims2 f, Dims2 c, int per, cudaStream_t st)
{
	if (f.nb != 1) {
		set_error(CDR_ERR_UNSUPPORTED, "periodic interpolation of a batch");
		return CDR_ERR_UNSUPPORTED;
	}
	const PerOI g = per_oi_geometry(f, c, per);
	if (!walk_matches(g.perx ? 0 : 2, g.IBEGC, g.IENDC, g.IIFC) ||
	    !walk_matches(g.pery ? 0 : 2, g.JBEGC, g.JENDC, g.JJFC)) {
		set_error(CDR_ERR_DIM, "periodic interpolation: column walk of a %dx%d -> %dx%d level", f.nx, f.ny, c.nx, c.ny);
		return CDR_ERR_DIM;
	}
	CDR_CUDA_TRY(cudaMemsetAsync(ci, 0, sizeof(double) * c.plane() * 8, st));
	dim3 blk(TX, TY);
	dim3 g1(ceil_div(g.IIC, TX), ceil_div(g.JJC, TY));
	dim3 g2(ceil_div(g.IENDC - g.IBEGC + 1, TX), ceil_div(g.JENDC - g.JBEGC + 1, TY));
	if (nstencil == 5) {
		k_oi_per_edges<5><<<g1, blk, 0, st>>>(so, ci, f, c, g);
		CDR_LAUNCH_CHECK();
		k_oi_per_corners<5><<<g2, blk, 0, st>>>(so, ci, f, c, g);
	} else {
		k_oi_per_edges<3><<<g1, blk, 0, st>>>(so, ci, f, c, g);
		CDR_LAUNCH_CHECK();
		k_oi_per_corners<3><<<g2, blk, 0, st>>>(so, ci, f, c, g);
	}
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

// ------------------------------------------------ coarsest dense Cholesky
// The coarsest operator with its wrap-around couplings as a dense N x N upper
// triangle, column-major (N = nx*ny, unknowns numbered row by row): the
// assembly of BMG2_SymStd_SETUP_cg_LU's periodic branches, one thread.
__global__ void k_cg_per_assemble(const double *__restrict__ so, int ns, Dims2 d, double *__restrict__ abd, int per)
{
	if (threadIdx.x != 0 || blockIdx.x != 0) return;
	const int II = d.nx + 2, JJ = d.ny + 2, I1 = II - 1, J1 = JJ - 1, I2 = I1 - 1, N = I2 * (J1 - 1);
	const bool perx = per & 1, pery = (per >> 1) & 1, nine = ns == 5;
	const size_t ps = d.plane();
	auto SO = [&](int I, int J, int K) { return so[K * ps + d.at(I - 1, J - 1)]; };
	auto ABD = [&](int i, int j) -> double & { return abd[(size_t)(j - 1) * N + (i - 1)]; };
	int KK = 1;
	ABD(1, 1) = SO(2, 2, KO);
	for (int I = 3; I <= I1; ++I) {
		KK = KK + 1;
		ABD(KK, KK) = SO(I, 2, KO);
		ABD(KK - 1, KK) = -SO(I, 2, KW);
	}
	if (perx) ABD(KK - I2 + 1, KK) = -SO(II, 2, KW);
	for (int J = 3; J <= J1; ++J) {
		if (perx) ABD(KK, KK + 1) = nine ? -SO(2, J, KSW) : 0.0;
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
		if (perx) {
			ABD(KK - I2 + 1, KK) = -SO(II, J, KW);
			ABD(KK - 2 * I2 + 1, KK) = nine ? -SO(II, J, KNW) : 0.0;
		}
	}
	if (pery) {
		KK = KK - I2;
		const int J2 = (J1 - 2) * I2;
		KK = KK + 1;
		ABD(KK - J2, KK) = -SO(2, JJ, KS);
		ABD(KK - J2 + 1, KK) = nine ? -SO(3, JJ, KSW) : 0.0;
		if (perx) ABD(I2, KK) = nine ? -SO(2, JJ, KNW) : 0.0;
		for (int I = 3; I <= I1; ++I) {
			KK = KK + 1;
			ABD(KK - J2, KK) = -SO(I, JJ, KS);
			ABD(KK - J2 - 1, KK) = nine ? -SO(I, JJ, KNW) : 0.0;
			ABD(KK - J2 + 1, KK) = nine ? -SO(I + 1, JJ, KSW) : 0.0;
		}
		ABD(KK - J2 + 1, KK) = 0.0;
		if (perx) ABD(1, KK) = nine ? -SO(II, JJ, KSW) : 0.0;
		if (perx) ABD(KK - 2 * I2 + 1, KK) = nine ? -SO(II, J1, KNW) : 0.0;
	}
}

// Unblocked upper Cholesky (the LAPACK DPOTF2 algorithm): column j's pivot
// from the sequential dot product of the column above it (one thread), then
// row j to its right, each entry by one thread: the sequential dot product
// of its column with column j, subtracted, scaled by the pivot's reciprocal.
// Every entry sees the serial routine's operations in its order.
__global__ void __launch_bounds__(1024) k_cg_per_factor(double *__restrict__ a, int n, int *info)
{
	__shared__ double rcp_s;
	__shared__ int stop_s;
	const int tid = threadIdx.x, nt = blockDim.x;
	int st = 0;
	for (int j = 0; j < n; ++j) {
		double *cj = a + (size_t)j * n;
		if (tid == 0) {
			double dot = 0.0;
			for (int i = 0; i < j; ++i) dot += cj[i] * cj[i];
			double ajj = cj[j] - dot;
			stop_s = !(ajj > 0.0);
			if (stop_s) cj[j] = ajj;
			else {
				ajj = sqrt(ajj);
				cj[j] = ajj;
				rcp_s = 1.0 / ajj;
			}
		}
		__syncthreads();
		if (stop_s) { st = j + 1; break; }
		const double r = rcp_s;
		for (int k = j + 1 + tid; k < n; k += nt) {
			double *ck = a + (size_t)k * n;
			double temp = 0.0;
			for (int i = 0; i < j; ++i) temp += ck[i] * cj[i];
			const double v = ck[j] + -1.0 * temp;
			ck[j] = r * v;
		}
		__syncthreads();
	}
	if (tid == 0 && info) *info = st;
}

int setup_cg_per_2d(const double *so, int nstencil, Dims2 d, double *abd, int *info, int per, cudaStream_t st)
{
	const size_t n = (size_t)d.nx * d.ny;
	CDR_CUDA_TRY(cudaMemsetAsync(abd, 0, sizeof(double) * n * n, st));
	k_cg_per_assemble<<<1, 1, 0, st>>>(so, nstencil, d, abd, per);
	CDR_LAUNCH_CHECK();
	k_cg_per_factor<<<1, 1024, 0, st>>>(abd, (int)n, info);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

// DPOTRS('U') for one right-hand side: U^T y = b (each entry's dot product
// over the earlier ones, applied in their order as they are final), then
// U x = y (column by column from the last); then the mean-zero shift of
// BMG2_SymStd_SOLVE_cg (sequential sum in the unknowns' order) and its ghost
// copies (y rows and x columns of the interior, the four corners when both
// directions are periodic).
__global__ void __launch_bounds__(1024) k_cg_per_solve(const double *__restrict__ a, double *__restrict__ q,
                                                       const double *__restrict__ qf, Dims2 d, int per)
{
	extern __shared__ double bb[];
	__shared__ double shift_s;
	__shared__ int nz_s;
	const int tid = threadIdx.x, nt = blockDim.x, nx = d.nx, n = d.nx * d.ny;
	for (int k = tid; k < n; k += nt) bb[k] = qf[d.at(k % nx + 1, k / nx + 1)];
	__syncthreads();
	for (int k = 0; k < n; ++k) {
		if (tid == 0) bb[k] = bb[k] / a[(size_t)k * n + k];
		__syncthreads();
		const double bk = bb[k];
		for (int i = k + 1 + tid; i < n; i += nt) bb[i] = bb[i] - a[(size_t)i * n + k] * bk;
		__syncthreads();
	}
	for (int k = n - 1; k >= 0; --k) {
		if (tid == 0) {
			nz_s = bb[k] != 0.0;
			if (nz_s) bb[k] = bb[k] / a[(size_t)k * n + k];
		}
		__syncthreads();
		if (nz_s) {
			const double bk = bb[k];
			const double *ck = a + (size_t)k * n;
			for (int i = tid; i < k; i += nt) bb[i] = bb[i] - bk * ck[i];
		}
		__syncthreads();
	}
	if (tid == 0) {
		double qint = 0.0, cint = 0.0;
		for (int k = 0; k < n; ++k) {
			qint = qint + bb[k];
			cint = cint + 1;
		}
		shift_s = -qint / cint;
	}
	__syncthreads();
	const double c = shift_s;
	for (int k = tid; k < n; k += nt) q[d.at(k % nx + 1, k / nx + 1)] = bb[k] + c;
	__syncthreads();
	const bool perx = per & 1, pery = (per >> 1) & 1;
	if (pery)
		for (int i = 1 + tid; i <= d.nx; i += nt) {
			q[d.at(i, d.ny + 1)] = q[d.at(i, 1)];
			q[d.at(i, 0)] = q[d.at(i, d.ny)];
		}
	if (perx)
		for (int j = 1 + tid; j <= d.ny; j += nt) {
			q[d.at(d.nx + 1, j)] = q[d.at(1, j)];
			q[d.at(0, j)] = q[d.at(d.nx, j)];
		}
	if (perx && pery && tid == 0) {
		q[d.at(0, 0)] = q[d.at(d.nx, d.ny)];
		q[d.at(d.nx + 1, 0)] = q[d.at(1, d.ny)];
		q[d.at(0, d.ny + 1)] = q[d.at(d.nx, 1)];
		q[d.at(d.nx + 1, d.ny + 1)] = q[d.at(1, 1)];
	}
}

int solve_cg_per_2d(const double *abd, double *x, const double *b, Dims2 d, int per, cudaStream_t st)
{
	const size_t sm = sizeof(double) * (size_t)d.nx * d.ny;
	if (sm > 48 * 1024) {
		set_error(CDR_ERR_DIM, "coarsest grid %dx%d too large for the dense periodic solve", d.nx, d.ny);
		return CDR_ERR_DIM;
	}
	k_cg_per_solve<<<1, 1024, sm, st>>>(abd, x, b, d, per);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

}  // namespace cdrgpu
