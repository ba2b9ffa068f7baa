// k2_point.cuh -- device helpers shared by the 2D point kernels.
#pragma once
#include "cdr_common.cuh"

namespace cdrgpu {

constexpr int TX = 32, TY = 8;  // 2D tile of the point kernels

// a*b + c: one fused multiply-add in FP32 (the preconditioner's kernels), a
// separately rounded product and sum in FP64 (the library is built without FMA
// contraction so that the FP64 kernels give the reference's bits; c + a*b and
// a*b + c are the same IEEE sum).
template <typename T>
__device__ __forceinline__ T madd(T a, T b, T c)
{
	if constexpr (sizeof(T) == 4) return __fmaf_rn(a, b, c);
	else return a * b + c;
}

// BMG2_SymStd_residual (src/2d/ftn/BMG2_SymStd_residual.f90:89-117).
template <typename T, int NS>
__device__ __forceinline__ T resid_at(const T *__restrict__ so, size_t ps, const T *__restrict__ q,
                                      const T *__restrict__ qf, size_t k, int pitch)
{
	const T *c = so, *w = so + ps, *s = so + 2 * ps;
	T a = madd(w[k], q[k - 1], qf[k]);
	a = madd(w[k + 1], q[k + 1], a);
	a = madd(s[k], q[k - pitch], a);
	a = madd(s[k + pitch], q[k + pitch], a);
	if (NS == 5) {
		const T *sw = so + 3 * ps, *nw = so + 4 * ps;
		a = madd(sw[k], q[k - pitch - 1], a);
		a = madd(nw[k + 1], q[k - pitch + 1], a);
		a = madd(nw[k + pitch], q[k + pitch - 1], a);
		a = madd(sw[k + pitch + 1], q[k + pitch + 1], a);
	}
	return madd(-c[k], q[k], a);
}

// One point of a Gauss-Seidel colour (BMG2_SymStd_relax_GS.f90:93-133):
// q(k) = (qf + couplings * q) * sor, in the reference's operand order.
template <typename T, int NS>
__device__ __forceinline__ void gs_at(const T *__restrict__ so, size_t ps, T *__restrict__ q,
                                      const T *__restrict__ qf, const T *__restrict__ sor, size_t k, int pitch)
{
	const T *w = so + ps, *s = so + 2 * ps;
	T acc = madd(w[k], q[k - 1], qf[k]);
	acc = madd(w[k + 1], q[k + 1], acc);
	acc = madd(s[k], q[k - pitch], acc);
	acc = madd(s[k + pitch], q[k + pitch], acc);
	if (NS == 5) {
		const T *sw = so + 3 * ps, *nw = so + 4 * ps;
		acc = madd(sw[k], q[k - pitch - 1], acc);
		acc = madd(nw[k + 1], q[k - pitch + 1], acc);
		acc = madd(nw[k + pitch], q[k + pitch - 1], acc);
		acc = madd(sw[k + pitch + 1], q[k + pitch + 1], acc);
	}
	q[k] = acc * sor[k];
}

// Coarse point (ic, jc) of BMG2_SymStd_restrict (src/2d/ftn/BMG2_SymStd_restrict.f90:72-92);
// it sits on fine (2ic-1, 2jc-1) (0-based, ghosts at 0).  TF/TC: fine and
// coarse types (equal except where an FP32 level hands over to an FP64 one;
// the sum is then formed in the coarse type).
template <typename TF, typename TC = TF>
__device__ __forceinline__ void restrict_at(const TC *__restrict__ ci, const TF *__restrict__ q, TC *__restrict__ qc,
                                            const Dims2 &f, const Dims2 &c, int ic, int jc)
{
	const size_t cps = c.plane();
	const int cp = c.pitch, fp = f.pitch;
	const size_t kc = c.at(ic, jc), kf = f.at(2 * ic - 1, 2 * jc - 1);
	const TC *cL = ci + IL * cps, *cR = ci + IR * cps, *cA = ci + IA * cps, *cB = ci + IB * cps;
	const TC *cSW = ci + ISW * cps, *cNW = ci + INW * cps, *cNE = ci + INE * cps, *cSE = ci + ISE * cps;
	auto Q = [&](size_t k) -> TC { return (TC)q[k]; };
	TC a = cNE[kc] * Q(kf - fp - 1);
	a = madd(cA[kc], Q(kf - fp), a);
	a = madd(cNW[kc + 1], Q(kf - fp + 1), a);
	a = madd(cR[kc], Q(kf - 1), a);
	a = a + Q(kf);
	a = madd(cL[kc + 1], Q(kf + 1), a);
	a = madd(cSE[kc + cp], Q(kf + fp - 1), a);
	a = madd(cB[kc + cp], Q(kf + fp), a);
	qc[kc] = madd(cSW[kc + cp + 1], Q(kf + fp + 1), a);
}

// Coarse cell (ic, jc) of BMG2_SymStd_interp_add (src/2d/ftn/BMG2_SymStd_interp_add.f90:101-137),
// ic in [1, nxf/2+1]: fine points (i, j), (i-1, j), (i, j-1), (i-1, j-1), i = 2ic-1.
// r/c is formed on the fly; the reference divides r by c on interior points
// only, and for even grid sizes its loop also reaches the ghost row/column,
// where r is added undivided.
// TF/TC as in restrict_at: the correction is formed in the coarse type and
// rounded to the fine one.
template <typename TF, typename TC = TF>
__device__ __forceinline__ void interp_at(const TC *__restrict__ ci, const TC *__restrict__ qc,
                                          const TF *__restrict__ res, const TF *__restrict__ soc, TF *__restrict__ q,
                                          const Dims2 &f, const Dims2 &c, int ic, int jc)
{
	const size_t cps = c.plane();
	const int cp = c.pitch, fp = f.pitch;
	const int i = 2 * ic - 1, j = 2 * jc - 1;
	const size_t kc = c.at(ic, jc), kf = f.at(i, j);
	auto rc = [&](size_t k, int ii, int jj) -> TC {
		return (ii <= f.nx && jj <= f.ny) ? (TC)(res[k] / soc[k]) : (TC)res[k];
	};
	auto Q = [&](size_t k) -> TC { return (TC)q[k]; };
	const TC qcc = qc[kc];
	q[kf] = (TF)(Q(kf) + qcc);
	if (ic >= 2) {
		const TC a = madd(ci[IL * cps + kc], qc[kc - 1], ci[IR * cps + kc] * qcc);
		const size_t k = kf - 1;
		q[k] = (TF)(Q(k) + a + rc(k, i - 1, j));
	}
	if (jc >= 2) {
		const TC aq = madd(ci[IB * cps + kc], qc[kc - cp], ci[IA * cps + kc] * qcc);
		const size_t k = kf - fp;
		q[k] = (TF)(Q(k) + aq + rc(k, i, j - 1));
	}
	if (ic >= 2 && jc >= 2) {
		TC a = madd(ci[INW * cps + kc], qc[kc - 1], ci[ISW * cps + kc] * qc[kc - cp - 1]);
		a = madd(ci[INE * cps + kc], qcc, a);
		a = madd(ci[ISE * cps + kc], qc[kc - cp], a);
		const size_t k = kf - fp - 1;
		q[k] = (TF)(Q(k) + a + rc(k, i - 1, j - 1));
	}
}

// Right-hand side of line relaxation at (i, j): b plus the couplings to the two
// neighbouring lines (relax_lines_x.f90:106-110, relax_lines_y.f90:102-106 operand order).
template <typename T, int NS, int DIR>
__device__ __forceinline__ T line_rhs(const T *__restrict__ so, size_t ps, const T *__restrict__ q,
                                      const T *__restrict__ qf, size_t k, int p)
{
	const T *w = so + ps, *s = so + 2 * ps;
	T a;
	if (DIR == CDR_DIR_X) {
		a = madd(s[k], q[k - p], qf[k]);
		a = madd(s[k + p], q[k + p], a);
	} else {
		a = madd(w[k], q[k - 1], qf[k]);
		a = madd(w[k + 1], q[k + 1], a);
	}
	if (NS == 5) {
		const T *sw = so + 3 * ps, *nw = so + 4 * ps;
		a = madd(sw[k], q[k - p - 1], a);
		a = madd(nw[k + 1], q[k - p + 1], a);
		a = madd(nw[k + p], q[k + p - 1], a);
		a = madd(sw[k + p + 1], q[k + p + 1], a);
	}
	return a;
}

// Per-problem size of the line-factor array of one direction (2 planes; y-line
// factors transposed, planes tpitch*(nx+2) apart).
__host__ __device__ __forceinline__ size_t line_factor_size(Dims2 d, int tpitch, int dir)
{
	return dir == CDR_DIR_X ? 2 * d.plane() : 2 * (size_t)tpitch * (d.nx + 2);
}

// y / d with a stored line pivot: FP64 factors keep d (DPTTS2 divides), FP32
// factors keep the reciprocal 1/d (the FP32 sweeps multiply).
template <typename TS>
__device__ __forceinline__ TS pivot_store(double d)
{
	return sizeof(TS) == 4 ? (TS)(1.0 / d) : (TS)d;
}
template <typename T>
__device__ __forceinline__ T pivot_div(T y, T dstored)
{
	return sizeof(T) == 4 ? y * dstored : y / dstored;
}

template <int NW>
__device__ __forceinline__ double block_sum(double v, double *sh)
{
	for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
	int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
	int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
	if (lane == 0) sh[warp] = v;
	__syncthreads();
	double t = 0;
	if (warp == 0) {
		t = lane < NW ? sh[lane] : 0.0;
		for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
	}
	return t;
}

}  // namespace cdrgpu
