// k2_krylov.cu -- flexible conjugate gradients (FCG(1)) around the 2D cycle.
//
// No counterpart in the reference: its solve (multilevel::solve,
// include/cedar/multilevel.h:278-298) repeats the cycle on the current iterate.
// Here the cycle (FP64, or FP32 inside FP64 recurrences) is the preconditioner
// z = M r of Notay's flexible CG:
//   beta = -(z . q_prev) / (p_prev . q_prev)      (0 on the first iteration)
//   p = z + beta p_prev,  q = A p,  alpha = (p . r) / (p . q)
//   x += alpha p,  r = b - A x
// The residual is formed anew from x every iteration (not updated as r -= alpha
// q): on high-contrast operators the updated residual drifts from b - A x by
// orders of magnitude before it converges, while the formed one stays at the
// FP64 floor eps |A||x|.  Couplings into the ghost ring are taken as zero
// (Dirichlet operators).  All of it is FP64.  Three kernels per iteration, each
// ending in a deterministic grid reduction: every block writes its partial
// sums, and the last block to finish (an atomic ticket) adds the partials in
// block order and updates the device scalars, so the host only reads |r|.
// p and x are double-buffered (device-side parity): A p and A x read neighbours.
#include "k2_point.cuh"
#include "kernels2d.cuh"

namespace cdrgpu {

namespace {

constexpr int kFcgBlocks = 148 * 6;  // grid of every FCG kernel (partials: 2 slots of this)

// Sum the NSUM per-thread values over the grid; the last block calls fin(totals).
template <int NSUM, typename F>
__device__ __forceinline__ void grid_sums(const double (&acc)[NSUM], double *__restrict__ partial,
                                          unsigned *__restrict__ ticket, F fin)
{
	__shared__ double sh[NSUM][TX * TY / 32];
	__shared__ bool last;
	const int tid = threadIdx.y * blockDim.x + threadIdx.x;
	double tot[NSUM];
#pragma unroll
	for (int s = 0; s < NSUM; ++s) tot[s] = block_sum<TX * TY / 32>(acc[s], sh[s]);
	if (tid == 0) {
#pragma unroll
		for (int s = 0; s < NSUM; ++s) partial[s * kFcgBlocks + blockIdx.x] = tot[s];
		__threadfence();
		last = atomicAdd(ticket, 1u) == gridDim.x - 1;
	}
	__syncthreads();
	if (!last || tid >= 32) return;
	__threadfence();
	double v[NSUM];
#pragma unroll
	for (int s = 0; s < NSUM; ++s) {
		v[s] = 0.0;
		for (int b = tid; b < (int)gridDim.x; b += 32) v[s] += __ldcg(partial + s * kFcgBlocks + b);
		for (int o = 16; o > 0; o >>= 1) v[s] += __shfl_down_sync(0xffffffffu, v[s], o);
	}
	if (tid == 0) {
		fin(v);
		*ticket = 0u;
	}
}

// Interior point t of the grid-stride loop -> (i, j); false when outside.
__device__ __forceinline__ bool tile_point(const Dims2 &d, int t, int &i, int &j)
{
	const int tiles_x = (d.nx + TX - 1) / TX;
	i = (t % tiles_x) * TX + threadIdx.x + 1;
	j = (t / tiles_x) * TY + threadIdx.y + 1;
	return i <= d.nx && j <= d.ny;
}

__device__ __forceinline__ int tile_count(const Dims2 &d) { return ((d.nx + TX - 1) / TX) * ((d.ny + TY - 1) / TY); }

// beta from z . q_prev
template <typename TZ>
__global__ void __launch_bounds__(TX *TY) k_fcg_beta(const TZ *__restrict__ z, const double *__restrict__ q, Dims2 d,
                                                     double *__restrict__ partial, FcgScalars *S)
{
	double acc[1] = {0.0};
	if (!S->first) {
		int i, j;
		for (int t = blockIdx.x; t < tile_count(d); t += gridDim.x)
			if (tile_point(d, t, i, j)) {
				const size_t k = d.at(i, j);
				acc[0] += (double)z[k] * q[k];
			}
	}
	grid_sums<1>(acc, partial, &S->ticket[0], [&](const double *v) {
		S->zq = v[0];
		S->beta = S->first ? 0.0 : -v[0] / S->pq;
	});
}

// p = z + beta p_prev (on the fly at the neighbours), q = A p on the interior
// (couplings to the ghost ring dropped), p . q and p . r
template <typename TZ, int NS>
__global__ void __launch_bounds__(TX *TY) k_fcg_dir(const double *__restrict__ so, const TZ *__restrict__ z,
                                                    double *__restrict__ p0, double *__restrict__ p1,
                                                    double *__restrict__ q, const double *__restrict__ r, Dims2 d,
                                                    double *__restrict__ partial, FcgScalars *S)
{
	const size_t ps = d.plane();
	const int pitch = d.pitch;
	const bool odd = S->iter & 1;
	const double *__restrict__ pold = odd ? p1 : p0;
	double *__restrict__ pnew = odd ? p0 : p1;
	const double beta = S->beta;
	const double *c = so, *w = so + ps, *s = so + 2 * ps;
	double acc[2] = {0.0, 0.0};
	auto P = [&](int ii, int jj) -> double {
		if (ii < 1 || ii > d.nx || jj < 1 || jj > d.ny) return 0.0;
		const size_t k = d.at(ii, jj);
		return (double)z[k] + beta * pold[k];
	};
	int i, j;
	for (int t = blockIdx.x; t < tile_count(d); t += gridDim.x)
		if (tile_point(d, t, i, j)) {
			const size_t k = d.at(i, j);
			const double pc = P(i, j);
			double nb = w[k] * P(i - 1, j) + w[k + 1] * P(i + 1, j) + s[k] * P(i, j - 1) + s[k + pitch] * P(i, j + 1);
			if (NS == 5) {
				const double *sw = so + 3 * ps, *nw = so + 4 * ps;
				nb += sw[k] * P(i - 1, j - 1) + nw[k + 1] * P(i + 1, j - 1) + nw[k + pitch] * P(i - 1, j + 1)
				      + sw[k + pitch + 1] * P(i + 1, j + 1);
			}
			const double qk = c[k] * pc - nb;
			pnew[k] = pc;
			q[k] = qk;
			acc[0] += pc * qk;
			acc[1] += pc * r[k];
		}
	grid_sums<2>(acc, partial, &S->ticket[1], [&](const double *v) {
		S->pq = v[0];
		S->alpha = v[1] / v[0];
	});
}

// x_new = x + alpha p and the true residual r = b - A x_new (x double-buffered
// by the same parity, the neighbours' x_new formed on the fly), |r|^2; the next
// preconditioner input (r in the cycle's precision) and a zero initial guess z
// (ghost ring included)
template <typename TZ, int NS>
__global__ void __launch_bounds__(TX *TY) k_fcg_update(const double *__restrict__ so, double *__restrict__ x0,
                                                       double *__restrict__ x1, const double *__restrict__ bb,
                                                       double *__restrict__ r, const double *__restrict__ p0,
                                                       const double *__restrict__ p1, TZ *__restrict__ rin,
                                                       TZ *__restrict__ z, Dims2 d, double *__restrict__ partial,
                                                       FcgScalars *S)
{
	const size_t ps = d.plane();
	const int pitch = d.pitch;
	const bool odd = S->iter & 1;
	const double *__restrict__ pnew = odd ? p0 : p1;
	const double *__restrict__ xold = odd ? x1 : x0;
	double *__restrict__ xnew = odd ? x0 : x1;
	const double alpha = S->alpha;
	const double *c = so, *w = so + ps, *s = so + 2 * ps;
	auto X = [&](int ii, int jj) -> double {
		if (ii < 1 || ii > d.nx || jj < 1 || jj > d.ny) return 0.0;
		const size_t k = d.at(ii, jj);
		return xold[k] + alpha * pnew[k];
	};
	double acc[1] = {0.0};
	int i, j;
	for (int t = blockIdx.x; t < tile_count(d); t += gridDim.x)
		if (tile_point(d, t, i, j)) {
			const size_t k = d.at(i, j);
			const double xc = X(i, j);
			double nb = w[k] * X(i - 1, j) + w[k + 1] * X(i + 1, j) + s[k] * X(i, j - 1) + s[k + pitch] * X(i, j + 1);
			if (NS == 5) {
				const double *sw = so + 3 * ps, *nw = so + 4 * ps;
				nb += sw[k] * X(i - 1, j - 1) + nw[k + 1] * X(i + 1, j - 1) + nw[k + pitch] * X(i - 1, j + 1)
				      + sw[k + pitch + 1] * X(i + 1, j + 1);
			}
			const double rk = bb[k] + nb - c[k] * xc;
			xnew[k] = xc;
			r[k] = rk;
			acc[0] += rk * rk;
			rin[k] = (TZ)rk;
			z[k] = TZ(0);
			if (i == 1) z[k - 1] = TZ(0);
			if (i == d.nx) z[k + 1] = TZ(0);
			if (j == 1) z[k - pitch] = TZ(0);
			if (j == d.ny) z[k + pitch] = TZ(0);
			if (i == 1 && j == 1) z[k - pitch - 1] = TZ(0);
			if (i == d.nx && j == 1) z[k - pitch + 1] = TZ(0);
			if (i == 1 && j == d.ny) z[k + pitch - 1] = TZ(0);
			if (i == d.nx && j == d.ny) z[k + pitch + 1] = TZ(0);
		}
	grid_sums<1>(acc, partial, &S->ticket[2], [&](const double *v) {
		S->rr = v[0];
		S->iter += 1;
		S->first = 0;
	});
}

// Start (or restart) from r: the preconditioner input, a zero z and first = 1.
template <typename TZ>
__global__ void __launch_bounds__(TX *TY) k_fcg_load(const double *__restrict__ r, TZ *__restrict__ rin,
                                                     TZ *__restrict__ z, Dims2 d, FcgScalars *S)
{
	const int i = blockIdx.x * TX + threadIdx.x, j = blockIdx.y * TY + threadIdx.y;
	if (i > d.nx + 1 || j > d.ny + 1) return;
	const size_t k = d.at(i, j);
	const bool in = i >= 1 && i <= d.nx && j >= 1 && j <= d.ny;
	rin[k] = in ? (TZ)r[k] : TZ(0);
	z[k] = TZ(0);
	if (i == 0 && j == 0) {
		S->first = 1;
		S->iter = 0;
	}
}

}  // namespace

template <typename TZ>
int fcg_load(const double *r, TZ *rin, TZ *z, Dims2 d, FcgScalars *S, cudaStream_t st)
{
	k_fcg_load<TZ><<<dim3(ceil_div(d.nx + 2, TX), ceil_div(d.ny + 2, TY)), dim3(TX, TY), 0, st>>>(r, rin, z, d, S);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int fcg_load<double>(const double *, double *, double *, Dims2, FcgScalars *, cudaStream_t);
template int fcg_load<float>(const double *, float *, float *, Dims2, FcgScalars *, cudaStream_t);

template <typename TZ>
int fcg_step(const double *so, int ns, TZ *z, TZ *rin, double *x0, double *x1, const double *b, double *r,
             double *p0, double *p1, double *q, Dims2 d, double *partial, FcgScalars *S, cudaStream_t st)
{
	const int nt = ceil_div(d.nx, TX) * ceil_div(d.ny, TY);
	const int nb = nt < kFcgBlocks ? nt : kFcgBlocks;
	const dim3 blk(TX, TY);
	k_fcg_beta<TZ><<<nb, blk, 0, st>>>(z, q, d, partial, S);
	CDR_LAUNCH_CHECK();
	if (ns == 5) k_fcg_dir<TZ, 5><<<nb, blk, 0, st>>>(so, z, p0, p1, q, r, d, partial, S);
	else k_fcg_dir<TZ, 3><<<nb, blk, 0, st>>>(so, z, p0, p1, q, r, d, partial, S);
	CDR_LAUNCH_CHECK();
	if (ns == 5) k_fcg_update<TZ, 5><<<nb, blk, 0, st>>>(so, x0, x1, b, r, p0, p1, rin, z, d, partial, S);
	else k_fcg_update<TZ, 3><<<nb, blk, 0, st>>>(so, x0, x1, b, r, p0, p1, rin, z, d, partial, S);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int fcg_step<double>(const double *, int, double *, double *, double *, double *, const double *, double *,
                              double *, double *, double *, Dims2, double *, FcgScalars *, cudaStream_t);
template int fcg_step<float>(const double *, int, float *, float *, double *, double *, const double *, double *,
                             double *, double *, double *, Dims2, double *, FcgScalars *, cudaStream_t);

}  // namespace cdrgpu
