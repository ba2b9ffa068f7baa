// k2_krylov.cu -- flexible conjugate gradients (FCG(1)) around the 2D cycle.
//
// No counterpart in the reference: its solve (multilevel::solve,
// include/cedar/multilevel.h:278-298) repeats the cycle on the current iterate.
// Here the cycle (FP64, or FP32 inside FP64 recurrences) is the preconditioner
// z = M r of Notay's flexible CG:
//   beta = -(z . q_prev) / (p_prev . q_prev)      (0 on the first iteration)
//   p = z + beta p_prev,  q = A p,  alpha = (p . r) / (p . q)
//   x += alpha p,  r = b - A x  (or r -= alpha q)
// By default the residual is formed anew from x every iteration: on
// high-contrast operators the updated residual r -= alpha q drifts from b - A x
// by orders of magnitude before it converges, while the formed one stays at
// the FP64 floor eps |A||x|.  With a replacement period m > 1 the solver forms
// it every m-th iteration and updates it in between (k_fcg_update_rec, one
// pass over the operator fewer).  The products read the ghost ring as the residual
// kernels do.  All of it is FP64.  Three kernels per iteration, each
// ending in a deterministic grid reduction: every block writes its partial
// sums, and the last block to finish (an atomic ticket) adds the partials in
// block order and updates the device scalars, so the host only reads |r|.
// p and x are double-buffered (device-side parity): A p and A x read neighbours.
#include "k2_point.cuh"
#include "kernels2d.cuh"

namespace cdrgpu {

namespace {

constexpr int FR = 4;  // rows per thread: each CTA covers 32 x 32 points, four independent rows in flight

// Sum the NSUM per-thread values over the grid; the last block to finish adds
// the blocks' partials in block order and calls fin(totals).
template <int NSUM, typename F>
__device__ __forceinline__ void grid_sums(const double (&acc)[NSUM], double *__restrict__ partial,
                                          unsigned *__restrict__ ticket, F fin)
{
	__shared__ double sh[NSUM][TX * TY / 32];
	__shared__ bool last;
	const int tid = threadIdx.y * blockDim.x + threadIdx.x;
	const int nb = gridDim.x * gridDim.y, bid = blockIdx.y * gridDim.x + blockIdx.x;
	double tot[NSUM];
#pragma unroll
	for (int s = 0; s < NSUM; ++s) tot[s] = block_sum<TX * TY / 32>(acc[s], sh[s]);
	if (tid == 0) {
#pragma unroll
		for (int s = 0; s < NSUM; ++s) partial[(size_t)s * nb + bid] = tot[s];
		__threadfence();
		last = atomicAdd(ticket, 1u) == (unsigned)nb - 1u;
	}
	__syncthreads();
	if (!last) return;
	__threadfence();
	double v[NSUM];
#pragma unroll
	for (int s = 0; s < NSUM; ++s) {
		double a = 0.0;
		for (int b = tid; b < nb; b += TX * TY) a += __ldcg(partial + (size_t)s * nb + b);
		v[s] = block_sum<TX * TY / 32>(a, sh[s]);
	}
	if (tid == 0) {
		fin(v);
		*ticket = 0u;
	}
}

// point (i, j) of row `row` of this thread; false outside the interior
__device__ __forceinline__ bool fcg_point(const Dims2 &d, int row, int &i, int &j)
{
	i = blockIdx.x * TX + threadIdx.x + 1;
	j = blockIdx.y * (TY * FR) + threadIdx.y + 1 + row * TY;
	return i <= d.nx && j <= d.ny;
}

// z = 0 at interior point (i, j) and, on the edges, at its ghost neighbours
// (skipped when z is null: a cycle whose first sweep starts from zero without
// reading its iterate)
template <typename TZ>
__device__ __forceinline__ void zero_z(TZ *__restrict__ z, size_t k, int i, int j, const Dims2 &d)
{
	const int pitch = d.pitch;
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

// The CTA's 32 x 32 points plus a one-point halo of u(k) = f(k), formed once
// per point into shared memory (0 beyond the ghost ring); the stencil products
// read their neighbours from there.
constexpr int HT = TX + 2;  // halo tile edge (TY * FR == TX)
static_assert(TY * FR == TX, "square tiles");

template <typename F>
__device__ __forceinline__ void fill_halo(double (&u)[HT][HT], const Dims2 &d, F f)
{
	const int i0 = blockIdx.x * TX, j0 = blockIdx.y * (TY * FR);  // halo origin (column i0, row j0)
	for (int e = threadIdx.y * TX + threadIdx.x; e < HT * HT; e += TX * TY) {
		const int li = e % HT, lj = e / HT, gi = i0 + li, gj = j0 + lj;
		u[lj][li] = gi <= d.nx + 1 && gj <= d.ny + 1 ? f((size_t)gj * d.pitch + gi) : 0.0;
	}
	__syncthreads();
}

// The preconditioner's output at k: z, or (SPLIT) the sum of an FP64 part z
// and an FP32 part zf (the FP32 cycle's fine level with a widened iterate:
// the interpolated iterate and the post-smoothing correction)
template <typename TZ, bool SPLIT>
__device__ __forceinline__ double zval(const TZ *__restrict__ z, const float *__restrict__ zf, size_t k)
{
	if constexpr (SPLIT) return (double)z[k] + (double)zf[k];
	else return (double)z[k];
}

// beta from z . q_prev
template <typename TZ, bool SPLIT>
__global__ void __launch_bounds__(TX *TY) k_fcg_beta(const TZ *__restrict__ z, const float *__restrict__ zf,
                                                     const double *__restrict__ q, Dims2 d,
                                                     double *__restrict__ partial, FcgScalars *S)
{
	double acc[1] = {0.0};
	if (!S->first) {
		int i, j;
#pragma unroll
		for (int row = 0; row < FR; ++row)
			if (fcg_point(d, row, i, j)) {
				const size_t k = d.at(i, j);
				acc[0] += zval<TZ, SPLIT>(z, zf, k) * q[k];
			}
	}
	grid_sums<1>(acc, partial, &S->ticket[0], [&](const double *v) {
		S->zq = v[0];
		S->beta = S->first ? 0.0 : -v[0] / S->pq;
	});
}

// p = z + beta p_prev (formed on the fly at the neighbours), q = A p, p . q and
// p . r.  The products read the ghost ring as the residual kernels do (the
// operator's couplings into it are zero); p is written on the interior only.
template <typename TZ, int NS, bool SPLIT>
__global__ void __launch_bounds__(TX *TY) k_fcg_dir(const double *__restrict__ so, const TZ *__restrict__ z,
                                                    const float *__restrict__ zf,
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
	const double *c = so, *w = so + ps, *s = so + 2 * ps, *sw = so + 3 * ps, *nw = so + 4 * ps;
	__shared__ double pt[HT][HT];
	fill_halo(pt, d, [&](size_t k) -> double { return madd(beta, pold[k], zval<TZ, SPLIT>(z, zf, k)); });
	double acc[2] = {0.0, 0.0};
	int i, j;
#pragma unroll
	for (int row = 0; row < FR; ++row)
		if (fcg_point(d, row, i, j)) {
			const size_t k = (size_t)j * pitch + i;
			const int li = threadIdx.x + 1, lj = threadIdx.y + 1 + row * TY;
			auto P = [&](int di, int dj) -> double { return pt[lj + dj][li + di]; };
			const double pc = P(0, 0);
			double nb = w[k] * P(-1, 0) + w[k + 1] * P(1, 0) + s[k] * P(0, -1) + s[k + pitch] * P(0, 1);
			if (NS == 5)
				nb += sw[k] * P(-1, -1) + nw[k + 1] * P(1, -1) + nw[k + pitch] * P(-1, 1) + sw[k + pitch + 1] * P(1, 1);
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
	const double *c = so, *w = so + ps, *s = so + 2 * ps, *sw = so + 3 * ps, *nw = so + 4 * ps;
	__shared__ double xt[HT][HT];
	fill_halo(xt, d, [&](size_t k) -> double { return madd(alpha, pnew[k], xold[k]); });
	double acc[1] = {0.0};
	int i, j;
#pragma unroll
	for (int row = 0; row < FR; ++row)
		if (fcg_point(d, row, i, j)) {
			const size_t k = (size_t)j * pitch + i;
			const int li = threadIdx.x + 1, lj = threadIdx.y + 1 + row * TY;
			auto X = [&](int di, int dj) -> double { return xt[lj + dj][li + di]; };
			const double xc = X(0, 0);
			double nb = w[k] * X(-1, 0) + w[k + 1] * X(1, 0) + s[k] * X(0, -1) + s[k + pitch] * X(0, 1);
			if (NS == 5)
				nb += sw[k] * X(-1, -1) + nw[k + 1] * X(1, -1) + nw[k + pitch] * X(-1, 1) + sw[k + pitch + 1] * X(1, 1);
			const double rk = bb[k] + nb - c[k] * xc;
			xnew[k] = xc;
			r[k] = rk;
			acc[0] += rk * rk;
			rin[k] = (TZ)rk;
			if (z) zero_z(z, k, i, j, d);
		}
	grid_sums<1>(acc, partial, &S->ticket[2], [&](const double *v) {
		S->rr = v[0];
		S->iter += 1;
		S->first = 0;
	});
}

// The same step with the residual updated instead of formed: x_new = x + alpha
// p, r -= alpha q (q = A p of this iteration; no pass over the operator),
// |r|^2, the preconditioner input and z = 0.
template <typename TZ>
__global__ void __launch_bounds__(TX *TY) k_fcg_update_rec(double *__restrict__ x0, double *__restrict__ x1,
                                                           double *__restrict__ r, const double *__restrict__ p0,
                                                           const double *__restrict__ p1,
                                                           const double *__restrict__ q, TZ *__restrict__ rin,
                                                           TZ *__restrict__ z, Dims2 d, double *__restrict__ partial,
                                                           FcgScalars *S)
{
	const int pitch = d.pitch;
	const bool odd = S->iter & 1;
	const double *__restrict__ pnew = odd ? p0 : p1;
	const double *__restrict__ xold = odd ? x1 : x0;
	double *__restrict__ xnew = odd ? x0 : x1;
	const double alpha = S->alpha;
	double acc[1] = {0.0};
	int i, j;
#pragma unroll
	for (int row = 0; row < FR; ++row)
		if (fcg_point(d, row, i, j)) {
			const size_t k = (size_t)j * pitch + i;
			xnew[k] = madd(alpha, pnew[k], xold[k]);
			const double rk = madd(-alpha, q[k], r[k]);
			r[k] = rk;
			acc[0] += rk * rk;
			rin[k] = (TZ)rk;
			if (z) zero_z(z, k, i, j, d);
		}
	grid_sums<1>(acc, partial, &S->ticket[2], [&](const double *v) {
		S->rr = v[0];
		S->iter += 1;
		S->first = 0;
	});
}

// Start from r: the preconditioner input, a zero z and (restart) first = 1,
// iter = 0; without restart the recurrences go on from the new r.
template <typename TZ>
__global__ void __launch_bounds__(TX *TY) k_fcg_load(const double *__restrict__ r, TZ *__restrict__ rin,
                                                     TZ *__restrict__ z, Dims2 d, FcgScalars *S, int restart)
{
	const int i = blockIdx.x * TX + threadIdx.x, j = blockIdx.y * TY + threadIdx.y;
	if (i > d.nx + 1 || j > d.ny + 1) return;
	const size_t k = d.at(i, j);
	const bool in = i >= 1 && i <= d.nx && j >= 1 && j <= d.ny;
	rin[k] = in ? (TZ)r[k] : TZ(0);
	z[k] = TZ(0);
	if (restart && i == 0 && j == 0) {
		S->first = 1;
		S->iter = 0;
	}
}

}  // namespace

template <typename TZ>
int fcg_load(const double *r, TZ *rin, TZ *z, Dims2 d, FcgScalars *S, cudaStream_t st, bool restart)
{
	k_fcg_load<TZ><<<dim3(ceil_div(d.nx + 2, TX), ceil_div(d.ny + 2, TY)), dim3(TX, TY), 0, st>>>(r, rin, z, d, S,
	                                                                                         restart ? 1 : 0);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int fcg_load<double>(const double *, double *, double *, Dims2, FcgScalars *, cudaStream_t, bool);
template int fcg_load<float>(const double *, float *, float *, Dims2, FcgScalars *, cudaStream_t, bool);

size_t fcg_scratch_doubles(Dims2 d) { return 2 * (size_t)ceil_div(d.nx, TX) * ceil_div(d.ny, TY * FR); }

template <typename TZ, typename TR>
int fcg_step(const double *so, int ns, const TZ *z, const float *zf, TR *rin, TR *zz, double *x0, double *x1,
             const double *b, double *r, double *p0, double *p1, double *q, Dims2 d, double *partial, FcgScalars *S,
             cudaStream_t st, bool formed)
{
	const dim3 nb(ceil_div(d.nx, TX), ceil_div(d.ny, TY * FR)), blk(TX, TY);
	if (zf) {
		k_fcg_beta<TZ, true><<<nb, blk, 0, st>>>(z, zf, q, d, partial, S);
		CDR_LAUNCH_CHECK();
		if (ns == 5) k_fcg_dir<TZ, 5, true><<<nb, blk, 0, st>>>(so, z, zf, p0, p1, q, r, d, partial, S);
		else k_fcg_dir<TZ, 3, true><<<nb, blk, 0, st>>>(so, z, zf, p0, p1, q, r, d, partial, S);
	} else {
		k_fcg_beta<TZ, false><<<nb, blk, 0, st>>>(z, nullptr, q, d, partial, S);
		CDR_LAUNCH_CHECK();
		if (ns == 5) k_fcg_dir<TZ, 5, false><<<nb, blk, 0, st>>>(so, z, nullptr, p0, p1, q, r, d, partial, S);
		else k_fcg_dir<TZ, 3, false><<<nb, blk, 0, st>>>(so, z, nullptr, p0, p1, q, r, d, partial, S);
	}
	CDR_LAUNCH_CHECK();
	if (!formed) k_fcg_update_rec<TR><<<nb, blk, 0, st>>>(x0, x1, r, p0, p1, q, rin, zz, d, partial, S);
	else if (ns == 5) k_fcg_update<TR, 5><<<nb, blk, 0, st>>>(so, x0, x1, b, r, p0, p1, rin, zz, d, partial, S);
	else k_fcg_update<TR, 3><<<nb, blk, 0, st>>>(so, x0, x1, b, r, p0, p1, rin, zz, d, partial, S);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int fcg_step<double, double>(const double *, int, const double *, const float *, double *, double *,
                                      double *, double *, const double *, double *, double *, double *, double *,
                                      Dims2, double *, FcgScalars *, cudaStream_t, bool);
template int fcg_step<float, float>(const double *, int, const float *, const float *, float *, float *, double *,
                                    double *, const double *, double *, double *, double *, double *, Dims2, double *,
                                    FcgScalars *, cudaStream_t, bool);
template int fcg_step<double, float>(const double *, int, const double *, const float *, float *, float *, double *,
                                     double *, const double *, double *, double *, double *, double *, Dims2,
                                     double *, FcgScalars *, cudaStream_t, bool);

}  // namespace cdrgpu
