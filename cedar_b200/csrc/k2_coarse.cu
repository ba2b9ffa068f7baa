// k2_coarse.cu -- the coarse end of a 2D V-cycle in one kernel launch.
//
// Below ~64x64 points a level's kernels are latency bound: each launch of the
// point, line and transfer kernels costs several microseconds however little
// work it has.  This kernel runs the whole sub-cycle from a coarse level down to
// the coarsest and back (cycle::vcycle::ncycle_helper,
// include/cedar/cycle/vcycle.h:57-115: pre-smoothing, residual, restriction,
// zero coarse iterate, ..., banded Cholesky, ..., interpolate-add,
// post-smoothing) with one CTA per problem and a barrier between steps.  Every
// point formula is the shared helper the separate kernels use (k2_point.cuh),
// and the line solves run DPTTS2's sequential substitutions on rows staged in
// shared memory (as the exact line kernels do), so the result is the one the
// separate kernels give in CDR_LINES_EXACT mode.
//
// Each level visit copies the level's operator, smoother factors, b, x and r
// into shared memory (compact rows), runs every smoothing phase there and
// writes x and r back: the barrier-separated phases then wait on shared memory
// instead of L2 (a first version that worked on L2 took 508 us per cycle for
// levels 64^2 .. 4^2, against ~300 us for the separate launches).  Levels of at
// most 32^2 are fused by default: FP32+IR and FP64 solves of the 2047^2 line-xy
// problem are 4-5 % faster than with separate launches; fusing from 64^2 is
// slower in FP32 (its 64-point sequential line solves dominate).
#include <algorithm>

#include "k2_point.cuh"
#include "kernels2d.cuh"

namespace cdrgpu {

constexpr int CC_THREADS = 1024;

// r = b - A x on the level (all interior points)
template <typename T, int NS>
__device__ void cc_residual(const CoarseLevel<T> &L)
{
	const Dims2 d{L.nx, L.ny, L.pitch};
	const int n = L.nx * L.ny;
	for (int e = threadIdx.x; e < n; e += CC_THREADS) {
		const size_t k = d.at(e % L.nx + 1, e / L.nx + 1);
		L.r[k] = resid_at<T, NS>(L.so, d.plane(), L.x, L.b, k, L.pitch);
	}
}

// coarse b = P^T r_fine
template <typename T>
__device__ void cc_restrict(const CoarseLevel<T> &F, const CoarseLevel<T> &C)
{
	const Dims2 f{F.nx, F.ny, F.pitch}, c{C.nx, C.ny, C.pitch};
	const int n = C.nx * C.ny;
	for (int e = threadIdx.x; e < n; e += CC_THREADS) restrict_at<T>(C.ci, F.r, C.b, f, c, e % C.nx + 1, e / C.nx + 1);
}

// x_fine += P x_coarse + r/c on the fine-only points
template <typename T>
__device__ void cc_interp(const CoarseLevel<T> &F, const CoarseLevel<T> &C)
{
	const Dims2 f{F.nx, F.ny, F.pitch}, c{C.nx, C.ny, C.pitch};
	const int mx = F.nx / 2 + 1, n = mx * (F.ny / 2 + 1);
	for (int e = threadIdx.x; e < n; e += CC_THREADS) interp_at<T>(C.ci, C.x, F.r, F.so, F.x, f, c, e % mx + 1, e / mx + 1);
}

// the whole coarse iterate, ghosts included, to zero (the cycle's memset)
template <typename T>
__device__ void cc_zero(const CoarseLevel<T> &L)
{
	const size_t n = (size_t)L.pitch * (L.ny + 2);
	for (size_t e = threadIdx.x; e < n; e += CC_THREADS) L.x[e] = T(0);
}

// one Gauss-Seidel sweep, colours in relax_point_2d's order
template <typename T, int NS>
__device__ void cc_gs(const CoarseLevel<T> &L, int updown)
{
	const Dims2 d{L.nx, L.ny, L.pitch};
	const size_t ps = d.plane();
	if (NS == 5) {
		const int order[4][2] = {{1, 1}, {1, 0}, {0, 1}, {0, 0}};  // (j odd?, i odd?)
		const int mx = (L.nx + 1) / 2, my = (L.ny + 1) / 2;
		for (int c = 0; c < 4; ++c) {
			const int o = updown == CDR_DOWN ? c : 3 - c;
			for (int e = threadIdx.x; e < mx * my; e += CC_THREADS) {
				const int i = (order[o][1] ? 1 : 2) + 2 * (e % mx), j = (order[o][0] ? 1 : 2) + 2 * (e / mx);
				if (i <= L.nx && j <= L.ny) gs_at<T, 5>(L.so, ps, L.x, L.b, L.sor, d.at(i, j), L.pitch);
			}
			__syncthreads();
		}
	} else {
		const int mx = (L.nx + 1) / 2;
		for (int c = 0; c < 2; ++c) {
			const int par = updown == CDR_DOWN ? c : 1 - c;
			for (int e = threadIdx.x; e < mx * L.ny; e += CC_THREADS) {
				const int j = e / mx + 1;
				const int i = (((1 + j) & 1) == par ? 1 : 2) + 2 * (e % mx);
				if (i <= L.nx) gs_at<T, 3>(L.so, ps, L.x, L.b, L.sor, d.at(i, j), L.pitch);
			}
			__syncthreads();
		}
	}
}

// One zebra line sweep (both colours, relax_lines_2d's order).  Each colour:
// the right-hand sides of its lines are formed by all threads into sm, then the
// substitutions run with the level's (shared-memory) pivots and multipliers:
// DPTTS2's sequential order in FP64 (one thread per line), affine-map scans over
// the lanes of one warp per line in FP32 (the preconditioner has no bitwise
// target; the separate FP32 kernels scan too).
template <typename T, int NS, int DIR>
__device__ void cc_lines(const CoarseLevel<T> &L, int updown, T *sm)
{
	const Dims2 d{L.nx, L.ny, L.pitch};
	const size_t ps = d.plane();
	const int n = DIR == CDR_DIR_X ? L.nx : L.ny;    // line length
	const int nl = DIR == CDR_DIR_X ? L.ny : L.nx;   // lines
	const T *fac = DIR == CDR_DIR_X ? L.sor : L.sory;
	const size_t eplane = DIR == CDR_DIR_X ? ps : (size_t)L.tpitch * (L.nx + 2);
	const int firsts[2] = {updown == CDR_DOWN ? 2 : 1, updown == CDR_DOWN ? 1 : 2};
	for (int c = 0; c < 2; ++c) {
		const int first = firsts[c];
		const int ml = first > nl ? 0 : (nl - first) / 2 + 1;  // lines of this colour
		T *R = sm;
		for (int e = threadIdx.x; e < ml * n; e += CC_THREADS) {
			const int g = e / n, m = e - g * n, lc = first + 2 * g;
			const size_t k = DIR == CDR_DIR_X ? d.at(m + 1, lc) : d.at(lc, m + 1);
			R[e] = line_rhs<T, NS, DIR>(L.so, ps, L.x, L.b, k, L.pitch);
		}
		__syncthreads();
		if constexpr (sizeof(T) == 8) {
			// FP64: DPTTS2's sequential substitutions, one thread per line
			if (threadIdx.x < ml) {
				const int lc = first + 2 * threadIdx.x;
				// factors of position p at dd[p], ee[p] (position 1 is r[0])
				const T *dd = fac + (DIR == CDR_DIR_X ? (size_t)lc * L.pitch : (size_t)lc * L.tpitch);
				const T *ee = dd + eplane;
				T *r = R + threadIdx.x * n;
				T y = r[0];
				for (int m = 1; m < n; ++m) {
					y = r[m] - y * ee[m + 1];
					r[m] = y;
				}
				T xv = pivot_div(y, dd[n]);
				r[n - 1] = xv;
				for (int m = n - 2; m >= 0; --m) {
					xv = pivot_div(r[m], dd[m + 1]) - xv * ee[m + 2];
					r[m] = xv;
				}
			}
		} else {
			// FP32: one warp per line, each lane a chunk of consecutive positions;
			// both substitutions as affine-map scans over the lanes (shuffles)
			const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
			const int cs = (n + 31) / 32;  // chunk length
			for (int g = warp; g < ml; g += CC_THREADS / 32) {
				const int lc = first + 2 * g;
				const T *dd = fac + (DIR == CDR_DIR_X ? (size_t)lc * L.pitch : (size_t)lc * L.tpitch);
				const T *ee = dd + eplane;
				T *r = R + g * n;
				const int lo = lane * cs < n ? lane * cs : n, hi = lo + cs < n ? lo + cs : n;
				// forward y(m) = r(m) - y(m-1) E(m+1), y(0) = r(0)
				T A = T(1), B = T(0);
				for (int m = lo; m < hi; ++m) {
					const T a = m == 0 ? T(0) : -ee[m + 1];
					B = madd(a, B, r[m]);
					A = a * A;
				}
				for (int off = 1; off < 32; off <<= 1) {
					const T a2 = __shfl_up_sync(0xffffffffu, A, off), b2 = __shfl_up_sync(0xffffffffu, B, off);
					if (lane >= off) { B = madd(A, b2, B); A = A * a2; }
				}
				T y = __shfl_up_sync(0xffffffffu, B, 1);
				if (lane == 0) y = T(0);
				for (int m = lo; m < hi; ++m) {
					y = m == 0 ? r[0] : madd(-y, ee[m + 1], r[m]);
					r[m] = pivot_div(y, dd[m + 1]);
				}
				__syncwarp();
				// backward x(m) = y(m)/D(m+1) - x(m+1) E(m+2), x(n-1) = y(n-1)/D(n)
				A = T(1);
				B = T(0);
				for (int m = hi - 1; m >= lo; --m) {
					const T a = m == n - 1 ? T(0) : -ee[m + 2];
					B = madd(a, B, r[m]);
					A = a * A;
				}
				for (int off = 1; off < 32; off <<= 1) {
					const T a2 = __shfl_down_sync(0xffffffffu, A, off), b2 = __shfl_down_sync(0xffffffffu, B, off);
					if (lane + off < 32) { B = madd(A, b2, B); A = A * a2; }
				}
				T xv = __shfl_down_sync(0xffffffffu, B, 1);
				if (lane == 31) xv = T(0);
				for (int m = hi - 1; m >= lo; --m) {
					xv = m == n - 1 ? r[m] : madd(-xv, ee[m + 2], r[m]);
					r[m] = xv;
				}
				__syncwarp();
			}
		}
		__syncthreads();
		for (int e = threadIdx.x; e < ml * n; e += CC_THREADS) {
			const int g = e / n, m = e - g * n, lc = first + 2 * g;
			L.x[DIR == CDR_DIR_X ? d.at(m + 1, lc) : d.at(lc, m + 1)] = R[e];
		}
		__syncthreads();
	}
}

template <typename T, int NS>
__device__ void cc_smooth(const CoarseCycle<T> &cc, const CoarseLevel<T> &L, int updown, T *sm)
{
	const int nrel = updown == CDR_DOWN ? cc.npre : cc.npost;
	for (int it = 0; it < nrel; ++it) {
		switch (cc.relax) {
		case CDR_RELAX_POINT: cc_gs<T, NS>(L, updown); break;
		case CDR_RELAX_LINE_X: cc_lines<T, NS, CDR_DIR_X>(L, updown, sm); break;
		case CDR_RELAX_LINE_Y: cc_lines<T, NS, CDR_DIR_Y>(L, updown, sm); break;
		default:
			if (updown == CDR_DOWN) {
				cc_lines<T, NS, CDR_DIR_X>(L, updown, sm);
				cc_lines<T, NS, CDR_DIR_Y>(L, updown, sm);
			} else {
				cc_lines<T, NS, CDR_DIR_Y>(L, updown, sm);
				cc_lines<T, NS, CDR_DIR_X>(L, updown, sm);
			}
		}
	}
}

// BMG2_SymStd_SOLVE_cg with DPBTRS('U') on the coarsest level: the factor and
// the right-hand side staged in shared memory, substitutions by one thread
// (k_cg_solve's operations)
template <typename T>
__device__ void cc_cg(const double *__restrict__ ab, const CoarseLevel<T> &L, double *xs)
{
	const Dims2 d{L.nx, L.ny, L.pitch};
	const int ldab = L.nx + 2, kd = L.nx + 1, n = L.nx * L.ny;
	double *abs = xs + n;
	for (int e = threadIdx.x; e < ldab * n; e += CC_THREADS) abs[e] = ab[e];
	for (int e = threadIdx.x; e < n; e += CC_THREADS) xs[e] = (double)L.b[d.at(e % L.nx + 1, e / L.nx + 1)];
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int j = 0; j < n; ++j) {
			double temp = xs[j];
			const int i0 = j - kd > 0 ? j - kd : 0;
			for (int i = i0; i < j; ++i) temp = temp - abs[(size_t)j * ldab + kd + i - j] * xs[i];
			xs[j] = temp / abs[(size_t)j * ldab + kd];
		}
		for (int j = n - 1; j >= 0; --j) {
			if (xs[j] != 0.0) {
				xs[j] = xs[j] / abs[(size_t)j * ldab + kd];
				const double temp = xs[j];
				const int i1 = j - kd > 0 ? j - kd : 0;
				for (int i = j - 1; i >= i1; --i) xs[i] = xs[i] - temp * abs[(size_t)j * ldab + kd + i - j];
			}
		}
	}
	__syncthreads();
	for (int e = threadIdx.x; e < n; e += CC_THREADS) L.x[d.at(e % L.nx + 1, e / L.nx + 1)] = (T)xs[e];
}

// Problem blockIdx.x of a batch: every array of every level moves by that
// problem's offset (problems back to back, problem step bstep).
template <typename T>
__device__ CoarseLevel<T> cc_level(const CoarseCycle<T> &cc, int l)
{
	CoarseLevel<T> L = cc.lv[l];
	const size_t p = (size_t)blockIdx.x * cc.bstep, pl = (size_t)L.pitch * (L.ny + 2);
	L.so += p * L.ns * pl;
	L.x += p * pl;
	L.b += p * pl;
	L.r += p * pl;
	if (L.sor) L.sor += p * 2 * pl;
	if (L.sory) L.sory += p * 2 * (size_t)L.tpitch * (L.nx + 2);
	if (L.ci) L.ci += p * 8 * pl;
	return L;
}

// Shared-memory copy of a level for one visit: its operator, smoother factors,
// b, x and r with compact rows (pitch nx+2; y-line factors tpitch ny+2).
template <typename T>
__device__ CoarseLevel<T> cc_view(const CoarseLevel<T> &G, int relax, T *base)
{
	CoarseLevel<T> S = G;
	S.pitch = G.nx + 2;
	S.tpitch = G.ny + 2;
	const size_t pl = (size_t)(G.nx + 2) * (G.ny + 2);
	T *p = base;
	S.so = p;
	p += G.ns * pl;
	if (relax == CDR_RELAX_POINT) { S.sor = p; p += pl; }
	else if (relax != CDR_RELAX_LINE_Y) { S.sor = p; p += 2 * pl; }
	else S.sor = nullptr;
	if (relax == CDR_RELAX_LINE_Y || relax == CDR_RELAX_LINE_XY) { S.sory = p; p += 2 * pl; }
	else S.sory = nullptr;
	S.b = p; p += pl;
	S.x = p; p += pl;
	S.r = p;
	S.ci = nullptr;
	return S;
}

// copy nplanes planes of (ny+2) rows of nx+2 elements between pitches
template <typename T>
__device__ void cc_copy(const T *__restrict__ src, int sp, size_t splane, T *__restrict__ dst, int dp, size_t dplane,
                        int rowlen, int rows, int nplanes)
{
	const int per = rowlen * rows;
	for (int e = threadIdx.x; e < per * nplanes; e += CC_THREADS) {
		const int q = e / per, rem = e - q * per, j = rem / rowlen, i = rem - j * rowlen;
		dst[(size_t)q * dplane + (size_t)j * dp + i] = src[(size_t)q * splane + (size_t)j * sp + i];
	}
}

template <typename T>
__device__ void cc_stage(const CoarseLevel<T> &G, const CoarseLevel<T> &S, int relax, bool with_r)
{
	const size_t gpl = (size_t)G.pitch * (G.ny + 2), spl = (size_t)S.pitch * (S.ny + 2);
	const int ii = G.nx + 2, jj = G.ny + 2;
	cc_copy<T>(G.so, G.pitch, gpl, const_cast<T *>(S.so), S.pitch, spl, ii, jj, G.ns);
	if (S.sor) cc_copy<T>(G.sor, G.pitch, gpl, const_cast<T *>(S.sor), S.pitch, spl, ii, jj, relax == CDR_RELAX_POINT ? 1 : 2);
	if (S.sory)  // transposed: nx+2 rows of ny+2 elements
		cc_copy<T>(G.sory, G.tpitch, (size_t)G.tpitch * ii, const_cast<T *>(S.sory), S.tpitch, (size_t)S.tpitch * ii, jj,
		           ii, 2);
	cc_copy<T>(G.b, G.pitch, gpl, S.b, S.pitch, spl, ii, jj, 1);
	cc_copy<T>(G.x, G.pitch, gpl, S.x, S.pitch, spl, ii, jj, 1);
	if (with_r) cc_copy<T>(G.r, G.pitch, gpl, S.r, S.pitch, spl, ii, jj, 1);
	__syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(CC_THREADS) k_coarse_cycle(CoarseCycle<T> cc)
{
	extern __shared__ __align__(16) unsigned char cc_smem[];
	T *lvl = reinterpret_cast<T *>(cc_smem);  // the visited level
	T *sm = lvl + cc.level_elems;              // line right-hand sides
	const int nl = cc.nl;
	for (int l = 0; l + 1 < nl; ++l) {
		const CoarseLevel<T> G = cc_level(cc, l), C = cc_level(cc, l + 1);
		const CoarseLevel<T> F = cc_view(G, cc.relax, lvl);
		// r too: restriction reads its ghost layer (zero) for odd edges
		cc_stage(G, F, cc.relax, true);
		if (F.ns == 5) cc_smooth<T, 5>(cc, F, CDR_DOWN, sm);
		else cc_smooth<T, 3>(cc, F, CDR_DOWN, sm);
		if (F.ns == 5) cc_residual<T, 5>(F);
		else cc_residual<T, 3>(F);
		__syncthreads();
		cc_restrict<T>(F, C);
		cc_zero<T>(C);
		// x and r of this level are needed again on the way up
		const size_t gpl = (size_t)G.pitch * (G.ny + 2), spl = (size_t)F.pitch * (F.ny + 2);
		cc_copy<T>(F.x, F.pitch, spl, G.x, G.pitch, gpl, G.nx + 2, G.ny + 2, 1);
		cc_copy<T>(F.r, F.pitch, spl, G.r, G.pitch, gpl, G.nx + 2, G.ny + 2, 1);
		__syncthreads();
	}
	{
		const CoarseLevel<T> Cg = cc_level(cc, nl - 1);
		const size_t nab = (size_t)(Cg.nx + 2) * Cg.nx * Cg.ny;
		cc_cg<T>(cc.abd + (size_t)blockIdx.x * cc.bstep * nab, Cg, reinterpret_cast<double *>(cc_smem));
		__syncthreads();
	}
	for (int l = nl - 2; l >= 0; --l) {
		const CoarseLevel<T> G = cc_level(cc, l), C = cc_level(cc, l + 1);
		const CoarseLevel<T> F = cc_view(G, cc.relax, lvl);
		cc_stage(G, F, cc.relax, true);
		cc_interp<T>(F, C);
		__syncthreads();
		if (F.ns == 5) cc_smooth<T, 5>(cc, F, CDR_UP, sm);
		else cc_smooth<T, 3>(cc, F, CDR_UP, sm);
		__syncthreads();
		cc_copy<T>(F.x, F.pitch, (size_t)F.pitch * (F.ny + 2), G.x, G.pitch, (size_t)G.pitch * (G.ny + 2), G.nx + 2,
		           G.ny + 2, 1);
		__syncthreads();
	}
}

// Elements of the shared copy of one level (cc_view's layout)
template <typename T>
size_t cc_level_elems(const CoarseLevel<T> &L, int relax)
{
	const size_t pl = (size_t)(L.nx + 2) * (L.ny + 2);
	size_t planes = L.ns + 3;  // so, b, x, r
	if (relax == CDR_RELAX_POINT) planes += 1;
	else if (relax != CDR_RELAX_LINE_Y) planes += 2;
	if (relax == CDR_RELAX_LINE_Y || relax == CDR_RELAX_LINE_XY) planes += 2;
	return planes * pl;
}

template <typename T>
size_t coarse_cycle_smem(const CoarseCycle<T> &cc, size_t *level_elems)
{
	size_t lvl = 0, lines = 0;
	for (int l = 0; l + 1 < cc.nl; ++l) {
		const CoarseLevel<T> &L = cc.lv[l];
		lvl = std::max(lvl, cc_level_elems(L, cc.relax));
		lines = std::max(lines, std::max((size_t)((L.ny + 1) / 2) * L.nx, (size_t)((L.nx + 1) / 2) * L.ny));
	}
	lvl = (lvl + 1) / 2 * 2;  // keep the line buffer 8-byte aligned
	*level_elems = lvl;
	const CoarseLevel<T> &Cg = cc.lv[cc.nl - 1];
	const size_t n = (size_t)Cg.nx * Cg.ny;
	return std::max((lvl + lines) * sizeof(T), (n + (size_t)(Cg.nx + 2) * n) * sizeof(double));
}

// Shared memory a fused coarse cycle from level descriptor lv[0..nl) needs
template <typename T>
size_t coarse_cycle_bytes(const CoarseCycle<T> &cc)
{
	size_t e;
	return coarse_cycle_smem(cc, &e);
}
template size_t coarse_cycle_bytes<double>(const CoarseCycle<double> &);
template size_t coarse_cycle_bytes<float>(const CoarseCycle<float> &);

template <typename T>
int coarse_cycle(const CoarseCycle<T> &cc, int nproblems, cudaStream_t st)
{
	if (cc.nl < 1 || cc.nl > kMaxCoarseLevels) {
		set_error(CDR_ERR_DIM, "fused coarse cycle over %d levels", cc.nl);
		return CDR_ERR_DIM;
	}
	CoarseCycle<T> c2 = cc;
	size_t lvl = 0;
	const size_t smem = coarse_cycle_smem(c2, &lvl);
	c2.level_elems = lvl;
	if (smem > kCoarseSmemMax) {
		set_error(CDR_ERR_DIM, "fused coarse cycle needs %zu bytes of shared memory", smem);
		return CDR_ERR_DIM;
	}
	k_coarse_cycle<T><<<nproblems, CC_THREADS, smem, st>>>(c2);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int coarse_cycle<double>(const CoarseCycle<double> &, int, cudaStream_t);

// Opt the fused kernels into the large shared-memory carve-out (once per
// process, before any graph capture: called from lines_prepare).
int coarse_prepare()
{
	CDR_CUDA_TRY(cudaFuncSetAttribute(k_coarse_cycle<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarseSmemMax));
	CDR_CUDA_TRY(cudaFuncSetAttribute(k_coarse_cycle<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarseSmemMax));
	return CDR_OK;
}
template int coarse_cycle<float>(const CoarseCycle<float> &, int, cudaStream_t);

}  // namespace cdrgpu
