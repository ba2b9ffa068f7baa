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
// and in FP64 the line solves run DPTTS2's sequential substitutions, so the
// result is the one the separate kernels give in CDR_LINES_EXACT mode.
//
// All levels of the sub-cycle live in shared memory for the whole launch (with
// compact rows): the operators, smoother factors and interpolation weights are
// staged once at entry, b of the first level is read and its x written back at
// exit, and nothing else touches global memory.  Loops map rows to warps and
// positions to lanes (no per-element division).  Levels of at most 32^2 are
// fused by default (the levels of the 2047^2 hierarchy below 63^2 need 83 KB in
// FP32, 166 KB in FP64; from 63^2 on they would not fit).
#include <algorithm>

#include "k2_point.cuh"
#include "kernels2d.cuh"

namespace cdrgpu {

constexpr int CC_THREADS = 1024;
constexpr int CC_WARPS = CC_THREADS / 32;

// f(i, j) for i in [i0, i1], j in [j0, j1]: rows over the warps, positions over the lanes
template <typename F>
__device__ __forceinline__ void cc_rows(int i0, int i1, int j0, int j1, F f)
{
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	for (int j = j0 + warp; j <= j1; j += CC_WARPS)
		for (int i = i0 + lane; i <= i1; i += 32) f(i, j);
}

// Planes of smoother factors kept for a relaxation type
__host__ __device__ inline int cc_sor_planes(int relax)
{
	return relax == CDR_RELAX_POINT ? 1 : relax == CDR_RELAX_LINE_Y ? 0 : 2;
}
__host__ __device__ inline int cc_sory_planes(int relax)
{
	return relax == CDR_RELAX_LINE_Y || relax == CDR_RELAX_LINE_XY ? 2 : 0;
}

// Elements of level l's shared copy (rows of nx+2): operator, factors, b, x, r
// (the coarsest keeps b and x only) and the interpolation weights of every
// level but the first.
template <typename T>
__host__ __device__ inline size_t cc_elems(const CoarseCycle<T> &cc, int l)
{
	const CoarseLevel<T> &L = cc.lv[l];
	const size_t pl = (size_t)(L.nx + 2) * (L.ny + 2);
	size_t planes = l == cc.nl - 1 ? 2 : L.ns + cc_sor_planes(cc.relax) + cc_sory_planes(cc.relax) + 3;
	if (l > 0) planes += 8;
	return planes * pl;
}

// Global arrays of problem blockIdx.x of a batch: every array of every level
// moves by that problem's offset (problems back to back, problem step bstep).
template <typename T>
__device__ CoarseLevel<T> cc_global(const CoarseCycle<T> &cc, int l)
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

// Shared copy of level l (compact rows: pitch nx+2, y-line factors tpitch ny+2)
template <typename T>
__device__ CoarseLevel<T> cc_view(const CoarseCycle<T> &cc, int l, T *base)
{
	size_t off = 0;
	for (int m = 0; m < l; ++m) off += cc_elems(cc, m);
	const CoarseLevel<T> &G = cc.lv[l];
	CoarseLevel<T> S = G;
	S.pitch = G.nx + 2;
	S.tpitch = G.ny + 2;
	const size_t pl = (size_t)(G.nx + 2) * (G.ny + 2);
	T *p = base + off;
	if (l < cc.nl - 1) {
		S.so = p;
		p += G.ns * pl;
		const int ns1 = cc_sor_planes(cc.relax), ns2 = cc_sory_planes(cc.relax);
		S.sor = ns1 ? p : nullptr;
		p += ns1 * pl;
		S.sory = ns2 ? p : nullptr;
		p += ns2 * pl;
	} else {
		S.so = S.sor = S.sory = nullptr;
	}
	S.b = p;
	p += pl;
	S.x = p;
	p += pl;
	if (l < cc.nl - 1) {
		S.r = p;
		p += pl;
	} else {
		S.r = nullptr;
	}
	S.ci = l > 0 ? p : nullptr;
	return S;
}

// copy nplanes planes of `rows` rows of rowlen elements between pitches
template <typename T>
__device__ void cc_copy(const T *__restrict__ src, int sp, size_t splane, T *__restrict__ dst, int dp, size_t dplane,
                        int rowlen, int rows, int nplanes)
{
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	for (int row = warp; row < rows * nplanes; row += CC_WARPS) {
		const int q = row / rows, j = row - q * rows;
		const T *s = src + (size_t)q * splane + (size_t)j * sp;
		T *d = dst + (size_t)q * dplane + (size_t)j * dp;
		for (int i = lane; i < rowlen; i += 32) d[i] = s[i];
	}
}

// The same copy from global into shared memory by asynchronous copies
// (cp.async, one element each, consecutive threads on consecutive elements of
// the flattened planes and rows): every load of the staging is in flight at
// once instead of one row per warp at a time; cc_stage_wait completes them.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst_smem, const T *src)
{
	const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
	if constexpr (sizeof(T) == 8)
		asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
	else
		asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}

template <typename T>
__device__ void cc_stage(const T *__restrict__ src, int sp, size_t splane, T *__restrict__ dst, int dp,
                         size_t dplane, int rowlen, int rows, int nplanes)
{
	const int per = rowlen * rows, total = per * nplanes;
	// quotients by FP64 reciprocals: (e + 1/2) / d lies at least 1/(2d) from an
	// integer, far beyond the product's rounding error, so the truncation is exact
	const double ip = 1.0 / per, ir = 1.0 / rowlen;
	for (int e = threadIdx.x; e < total; e += CC_THREADS) {
		const int q = (int)((e + 0.5) * ip), rem = e - q * per, j = (int)((rem + 0.5) * ir), i = rem - j * rowlen;
		cp_async_elem(dst + (size_t)q * dplane + (size_t)j * dp + i, src + (size_t)q * splane + (size_t)j * sp + i);
	}
}

__device__ __forceinline__ void cc_stage_wait()
{
	asm volatile("cp.async.wait_all;\n" ::: "memory");
}

template <typename T>
__device__ void cc_fill(T *p, size_t n)
{
	for (size_t e = threadIdx.x; e < n; e += CC_THREADS) p[e] = T(0);
}

// r = b - A x on the level (all interior points)
template <typename T, int NS>
__device__ void cc_residual(const CoarseLevel<T> &L)
{
	const size_t ps = (size_t)L.pitch * (L.ny + 2);
	cc_rows(1, L.nx, 1, L.ny, [&](int i, int j) {
		const size_t k = (size_t)j * L.pitch + i;
		L.r[k] = resid_at<T, NS>(L.so, ps, L.x, L.b, k, L.pitch);
	});
}

// coarse b = P^T r_fine
template <typename T>
__device__ void cc_restrict(const CoarseLevel<T> &F, const CoarseLevel<T> &C)
{
	const Dims2 f{F.nx, F.ny, F.pitch}, c{C.nx, C.ny, C.pitch};
	cc_rows(1, C.nx, 1, C.ny, [&](int ic, int jc) { restrict_at<T>(C.ci, F.r, C.b, f, c, ic, jc); });
}

// x_fine += P x_coarse + r/c on the fine-only points
template <typename T>
__device__ void cc_interp(const CoarseLevel<T> &F, const CoarseLevel<T> &C)
{
	const Dims2 f{F.nx, F.ny, F.pitch}, c{C.nx, C.ny, C.pitch};
	cc_rows(1, F.nx / 2 + 1, 1, F.ny / 2 + 1, [&](int ic, int jc) { interp_at<T>(C.ci, C.x, F.r, F.so, F.x, f, c, ic, jc); });
}

template <typename T, int NS>
__device__ void cc_gs(const CoarseLevel<T> &L, int updown)
{
	const size_t ps = (size_t)L.pitch * (L.ny + 2);
	if (NS == 5) {
		const int order[4][2] = {{1, 1}, {1, 0}, {0, 1}, {0, 0}};  // (j odd?, i odd?)
		for (int c = 0; c < 4; ++c) {
			const int o = updown == CDR_DOWN ? c : 3 - c;
			const int i0 = order[o][1] ? 1 : 2, j0 = order[o][0] ? 1 : 2;
			cc_rows(0, (L.nx - i0) / 2, 0, (L.ny - j0) / 2, [&](int a, int b) {
				gs_at<T, 5>(L.so, ps, L.x, L.b, L.sor, (size_t)(j0 + 2 * b) * L.pitch + i0 + 2 * a, L.pitch);
			});
			__syncthreads();
		}
	} else {
		for (int c = 0; c < 2; ++c) {
			const int par = updown == CDR_DOWN ? c : 1 - c;
			const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
			for (int j = 1 + warp; j <= L.ny; j += CC_WARPS) {
				const int i0 = ((1 + j) & 1) == par ? 1 : 2;
				for (int i = i0 + 2 * lane; i <= L.nx; i += 64)
					gs_at<T, 3>(L.so, ps, L.x, L.b, L.sor, (size_t)j * L.pitch + i, L.pitch);
			}
			__syncthreads();
		}
	}
}

// One zebra line sweep (both colours, relax_lines_2d's order).  Each colour:
// each line's warp forms its right-hand sides into sm (the other warps solve
// lines of the same colour, which this line does not read), then the
// substitutions run with the level's (shared-memory) pivots and multipliers:
// DPTTS2's sequential order in FP64 (one warp per line), affine-map scans over
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
	// x of position m (0-based) of line lc: the solves write their lines' x
	// directly (lines of one colour read only lines of the other)
	auto xat = [&](int lc, int m) -> size_t { return DIR == CDR_DIR_X ? d.at(m + 1, lc) : d.at(lc, m + 1); };
	for (int c = 0; c < 2; ++c) {
		const int first = firsts[c];
		const int ml = first > nl ? 0 : (nl - first) / 2 + 1;  // lines of this colour
		T *R = sm;
		if constexpr (sizeof(T) == 8) {
			// FP64: DPTTS2's sequential substitutions, one warp per line: the
			// line's right-hand sides and the quotients of the backward
			// substitution (which do not depend on its recurrence) by all lanes,
			// the two recurrences by lane 0, four positions per step with their
			// operands loaded ahead of the arithmetic
			const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
			for (int g = warp; g < ml; g += CC_THREADS / 32) {
				const int lc = first + 2 * g;
				// factors of position p at dd[p], ee[p] (position 1 is r[0])
				const T *dd = fac + (DIR == CDR_DIR_X ? (size_t)lc * L.pitch : (size_t)lc * L.tpitch);
				const T *ee = dd + eplane;
				T *r = R + g * n;
				for (int m = lane; m < n; m += 32) r[m] = line_rhs<T, NS, DIR>(L.so, ps, L.x, L.b, xat(lc, m), L.pitch);
				__syncwarp();
				if (lane == 0) {  // y(m) = r(m) - y(m-1) e(m+1), y(0) = r(0)
					T y = r[0];
					int m = 1;
					for (; m + 3 < n; m += 4) {
						const T e0 = ee[m + 1], e1 = ee[m + 2], e2 = ee[m + 3], e3 = ee[m + 4];
						const T a0 = r[m], a1 = r[m + 1], a2 = r[m + 2], a3 = r[m + 3];
						y = a0 - y * e0;
						r[m] = y;
						y = a1 - y * e1;
						r[m + 1] = y;
						y = a2 - y * e2;
						r[m + 2] = y;
						y = a3 - y * e3;
						r[m + 3] = y;
					}
					for (; m < n; ++m) {
						y = r[m] - y * ee[m + 1];
						r[m] = y;
					}
				}
				__syncwarp();
				for (int m = lane; m < n; m += 32) r[m] = pivot_div(r[m], dd[m + 1]);
				__syncwarp();
				if (lane == 0) {  // x(m) = y(m)/d(m+1) - x(m+1) e(m+2), x(n-1) = y(n-1)/d(n)
					T xv = r[n - 1];
					L.x[xat(lc, n - 1)] = xv;
					int m = n - 2;
					for (; m >= 3; m -= 4) {
						const T e0 = ee[m + 2], e1 = ee[m + 1], e2 = ee[m], e3 = ee[m - 1];
						const T q0 = r[m], q1 = r[m - 1], q2 = r[m - 2], q3 = r[m - 3];
						xv = q0 - xv * e0;
						L.x[xat(lc, m)] = xv;
						xv = q1 - xv * e1;
						L.x[xat(lc, m - 1)] = xv;
						xv = q2 - xv * e2;
						L.x[xat(lc, m - 2)] = xv;
						xv = q3 - xv * e3;
						L.x[xat(lc, m - 3)] = xv;
					}
					for (; m >= 0; --m) {
						xv = r[m] - xv * ee[m + 2];
						L.x[xat(lc, m)] = xv;
					}
				}
				__syncwarp();
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
				// the line's right-hand sides by its own warp (the other warps solve
				// lines of the same colour, which this line does not read)
				for (int m = lane; m < n; m += 32) r[m] = line_rhs<T, NS, DIR>(L.so, ps, L.x, L.b, xat(lc, m), L.pitch);
				__syncwarp();
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
					L.x[xat(lc, m)] = xv;
				}
				__syncwarp();
			}
		}
		__syncthreads();  // this colour's lines are written into x
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
		default:  // x then y down, y then x up: one copy of each direction's code
			for (int h = 0; h < 2; ++h) {
				if ((h == 0) == (updown == CDR_DOWN)) cc_lines<T, NS, CDR_DIR_X>(L, updown, sm);
				else cc_lines<T, NS, CDR_DIR_Y>(L, updown, sm);
			}
		}
	}
}

// BMG2_SymStd_SOLVE_cg with DPBTRS('U') on the coarsest level: the right-hand
// side in shared memory (xs) and the factor after it (staged with the levels),
// the substitutions by one thread (k_cg_solve's operations)
template <typename T>
__device__ void cc_cg(const CoarseLevel<T> &L, double *xs)
{
	const int ldab = L.nx + 2, kd = L.nx + 1, n = L.nx * L.ny;
	const double *abs = xs + n;
	cc_rows(1, L.nx, 1, L.ny, [&](int i, int j) { xs[(j - 1) * L.nx + i - 1] = (double)L.b[(size_t)j * L.pitch + i]; });
	__syncthreads();
	if (threadIdx.x == 0) {
		constexpr int KW = 6;
		if (kd < KW) {
			// the same operations in the same order, the band's last KW entries of
			// xs in registers (w[t] = xs[j - KW + t]) and each row's multipliers
			// loaded ahead of the recurrence
			double w[KW];
#pragma unroll
			for (int t = 0; t < KW; ++t) w[t] = 0.0;
			for (int j = 0; j < n; ++j) {
				const double *arow = abs + (size_t)j * ldab + kd - j;  // arow[i]: row j, column i
				double a[KW];
#pragma unroll
				for (int t = 0; t < KW; ++t) {
					const int i = j - KW + t;
					a[t] = i >= 0 && i >= j - kd ? arow[i] : 0.0;
				}
				double temp = xs[j];
#pragma unroll
				for (int t = 0; t < KW; ++t) {
					const int i = j - KW + t;
					if (i >= 0 && i >= j - kd) temp = temp - a[t] * w[t];
				}
				const double v = temp / abs[(size_t)j * ldab + kd];
				xs[j] = v;
#pragma unroll
				for (int t = 0; t < KW - 1; ++t) w[t] = w[t + 1];
				w[KW - 1] = v;
			}
			// backward: cur = xs[j] with the updates of the rows below applied,
			// w[t] = xs[j - KW + t] pending
#pragma unroll
			for (int t = 0; t < KW; ++t) {
				const int i = n - 1 - KW + t;
				w[t] = i >= 0 ? xs[i] : 0.0;
			}
			double cur = xs[n - 1];
			for (int j = n - 1; j >= 0; --j) {
				if (cur != 0.0) {
					cur = cur / abs[(size_t)j * ldab + kd];
					const double temp = cur;
					const double *arow = abs + (size_t)j * ldab + kd - j;
#pragma unroll
					for (int t = KW - 1; t >= 0; --t) {
						const int i = j - KW + t;
						if (i >= 0 && i >= j - kd) w[t] = w[t] - temp * arow[i];
					}
				}
				xs[j] = cur;
				cur = w[KW - 1];
#pragma unroll
				for (int t = KW - 1; t >= 1; --t) w[t] = w[t - 1];
				const int i = j - 1 - KW;  // no row at or below j updates it
				w[0] = i >= 0 ? xs[i] : 0.0;
			}
		} else {
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
	}
	__syncthreads();
	cc_rows(1, L.nx, 1, L.ny, [&](int i, int j) { L.x[(size_t)j * L.pitch + i] = (T)xs[(j - 1) * L.nx + i - 1]; });
}

// Shared-memory map: the levels' copies (cc_view), the line right-hand sides,
// then (8-byte aligned) the coarsest solve's vector and factor in FP64.
template <typename T>
__host__ __device__ inline void cc_layout(const CoarseCycle<T> &cc, size_t *levels, size_t *lines, size_t *dbl)
{
	size_t lv = 0, ln = 0;
	for (int l = 0; l < cc.nl; ++l) {
		lv += cc_elems(cc, l);
		if (l + 1 < cc.nl) {
			const CoarseLevel<T> &L = cc.lv[l];
			const size_t a = (size_t)((L.ny + 1) / 2) * L.nx, b = (size_t)((L.nx + 1) / 2) * L.ny;
			ln = ln > a ? ln : a;
			ln = ln > b ? ln : b;
		}
	}
	const CoarseLevel<T> &Cg = cc.lv[cc.nl - 1];
	const size_t n = (size_t)Cg.nx * Cg.ny;
	*levels = lv;
	*lines = ln;
	*dbl = n + (size_t)(Cg.nx + 2) * n;
}

template <typename T>
__global__ void __launch_bounds__(CC_THREADS) k_coarse_cycle(CoarseCycle<T> cc)
{
	extern __shared__ __align__(16) unsigned char cc_smem[];
	T *base = reinterpret_cast<T *>(cc_smem);
	size_t nlv, nln, ndbl;
	cc_layout(cc, &nlv, &nln, &ndbl);
	T *sm = base + nlv;  // line right-hand sides
	double *xs = reinterpret_cast<double *>(cc_smem + ((nlv + nln) * sizeof(T) + 7) / 8 * 8);
	const int nl = cc.nl;
	// stage: operators, factors and weights of every level; b of the first level;
	// x, r and the other b zero (ghost rings included)
	for (int l = 0; l < nl; ++l) {
		const CoarseLevel<T> G = cc_global(cc, l), S = cc_view(cc, l, base);
		const size_t gpl = (size_t)G.pitch * (G.ny + 2), spl = (size_t)S.pitch * (S.ny + 2);
		const int ii = G.nx + 2, jj = G.ny + 2;
		if (l < nl - 1) {
			cc_stage<T>(G.so, G.pitch, gpl, const_cast<T *>(S.so), S.pitch, spl, ii, jj, G.ns);
			if (S.sor) cc_stage<T>(G.sor, G.pitch, gpl, const_cast<T *>(S.sor), S.pitch, spl, ii, jj, cc_sor_planes(cc.relax));
			if (S.sory)  // transposed: nx+2 rows of ny+2 elements
				cc_stage<T>(G.sory, G.tpitch, (size_t)G.tpitch * ii, const_cast<T *>(S.sory), S.tpitch,
				            (size_t)S.tpitch * ii, jj, ii, 2);
			cc_fill(S.r, spl);
		}
		if (l > 0) cc_stage<T>(G.ci, G.pitch, gpl, const_cast<T *>(S.ci), S.pitch, spl, ii, jj, 8);
		if (l == 0) cc_stage<T>(G.b, G.pitch, gpl, S.b, S.pitch, spl, ii, jj, 1);
		else cc_fill(S.b, spl);
		cc_fill(S.x, spl);
	}
	{  // the coarsest level's band factor, after its right-hand side xs
		const CoarseLevel<T> &Cg = cc.lv[nl - 1];
		const int n = Cg.nx * Cg.ny, nab = (Cg.nx + 2) * n;
		cc_stage<double>(cc.abd + (size_t)blockIdx.x * cc.bstep * nab, 0, 0, xs + n, 0, 0, nab, 1, 1);
	}
	cc_stage_wait();
	__syncthreads();
	// The cycle as one sequence of steps (down: smooth, residual, restriction,
	// and the coarsest solve after the last; up: interpolation, smooth), so that
	// the code of each kind of step exists once: the first fetch of a code
	// region from instruction memory costs several microseconds, and separate
	// copies for the two legs paid it twice.
	if (nl == 1) {
		cc_cg<T>(cc_view(cc, 0, base), xs);
		__syncthreads();
	}
	for (int step = 0; step < 2 * (nl - 1); ++step) {
		const bool down = step < nl - 1;
		const int l = down ? step : 2 * (nl - 1) - 1 - step;
		const CoarseLevel<T> F = cc_view(cc, l, base), C = cc_view(cc, l + 1, base);
		if (!down) {
			cc_interp<T>(F, C);
			__syncthreads();
		}
		const int updown = down ? CDR_DOWN : CDR_UP;
		if (F.ns == 5) cc_smooth<T, 5>(cc, F, updown, sm);
		else cc_smooth<T, 3>(cc, F, updown, sm);
		if (down) {
			if (F.ns == 5) cc_residual<T, 5>(F);
			else cc_residual<T, 3>(F);
			__syncthreads();
			cc_restrict<T>(F, C);
			cc_fill(C.x, (size_t)C.pitch * (C.ny + 2));
			__syncthreads();
			if (l == nl - 2) {
				cc_cg<T>(cc_view(cc, nl - 1, base), xs);
				__syncthreads();
			}
		} else {
			__syncthreads();
		}
	}
	{
		const CoarseLevel<T> G = cc_global(cc, 0), S = cc_view(cc, 0, base);
		cc_copy<T>(S.x, S.pitch, 0, G.x, G.pitch, 0, G.nx + 2, G.ny + 2, 1);
	}
}

template <typename T>
size_t coarse_cycle_smem(const CoarseCycle<T> &cc)
{
	size_t nlv, nln, ndbl;
	cc_layout(cc, &nlv, &nln, &ndbl);
	return ((nlv + nln) * sizeof(T) + 7) / 8 * 8 + ndbl * sizeof(double);
}

// Shared memory a fused coarse cycle from level descriptor lv[0..nl) needs
template <typename T>
size_t coarse_cycle_bytes(const CoarseCycle<T> &cc)
{
	return coarse_cycle_smem(cc);
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
	const size_t smem = coarse_cycle_smem(cc);
	if (smem > kCoarseSmemMax) {
		set_error(CDR_ERR_DIM, "fused coarse cycle needs %zu bytes of shared memory", smem);
		return CDR_ERR_DIM;
	}
	k_coarse_cycle<T><<<nproblems, CC_THREADS, smem, st>>>(cc);
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
