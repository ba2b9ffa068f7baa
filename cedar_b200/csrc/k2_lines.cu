// k2_lines.cu -- zebra line Gauss-Seidel for 2D BoxMG on sm_100a.
//
// The reference forms each line's right-hand side from the two neighbouring
// lines and calls LAPACK DPTTRS on the line's L*D*L^T factors
// (src/2d/ftn/BMG2_SymStd_relax_lines_x.f90:99-131, ..._y.f90:95-129).  Here one
// CTA owns G whole lines of one colour:
//   1. the right-hand sides are formed with coalesced loads into shared memory
//      (x-lines: consecutive threads walk i; y-lines: consecutive threads walk
//      the G lines of a row, so each row segment is one or two 128-byte lines);
//   2. the two substitutions of DPTTRS, y(i) = r(i) - y(i-1) e(i) and
//      x(i) = y(i)/d(i) - x(i+1) e(i+1), are first-order affine recurrences.
//      Each of the 256/G threads of a line composes the affine map of its
//      contiguous chunk, a segmented scan over the chunk maps gives every chunk
//      its incoming value, and the chunk is then re-run with the exact LAPACK
//      update (so every element sees the DPTTS2 operation on its inputs);
//   3. the solution is written back with the coalesced mapping of step 1.
// Both colours of a sweep are two launches: lines of one colour read only lines
// of the other colour.  With CDR_LINES_EXACT the substitutions instead run in
// DPTTS2's sequential order (one thread per line): slower, bit-identical.
#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>

#include "k2_bulk.cuh"
#include "k2_point.cuh"
#include "kernels2d.cuh"

namespace cdrgpu {

constexpr int LT = 256;  // threads per CTA

// ------------------------------------------------------------------ setup
// BMG2_SymStd_SETUP_lines_{x,y} + DPTTRF: per line d = c, e = -w (x) or -s (y),
// then e(i) <- e(i)/d(i-1), d(i) <- d(i) - e(i)*e_old(i).  Always FP64; TS is
// the storage type of the factors.  FP32 factors (the preconditioner's) keep the
// reciprocal pivots 1/d, formed in FP64 and rounded once, so that the FP32 sweeps
// multiply instead of divide; FP64 factors keep d, as DPTTRF does.
template <typename TS, int DIR>
__global__ void k_lines_setup(const double *__restrict__ so, int ns, TS *__restrict__ sor, Dims2 d, int tpitch,
                              int *__restrict__ info)
{
	const int line = blockIdx.x * blockDim.x + threadIdx.x + 1;
	const int nl = DIR == CDR_DIR_X ? d.ny : d.nx;
	const int n = DIR == CDR_DIR_X ? d.nx : d.ny;
	if (line > nl) return;
	const size_t ps = d.plane();
	so += d.bofs(ns * ps);
	sor += d.bofs(line_factor_size(d, tpitch, DIR));
	const double *c = so, *off = so + (DIR == CDR_DIR_X ? 1 : 2) * ps;
	// element at line position p (1..n): grid offset and factor offset
	auto g = [&](int p) -> size_t { return DIR == CDR_DIR_X ? d.at(p, line) : d.at(line, p); };
	const size_t fps = DIR == CDR_DIR_X ? ps : (size_t)tpitch * (d.nx + 2);
	auto fo = [&](int p) -> size_t { return DIR == CDR_DIR_X ? d.at(p, line) : (size_t)line * tpitch + p; };
	double dprev = c[g(1)];
	sor[fo(1)] = pivot_store<TS>(dprev);
	sor[fps + fo(1)] = (TS)(-off[g(1)]);
	int st = 0;
	for (int p = 1; p < n; ++p) {
		if (dprev <= 0.0 && !st) st = p;
		double ei = -off[g(p + 1)];
		double e = ei / dprev;
		double dn = c[g(p + 1)] - e * ei;
		sor[fps + fo(p + 1)] = (TS)e;
		sor[fo(p + 1)] = pivot_store<TS>(dn);
		dprev = dn;
	}
	if (dprev <= 0.0 && !st) st = n;
	if (st && info) atomicCAS(info, 0, line);
}

template <typename TS>
int setup_lines_2d(const double *so, int nstencil, TS *sor, Dims2 d, int tpitch, int dir, int *info, cudaStream_t st)
{
	if (dir == CDR_DIR_Y && tpitch < d.ny + 2) {
		set_error(CDR_ERR_DIM, "y-line factor pitch %d < ny+2 = %d", tpitch, d.ny + 2);
		return CDR_ERR_DIM;
	}
	const int nl = dir == CDR_DIR_X ? d.ny : d.nx;
	const dim3 grd(ceil_div(nl, 128), 1, d.nb);
	if (dir == CDR_DIR_X) k_lines_setup<TS, CDR_DIR_X><<<grd, 128, 0, st>>>(so, nstencil, sor, d, tpitch, info);
	else k_lines_setup<TS, CDR_DIR_Y><<<grd, 128, 0, st>>>(so, nstencil, sor, d, tpitch, info);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int setup_lines_2d<double>(const double *, int, double *, Dims2, int, int, int *, cudaStream_t);
template int setup_lines_2d<float>(const double *, int, float *, Dims2, int, int, int *, cudaStream_t);

// ------------------------------------------------------------------ relax
// Segmented inclusive scan of affine maps over the tpl threads of a line.
// forward: element t composes (later) t o (earlier) t-off; backward: t o t+off.
template <typename T>
__device__ __forceinline__ void affine_scan(T &A, T &B, T *sA, T *sB, int t, int tpl, bool forward)
{
	const int tid = threadIdx.x;
	for (int off = 1; off < tpl; off <<= 1) {
		sA[tid] = A;
		sB[tid] = B;
		__syncthreads();
		if (forward ? t >= off : t + off < tpl) {
			int o = forward ? tid - off : tid + off;
			T a2 = sA[o], b2 = sB[o];
			B = A * b2 + B;
			A = A * a2;
		}
		__syncthreads();
	}
	sA[tid] = A;
	sB[tid] = B;
	__syncthreads();
}

template <typename T, int NS, int DIR, bool EXACT>
__global__ void __launch_bounds__(LT) k_lines(const T *__restrict__ so, T *__restrict__ q, const T *__restrict__ qf,
                                              const T *__restrict__ sor, Dims2 d, int tpitch, int first, int G)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T *sA = reinterpret_cast<T *>(smem_raw);
	T *sB = sA + LT;
	T *buf = sB + LT;
	const size_t ps = d.plane();
	const int p = d.pitch;
	so += d.bofs(NS * ps);
	q += d.bofs(ps);
	qf += d.bofs(ps);
	sor += d.bofs(line_factor_size(d, tpitch, DIR));
	const int n = DIR == CDR_DIR_X ? d.nx : d.ny;     // line length
	const int nl = DIR == CDR_DIR_X ? d.ny : d.nx;    // lines in the grid
	const int l0 = blockIdx.x * G;                    // first line (of this colour) of the CTA
	auto line_coord = [&](int g) { return first + 2 * (l0 + g); };
	int gmax = G;
	while (gmax > 0 && line_coord(gmax - 1) > nl) --gmax;

	// 1. right-hand sides
	for (int idx = threadIdx.x; idx < gmax * n; idx += LT) {
		int g, m;
		if (DIR == CDR_DIR_X) { g = idx / n; m = idx - g * n; }
		else { m = idx / gmax; g = idx - m * gmax; }
		int lc = line_coord(g);
		size_t k = DIR == CDR_DIR_X ? d.at(m + 1, lc) : d.at(lc, m + 1);
		buf[g * n + m] = line_rhs<T, NS, DIR>(so, ps, q, qf, k, p);
	}
	__syncthreads();

	// 2. substitutions
	const int tpl = LT / G;
	const int g = threadIdx.x / tpl, t = threadIdx.x - g * tpl;
	const bool active = g < gmax;
	const int lc = active ? line_coord(g) : 1;
	const T *D, *E;
	if (DIR == CDR_DIR_X) {
		D = sor + (size_t)lc * p;
		E = sor + ps + (size_t)lc * p;
	} else {
		D = sor + (size_t)lc * tpitch;
		E = sor + (size_t)tpitch * (d.nx + 2) + (size_t)lc * tpitch;
	}
	T *r = buf + g * n;  // r[m] is line position m+1
	if (EXACT) {
		// DPTTS2 in its own order, one thread per line: bit-identical to LAPACK.
		if (active && t == 0) {
			for (int m = 1; m < n; ++m) r[m] = r[m] - r[m - 1] * E[m + 1];
			r[n - 1] = pivot_div(r[n - 1], D[n]);
			for (int m = n - 2; m >= 0; --m) r[m] = pivot_div(r[m], D[m + 1]) - r[m + 1] * E[m + 2];
		}
		__syncthreads();
	} else {
		const int K = (n + tpl - 1) / tpl;
		const int lo = t * K < n ? t * K : n, hi = lo + K < n ? lo + K : n;
		// forward: y(m) = r(m) - y(m-1) * E(m+1)
		T A = T(1), B = T(0);
		if (active)
			for (int m = lo; m < hi; ++m) {
				T a = m == 0 ? T(0) : -E[m + 1];
				B = a * B + r[m];
				A = a * A;
			}
		affine_scan<T>(A, B, sA, sB, t, tpl, true);
		if (active) {
			T y = t == 0 ? T(0) : sB[threadIdx.x - 1];
			for (int m = lo; m < hi; ++m) {
				y = m == 0 ? r[0] : r[m] - y * E[m + 1];
				r[m] = y;
			}
		}
		__syncthreads();
		// backward: x(m) = y(m)/D(m+1) - x(m+1) * E(m+2)
		A = T(1);
		B = T(0);
		if (active)
			for (int m = hi - 1; m >= lo; --m) {
				T a = m == n - 1 ? T(0) : -E[m + 2];
				B = a * B + pivot_div(r[m], D[m + 1]);
				A = a * A;
			}
		affine_scan<T>(A, B, sA, sB, t, tpl, false);
		if (active) {
			T x = t == tpl - 1 ? T(0) : sB[threadIdx.x + 1];
			for (int m = hi - 1; m >= lo; --m) {
				x = m == n - 1 ? pivot_div(r[m], D[m + 1]) : pivot_div(r[m], D[m + 1]) - x * E[m + 2];
				r[m] = x;
			}
		}
		__syncthreads();
	}

	// 3. write back
	for (int idx = threadIdx.x; idx < gmax * n; idx += LT) {
		int gg, m;
		if (DIR == CDR_DIR_X) { gg = idx / n; m = idx - gg * n; }
		else { m = idx / gmax; gg = idx - m * gmax; }
		int c2 = line_coord(gg);
		size_t k = DIR == CDR_DIR_X ? d.at(m + 1, c2) : d.at(c2, m + 1);
		q[k] = buf[gg * n + m];
	}
}


// ------------------------------------------------------------ fast line sweep
// Register-chunk form of the zebra sweep.  Thread t of a line owns positions
// [t*K, t*K+K) of the line (0-based, ghost at 0; only 1..n are solved) and keeps
// their right-hand sides in registers.  x-lines: the threads of a line are
// consecutive lanes, so each thread reads its chunk with 16-byte vector loads
// and a warp covers 32*K contiguous elements of a row.  y-lines: the lanes of a
// warp are line-fastest (G lines side by side, stride-2 columns), so every row
// segment a warp touches is shared by its G lines; the factors of y-lines are
// stored transposed (line-contiguous) and still load as vectors.  The affine
// maps of the chunks are scanned with warp shuffles and, across warps, through
// shared memory (one slot per line and warp).
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; };
template <> struct Vec16<double> { using type = double2; };

template <typename T, int K>
__device__ __forceinline__ void vload(const T *__restrict__ p, T (&v)[K])
{
	using VT = typename Vec16<T>::type;
	constexpr int W = 16 / sizeof(T);
	const VT *pv = reinterpret_cast<const VT *>(p);
#pragma unroll
	for (int c = 0; c < K / W; ++c) {
		VT t = pv[c];
		const T *e = reinterpret_cast<const T *>(&t);
#pragma unroll
		for (int w = 0; w < W; ++w) v[c * W + w] = e[w];
	}
}

template <typename T, int K>
__device__ __forceinline__ void vstore(T *__restrict__ p, const T (&v)[K])
{
	using VT = typename Vec16<T>::type;
	constexpr int W = 16 / sizeof(T);
	VT *pv = reinterpret_cast<VT *>(p);
#pragma unroll
	for (int c = 0; c < K / W; ++c) {
		VT t;
		T *e = reinterpret_cast<T *>(&t);
#pragma unroll
		for (int w = 0; w < W; ++w) e[w] = v[c * W + w];
		pv[c] = t;
	}
}

// compose (A,B) <- (A,B) o (a2,b2): apply (a2,b2) first
template <typename T>
__device__ __forceinline__ void after(T &A, T &B, T a2, T b2)
{
	B = madd(A, b2, B);
	A = A * a2;
}

// Exclusive scan of the chunk maps of a line.  forward: element u composes the
// maps of the chunks before it (lower t); backward: after it (higher t).  S is
// the lane distance between consecutive chunks of a line in a warp, CW the
// number of chunks of one line in a warp, NWG the number of warps a line spans;
// slot(g, k) indexes the shared-memory carry of line g, warp group k.
// Returns the map's value at 0 (the incoming value of the chunk).
template <typename T>
__device__ __forceinline__ T scan_incoming(T A, T B, bool forward, int u, int S, int CW, int NWG, int k, int slot_self,
                                           int slot_stride, T *sA, T *sB)
{
	const unsigned full = 0xffffffffu;
	// inclusive within the warp segment
	for (int off = 1; off < CW; off <<= 1) {
		T a2 = forward ? __shfl_up_sync(full, A, off * S) : __shfl_down_sync(full, A, off * S);
		T b2 = forward ? __shfl_up_sync(full, B, off * S) : __shfl_down_sync(full, B, off * S);
		if (forward ? u >= off : u + off < CW) after(A, B, a2, b2);
	}
	// exclusive within the warp segment
	T ae = forward ? __shfl_up_sync(full, A, S) : __shfl_down_sync(full, A, S);
	T be = forward ? __shfl_up_sync(full, B, S) : __shfl_down_sync(full, B, S);
	const bool first = forward ? u == 0 : u == CW - 1;
	if (first) { ae = T(1); be = T(0); }
	if (NWG == 1) return be;
	// carry across warps: slot of group k holds the inclusive map of the whole group
	const bool last = forward ? u == CW - 1 : u == 0;
	__syncthreads();
	if (last) { sA[slot_self] = A; sB[slot_self] = B; }
	__syncthreads();
	T ca = T(1), cb = T(0);
	if (forward) {
		for (int kk = 0; kk < k; ++kk) {  // carry = M_{k-1} o ... o M_0
			int sl = slot_self + (kk - k) * slot_stride;
			T a2 = sA[sl], b2 = sB[sl];
			T na = a2 * ca, nb = madd(a2, cb, b2);
			ca = na; cb = nb;
		}
	} else {
		for (int kk = NWG - 1; kk > k; --kk) {  // carry = M_{k+1} o ... o M_{NWG-1}
			int sl = slot_self + (kk - k) * slot_stride;
			T a2 = sA[sl], b2 = sB[sl];
			T na = a2 * ca, nb = madd(a2, cb, b2);
			ca = na; cb = nb;
		}
	}
	return madd(ae, cb, be);
}

constexpr int FAST_BLOCK_X = 256, FAST_BLOCK_Y = 1024;

template <typename T, int NS, int DIR, int K, bool XL = DIR == CDR_DIR_X>
__global__ void __launch_bounds__(XL ? FAST_BLOCK_X : FAST_BLOCK_Y, XL ? 2 : 1)
    k_lines_fast(const T *__restrict__ so, T *__restrict__ q, const T *__restrict__ qf, const T *__restrict__ sor,
                 Dims2 d, int tpitch, int first, int tpl_log2)
{
	// one carry slot per (warp, line of the warp): at most 32 warps x 32 lines
	__shared__ T sA[FAST_BLOCK_Y], sB[FAST_BLOCK_Y];
	const int TPL = 1 << tpl_log2;
	const int G = blockDim.x >> tpl_log2;  // lines per CTA
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	int g, t;
	if (XL) { g = tid >> tpl_log2; t = tid & (TPL - 1); }
	else { g = tid % G; t = tid / G; }
	const int n = DIR == CDR_DIR_X ? d.nx : d.ny;
	const int nl = DIR == CDR_DIR_X ? d.ny : d.nx;
	const int lc = first + 2 * (blockIdx.x * G + g);
	const bool active = lc <= nl;
	const int p0 = t * K;
	const bool has = active && p0 <= n;
	// Chunks cover positions 0 .. TPL*K - 1 (position 0 is the ghost).  Where
	// TPL*K == n, position n is left over and the last chunk takes it as one more
	// element (rx, its rhs and then its solution): a level of 2^k + 1 positions
	// then runs on 2^k / K threads per line instead of twice that.
	const bool xtra = has && t == TPL - 1 && p0 + K == n;
	T rx = T(0);
	const size_t ps = d.plane();
	const int P = d.pitch;
	so += d.bofs(NS * ps);
	q += d.bofs(ps);
	qf += d.bofs(ps);
	sor += d.bofs(line_factor_size(d, tpitch, DIR));
	const T *D = DIR == CDR_DIR_X ? sor + (size_t)lc * P : sor + (size_t)lc * tpitch;
	const T *E = DIR == CDR_DIR_X ? sor + ps + (size_t)lc * P : sor + (size_t)tpitch * (d.nx + 2) + (size_t)lc * tpitch;

	// 1. right-hand sides of the chunk
	T r[K];
#pragma unroll
	for (int m = 0; m < K; ++m) r[m] = T(0);
	if (has) {
		if (DIR == CDR_DIR_X) {
			const size_t k0 = d.at(p0, lc);
			const T *w = so + ps, *s = so + 2 * ps, *sw = so + 3 * ps, *nw = so + 4 * ps;
			T b_[K], qm[K], qp[K], s0[K], s1[K];
			vload<T, K>(qf + k0, b_);
			vload<T, K>(q + k0 - P, qm);
			vload<T, K>(q + k0 + P, qp);
			vload<T, K>(s + k0, s0);
			vload<T, K>(s + k0 + P, s1);
#pragma unroll
			for (int m = 0; m < K; ++m) r[m] = madd(s1[m], qp[m], madd(s0[m], qm[m], b_[m]));
			const size_t kx = k0 + K;  // position n when xtra
			if (xtra) rx = madd(s[kx + P], q[kx + P], madd(s[kx], q[kx - P], qf[kx]));
			if (NS == 5) {
				T sw0[K], nw0[K], nw1[K], sw1[K];
				vload<T, K>(sw + k0, sw0);
				vload<T, K>(nw + k0, nw0);
				vload<T, K>(nw + k0 + P, nw1);
				vload<T, K>(sw + k0 + P, sw1);
				const T qm_l = p0 >= 1 ? q[k0 - P - 1] : T(0), qp_l = p0 >= 1 ? q[k0 + P - 1] : T(0);
				const bool rin = p0 + K <= n + 1;
				const T qm_r = rin ? q[k0 - P + K] : T(0), qp_r = rin ? q[k0 + P + K] : T(0);
				const T nw0_r = rin ? nw[k0 + K] : T(0), sw1_r = rin ? sw[k0 + P + K] : T(0);
#pragma unroll
				for (int m = 0; m < K; ++m) {
					const T qml = m > 0 ? qm[m - 1] : qm_l, qmr = m < K - 1 ? qm[m + 1] : qm_r;
					const T qpl = m > 0 ? qp[m - 1] : qp_l, qpr = m < K - 1 ? qp[m + 1] : qp_r;
					const T nwr = m < K - 1 ? nw0[m + 1] : nw0_r, swr = m < K - 1 ? sw1[m + 1] : sw1_r;
					// operand order of relax_lines_x.f90:106-110
					T a = madd(s0[m], qm[m], b_[m]);
					a = madd(s1[m], qp[m], a);
					a = madd(sw0[m], qml, a);
					a = madd(nwr, qmr, a);
					a = madd(nw1[m], qpl, a);
					r[m] = madd(swr, qpr, a);
				}
				if (xtra) {
					T a = madd(s[kx], q[kx - P], qf[kx]);
					a = madd(s[kx + P], q[kx + P], a);
					a = madd(sw[kx], qm[K - 1], a);
					a = madd(nw[kx + 1], q[kx - P + 1], a);
					a = madd(nw[kx + P], qp[K - 1], a);
					rx = madd(sw[kx + P + 1], q[kx + P + 1], a);
				}
			}
		} else {
			const int i = lc;
#pragma unroll
			for (int m = 0; m < K; ++m) {
				const int jj = p0 + m;
				if (jj < 1 || jj > n) continue;
				r[m] = line_rhs<T, NS, CDR_DIR_Y>(so, ps, q, qf, d.at(i, jj), P);
			}
			if (xtra) rx = line_rhs<T, NS, CDR_DIR_Y>(so, ps, q, qf, d.at(i, n), P);
		}
	}

	// scan geometry
	int S, CW, NWG, kgrp, slot, sstride;
	if (XL) {
		S = 1;
		CW = TPL < 32 ? TPL : 32;
		NWG = TPL > 32 ? TPL / 32 : 1;
		kgrp = TPL > 32 ? (tid - (g << tpl_log2)) >> 5 : 0;
		slot = warp;
		sstride = 1;
	} else {
		S = G < 32 ? G : 32;
		CW = 32 / S;
		NWG = blockDim.x / 32;
		kgrp = warp;
		slot = warp * (32 / CW) + (lane % S);  // one slot per (warp, line of the warp)
		sstride = 32 / CW;
	}
	const int u = XL ? (lane & (CW - 1)) : lane / S;
	const bool full = p0 >= 1 && p0 + K - 1 <= n;  // no ghost or beyond-end position in the chunk

	// 2a. forward substitution y(p) = r(p) - y(p-1) E(p)
	T Ev[K];
	if (has) vload<T, K>(E + p0, Ev);
	T A = T(1), B = T(0);
	if (has) {
#pragma unroll
		for (int m = 0; m < K; ++m) {
			const int pos = p0 + m;
			if (!full && (pos < 1 || pos > n)) continue;
			const T a = (!full && pos == 1) ? T(0) : -Ev[m];
			B = madd(a, B, r[m]);
			A = a * A;
		}
		if (xtra) {
			const T a = -E[n];
			B = madd(a, B, rx);
			A = a * A;
		}
	}
	T y = scan_incoming<T>(A, B, true, u, S, CW, NWG, kgrp, slot, sstride, sA, sB);
	if (has) {
#pragma unroll
		for (int m = 0; m < K; ++m) {
			const int pos = p0 + m;
			if (!full && (pos < 1 || pos > n)) continue;
			y = (!full && pos == 1) ? r[m] : madd(-y, Ev[m], r[m]);
			r[m] = y;
		}
		if (xtra) rx = pivot_div(madd(-y, E[n], rx), D[n]);
		// y(p)/D(p), the first operation of the DPTTS2 back substitution, in place
		constexpr int W = 16 / sizeof(T);
#pragma unroll
		for (int c = 0; c < K / W; ++c) {
			T dv[W];
			vload<T, W>(D + p0 + c * W, dv);
#pragma unroll
			for (int w = 0; w < W; ++w) {
				const int m = c * W + w, pos = p0 + m;
				if (full || (pos >= 1 && pos <= n)) r[m] = pivot_div(r[m], dv[w]);
			}
		}
	}
	// 2b. backward substitution x(p) = y(p)/D(p) - x(p+1) E(p+1)
	const T Enext = has && p0 + K <= n ? E[p0 + K] : T(0);
	A = T(1);
	B = T(0);
	if (has) {
		if (xtra) {
			B = madd(T(0), B, rx);
			A = T(0) * A;
		}
#pragma unroll
		for (int m = K - 1; m >= 0; --m) {
			const int pos = p0 + m;
			if (!full && (pos < 1 || pos > n)) continue;
			const T e1 = m < K - 1 ? Ev[m + 1] : Enext;
			const T a = pos == n ? T(0) : -e1;
			B = madd(a, B, r[m]);
			A = a * A;
		}
	}
	if (NWG > 1) __syncthreads();  // the forward carries are still being read
	T x = scan_incoming<T>(A, B, false, u, S, CW, NWG, kgrp, slot, sstride, sA, sB);
	if (has) {
		if (xtra) x = rx;
#pragma unroll
		for (int m = K - 1; m >= 0; --m) {
			const int pos = p0 + m;
			if (!full && (pos < 1 || pos > n)) continue;
			const T e1 = m < K - 1 ? Ev[m + 1] : Enext;
			x = pos == n ? r[m] : madd(-x, e1, r[m]);
			r[m] = x;
		}
	}

	// 3. write back the interior positions of the chunk
	if (has) {
		if (DIR == CDR_DIR_X) {
			const size_t k0 = d.at(p0, lc);
			if (xtra) q[k0 + K] = rx;
			if (p0 >= 1 && p0 + K - 1 <= n) vstore<T, K>(q + k0, r);
			else {
#pragma unroll
				for (int m = 0; m < K; ++m) {
					const int pos = p0 + m;
					if (pos >= 1 && pos <= n) q[k0 + m] = r[m];
				}
			}
		} else {
#pragma unroll
			for (int m = 0; m < K; ++m) {
				const int pos = p0 + m;
				if (pos >= 1 && pos <= n) q[d.at(lc, pos)] = r[m];
			}
			if (xtra) q[d.at(lc, n)] = rx;
		}
	}
}

// ---------------------------------------------------------- streamed x-lines
// x-lines of one problem with 32K <= n <= 256K: a persistent CTA walks the
// lines of a colour (l = blockIdx.x, + gridDim.x, ...).  Each line's rows --
// b, x of the two neighbouring lines, the off-line couplings of rows j and j+1
// and the line's factors, 7 or 11 rows -- arrive in shared memory by bulk
// asynchronous copies (cp.async.bulk) completing on one mbarrier.  Every
// thread takes its chunk of the rows into registers, the stage is released at
// once and the next line's rows are requested, and the scans of the current
// line then run while DRAM streams the next one (one stage per CTA, so two
// CTAs share an SM).  The arithmetic is k_lines_fast's x-line path with the
// same K: results are bit-identical to it.  Every wait on the stage is
// bounded (g_xstream_wait_ns of the global timer); a CTA that gives up counts
// itself in g_xstream_timeouts, waits (bounded) for the copy it has in flight,
// so that nothing lands in shared memory after it has left, and returns.
namespace {
__device__ unsigned g_xstream_timeouts;
__device__ unsigned long long g_xstream_wait_ns = kWaitLimitNs;
}  // namespace
static_assert(kStreamWaitDefaultNs == kWaitLimitNs, "one default wait limit");

int lines_stream_timeouts(cudaStream_t st, unsigned *count)
{
	unsigned v = 0;
	*count = 0;
	CDR_CUDA_TRY(cudaMemcpyFromSymbolAsync(&v, g_xstream_timeouts, sizeof v, 0, cudaMemcpyDeviceToHost, st));
	CDR_CUDA_TRY(cudaStreamSynchronize(st));
	if (v) {
		const unsigned z = 0;
		CDR_CUDA_TRY(cudaMemcpyToSymbolAsync(g_xstream_timeouts, &z, sizeof z, 0, cudaMemcpyHostToDevice, st));
		CDR_CUDA_TRY(cudaStreamSynchronize(st));
	}
	*count = v;
	return CDR_OK;
}

int lines_stream_add_timeouts(unsigned n)
{
	unsigned v = 0;
	CDR_CUDA_TRY(cudaMemcpyFromSymbol(&v, g_xstream_timeouts, sizeof v));
	v += n;
	CDR_CUDA_TRY(cudaMemcpyToSymbol(g_xstream_timeouts, &v, sizeof v));
	return CDR_OK;
}

int lines_stream_set_wait(unsigned long long ns)
{
	CDR_CUDA_TRY(cudaMemcpyToSymbol(g_xstream_wait_ns, &ns, sizeof ns));
	return CDR_OK;
}

constexpr int XS_BLOCK = 256;
constexpr int XS_SMEM_MAX = 226 * 1024;  // dynamic part; the kernel's static carries take the rest
template <int NS>
__host__ __device__ constexpr int xs_rows()
{
	return NS == 5 ? 11 : 7;
}
// dynamic shared memory of the streamed kernel: the barrier (padded to 128
// bytes), then one stage of R rows with the level's pitch
template <typename T, int NS>
static size_t xs_smem(int pitch)
{
	return 128 + (size_t)xs_rows<NS>() * pitch * sizeof(T);
}

template <typename T, int NS, int K>
__global__ void __launch_bounds__(XS_BLOCK, 2) k_lines_xstream(const T *__restrict__ so, T *__restrict__ q,
                                                               const T *__restrict__ qf, const T *__restrict__ sor,
                                                               Dims2 d, int first, int nlines)
{
	extern __shared__ __align__(128) unsigned char xs_raw[];
	__shared__ T sA[XS_BLOCK / 32], sB[XS_BLOCK / 32];
	constexpr int R = xs_rows<NS>();
	uint64_t *bar = reinterpret_cast<uint64_t *>(xs_raw);
	T *rows = reinterpret_cast<T *>(xs_raw + 128);
	const int P = d.pitch, n = d.nx;
	const size_t ps = d.plane();
	const unsigned row_bytes = ((unsigned)(n + 2) * sizeof(T) + 15u) & ~15u;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int TPL = blockDim.x;  // threads of the line: chunks of K positions
	const T *s = so + 2 * ps, *sw = so + (NS == 5 ? 3 : 0) * ps, *nw = so + (NS == 5 ? 4 : 0) * ps;
	const T *Dp = sor, *Ep = sor + ps;

	// rows of line index li: b, x(j-1), x(j+1), s(j), s(j+1), d, e [, sw(j), sw(j+1), nw(j), nw(j+1)]
	auto issue = [&](int li) {
		const size_t j = (size_t)(first + 2 * li) * P;
		const T *src[11] = {qf + j, q + j - P, q + j + P, s + j, s + j + P, Dp + j, Ep + j,
		                    sw + j, sw + j + P, nw + j, nw + j + P};
		asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
		mbar_expect_tx(bar, R * row_bytes);
#pragma unroll
		for (int r = 0; r < R; ++r) bulk_g2s(rows + (size_t)r * P, src[r], row_bytes, bar);
	};

	if (tid == 0) {
		mbar_init(bar, 1);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	__syncthreads();
	const int G = gridDim.x;
	if (tid == 0 && (int)blockIdx.x < nlines) issue(blockIdx.x);

	// scan geometry of one line per CTA (k_lines_fast's x-line case with G = 1)
	const int CW = TPL < 32 ? TPL : 32, NWG = TPL > 32 ? TPL / 32 : 1, kgrp = TPL > 32 ? warp : 0;
	const int u = lane & (CW - 1);
	const int p0 = tid * K;
	const bool has = p0 <= n;
	const bool xtra = has && tid == TPL - 1 && p0 + K == n;
	const bool full = p0 >= 1 && p0 + K - 1 <= n;
	const T *rb = rows, *rqm = rows + P, *rqp = rows + 2 * P, *rs0 = rows + 3 * P, *rs1 = rows + 4 * P;
	const T *rD = rows + 5 * P, *rE = rows + 6 * P;

	// K-element chunk (two 16-byte pieces) from a staged row, the two pieces read
	// in an order swapped for every other group of four lanes, so that a warp's
	// 16-byte loads hit all 32 banks (lanes 32 bytes apart would otherwise meet
	// in pairs)
	constexpr int W = 16 / sizeof(T);
	static_assert(K == 2 * W, "two 16-byte pieces per chunk");
	const int rot = (lane >> 2) & 1;
	auto sload = [&](const T *p, T(&v)[K]) {
		using VT = typename Vec16<T>::type;
		const VT *pv = reinterpret_cast<const VT *>(p);
		const VT ta = pv[rot], tb = pv[rot ^ 1];
		const T *ea = reinterpret_cast<const T *>(&ta), *eb = reinterpret_cast<const T *>(&tb);
#pragma unroll
		for (int w = 0; w < W; ++w) {
			v[w] = rot ? eb[w] : ea[w];
			v[W + w] = rot ? ea[w] : eb[w];
		}
	};
	const unsigned long long wait_ns = g_xstream_wait_ns;
	int k = 0;
	for (int li = blockIdx.x; li < nlines; li += G, ++k) {
		const bool ok = mbar_wait_bounded(bar, (unsigned)k & 1u, wait_ns);
		if (!__syncthreads_and(ok)) {
			// give up: count, then wait (bounded) for this line's copy, the one in flight
			if (tid == 0) {
				atomicAdd(&g_xstream_timeouts, 1u);
				mbar_wait_bounded(bar, (unsigned)k & 1u, kDrainLimitNs);
			}
			return;
		}
		const int lc = first + 2 * li;

		// 1. everything this thread needs from the stage into registers, and the
		// right-hand sides of the chunk
		T r[K], Ev[K], dv[K];
		T rx = T(0), Ex = T(0), Dx = T(0), Enext = T(0);
#pragma unroll
		for (int m = 0; m < K; ++m) r[m] = T(0);
		if (has) {
			T b_[K], qm[K], qp[K], s0[K], s1[K];
			sload(rb + p0, b_);
			sload(rqm + p0, qm);
			sload(rqp + p0, qp);
			sload(rs0 + p0, s0);
			sload(rs1 + p0, s1);
			sload(rE + p0, Ev);
			sload(rD + p0, dv);
			Enext = p0 + K <= n ? rE[p0 + K] : T(0);
			if (xtra) {
				Ex = rE[n];
				Dx = rD[n];
			}
#pragma unroll
			for (int m = 0; m < K; ++m) r[m] = madd(s1[m], qp[m], madd(s0[m], qm[m], b_[m]));
			if (xtra) rx = madd(rs1[n], rqp[n], madd(rs0[n], rqm[n], rb[n]));
			if (NS == 5) {
				const T *rsw0 = rows + 7 * P, *rsw1 = rows + 8 * P, *rnw0 = rows + 9 * P, *rnw1 = rows + 10 * P;
				T sw0[K], nw0[K], nw1[K], sw1[K];
				sload(rsw0 + p0, sw0);
				sload(rnw0 + p0, nw0);
				sload(rnw1 + p0, nw1);
				sload(rsw1 + p0, sw1);
				const T qm_l = p0 >= 1 ? rqm[p0 - 1] : T(0), qp_l = p0 >= 1 ? rqp[p0 - 1] : T(0);
				const bool rin = p0 + K <= n + 1;
				const T qm_r = rin ? rqm[p0 + K] : T(0), qp_r = rin ? rqp[p0 + K] : T(0);
				const T nw0_r = rin ? rnw0[p0 + K] : T(0), sw1_r = rin ? rsw1[p0 + K] : T(0);
#pragma unroll
				for (int m = 0; m < K; ++m) {
					const T qml = m > 0 ? qm[m - 1] : qm_l, qmr = m < K - 1 ? qm[m + 1] : qm_r;
					const T qpl = m > 0 ? qp[m - 1] : qp_l, qpr = m < K - 1 ? qp[m + 1] : qp_r;
					const T nwr = m < K - 1 ? nw0[m + 1] : nw0_r, swr = m < K - 1 ? sw1[m + 1] : sw1_r;
					// operand order of relax_lines_x.f90:106-110
					T a = madd(s0[m], qm[m], b_[m]);
					a = madd(s1[m], qp[m], a);
					a = madd(sw0[m], qml, a);
					a = madd(nwr, qmr, a);
					a = madd(nw1[m], qpl, a);
					r[m] = madd(swr, qpr, a);
				}
				if (xtra) {
					T a = madd(rs0[n], rqm[n], rb[n]);
					a = madd(rs1[n], rqp[n], a);
					a = madd(rsw0[n], qm[K - 1], a);
					a = madd(rnw0[n + 1], rqm[n + 1], a);
					a = madd(rnw1[n], qp[K - 1], a);
					rx = madd(rsw1[n + 1], rqp[n + 1], a);
				}
			}
		}
		__syncthreads();  // the stage is read: the next line's rows may come in
		if (tid == 0 && li + G < nlines) issue(li + G);

		// 2a. forward substitution y(p) = r(p) - y(p-1) E(p)
		T A = T(1), B = T(0);
		if (has) {
#pragma unroll
			for (int m = 0; m < K; ++m) {
				const int pos = p0 + m;
				if (!full && (pos < 1 || pos > n)) continue;
				const T a = (!full && pos == 1) ? T(0) : -Ev[m];
				B = madd(a, B, r[m]);
				A = a * A;
			}
			if (xtra) {
				const T a = -Ex;
				B = madd(a, B, rx);
				A = a * A;
			}
		}
		T y = scan_incoming<T>(A, B, true, u, 1, CW, NWG, kgrp, warp, 1, sA, sB);
		if (has) {
#pragma unroll
			for (int m = 0; m < K; ++m) {
				const int pos = p0 + m;
				if (!full && (pos < 1 || pos > n)) continue;
				y = (!full && pos == 1) ? r[m] : madd(-y, Ev[m], r[m]);
				r[m] = y;
			}
			if (xtra) rx = pivot_div(madd(-y, Ex, rx), Dx);
#pragma unroll
			for (int m = 0; m < K; ++m) {
				const int pos = p0 + m;
				if (full || (pos >= 1 && pos <= n)) r[m] = pivot_div(r[m], dv[m]);
			}
		}
		// 2b. backward substitution x(p) = y(p)/D(p) - x(p+1) E(p+1)
		A = T(1);
		B = T(0);
		if (has) {
			if (xtra) {
				B = madd(T(0), B, rx);
				A = T(0) * A;
			}
#pragma unroll
			for (int m = K - 1; m >= 0; --m) {
				const int pos = p0 + m;
				if (!full && (pos < 1 || pos > n)) continue;
				const T e1 = m < K - 1 ? Ev[m + 1] : Enext;
				const T a = pos == n ? T(0) : -e1;
				B = madd(a, B, r[m]);
				A = a * A;
			}
		}
		if (NWG > 1) __syncthreads();  // the forward carries are still being read
		T x = scan_incoming<T>(A, B, false, u, 1, CW, NWG, kgrp, warp, 1, sA, sB);
		if (has) {
			if (xtra) x = rx;
#pragma unroll
			for (int m = K - 1; m >= 0; --m) {
				const int pos = p0 + m;
				if (!full && (pos < 1 || pos > n)) continue;
				const T e1 = m < K - 1 ? Ev[m + 1] : Enext;
				x = pos == n ? r[m] : madd(-x, e1, r[m]);
				r[m] = x;
			}
			// 3. write the line back
			T *qo = q + (size_t)lc * P;
			if (xtra) qo[n] = rx;
			if (full) vstore<T, K>(qo + p0, r);
			else {
#pragma unroll
				for (int m = 0; m < K; ++m) {
					const int pos = p0 + m;
					if (pos >= 1 && pos <= n) qo[pos] = r[m];
				}
			}
		}
	}
}


// Opt every line kernel into the large dynamic shared-memory carve-out once per
// process (before any graph capture: the solver calls this at creation).
int lines_prepare()
{
	static bool done = false;
	if (done) return CDR_OK;
	const int big = 227 * 1024;
#define CDR_LINES_ATTR(T, NS, DIR, EX) \
	CDR_CUDA_TRY(cudaFuncSetAttribute(k_lines<T, NS, DIR, EX>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))
	CDR_LINES_ATTR(double, 5, CDR_DIR_X, false); CDR_LINES_ATTR(double, 5, CDR_DIR_Y, false);
	CDR_LINES_ATTR(double, 3, CDR_DIR_X, false); CDR_LINES_ATTR(double, 3, CDR_DIR_Y, false);
	CDR_LINES_ATTR(float, 5, CDR_DIR_X, false); CDR_LINES_ATTR(float, 5, CDR_DIR_Y, false);
	CDR_LINES_ATTR(float, 3, CDR_DIR_X, false); CDR_LINES_ATTR(float, 3, CDR_DIR_Y, false);
	CDR_LINES_ATTR(double, 5, CDR_DIR_X, true); CDR_LINES_ATTR(double, 5, CDR_DIR_Y, true);
	CDR_LINES_ATTR(double, 3, CDR_DIR_X, true); CDR_LINES_ATTR(double, 3, CDR_DIR_Y, true);
	CDR_LINES_ATTR(float, 5, CDR_DIR_X, true); CDR_LINES_ATTR(float, 5, CDR_DIR_Y, true);
	CDR_LINES_ATTR(float, 3, CDR_DIR_X, true); CDR_LINES_ATTR(float, 3, CDR_DIR_Y, true);
#undef CDR_LINES_ATTR
#define CDR_XS_ATTR(T, NS, K) \
	CDR_CUDA_TRY(cudaFuncSetAttribute(k_lines_xstream<T, NS, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, XS_SMEM_MAX))
	CDR_XS_ATTR(float, 5, 8); CDR_XS_ATTR(float, 3, 8); CDR_XS_ATTR(double, 5, 4); CDR_XS_ATTR(double, 3, 4);
#undef CDR_XS_ATTR
	CDR_TRY(coarse_prepare());
	done = true;
	return CDR_OK;
}

// Lines per CTA: the largest power of two with G*n*sizeof(T) within the shared
// memory budget (x-lines: small, rows are contiguous; y-lines: at least 4 lines
// so that each row segment read is a useful 32-byte sector group).
template <typename T>
static int lines_per_cta(int n, int dir)
{
	const size_t budget = dir == CDR_DIR_X ? 32 * 1024 : (sizeof(T) == 8 ? 68 * 1024 : 68 * 1024);
	int G = 1;
	while (G < 32 && (size_t)(2 * G) * n * sizeof(T) <= budget) G *= 2;
	return G;
}

// ---------------------------------------------------------------- launch shapes
// The register-chunk kernel's shape: K elements per thread and, for y-lines,
// the CTA size cap (x-lines always run FAST_BLOCK_X threads).  The default is
// K = 8 (16 for FP32 y-lines longer than 1024 points) and the largest CTA;
// lines_autotune times the candidates on a level's own arrays at setup and
// records the fastest per (direction, type, stencil, n, lines, single problem
// or batch).  The
// record lives for the process, so every solver of one shape in a process
// runs the same launches (FP32 results depend on the chunking).
namespace {
struct LineKey {
	int dir, tsize, ns, n, nl, nb;
	bool operator<(const LineKey &o) const
	{
		return std::tie(dir, tsize, ns, n, nl, nb) < std::tie(o.dir, o.tsize, o.ns, o.n, o.nl, o.nb);
	}
};
std::mutex g_shape_mu;
std::map<LineKey, LineShape> &shape_table()
{
	static std::map<LineKey, LineShape> t;
	return t;
}
}  // namespace

template <typename T>
static LineShape default_shape(int n, int dir, int nb = 1)
{
	// FP32 x-lines longer than 1024 points: the streamed kernel (K = 8, the same
	// results as the register-chunk kernel; a batch or a misaligned level falls
	// back to that kernel with the same K)
	const int stream = dir == CDR_DIR_X && sizeof(T) == 4 && n > 1024 ? 1 : 0;
	if (dir == CDR_DIR_Y && sizeof(T) == 4) {
		// FP32 y-lines: for a single problem, K = 4 in small CTAs for short lines
		// (the shapes the timing picks there inside a cycle); K = 16 for lines
		// longer than 1024 points
		if (nb == 1 && n <= 160) return LineShape{4, 256, 0};
		if (nb == 1 && n <= 320) return LineShape{4, 128, 0};
		return LineShape{n > 8 * 128 ? 16 : 8, FAST_BLOCK_Y, 0};
	}
	return LineShape{8, FAST_BLOCK_Y, stream};
}

template <typename T>
static bool shape_ok(LineShape sh, int n, int dir)
{
	const bool kok = sizeof(T) == 4 ? (sh.K == 4 || sh.K == 8 || sh.K == 16) : (sh.K == 2 || sh.K == 4 || sh.K == 8);
	if (!kok || n > 256 * sh.K) return false;
	int tpl = 1;
	while (tpl * sh.K < n) tpl *= 2;
	if (dir == CDR_DIR_X) return tpl <= FAST_BLOCK_X && sh.cap >= 32;
	return sh.cap >= 32 && sh.cap <= FAST_BLOCK_Y && tpl <= sh.cap;
}

template <typename T>
static LineShape shape_for(int n, int nl, int ns, int nb, int dir)
{
	std::lock_guard<std::mutex> lk(g_shape_mu);
	auto it = shape_table().find(LineKey{dir, (int)sizeof(T), ns, n, nl, nb > 1 ? 2 : 1});
	return it == shape_table().end() ? default_shape<T>(n, dir, nb) : it->second;
}

template <typename T, int NS, int DIR, int K>
static int launch_fast(const T *so, T *x, const T *b, const T *sor, Dims2 d, int tpitch, int first, int nlines,
                       int cap, cudaStream_t st)
{
	const int n = DIR == CDR_DIR_X ? d.nx : d.ny;
	int tpl_log2 = 0;
	while ((1 << tpl_log2) * K < n) ++tpl_log2;  // chunks cover 0 .. n - 1, the last one also n
	const int TPL = 1 << tpl_log2;
	// x: cap CTA threads (at least one line, at most FAST_BLOCK_X); y: up to 32
	// lines, at most cap threads
	const int block = DIR == CDR_DIR_X ? std::min(FAST_BLOCK_X, std::max(TPL, cap)) : (TPL * 32 < cap ? TPL * 32 : cap);
	const int G = block / TPL;
	k_lines_fast<T, NS, DIR, K><<<dim3(ceil_div(nlines, G), 1, d.nb), block, 0, st>>>(so, x, b, sor, d, tpitch, first,
	                                                                                  tpl_log2);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

// The streamed x-line kernel: K = 8 (FP32) or 4 (FP64) elements per thread, one
// line per CTA step (TPL = 32 .. 256 threads), a single problem, both stages
// within the shared-memory budget.
template <typename T>
__host__ __device__ constexpr int xs_K()
{
	return sizeof(T) == 4 ? 8 : 4;
}

template <typename T, int NS>
static bool xs_ok(Dims2 d)
{
	const int K = xs_K<T>(), n = d.nx;
	return d.nb == 1 && n >= 32 * K && n <= XS_BLOCK * K && xs_smem<T, NS>(d.pitch) <= XS_SMEM_MAX;
}

// CTAs per SM of the streamed kernel for a (block, shared memory) pair, and the
// SM count: looked up once per pair
template <typename T, int NS>
static int xs_grid_cap(int block, size_t smem)
{
	static std::mutex mu;
	static std::map<std::pair<int, size_t>, int> cache;
	std::lock_guard<std::mutex> lk(mu);
	auto it = cache.find({block, smem});
	if (it != cache.end()) return it->second;
	int dev = 0, sms = 0, per_sm = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
	    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lines_xstream<T, NS, xs_K<T>()>, block, smem) != cudaSuccess)
		return 0;
	const int cap = sms * (per_sm > 0 ? per_sm : 1);
	cache[{block, smem}] = cap;
	return cap;
}

template <typename T, int NS>
static int launch_xstream(const T *so, T *x, const T *b, const T *sor, Dims2 d, int first, int nlines, cudaStream_t st)
{
	constexpr int K = xs_K<T>();
	int tpl = 1;
	while (tpl * K < d.nx) tpl *= 2;
	const size_t smem = xs_smem<T, NS>(d.pitch);
	CDR_TRY(lines_prepare());
	const int cap = xs_grid_cap<T, NS>(tpl, smem);
	if (cap <= 0) {
		set_error(CDR_ERR_CUDA, "occupancy query for the streamed line kernel failed");
		return CDR_ERR_CUDA;
	}
	const int grid = nlines < cap ? nlines : cap;
	k_lines_xstream<T, NS, K><<<grid, tpl, smem, st>>>(so, x, b, sor, d, first, nlines);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

template <typename T, int NS, int DIR>
static int launch_lines(const T *so, T *x, const T *b, const T *sor, Dims2 d, int tpitch, int first, bool exact,
                        cudaStream_t st, const LineShape *force = nullptr)
{
	const int n = DIR == CDR_DIR_X ? d.nx : d.ny;
	const int nl = DIR == CDR_DIR_X ? d.ny : d.nx;
	const int nlines = first > nl ? 0 : (nl - first) / 2 + 1;
	if (nlines == 0) return CDR_OK;
	// The register-chunk kernel reads whole 16-byte-aligned chunks of K elements:
	// rows (x) or factor lines (y) must have a pitch that is a multiple of K and
	// 16-byte aligned base pointers; lines up to 256*K - 1 points.
	const int fpitch = DIR == CDR_DIR_X ? d.pitch : tpitch;
	const bool aligned = ((uintptr_t)so | (uintptr_t)x | (uintptr_t)b | (uintptr_t)sor) % 16 == 0;
	LineShape sh = force ? *force : shape_for<T>(n, nl, NS, d.nb, DIR);
	if (!shape_ok<T>(sh, n, DIR)) sh = default_shape<T>(n, DIR, d.nb);
	if (!exact && aligned && d.pitch % 16 == 0 && fpitch % 16 == 0 && shape_ok<T>(sh, n, DIR)) {
		if constexpr (DIR == CDR_DIR_X)
			if (sh.stream && sh.K == xs_K<T>() && xs_ok<T, NS>(d))
				return launch_xstream<T, NS>(so, x, b, sor, d, first, nlines, st);
		if constexpr (sizeof(T) == 4) {
			if (sh.K == 4) return launch_fast<T, NS, DIR, 4>(so, x, b, sor, d, tpitch, first, nlines, sh.cap, st);
			if (sh.K == 16) return launch_fast<T, NS, DIR, 16>(so, x, b, sor, d, tpitch, first, nlines, sh.cap, st);
		} else {
			if (sh.K == 2) return launch_fast<T, NS, DIR, 2>(so, x, b, sor, d, tpitch, first, nlines, sh.cap, st);
			if (sh.K == 4) return launch_fast<T, NS, DIR, 4>(so, x, b, sor, d, tpitch, first, nlines, sh.cap, st);
		}
		return launch_fast<T, NS, DIR, 8>(so, x, b, sor, d, tpitch, first, nlines, sh.cap, st);
	}
	const int G = lines_per_cta<T>(n, DIR);
	size_t smem = sizeof(T) * (2 * LT + (size_t)G * n);
	if (smem > 227 * 1024) {
		set_error(CDR_ERR_DIM, "line length %d too long for one CTA", n);
		return CDR_ERR_DIM;
	}
	CDR_TRY(lines_prepare());
	const dim3 grd(ceil_div(nlines, G), 1, d.nb);
	if (exact) k_lines<T, NS, DIR, true><<<grd, LT, smem, st>>>(so, x, b, sor, d, tpitch, first, G);
	else k_lines<T, NS, DIR, false><<<grd, LT, smem, st>>>(so, x, b, sor, d, tpitch, first, G);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

template <typename T, int NS, int DIR>
static int tune_dir(const T *so, T *x, const T *b, const T *sor, Dims2 d, int tpitch, cudaStream_t st)
{
	const int n = DIR == CDR_DIR_X ? d.nx : d.ny;
	const int nl = DIR == CDR_DIR_X ? d.ny : d.nx;
	const LineKey key{DIR, (int)sizeof(T), NS, n, nl, d.nb > 1 ? 2 : 1};
	{
		std::lock_guard<std::mutex> lk(g_shape_mu);
		if (shape_table().count(key)) return CDR_OK;
	}
	// FP32 results depend on K (and, for y-lines, on the lines per CTA) through
	// the order in which the scans compose their maps, and the FP32 cycle's
	// outer iteration count moves with that rounding: for a single problem,
	// FP32 x-lines try only shapes with the default K (bit-identical among
	// themselves) and FP32 y-lines keep the default, so that every run of an FP32
	// solve gives the same bits.  Batches (many small problems, or the planes of
	// a 3D plane smoother) time every candidate.
	const int kdef = default_shape<T>(n, DIR, d.nb).K;
	const bool fixed_bits = sizeof(T) == 4 && d.nb == 1;
	if (fixed_bits && DIR == CDR_DIR_Y) {
		std::lock_guard<std::mutex> lk(g_shape_mu);
		shape_table()[key] = default_shape<T>(n, DIR, d.nb);
		return CDR_OK;
	}
	const int ks[3] = {sizeof(T) == 4 ? 4 : 2, sizeof(T) == 4 ? 8 : 4, sizeof(T) == 4 ? 16 : 8};
	// small CTAs spread the few lines of a coarse level over more SMs
	const int caps[6] = {32, 64, 128, 256, 512, FAST_BLOCK_Y};
	// Each candidate is timed on one sweep (both colours) after L2 has been
	// overwritten, best of three: the sweep of a level inside a cycle finds its
	// arrays in DRAM, and a level that fits in L2 would otherwise favour shapes
	// that only win on L2-resident data.
	int dev = 0, l2 = 0;
	CDR_CUDA_TRY(cudaGetDevice(&dev));
	CDR_CUDA_TRY(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
	const size_t flush_bytes = 2 * (size_t)(l2 > 0 ? l2 : 128 << 20);
	void *flush = nullptr;
	if (cudaMalloc(&flush, flush_bytes) != cudaSuccess) {  // no room: time without the flush
		cudaGetLastError();
		flush = nullptr;
	}
	cudaEvent_t e0, e1;
	CDR_CUDA_TRY(cudaEventCreate(&e0));
	CDR_CUDA_TRY(cudaEventCreate(&e1));
	int rc = CDR_OK;
	auto time_shape = [&](const LineShape &sh) -> float {
		float ms = 1e30f;
		for (int rep = 0; rep < 3 && rc == CDR_OK; ++rep) {
			if ((flush && cudaMemsetAsync(flush, rep, flush_bytes, st) != cudaSuccess) ||
			    cudaEventRecord(e0, st) != cudaSuccess) {
				rc = CDR_ERR_CUDA;
				break;
			}
			for (int f = 1; f <= 2 && rc == CDR_OK; ++f) rc = launch_lines<T, NS, DIR>(so, x, b, sor, d, tpitch, f, false, st, &sh);
			if (rc != CDR_OK) break;
			float t = 0.f;
			if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
			    cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) {
				rc = CDR_ERR_CUDA;
				break;
			}
			ms = t < ms ? t : ms;
		}
		return ms;
	};
	// the default shape stands unless a candidate is at least 5 % faster (10 %
	// for a level larger than a quarter of L2: single cold sweeps of those vary
	// by a few per cent from run to run)
	const size_t level_bytes = 12 * d.plane() * sizeof(T) * (size_t)d.nb;
	const float margin = 4 * level_bytes > flush_bytes / 2 ? 0.90f : 0.95f;
	LineShape best = default_shape<T>(n, DIR, d.nb);
	float best_ms = time_shape(best);
	for (int a = 0; a < 3 && rc == CDR_OK; ++a)
		for (int c = 0; c < (DIR == CDR_DIR_X ? 4 : 6) && rc == CDR_OK; ++c) {
			const LineShape sh{ks[a], caps[c]};
			if (!shape_ok<T>(sh, n, DIR) || (fixed_bits && sh.K != kdef)) continue;
			const float ms = time_shape(sh);
			if (ms < margin * best_ms) { best_ms = ms; best = sh; }
		}
	if (DIR == CDR_DIR_X && rc == CDR_OK && xs_ok<T, NS>(d) && (!fixed_bits || xs_K<T>() == kdef)) {
		const LineShape sh{xs_K<T>(), FAST_BLOCK_X, 1};
		const float ms = time_shape(sh);
		if (ms < margin * best_ms) { best_ms = ms; best = sh; }
	}
	cudaStreamSynchronize(st);
	if (flush) cudaFree(flush);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if (rc != CDR_OK) return rc;
	std::lock_guard<std::mutex> lk(g_shape_mu);
	shape_table()[key] = best;
	return CDR_OK;
}

template <typename T>
int lines_autotune(const T *so, int nstencil, T *x, const T *b, const T *sor, Dims2 d, int tpitch, int dir,
                   cudaStream_t st)
{
	if (dir == CDR_DIR_X) {
		if (nstencil == 5) return tune_dir<T, 5, CDR_DIR_X>(so, x, b, sor, d, tpitch, st);
		return tune_dir<T, 3, CDR_DIR_X>(so, x, b, sor, d, tpitch, st);
	}
	if (nstencil == 5) return tune_dir<T, 5, CDR_DIR_Y>(so, x, b, sor, d, tpitch, st);
	return tune_dir<T, 3, CDR_DIR_Y>(so, x, b, sor, d, tpitch, st);
}
template int lines_autotune<double>(const double *, int, double *, const double *, const double *, Dims2, int, int,
                                    cudaStream_t);
template int lines_autotune<float>(const float *, int, float *, const float *, const float *, Dims2, int, int,
                                   cudaStream_t);

bool lines_set_shape(int dir, int tsize, int ns, int n, int nl, int nb, LineShape sh)
{
	bool ok;
	if (tsize == 4) ok = shape_ok<float>(sh, n, dir);
	else ok = shape_ok<double>(sh, n, dir);
	if (sh.stream) ok = dir == CDR_DIR_X && nb == 1 && sh.K == (tsize == 4 ? 8 : 4);
	if (!ok) return false;
	std::lock_guard<std::mutex> lk(g_shape_mu);
	shape_table()[LineKey{dir, tsize, ns, n, nl, nb > 1 ? 2 : 1}] = sh;
	return true;
}

bool lines_shape(int dir, int tsize, int ns, int n, int nl, int nb, LineShape *out)
{
	std::lock_guard<std::mutex> lk(g_shape_mu);
	auto it = shape_table().find(LineKey{dir, tsize, ns, n, nl, nb > 1 ? 2 : 1});
	if (it == shape_table().end()) return false;
	*out = it->second;
	return true;
}

template <typename T>
int relax_lines_2d(const T *so, int nstencil, T *x, const T *b, const T *sor, Dims2 d, int tpitch, int dir,
                   int updown, int flags, cudaStream_t st)
{
	const bool exact = (flags & CDR_LINES_EXACT) != 0;
	const LineShape dflt = default_shape<T>(dir == CDR_DIR_X ? d.nx : d.ny, dir, d.nb);
	const LineShape streamed{xs_K<T>(), FAST_BLOCK_X, 1};
	const LineShape *force = (flags & CDR_LINES_NOTUNE) ? &dflt : nullptr;
	if ((flags & CDR_LINES_STREAM) && dir == CDR_DIR_X) force = &streamed;
	// DOWN: lines with Fortran start index 3 (0-based even) first, then 2 (odd);
	// UP: the opposite (relax_lines_x.f90:82-97).
	const int firsts[2] = {updown == CDR_DOWN ? 2 : 1, updown == CDR_DOWN ? 1 : 2};
	for (int c = 0; c < 2; ++c) {
		int f = firsts[c];
		if (dir == CDR_DIR_X) {
			if (nstencil == 5) CDR_TRY((launch_lines<T, 5, CDR_DIR_X>(so, x, b, sor, d, tpitch, f, exact, st, force)));
			else CDR_TRY((launch_lines<T, 3, CDR_DIR_X>(so, x, b, sor, d, tpitch, f, exact, st, force)));
		} else {
			if (nstencil == 5) CDR_TRY((launch_lines<T, 5, CDR_DIR_Y>(so, x, b, sor, d, tpitch, f, exact, st, force)));
			else CDR_TRY((launch_lines<T, 3, CDR_DIR_Y>(so, x, b, sor, d, tpitch, f, exact, st, force)));
		}
	}
	return CDR_OK;
}
template int relax_lines_2d<double>(const double *, int, double *, const double *, const double *, Dims2, int, int,
                                    int, int, cudaStream_t);
template int relax_lines_2d<float>(const float *, int, float *, const float *, const float *, Dims2, int, int, int,
                                   int, cudaStream_t);

}  // namespace cdrgpu
