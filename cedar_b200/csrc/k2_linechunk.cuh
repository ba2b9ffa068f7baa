// k2_linechunk.cuh -- the register-chunk zebra line sweep of one line and its
// scan (device code of the line kernels in k2_lines.cu), and the launch-shape
// rules that fix its chunks per line length.
#pragma once
#include "k2_point.cuh"

namespace cdrgpu {

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

// vload through L2 only (values other CTAs have written since the launch began)
template <typename T, int K, bool CG>
__device__ __forceinline__ void vload_q(const T *__restrict__ p, T (&v)[K])
{
	if constexpr (!CG) {
		vload<T, K>(p, v);
	} else {
		using VT = typename Vec16<T>::type;
		constexpr int W = 16 / sizeof(T);
		const VT *pv = reinterpret_cast<const VT *>(p);
#pragma unroll
		for (int c = 0; c < K / W; ++c) {
			VT t = __ldcg(pv + c);
			const T *e = reinterpret_cast<const T *>(&t);
#pragma unroll
			for (int w = 0; w < W; ++w) v[c * W + w] = e[w];
		}
	}
}

// compose (A,B) <- (A,B) o (a2,b2): apply (a2,b2) first
template <typename T>
__device__ __forceinline__ void after(T &A, T &B, T a2, T b2)
{
	B = madd(A, b2, B);
	A = A * a2;
}

// Incoming value of a chunk (its exclusive prefix map applied to 0) by a tree
// fixed over chunk indices, so that the bits do not depend on how the chunks
// of a line are laid over lanes, warps and CTAs: positions s along the scan
// direction (s = t forward, TPL - 1 - t backward) form groups of SG = 4; an
// inclusive Kogge-Stone scan inside each group (warp shuffles, partner s - o
// for o = 1, 2), then a scan of the ng <= 64 group totals by one warp per line
// through shared memory (ng <= 32: Kogge-Stone over the groups, o = 1 .. 16;
// else lane k pairs groups 2k and 2k + 1 and the Kogge-Stone runs over the
// pairs), and the chunk's incoming map is its in-group exclusive prefix
// composed after the prefix of the groups before it.  LS is the lane distance
// between consecutive chunks of a line (groups must lie inside a warp:
// SG * LS <= 32, or the whole line when TPL <= SG); `line` indexes the line
// among the CTA's nlines; gA/gB hold nlines * ng entries.  Every thread of the
// CTA calls it (threads of no chunk with identity maps): the __syncthreads
// are uniform.
constexpr int SG = 4;

template <typename T>
__device__ __forceinline__ T canon_incoming(T A, T B, bool forward, int t, int TPL, int LS, int line, int nlines,
                                            T *gA, T *gB)
{
	const unsigned full = 0xffffffffu;
	const int s = forward ? t : TPL - 1 - t;
	const int u = s & (SG - 1);
#pragma unroll
	for (int o = 1; o < SG; o <<= 1) {
		const T a2 = forward ? __shfl_up_sync(full, A, o * LS) : __shfl_down_sync(full, A, o * LS);
		const T b2 = forward ? __shfl_up_sync(full, B, o * LS) : __shfl_down_sync(full, B, o * LS);
		if (u >= o && s < TPL) after(A, B, a2, b2);
	}
	T ae = forward ? __shfl_up_sync(full, A, LS) : __shfl_down_sync(full, A, LS);
	T be = forward ? __shfl_up_sync(full, B, LS) : __shfl_down_sync(full, B, LS);
	if (u == 0) {
		ae = T(1);
		be = T(0);
	}
	const int ng = (TPL + SG - 1) / SG;
	if (ng == 1) return be;
	const bool real = t < TPL && line < nlines;
	__syncthreads();  // earlier readers of gA / gB are done
	if (real && (u == SG - 1 || s == TPL - 1)) {
		gA[line * ng + s / SG] = A;
		gB[line * ng + s / SG] = B;
	}
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
	for (int l = warp; l < nlines; l += nw) {
		T *la = gA + l * ng, *lb = gB + l * ng;
		if (ng <= 32) {
			T ga = lane < ng ? la[lane] : T(1), gb = lane < ng ? lb[lane] : T(0);
#pragma unroll
			for (int o = 1; o < 32; o <<= 1) {
				const T a2 = __shfl_up_sync(full, ga, o), b2 = __shfl_up_sync(full, gb, o);
				if (lane >= o) after(ga, gb, a2, b2);
			}
			if (lane < ng) {
				la[lane] = ga;
				lb[lane] = gb;
			}
		} else {
			const int k0 = 2 * lane, k1 = k0 + 1;
			const T a0 = k0 < ng ? la[k0] : T(1), b0 = k0 < ng ? lb[k0] : T(0);
			const T a1 = k1 < ng ? la[k1] : T(1), b1 = k1 < ng ? lb[k1] : T(0);
			T pa = a1, pb = b1;  // the pair: group 2k+1 after group 2k
			after(pa, pb, a0, b0);
#pragma unroll
			for (int o = 1; o < 32; o <<= 1) {
				const T a2 = __shfl_up_sync(full, pa, o), b2 = __shfl_up_sync(full, pb, o);
				if (lane >= o) after(pa, pb, a2, b2);
			}
			T ea = __shfl_up_sync(full, pa, 1), eb = __shfl_up_sync(full, pb, 1);
			if (lane == 0) {
				ea = T(1);
				eb = T(0);
			}
			T qa = a0, qb = b0;  // group 2k after the pairs before it
			after(qa, qb, ea, eb);
			if (k0 < ng) {
				la[k0] = qa;
				lb[k0] = qb;
			}
			if (k1 < ng) {
				la[k1] = pa;
				lb[k1] = pb;
			}
		}
	}
	__syncthreads();
	const int k = s / SG;
	if (k == 0 || !real) return be;
	return madd(ae, gB[line * ng + k - 1], be);
}

constexpr int FAST_BLOCK_X = 256, FAST_BLOCK_Y = 1024;

// G lines of one colour per CTA.  x-lines: thread tid works on chunk
// t = tid % TPL of line g = tid / TPL (blockDim = G * TPL); y-lines: chunk
// t = tid / G of line g = tid % G (blockDim >= G * TPL, a multiple of 32; the
// threads beyond G * TPL hold no chunk).  G * SG <= 32 for y-lines unless
// TPL <= SG (the scan's groups lie inside a warp): a warp then reads 8 lines,
// 16 columns of one row (two 32-byte sectors), per row of its chunks.
// CTA thread bound of the y-line kernel: 1024 (FP32) or 512 (FP64) threads
template <typename T>
__host__ __device__ constexpr int yblock_max()
{
	return sizeof(T) == 4 ? FAST_BLOCK_Y : FAST_BLOCK_Y / 2;
}

// Right-hand side of a y-line at (i, j) (relax_lines_y.f90:102-106 operand
// order, as line_rhs); CG reads x through L2 only (values other CTAs of the
// same launch have written).
template <typename T, int NS, bool CG>
__device__ __forceinline__ T yline_rhs(const T *__restrict__ so, size_t ps, const T *__restrict__ q,
                                       const T *__restrict__ qf, size_t k, int p)
{
	auto Q = [&](size_t i) -> T {
		if constexpr (CG) return __ldcg(q + i);
		else return q[i];
	};
	const T *w = so + ps;
	T a = madd(w[k], Q(k - 1), qf[k]);
	a = madd(w[k + 1], Q(k + 1), a);
	if (NS == 5) {
		const T *sw = so + 3 * ps, *nw = so + 4 * ps;
		a = madd(sw[k], Q(k - p - 1), a);
		a = madd(nw[k + 1], Q(k - p + 1), a);
		a = madd(nw[k + p], Q(k + p - 1), a);
		a = madd(sw[k + p + 1], Q(k + p + 1), a);
	}
	return a;
}

// One chunk (t of TPL) of line lc (0: none) of the CTA's G lines, the whole
// sweep of a line: right-hand sides, both substitutions by the scans, write
// back.  g is the line's slot among the CTA's lines; sA/sB hold G*TPL/SG
// scan totals.  Every thread of the CTA calls it.  CG: the iterate is
// read through L2 only (other CTAs of the launch have written it since).
// ZERO: the iterate is zero on entry (its interior is not read), as at the
// first sweep after a coarse-grid iterate is cleared.  nslots: line slots of
// the CTA's scans when it holds several groups of G y-lines (g is then the
// slot, G the lines of one group: the lane distance of a line's chunks).
// PACK (y-lines): yc holds the lines' couplings in line order
// (pack_ylines_2d), read as vectors.
template <typename T, int NS, int DIR, int K, bool CG = false, bool ZERO = false, bool PACK = false,
          bool XL = DIR == CDR_DIR_X>
__device__ __forceinline__ void line_chunk(const T *__restrict__ so, T *__restrict__ q, const T *__restrict__ qf,
                                           const T *__restrict__ sor, const Dims2 &d, int tpitch, int lc, int g,
                                           int t, int TPL, int G, T *sA, T *sB, int nslots = 0,
                                           const T *__restrict__ yc = nullptr)
{
	const int NL = nslots > 0 ? nslots : G;  // line slots of the CTA's scans (g < NL)
	const int n = DIR == CDR_DIR_X ? d.nx : d.ny;
	const int nl = DIR == CDR_DIR_X ? d.ny : d.nx;
	const bool active = lc >= 1 && lc <= nl;
	const int p0 = t * K;
	const bool has = active && t < TPL && p0 <= n;
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
	if (has && ZERO) {
		// the iterate is zero: the right-hand side is b (b + a 0 for every
		// coupling a, up to the sign of an exact zero); nothing else is read
		if (DIR == CDR_DIR_X) {
			const size_t k0 = d.at(p0, lc);
			vload<T, K>(qf + k0, r);
			if (xtra) rx = qf[k0 + K];
		} else {
#pragma unroll
			for (int m = 0; m < K; ++m) {
				const int jj = p0 + m;
				if (jj < 1 || jj > n) continue;
				r[m] = qf[d.at(lc, jj)];
			}
			if (xtra) rx = qf[d.at(lc, n)];
		}
	} else if (has) {
		if (DIR == CDR_DIR_X) {
			// operand order of relax_lines_x.f90:106-110, in stages so that only
			// the two neighbour rows and one coupling row are live at a time
			const size_t k0 = d.at(p0, lc);
			const T *w = so + ps, *s = so + 2 * ps, *sw = so + 3 * ps, *nw = so + 4 * ps;
			auto Q = [&](size_t i) -> T {
				if constexpr (CG) return __ldcg(q + i);
				else return q[i];
			};
			T qm[K], qp[K], c[K];
			vload<T, K>(qf + k0, r);
			vload_q<T, K, CG>(q + k0 - P, qm);
			vload<T, K>(s + k0, c);
#pragma unroll
			for (int m = 0; m < K; ++m) r[m] = madd(c[m], qm[m], r[m]);
			vload_q<T, K, CG>(q + k0 + P, qp);
			vload<T, K>(s + k0 + P, c);
#pragma unroll
			for (int m = 0; m < K; ++m) r[m] = madd(c[m], qp[m], r[m]);
			const size_t kx = k0 + K;  // position n when xtra
			if (xtra) rx = madd(s[kx + P], Q(kx + P), madd(s[kx], Q(kx - P), qf[kx]));
			if (NS == 5) {
				const T qm_l = p0 >= 1 ? Q(k0 - P - 1) : T(0), qp_l = p0 >= 1 ? Q(k0 + P - 1) : T(0);
				const bool rin = p0 + K <= n + 1;
				const T qm_r = rin ? Q(k0 - P + K) : T(0), qp_r = rin ? Q(k0 + P + K) : T(0);
				vload<T, K>(sw + k0, c);
#pragma unroll
				for (int m = 0; m < K; ++m) r[m] = madd(c[m], m > 0 ? qm[m - 1] : qm_l, r[m]);
				vload<T, K>(nw + k0, c);
				const T nw0_r = rin ? nw[k0 + K] : T(0);
#pragma unroll
				for (int m = 0; m < K; ++m) r[m] = madd(m < K - 1 ? c[m + 1] : nw0_r, m < K - 1 ? qm[m + 1] : qm_r, r[m]);
				vload<T, K>(nw + k0 + P, c);
#pragma unroll
				for (int m = 0; m < K; ++m) r[m] = madd(c[m], m > 0 ? qp[m - 1] : qp_l, r[m]);
				vload<T, K>(sw + k0 + P, c);
				const T sw1_r = rin ? sw[k0 + P + K] : T(0);
#pragma unroll
				for (int m = 0; m < K; ++m) r[m] = madd(m < K - 1 ? c[m + 1] : sw1_r, m < K - 1 ? qp[m + 1] : qp_r, r[m]);
				if (xtra) {
					T a = madd(s[kx], Q(kx - P), qf[kx]);
					a = madd(s[kx + P], Q(kx + P), a);
					a = madd(sw[kx], qm[K - 1], a);
					a = madd(nw[kx + 1], Q(kx - P + 1), a);
					a = madd(nw[kx + P], qp[K - 1], a);
					rx = madd(sw[kx + P + 1], Q(kx + P + 1), a);
				}
			}
		} else if constexpr (PACK) {
			// yline_rhs's operations in its order, the couplings from the line's
			// packed planes (vector loads), the neighbour columns' rows loaded once
			// per half-chunk of 8 positions
			auto Q = [&](size_t e) -> T {
				if constexpr (CG) return __ldcg(q + e);
				else return q[e];
			};
			const size_t fps = (size_t)tpitch * (d.nx + 2);
			// the problem's planes of packed couplings, line lc: plane m at cpl + m * fps
			const T *cpl = yc + d.bofs((size_t)(NS == 5 ? 6 : 2) * fps) + (size_t)lc * tpitch;
			const size_t kq = d.at(lc, 0);
			constexpr int H = 8;
			static_assert(K % H == 0, "half-chunks of 8");
#pragma unroll
			for (int h = 0; h < K; h += H) {
				T qL[H + 2], qR[H + 2];  // columns lc - 1 and lc + 1, rows p0 + h - 1 .. p0 + h + H
#pragma unroll
				for (int e = 0; e < H + 2; ++e) {
					const int row = p0 + h - 1 + e;
					const bool in = row >= 0 && row <= n + 1;
					qL[e] = in ? Q(kq + (size_t)row * P - 1) : T(0);
					qR[e] = in ? Q(kq + (size_t)row * P + 1) : T(0);
				}
				T a[H], c[H];
#pragma unroll
				for (int m = 0; m < H; ++m) {
					const int pos = p0 + h + m;
					a[m] = pos >= 1 && pos <= n ? qf[kq + (size_t)pos * P] : T(0);
				}
				vload<T, H>(cpl + p0 + h, c);  // w(i, j)
#pragma unroll
				for (int m = 0; m < H; ++m) a[m] = madd(c[m], qL[m + 1], a[m]);
				vload<T, H>(cpl + fps + p0 + h, c);  // w(i+1, j)
#pragma unroll
				for (int m = 0; m < H; ++m) a[m] = madd(c[m], qR[m + 1], a[m]);
				if (NS == 5) {
					vload<T, H>(cpl + 2 * fps + p0 + h, c);  // sw(i, j)
#pragma unroll
					for (int m = 0; m < H; ++m) a[m] = madd(c[m], qL[m], a[m]);
					vload<T, H>(cpl + 3 * fps + p0 + h, c);  // nw(i+1, j)
#pragma unroll
					for (int m = 0; m < H; ++m) a[m] = madd(c[m], qR[m], a[m]);
					vload<T, H>(cpl + 4 * fps + p0 + h, c);  // nw(i, j+1)
#pragma unroll
					for (int m = 0; m < H; ++m) a[m] = madd(c[m], qL[m + 2], a[m]);
					vload<T, H>(cpl + 5 * fps + p0 + h, c);  // sw(i+1, j+1)
#pragma unroll
					for (int m = 0; m < H; ++m) a[m] = madd(c[m], qR[m + 2], a[m]);
				}
#pragma unroll
				for (int m = 0; m < H; ++m) r[h + m] = a[m];
			}
			if (xtra) rx = yline_rhs<T, NS, CG>(so, ps, q, qf, d.at(lc, n), P);
		} else {
			const int i = lc;
#pragma unroll
			for (int m = 0; m < K; ++m) {
				const int jj = p0 + m;
				if (jj < 1 || jj > n) continue;
				r[m] = yline_rhs<T, NS, CG>(so, ps, q, qf, d.at(i, jj), P);
			}
			if (xtra) rx = yline_rhs<T, NS, CG>(so, ps, q, qf, d.at(i, n), P);
		}
	}

	const int LS = XL ? 1 : G;  // lane distance of consecutive chunks of a line
	const bool full = p0 >= 1 && p0 + K - 1 <= n;  // no ghost or beyond-end position in the chunk

	// 2a. forward substitution y(p) = r(p) - y(p-1) E(p)
	T Ev[K];
	if (has) vload<T, K>(E + p0, Ev);
	// short chunks: the pivots are loaded here too, before the scan's barriers
	constexpr bool PRED = K <= 8;
	T Dv[PRED ? K : 1];
	if constexpr (PRED)
		if (has) vload<T, K>(D + p0, Dv);
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
	T y = canon_incoming<T>(A, B, true, t, TPL, LS, g, NL, sA, sB);
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
			if constexpr (PRED) {
#pragma unroll
				for (int w = 0; w < W; ++w) dv[w] = Dv[c * W + w];
			} else {
				vload<T, W>(D + p0 + c * W, dv);
			}
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
	T x = canon_incoming<T>(A, B, false, t, TPL, LS, g, NL, sA, sB);
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

// Elements per thread of the register-chunk kernels for lines of n points in
// direction dir (0: none): 8 up to 2048 points, with y-lines of more than 1024
// points at 16 (a whole line within 128 threads, so that a CTA holds the 8
// lines a warp's row reads need), and 16 up to 4096 (FP32 x-lines, y-lines).
// K depends on the line only, so the chunks of a line and the scan's tree over
// them (and with them every bit of a sweep) are the same for every launch shape.
template <typename T>
__host__ __device__ inline int canon_K(int n, int dir)
{
	if (dir == CDR_DIR_Y && n > 1024 && n <= 16 * 256) return 16;
	if (n <= 8 * 256) return 8;
	if (sizeof(T) == 4 && n <= 16 * 256) return 16;
	return 0;
}

// log2 of the threads of a line: chunks cover 0 .. n - 1, the last one also n
__host__ __device__ inline int tpl_log2_of(int n, int K)
{
	int l = 0;
	while ((1 << l) * K < n) ++l;
	return l;
}

// y-lines per CTA for a CTA thread cap: the scan's groups of SG chunks must lie
// inside a warp (G * SG <= 32), or the whole line when TPL <= SG
__host__ __device__ inline int ylines_per_cta(int TPL, int cap)
{
	const int gmax = TPL > SG ? 32 / SG : 32 / TPL;  // at most 8 (TPL > 4) or 32 lines
	int G = cap / TPL;
	if (G < 1) G = 1;
	if (G > gmax) G = gmax;
	return G;
}

}  // namespace cdrgpu
