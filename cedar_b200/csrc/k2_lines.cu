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
#include "k2_linechunk.cuh"
#include "k2_point.cuh"
#include "kernels2d.cuh"

namespace cdrgpu {

constexpr int LT = 256;  // threads per CTA
// FP32 y-line CTAs of at most this many threads run a kernel instance built
// for two such CTAs per SM (up to 128 registers per thread instead of 64)
constexpr int YSMALL_BLOCK = 256;

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


// The register-chunk sweep of a line (line_chunk) and its scan: k2_linechunk.cuh.

// G lines of one colour per CTA.  x-lines: thread tid works on chunk
// t = tid % TPL of line g = tid / TPL (blockDim = G * TPL); y-lines: chunk
// t = tid / G of line g = tid % G (blockDim >= G * TPL, a multiple of 32; the
// threads beyond G * TPL hold no chunk).  G * SG <= 32 for y-lines unless
// TPL <= SG (the scan's groups lie inside a warp): a warp then reads 8 lines,
// 16 columns of one row (two 32-byte sectors), per row of its chunks.
template <typename T, int NS, int DIR, int K, int LB = 0, bool ZERO = false, bool PACK = false,
          bool XL = DIR == CDR_DIR_X>
__global__ void __launch_bounds__(XL ? FAST_BLOCK_X : (LB ? LB : yblock_max<T>()), XL || LB ? 2 : 1)
    k_lines_fast(const T *__restrict__ so, T *__restrict__ q, const T *__restrict__ qf, const T *__restrict__ sor,
                 Dims2 d, int tpitch, int first, int tpl_log2, int G, const T *__restrict__ yc)
{
	// group totals of the scans: lines * groups = blockDim / SG at most
	__shared__ T sA[FAST_BLOCK_Y / SG], sB[FAST_BLOCK_Y / SG];
	const int TPL = 1 << tpl_log2;
	const int tid = threadIdx.x;
	int g, t;
	if (XL) { g = tid >> tpl_log2; t = tid & (TPL - 1); }
	else { g = tid % G; t = tid / G; }
	line_chunk<T, NS, DIR, K, false, ZERO, PACK>(so, q, qf, sor, d, tpitch, first + 2 * (blockIdx.x * G + g), g, t,
	                                             TPL, G, sA, sB, 0, yc);
}

// Give-ups of the bounded waits of the line kernels (streamed x-lines, the
// fused y-line sweep) and the limit of those waits (device globals).
namespace {
__device__ unsigned g_xstream_timeouts;
__device__ unsigned long long g_xstream_wait_ns = kWaitLimitNs;
}  // namespace
static_assert(kStreamWaitDefaultNs == kWaitLimitNs, "one default wait limit");

// ------------------------------------------------- both colours in one launch
// y-line sweep of a single problem, both colours in one launch.  Columns are
// taken in pairs (p2, p1 = p2 + 1), p1 of the colour swept first; virtual
// block vb (a ticket drawn at start, so that vb - 1 is already running) owns
// pairs vb*G .. vb*G + G - 1.  Phase 1 solves its p1 lines, which read the
// old x of the p2 columns beside them (its own and the next block's first);
// phase 2 solves its p2 lines, which read the new x of the p1 columns (its
// own and the previous block's last).  Between the phases the block raises
// its flag and waits for block vb - 1's: that block has then written its last
// p1 line and read the old x of our first p2 line, which phase 2 overwrites.
// The waiting block resets the flag it consumed, and the last block raises
// none, so all flags are 0 again when the launch ends.  Every coupling column
// is read by phase 1 and again, moments later, by phase 2 of the same or the
// next block: the second read comes from L2, so the sweep moves each array
// through DRAM about once instead of once per colour.  Each line gets the
// arithmetic of line_chunk: the result equals two k_lines_fast launches bit for
// bit.  sync[0] is the ticket counter, sync[1 + vb] block vb's flag.  The wait
// is bounded (g_xstream_wait_ns); a block that gives up counts itself in
// g_xstream_timeouts and leaves its p2 lines unsolved.
namespace {
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
	unsigned v;
	asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}
}  // namespace

template <typename T, int NS, int K, int LB = 0, bool Z1 = false, bool PK = false>
__global__ void __launch_bounds__(LB ? LB : yblock_max<T>(), LB ? 2 : 1)
    k_ylines_pair(const T *__restrict__ so, T *__restrict__ q, const T *__restrict__ qf, const T *__restrict__ sor,
                  Dims2 d, int tpitch, int c2, int tpl_log2, int G, unsigned *__restrict__ sync, int nvb,
                  const T *__restrict__ yc)
{
	__shared__ T sA[FAST_BLOCK_Y / SG], sB[FAST_BLOCK_Y / SG];
	__shared__ int s_vb, s_ok;
	const int TPL = 1 << tpl_log2;
	const int tid = threadIdx.x, g = tid % G, t = tid / G;
	if (tid == 0) {
		const unsigned v = atomicAdd(&sync[0], 1u);
		if (v == gridDim.x - 1) atomicExch(&sync[0], 0u);  // every block has its ticket
		s_vb = (int)v;
	}
	__syncthreads();
	const int vb = s_vb;
	const int p2 = 2 * (vb * G + g) + c2, p1 = p2 + 1;
	line_chunk<T, NS, CDR_DIR_Y, K, false, Z1, PK && !Z1>(so, q, qf, sor, d, tpitch, p1, g, t, TPL, G, sA, sB, 0, yc);
	__threadfence();  // this thread's phase-1 lines reach L2 before phase 2 reads them there
	__syncthreads();  // phase 1 read and written by every thread
	if (tid == 0) {
		int ok = 1;
		if (vb + 1 < nvb) {
			__threadfence();
			atomicExch(&sync[1 + vb], 1u);
		}
		if (vb > 0) {
			const unsigned long long limit = g_xstream_wait_ns;
			ok = 0;
			if (limit > 0) {
				const unsigned long long t0 = globaltimer_ns();
				for (int it = 0; it < (1 << 22); ++it) {
					if (ld_acquire(&sync[vb])) { ok = 1; break; }
					if (globaltimer_ns() - t0 > limit) break;
					__nanosleep(64);
				}
			}
			if (ok) {
				atomicExch(&sync[vb], 0u);
				__threadfence();
			} else {
				atomicAdd(&g_xstream_timeouts, 1u);
			}
		}
		s_ok = ok;
	}
	__syncthreads();
	if (!s_ok) return;
	line_chunk<T, NS, CDR_DIR_Y, K, true, false, PK>(so, q, qf, sor, d, tpitch, p2, g, t, TPL, G, sA, sB, 0, yc);
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
	__shared__ T sA[XS_BLOCK / SG], sB[XS_BLOCK / SG];  // group totals of the scans
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
		T y = canon_incoming<T>(A, B, true, tid, TPL, 1, 0, 1, sA, sB);
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
		T x = canon_incoming<T>(A, B, false, tid, TPL, 1, 0, 1, sA, sB);
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
	CDR_XS_ATTR(float, 5, 8); CDR_XS_ATTR(float, 3, 8);
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
// The register-chunk kernels run K elements per thread with K fixed by the
// line length (8 up to 2048 points, 16 up to 4096 for FP32), so the chunks of
// a line, and with them the scan's tree and every bit of the result, are the
// same whatever the launch shape.  The shape is then free: the CTA size (x) or
// the lines per CTA (y), and for x-lines the streamed kernel.  lines_autotune
// times the candidates on a level's own arrays at setup and records the
// fastest per (direction, type, stencil, n, lines, single problem or batch)
// for the process.
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
	// FP32 x-lines longer than 1024 points of a single problem: the streamed
	// kernel (a batch or a misaligned level falls back to the register-chunk one)
	const int stream = dir == CDR_DIR_X && sizeof(T) == 4 && n > 1024 && nb == 1 ? 1 : 0;
	return LineShape{canon_K<T>(n, dir), dir == CDR_DIR_X ? FAST_BLOCK_X : yblock_max<T>(), stream};
}

template <typename T>
static bool shape_ok(LineShape sh, int n, int dir)
{
	const int K = canon_K<T>(n, dir);
	if (K == 0 || sh.K != K || sh.cap < 32) return false;
	return dir == CDR_DIR_X ? sh.cap <= FAST_BLOCK_X || sh.stream : sh.cap <= yblock_max<T>();
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
                       int cap, cudaStream_t st, bool zero, const T *yc = nullptr)
{
	const bool pack = yc != nullptr;
	const int n = DIR == CDR_DIR_X ? d.nx : d.ny;
	const int tpl_log2 = tpl_log2_of(n, K);
	const int TPL = 1 << tpl_log2;
	int G, block;
	if (DIR == CDR_DIR_X) {  // cap CTA threads, at least one line, at most FAST_BLOCK_X
		block = std::min(FAST_BLOCK_X, std::max(TPL, cap));
		G = block / TPL;
	} else {
		G = ylines_per_cta(TPL, cap);
		block = (G * TPL + 31) / 32 * 32;
	}
	const dim3 grd(ceil_div(nlines, G), 1, d.nb);
	constexpr bool ysmall = DIR == CDR_DIR_Y && sizeof(T) == 4;
	if constexpr (DIR == CDR_DIR_Y) {
		// packed couplings (zero-start sweeps read no couplings)
		if (pack && !zero) {
			if (ysmall && block <= YSMALL_BLOCK)
				k_lines_fast<T, NS, DIR, K, ysmall ? YSMALL_BLOCK : 0, false, true><<<grd, block, 0, st>>>(
				    so, x, b, sor, d, tpitch, first, tpl_log2, G, yc);
			else
				k_lines_fast<T, NS, DIR, K, 0, false, true><<<grd, block, 0, st>>>(so, x, b, sor, d, tpitch, first,
				                                                                    tpl_log2, G, yc);
			CDR_LAUNCH_CHECK();
			return CDR_OK;
		}
	}
	if (ysmall && block <= YSMALL_BLOCK) {
		constexpr int LB = ysmall ? YSMALL_BLOCK : 0;
		if (zero)
			k_lines_fast<T, NS, DIR, K, LB, true><<<grd, block, 0, st>>>(so, x, b, sor, d, tpitch, first, tpl_log2, G, yc);
		else
			k_lines_fast<T, NS, DIR, K, LB><<<grd, block, 0, st>>>(so, x, b, sor, d, tpitch, first, tpl_log2, G, yc);
	} else if (zero) {
		k_lines_fast<T, NS, DIR, K, 0, true><<<grd, block, 0, st>>>(so, x, b, sor, d, tpitch, first, tpl_log2, G, yc);
	} else {
		k_lines_fast<T, NS, DIR, K><<<grd, block, 0, st>>>(so, x, b, sor, d, tpitch, first, tpl_log2, G, yc);
	}
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

// The streamed x-line kernel (FP32, K = 8, the register-chunk kernel's K for
// these lengths): one line per CTA step (TPL = 32 .. 256 threads), a single
// problem, the stage within the shared-memory budget.
template <typename T, int NS>
static bool xs_ok(Dims2 d)
{
	const int n = d.nx;
	return sizeof(T) == 4 && canon_K<T>(n, CDR_DIR_X) == 8 && d.nb == 1 && n >= 32 * 8 && n <= XS_BLOCK * 8 &&
	       xs_smem<T, NS>(d.pitch) <= XS_SMEM_MAX;
}

// CTAs per SM of the streamed kernel for a (block, shared memory) pair, and the
// SM count: looked up once per pair
template <int NS>
static int xs_grid_cap(int block, size_t smem)
{
	static std::mutex mu;
	static std::map<std::pair<int, size_t>, int> cache;
	std::lock_guard<std::mutex> lk(mu);
	auto it = cache.find({block, smem});
	if (it != cache.end()) return it->second;
	int dev = 0, sms = 0, per_sm = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
	    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lines_xstream<float, NS, 8>, block, smem) != cudaSuccess)
		return 0;
	const int cap = sms * (per_sm > 0 ? per_sm : 1);
	cache[{block, smem}] = cap;
	return cap;
}

template <int NS>
static int launch_xstream(const float *so, float *x, const float *b, const float *sor, Dims2 d, int first, int nlines,
                          cudaStream_t st)
{
	const int tpl = 1 << tpl_log2_of(d.nx, 8);
	const size_t smem = xs_smem<float, NS>(d.pitch);
	CDR_TRY(lines_prepare());
	const int cap = xs_grid_cap<NS>(tpl, smem);
	if (cap <= 0) {
		set_error(CDR_ERR_CUDA, "occupancy query for the streamed line kernel failed");
		return CDR_ERR_CUDA;
	}
	const int grid = nlines < cap ? nlines : cap;
	k_lines_xstream<float, NS, 8><<<grid, tpl, smem, st>>>(so, x, b, sor, d, first, nlines);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

// Words of the sync buffer of the fused y-line sweep of a level: a ticket
// counter and one flag per virtual block (at most one block per column pair).
size_t lines_sync_words(Dims2 d) { return 2 + (size_t)d.nx / 2 + 1; }

template <typename T, int NS, int K>
static int launch_ypair(const T *so, T *x, const T *b, const T *sor, Dims2 d, int tpitch, int updown, int cap,
                        unsigned *sync, cudaStream_t st, bool zero = false, const T *yc = nullptr)
{
	const bool pack = yc != nullptr;
	const int tpl_log2 = tpl_log2_of(d.ny, K), TPL = 1 << tpl_log2;
	const int G = ylines_per_cta(TPL, cap);
	const int block = (G * TPL + 31) / 32 * 32;
	// DOWN sweeps the even lines first (relax_lines_y.f90:82-97): pairs (odd, even)
	const int c2 = updown == CDR_DOWN ? 1 : 0;
	const int npairs = (d.nx - c2) / 2 + 1, nvb = ceil_div(npairs, G);
	constexpr int LB = sizeof(T) == 4 ? YSMALL_BLOCK : 0;
	const bool small = LB && block <= LB;
	// zero start and packed couplings: the first colour reads b only, the second the packed couplings
	if (small) {
		if (zero && pack)
			k_ylines_pair<T, NS, K, LB, true, true><<<nvb, block, 0, st>>>(so, x, b, sor, d, tpitch, c2, tpl_log2, G, sync, nvb, yc);
		else if (zero)
			k_ylines_pair<T, NS, K, LB, true><<<nvb, block, 0, st>>>(so, x, b, sor, d, tpitch, c2, tpl_log2, G, sync, nvb, yc);
		else if (pack)
			k_ylines_pair<T, NS, K, LB, false, true><<<nvb, block, 0, st>>>(so, x, b, sor, d, tpitch, c2, tpl_log2, G, sync, nvb, yc);
		else
			k_ylines_pair<T, NS, K, LB><<<nvb, block, 0, st>>>(so, x, b, sor, d, tpitch, c2, tpl_log2, G, sync, nvb, yc);
	} else {
		if (zero && pack)
			k_ylines_pair<T, NS, K, 0, true, true><<<nvb, block, 0, st>>>(so, x, b, sor, d, tpitch, c2, tpl_log2, G, sync, nvb, yc);
		else if (zero)
			k_ylines_pair<T, NS, K, 0, true><<<nvb, block, 0, st>>>(so, x, b, sor, d, tpitch, c2, tpl_log2, G, sync, nvb, yc);
		else if (pack)
			k_ylines_pair<T, NS, K, 0, false, true><<<nvb, block, 0, st>>>(so, x, b, sor, d, tpitch, c2, tpl_log2, G, sync, nvb, yc);
		else
			k_ylines_pair<T, NS, K><<<nvb, block, 0, st>>>(so, x, b, sor, d, tpitch, c2, tpl_log2, G, sync, nvb, yc);
	}
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

// The register-chunk kernels read whole 16-byte-aligned chunks of K elements:
// rows (x) or factor lines (y) must have a pitch that is a multiple of K and
// 16-byte aligned base pointers; lines up to 256*K points (16*256 FP32).
template <typename T>
static bool fast_lines_ok(const T *so, const T *x, const T *b, const T *sor, Dims2 d, int tpitch, int dir, bool exact)
{
	const int n = dir == CDR_DIR_X ? d.nx : d.ny;
	const int fpitch = dir == CDR_DIR_X ? d.pitch : tpitch;
	const bool aligned = ((uintptr_t)so | (uintptr_t)x | (uintptr_t)b | (uintptr_t)sor) % 16 == 0;
	const int K = canon_K<T>(n, dir);
	return !exact && aligned && d.pitch % 16 == 0 && fpitch % 16 == 0 && K != 0 &&
	       (K == 8 || sizeof(T) == 4 || dir == CDR_DIR_Y);
}

// One colour of lines.  zero: x is zero on entry (the register-chunk kernels
// only; the streamed x-line kernel's bits are the register-chunk kernel's).
template <typename T, int NS, int DIR>
static int launch_lines(const T *so, T *x, const T *b, const T *sor, Dims2 d, int tpitch, int first, bool exact,
                        cudaStream_t st, const LineShape *force = nullptr, bool zero = false, const T *yc = nullptr)
{
	const int n = DIR == CDR_DIR_X ? d.nx : d.ny;
	const int nl = DIR == CDR_DIR_X ? d.ny : d.nx;
	const int nlines = first > nl ? 0 : (nl - first) / 2 + 1;
	if (nlines == 0) return CDR_OK;
	LineShape sh = force ? *force : shape_for<T>(n, nl, NS, d.nb, DIR);
	if (!shape_ok<T>(sh, n, DIR)) sh = default_shape<T>(n, DIR, d.nb);
	if (fast_lines_ok<T>(so, x, b, sor, d, tpitch, DIR, exact) && shape_ok<T>(sh, n, DIR)) {
		if constexpr (DIR == CDR_DIR_X && sizeof(T) == 4)
			if (sh.stream && xs_ok<T, NS>(d)) {
				if (!zero) return launch_xstream<NS>(so, x, b, sor, d, first, nlines, st);
				sh.cap = FAST_BLOCK_X;
			}
		if (sh.K == 16) {
			if constexpr (sizeof(T) == 4 || DIR == CDR_DIR_Y)
				return launch_fast<T, NS, DIR, 16>(so, x, b, sor, d, tpitch, first, nlines, sh.cap, st, zero, yc);
		} else {
			return launch_fast<T, NS, DIR, 8>(so, x, b, sor, d, tpitch, first, nlines, sh.cap, st, zero, yc);
		}
	}
	if (zero) {
		set_error(CDR_ERR_ARG, "zero-start line sweep needs the register-chunk kernel");
		return CDR_ERR_ARG;
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
static int tune_dir(const T *so, T *x, const T *b, const T *sor, Dims2 d, int tpitch, cudaStream_t st,
                    unsigned *ysync, const T *yc)
{
	const int n = DIR == CDR_DIR_X ? d.nx : d.ny;
	const int nl = DIR == CDR_DIR_X ? d.ny : d.nx;
	const LineKey key{DIR, (int)sizeof(T), NS, n, nl, d.nb > 1 ? 2 : 1};
	{
		std::lock_guard<std::mutex> lk(g_shape_mu);
		if (shape_table().count(key)) return CDR_OK;
	}
	// every candidate gives the same bits (the chunks are fixed by the line
	// length); x: CTA sizes, y: lines per CTA
	const int K = canon_K<T>(n, DIR);
	if (K == 0) {
		std::lock_guard<std::mutex> lk(g_shape_mu);
		shape_table()[key] = default_shape<T>(n, DIR, d.nb);
		return CDR_OK;
	}
	const int TPL = 1 << tpl_log2_of(n, K);
	const int caps_x[4] = {32, 64, 128, 256};
	const int caps_y[4] = {TPL, 2 * TPL, 4 * TPL, 8 * TPL};
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
			if (DIR == CDR_DIR_Y && ysync && d.nb == 1 && sh.pair) {  // both colours in one launch
				rc = sh.K == 16 ? launch_ypair<T, NS, 16>(so, x, b, sor, d, tpitch, CDR_DOWN, sh.cap, ysync, st, false, yc)
				                : launch_ypair<T, NS, 8>(so, x, b, sor, d, tpitch, CDR_DOWN, sh.cap, ysync, st, false, yc);
			} else {
				for (int f = 1; f <= 2 && rc == CDR_OK; ++f)
					rc = launch_lines<T, NS, DIR>(so, x, b, sor, d, tpitch, f, false, st, &sh, false, yc);
			}
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
	// y-lines of a single problem: both colours in one launch or one launch per
	// colour (the default: the one-launch form's phase hand-over costs more than
	// the second launch on a B200 at every size measured, 127^2 to 2047^2)
	const int npair = DIR == CDR_DIR_Y && ysync && d.nb == 1 ? 2 : 1;
	for (int pr = 0; pr < npair && rc == CDR_OK; ++pr)
		for (int c = 0; c < 4 && rc == CDR_OK; ++c) {
			LineShape sh{K, DIR == CDR_DIR_X ? caps_x[c] : std::max(32, caps_y[c]), 0};
			sh.pair = pr == 0 ? 1 : 0;
			if (!shape_ok<T>(sh, n, DIR)) continue;
			if (DIR == CDR_DIR_X && sh.cap < TPL && caps_x[c] != 32) continue;  // same CTA as a smaller cap
			const float ms = time_shape(sh);
			if (ms < margin * best_ms) { best_ms = ms; best = sh; }
		}
	if (DIR == CDR_DIR_X && rc == CDR_OK && xs_ok<T, NS>(d)) {
		const LineShape sh{K, FAST_BLOCK_X, 1};
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
                   cudaStream_t st, unsigned *ysync, const T *ycpl)
{
	if (dir == CDR_DIR_X) {
		if (nstencil == 5) return tune_dir<T, 5, CDR_DIR_X>(so, x, b, sor, d, tpitch, st, ysync, nullptr);
		return tune_dir<T, 3, CDR_DIR_X>(so, x, b, sor, d, tpitch, st, ysync, nullptr);
	}
	if (nstencil == 5) return tune_dir<T, 5, CDR_DIR_Y>(so, x, b, sor, d, tpitch, st, ysync, ycpl);
	return tune_dir<T, 3, CDR_DIR_Y>(so, x, b, sor, d, tpitch, st, ysync, ycpl);
}
template int lines_autotune<double>(const double *, int, double *, const double *, const double *, Dims2, int, int,
                                    cudaStream_t, unsigned *, const double *);
template int lines_autotune<float>(const float *, int, float *, const float *, const float *, Dims2, int, int,
                                   cudaStream_t, unsigned *, const float *);

bool lines_set_shape(int dir, int tsize, int ns, int n, int nl, int nb, LineShape sh)
{
	bool ok;
	if (tsize == 4) ok = shape_ok<float>(sh, n, dir);
	else ok = shape_ok<double>(sh, n, dir);
	if (sh.stream) ok = ok && dir == CDR_DIR_X && nb == 1 && tsize == 4 && sh.K == 8;
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
                   int updown, int flags, cudaStream_t st, unsigned *ysync, const T *ycpl)
{
	const bool exact = (flags & CDR_LINES_EXACT) != 0;
	bool zero = (flags & CDR_LINES_ZERO_START) != 0;
	if (zero && !fast_lines_ok<T>(so, x, b, sor, d, tpitch, dir, exact)) {
		// the sequential or shared-memory kernels read x: clear it (each of the
		// batch's problems, bstep planes apart)
		CDR_CUDA_TRY(cudaMemset2DAsync(x, sizeof(T) * (size_t)d.bstep * d.plane(), 0, sizeof(T) * d.plane(), d.nb, st));
		zero = false;
	}
	// packed y couplings: the caller's array, or (CDR_LINES_YPACKED, a single
	// problem) the planes after the two factor planes of sor
	const T *yc = nullptr;
	if (dir == CDR_DIR_Y) {
		if (ycpl) yc = ycpl;
		else if ((flags & CDR_LINES_YPACKED) && d.nb == 1) yc = sor + 2 * (size_t)tpitch * (d.nx + 2);
	}
	const LineShape dflt = default_shape<T>(dir == CDR_DIR_X ? d.nx : d.ny, dir, d.nb);
	const LineShape streamed{canon_K<T>(d.nx, CDR_DIR_X), FAST_BLOCK_X, 1};
	const LineShape *force = (flags & CDR_LINES_NOTUNE) ? &dflt : nullptr;
	if ((flags & CDR_LINES_STREAM) && dir == CDR_DIR_X) force = &streamed;
	// y-lines of a single problem with a sync buffer: both colours in one launch
	// where the tuned shape says so or the caller asks for it (CDR_LINES_YPAIR)
	if (dir == CDR_DIR_Y && ysync && !exact && d.nb == 1 && d.nx >= 2 &&
	    ((uintptr_t)so | (uintptr_t)x | (uintptr_t)b | (uintptr_t)sor) % 16 == 0 && d.pitch % 16 == 0 &&
	    tpitch % 16 == 0) {
		LineShape sh = force ? *force : shape_for<T>(d.ny, d.nx, nstencil, d.nb, dir);
		if (!shape_ok<T>(sh, d.ny, dir)) sh = dflt;
		if (shape_ok<T>(sh, d.ny, dir) && (sh.pair || (flags & CDR_LINES_YPAIR))) {
			if (sh.K == 16) {
				if (nstencil == 5)
					return launch_ypair<T, 5, 16>(so, x, b, sor, d, tpitch, updown, sh.cap, ysync, st, zero, yc);
				return launch_ypair<T, 3, 16>(so, x, b, sor, d, tpitch, updown, sh.cap, ysync, st, zero, yc);
			}
			if (nstencil == 5)
				return launch_ypair<T, 5, 8>(so, x, b, sor, d, tpitch, updown, sh.cap, ysync, st, zero, yc);
			return launch_ypair<T, 3, 8>(so, x, b, sor, d, tpitch, updown, sh.cap, ysync, st, zero, yc);
		}
	}
	// DOWN: lines with Fortran start index 3 (0-based even) first, then 2 (odd);
	// UP: the opposite (relax_lines_x.f90:82-97).
	const int firsts[2] = {updown == CDR_DOWN ? 2 : 1, updown == CDR_DOWN ? 1 : 2};
	for (int c = 0; c < 2; ++c) {
		const int f = firsts[c];
		const bool z = zero && c == 0;  // the second colour reads the first's new lines only
		if (dir == CDR_DIR_X) {
			if (nstencil == 5) CDR_TRY((launch_lines<T, 5, CDR_DIR_X>(so, x, b, sor, d, tpitch, f, exact, st, force, z)));
			else CDR_TRY((launch_lines<T, 3, CDR_DIR_X>(so, x, b, sor, d, tpitch, f, exact, st, force, z)));
		} else {
			if (nstencil == 5)
				CDR_TRY((launch_lines<T, 5, CDR_DIR_Y>(so, x, b, sor, d, tpitch, f, exact, st, force, z, yc)));
			else CDR_TRY((launch_lines<T, 3, CDR_DIR_Y>(so, x, b, sor, d, tpitch, f, exact, st, force, z, yc)));
		}
	}
	return CDR_OK;
}
template int relax_lines_2d<double>(const double *, int, double *, const double *, const double *, Dims2, int, int,
                                    int, int, cudaStream_t, unsigned *, const double *);
template int relax_lines_2d<float>(const float *, int, float *, const float *, const float *, Dims2, int, int, int,
                                   int, cudaStream_t, unsigned *, const float *);

// ---------------------------------------------------- packed y-line couplings
// For the y-line sweep: the couplings that line i's right-hand side reads at
// position j, one plane each in line order (line-contiguous, tpitch, like the
// transposed y factors): w(i,j), w(i+1,j) [, sw(i,j), nw(i+1,j), nw(i,j+1),
// sw(i+1,j+1)] -- the operands of relax_lines_y.f90:102-106 other than b and
// x.  The sweep then reads them with vector loads of the line's own
// contiguous segments instead of strided loads shared by the two colours.
// Problem z of a batch (bstep apart) at yc + z * bstep * planes * tpitch * (nx+2).
template <typename T, int NS>
__global__ void k_pack_ylines(const T *__restrict__ so, T *__restrict__ yc, Dims2 d, int tpitch)
{
	const int j = blockIdx.x * blockDim.x + threadIdx.x + 1, i = blockIdx.y + 1;
	if (j > d.ny || i > d.nx) return;
	const size_t ps = d.plane(), fps = (size_t)tpitch * (d.nx + 2);
	so += d.bofs(NS * ps);
	yc += d.bofs((size_t)(NS == 5 ? 6 : 2) * fps);
	const int P = d.pitch;
	const size_t k = d.at(i, j), o = (size_t)i * tpitch + j;
	const T *w = so + ps;
	yc[o] = w[k];
	yc[fps + o] = w[k + 1];
	if (NS == 5) {
		const T *sw = so + 3 * ps, *nw = so + 4 * ps;
		yc[2 * fps + o] = sw[k];
		yc[3 * fps + o] = nw[k + 1];
		yc[4 * fps + o] = nw[k + P];
		yc[5 * fps + o] = sw[k + P + 1];
	}
}

template <typename T>
int pack_ylines_2d(const T *so, int nstencil, T *yc, Dims2 d, int tpitch, cudaStream_t st)
{
	if (tpitch < d.ny + 2) {
		set_error(CDR_ERR_DIM, "packed y-line couplings: tpitch %d < ny+2", tpitch);
		return CDR_ERR_DIM;
	}
	const dim3 g(ceil_div(d.ny, 256), d.nx, d.nb);
	if (nstencil == 5) k_pack_ylines<T, 5><<<g, 256, 0, st>>>(so, yc, d, tpitch);
	else k_pack_ylines<T, 3><<<g, 256, 0, st>>>(so, yc, d, tpitch);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int pack_ylines_2d<double>(const double *, int, double *, Dims2, int, cudaStream_t);
template int pack_ylines_2d<float>(const float *, int, float *, Dims2, int, cudaStream_t);

}  // namespace cdrgpu
