// k2_cginv.cu -- the coarsest 2D solve as a product with the explicit inverse.
//
// The reference solves the coarsest level with the banded Cholesky factor of
// BMG2_SymStd_SETUP_cg_LU (DPBTRS: two triangular sweeps over n unknowns with
// bandwidth nx+1, src/2d/ftn/BMG2_SymStd_SOLVE_cg.f90).  On the GPU those sweeps
// are one sequential chain; for a coarsest level of a few thousand unknowns
// (e.g. 63^2, selected with solver.num-levels) it costs about a millisecond.
// With settings.coarse_solve = CDR_COARSE_INVERSE the setup instead forms
// A^{-1} from the same factor (one column per thread, both sweeps per column,
// FP64) and each cycle applies it as a matrix-vector product (memory bound,
// ~n^2 words per solve).  The result equals DPBTRS's to rounding, not bitwise.
#include <cstdint>
#include <type_traits>

#include "k2_bulk.cuh"
#include "k2_point.cuh"
#include "kernels2d.cuh"

namespace cdrgpu {

namespace {

// Column c of A^{-1} = U^{-1} U^{-T} e_c by the two sweeps of DPBTRS ('U'
// band storage, U(i, j) at ab[j*ldab + kd + i - j]), one column per thread, 32
// columns per CTA, the warp walking j in step so that every lane uses the same
// factor column, which is staged in shared memory one step ahead.  Forward:
// y(j) = (e_c(j) - sum_i U(i, j) y(i)) / U(j, j); backward (DTBSV's column
// form): x(j) = y(j) / U(j, j), then y(i) -= x(j) U(i, j) for the kd rows
// above.  The active window of each column lives in a shared-memory ring; y is
// parked in ainv[j*n + c] (row c of the symmetric inverse, 32 consecutive words
// per warp) and overwritten by x.
constexpr int CGI_RING = 128;  // ring slots per column (>= kd + 2)

__global__ void __launch_bounds__(32) k_cg_inverse(const double *__restrict__ ab, int n, int kd, int ldab,
                                                   double *__restrict__ ainv)
{
	__shared__ double ring[CGI_RING][32];
	__shared__ double ucol[2][CGI_RING];
	const int lane = threadIdx.x, c0 = blockIdx.x * 32, c = c0 + lane;
	const bool on = c < n;
	constexpr int M = CGI_RING - 1;
	for (int j = 0; j < CGI_RING; ++j) ring[j][lane] = 0.0;
	auto stage = [&](int j, int buf) {
		for (int e = lane; e <= kd; e += 32) ucol[buf][e] = ab[(size_t)j * ldab + e];
	};
	stage(c0, 0);
	__syncwarp();
	// forward from the warp's first column; y(j) = 0 for j < c
	for (int j = c0; j < n; ++j) {
		const int buf = (j - c0) & 1;
		if (j + 1 < n) stage(j + 1, buf ^ 1);
		double t = j == c ? 1.0 : 0.0;
		if (on && j > c) {
			const int i0 = j - kd > c ? j - kd : c;
			const double *col = ucol[buf] + kd - j;
			for (int i = i0; i < j; ++i) t -= col[i] * ring[i & M][lane];
		}
		const double y = (on && j >= c) ? t / ucol[buf][kd] : 0.0;
		ring[j & M][lane] = y;
		if (on) ainv[(size_t)j * n + c] = y;
		__syncwarp();
	}
	if (on)
		for (int j = 0; j < c0 && j < n; ++j) ainv[(size_t)j * n + c] = 0.0;  // y below the warp's first column
	// backward; the ring holds y (being updated) for rows (j - kd - 1, j]
	stage(n - 1, 0);
	__syncwarp();
	for (int j = n - 1; j >= 0; --j) {
		const int buf = (n - 1 - j) & 1;
		if (j > 0) stage(j - 1, buf ^ 1);
		// y(j - 1 - kd) enters the window for the next step (untouched by the backward sweep so far)
		const int e = j - 1 - kd;
		const double yin = (on && e >= 0) ? ainv[(size_t)e * n + c] : 0.0;
		const double x = ring[j & M][lane] / ucol[buf][kd];
		if (on) ainv[(size_t)j * n + c] = x;
		const int i0 = j - kd > 0 ? j - kd : 0;
		const double *col = ucol[buf] + kd - j;
		for (int i = i0; i < j; ++i) ring[i & M][lane] -= x * col[i];
		if (e >= 0) ring[e & M][lane] = yin;
		__syncwarp();
	}
}

// x(interior) = A^{-1} b(interior): b compacted into shared memory in the
// inverse's type, one warp per row, 16-byte row loads (four independent FP64
// accumulators per lane, so that each lane keeps four loads in flight) where
// the row length is a multiple of the vector width, FP64 accumulation.  A
// product of two FP32 (or the FP64) values is summed in FP64.
template <typename T>
__global__ void __launch_bounds__(256) k_cg_inv_apply(const T *__restrict__ ainv, T *__restrict__ q,
                                                      const T *__restrict__ qf, Dims2 d)
{
	extern __shared__ __align__(16) unsigned char cgi_raw[];
	T *bs = reinterpret_cast<T *>(cgi_raw);
	constexpr int V = 16 / sizeof(T);
	using VT = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
	const int n = d.nx * d.ny;
	for (int e = threadIdx.x; e < n; e += blockDim.x) bs[e] = qf[d.at(e % d.nx + 1, e / d.nx + 1)];
	__syncthreads();
	const int lane = threadIdx.x & 31;
	const int warps = gridDim.x * (blockDim.x >> 5);
	const bool vec = n % V == 0;
	for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
		const T *row = ainv + (size_t)r * n;
		double a[4] = {0.0, 0.0, 0.0, 0.0};
		if (vec) {
			const VT *rv = reinterpret_cast<const VT *>(row);
			const int nv = n / V;
			int j = lane;
			for (; j + 96 < nv; j += 128) {
#pragma unroll
				for (int u = 0; u < 4; ++u) {
					const VT w = __ldcs(rv + j + 32 * u);
					const VT bv = reinterpret_cast<const VT *>(bs)[j + 32 * u];
					const T *wt = reinterpret_cast<const T *>(&w), *bb = reinterpret_cast<const T *>(&bv);
#pragma unroll
					for (int v = 0; v < V; ++v) a[u] += (double)wt[v] * (double)bb[v];
				}
			}
			for (; j < nv; j += 32) {
				const VT w = __ldcs(rv + j);
				const VT bv = reinterpret_cast<const VT *>(bs)[j];
				const T *wt = reinterpret_cast<const T *>(&w), *bb = reinterpret_cast<const T *>(&bv);
#pragma unroll
				for (int v = 0; v < V; ++v) a[0] += (double)wt[v] * (double)bb[v];
			}
		} else {
			for (int j = lane; j < n; j += 32) a[0] += (double)row[j] * (double)bs[j];
		}
		double s = (a[0] + a[1]) + (a[2] + a[3]);
		for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
		if (lane == 0) q[d.at(r % d.nx + 1, r / d.nx + 1)] = (T)s;
	}
}

// The same product with the inverse's rows streamed into shared memory by bulk
// asynchronous copies, IA_STAGES rows ahead per CTA (one mbarrier per stage;
// two stages leave room for four CTAs per SM, whose rows overlap),
// so that DRAM keeps streaming while the CTA sums the current row: one row per
// CTA step, 256 threads, 16-byte row loads from shared memory, FP64 partial
// sums reduced in a fixed order.  Rows must be 16-byte multiples.  Every wait
// is bounded (g_inv_wait_ns of the global timer); a CTA that gives up is
// counted in g_inv_timeouts, waits (bounded) for every copy it has in flight
// (the stage it gave up on and the ones issued after it) and returns.
constexpr int IA_STAGES = 2, IA_BLOCK = 256;
__device__ unsigned g_inv_timeouts;
__device__ unsigned long long g_inv_wait_ns = kWaitLimitNs;

template <typename T>
__global__ void __launch_bounds__(IA_BLOCK) k_cg_inv_apply_bulk(const T *__restrict__ ainv, T *__restrict__ q,
                                                                const T *__restrict__ qf, Dims2 d)
{
	extern __shared__ __align__(128) unsigned char ia_raw[];
	__shared__ double red[IA_BLOCK / 32];
	constexpr int V = 16 / sizeof(T);
	using VT = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
	const int n = d.nx * d.ny;
	uint64_t *bar = reinterpret_cast<uint64_t *>(ia_raw);
	T *bs = reinterpret_cast<T *>(ia_raw + 128);
	T *rows = bs + ((n + 31) & ~31);
	const unsigned row_bytes = (unsigned)n * sizeof(T);
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, G = gridDim.x;
	auto issue = [&](int r, int st) {
		asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
		mbar_expect_tx(&bar[st], row_bytes);
		bulk_g2s(rows + (size_t)st * n, ainv + (size_t)r * n, row_bytes, &bar[st]);
	};
	if (tid == 0) {
		for (int st = 0; st < IA_STAGES; ++st) mbar_init(&bar[st], 1);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	__syncthreads();
	if (tid == 0)
		for (int st = 0; st < IA_STAGES; ++st)
			if ((int)blockIdx.x + st * G < n) issue(blockIdx.x + st * G, st);
	for (int e = tid; e < n; e += IA_BLOCK) {  // b compacted while the first rows arrive
		const int jj = e / d.nx;
		bs[e] = qf[d.at(e - jj * d.nx + 1, jj + 1)];
	}
	__syncthreads();
	const unsigned long long wait_ns = g_inv_wait_ns;
	int k = 0;
	for (int r = blockIdx.x; r < n; r += G, ++k) {
		const int st = k % IA_STAGES;
		const bool ok = mbar_wait_bounded(&bar[st], (unsigned)(k / IA_STAGES) & 1u, wait_ns);
		if (!__syncthreads_and(ok)) {
			// give up: wait (bounded) for the copies in flight -- this stage's and
			// those of the rows issued after it -- then leave
			if (tid == 0) {
				atomicAdd(&g_inv_timeouts, 1u);
				for (int s2 = 0; s2 < IA_STAGES; ++s2)
					if (r + s2 * G < n)
						mbar_wait_bounded(&bar[(k + s2) % IA_STAGES], (unsigned)((k + s2) / IA_STAGES) & 1u,
						                  kDrainLimitNs);
			}
			return;
		}
		const VT *row = reinterpret_cast<const VT *>(rows + (size_t)st * n);
		const VT *bv = reinterpret_cast<const VT *>(bs);
		double a = 0.0;
		for (int j = tid; j < n / V; j += IA_BLOCK) {
			const VT w = row[j], x = bv[j];
			const T *wt = reinterpret_cast<const T *>(&w), *xt = reinterpret_cast<const T *>(&x);
#pragma unroll
			for (int v = 0; v < V; ++v) a += (double)wt[v] * (double)xt[v];
		}
		for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
		if (lane == 0) red[warp] = a;
		__syncthreads();  // the stage is read, the warp sums are in
		if (tid == 0) {
			double sum = 0.0;
#pragma unroll
			for (int w = 0; w < IA_BLOCK / 32; ++w) sum += red[w];
			q[d.at(r % d.nx + 1, r / d.nx + 1)] = (T)sum;
			if (r + IA_STAGES * G < n) issue(r + IA_STAGES * G, st);
		}
		__syncthreads();  // red[] is free again
	}
}

template <typename T>
size_t inv_bulk_smem(int n)
{
	return 128 + sizeof(T) * ((size_t)((n + 31) & ~31) + (size_t)IA_STAGES * n);
}

}  // namespace

int cg_inv_timeouts(cudaStream_t st, unsigned *count)
{
	unsigned v = 0;
	*count = 0;
	CDR_CUDA_TRY(cudaMemcpyFromSymbolAsync(&v, g_inv_timeouts, sizeof v, 0, cudaMemcpyDeviceToHost, st));
	CDR_CUDA_TRY(cudaStreamSynchronize(st));
	if (v) {
		const unsigned z = 0;
		CDR_CUDA_TRY(cudaMemcpyToSymbolAsync(g_inv_timeouts, &z, sizeof z, 0, cudaMemcpyHostToDevice, st));
		CDR_CUDA_TRY(cudaStreamSynchronize(st));
	}
	*count = v;
	return CDR_OK;
}

int cg_inv_add_timeouts(unsigned n)
{
	unsigned v = 0;
	CDR_CUDA_TRY(cudaMemcpyFromSymbol(&v, g_inv_timeouts, sizeof v));
	v += n;
	CDR_CUDA_TRY(cudaMemcpyToSymbol(g_inv_timeouts, &v, sizeof v));
	return CDR_OK;
}

int cg_inv_set_wait(unsigned long long ns)
{
	CDR_CUDA_TRY(cudaMemcpyToSymbol(g_inv_wait_ns, &ns, sizeof ns));
	return CDR_OK;
}

int cg_inverse_2d(const double *abd, Dims2 d, double *ainv, cudaStream_t st)
{
	const int n = d.nx * d.ny, kd = d.nx + 1, ldab = d.nx + 2;
	if (kd + 2 > CGI_RING) {
		set_error(CDR_ERR_DIM, "coarsest grid %dx%d too wide for the inverse (bandwidth %d)", d.nx, d.ny, kd);
		return CDR_ERR_DIM;
	}
	k_cg_inverse<<<ceil_div(n, 32), 32, 0, st>>>(abd, n, kd, ldab, ainv);
	CDR_LAUNCH_CHECK();
	// the streamed product's shared-memory opt-in (setup time, before any capture)
	const size_t big = 226 * 1024;
	CDR_CUDA_TRY(cudaFuncSetAttribute(k_cg_inv_apply_bulk<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big));
	CDR_CUDA_TRY(cudaFuncSetAttribute(k_cg_inv_apply_bulk<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big));
	return CDR_OK;
}

template <typename T>
int solve_cg_inv_2d(const T *ainv, T *x, const T *b, Dims2 d, cudaStream_t st)
{
	const int n = d.nx * d.ny;
	const size_t sm = sizeof(T) * (size_t)n;
	if (sm > 48 * 1024) {
		set_error(CDR_ERR_DIM, "coarsest grid %dx%d too large for the inverse product", d.nx, d.ny);
		return CDR_ERR_DIM;
	}
	const size_t smb = inv_bulk_smem<T>(n);
	if ((n * sizeof(T)) % 16 == 0 && (uintptr_t)ainv % 16 == 0 && smb <= 226 * 1024) {
		static const int slots = [] {
			int dev = 0, sms = 0;
			if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
				return 148;
			return sms;
		}();
		const int per_sm = (int)((228 * 1024) / (smb + 1024));
		const int g = slots * (per_sm > 0 ? per_sm : 1);
		k_cg_inv_apply_bulk<T><<<n < g ? n : g, IA_BLOCK, smb, st>>>(ainv, x, b, d);
		CDR_LAUNCH_CHECK();
		return CDR_OK;
	}
	const int rows_per_cta = 256 / 32, grid = ceil_div(n, rows_per_cta) < 148 * 4 ? ceil_div(n, rows_per_cta) : 148 * 4;
	k_cg_inv_apply<T><<<grid, 256, sm, st>>>(ainv, x, b, d);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int solve_cg_inv_2d<double>(const double *, double *, const double *, Dims2, cudaStream_t);
template int solve_cg_inv_2d<float>(const float *, float *, const float *, Dims2, cudaStream_t);

}  // namespace cdrgpu
