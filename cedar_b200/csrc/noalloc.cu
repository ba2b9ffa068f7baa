// noalloc.cu -- residual and l2 norm without any device allocation.
//
// Some callers of this library cannot allocate device memory when they call it:
// a solver plugin whose host application owns every device allocation (the
// application budgets memory up front and forbids cudaMalloc/cudaFree during a
// run, or would have cudaFree synchronize its pipelines), or code that runs
// where it must not go through another framework's caching allocator.  The
// regular cdr_gpu_residual_2d_f64 needs caller-provided scratch for the partial
// sums of ||r||^2; this variant needs none: its partial sums live in a fixed
// array of device memory that is reserved when the library is loaded.
//
// Limits and behaviour:
//  * the array holds NOALLOC_MAX_TILES = 65536 partial sums (512 KiB), one per
//    32x8 tile of the grid, so the grid may have at most 65536 tiles (for
//    example 4096 x 4096 interior points); larger grids are rejected with
//    CDR_ERR_DIM before anything is launched;
//  * every GPU that loads the library holds the array until the process exits;
//  * the first call on a device looks up the array's device address (once per
//    device, with that device current); make that first call before any
//    stream capture.  The address is kept for the life of the process, so the
//    entry point must not be called on a device after cudaDeviceReset of it;
//  * every call uses the same array and overwrites the partial sums it reads,
//    so calls whose kernels overlap on the GPU (different streams, or different
//    host threads, without ordering between them) race and give wrong norms.
#include <mutex>

#include "k2_point.cuh"

namespace cdrgpu {

constexpr int NOALLOC_MAX_TILES = 65536;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_TILES];

static std::mutex g_noalloc_mutex;
static double *g_noalloc_ptr[NOALLOC_MAX_DEVICES];

// Device address of the partial-sum array on the current device.
static int noalloc_scratch(double **out)
{
	int dev = 0;
	CDR_CUDA_TRY(cudaGetDevice(&dev));
	if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
		set_error(CDR_ERR_UNSUPPORTED, "device ordinal %d beyond %d", dev, NOALLOC_MAX_DEVICES);
		return CDR_ERR_UNSUPPORTED;
	}
	std::lock_guard<std::mutex> lock(g_noalloc_mutex);
	if (!g_noalloc_ptr[dev]) {
		void *p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
		if (e != cudaSuccess || !p) {
			set_error(CDR_ERR_CUDA, "cudaGetSymbolAddress(partial-sum array) on device %d: %s", dev,
			          cudaGetErrorString(e));
			return CDR_ERR_CUDA;
		}
		g_noalloc_ptr[dev] = static_cast<double *>(p);
	}
	*out = g_noalloc_ptr[dev];
	return CDR_OK;
}

// One 32x8 tile per CTA: r = b - A x on the tile, partial[tile] = sum of r^2.
template <int NS>
__global__ void __launch_bounds__(TX *TY) k_residual_tile_norm(const double *__restrict__ so, const double *__restrict__ q,
                                                               const double *__restrict__ qf, double *__restrict__ res,
                                                               Dims2 d, double *__restrict__ partial)
{
	__shared__ double sh[TX * TY / 32];
	const int tiles_x = (d.nx + TX - 1) / TX;
	const int i = (blockIdx.x % tiles_x) * TX + threadIdx.x + 1;
	const int j = (blockIdx.x / tiles_x) * TY + threadIdx.y + 1;
	double acc = 0.0;
	if (i <= d.nx && j <= d.ny) {
		const size_t k = d.at(i, j);
		const double r = resid_at<double, NS>(so, d.plane(), q, qf, k, d.pitch);
		res[k] = r;
		acc = r * r;
	}
	const double s = block_sum<TX * TY / 32>(acc, sh);
	if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(1024) k_noalloc_norm_finish(const double *__restrict__ partial, int n, double *out)
{
	__shared__ double sh[32];
	double v = 0;
	for (int i = threadIdx.x; i < n; i += blockDim.x) v += partial[i];
	for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
	if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
	__syncthreads();
	if (threadIdx.x < 32) {
		v = sh[threadIdx.x];
		for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
		if (threadIdx.x == 0) *out = sqrt(v);
	}
}

}  // namespace cdrgpu

using namespace cdrgpu;

extern "C" int cdr_gpu_residual_2d_f64_noalloc(const double *so, int nstencil, const double *x, const double *b,
                                               double *r, int nx, int ny, int pitch, double *norm_out,
                                               cudaStream_t stream)
{
	if (nx < 1 || ny < 1 || pitch < nx + 2) {
		set_error(CDR_ERR_DIM, "bad grid nx=%d ny=%d pitch=%d", nx, ny, pitch);
		return CDR_ERR_DIM;
	}
	if (nstencil != 3 && nstencil != 5) {
		set_error(CDR_ERR_ARG, "nstencil must be 3 (five_pt) or 5 (nine_pt), got %d", nstencil);
		return CDR_ERR_ARG;
	}
	if (!so || !x || !b || !r || !norm_out) {
		set_error(CDR_ERR_ARG, "null pointer argument");
		return CDR_ERR_ARG;
	}
	const long long tiles = (long long)((nx + TX - 1) / TX) * ((ny + TY - 1) / TY);
	if (tiles > NOALLOC_MAX_TILES) {
		set_error(CDR_ERR_DIM,
		          "grid %dx%d needs %lld partial sums but the fixed scratch of the no-allocation residual holds %d "
		          "(one per 32x8 tile, e.g. at most 4096x4096 points); use cdr_gpu_residual_2d_f64 with caller scratch",
		          nx, ny, tiles, NOALLOC_MAX_TILES);
		return CDR_ERR_DIM;
	}
	double *partial = nullptr;
	CDR_TRY(noalloc_scratch(&partial));
	const Dims2 d{nx, ny, pitch};
	if (nstencil == 5)
		k_residual_tile_norm<5><<<(unsigned)tiles, dim3(TX, TY), 0, stream>>>(so, x, b, r, d, partial);
	else
		k_residual_tile_norm<3><<<(unsigned)tiles, dim3(TX, TY), 0, stream>>>(so, x, b, r, d, partial);
	CDR_LAUNCH_CHECK();
	k_noalloc_norm_finish<<<1, 1024, 0, stream>>>(partial, (int)tiles, norm_out);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
