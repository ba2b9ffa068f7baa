// cdr_common.cuh -- shared definitions for the cedar_b200 CUDA library.
//
// Device layout of a 2D level (same logical layout as Cedar's arrays,
// include/cedar/stencil_op_nd.h:41-78): one ghost ring, i fastest, every stencil
// direction in its own plane.  Rows are padded to a pitch (elements) so that
// row starts are 128/256-byte aligned; planes are pitch*jj elements apart.
// Index (i, j, k) with 0-based i in [0, nx+1], j in [0, ny+1] (ghosts at 0 and
// n+1) lives at p[k*pitch*jj + j*pitch + i].
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/cdr_gpu.h"

namespace cdrgpu {

// Stencil plane numbers (Cedar 2D enum, include/cedar/2d/base_types.h:4-14).
enum : int { PC = 0, PW = 1, PS = 2, PSW = 3, PNW = 4 };
// Interpolation planes (include/cedar/2d/prolong_op.h:14).
enum : int { IL = 0, IR = 1, IA = 2, IB = 3, ISW = 4, INW = 5, INE = 6, ISE = 7 };

struct Dims2 {
	int nx, ny;     // interior points
	int pitch;      // elements per row (>= nx + 2)
	// Batches of independent problems of this size: a launch covers nb of them
	// (grid z); entry z of the batch is problem z*bstep of the arrays, whose
	// problems lie back to back (an array of P planes holds P*plane() elements
	// per problem).  A single problem has nb = bstep = 1.
	int nb = 1, bstep = 1;
	__host__ __device__ int ii() const { return nx + 2; }
	__host__ __device__ int jj() const { return ny + 2; }
	__host__ __device__ size_t plane() const { return (size_t)pitch * (ny + 2); }
	__host__ __device__ size_t at(int i, int j) const { return (size_t)j * pitch + i; }
#ifdef __CUDACC__
	// element offset of this CTA's problem in an array of `per` elements per problem
	__device__ __forceinline__ size_t bofs(size_t per) const { return (size_t)blockIdx.z * (size_t)bstep * per; }
#endif
};

// Counts kernel launches issued by this library (graph replays add the
// launches of the captured cycle).
void count_launches(long long n);

// Records the first error of this thread; the C ABI returns it and
// cdr_gpu_last_error() reports its text.
void set_error(int code, const char *fmt, ...);

#define CDR_CUDA_TRY(expr)                                                          \
	do {                                                                            \
		cudaError_t _e = (expr);                                                    \
		if (_e != cudaSuccess) {                                                    \
			::cdrgpu::set_error(CDR_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #expr, \
			                    cudaGetErrorString(_e));                            \
			return CDR_ERR_CUDA;                                                    \
		}                                                                           \
	} while (0)

#define CDR_LAUNCH_CHECK()                                                          \
	do {                                                                            \
		::cdrgpu::count_launches(1);                                                \
		cudaError_t _e = cudaGetLastError();                                        \
		if (_e != cudaSuccess) {                                                    \
			::cdrgpu::set_error(CDR_ERR_CUDA, "%s:%d launch: %s", __FILE__, __LINE__,  \
			                    cudaGetErrorString(_e));                            \
			return CDR_ERR_CUDA;                                                    \
		}                                                                           \
	} while (0)

#define CDR_TRY(expr)                                                               \
	do {                                                                            \
		int _s = (expr);                                                            \
		if (_s != CDR_OK) return _s;                                                \
	} while (0)

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace cdrgpu
