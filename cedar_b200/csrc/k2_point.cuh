// k2_point.cuh -- device helpers shared by the 2D point kernels.
#pragma once
#include "cdr_common.cuh"

namespace cdrgpu {

constexpr int TX = 32, TY = 8;  // 2D tile of the point kernels

// BMG2_SymStd_residual (src/2d/ftn/BMG2_SymStd_residual.f90:89-117).
template <typename T, int NS>
__device__ __forceinline__ T resid_at(const T *__restrict__ so, size_t ps, const T *__restrict__ q,
                                      const T *__restrict__ qf, size_t k, int pitch)
{
	const T *c = so, *w = so + ps, *s = so + 2 * ps;
	if (NS == 5) {
		const T *sw = so + 3 * ps, *nw = so + 4 * ps;
		return qf[k] + w[k] * q[k - 1] + w[k + 1] * q[k + 1] + s[k] * q[k - pitch] + s[k + pitch] * q[k + pitch]
		       + sw[k] * q[k - pitch - 1] + nw[k + 1] * q[k - pitch + 1] + nw[k + pitch] * q[k + pitch - 1]
		       + sw[k + pitch + 1] * q[k + pitch + 1] - c[k] * q[k];
	} else {
		return qf[k] + w[k] * q[k - 1] + w[k + 1] * q[k + 1] + s[k] * q[k - pitch] + s[k + pitch] * q[k + pitch]
		       - c[k] * q[k];
	}
}

template <int NW>
__device__ __forceinline__ double block_sum(double v, double *sh)
{
	for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
	int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
	int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
	if (lane == 0) sh[warp] = v;
	__syncthreads();
	double t = 0;
	if (warp == 0) {
		t = lane < NW ? sh[lane] : 0.0;
		for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
	}
	return t;
}

}  // namespace cdrgpu
