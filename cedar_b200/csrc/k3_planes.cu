// k3_planes.cu -- plane relaxation of the 3D solver: the data movement between a
// 3D level and the batch of 2D plane problems.
//
// Plane ipl (1-based) of direction xy is the k = ipl slice, of xz the j = ipl
// slice and of yz the i = ipl slice; its 2D grid is (i, j), (i, k) and (j, k)
// respectively (include/cedar/3d/relax_planes.h:73-149).  The plane problems of
// a direction are the entries of a Batch2 (problem ipl-1).  Indices below are
// the reference's C++ ones: 0-based with the ghost layer at 0 and n+1.
#include "k2_point.cuh"
#include "kernels3d.cuh"

namespace cdrgpu {

namespace {

__device__ __forceinline__ size_t o3(const Dims3 &F, int i, int j, int k)
{
	return ((size_t)k * (F.ny + 2) + j) * F.pitch + i;
}

// 3D grid index of plane point (a, b) of plane ipl
__device__ __forceinline__ size_t plane_at(const Dims3 &F, int dir, int ipl, int a, int b)
{
	return dir == 0 ? o3(F, a, b, ipl) : dir == 1 ? o3(F, a, ipl, b) : o3(F, ipl, a, b);
}

}  // namespace

// copy_coeff for xxvii_pt -> nine_pt (include/cedar/3d/relax_planes.h:110-149):
// 2D planes c, w, s, sw, nw from the 3D planes
//   xy: p, pw, ps, psw, pnw;  xz: p, pw, b, bw, be;  yz: p, ps, b, bs, bn.
// xz copies the interior k rows only (so3.range(2)), the others the ghost rows too.
// copy_coeff for seven_pt -> five_pt (include/cedar/3d/relax_planes.h:77-107)
// takes the first three of each list (c, w, s), with the same row ranges.
template <int NS2>
__global__ void k3_plane_coeff(const double *__restrict__ so, Dims3 F, int dir, double *__restrict__ so2, int n1,
                               int n2, int pitch2)
{
	const int a = blockIdx.x * TX + threadIdx.x, b = blockIdx.y * TY + threadIdx.y, ipl = blockIdx.z + 1;
	if (a > n1 + 1 || b > n2 + 1) return;
	if (dir == 1 && (b < 1 || b > n2)) return;
	const size_t plane2 = (size_t)pitch2 * (n2 + 2);
	so2 += (size_t)(ipl - 1) * NS2 * plane2 + (size_t)b * pitch2 + a;
	const size_t g = plane_at(F, dir, ipl, a, b), P = F.plane();
	const int src[3][5] = {{KP, KPW, KPS, KPSW, KPNW}, {KP, KPW, KB, KBW, KBE}, {KP, KPS, KB, KBS, KBN}};
#pragma unroll
	for (int q = 0; q < NS2; ++q) so2[q * plane2] = so[(size_t)(src[dir][q] - 1) * P + g];
}

// copy32 (TO_PLANE) / copy23 (src/3d/relax_planes.cc:185-238): the whole plane,
// ghost layer included, for planes ipl = first+1, first+1+step, ...
template <typename T, bool TO_PLANE>
__global__ void k3_plane_copy(T *__restrict__ x3, Dims3 F, int dir, int first, int step, T *__restrict__ x2, int n1,
                              int n2, int pitch2)
{
	const int a = blockIdx.x * TX + threadIdx.x, b = blockIdx.y * TY + threadIdx.y;
	const int ipl = first + 1 + blockIdx.z * step;
	if (a > n1 + 1 || b > n2 + 1) return;
	const size_t k2 = (size_t)(ipl - 1) * pitch2 * (n2 + 2) + (size_t)b * pitch2 + a;
	const size_t k3 = plane_at(F, dir, ipl, a, b);
	if (TO_PLANE) x2[k2] = x3[k3];
	else x3[k3] = x2[k2];
}

template <typename T, bool TO_PLANE>
__global__ void __launch_bounds__(TX *TY) k3_plane_copy_yz(T *__restrict__ x3, Dims3 F, int first, int step,
                                                           int count, T *__restrict__ x2, int n1, int n2, int pitch2);

template <typename T>
int plane_copy(T *x3, Dims3 F, int dir, int first, int step, int count, T *x2, int n1, int n2, int pitch2,
               bool to_plane, cudaStream_t st)
{
	if (dir == 2) {  // yz planes: through a shared-memory transpose
		const dim3 grd(ceil_div(count, TX), ceil_div(n1 + 2, TX), n2 + 2);
		if (to_plane) k3_plane_copy_yz<T, true><<<grd, dim3(TX, TY), 0, st>>>(x3, F, first, step, count, x2, n1, n2, pitch2);
		else k3_plane_copy_yz<T, false><<<grd, dim3(TX, TY), 0, st>>>(x3, F, first, step, count, x2, n1, n2, pitch2);
		CDR_LAUNCH_CHECK();
		return CDR_OK;
	}
	const dim3 grd(ceil_div(n1 + 2, TX), ceil_div(n2 + 2, TY), count);
	if (to_plane) k3_plane_copy<T, true><<<grd, dim3(TX, TY), 0, st>>>(x3, F, dir, first, step, x2, n1, n2, pitch2);
	else k3_plane_copy<T, false><<<grd, dim3(TX, TY), 0, st>>>(x3, F, dir, first, step, x2, n1, n2, pitch2);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int plane_copy<double>(double *, Dims3, int, int, int, int, double *, int, int, int, bool, cudaStream_t);
template int plane_copy<float>(float *, Dims3, int, int, int, int, float *, int, int, int, bool, cudaStream_t);

// copy_rhs for xxvii_pt (src/3d/relax_planes.cc:43-72 xy, :95-127 xz, :146-178 yz):
// b2 = b + the couplings to the two neighbouring planes, on the plane interior,
// in the reference's operand order.
// NS == 4 (seven_pt, src/3d/relax_planes.cc:25-38 xy, :76-90 xz, :126-140 yz):
// one coupling to each neighbouring plane.
template <typename T, int NS>
__global__ void __launch_bounds__(TX *TY) k3_plane_rhs(const T *__restrict__ so, const T *__restrict__ x,
                                                       const T *__restrict__ bb, Dims3 F, int dir, int first, int step,
                                                       T *__restrict__ b2, int n1, int n2, int pitch2)
{
	const int p = blockIdx.x * TX + threadIdx.x + 1, q = blockIdx.y * TY + threadIdx.y + 1;
	const int ipl = first + 1 + blockIdx.z * step;
	if (p > n1 || q > n2) return;
	const size_t P = F.plane();
#define X3(a, i, j, k) a[o3(F, i, j, k)]
#define S3(pl, i, j, k) so[(size_t)((pl)-1) * P + o3(F, i, j, k)]
	T v;
	if (NS == 4) {
		if (dir == 0) {
			const int i = p, j = q, k = ipl;
			v = X3(bb, i, j, k) + S3(KB, i, j, k) * X3(x, i, j, k - 1) + S3(KB, i, j, k + 1) * X3(x, i, j, k + 1);
		} else if (dir == 1) {
			const int i = p, k = q, j = ipl;
			v = X3(bb, i, j, k) + S3(KPS, i, j, k) * X3(x, i, j - 1, k) + S3(KPS, i, j + 1, k) * X3(x, i, j + 1, k);
		} else {
			const int j = p, k = q, i = ipl;
			v = X3(bb, i, j, k) + S3(KPW, i, j, k) * X3(x, i - 1, j, k) + S3(KPW, i + 1, j, k) * X3(x, i + 1, j, k);
		}
	} else if (dir == 0) {
		const int i = p, j = q, k = ipl;
		v = X3(bb, i, j, k) + S3(KB, i, j, k) * X3(x, i, j, k - 1) + S3(KBW, i, j, k) * X3(x, i - 1, j, k - 1)
		    + S3(KBNW, i, j + 1, k) * X3(x, i - 1, j + 1, k - 1) + S3(KBN, i, j + 1, k) * X3(x, i, j + 1, k - 1)
		    + S3(KBNE, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k - 1) + S3(KBE, i + 1, j, k) * X3(x, i + 1, j, k - 1)
		    + S3(KBSE, i + 1, j, k) * X3(x, i + 1, j - 1, k - 1) + S3(KBS, i, j, k) * X3(x, i, j - 1, k - 1)
		    + S3(KBSW, i, j, k) * X3(x, i - 1, j - 1, k - 1) + S3(KBE, i, j, k + 1) * X3(x, i - 1, j, k + 1)
		    + S3(KBSE, i, j + 1, k + 1) * X3(x, i - 1, j + 1, k + 1) + S3(KBS, i, j + 1, k + 1) * X3(x, i, j + 1, k + 1)
		    + S3(KBSW, i + 1, j + 1, k + 1) * X3(x, i + 1, j + 1, k + 1) + S3(KBW, i + 1, j, k + 1) * X3(x, i + 1, j, k + 1)
		    + S3(KB, i, j, k + 1) * X3(x, i, j, k + 1) + S3(KBNW, i + 1, j, k + 1) * X3(x, i + 1, j - 1, k + 1)
		    + S3(KBN, i, j, k + 1) * X3(x, i, j - 1, k + 1) + S3(KBNE, i, j, k + 1) * X3(x, i - 1, j - 1, k + 1);
	} else if (dir == 1) {
		const int i = p, k = q, j = ipl;
		v = X3(bb, i, j, k) + S3(KPNW, i, j + 1, k) * X3(x, i - 1, j + 1, k) + S3(KPS, i, j + 1, k) * X3(x, i, j + 1, k)
		    + S3(KPSW, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k) + S3(KBNW, i, j + 1, k) * X3(x, i - 1, j + 1, k - 1)
		    + S3(KBN, i, j + 1, k) * X3(x, i, j + 1, k - 1) + S3(KBNE, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k - 1)
		    + S3(KBSE, i, j + 1, k + 1) * X3(x, i - 1, j + 1, k + 1) + S3(KBS, i, j + 1, k + 1) * X3(x, i, j + 1, k + 1)
		    + S3(KBSW, i + 1, j + 1, k + 1) * X3(x, i + 1, j + 1, k + 1) + S3(KPSW, i, j, k) * X3(x, i - 1, j - 1, k)
		    + S3(KPS, i, j, k) * X3(x, i, j - 1, k) + S3(KPNW, i + 1, j, k) * X3(x, i + 1, j - 1, k)
		    + S3(KBSW, i, j, k) * X3(x, i - 1, j - 1, k - 1) + S3(KBS, i, j, k) * X3(x, i, j - 1, k - 1)
		    + S3(KBSE, i + 1, j, k) * X3(x, i + 1, j - 1, k - 1) + S3(KBNE, i, j, k + 1) * X3(x, i - 1, j - 1, k + 1)
		    + S3(KBN, i, j, k + 1) * X3(x, i, j - 1, k + 1) + S3(KBNW, i + 1, j, k + 1) * X3(x, i + 1, j - 1, k + 1);
	} else {
		const int j = p, k = q, i = ipl;
		v = X3(bb, i, j, k) + S3(KPNW, i, j + 1, k) * X3(x, i - 1, j + 1, k) + S3(KPW, i, j, k) * X3(x, i - 1, j, k)
		    + S3(KPSW, i, j, k) * X3(x, i - 1, j - 1, k) + S3(KBNW, i, j + 1, k) * X3(x, i - 1, j + 1, k - 1)
		    + S3(KBW, i, j, k) * X3(x, i - 1, j, k - 1) + S3(KBSW, i, j, k) * X3(x, i - 1, j - 1, k - 1)
		    + S3(KBSE, i, j + 1, k + 1) * X3(x, i - 1, j + 1, k + 1) + S3(KBE, i, j, k + 1) * X3(x, i - 1, j, k + 1)
		    + S3(KBNE, i, j, k + 1) * X3(x, i - 1, j - 1, k + 1) + S3(KPSW, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k)
		    + S3(KPW, i + 1, j, k) * X3(x, i + 1, j, k) + S3(KPNW, i + 1, j, k) * X3(x, i + 1, j - 1, k)
		    + S3(KBNE, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k - 1) + S3(KBE, i + 1, j, k) * X3(x, i + 1, j, k - 1)
		    + S3(KBSE, i + 1, j, k) * X3(x, i + 1, j - 1, k - 1) + S3(KBSW, i + 1, j + 1, k + 1) * X3(x, i + 1, j + 1, k + 1)
		    + S3(KBW, i + 1, j, k + 1) * X3(x, i + 1, j, k + 1) + S3(KBNW, i + 1, j, k + 1) * X3(x, i + 1, j - 1, k + 1);
	}
#undef X3
#undef S3
	b2[(size_t)(ipl - 1) * pitch2 * (n2 + 2) + (size_t)q * pitch2 + p] = v;
}

// yz planes (fixed i): the 3D arrays run along i, across the planes, and the
// planes' 2D arrays along j.  A CTA takes 32 planes of the colour x 32 j at one
// k: it forms (rhs) or reads the values with consecutive threads on
// consecutive planes, and writes them through a shared-memory transpose with
// consecutive threads on consecutive j (and the reverse for the copy back).
// The same values as the kernels above, moved in coalesced rows.
template <typename T, int NS>
__global__ void __launch_bounds__(TX *TY) k3_plane_rhs_yz(const T *__restrict__ so, const T *__restrict__ x,
                                                          const T *__restrict__ bb, Dims3 F, int first, int step,
                                                          int count, T *__restrict__ b2, int n1, int n2, int pitch2)
{
	__shared__ T tile[TX][TX + 1];
	const int z0 = blockIdx.x * TX, a0 = blockIdx.y * TX + 1, q = blockIdx.z + 1;
	const size_t P = F.plane();
#define X3(a, i, j, k) a[o3(F, i, j, k)]
#define S3(pl, i, j, k) so[(size_t)((pl)-1) * P + o3(F, i, j, k)]
	for (int r = threadIdx.y; r < TX; r += TY) {
		const int zi = z0 + threadIdx.x, p = a0 + r;
		if (zi >= count || p > n1) continue;
		const int j = p, k = q, i = first + 1 + zi * step;
		T v;
		if (NS == 4) {
			v = X3(bb, i, j, k) + S3(KPW, i, j, k) * X3(x, i - 1, j, k) + S3(KPW, i + 1, j, k) * X3(x, i + 1, j, k);
		} else {
			v = X3(bb, i, j, k) + S3(KPNW, i, j + 1, k) * X3(x, i - 1, j + 1, k) + S3(KPW, i, j, k) * X3(x, i - 1, j, k)
			    + S3(KPSW, i, j, k) * X3(x, i - 1, j - 1, k) + S3(KBNW, i, j + 1, k) * X3(x, i - 1, j + 1, k - 1)
			    + S3(KBW, i, j, k) * X3(x, i - 1, j, k - 1) + S3(KBSW, i, j, k) * X3(x, i - 1, j - 1, k - 1)
			    + S3(KBSE, i, j + 1, k + 1) * X3(x, i - 1, j + 1, k + 1) + S3(KBE, i, j, k + 1) * X3(x, i - 1, j, k + 1)
			    + S3(KBNE, i, j, k + 1) * X3(x, i - 1, j - 1, k + 1) + S3(KPSW, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k)
			    + S3(KPW, i + 1, j, k) * X3(x, i + 1, j, k) + S3(KPNW, i + 1, j, k) * X3(x, i + 1, j - 1, k)
			    + S3(KBNE, i + 1, j + 1, k) * X3(x, i + 1, j + 1, k - 1) + S3(KBE, i + 1, j, k) * X3(x, i + 1, j, k - 1)
			    + S3(KBSE, i + 1, j, k) * X3(x, i + 1, j - 1, k - 1)
			    + S3(KBSW, i + 1, j + 1, k + 1) * X3(x, i + 1, j + 1, k + 1)
			    + S3(KBW, i + 1, j, k + 1) * X3(x, i + 1, j, k + 1) + S3(KBNW, i + 1, j, k + 1) * X3(x, i + 1, j - 1, k + 1);
		}
		tile[threadIdx.x][r] = v;
	}
#undef X3
#undef S3
	__syncthreads();
	for (int r = threadIdx.y; r < TX; r += TY) {
		const int zi = z0 + r, p = a0 + threadIdx.x;
		if (zi >= count || p > n1) continue;
		const int ipl = first + 1 + zi * step;
		b2[(size_t)(ipl - 1) * pitch2 * (n2 + 2) + (size_t)q * pitch2 + p] = tile[r][threadIdx.x];
	}
}

template <typename T, bool TO_PLANE>
__global__ void __launch_bounds__(TX *TY) k3_plane_copy_yz(T *__restrict__ x3, Dims3 F, int first, int step,
                                                           int count, T *__restrict__ x2, int n1, int n2, int pitch2)
{
	__shared__ T tile[TX][TX + 1];
	const int z0 = blockIdx.x * TX, a0 = blockIdx.y * TX, b = blockIdx.z;
	const size_t pl2 = (size_t)pitch2 * (n2 + 2);
	// 3D side: consecutive threads on consecutive planes (i); plane side:
	// consecutive threads on consecutive a (j)
	if (TO_PLANE) {
		for (int r = threadIdx.y; r < TX; r += TY) {
			const int zi = z0 + threadIdx.x, a = a0 + r;
			if (zi < count && a <= n1 + 1) tile[threadIdx.x][r] = x3[o3(F, first + 1 + zi * step, a, b)];
		}
		__syncthreads();
		for (int r = threadIdx.y; r < TX; r += TY) {
			const int zi = z0 + r, a = a0 + threadIdx.x;
			if (zi < count && a <= n1 + 1) x2[(size_t)(first + zi * step) * pl2 + (size_t)b * pitch2 + a] = tile[r][threadIdx.x];
		}
	} else {
		for (int r = threadIdx.y; r < TX; r += TY) {
			const int zi = z0 + r, a = a0 + threadIdx.x;
			if (zi < count && a <= n1 + 1) tile[r][threadIdx.x] = x2[(size_t)(first + zi * step) * pl2 + (size_t)b * pitch2 + a];
		}
		__syncthreads();
		for (int r = threadIdx.y; r < TX; r += TY) {
			const int zi = z0 + threadIdx.x, a = a0 + r;
			if (zi < count && a <= n1 + 1) x3[o3(F, first + 1 + zi * step, a, b)] = tile[threadIdx.x][r];
		}
	}
}

template <typename T>
int plane_rhs(const T *so, const T *x, const T *b, Dims3 F, int dir, int first, int step, int count, T *b2, int n1,
              int n2, int pitch2, cudaStream_t st, int ns)
{
	if (dir == 2) {
		const dim3 grd(ceil_div(count, TX), ceil_div(n1, TX), n2);
		if (ns == 4) k3_plane_rhs_yz<T, 4><<<grd, dim3(TX, TY), 0, st>>>(so, x, b, F, first, step, count, b2, n1, n2, pitch2);
		else k3_plane_rhs_yz<T, 14><<<grd, dim3(TX, TY), 0, st>>>(so, x, b, F, first, step, count, b2, n1, n2, pitch2);
		CDR_LAUNCH_CHECK();
		return CDR_OK;
	}
	const dim3 grd(ceil_div(n1, TX), ceil_div(n2, TY), count);
	if (ns == 4) k3_plane_rhs<T, 4><<<grd, dim3(TX, TY), 0, st>>>(so, x, b, F, dir, first, step, b2, n1, n2, pitch2);
	else k3_plane_rhs<T, 14><<<grd, dim3(TX, TY), 0, st>>>(so, x, b, F, dir, first, step, b2, n1, n2, pitch2);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int plane_rhs<double>(const double *, const double *, const double *, Dims3, int, int, int, int, double *,
                               int, int, int, cudaStream_t, int);
template int plane_rhs<float>(const float *, const float *, const float *, Dims3, int, int, int, int, float *, int,
                              int, int, cudaStream_t, int);

int plane_coeff(const double *so, Dims3 F, int dir, double *so2, int n, int n1, int n2, int pitch2, cudaStream_t st,
                int ns)
{
	const int ns2 = ns == 4 ? 3 : 5;
	CDR_CUDA_TRY(cudaMemsetAsync(so2, 0, sizeof(double) * ns2 * (size_t)pitch2 * (n2 + 2) * n, st));
	const dim3 grd(ceil_div(n1 + 2, TX), ceil_div(n2 + 2, TY), n);
	if (ns == 4) k3_plane_coeff<3><<<grd, dim3(TX, TY), 0, st>>>(so, F, dir, so2, n1, n2, pitch2);
	else k3_plane_coeff<5><<<grd, dim3(TX, TY), 0, st>>>(so, F, dir, so2, n1, n2, pitch2);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

}  // namespace cdrgpu
