// k2_fe.cu -- bilinear (Q1) finite elements of -div(K grad u) on the device.
//
// The reference has only constant-coefficient gallery operators
// (src/2d/gallery.cc:7-113); heterogeneous problems and the differentiable
// solve need the operator assembled from per-cell coefficients, and its
// derivative.  A cell (cj, ci) of the (ny+1) x (nx+1) cell mesh has corner
// nodes (ci + a, cj + b), a, b in {0, 1}, in the ghost-inclusive node index
// (boundary nodes 0 and n+1 carry the Dirichlet zero).  K = diag(kx, ky) is
// constant per cell; on a square cell the element matrix is
//   A_e = kx * Ex + ky * Ey,  Ex = K1 (x) M1,  Ey = M1 (x) K1,
//   K1 = [[1,-1],[-1,1]],  M1 = [[2,1],[1,2]] / 6,
// with local node l = a + 2b.  The stencil is written in Cedar's storage
// (c, w, s, sw, nw; couplings negated; none into the ghost ring), summing cell
// contributions in a fixed order (cells (j,i), (j,i-1), (j-1,i), (j-1,i-1)
// of node (i, j)), so that it is bit-identical to the host assembler.
#include "k2_point.cuh"

namespace cdrgpu {

// Q1 element entries; a*, b* are local node coordinates in {0, 1}
__device__ __forceinline__ double q1_k1(int p, int q) { return p == q ? 1.0 : -1.0; }
__device__ __forceinline__ double q1_m1(int p, int q) { return (p == q ? 2.0 : 1.0) / 6.0; }
__device__ __forceinline__ double q1_ex(int a1, int b1, int a2, int b2) { return q1_k1(a1, a2) * q1_m1(b1, b2); }
__device__ __forceinline__ double q1_ey(int a1, int b1, int a2, int b2) { return q1_m1(a1, a2) * q1_k1(b1, b2); }

struct CellK {
	const double *kx, *ky;
	int cp;  // cell pitch
	__device__ double x(int cj, int ci) const { return kx[(size_t)cj * cp + ci]; }
	__device__ double y(int cj, int ci) const { return ky[(size_t)cj * cp + ci]; }
	// contribution kx*Ex[l1,l2] + ky*Ey[l1,l2] of cell (cj, ci)
	__device__ double e(int cj, int ci, int a1, int b1, int a2, int b2) const
	{
		return x(cj, ci) * q1_ex(a1, b1, a2, b2) + y(cj, ci) * q1_ey(a1, b1, a2, b2);
	}
};

__global__ void k_fe_assemble(CellK K, double *__restrict__ so, Dims2 d)
{
	const int i = blockIdx.x * TX + threadIdx.x + 1, j = blockIdx.y * TY + threadIdx.y + 1;
	if (i > d.nx || j > d.ny) return;
	const size_t ps = d.plane(), k = d.at(i, j);
	// diagonal: local node (a, b) of cell (j - b, i - a)
	double diag = 0.0;
	diag = diag + K.e(j, i, 0, 0, 0, 0);
	diag = diag + K.e(j, i - 1, 1, 0, 1, 0);
	diag = diag + K.e(j - 1, i, 0, 1, 0, 1);
	diag = diag + K.e(j - 1, i - 1, 1, 1, 1, 1);
	so[k] = diag;
	// coupling (i-1, j)-(i, j): bottom edge of cell (j, i-1), top edge of cell (j-1, i-1)
	if (i >= 2) {
		double aw = 0.0;
		aw = aw + K.e(j, i - 1, 0, 0, 1, 0);
		aw = aw + K.e(j - 1, i - 1, 0, 1, 1, 1);
		so[ps + k] = -aw;
	}
	// coupling (i, j-1)-(i, j): left edge of cell (j-1, i), right edge of cell (j-1, i-1)
	if (j >= 2) {
		double as = 0.0;
		as = as + K.e(j - 1, i, 0, 0, 0, 1);
		as = as + K.e(j - 1, i - 1, 1, 0, 1, 1);
		so[2 * ps + k] = -as;
	}
	// diagonals of cell (j-1, i-1), whose NE corner is (i, j)
	if (i >= 2 && j >= 2) {
		so[3 * ps + k] = -K.e(j - 1, i - 1, 0, 0, 1, 1);
		so[4 * ps + k] = -K.e(j - 1, i - 1, 1, 0, 0, 1);
	}
}

// dL/dkx_e = -lam_e^T Ex u_e and dL/dky_e = -lam_e^T Ey u_e per cell, for
// A(k) u = f and lam = A^{-T} dL/du (A is symmetric); boundary nodes carry 0.
__global__ void k_fe_grad(const double *__restrict__ u, const double *__restrict__ lam, Dims2 d,
                          double *__restrict__ gkx, double *__restrict__ gky, int cp)
{
	const int ci = blockIdx.x * TX + threadIdx.x, cj = blockIdx.y * TY + threadIdx.y;
	if (ci > d.nx || cj > d.ny) return;
	double ul[4], ll[4];
#pragma unroll
	for (int l = 0; l < 4; ++l) {
		const int a = l & 1, b = l >> 1;
		const int ni = ci + a, nj = cj + b;
		const bool inner = ni >= 1 && ni <= d.nx && nj >= 1 && nj <= d.ny;
		ul[l] = inner ? u[d.at(ni, nj)] : 0.0;
		ll[l] = inner ? lam[d.at(ni, nj)] : 0.0;
	}
	double sx = 0.0, sy = 0.0;
#pragma unroll
	for (int l1 = 0; l1 < 4; ++l1)
#pragma unroll
		for (int l2 = 0; l2 < 4; ++l2) {
			sx += ll[l1] * q1_ex(l1 & 1, l1 >> 1, l2 & 1, l2 >> 1) * ul[l2];
			sy += ll[l1] * q1_ey(l1 & 1, l1 >> 1, l2 & 1, l2 >> 1) * ul[l2];
		}
	gkx[(size_t)cj * cp + ci] = -sx;
	gky[(size_t)cj * cp + ci] = -sy;
}

}  // namespace cdrgpu

using namespace cdrgpu;

extern "C" {

int cdr_gpu_fe_assemble_2d_f64(const double *kx, const double *ky, int cell_pitch, double *so, int nx, int ny,
                               int pitch, cudaStream_t stream)
{
	if (!kx || !ky || !so) { set_error(CDR_ERR_ARG, "null pointer"); return CDR_ERR_ARG; }
	if (nx < 1 || ny < 1 || pitch < nx + 2 || cell_pitch < nx + 1) {
		set_error(CDR_ERR_DIM, "bad grid nx=%d ny=%d pitch=%d cell_pitch=%d", nx, ny, pitch, cell_pitch);
		return CDR_ERR_DIM;
	}
	const Dims2 d{nx, ny, pitch};
	CDR_CUDA_TRY(cudaMemsetAsync(so, 0, sizeof(double) * d.plane() * 5, stream));
	k_fe_assemble<<<dim3(ceil_div(nx, TX), ceil_div(ny, TY)), dim3(TX, TY), 0, stream>>>(CellK{kx, ky, cell_pitch}, so,
	                                                                                     d);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

int cdr_gpu_fe_grad_2d_f64(const double *u, const double *lam, int nx, int ny, int pitch, double *gkx, double *gky,
                           int cell_pitch, cudaStream_t stream)
{
	if (!u || !lam || !gkx || !gky) { set_error(CDR_ERR_ARG, "null pointer"); return CDR_ERR_ARG; }
	if (nx < 1 || ny < 1 || pitch < nx + 2 || cell_pitch < nx + 1) {
		set_error(CDR_ERR_DIM, "bad grid nx=%d ny=%d pitch=%d cell_pitch=%d", nx, ny, pitch, cell_pitch);
		return CDR_ERR_DIM;
	}
	const Dims2 d{nx, ny, pitch};
	k_fe_grad<<<dim3(ceil_div(nx + 1, TX), ceil_div(ny + 1, TY)), dim3(TX, TY), 0, stream>>>(u, lam, d, gkx, gky,
	                                                                                        cell_pitch);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Trilinear (Q1) elements in 3D: -div(k grad u), k scalar per cell, cube cells
// of side h = 1/(nx+1).  A_e = h * k * (Ex + Ey + Ez) with
// Ex = K1 (x) M1 (x) M1, Ey = M1 (x) K1 (x) M1, Ez = M1 (x) M1 (x) K1, local node
// l = a + 2b + 4c.  Entry of plane q at node s couples nodes s + oa and s + ob
// (offsets per plane below, both nodes interior) and equals minus the sum over
// the element pairs (l1, l2) with o(l2) - o(l1) = ob - oa, in the order
// l1 = 0..7, l2 = 0..7, of k(cell (s + oa) - o(l1)) * A_e[l1, l2]; the p plane
// is the plain sum at offset 0.  This fixed order makes the result identical to
// the host assembler in the package's gallery.
namespace cdrgpu {

__device__ __forceinline__ double q1_ae3(double h, int l1, int l2)
{
	const int a1 = l1 & 1, b1 = (l1 >> 1) & 1, c1 = l1 >> 2, a2 = l2 & 1, b2 = (l2 >> 1) & 1, c2 = l2 >> 2;
	const double ex = q1_k1(a1, a2) * q1_m1(b1, b2) * q1_m1(c1, c2);
	const double ey = q1_m1(a1, a2) * q1_k1(b1, b2) * q1_m1(c1, c2);
	const double ez = q1_m1(a1, a2) * q1_m1(b1, b2) * q1_k1(c1, c2);
	return h * (ex + ey + ez);
}

// (oa, ob) of the 14 planes p pw ps b psw pnw bw bnw bn bne be bse bs bsw, as (x, y, z)
__constant__ signed char c_planes3[14][2][3] = {
    {{0, 0, 0}, {0, 0, 0}},    {{0, 0, 0}, {-1, 0, 0}},    {{0, 0, 0}, {0, -1, 0}},   {{0, 0, 0}, {0, 0, -1}},
    {{0, 0, 0}, {-1, -1, 0}},  {{0, -1, 0}, {-1, 0, 0}},   {{0, 0, 0}, {-1, 0, -1}},  {{0, -1, 0}, {-1, 0, -1}},
    {{0, -1, 0}, {0, 0, -1}},  {{-1, -1, 0}, {0, 0, -1}},  {{-1, 0, 0}, {0, 0, -1}},  {{-1, 0, 0}, {0, -1, -1}},
    {{0, 0, 0}, {0, -1, -1}},  {{0, 0, 0}, {-1, -1, -1}}};

__global__ void k_fe_assemble3(const double *__restrict__ kc, int cp, int cs, double *__restrict__ so, int nx, int ny,
                               int nz, int pitch)
{
	const int i = blockIdx.x * TX + threadIdx.x + 1, j = blockIdx.y * TY + threadIdx.y + 1, k = blockIdx.z + 1;
	if (i > nx || j > ny) return;
	const double h = 1.0 / (nx + 1);
	const size_t slice = (size_t)pitch * (ny + 2), plane = slice * (nz + 2);
	const size_t at = (size_t)k * slice + (size_t)j * pitch + i;
	for (int q = 0; q < 14; ++q) {
		const int ax = i + c_planes3[q][0][0], ay = j + c_planes3[q][0][1], az = k + c_planes3[q][0][2];
		const int bx = i + c_planes3[q][1][0], by = j + c_planes3[q][1][1], bz = k + c_planes3[q][1][2];
		if (ax < 1 || ay < 1 || az < 1 || bx < 1 || by < 1 || bz < 1) continue;  // upper bounds hold for s interior
		const int dx = bx - ax, dy = by - ay, dz = bz - az;
		double acc = 0.0;
		for (int l1 = 0; l1 < 8; ++l1)
			for (int l2 = 0; l2 < 8; ++l2) {
				if (((l2 & 1) - (l1 & 1)) != dx || (((l2 >> 1) & 1) - ((l1 >> 1) & 1)) != dy || ((l2 >> 2) - (l1 >> 2)) != dz)
					continue;
				const int ci = ax - (l1 & 1), cj = ay - ((l1 >> 1) & 1), ck = az - (l1 >> 2);
				acc = acc + kc[(size_t)ck * cs + (size_t)cj * cp + ci] * q1_ae3(h, l1, l2);
			}
		so[(size_t)q * plane + at] = q == 0 ? acc : -acc;
	}
}

}  // namespace cdrgpu

extern "C" int cdr_gpu_fe_assemble_3d_f64(const double *k, int cell_pitch, int cell_slice, double *so, int nx, int ny,
                                          int nz, int pitch, cudaStream_t stream)
{
	if (!k || !so) { set_error(CDR_ERR_ARG, "null pointer"); return CDR_ERR_ARG; }
	if (nx < 1 || ny < 1 || nz < 1 || pitch < nx + 2 || cell_pitch < nx + 1 ||
	    (size_t)cell_slice < (size_t)cell_pitch * (ny + 1)) {
		set_error(CDR_ERR_DIM, "bad grid nx=%d ny=%d nz=%d pitch=%d cell_pitch=%d cell_slice=%d", nx, ny, nz, pitch,
		          cell_pitch, cell_slice);
		return CDR_ERR_DIM;
	}
	const size_t plane = (size_t)pitch * (ny + 2) * (nz + 2);
	CDR_CUDA_TRY(cudaMemsetAsync(so, 0, sizeof(double) * plane * 14, stream));
	k_fe_assemble3<<<dim3(ceil_div(nx, TX), ceil_div(ny, TY), nz), dim3(TX, TY), 0, stream>>>(k, cell_pitch, cell_slice,
	                                                                                         so, nx, ny, nz, pitch);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
