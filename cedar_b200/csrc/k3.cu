// k3.cu -- 3D BoxMG kernels (27- and 7-point fine operators) for sm_100a.
//
// Layout: Cedar's 3D arrays with one ghost layer, i fastest, rows padded to a
// pitch; a k-slice is pitch*(ny+2) elements, a stencil plane
// pitch*(ny+2)*(nz+2).  Stencil planes (include/cedar/3d/base_types.h:4-20,
// 1-based as in src/3d/ftn/BMG_stencils_f90.h): kp kpw kps kb kpsw kpnw kbw kbnw
// kbn kbne kbe kbse kbs kbsw; interpolation weights: 26 planes lxyl .. ltse.
// A seven-point operator (include/cedar/3d/base_types.h seven_pt) keeps the
// first four planes only: p, pw, ps, b.
// Kernel bodies address arrays with the reference's 1-based (I, J, K) through
// the macros below and keep its operand order, so they reproduce its bits
// (the library is built without FMA contraction).
#include "k2_point.cuh"
#include "kernels3d.cuh"

namespace cdrgpu {

#define SO(i, j, k, p) so[(size_t)((p)-1) * F.plane() + F.at1(i, j, k)]
#define Q(i, j, k) q[F.at1(i, j, k)]
#define QF(i, j, k) qf[F.at1(i, j, k)]
#define CI(i, j, k, l) ci[(size_t)((l)-1) * C.plane() + C.at1(i, j, k)]
#define QC(i, j, k) qc[C.at1(i, j, k)]

// qf plus the 26 neighbour terms of BMG3_SymStd_residual.f90:76-101, in its
// order; xq(i, j, k) supplies the iterate (a plain load, or x + e in the
// refinement step)
template <typename T, typename XQ>
__device__ __forceinline__ T nb27(const T *__restrict__ so, XQ xq, T qf, Dims3 F, int i, int j, int k)
{
	T nb = qf + SO(i, j, k, KPW) * xq(i - 1, j, k);
	nb = nb + SO(i, j + 1, k, KPNW) * xq(i - 1, j + 1, k) + SO(i, j + 1, k, KPS) * xq(i, j + 1, k)
	     + SO(i + 1, j + 1, k, KPSW) * xq(i + 1, j + 1, k) + SO(i + 1, j, k, KPW) * xq(i + 1, j, k)
	     + SO(i + 1, j, k, KPNW) * xq(i + 1, j - 1, k) + SO(i, j, k, KPS) * xq(i, j - 1, k)
	     + SO(i, j, k, KPSW) * xq(i - 1, j - 1, k) + SO(i, j, k, KB) * xq(i, j, k - 1)
	     + SO(i, j, k, KBW) * xq(i - 1, j, k - 1) + SO(i, j + 1, k, KBNW) * xq(i - 1, j + 1, k - 1)
	     + SO(i, j + 1, k, KBN) * xq(i, j + 1, k - 1) + SO(i + 1, j + 1, k, KBNE) * xq(i + 1, j + 1, k - 1)
	     + SO(i + 1, j, k, KBE) * xq(i + 1, j, k - 1) + SO(i + 1, j, k, KBSE) * xq(i + 1, j - 1, k - 1)
	     + SO(i, j, k, KBS) * xq(i, j - 1, k - 1) + SO(i, j, k, KBSW) * xq(i - 1, j - 1, k - 1)
	     + SO(i, j, k + 1, KB) * xq(i, j, k + 1) + SO(i, j, k + 1, KBE) * xq(i - 1, j, k + 1)
	     + SO(i, j + 1, k + 1, KBSE) * xq(i - 1, j + 1, k + 1) + SO(i, j + 1, k + 1, KBS) * xq(i, j + 1, k + 1)
	     + SO(i + 1, j + 1, k + 1, KBSW) * xq(i + 1, j + 1, k + 1) + SO(i + 1, j, k + 1, KBW) * xq(i + 1, j, k + 1)
	     + SO(i + 1, j, k + 1, KBNW) * xq(i + 1, j - 1, k + 1) + SO(i, j, k + 1, KBN) * xq(i, j - 1, k + 1)
	     + SO(i, j, k + 1, KBNE) * xq(i - 1, j - 1, k + 1);
	return nb;
}

// qf plus the 6 neighbour terms of the seven-point branch
// (BMG3_SymStd_residual.f90:104-119), in its order.
template <typename T, typename XQ>
__device__ __forceinline__ T nb7(const T *__restrict__ so, XQ xq, T qf, Dims3 F, int i, int j, int k)
{
	return qf + SO(i, j, k, KPW) * xq(i - 1, j, k) + SO(i, j + 1, k, KPS) * xq(i, j + 1, k)
	       + SO(i + 1, j, k, KPW) * xq(i + 1, j, k) + SO(i, j, k, KPS) * xq(i, j - 1, k)
	       + SO(i, j, k, KB) * xq(i, j, k - 1) + SO(i, j, k + 1, KB) * xq(i, j, k + 1);
}

// Neighbour sum of an NS-plane operator: 14 (27-point) or 4 (seven-point).
template <int NS, typename T, typename XQ>
__device__ __forceinline__ T nbs(const T *__restrict__ so, XQ xq, T qf, Dims3 F, int i, int j, int k)
{
	if constexpr (NS == 4) return nb7<T>(so, xq, qf, F, i, j, k);
	else return nb27<T>(so, xq, qf, F, i, j, k);
}

template <typename T>
struct Load3 {
	const T *__restrict__ q;
	Dims3 F;
	__device__ __forceinline__ T operator()(int i, int j, int k) const { return q[F.at1(i, j, k)]; }
};

// --------------------------------------------------------------- residual
// BMG3_SymStd_residual (src/3d/ftn/BMG3_SymStd_residual.f90:67-121); grid-stride
// over 32x8 tiles of every k-slice, FP64 partial sums of r^2 per block.
template <typename T, bool NORM, int NS>
__global__ void __launch_bounds__(TX *TY) k3_residual(const T *__restrict__ so, const T *__restrict__ q,
                                                      const T *__restrict__ qf, T *__restrict__ res, Dims3 F,
                                                      double *__restrict__ partial)
{
	__shared__ double sh[TX * TY / 32];
	const int tx = (F.nx + TX - 1) / TX, ty = (F.ny + TY - 1) / TY;
	const long ntiles = (long)tx * ty * F.nz;
	double acc = 0.0;
	for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
		const int kk = (int)(t / ((long)tx * ty));
		const int rem = (int)(t - (long)kk * tx * ty);
		const int i = (rem % tx) * TX + threadIdx.x + 2, j = (rem / tx) * TY + threadIdx.y + 2, k = kk + 2;
		if (i <= F.nx + 1 && j <= F.ny + 1) {
			const T r = nbs<NS, T>(so, Load3<T>{q, F}, QF(i, j, k), F, i, j, k) - SO(i, j, k, KP) * Q(i, j, k);
			res[F.at1(i, j, k)] = r;
			if (NORM) acc += (double)r * (double)r;
		}
	}
	if (NORM) {
		const double s = block_sum<TX * TY / 32>(acc, sh);
		if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x] = s;
	}
}

__global__ void __launch_bounds__(1024) k3_norm_finish(const double *__restrict__ partial, int n, double *out)
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

template <typename T>
int residual_3d(const T *so, const T *x, const T *b, T *r, Dims3 F, double *norm_out, double *partial, cudaStream_t st,
                int ns)
{
	const long ntiles = (long)ceil_div(F.nx, TX) * ceil_div(F.ny, TY) * F.nz;
	const int nb = ntiles < 2048 ? (int)ntiles : 2048;
	if (norm_out) {
		if (ns == 4) k3_residual<T, true, 4><<<nb, dim3(TX, TY), 0, st>>>(so, x, b, r, F, partial);
		else k3_residual<T, true, 14><<<nb, dim3(TX, TY), 0, st>>>(so, x, b, r, F, partial);
		CDR_LAUNCH_CHECK();
		k3_norm_finish<<<1, 1024, 0, st>>>(partial, nb, norm_out);
	} else {
		const int nb2 = ntiles < 148 * 64 ? (int)ntiles : 148 * 64;
		if (ns == 4) k3_residual<T, false, 4><<<nb2, dim3(TX, TY), 0, st>>>(so, x, b, r, F, nullptr);
		else k3_residual<T, false, 14><<<nb2, dim3(TX, TY), 0, st>>>(so, x, b, r, F, nullptr);
	}
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int residual_3d<double>(const double *, const double *, const double *, double *, Dims3, double *, double *,
                                 cudaStream_t, int);
template int residual_3d<float>(const float *, const float *, const float *, float *, Dims3, double *, double *,
                                cudaStream_t, int);

// ----------------------------------------------------------------- smoother
// BMG3_SymStd_SETUP_recip (src/3d/ftn/BMG3_SymStd_SETUP_recip.f90:63-69)
template <typename T>
__global__ void k3_recip(const T *__restrict__ so, T *__restrict__ sor, Dims3 F)
{
	const int i = blockIdx.x * TX + threadIdx.x + 2, j = blockIdx.y * TY + threadIdx.y + 2, k = blockIdx.z + 2;
	if (i > F.nx + 1 || j > F.ny + 1) return;
	sor[F.at1(i, j, k)] = T(1) / SO(i, j, k, KP);
}

// One colour of BMG3_SymStd_relax_GS (src/3d/ftn/BMG3_SymStd_relax_GS.f90:94-136):
// colour pts has parities (i, j, k) = bits of pts-1.
template <typename T>
__global__ void __launch_bounds__(TX *TY) k3_gs_colour(const T *__restrict__ so, T *__restrict__ q,
                                                       const T *__restrict__ qf, const T *__restrict__ sor, Dims3 F,
                                                       int pi, int pj, int pk)
{
	const int i = 2 + pi + 2 * (blockIdx.x * TX + threadIdx.x);
	const int j = 2 + pj + 2 * (blockIdx.y * TY + threadIdx.y);
	const int k = 2 + pk + 2 * blockIdx.z;
	if (i > F.nx + 1 || j > F.ny + 1 || k > F.nz + 1) return;
	const T acc = nb27<T>(so, Load3<T>{q, F}, QF(i, j, k), F, i, j, k);
	Q(i, j, k) = acc * sor[F.at1(i, j, k)];
}

// One colour of the seven-point branch of BMG3_SymStd_relax_GS
// (BMG3_SymStd_relax_GS.f90:141-180): colour pts (0 or 1) holds the points
// with I + J + K + pts even.
template <typename T>
__global__ void __launch_bounds__(TX *TY) k3_gs7_colour(const T *__restrict__ so, T *__restrict__ q,
                                                        const T *__restrict__ qf, const T *__restrict__ sor, Dims3 F,
                                                        int pts)
{
	const int j = 2 + blockIdx.y * TY + threadIdx.y, k = 2 + blockIdx.z;
	const int i = 2 + ((j + k + pts) & 1) + 2 * (blockIdx.x * TX + threadIdx.x);
	if (i > F.nx + 1 || j > F.ny + 1) return;
	Q(i, j, k) = nb7<T>(so, Load3<T>{q, F}, QF(i, j, k), F, i, j, k) * sor[F.at1(i, j, k)];
}

template <typename T>
int relax_point_3d(const T *so, T *x, const T *b, const T *sor, Dims3 F, int updown, cudaStream_t st, int ns)
{
	if (ns == 4) {  // UP (and the non-symmetric sweep): colour 0 then 1; DOWN: 1 then 0
		const dim3 blk(TX, TY), grd(ceil_div((F.nx + 1) / 2, TX), ceil_div(F.ny, TY), F.nz);
		for (int c = 0; c < 2; ++c) {
			k3_gs7_colour<T><<<grd, blk, 0, st>>>(so, x, b, sor, F, updown == CDR_DOWN ? 1 - c : c);
			CDR_LAUNCH_CHECK();
		}
		return CDR_OK;
	}
	const dim3 blk(TX, TY), grd(ceil_div((F.nx + 1) / 2, TX), ceil_div((F.ny + 1) / 2, TY), (F.nz + 1) / 2);
	for (int c = 0; c < 8; ++c) {
		const int pts = updown == CDR_UP ? c + 1 : 8 - c;  // UP 1..8, DOWN 8..1
		const int bits = pts - 1;
		k3_gs_colour<T><<<grd, blk, 0, st>>>(so, x, b, sor, F, bits & 1, (bits >> 1) & 1, (bits >> 2) & 1);
		CDR_LAUNCH_CHECK();
	}
	return CDR_OK;
}
template int relax_point_3d<double>(const double *, double *, const double *, const double *, Dims3, int, cudaStream_t,
                                    int);
template int relax_point_3d<float>(const float *, float *, const float *, const float *, Dims3, int, cudaStream_t, int);

template <typename T>
int setup_recip_3d(const T *so, T *sor, Dims3 F, cudaStream_t st)
{
	k3_recip<T><<<dim3(ceil_div(F.nx, TX), ceil_div(F.ny, TY), F.nz), dim3(TX, TY), 0, st>>>(so, sor, F);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int setup_recip_3d<double>(const double *, double *, Dims3, cudaStream_t);

// ----------------------------------------------------------------- transfers
// BMG3_SymStd_restrict (src/3d/ftn/BMG3_SymStd_restrict.f90:114-154)
template <typename T>
__global__ void __launch_bounds__(TX *TY) k3_restrict(const T *__restrict__ ci, const T *__restrict__ q,
                                                      T *__restrict__ qc, Dims3 F, Dims3 C)
{
	const int ic = blockIdx.x * TX + threadIdx.x + 2, jc = blockIdx.y * TY + threadIdx.y + 2, kc = blockIdx.z + 2;
	if (ic > C.nx + 1 || jc > C.ny + 1) return;
	const int i = 2 * ic - 2, j = 2 * jc - 2, k = 2 * kc - 2;
	QC(ic, jc, kc) = CI(ic, jc, kc, LXYNE) * Q(i - 1, j - 1, k) + CI(ic, jc, kc, LXYA) * Q(i, j - 1, k)
	                 + CI(ic + 1, jc, kc, LXYNW) * Q(i + 1, j - 1, k) + CI(ic, jc, kc, LXYR) * Q(i - 1, j, k) + Q(i, j, k)
	                 + CI(ic + 1, jc, kc, LXYL) * Q(i + 1, j, k) + CI(ic, jc + 1, kc, LXYSE) * Q(i - 1, j + 1, k)
	                 + CI(ic, jc + 1, kc, LXYB) * Q(i, j + 1, k) + CI(ic + 1, jc + 1, kc, LXYSW) * Q(i + 1, j + 1, k)
	                 + CI(ic, jc, kc, LTNE) * Q(i - 1, j - 1, k - 1) + CI(ic, jc, kc, LYZNW) * Q(i, j - 1, k - 1)
	                 + CI(ic + 1, jc, kc, LTNW) * Q(i + 1, j - 1, k - 1) + CI(ic, jc, kc, LXZNE) * Q(i - 1, j, k - 1)
	                 + CI(ic, jc, kc, LXZA) * Q(i, j, k - 1) + CI(ic + 1, jc, kc, LXZNW) * Q(i + 1, j, k - 1)
	                 + CI(ic, jc + 1, kc, LTSE) * Q(i - 1, j + 1, k - 1) + CI(ic, jc + 1, kc, LYZNE) * Q(i, j + 1, k - 1)
	                 + CI(ic + 1, jc + 1, kc, LTSW) * Q(i + 1, j + 1, k - 1) + CI(ic, jc, kc + 1, LBNE) * Q(i - 1, j - 1, k + 1)
	                 + CI(ic, jc, kc + 1, LYZSW) * Q(i, j - 1, k + 1) + CI(ic + 1, jc, kc + 1, LBNW) * Q(i + 1, j - 1, k + 1)
	                 + CI(ic, jc, kc + 1, LXZSE) * Q(i - 1, j, k + 1) + CI(ic, jc, kc + 1, LXZB) * Q(i, j, k + 1)
	                 + CI(ic + 1, jc, kc + 1, LXZSW) * Q(i + 1, j, k + 1) + CI(ic, jc + 1, kc + 1, LBSE) * Q(i - 1, j + 1, k + 1)
	                 + CI(ic, jc + 1, kc + 1, LYZSE) * Q(i, j + 1, k + 1) + CI(ic + 1, jc + 1, kc + 1, LBSW) * Q(i + 1, j + 1, k + 1);
}

// BMG3_SymStd_interp_add (src/3d/ftn/BMG3_SymStd_interp_add.f90:108-239).  The
// reference's three loop nests write disjoint sets of fine points and each
// update reads only its own target in q, so one thread per (IC, JC, KC) does the
// writes of all three nests.  r/c is formed on the fly (the reference divides
// r in place on interior points; a ghost-layer point, reached for even sizes,
// adds r undivided).
template <typename T>
__global__ void __launch_bounds__(TX *TY) k3_interp_add(const T *__restrict__ ci, const T *__restrict__ qc,
                                                        const T *__restrict__ res, const T *__restrict__ so,
                                                        T *__restrict__ q, Dims3 F, Dims3 C)
{
	const int ic = blockIdx.x * TX + threadIdx.x + 2, jc = blockIdx.y * TY + threadIdx.y + 2, kc = blockIdx.z + 2;
	const int iic1 = C.nx + 1, kkc1 = C.nz + 1;
	const int iicf1 = F.nx / 2 + 2, jjcf1 = F.ny / 2 + 2, kkcf1 = F.nz / 2 + 2;
	if (ic > iicf1 || jc > jjcf1) return;
	auto RES = [&](int i, int j, int k) -> T {
		const size_t o = F.at1(i, j, k);
		const bool in = i >= 2 && i <= F.nx + 1 && j >= 2 && j <= F.ny + 1 && k >= 2 && k <= F.nz + 1;
		return in ? res[o] / so[o] : res[o];
	};
	if (kc <= kkc1) {  // coarse-aligned k-planes, k = 2KC-2: the 2D pattern
		const int k = 2 * kc - 2, i = 2 * ic - 2, j = 2 * jc - 2;
		Q(i, j, k) = Q(i, j, k) + QC(ic, jc, kc);
		if (ic >= 3) {
			const T a = CI(ic, jc, kc, LXYR) * QC(ic, jc, kc) + CI(ic, jc, kc, LXYL) * QC(ic - 1, jc, kc);
			Q(i - 1, j, k) = Q(i - 1, j, k) + a + RES(i - 1, j, k);
		}
		if (jc >= 3) {
			const T aq = CI(ic, jc, kc, LXYA) * QC(ic, jc, kc) + CI(ic, jc, kc, LXYB) * QC(ic, jc - 1, kc);
			Q(i, j - 1, k) = Q(i, j - 1, k) + aq + RES(i, j - 1, k);
		}
		if (ic >= 3 && jc >= 3) {
			const T a = CI(ic, jc, kc, LXYSW) * QC(ic - 1, jc - 1, kc) + CI(ic, jc, kc, LXYNW) * QC(ic - 1, jc, kc)
			            + CI(ic, jc, kc, LXYNE) * QC(ic, jc, kc) + CI(ic, jc, kc, LXYSE) * QC(ic, jc - 1, kc);
			Q(i - 1, j - 1, k) = Q(i - 1, j - 1, k) + a + RES(i - 1, j - 1, k);
		}
	}
	if (kc < 3 || kc > kkcf1) return;
	const int k = 2 * kc - 3, j = 2 * jc - 2;
	if (ic <= iic1) {  // fine-only k-planes, coarse-aligned x: i = 2IC-2
		const int i = 2 * ic - 2;
		Q(i, j, k) = Q(i, j, k) + CI(ic, jc, kc, LXZA) * QC(ic, jc, kc) + CI(ic, jc, kc, LXZB) * QC(ic, jc, kc - 1)
		             + RES(i, j, k);
		if (jc >= 3)
			Q(i, j - 1, k) = Q(i, j - 1, k) + CI(ic, jc, kc, LYZNW) * QC(ic, jc, kc) + CI(ic, jc, kc, LYZNE) * QC(ic, jc - 1, kc)
			                 + CI(ic, jc, kc, LYZSW) * QC(ic, jc, kc - 1) + CI(ic, jc, kc, LYZSE) * QC(ic, jc - 1, kc - 1)
			                 + RES(i, j - 1, k);
	}
	if (ic >= 3) {  // fine-only k-planes, fine-only x: i = 2IC-3
		const int i = 2 * ic - 3;
		Q(i, j, k) = Q(i, j, k) + CI(ic, jc, kc, LXZNW) * QC(ic - 1, jc, kc) + CI(ic, jc, kc, LXZNE) * QC(ic, jc, kc)
		             + CI(ic, jc, kc, LXZSW) * QC(ic - 1, jc, kc - 1) + CI(ic, jc, kc, LXZSE) * QC(ic, jc, kc - 1)
		             + RES(i, j, k);
		if (jc >= 3)
			Q(i, j - 1, k) = Q(i, j - 1, k) + CI(ic, jc, kc, LTNW) * QC(ic - 1, jc, kc) + CI(ic, jc, kc, LTNE) * QC(ic, jc, kc)
			                 + CI(ic, jc, kc, LTSW) * QC(ic - 1, jc - 1, kc) + CI(ic, jc, kc, LTSE) * QC(ic, jc - 1, kc)
			                 + CI(ic, jc, kc, LBNW) * QC(ic - 1, jc, kc - 1) + CI(ic, jc, kc, LBNE) * QC(ic, jc, kc - 1)
			                 + CI(ic, jc, kc, LBSW) * QC(ic - 1, jc - 1, kc - 1) + CI(ic, jc, kc, LBSE) * QC(ic, jc - 1, kc - 1)
			                 + RES(i, j - 1, k);
	}
}

template <typename T>
int restrict_3d(const T *ci, const T *rf, T *bc, Dims3 F, Dims3 C, cudaStream_t st)
{
	k3_restrict<T><<<dim3(ceil_div(C.nx, TX), ceil_div(C.ny, TY), C.nz), dim3(TX, TY), 0, st>>>(ci, rf, bc, F, C);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int restrict_3d<double>(const double *, const double *, double *, Dims3, Dims3, cudaStream_t);
template int restrict_3d<float>(const float *, const float *, float *, Dims3, Dims3, cudaStream_t);

template <typename T>
int interp_add_3d(const T *ci, const T *xc, const T *rf, const T *sof, T *xf, Dims3 F, Dims3 C, cudaStream_t st)
{
	const dim3 grd(ceil_div(F.nx / 2 + 1, TX), ceil_div(F.ny / 2 + 1, TY), F.nz / 2 + 1);
	k3_interp_add<T><<<grd, dim3(TX, TY), 0, st>>>(ci, xc, rf, sof, xf, F, C);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int interp_add_3d<double>(const double *, const double *, const double *, const double *, double *, Dims3,
                                   Dims3, cudaStream_t);
template int interp_add_3d<float>(const float *, const float *, const float *, const float *, float *, Dims3, Dims3,
                                  cudaStream_t);

// ------------------------------------------------ operator-induced interpolation
// BMG3_SymStd_SETUP_interp_OI (src/3d/ftn/BMG3_SymStd_SETUP_interp_OI.f90:121-537),
// non-periodic, 27-point fine operator.  Launch 0: edge weights (x-, y-, z-edges);
// launch 1: face weights (xy, xz, yz), which read edge weights; launch 2:
// interior weights, which read face and edge weights.  Every thread handles one
// (IC, JC, KC) and the fine point (2IC-2, 2JC-2, 2KC-2) the formulas are centred on.
__device__ __forceinline__ double dmin2(double a, double b) { return a < b ? a : b; }

__global__ void __launch_bounds__(TX *TY) k3_oi(const double *__restrict__ so, double *__restrict__ ci, Dims3 F,
                                                Dims3 C, int phase)
{
	const int ic = blockIdx.x * TX + threadIdx.x + 2, jc = blockIdx.y * TY + threadIdx.y + 2, kc = blockIdx.z + 2;
	const int iic1 = C.nx + 1, jjc1 = C.ny + 1, kkc1 = C.nz + 1;
	const int iicf1 = F.nx / 2 + 2, jjcf1 = F.ny / 2 + 2, kkcf1 = F.nz / 2 + 2;
	const double emach = 1.1102230246251565e-16;
	const int i = 2 * ic - 2, j = 2 * jc - 2, k = 2 * kc - 2;
	double a, b, c, ep, dnw, dn, dne, dw, de, dsw, ds, dse, dp, sum;
	if (phase == 0) {
		if (kc <= kkc1 && jc <= jjc1 && ic >= 3 && ic <= iicf1) {  // x-edges: lxyl, lxyr
			a = SO(i - 1, j + 1, k, KPNW) + SO(i - 1, j, k, KPW) + SO(i - 1, j, k, KPSW) + SO(i - 1, j + 1, k, KBNW)
			    + SO(i - 1, j, k, KBW) + SO(i - 1, j, k, KBSW) + SO(i - 1, j + 1, k + 1, KBSE) + SO(i - 1, j, k + 1, KBE)
			    + SO(i - 1, j, k + 1, KBNE);
			b = SO(i, j + 1, k, KPSW) + SO(i, j, k, KPW) + SO(i, j, k, KPNW) + SO(i, j + 1, k, KBNE) + SO(i, j, k, KBE)
			    + SO(i, j, k, KBSE) + SO(i, j + 1, k + 1, KBSW) + SO(i, j, k + 1, KBW) + SO(i, j, k + 1, KBNW);
			c = a + b + SO(i - 1, j, k, KPS) + SO(i - 1, j + 1, k, KPS) + SO(i - 1, j + 1, k, KBN) + SO(i - 1, j, k, KB)
			    + SO(i - 1, j, k, KBS) + SO(i - 1, j + 1, k + 1, KBS) + SO(i - 1, j, k + 1, KB) + SO(i - 1, j, k + 1, KBN);
			ep = dmin2(fabs(a / SO(i - 1, j, k, KP)), fabs(b / SO(i - 1, j, k, KP)));
			c = a + b + (SO(i - 1, j, k, KP) - c) * fmax(SO(i - 1, j, k, KP) - (1.0 + ep) * c, 0.0)
			            / (fabs(SO(i - 1, j, k, KP) - (1.0 + ep) * c) + emach);
			CI(ic, jc, kc, LXYL) = a / c;
			CI(ic, jc, kc, LXYR) = b / c;
		}
		if (kc <= kkc1 && jc >= 3 && jc <= jjcf1 && ic <= iic1) {  // y-edges: lxya, lxyb
			a = SO(i, j, k, KPNW) + SO(i, j, k, KPS) + SO(i + 1, j, k, KPSW) + SO(i, j, k, KBNW) + SO(i, j, k, KBN)
			    + SO(i + 1, j, k, KBNE) + SO(i, j, k + 1, KBSE) + SO(i, j, k + 1, KBS) + SO(i + 1, j, k + 1, KBSW);
			b = SO(i, j - 1, k, KPSW) + SO(i, j - 1, k, KPS) + SO(i + 1, j - 1, k, KPNW) + SO(i, j - 1, k, KBSW)
			    + SO(i, j - 1, k, KBS) + SO(i + 1, j - 1, k, KBSE) + SO(i, j - 1, k + 1, KBNE) + SO(i, j - 1, k + 1, KBN)
			    + SO(i + 1, j - 1, k + 1, KBNW);
			ep = dmin2(fabs(a / SO(i, j - 1, k, KP)), fabs(b / SO(i, j - 1, k, KP)));
			c = a + b + SO(i, j - 1, k, KPW) + SO(i + 1, j - 1, k, KPW) + SO(i, j - 1, k, KBW) + SO(i, j - 1, k, KB)
			    + SO(i + 1, j - 1, k, KBE) + SO(i, j - 1, k + 1, KBE) + SO(i, j - 1, k + 1, KB) + SO(i + 1, j - 1, k + 1, KBW);
			c = a + b + (SO(i, j - 1, k, KP) - c) * fmax(SO(i, j - 1, k, KP) - (1.0 + ep) * c, 0.0)
			            / (fabs(SO(i, j - 1, k, KP) - (1.0 + ep) * c) + emach);
			CI(ic, jc, kc, LXYA) = a / c;
			CI(ic, jc, kc, LXYB) = b / c;
		}
		if (kc >= 3 && kc <= kkcf1 && jc <= jjc1 && ic <= iic1) {  // z-edges: lxza, lxzb
			a = SO(i, j + 1, k, KBSE) + SO(i, j + 1, k, KBS) + SO(i + 1, j + 1, k, KBSW) + SO(i, j, k, KBE) + SO(i, j, k, KB)
			    + SO(i + 1, j, k, KBW) + SO(i, j, k, KBNE) + SO(i, j, k, KBN) + SO(i + 1, j, k, KBNW);
			b = SO(i, j + 1, k - 1, KBNW) + SO(i, j + 1, k - 1, KBN) + SO(i + 1, j + 1, k - 1, KBNE) + SO(i, j, k - 1, KBW)
			    + SO(i, j, k - 1, KB) + SO(i + 1, j, k - 1, KBE) + SO(i, j, k - 1, KBSW) + SO(i, j, k - 1, KBS)
			    + SO(i + 1, j, k - 1, KBSE);
			c = a + b + SO(i, j, k - 1, KPW) + SO(i + 1, j, k - 1, KPW) + SO(i, j + 1, k - 1, KPNW) + SO(i, j + 1, k - 1, KPS)
			    + SO(i + 1, j + 1, k - 1, KPSW) + SO(i, j, k - 1, KPSW) + SO(i, j, k - 1, KPS) + SO(i + 1, j, k - 1, KPNW);
			ep = dmin2(fabs(a / SO(i, j, k - 1, KP)), fabs(b / SO(i, j, k - 1, KP)));
			c = a + b + (SO(i, j, k - 1, KP) - c) * fmax(SO(i, j, k - 1, KP) - (1.0 + ep) * c, 0.0)
			            / (fabs(SO(i, j, k - 1, KP) - (1.0 + ep) * c) + emach);
			CI(ic, jc, kc, LXZA) = a / c;
			CI(ic, jc, kc, LXZB) = b / c;
		}
	} else if (phase == 1) {
		if (kc <= kkc1 && jc >= 3 && jc <= jjcf1 && ic >= 3 && ic <= iicf1) {  // xy faces
			dnw = SO(i - 1, j, k, KPNW) + SO(i - 1, j, k, KBNW) + SO(i - 1, j, k + 1, KBSE);
			dn = SO(i - 1, j, k, KPS) + SO(i - 1, j, k, KBN) + SO(i - 1, j, k + 1, KBS);
			dne = SO(i, j, k, KPSW) + SO(i, j, k, KBNE) + SO(i, j, k + 1, KBSW);
			dw = SO(i - 1, j - 1, k, KPW) + SO(i - 1, j - 1, k, KBW) + SO(i - 1, j - 1, k + 1, KBE);
			de = SO(i, j - 1, k, KPW) + SO(i, j - 1, k, KBE) + SO(i, j - 1, k + 1, KBW);
			dsw = SO(i - 1, j - 1, k, KPSW) + SO(i - 1, j - 1, k, KBSW) + SO(i - 1, j - 1, k + 1, KBNE);
			ds = SO(i - 1, j - 1, k, KPS) + SO(i - 1, j - 1, k, KBS) + SO(i - 1, j - 1, k + 1, KBN);
			dse = SO(i, j - 1, k, KPNW) + SO(i, j - 1, k, KBSE) + SO(i, j - 1, k + 1, KBNW);
			const double o = SO(i - 1, j - 1, k, KP);
			ep = dmin2(dmin2(dmin2(fabs((dsw + dw + dnw) / o), fabs((dnw + dn + dne) / o)), fabs((dne + de + dse) / o)),
			           fabs((dse + ds + dsw) / o));
			dp = dw + dnw + dn + dne + de + dse + ds + dsw;
			sum = o - SO(i - 1, j - 1, k, KB) - SO(i - 1, j - 1, k + 1, KB);
			dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
			dp = 1.0 / dp;
			CI(ic, jc, kc, LXYNW) = dp * (dnw + CI(ic - 1, jc, kc, LXYA) * dw + CI(ic, jc, kc, LXYL) * dn);
			CI(ic, jc, kc, LXYNE) = dp * (dne + CI(ic, jc, kc, LXYR) * dn + CI(ic, jc, kc, LXYA) * de);
			CI(ic, jc, kc, LXYSE) = dp * (dse + CI(ic, jc, kc, LXYB) * de + CI(ic, jc - 1, kc, LXYR) * ds);
			CI(ic, jc, kc, LXYSW) = dp * (dsw + CI(ic, jc - 1, kc, LXYL) * ds + CI(ic - 1, jc, kc, LXYB) * dw);
		}
		if (kc >= 3 && kc <= kkcf1 && jc <= jjc1 && ic >= 3 && ic <= iicf1) {  // xz faces
			dnw = SO(i - 1, j + 1, k, KBSE) + SO(i - 1, j, k, KBE) + SO(i - 1, j, k, KBNE);
			dn = SO(i - 1, j + 1, k, KBS) + SO(i - 1, j, k, KB) + SO(i - 1, j, k, KBN);
			dne = SO(i, j + 1, k, KBSW) + SO(i, j, k, KBW) + SO(i, j, k, KBNW);
			dw = SO(i - 1, j + 1, k - 1, KPNW) + SO(i - 1, j, k - 1, KPW) + SO(i - 1, j, k - 1, KPSW);
			de = SO(i, j + 1, k - 1, KPSW) + SO(i, j, k - 1, KPW) + SO(i, j, k - 1, KPNW);
			dsw = SO(i - 1, j + 1, k - 1, KBNW) + SO(i - 1, j, k - 1, KBW) + SO(i - 1, j, k - 1, KBSW);
			ds = SO(i - 1, j + 1, k - 1, KBN) + SO(i - 1, j, k - 1, KB) + SO(i - 1, j, k - 1, KBS);
			dse = SO(i, j + 1, k - 1, KBNE) + SO(i, j, k - 1, KBE) + SO(i, j, k - 1, KBSE);
			const double o = SO(i - 1, j, k - 1, KP);
			ep = dmin2(dmin2(dmin2(fabs((dsw + dw + dnw) / o), fabs((dnw + dn + dne) / o)), fabs((dne + de + dse) / o)),
			           fabs((dse + ds + dsw) / o));
			dp = dw + dnw + dn + dne + de + dse + ds + dsw;
			sum = o - SO(i - 1, j + 1, k - 1, KPS) - SO(i - 1, j, k - 1, KPS);
			dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
			dp = 1.0 / dp;
			CI(ic, jc, kc, LXZNW) = dp * (dnw + CI(ic - 1, jc, kc, LXZA) * dw + CI(ic, jc, kc, LXYL) * dn);
			CI(ic, jc, kc, LXZNE) = dp * (dne + CI(ic, jc, kc, LXYR) * dn + CI(ic, jc, kc, LXZA) * de);
			CI(ic, jc, kc, LXZSE) = dp * (dse + CI(ic, jc, kc, LXZB) * de + CI(ic, jc, kc - 1, LXYR) * ds);
			CI(ic, jc, kc, LXZSW) = dp * (dsw + CI(ic, jc, kc - 1, LXYL) * ds + CI(ic - 1, jc, kc, LXZB) * dw);
		}
		if (kc >= 3 && kc <= kkcf1 && jc >= 3 && jc <= jjcf1 && ic <= iic1) {  // yz faces
			dnw = SO(i, j, k, KBSE) + SO(i, j, k, KBS) + SO(i + 1, j, k, KBSW);
			dn = SO(i, j - 1, k, KBE) + SO(i, j - 1, k, KB) + SO(i + 1, j - 1, k, KBW);
			dne = SO(i, j - 1, k, KBNE) + SO(i, j - 1, k, KBN) + SO(i + 1, j - 1, k, KBNW);
			dw = SO(i, j, k - 1, KPNW) + SO(i, j, k - 1, KPS) + SO(i + 1, j, k - 1, KPSW);
			de = SO(i, j - 1, k - 1, KPSW) + SO(i, j - 1, k - 1, KPS) + SO(i + 1, j - 1, k - 1, KPNW);
			dsw = SO(i, j, k - 1, KBNW) + SO(i, j, k - 1, KBN) + SO(i + 1, j, k - 1, KBNE);
			ds = SO(i, j - 1, k - 1, KBW) + SO(i, j - 1, k - 1, KB) + SO(i + 1, j - 1, k - 1, KBE);
			dse = SO(i, j - 1, k - 1, KBSW) + SO(i, j - 1, k - 1, KBS) + SO(i + 1, j - 1, k - 1, KBSE);
			const double o = SO(i, j - 1, k - 1, KP);
			ep = dmin2(dmin2(dmin2(fabs((dsw + dw + dnw) / o), fabs((dnw + dn + dne) / o)), fabs((dne + de + dse) / o)),
			           fabs((dse + ds + dsw) / o));
			dp = dw + dnw + dn + dne + de + dse + ds + dsw;
			sum = o - SO(i, j - 1, k - 1, KPW) - SO(i + 1, j - 1, k - 1, KPW);
			dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
			dp = 1.0 / dp;
			CI(ic, jc, kc, LYZNW) = dp * (dnw + CI(ic, jc, kc, LXZA) * dw + CI(ic, jc, kc, LXYA) * dn);
			CI(ic, jc, kc, LYZNE) = dp * (dne + CI(ic, jc, kc, LXYB) * dn + CI(ic, jc - 1, kc, LXZA) * de);
			CI(ic, jc, kc, LYZSE) = dp * (dse + CI(ic, jc - 1, kc, LXZB) * de + CI(ic, jc, kc - 1, LXYB) * ds);
			CI(ic, jc, kc, LYZSW) = dp * (dsw + CI(ic, jc, kc - 1, LXYA) * ds + CI(ic, jc, kc, LXZB) * dw);
		}
	} else {
		if (!(kc >= 3 && kc <= kkcf1 && jc >= 3 && jc <= jjcf1 && ic >= 3 && ic <= iicf1)) return;
		double yp = SO(i - 1, j - 1, k - 1, KPW) + SO(i - 1, j, k - 1, KPNW) + SO(i - 1, j, k - 1, KPS)
		            + SO(i, j, k - 1, KPSW) + SO(i, j - 1, k - 1, KPW) + SO(i, j - 1, k - 1, KPNW)
		            + SO(i - 1, j - 1, k - 1, KPS) + SO(i - 1, j - 1, k - 1, KPSW) + SO(i - 1, j - 1, k - 1, KB)
		            + SO(i - 1, j - 1, k - 1, KBW) + SO(i - 1, j, k - 1, KBNW) + SO(i - 1, j, k - 1, KBN)
		            + SO(i, j, k - 1, KBNE) + SO(i, j - 1, k - 1, KBE) + SO(i, j - 1, k - 1, KBSE)
		            + SO(i - 1, j - 1, k - 1, KBS) + SO(i - 1, j - 1, k - 1, KBSW) + SO(i - 1, j - 1, k, KB)
		            + SO(i - 1, j - 1, k, KBE) + SO(i - 1, j, k, KBSE) + SO(i - 1, j, k, KBS) + SO(i, j, k, KBSW)
		            + SO(i, j - 1, k, KBW) + SO(i, j - 1, k, KBNW) + SO(i - 1, j - 1, k, KBN) + SO(i - 1, j - 1, k, KBNE);
		const double o = SO(i - 1, j - 1, k - 1, KP);
		const double m1 = fabs(SO(i - 1, j - 1, k - 1, KPW) + SO(i - 1, j, k - 1, KPNW) + SO(i - 1, j, k, KBSE)
		                       + SO(i - 1, j - 1, k, KBE) + SO(i - 1, j - 1, k, KBNE) + SO(i - 1, j - 1, k - 1, KPSW)
		                       + SO(i - 1, j - 1, k - 1, KBSW) + SO(i - 1, j - 1, k - 1, KBW) + SO(i - 1, j, k - 1, KBNW))
		                  / o;
		const double m2 = fabs(SO(i, j - 1, k - 1, KPW) + SO(i, j, k - 1, KPSW) + SO(i, j, k, KBSW) + SO(i, j - 1, k, KBW)
		                       + SO(i, j - 1, k, KBNW) + SO(i, j - 1, k - 1, KPNW) + SO(i, j - 1, k - 1, KBSE)
		                       + SO(i, j - 1, k - 1, KBE) + SO(i, j, k - 1, KBNE))
		                  / o;
		const double m3 = fabs(SO(i - 1, j, k - 1, KPS) + SO(i - 1, j, k - 1, KPNW) + SO(i - 1, j, k, KBSE) + SO(i - 1, j, k, KBS)
		                       + SO(i, j, k, KBSW) + SO(i, j, k - 1, KPSW) + SO(i, j, k - 1, KBNE) + SO(i - 1, j, k - 1, KBN)
		                       + SO(i - 1, j, k - 1, KBNW));
		const double m4 = fabs(SO(i - 1, j - 1, k - 1, KPS) + SO(i - 1, j - 1, k - 1, KPSW) + SO(i - 1, j - 1, k, KBNE)
		                       + SO(i - 1, j - 1, k, KBN) + SO(i, j - 1, k, KBNW) + SO(i, j - 1, k - 1, KPNW)
		                       + SO(i, j - 1, k - 1, KBSE) + SO(i - 1, j - 1, k - 1, KBS) + SO(i, j - 1, k - 1, KBSE))
		                  / o;
		double ypw = dmin2(dmin2(dmin2(m1, m2), m3), m4);  // third argument undivided, as the reference
		const double m5 = fabs(SO(i - 1, j - 1, k - 1, KB) + SO(i - 1, j - 1, k - 1, KBW) + SO(i - 1, j, k - 1, KBNW)
		                       + SO(i - 1, j, k - 1, KBN) + SO(i, j, k - 1, KBNE) + SO(i, j - 1, k - 1, KBE)
		                       + SO(i, j - 1, k - 1, KBSE) + SO(i - 1, j - 1, k - 1, KBS) + SO(i - 1, j - 1, k - 1, KBSW));
		const double m6 = fabs(SO(i - 1, j - 1, k, KB) + SO(i - 1, j - 1, k, KBE) + SO(i - 1, j, k, KBSE) + SO(i - 1, j, k, KBS)
		                       + SO(i, j, k, KBSW) + SO(i, j - 1, k, KBW) + SO(i, j - 1, k, KBNW) + SO(i - 1, j - 1, k, KBN)
		                       + SO(i - 1, j - 1, k, KBNE))
		                  / o;
		ypw = dmin2(dmin2(ypw, m5), m6);  // fifth argument undivided, as the reference
		yp = yp + (o - yp) * fmax(o - (1.0 + ypw) * yp, 0.0) / (fabs(o - (1.0 + ypw) * yp) + emach);
		yp = 1.0 / yp;
		CI(ic, jc, kc, LTNW) = yp * (SO(i - 1, j, k, KBSE) + CI(ic - 1, jc, kc, LYZNW) * SO(i - 1, j - 1, k - 1, KPW)
		                             + CI(ic - 1, jc, kc, LXZA) * SO(i - 1, j, k - 1, KPNW) + CI(ic, jc, kc, LXZNW) * SO(i - 1, j, k - 1, KPS)
		                             + CI(ic - 1, jc, kc, LXYA) * SO(i - 1, j - 1, k, KBE) + CI(ic, jc, kc, LXYL) * SO(i - 1, j, k, KBS)
		                             + CI(ic, jc, kc, LXYNW) * SO(i - 1, j - 1, k, KB));
		CI(ic, jc, kc, LTNE) = yp * (SO(i, j, k, KBSW) + CI(ic, jc, kc, LXZNE) * SO(i - 1, j, k - 1, KPS)
		                             + CI(ic, jc, kc, LXZA) * SO(i, j, k - 1, KPSW) + CI(ic, jc, kc, LYZNW) * SO(i, j - 1, k - 1, KPW)
		                             + CI(ic, jc, kc, LXYR) * SO(i - 1, j, k, KBS) + CI(ic, jc, kc, LXYA) * SO(i, j - 1, k, KBW)
		                             + CI(ic, jc, kc, LXYNE) * SO(i - 1, j - 1, k, KB));
		CI(ic, jc, kc, LBNW) = yp * (SO(i - 1, j, k - 1, KBNW) + CI(ic - 1, jc, kc - 1, LXYA) * SO(i - 1, j - 1, k - 1, KBW)
		                             + CI(ic, jc, kc - 1, LXYL) * SO(i - 1, j, k - 1, KBN) + CI(ic, jc, kc - 1, LXYNW) * SO(i - 1, j - 1, k - 1, KB)
		                             + CI(ic - 1, jc, kc, LYZSW) * SO(i - 1, j - 1, k - 1, KPW) + CI(ic - 1, jc, kc, LXZB) * SO(i - 1, j, k - 1, KPNW)
		                             + CI(ic, jc, kc, LXZSW) * SO(i - 1, j, k - 1, KPS));
		CI(ic, jc, kc, LBNE) = yp * (SO(i, j, k - 1, KBNE) + CI(ic, jc, kc - 1, LXYNE) * SO(i - 1, j - 1, k - 1, KB)
		                             + CI(ic, jc, kc - 1, LXYR) * SO(i - 1, j, k - 1, KBN) + CI(ic, jc, kc - 1, LXYA) * SO(i, j - 1, k - 1, KBE)
		                             + CI(ic, jc, kc, LXZSE) * SO(i - 1, j, k - 1, KPS) + CI(ic, jc, kc, LXZB) * SO(i, j, k - 1, KPSW)
		                             + CI(ic, jc, kc, LYZSW) * SO(i, j - 1, k - 1, KPW));
		CI(ic, jc, kc, LBSW) = yp * (SO(i - 1, j - 1, k - 1, KBSW) + CI(ic - 1, jc, kc - 1, LXYB) * SO(i - 1, j - 1, k - 1, KBW)
		                             + CI(ic, jc, kc - 1, LXYSW) * SO(i - 1, j - 1, k - 1, KB) + CI(ic, jc - 1, kc - 1, LXYL) * SO(i - 1, j - 1, k - 1, KBS)
		                             + CI(ic - 1, jc, kc, LYZSE) * SO(i - 1, j - 1, k - 1, KPW) + CI(ic, jc - 1, kc, LXZSW) * SO(i - 1, j - 1, k - 1, KPS)
		                             + CI(ic - 1, jc - 1, kc, LXZB) * SO(i - 1, j - 1, k - 1, KPSW));
		CI(ic, jc, kc, LTSW) = yp * (SO(i - 1, j - 1, k, KBNE) + CI(ic - 1, jc, kc, LXYB) * SO(i - 1, j - 1, k, KBE)
		                             + CI(ic, jc, kc, LXYSW) * SO(i - 1, j - 1, k, KB) + CI(ic, jc - 1, kc, LXYL) * SO(i - 1, j - 1, k, KBN)
		                             + CI(ic - 1, jc, kc, LYZNE) * SO(i - 1, j - 1, k - 1, KPW) + CI(ic, jc - 1, kc, LXZNW) * SO(i - 1, j - 1, k - 1, KPS)
		                             + CI(ic - 1, jc - 1, kc, LXZA) * SO(i - 1, j - 1, k - 1, KPSW));
		CI(ic, jc, kc, LTSE) = yp * (SO(i, j - 1, k, KBNW) + CI(ic, jc - 1, kc, LXYR) * SO(i - 1, j - 1, k, KBN)
		                             + CI(ic, jc, kc, LXYSE) * SO(i - 1, j - 1, k, KB) + CI(ic, jc, kc, LXYB) * SO(i, j - 1, k, KBW)
		                             + CI(ic, jc - 1, kc, LXZNE) * SO(i - 1, j - 1, k - 1, KPS) + CI(ic, jc, kc, LYZNE) * SO(i, j - 1, k - 1, KPW)
		                             + CI(ic, jc - 1, kc, LXZA) * SO(i, j - 1, k - 1, KPNW));
		CI(ic, jc, kc, LBSE) = yp * (SO(i, j - 1, k - 1, KBSE) + CI(ic, jc - 1, kc - 1, LXYR) * SO(i - 1, j - 1, k - 1, KBS)
		                             + CI(ic, jc, kc - 1, LXYSE) * SO(i - 1, j - 1, k - 1, KB) + CI(ic, jc, kc - 1, LXYB) * SO(i, j - 1, k - 1, KBE)
		                             + CI(ic, jc - 1, kc, LXZSE) * SO(i - 1, j - 1, k - 1, KPS) + CI(ic, jc, kc, LYZSE) * SO(i, j - 1, k - 1, KPW)
		                             + CI(ic, jc - 1, kc, LXZB) * SO(i, j - 1, k - 1, KPNW));
	}
}

// The seven-point branch of BMG3_SymStd_SETUP_interp_OI
// (BMG3_SymStd_SETUP_interp_OI.f90:543-807), same three phases.  Kept from the
// reference: the x-edge ep divides |b| (not b) by so(kp), and the interior
// correction is added after the product ((o - dp) * ... + dp).
__global__ void __launch_bounds__(TX *TY) k3_oi7(const double *__restrict__ so, double *__restrict__ ci, Dims3 F,
                                                 Dims3 C, int phase)
{
	const int ic = blockIdx.x * TX + threadIdx.x + 2, jc = blockIdx.y * TY + threadIdx.y + 2, kc = blockIdx.z + 2;
	const int iic1 = C.nx + 1, jjc1 = C.ny + 1, kkc1 = C.nz + 1;
	const int iicf1 = F.nx / 2 + 2, jjcf1 = F.ny / 2 + 2, kkcf1 = F.nz / 2 + 2;
	const double emach = 1.1102230246251565e-16;
	const int i = 2 * ic - 2, j = 2 * jc - 2, k = 2 * kc - 2;
	double a, b, c, ep, dn, dw, de, ds, dp, sum, o;
	if (phase == 0) {
		if (kc <= kkc1 && jc <= jjc1 && ic >= 3 && ic <= iicf1) {  // x-edges: lxyl, lxyr
			a = SO(i - 1, j, k, KPW);
			b = SO(i, j, k, KPW);
			ep = dmin2(fabs(a / SO(i - 1, j, k, KP)), fabs(b) / SO(i - 1, j, k, KP));
			c = a + b + SO(i - 1, j, k, KPS) + SO(i - 1, j + 1, k, KPS) + SO(i - 1, j, k, KB) + SO(i - 1, j, k + 1, KB);
			c = a + b + (SO(i - 1, j, k, KP) - c) * fmax(SO(i - 1, j, k, KP) - (1.0 + ep) * c, 0.0)
			            / (fabs(SO(i - 1, j, k, KP) - (1.0 + ep) * c) + emach);
			CI(ic, jc, kc, LXYL) = a / c;
			CI(ic, jc, kc, LXYR) = b / c;
		}
		if (kc <= kkc1 && jc >= 3 && jc <= jjcf1 && ic <= iic1) {  // y-edges: lxya, lxyb
			a = SO(i, j, k, KPS);
			b = SO(i, j - 1, k, KPS);
			c = a + b + SO(i, j - 1, k, KPW) + SO(i + 1, j - 1, k, KPW) + SO(i, j - 1, k, KB) + SO(i, j - 1, k + 1, KB);
			ep = dmin2(fabs(a / SO(i, j - 1, k, KP)), fabs(b / SO(i, j - 1, k, KP)));
			c = a + b + (SO(i, j - 1, k, KP) - c) * fmax(SO(i, j - 1, k, KP) - (1.0 + ep) * c, 0.0)
			            / (fabs(SO(i, j - 1, k, KP) - (1.0 + ep) * c) + emach);
			CI(ic, jc, kc, LXYA) = a / c;
			CI(ic, jc, kc, LXYB) = b / c;
		}
		if (kc >= 3 && kc <= kkcf1 && jc <= jjc1 && ic <= iic1) {  // z-edges: lxza, lxzb
			a = SO(i, j, k, KB);
			b = SO(i, j, k - 1, KB);
			c = a + b + SO(i, j, k - 1, KPW) + SO(i + 1, j, k - 1, KPW) + SO(i, j + 1, k - 1, KPS) + SO(i, j, k - 1, KPS);
			ep = dmin2(fabs(a / SO(i, j, k - 1, KP)), fabs(b / SO(i, j, k - 1, KP)));
			c = a + b + (SO(i, j, k - 1, KP) - c) * fmax(SO(i, j, k - 1, KP) - (1.0 + ep) * c, 0.0)
			            / (fabs(SO(i, j, k - 1, KP) - (1.0 + ep) * c) + emach);
			CI(ic, jc, kc, LXZA) = a / c;
			CI(ic, jc, kc, LXZB) = b / c;
		}
	} else if (phase == 1) {
		if (ic >= 3 && ic <= iicf1 && jc >= 3 && jc <= jjcf1 && kc <= kkc1) {  // xy faces
			o = SO(i - 1, j - 1, k, KP);
			dn = SO(i - 1, j, k, KPS);
			dw = SO(i - 1, j - 1, k, KPW);
			de = SO(i, j - 1, k, KPW);
			ds = SO(i - 1, j - 1, k, KPS);
			dp = dw + dn + de + ds;
			sum = o - SO(i - 1, j - 1, k, KB) - SO(i - 1, j - 1, k + 1, KB);
			ep = dmin2(dmin2(dmin2(fabs(dw / o), fabs(dn / o)), fabs(de / o)), fabs(ds / o));
			dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
			dp = 1.0 / dp;
			CI(ic, jc, kc, LXYNW) = dp * (CI(ic - 1, jc, kc, LXYA) * dw + CI(ic, jc, kc, LXYL) * dn);
			CI(ic, jc, kc, LXYNE) = dp * (CI(ic, jc, kc, LXYR) * dn + CI(ic, jc, kc, LXYA) * de);
			CI(ic, jc, kc, LXYSE) = dp * (CI(ic, jc, kc, LXYB) * de + CI(ic, jc - 1, kc, LXYR) * ds);
			CI(ic, jc, kc, LXYSW) = dp * (CI(ic, jc - 1, kc, LXYL) * ds + CI(ic - 1, jc, kc, LXYB) * dw);
		}
		if (kc >= 3 && kc <= kkcf1 && jc <= jjc1 && ic >= 3 && ic <= iicf1) {  // xz faces
			o = SO(i - 1, j, k - 1, KP);
			dn = SO(i - 1, j, k, KB);
			dw = SO(i - 1, j, k - 1, KPW);
			de = SO(i, j, k - 1, KPW);
			ds = SO(i - 1, j, k - 1, KB);
			dp = dw + dn + de + ds;
			sum = o - SO(i - 1, j + 1, k - 1, KPS) - SO(i - 1, j, k - 1, KPS);
			ep = dmin2(dmin2(dmin2(fabs(dw / o), fabs(dn / o)), fabs(de / o)), fabs(ds / o));
			dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
			dp = 1.0 / dp;
			CI(ic, jc, kc, LXZNW) = dp * (CI(ic - 1, jc, kc, LXZA) * dw + CI(ic, jc, kc, LXYL) * dn);
			CI(ic, jc, kc, LXZNE) = dp * (CI(ic, jc, kc, LXYR) * dn + CI(ic, jc, kc, LXZA) * de);
			CI(ic, jc, kc, LXZSE) = dp * (CI(ic, jc, kc, LXZB) * de + CI(ic, jc, kc - 1, LXYR) * ds);
			CI(ic, jc, kc, LXZSW) = dp * (CI(ic, jc, kc - 1, LXYL) * ds + CI(ic - 1, jc, kc, LXZB) * dw);
		}
		if (kc >= 3 && kc <= kkcf1 && jc >= 3 && jc <= jjcf1 && ic <= iic1) {  // yz faces
			o = SO(i, j - 1, k - 1, KP);
			dn = SO(i, j - 1, k, KB);
			dw = SO(i, j, k - 1, KPS);
			de = SO(i, j - 1, k - 1, KPS);
			ds = SO(i, j - 1, k - 1, KB);
			dp = dw + dn + de + ds;
			sum = o - SO(i, j - 1, k - 1, KPW) - SO(i + 1, j - 1, k - 1, KPW);
			ep = dmin2(dmin2(dmin2(fabs(dw / o), fabs(dn / o)), fabs(de / o)), fabs(ds / o));
			dp = dp + (sum - dp) * fmax(sum - (1.0 + ep) * dp, 0.0) / (fabs(sum - (1.0 + ep) * dp) + emach);
			dp = 1.0 / dp;
			CI(ic, jc, kc, LYZNW) = dp * (CI(ic, jc, kc, LXZA) * dw + CI(ic, jc, kc, LXYA) * dn);
			CI(ic, jc, kc, LYZNE) = dp * (CI(ic, jc, kc, LXYB) * dn + CI(ic, jc - 1, kc, LXZA) * de);
			CI(ic, jc, kc, LYZSE) = dp * (CI(ic, jc - 1, kc, LXZB) * de + CI(ic, jc, kc - 1, LXYB) * ds);
			CI(ic, jc, kc, LYZSW) = dp * (CI(ic, jc, kc - 1, LXYA) * ds + CI(ic, jc, kc, LXZB) * dw);
		}
	} else if (kc >= 3 && kc <= kkcf1 && jc >= 3 && jc <= jjcf1 && ic >= 3 && ic <= iicf1) {  // interior points
		o = SO(i - 1, j - 1, k - 1, KP);
		const double sw = SO(i - 1, j - 1, k - 1, KPW), sn = SO(i - 1, j, k - 1, KPS), se = SO(i, j - 1, k - 1, KPW);
		const double ss = SO(i - 1, j - 1, k - 1, KPS), sb = SO(i - 1, j - 1, k - 1, KB), st = SO(i - 1, j - 1, k, KB);
		dp = sw + sn + se + ss + sb + st;
		ep = dmin2(dmin2(dmin2(dmin2(dmin2(fabs(sw / o), fabs(sn / o)), fabs(se / o)), fabs(ss / o)), fabs(sb / o)),
		           fabs(st / o));
		dp = (o - dp) * fmax(o - (1.0 + ep) * dp, 0.0) / (fabs(o - (1.0 + ep) * dp) + emach) + dp;
		dp = 1.0 / dp;
		CI(ic, jc, kc, LTNW) = dp * (CI(ic - 1, jc, kc, LYZNW) * sw + CI(ic, jc, kc, LXZNW) * sn + CI(ic, jc, kc, LXYNW) * st);
		CI(ic, jc, kc, LTNE) = dp * (CI(ic, jc, kc, LXZNE) * sn + CI(ic, jc, kc, LYZNW) * se + CI(ic, jc, kc, LXYNE) * st);
		CI(ic, jc, kc, LBNW) =
		    dp * (CI(ic, jc, kc - 1, LXYNW) * sb + CI(ic - 1, jc, kc, LYZSW) * sw + CI(ic, jc, kc, LXZSW) * sn);
		CI(ic, jc, kc, LBNE) = dp * (CI(ic, jc, kc - 1, LXYNE) * sb + CI(ic, jc, kc, LXZSE) * sn + CI(ic, jc, kc, LYZSW) * se);
		CI(ic, jc, kc, LBSW) =
		    dp * (CI(ic, jc, kc - 1, LXYSW) * sb + CI(ic - 1, jc, kc, LYZSE) * sw + CI(ic, jc - 1, kc, LXZSW) * ss);
		CI(ic, jc, kc, LTSW) =
		    dp * (CI(ic, jc, kc, LXYSW) * st + CI(ic - 1, jc, kc, LYZNE) * sw + CI(ic, jc - 1, kc, LXZNW) * ss);
		CI(ic, jc, kc, LTSE) = dp * (CI(ic, jc, kc, LXYSE) * st + CI(ic, jc - 1, kc, LXZNE) * ss + CI(ic, jc, kc, LYZNE) * se);
		CI(ic, jc, kc, LBSE) =
		    dp * (CI(ic, jc, kc - 1, LXYSE) * sb + CI(ic, jc - 1, kc, LXZSE) * ss + CI(ic, jc, kc, LYZSE) * se);
	}
}

int setup_interp_3d(const double *so, double *ci, Dims3 F, Dims3 C, cudaStream_t st, int ns)
{
	CDR_CUDA_TRY(cudaMemsetAsync(ci, 0, sizeof(double) * C.plane() * 26, st));
	const dim3 grd(ceil_div(F.nx / 2 + 1, TX), ceil_div(F.ny / 2 + 1, TY), F.nz / 2 + 1);
	for (int ph = 0; ph < 3; ++ph) {
		if (ns == 4) k3_oi7<<<grd, dim3(TX, TY), 0, st>>>(so, ci, F, C, ph);
		else k3_oi<<<grd, dim3(TX, TY), 0, st>>>(so, ci, F, C, ph);
		CDR_LAUNCH_CHECK();
	}
	return CDR_OK;
}

// ------------------------------------------------------------- Galerkin (P^T A P)
// Same loops, order and skips as the CPU restatement of the product that
// BMG3_SymStd_SETUP_ITLI27_ex expands (cdr3 oracle).
// A seven-point operator (NS == 4) has no planes beyond kb: those couplings
// read as 0, as the zero-filled planes of a 14-plane copy would.
template <int NS>
__device__ __forceinline__ double a3(const double *__restrict__ so, Dims3 F, int i, int j, int k, int di, int dj, int dk)
{
	auto S = [&](int ii, int jj, int kk, int p) -> double { return (NS == 4 && p > KB) ? 0.0 : SO(ii, jj, kk, p); };
	if (di == 0 && dj == 0 && dk == 0) return SO(i, j, k, KP);
	double c = 0.0;
	switch ((dk + 1) * 9 + (dj + 1) * 3 + (di + 1)) {
	case 9 + 3 + 0: c = S(i, j, k, KPW); break;
	case 9 + 6 + 0: c = S(i, j + 1, k, KPNW); break;
	case 9 + 6 + 1: c = S(i, j + 1, k, KPS); break;
	case 9 + 6 + 2: c = S(i + 1, j + 1, k, KPSW); break;
	case 9 + 3 + 2: c = S(i + 1, j, k, KPW); break;
	case 9 + 0 + 2: c = S(i + 1, j, k, KPNW); break;
	case 9 + 0 + 1: c = S(i, j, k, KPS); break;
	case 9 + 0 + 0: c = S(i, j, k, KPSW); break;
	case 0 + 3 + 1: c = S(i, j, k, KB); break;
	case 0 + 3 + 0: c = S(i, j, k, KBW); break;
	case 0 + 6 + 0: c = S(i, j + 1, k, KBNW); break;
	case 0 + 6 + 1: c = S(i, j + 1, k, KBN); break;
	case 0 + 6 + 2: c = S(i + 1, j + 1, k, KBNE); break;
	case 0 + 3 + 2: c = S(i + 1, j, k, KBE); break;
	case 0 + 0 + 2: c = S(i + 1, j, k, KBSE); break;
	case 0 + 0 + 1: c = S(i, j, k, KBS); break;
	case 0 + 0 + 0: c = S(i, j, k, KBSW); break;
	case 18 + 3 + 1: c = S(i, j, k + 1, KB); break;
	case 18 + 3 + 0: c = S(i, j, k + 1, KBE); break;
	case 18 + 6 + 0: c = S(i, j + 1, k + 1, KBSE); break;
	case 18 + 6 + 1: c = S(i, j + 1, k + 1, KBS); break;
	case 18 + 6 + 2: c = S(i + 1, j + 1, k + 1, KBSW); break;
	case 18 + 3 + 2: c = S(i + 1, j, k + 1, KBW); break;
	case 18 + 0 + 2: c = S(i + 1, j, k + 1, KBNW); break;
	case 18 + 0 + 1: c = S(i, j, k + 1, KBN); break;
	case 18 + 0 + 0: c = S(i, j, k + 1, KBNE); break;
	}
	return -c;
}

__device__ __forceinline__ double p3(const double *__restrict__ ci, Dims3 C, int ic, int jc, int kc, int dx, int dy, int dz)
{
	if (dz == 0) {
		if (dx == 0 && dy == 0) return 1.0;
		if (dy == 0) return dx < 0 ? CI(ic, jc, kc, LXYR) : CI(ic + 1, jc, kc, LXYL);
		if (dx == 0) return dy < 0 ? CI(ic, jc, kc, LXYA) : CI(ic, jc + 1, kc, LXYB);
		if (dy < 0) return dx < 0 ? CI(ic, jc, kc, LXYNE) : CI(ic + 1, jc, kc, LXYNW);
		return dx < 0 ? CI(ic, jc + 1, kc, LXYSE) : CI(ic + 1, jc + 1, kc, LXYSW);
	}
	const int ko = dz < 0 ? 0 : 1;
	if (dx == 0 && dy == 0) return dz < 0 ? CI(ic, jc, kc, LXZA) : CI(ic, jc, kc + 1, LXZB);
	if (dx == 0) {
		if (dy < 0) return dz < 0 ? CI(ic, jc, kc, LYZNW) : CI(ic, jc, kc + 1, LYZSW);
		return dz < 0 ? CI(ic, jc + 1, kc, LYZNE) : CI(ic, jc + 1, kc + 1, LYZSE);
	}
	if (dy == 0) {
		if (dx < 0) return dz < 0 ? CI(ic, jc, kc, LXZNE) : CI(ic, jc, kc + 1, LXZSE);
		return dz < 0 ? CI(ic + 1, jc, kc, LXZNW) : CI(ic + 1, jc, kc + 1, LXZSW);
	}
	const int io = dx < 0 ? 0 : 1, jo = dy < 0 ? 0 : 1;
	int l;
	if (dz < 0) l = dy < 0 ? (dx < 0 ? LTNE : LTNW) : (dx < 0 ? LTSE : LTSW);
	else l = dy < 0 ? (dx < 0 ? LBNE : LBNW) : (dx < 0 ? LBSE : LBSW);
	return CI(ic + io, jc + jo, kc + ko, l);
}

template <int NS>
__device__ double rap3(const double *__restrict__ so, const double *__restrict__ ci, Dims3 F, Dims3 C, int i1, int j1,
                       int k1, int i2, int j2, int k2)
{
	const int F1x = 2 * i1 - 2, F1y = 2 * j1 - 2, F1z = 2 * k1 - 2;
	double tot = 0.0;
#pragma unroll 1
	for (int dz1 = -1; dz1 <= 1; ++dz1)
#pragma unroll 1
		for (int dy1 = -1; dy1 <= 1; ++dy1)
			for (int dx1 = -1; dx1 <= 1; ++dx1) {
				const int fx = F1x + dx1, fy = F1y + dy1, fz = F1z + dz1;
				if (fx < 2 || fx > F.nx + 1 || fy < 2 || fy > F.ny + 1 || fz < 2 || fz > F.nz + 1) continue;
				double inner = 0.0;
				for (int ddz = -1; ddz <= 1; ++ddz)
					for (int ddy = -1; ddy <= 1; ++ddy)
						for (int ddx = -1; ddx <= 1; ++ddx) {
							const int ex = dx1 + ddx - 2 * (i2 - i1), ey = dy1 + ddy - 2 * (j2 - j1), ez = dz1 + ddz - 2 * (k2 - k1);
							if (ex < -1 || ex > 1 || ey < -1 || ey > 1 || ez < -1 || ez > 1) continue;
							inner += a3<NS>(so, F, fx, fy, fz, ddx, ddy, ddz) * p3(ci, C, i2, j2, k2, ex, ey, ez);
						}
				tot += p3(ci, C, i1, j1, k1, dx1, dy1, dz1) * inner;
			}
	return tot;
}

// One thread per (coarse point, stencil plane): the 14 entries are independent.
template <int NS>
__global__ void __launch_bounds__(TX *TY) k3_galerkin(const double *__restrict__ so, const double *__restrict__ ci,
                                                      double *__restrict__ soc, Dims3 F, Dims3 C)
{
	const int ic = blockIdx.x * TX + threadIdx.x + 2, jc = blockIdx.y * TY + threadIdx.y + 2;
	const int kc = blockIdx.z / 14 + 2, pl = blockIdx.z % 14 + 1;
	if (ic > C.nx + 1 || jc > C.ny + 1) return;
	// (fine-side coarse point, partner coarse point) offsets of each plane, and
	// the sign: KP = R(c,c); the others -R(c1, c2) (BMG3_SymStd_SETUP_ITLI27_ex)
	int a1 = 0, b1 = 0, c1 = 0, a2 = 0, b2 = 0, c2 = 0;
	switch (pl) {
	case KP: break;
	case KPW: a2 = -1; break;
	case KPS: b2 = -1; break;
	case KB: c2 = -1; break;
	case KPSW: a2 = -1; b2 = -1; break;
	case KPNW: b1 = -1; a2 = -1; break;
	case KBW: a2 = -1; c2 = -1; break;
	case KBNW: b1 = -1; a2 = -1; c2 = -1; break;
	case KBN: b1 = -1; c2 = -1; break;
	case KBNE: a1 = -1; b1 = -1; c2 = -1; break;
	case KBE: a1 = -1; c2 = -1; break;
	case KBSE: a1 = -1; b2 = -1; c2 = -1; break;
	case KBS: b2 = -1; c2 = -1; break;
	case KBSW: a2 = -1; b2 = -1; c2 = -1; break;
	}
	const double v = rap3<NS>(so, ci, F, C, ic + a1, jc + b1, kc + c1, ic + a2, jc + b2, kc + c2);
	soc[(size_t)(pl - 1) * C.plane() + C.at1(ic, jc, kc)] = pl == KP ? v : -v;
}

int galerkin_3d(const double *so, const double *ci, double *soc, Dims3 F, Dims3 C, cudaStream_t st, int ns)
{
	CDR_CUDA_TRY(cudaMemsetAsync(soc, 0, sizeof(double) * C.plane() * 14, st));
	const dim3 grd(ceil_div(C.nx, TX), ceil_div(C.ny, TY), C.nz * 14);
	if (ns == 4) k3_galerkin<4><<<grd, dim3(TX, TY), 0, st>>>(so, ci, soc, F, C);
	else k3_galerkin<14><<<grd, dim3(TX, TY), 0, st>>>(so, ci, soc, F, C);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

// ---------------------------------------------------------- coarsest Cholesky
// ABD fill of BMG3_SymStd_SETUP_cg_LU (src/3d/ftn/BMG3_SymStd_SETUP_cg_LU.f90:106-130),
// KD = IBW = (II-2)*(JJ-1)+1, then DPBTF2('U') as in 2D.
// NS == 4: a seven-point operator (a one-level hierarchy); the couplings it
// lacks enter the band as -0.0, as from zero-filled planes.
template <int NS>
__global__ void k3_cg_factor(const double *__restrict__ so, Dims3 F, double *__restrict__ abd, int nabd1, int *info)
{
	auto S = [&](int ii, int jj, int kk, int p) -> double { return (NS == 4 && p > KB) ? 0.0 : SO(ii, jj, kk, p); };
	if (threadIdx.x != 0 || blockIdx.x != 0) return;
	const int II = F.nx + 2, JJ = F.ny + 2, KK = F.nz + 2;
	const int i1 = II - 1, j1 = JJ - 1, k1 = KK - 1, i2 = i1 - 1;
	const int ibw = i2 * j1 + 1;
	const int n = F.nx * F.ny * F.nz;
	for (size_t e = 0; e < (size_t)nabd1 * n; ++e) abd[e] = 0.0;
#define ABD(r, c) abd[(size_t)((c)-1) * nabd1 + ((r)-1)]
	int kl = 0;
	for (int k = 2; k <= k1; ++k)
		for (int j = 2; j <= j1; ++j)
			for (int i = 2; i <= i1; ++i) {
				kl++;
				ABD(ibw + 1, kl) = S(i, j, k, KP);
				ABD(ibw, kl) = -S(i, j, k, KPW);
				ABD(ibw - i1 + 3, kl) = -S(i + 1, j, k, KPNW);
				ABD(ibw - i1 + 2, kl) = -S(i, j, k, KPS);
				ABD(ibw - i1 + 1, kl) = -S(i, j, k, KPSW);
				ABD(ibw - (j1 - 2) * i2 + 2, kl) = -S(i + 1, j + 1, k, KBNE);
				ABD(ibw - (j1 - 2) * i2 + 1, kl) = -S(i, j + 1, k, KBN);
				ABD(ibw - (j1 - 2) * i2, kl) = -S(i, j + 1, k, KBNW);
				ABD(ibw - (j1 - 1) * i2 + 2, kl) = -S(i + 1, j, k, KBE);
				ABD(ibw - (j1 - 1) * i2 + 1, kl) = -S(i, j, k, KB);
				ABD(ibw - (j1 - 1) * i2, kl) = -S(i, j, k, KBW);
				ABD(3, kl) = -S(i + 1, j, k, KBSE);
				ABD(2, kl) = -S(i, j, k, KBS);
				ABD(1, kl) = -S(i, j, k, KBSW);
			}
#undef ABD
	// DPBTF2('U', n, kd = ibw)
	const int kd = ibw, ldab = nabd1, kld = ldab - 1;
	int stt = 0;
	for (int jj = 0; jj < n; ++jj) {
		double ajj = abd[(size_t)jj * ldab + kd];
		if (ajj <= 0.0) { stt = jj + 1; break; }
		ajj = sqrt(ajj);
		abd[(size_t)jj * ldab + kd] = ajj;
		const int kn = kd < n - jj - 1 ? kd : n - jj - 1;
		if (kn > 0) {
			const double rcp = 1.0 / ajj;
			double *xv = abd + (size_t)(jj + 1) * ldab + (kd - 1);
			for (int p = 0; p < kn; ++p) xv[(size_t)p * kld] = rcp * xv[(size_t)p * kld];
			double *a = abd + (size_t)(jj + 1) * ldab + kd;
			for (int qq = 0; qq < kn; ++qq) {
				const double xq = xv[(size_t)qq * kld];
				if (xq != 0.0) {
					const double temp = -1.0 * xq;
					for (int p = 0; p <= qq; ++p)
						a[(size_t)p + (size_t)qq * kld] = a[(size_t)p + (size_t)qq * kld] + xv[(size_t)p * kld] * temp;
				}
			}
		}
	}
	if (info) *info = stt;
}

// BMG3_SymStd_SOLVE_cg (src/3d/ftn/BMG3_SymStd_SOLVE_cg.f90:105-131) with DPBTRS('U')
template <typename T>
__global__ void k3_cg_solve(const double *__restrict__ ab, int ldab, T *__restrict__ q, const T *__restrict__ qf, Dims3 F)
{
	extern __shared__ double xs[];
	if (threadIdx.x != 0 || blockIdx.x != 0) return;
	const int kd = F.nx * (F.ny + 1) + 1, n = F.nx * F.ny * F.nz;
	int kk = 0;
	for (int k = 2; k <= F.nz + 1; ++k)
		for (int j = 2; j <= F.ny + 1; ++j)
			for (int i = 2; i <= F.nx + 1; ++i) xs[kk++] = (double)QF(i, j, k);
	for (int j = 0; j < n; ++j) {
		double temp = xs[j];
		const int i0 = j - kd > 0 ? j - kd : 0;
		for (int i = i0; i < j; ++i) temp = temp - ab[(size_t)j * ldab + kd + i - j] * xs[i];
		xs[j] = temp / ab[(size_t)j * ldab + kd];
	}
	for (int j = n - 1; j >= 0; --j) {
		if (xs[j] != 0.0) {
			xs[j] = xs[j] / ab[(size_t)j * ldab + kd];
			const double temp = xs[j];
			const int i1 = j - kd > 0 ? j - kd : 0;
			for (int i = j - 1; i >= i1; --i) xs[i] = xs[i] - temp * ab[(size_t)j * ldab + kd + i - j];
		}
	}
	kk = 0;
	for (int k = 2; k <= F.nz + 1; ++k)
		for (int j = 2; j <= F.ny + 1; ++j)
			for (int i = 2; i <= F.nx + 1; ++i) Q(i, j, k) = (T)xs[kk++];
}

int setup_cg_3d(const double *so, Dims3 F, double *abd, int *info, cudaStream_t st, int ns)
{
	if (ns == 4) k3_cg_factor<4><<<1, 32, 0, st>>>(so, F, abd, F.nx * (F.ny + 1) + 2, info);
	else k3_cg_factor<14><<<1, 32, 0, st>>>(so, F, abd, F.nx * (F.ny + 1) + 2, info);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

template <typename T>
int solve_cg_3d(const double *abd, T *x, const T *b, Dims3 F, cudaStream_t st)
{
	const size_t sm = sizeof(double) * (size_t)F.nx * F.ny * F.nz;
	if (sm > 48 * 1024) {
		set_error(CDR_ERR_DIM, "coarsest grid %dx%dx%d too large for the direct solve", F.nx, F.ny, F.nz);
		return CDR_ERR_DIM;
	}
	k3_cg_solve<T><<<1, 32, sm, st>>>(abd, F.nx * (F.ny + 1) + 2, x, b, F);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}
template int solve_cg_3d<double>(const double *, double *, const double *, Dims3, cudaStream_t);
template int solve_cg_3d<float>(const double *, float *, const float *, Dims3, cudaStream_t);

// Outer refinement step of the mixed-precision 3D solve (as the 2D one):
//   x_out = x_in + e32, r64 = b - A x_out, r32 = (float) r64, ||r64||^2 per
//   block.  Each thread forms x_in + e32 over its 27-point neighbourhood on the
//   fly; x_in and x_out are different buffers.  apply = 0 skips e.
struct LoadIR3 {
	const double *__restrict__ x;
	const float *__restrict__ e;
	Dims3 F, E;
	int apply;
	__device__ __forceinline__ double operator()(int i, int j, int k) const
	{
		const double v = x[F.at1(i, j, k)];
		return apply ? v + (double)e[E.at1(i, j, k)] : v;
	}
};

template <int NS>
__global__ void __launch_bounds__(TX *TY) k3_ir_residual(const double *__restrict__ so, const double *__restrict__ x,
                                                         const float *__restrict__ e, const double *__restrict__ b,
                                                         double *__restrict__ xo, float *__restrict__ r32, Dims3 F,
                                                         Dims3 E, double *__restrict__ partial, int apply)
{
	__shared__ double sh[TX * TY / 32];
	const int tx = (F.nx + TX - 1) / TX, ty = (F.ny + TY - 1) / TY;
	const long ntiles = (long)tx * ty * F.nz;
	const LoadIR3 xq{x, e, F, E, apply};
	double acc = 0.0;
	for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
		const int kk = (int)(t / ((long)tx * ty));
		const int rem = (int)(t - (long)kk * tx * ty);
		const int i = (rem % tx) * TX + threadIdx.x + 2, j = (rem / tx) * TY + threadIdx.y + 2, k = kk + 2;
		if (i <= F.nx + 1 && j <= F.ny + 1) {
			const double xc = xq(i, j, k);
			const double r = nbs<NS, double>(so, xq, b[F.at1(i, j, k)], F, i, j, k) - SO(i, j, k, KP) * xc;
			acc += r * r;
			r32[E.at1(i, j, k)] = (float)r;
			xo[F.at1(i, j, k)] = xc;
		}
	}
	const double s = block_sum<TX * TY / 32>(acc, sh);
	if (threadIdx.x == 0 && threadIdx.y == 0) partial[blockIdx.x] = s;
}

int ir_residual_3d(const double *so, const double *x, const float *e, const double *b, double *xo, float *r32,
                   Dims3 d, Dims3 d32, double *norm_out, double *partial, int apply, cudaStream_t st, int ns)
{
	const long ntiles = (long)ceil_div(d.nx, TX) * ceil_div(d.ny, TY) * d.nz;
	const int nb = ntiles < 2048 ? (int)ntiles : 2048;
	if (ns == 4) k3_ir_residual<4><<<nb, dim3(TX, TY), 0, st>>>(so, x, e, b, xo, r32, d, d32, partial, apply);
	else k3_ir_residual<14><<<nb, dim3(TX, TY), 0, st>>>(so, x, e, b, xo, r32, d, d32, partial, apply);
	CDR_LAUNCH_CHECK();
	k3_norm_finish<<<1, 1024, 0, st>>>(partial, nb, norm_out);
	CDR_LAUNCH_CHECK();
	return CDR_OK;
}

#undef SO
#undef Q
#undef QF
#undef CI
#undef QC

}  // namespace cdrgpu
