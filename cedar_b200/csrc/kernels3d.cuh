// kernels3d.cuh -- host-side launchers of the 3D kernels (internal C++ API).
//
// Device layout of a 3D level (Cedar's, include/cedar/3d/stencil_op.h): one
// ghost layer, i fastest, rows padded to a pitch; a k-slice is pitch*(ny+2)
// elements, a stencil plane pitch*(ny+2)*(nz+2).  14 stencil planes (27-point
// operators) or 4 (a seven-point fine operator: p, pw, ps, b), 26 interpolation
// planes on the coarse grid.  Launchers taking ns accept either.
#pragma once
#include "cdr_common.cuh"

namespace cdrgpu {

// stencil planes p pw ps b psw pnw bw bnw bn bne be bse bs bsw (1-based, as the
// reference's kp .. kbsw, src/3d/ftn/BMG_stencils_f90.h:46-48) and the 26
// interpolation planes lxyl .. ltse
enum : int { KP = 1, KPW, KPS, KB, KPSW, KPNW, KBW, KBNW, KBN, KBNE, KBE, KBSE, KBS, KBSW };
enum : int { LXYL = 1, LXYR, LXYA, LXYB, LXZA, LXZB, LXYNE, LXYSE, LXYSW, LXYNW, LXZSW, LXZNW, LXZNE, LXZSE,
             LYZSW, LYZNW, LYZNE, LYZSE, LBSW, LBNW, LBNE, LBSE, LTSW, LTNW, LTNE, LTSE };

struct Dims3 {
	int nx, ny, nz, pitch;
	__host__ __device__ size_t slice() const { return (size_t)pitch * (ny + 2); }
	__host__ __device__ size_t plane() const { return slice() * (nz + 2); }
	// the reference's 1-based index (I, J, K) -> offset
	__host__ __device__ size_t at1(int i, int j, int k) const
	{
		return ((size_t)(k - 1) * (ny + 2) + (j - 1)) * pitch + (i - 1);
	}
};

template <typename T>
int residual_3d(const T *so, const T *x, const T *b, T *r, Dims3 d, double *norm_out, double *partial, cudaStream_t st,
                int ns = 14);
template <typename T>
int setup_recip_3d(const T *so, T *sor, Dims3 d, cudaStream_t st);
template <typename T>
int relax_point_3d(const T *so, T *x, const T *b, const T *sor, Dims3 d, int updown, cudaStream_t st, int ns = 14);
template <typename T>
int restrict_3d(const T *ci, const T *rf, T *bc, Dims3 f, Dims3 c, cudaStream_t st);
template <typename T>
int interp_add_3d(const T *ci, const T *xc, const T *rf, const T *sof, T *xf, Dims3 f, Dims3 c, cudaStream_t st);
int setup_interp_3d(const double *so, double *ci, Dims3 f, Dims3 c, cudaStream_t st, int ns = 14);
int galerkin_3d(const double *so, const double *ci, double *soc, Dims3 f, Dims3 c, cudaStream_t st, int ns = 14);
int setup_cg_3d(const double *so, Dims3 d, double *abd, int *info, cudaStream_t st, int ns = 14);
template <typename T>
int solve_cg_3d(const double *abd, T *x, const T *b, Dims3 d, cudaStream_t st);
int ir_residual_3d(const double *so, const double *x, const float *e, const double *b, double *xo, float *r32,
                   Dims3 d, Dims3 d32, double *norm_out, double *partial, int apply, cudaStream_t st, int ns = 14);

// Plane relaxation data movement (dir 0 = xy, 1 = xz, 2 = yz); plane problems
// are (n1, n2) grids of row pitch pitch2, problem ipl-1 for plane ipl.
// ns: planes of the 3D operator (14, or 4 for seven-point, whose plane
// problems are five-point: 3 planes each instead of 5)
int plane_coeff(const double *so, Dims3 F, int dir, double *so2, int n, int n1, int n2, int pitch2, cudaStream_t st,
                int ns = 14);
template <typename T>
int plane_copy(T *x3, Dims3 F, int dir, int first, int step, int count, T *x2, int n1, int n2, int pitch2,
               bool to_plane, cudaStream_t st);
template <typename T>
int plane_rhs(const T *so, const T *x, const T *b, Dims3 F, int dir, int first, int step, int count, T *b2, int n1,
              int n2, int pitch2, cudaStream_t st, int ns = 14);

// rows of the banded coarse-grid factor: KD + 1 with KD = nx*(ny+1) + 1
inline int cg3_ldab(Dims3 d) { return d.nx * (d.ny + 1) + 2; }

}  // namespace cdrgpu
