// capi3d.cu -- extern "C" entry points of the individual 3D kernels.
#include "kernels3d.cuh"

namespace {
using namespace cdrgpu;

int check_grid3(int nx, int ny, int nz, int pitch)
{
	if (nx < 1 || ny < 1 || nz < 1 || pitch < nx + 2) {
		set_error(CDR_ERR_DIM, "bad grid nx=%d ny=%d nz=%d pitch=%d", nx, ny, nz, pitch);
		return CDR_ERR_DIM;
	}
	return CDR_OK;
}

// coarse size rule of cdr3::solver (include/cedar/3d/solver.h): (n-1)/2+1 per axis
int check_pair3(int nxf, int nyf, int nzf, int pf, int nxc, int nyc, int nzc, int pc)
{
	CDR_TRY(check_grid3(nxf, nyf, nzf, pf));
	CDR_TRY(check_grid3(nxc, nyc, nzc, pc));
	if (nxc != (nxf - 1) / 2 + 1 || nyc != (nyf - 1) / 2 + 1 || nzc != (nzf - 1) / 2 + 1) {
		set_error(CDR_ERR_DIM, "coarse grid %dx%dx%d is not the coarsening of %dx%dx%d", nxc, nyc, nzc, nxf, nyf, nzf);
		return CDR_ERR_DIM;
	}
	return CDR_OK;
}

int check_ns3(int ns)
{
	if (ns != 4 && ns != 14) {
		set_error(CDR_ERR_ARG, "nstencil %d: 3D operators have 4 (seven-point) or 14 (27-point) planes", ns);
		return CDR_ERR_ARG;
	}
	return CDR_OK;
}

#define NONNULL3(p)                                                \
	do {                                                           \
		if (!(p)) {                                                \
			set_error(CDR_ERR_ARG, "null pointer argument %s", #p); \
			return CDR_ERR_ARG;                                    \
		}                                                          \
	} while (0)

}  // namespace

extern "C" {

int cdr_gpu_residual_3d_f64(const double *so, int nstencil, const double *x, const double *b, double *r, int nx,
                            int ny, int nz, int pitch, double *norm_out, void *scratch, cudaStream_t s)
{
	CDR_TRY(check_grid3(nx, ny, nz, pitch));
	CDR_TRY(check_ns3(nstencil));
	NONNULL3(so); NONNULL3(x); NONNULL3(b); NONNULL3(r);
	if (norm_out) NONNULL3(scratch);
	return residual_3d<double>(so, x, b, r, Dims3{nx, ny, nz, pitch}, norm_out, (double *)scratch, s, nstencil);
}

int cdr_gpu_residual_3d_f32(const float *so, int nstencil, const float *x, const float *b, float *r, int nx, int ny,
                            int nz, int pitch, double *norm_out, void *scratch, cudaStream_t s)
{
	CDR_TRY(check_grid3(nx, ny, nz, pitch));
	CDR_TRY(check_ns3(nstencil));
	NONNULL3(so); NONNULL3(x); NONNULL3(b); NONNULL3(r);
	if (norm_out) NONNULL3(scratch);
	return residual_3d<float>(so, x, b, r, Dims3{nx, ny, nz, pitch}, norm_out, (double *)scratch, s, nstencil);
}

int cdr_gpu_setup_recip_3d_f64(const double *so, double *sor, int nx, int ny, int nz, int pitch, cudaStream_t s)
{
	CDR_TRY(check_grid3(nx, ny, nz, pitch));
	NONNULL3(so); NONNULL3(sor);
	return setup_recip_3d<double>(so, sor, Dims3{nx, ny, nz, pitch}, s);
}

int cdr_gpu_relax_point_3d_f64(const double *so, int nstencil, double *x, const double *b, const double *sor, int nx,
                               int ny, int nz, int pitch, int updown, cudaStream_t s)
{
	CDR_TRY(check_grid3(nx, ny, nz, pitch));
	CDR_TRY(check_ns3(nstencil));
	NONNULL3(so); NONNULL3(x); NONNULL3(b); NONNULL3(sor);
	return relax_point_3d<double>(so, x, b, sor, Dims3{nx, ny, nz, pitch}, updown, s, nstencil);
}

int cdr_gpu_relax_point_3d_f32(const float *so, int nstencil, float *x, const float *b, const float *sor, int nx,
                               int ny, int nz, int pitch, int updown, cudaStream_t s)
{
	CDR_TRY(check_grid3(nx, ny, nz, pitch));
	CDR_TRY(check_ns3(nstencil));
	NONNULL3(so); NONNULL3(x); NONNULL3(b); NONNULL3(sor);
	return relax_point_3d<float>(so, x, b, sor, Dims3{nx, ny, nz, pitch}, updown, s, nstencil);
}

int cdr_gpu_restrict_3d_f64(const double *ci, const double *rf, double *bc, int nxf, int nyf, int nzf, int pf,
                            int nxc, int nyc, int nzc, int pc, cudaStream_t s)
{
	CDR_TRY(check_pair3(nxf, nyf, nzf, pf, nxc, nyc, nzc, pc));
	NONNULL3(ci); NONNULL3(rf); NONNULL3(bc);
	return restrict_3d<double>(ci, rf, bc, Dims3{nxf, nyf, nzf, pf}, Dims3{nxc, nyc, nzc, pc}, s);
}

int cdr_gpu_interp_add_3d_f64(const double *ci, const double *xc, const double *rf, const double *sof, double *xf,
                              int nxf, int nyf, int nzf, int pf, int nxc, int nyc, int nzc, int pc, cudaStream_t s)
{
	CDR_TRY(check_pair3(nxf, nyf, nzf, pf, nxc, nyc, nzc, pc));
	NONNULL3(ci); NONNULL3(xc); NONNULL3(rf); NONNULL3(sof); NONNULL3(xf);
	return interp_add_3d<double>(ci, xc, rf, sof, xf, Dims3{nxf, nyf, nzf, pf}, Dims3{nxc, nyc, nzc, pc}, s);
}

int cdr_gpu_setup_interp_3d_f64(const double *so, int nstencil, double *ci, int nxf, int nyf, int nzf, int pf,
                                int nxc, int nyc, int nzc, int pc, cudaStream_t s)
{
	CDR_TRY(check_pair3(nxf, nyf, nzf, pf, nxc, nyc, nzc, pc));
	CDR_TRY(check_ns3(nstencil));
	NONNULL3(so); NONNULL3(ci);
	return setup_interp_3d(so, ci, Dims3{nxf, nyf, nzf, pf}, Dims3{nxc, nyc, nzc, pc}, s, nstencil);
}

int cdr_gpu_galerkin_3d_f64(const double *so, int nstencil, const double *ci, double *soc, int nxf, int nyf, int nzf,
                            int pf, int nxc, int nyc, int nzc, int pc, cudaStream_t s)
{
	CDR_TRY(check_pair3(nxf, nyf, nzf, pf, nxc, nyc, nzc, pc));
	CDR_TRY(check_ns3(nstencil));
	NONNULL3(so); NONNULL3(ci); NONNULL3(soc);
	return galerkin_3d(so, ci, soc, Dims3{nxf, nyf, nzf, pf}, Dims3{nxc, nyc, nzc, pc}, s, nstencil);
}

int cdr_gpu_setup_cg_3d_f64(const double *so, int nstencil, int nx, int ny, int nz, int pitch, double *abd,
                            int *info, cudaStream_t s)
{
	CDR_TRY(check_grid3(nx, ny, nz, pitch));
	CDR_TRY(check_ns3(nstencil));
	NONNULL3(so); NONNULL3(abd);
	return setup_cg_3d(so, Dims3{nx, ny, nz, pitch}, abd, info, s, nstencil);
}

int cdr_gpu_solve_cg_3d_f64(const double *abd, double *x, const double *b, int nx, int ny, int nz, int pitch,
                            cudaStream_t s)
{
	CDR_TRY(check_grid3(nx, ny, nz, pitch));
	NONNULL3(abd); NONNULL3(x); NONNULL3(b);
	return solve_cg_3d<double>(abd, x, b, Dims3{nx, ny, nz, pitch}, s);
}

}  // extern "C"
