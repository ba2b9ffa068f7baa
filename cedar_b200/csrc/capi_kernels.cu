// capi_kernels.cu -- extern "C" entry points of the individual 2D kernels.
#include <cstdarg>
#include <cstring>
#include <atomic>

#include "kernels2d.cuh"

namespace cdrgpu {

static thread_local char g_err[512] = "";
static std::atomic<long long> g_launches{0};

void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void set_error(int code, const char *fmt, ...)
{
	va_list ap;
	va_start(ap, fmt);
	int n = snprintf(g_err, sizeof(g_err), "[%d] ", code);
	vsnprintf(g_err + n, sizeof(g_err) - n, fmt, ap);
	va_end(ap);
}

static int check_grid(int nx, int ny, int pitch)
{
	if (nx < 1 || ny < 1 || pitch < nx + 2) {
		set_error(CDR_ERR_DIM, "bad grid nx=%d ny=%d pitch=%d", nx, ny, pitch);
		return CDR_ERR_DIM;
	}
	return CDR_OK;
}

static int check_ns(int ns)
{
	if (ns != 3 && ns != 5) {
		set_error(CDR_ERR_ARG, "nstencil must be 3 (five_pt) or 5 (nine_pt), got %d", ns);
		return CDR_ERR_ARG;
	}
	return CDR_OK;
}

static int check_pair(int nxf, int nyf, int pf, int nxc, int nyc, int pc)
{
	CDR_TRY(check_grid(nxf, nyf, pf));
	CDR_TRY(check_grid(nxc, nyc, pc));
	// coarse size rule of cdr2::solver::setup_space (include/cedar/2d/solver.h:93-94)
	if (nxc != (nxf - 1) / 2 + 1 || nyc != (nyf - 1) / 2 + 1) {
		set_error(CDR_ERR_DIM, "coarse grid %dx%d is not the coarsening of %dx%d", nxc, nyc, nxf, nyf);
		return CDR_ERR_DIM;
	}
	return CDR_OK;
}

#define CDR_NONNULL(p)                                             \
	do {                                                           \
		if (!(p)) {                                                \
			set_error(CDR_ERR_ARG, "null pointer argument %s", #p); \
			return CDR_ERR_ARG;                                    \
		}                                                          \
	} while (0)

}  // namespace cdrgpu

using namespace cdrgpu;

extern "C" {

const char *cdr_gpu_last_error(void) { return g_err; }
int cdr_gpu_version(void) { return 100; }
long long cdr_gpu_launch_count(void) { return g_launches.load(); }
size_t cdr_gpu_norm_scratch_bytes(void) { return kNormScratchBytes; }

int cdr_gpu_lines_stream_status(cudaStream_t s)
{
	unsigned to = 0;
	CDR_TRY(lines_stream_timeouts(s, &to));
	if (to) {
		set_error(CDR_ERR_NUMERIC, "%u streamed line-sweep CTAs gave up waiting for their rows", to);
		return CDR_ERR_NUMERIC;
	}
	return CDR_OK;
}

int cdr_gpu_set_wait_limit_ns(long long ns)
{
	const unsigned long long v = ns < 0 ? kStreamWaitDefaultNs : (unsigned long long)ns;
	CDR_TRY(lines_stream_set_wait(v));
	return cg_inv_set_wait(v);
}

int cdr_gpu_inject_timeouts(unsigned lines, unsigned inverse)
{
	CDR_TRY(lines_stream_add_timeouts(lines));
	return cg_inv_add_timeouts(inverse);
}

int cdr_gpu_lines_set_shape(int dir, int fp32, int nstencil, int n, int nlines, int batch, int K, int cap)
{
	LineShape sh;
	sh.K = K;
	sh.cap = cap == 0 ? 256 : cap;
	sh.stream = cap == 0 ? 1 : 0;
	if (!lines_set_shape(dir, fp32 ? 4 : 8, nstencil, n, nlines, batch ? 2 : 1, sh)) {
		set_error(CDR_ERR_ARG, "line shape K=%d cap=%d cannot run lines of %d points", K, cap, n);
		return CDR_ERR_ARG;
	}
	return CDR_OK;
}

int cdr_gpu_lines_shape(int dir, int fp32, int nstencil, int n, int nlines, int batch, int *K, int *cap)
{
	LineShape sh;
	if (!lines_shape(dir, fp32 ? 4 : 8, nstencil, n, nlines, batch ? 2 : 1, &sh)) {
		set_error(CDR_ERR_ARG, "no tuned line shape for n=%d lines=%d", n, nlines);
		return CDR_ERR_ARG;
	}
	if (K) *K = sh.K;
	if (cap) *cap = sh.stream ? 0 : sh.cap;
	return CDR_OK;
}

#define RESID_IMPL(T, SUF)                                                                                      \
	int cdr_gpu_residual_2d_##SUF(const T *so, int ns, const T *x, const T *b, T *r, int nx, int ny, int pitch,  \
	                              double *norm_out, void *scratch, cudaStream_t s)                              \
	{                                                                                                           \
		CDR_TRY(check_grid(nx, ny, pitch));                                                                     \
		CDR_TRY(check_ns(ns));                                                                                  \
		CDR_NONNULL(so); CDR_NONNULL(x); CDR_NONNULL(b); CDR_NONNULL(r);                                        \
		if (norm_out) CDR_NONNULL(scratch);                                                                     \
		return residual_2d<T>(so, ns, x, b, r, Dims2{nx, ny, pitch}, norm_out, (double *)scratch, s);          \
	}
RESID_IMPL(double, f64)
RESID_IMPL(float, f32)

#define RECIP_IMPL(T, SUF)                                                                            \
	int cdr_gpu_setup_recip_2d_##SUF(const T *so, T *sor, int nx, int ny, int pitch, cudaStream_t s)   \
	{                                                                                                 \
		CDR_TRY(check_grid(nx, ny, pitch));                                                           \
		CDR_NONNULL(so); CDR_NONNULL(sor);                                                            \
		return setup_recip_2d<T>(so, sor, Dims2{nx, ny, pitch}, s);                                    \
	}
RECIP_IMPL(double, f64)
RECIP_IMPL(float, f32)

#define POINT_IMPL(T, SUF)                                                                                       \
	int cdr_gpu_relax_point_2d_##SUF(const T *so, int ns, T *x, const T *b, const T *sor, int nx, int ny,         \
	                                 int pitch, int updown, cudaStream_t s)                                      \
	{                                                                                                            \
		CDR_TRY(check_grid(nx, ny, pitch));                                                                      \
		CDR_TRY(check_ns(ns));                                                                                   \
		CDR_NONNULL(so); CDR_NONNULL(x); CDR_NONNULL(b); CDR_NONNULL(sor);                                       \
		return relax_point_2d<T>(so, ns, x, b, sor, Dims2{nx, ny, pitch}, updown, s);                            \
	}
POINT_IMPL(double, f64)
POINT_IMPL(float, f32)

#define LSETUP_IMPL(T, SUF)                                                                                      \
	int cdr_gpu_setup_lines_2d_##SUF(const double *so, int ns, T *sor, int nx, int ny, int pitch, int tpitch,    \
	                                 int dir, int *info, cudaStream_t s)                                         \
	{                                                                                                            \
		CDR_TRY(check_grid(nx, ny, pitch));                                                                      \
		CDR_TRY(check_ns(ns));                                                                                   \
		CDR_NONNULL(so); CDR_NONNULL(sor);                                                                       \
		if (dir != CDR_DIR_X && dir != CDR_DIR_Y) { set_error(CDR_ERR_ARG, "bad dir %d", dir); return CDR_ERR_ARG; } \
		return setup_lines_2d<T>(so, ns, sor, Dims2{nx, ny, pitch}, tpitch, dir, info, s);                      \
	}
LSETUP_IMPL(double, f64)
LSETUP_IMPL(float, f32)

#define LRELAX_IMPL(T, SUF)                                                                                      \
	int cdr_gpu_relax_lines_2d_##SUF(const T *so, int ns, T *x, const T *b, const T *sor, int nx, int ny,         \
	                                 int pitch, int tpitch, int dir, int updown, int flags, cudaStream_t s)      \
	{                                                                                                            \
		CDR_TRY(check_grid(nx, ny, pitch));                                                                      \
		CDR_TRY(check_ns(ns));                                                                                   \
		CDR_NONNULL(so); CDR_NONNULL(x); CDR_NONNULL(b); CDR_NONNULL(sor);                                       \
		if (dir != CDR_DIR_X && dir != CDR_DIR_Y) { set_error(CDR_ERR_ARG, "bad dir %d", dir); return CDR_ERR_ARG; } \
		if (dir == CDR_DIR_Y && tpitch < ny + 2) { set_error(CDR_ERR_DIM, "tpitch %d < ny+2", tpitch); return CDR_ERR_DIM; } \
		return relax_lines_2d<T>(so, ns, x, b, sor, Dims2{nx, ny, pitch}, tpitch, dir, updown, flags, s);       \
	}
LRELAX_IMPL(double, f64)
LRELAX_IMPL(float, f32)

size_t cdr_gpu_lines_sync_words(int nx) { return lines_sync_words(Dims2{nx > 0 ? nx : 0, 1, nx + 2}); }

#define LRELAX_SYNC_IMPL(T, SUF)                                                                                 \
	int cdr_gpu_relax_lines_2d_sync_##SUF(const T *so, int ns, T *x, const T *b, const T *sor, int nx, int ny,    \
	                                      int pitch, int tpitch, int dir, int updown, int flags, unsigned *sync,  \
	                                      cudaStream_t s)                                                         \
	{                                                                                                            \
		CDR_TRY(check_grid(nx, ny, pitch));                                                                      \
		CDR_TRY(check_ns(ns));                                                                                   \
		CDR_NONNULL(so); CDR_NONNULL(x); CDR_NONNULL(b); CDR_NONNULL(sor); CDR_NONNULL(sync);                    \
		if (dir != CDR_DIR_X && dir != CDR_DIR_Y) { set_error(CDR_ERR_ARG, "bad dir %d", dir); return CDR_ERR_ARG; } \
		if (dir == CDR_DIR_Y && tpitch < ny + 2) { set_error(CDR_ERR_DIM, "tpitch %d < ny+2", tpitch); return CDR_ERR_DIM; } \
		return relax_lines_2d<T>(so, ns, x, b, sor, Dims2{nx, ny, pitch}, tpitch, dir, updown, flags, s, sync);  \
	}
LRELAX_SYNC_IMPL(double, f64)
LRELAX_SYNC_IMPL(float, f32)

#define PACKY_IMPL(T, SUF)                                                                                       \
	int cdr_gpu_pack_ylines_2d_##SUF(const T *so, int ns, T *sor, int nx, int ny, int pitch, int tpitch,         \
	                                 cudaStream_t s)                                                            \
	{                                                                                                           \
		CDR_TRY(check_grid(nx, ny, pitch));                                                                     \
		CDR_TRY(check_ns(ns));                                                                                  \
		CDR_NONNULL(so); CDR_NONNULL(sor);                                                                      \
		return pack_ylines_2d<T>(so, ns, sor + 2 * (size_t)tpitch * (nx + 2), Dims2{nx, ny, pitch}, tpitch, s);  \
	}
PACKY_IMPL(double, f64)
PACKY_IMPL(float, f32)


#define RESTRICT_IMPL(T, SUF)                                                                                   \
	int cdr_gpu_restrict_2d_##SUF(const T *ci, const T *rf, T *bc, int nxf, int nyf, int pf, int nxc, int nyc,  \
	                              int pc, cudaStream_t s)                                                       \
	{                                                                                                           \
		CDR_TRY(check_pair(nxf, nyf, pf, nxc, nyc, pc));                                                        \
		CDR_NONNULL(ci); CDR_NONNULL(rf); CDR_NONNULL(bc);                                                      \
		return restrict_2d<T>(ci, rf, bc, Dims2{nxf, nyf, pf}, Dims2{nxc, nyc, pc}, s);                         \
	}
RESTRICT_IMPL(double, f64)
RESTRICT_IMPL(float, f32)

#define INTERP_IMPL(T, SUF)                                                                                     \
	int cdr_gpu_interp_add_2d_##SUF(const T *ci, const T *xc, const T *rf, const T *sof, T *xf, int nxf,        \
	                                int nyf, int pf, int nxc, int nyc, int pc, cudaStream_t s)                  \
	{                                                                                                           \
		CDR_TRY(check_pair(nxf, nyf, pf, nxc, nyc, pc));                                                        \
		CDR_NONNULL(ci); CDR_NONNULL(xc); CDR_NONNULL(rf); CDR_NONNULL(sof); CDR_NONNULL(xf);                   \
		return interp_add_2d<T>(ci, xc, rf, sof, xf, Dims2{nxf, nyf, pf}, Dims2{nxc, nyc, pc}, s);              \
	}
INTERP_IMPL(double, f64)
INTERP_IMPL(float, f32)

int cdr_gpu_rowsum_excess_2d(const double *so, int ns, float *dg, int nx, int ny, int pitch, cudaStream_t s)
{
	CDR_TRY(check_grid(nx, ny, pitch));
	CDR_TRY(check_ns(ns));
	CDR_NONNULL(so); CDR_NONNULL(dg);
	return rowsum_excess_2d(so, ns, dg, Dims2{nx, ny, pitch}, s);
}

int cdr_gpu_residual_2d_wide(const float *so, const float *dg, int ns, const double *x, const float *b, float *r,
                             float *zero, int nx, int ny, int pitch, cudaStream_t s)
{
	CDR_TRY(check_grid(nx, ny, pitch));
	CDR_TRY(check_ns(ns));
	CDR_NONNULL(so); CDR_NONNULL(dg); CDR_NONNULL(x); CDR_NONNULL(b); CDR_NONNULL(r); CDR_NONNULL(zero);
	return residual_2d_wide(so, dg, ns, x, b, r, zero, Dims2{nx, ny, pitch}, s);
}

int cdr_gpu_interp_add_2d_wide(const float *ci, const float *xc, const float *rf, const float *sof, int nsf,
                               const float *xin, double *xout, int nxf, int nyf, int pf, int nxc, int nyc, int pc,
                               cudaStream_t s)
{
	CDR_TRY(check_pair(nxf, nyf, pf, nxc, nyc, pc));
	CDR_TRY(check_ns(nsf));
	CDR_NONNULL(ci); CDR_NONNULL(xc); CDR_NONNULL(rf); CDR_NONNULL(sof); CDR_NONNULL(xin); CDR_NONNULL(xout);
	return interp_add_2d_wide(ci, xc, rf, sof, xin, xout, Dims2{nxf, nyf, pf}, Dims2{nxc, nyc, pc}, s, nsf);
}

int cdr_gpu_setup_interp_2d_f64(const double *so, int ns, double *ci, int nxf, int nyf, int pf, int nxc, int nyc,
                                int pc, cudaStream_t s)
{
	CDR_TRY(check_pair(nxf, nyf, pf, nxc, nyc, pc));
	CDR_TRY(check_ns(ns));
	CDR_NONNULL(so); CDR_NONNULL(ci);
	return setup_interp_2d(so, ns, ci, Dims2{nxf, nyf, pf}, Dims2{nxc, nyc, pc}, s);
}

int cdr_gpu_galerkin_2d_f64(const double *so, int ns, const double *ci, double *soc, int nxf, int nyf, int pf,
                            int nxc, int nyc, int pc, cudaStream_t s)
{
	CDR_TRY(check_pair(nxf, nyf, pf, nxc, nyc, pc));
	CDR_TRY(check_ns(ns));
	CDR_NONNULL(so); CDR_NONNULL(ci); CDR_NONNULL(soc);
	return galerkin_2d(so, ns, ci, soc, Dims2{nxf, nyf, pf}, Dims2{nxc, nyc, pc}, s);
}

int cdr_gpu_setup_cg_2d_f64(const double *so, int ns, int nx, int ny, int pitch, double *abd, int *info,
                            cudaStream_t s)
{
	CDR_TRY(check_grid(nx, ny, pitch));
	CDR_TRY(check_ns(ns));
	CDR_NONNULL(so); CDR_NONNULL(abd);
	return setup_cg_2d(so, ns, Dims2{nx, ny, pitch}, abd, info, s);
}

int cdr_gpu_solve_cg_2d_f64(const double *abd, double *x, const double *b, int nx, int ny, int pitch, cudaStream_t s)
{
	CDR_TRY(check_grid(nx, ny, pitch));
	CDR_NONNULL(abd); CDR_NONNULL(x); CDR_NONNULL(b);
	return solve_cg_2d<double>(abd, x, b, Dims2{nx, ny, pitch}, s);
}

int cdr_gpu_solve_cg_2d_f32(const double *abd, float *x, const float *b, int nx, int ny, int pitch, cudaStream_t s)
{
	CDR_TRY(check_grid(nx, ny, pitch));
	CDR_NONNULL(abd); CDR_NONNULL(x); CDR_NONNULL(b);
	return solve_cg_2d<float>(abd, x, b, Dims2{nx, ny, pitch}, s);
}

}  // extern "C"
