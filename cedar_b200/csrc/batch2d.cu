// batch2d.cu -- batched 2D BoxMG hierarchies (see batch2d.cuh).
#include <cmath>

#include "batch2d.cuh"

namespace cdrgpu {

namespace {

template <typename T> struct BA;
template <> struct BA<double> {
	static double *so(B2Level &L) { return L.so; }
	static double *x(B2Level &L) { return L.x; }
	static double *b(B2Level &L) { return L.b; }
	static double *r(B2Level &L) { return L.r; }
	static double *sor(B2Level &L) { return L.sor; }
	static double *sory(B2Level &L) { return L.sory; }
	static double *yc(B2Level &L) { return L.yc; }
	static double *ci(B2Level &L) { return L.ci; }
};
template <> struct BA<float> {
	static float *so(B2Level &L) { return L.so32; }
	static float *x(B2Level &L) { return L.x32; }
	static float *b(B2Level &L) { return L.b32; }
	static float *r(B2Level &L) { return L.r32; }
	static float *sor(B2Level &L) { return L.sor32; }
	static float *sory(B2Level &L) { return L.sory32; }
	static float *yc(B2Level &L) { return L.yc32; }
	static float *ci(B2Level &L) { return L.ci32; }
};

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

}  // namespace

int num_levels_2d(int nx, int ny, int min_coarse)
{
	float nxc, nyc;
	int ng = 0;
	do {
		ng++;
		nxc = (float)((nx - 1) / (1 << ng) + 1);
		nyc = (float)((ny - 1) / (1 << ng) + 1);
	} while ((nxc < nyc ? nxc : nyc) >= min_coarse);
	return ng;
}

// The owner synchronises its stream before destroying the batch (and may have
// destroyed the stream since); cudaFree itself waits for work on the memory.
Batch2::~Batch2()
{
	for (void *p : allocs_) cudaFree(p);
}

template <typename T>
int Batch2::alloc(T **p, size_t n)
{
	void *q = nullptr;
	CDR_CUDA_TRY(cudaMalloc(&q, n * sizeof(T) + 256));
	CDR_CUDA_TRY(cudaMemsetAsync(q, 0, n * sizeof(T) + 256, st));
	allocs_.push_back(q);
	*p = (T *)q;
	return CDR_OK;
}

int Batch2::init(const cdr_gpu_settings &settings, int ns, int nx, int ny, int nbatch, cudaStream_t stream,
                 bool external32)
{
	s = settings;
	nb = nbatch;
	st = stream;
	if (nb < 1 || nb > 65535) {
		set_error(CDR_ERR_DIM, "batch of %d problems (1..65535)", nb);
		return CDR_ERR_DIM;
	}
	int nl = num_levels_2d(nx, ny, s.min_coarse);
	if (s.num_levels > 0 && s.num_levels < nl) nl = s.num_levels;
	lv.resize(nl);
	const bool lines = s.relaxation != CDR_RELAX_POINT;
	for (int l = 0; l < nl; ++l) {
		B2Level &L = lv[l];
		if (l == 0) { L.nx = nx; L.ny = ny; L.ns = ns; }
		else {
			// cdr2::solver::setup_space (include/cedar/2d/solver.h:93-94)
			L.nx = (int)((lv[l - 1].nx - 1) / 2. + 1);
			L.ny = (int)((lv[l - 1].ny - 1) / 2. + 1);
			L.ns = 5;
		}
		// rows padded to 16 elements (the register-chunk line kernels read 16-byte chunks)
		L.pitch = round_up(L.nx + 2, 16);
		L.tpitch = round_up(L.ny + 2, 16);
		const size_t pl = L.plane() * nb;
		CDR_TRY(alloc(&L.so, pl * L.ns));
		CDR_TRY(alloc(&L.x, pl));
		CDR_TRY(alloc(&L.b, pl));
		CDR_TRY(alloc(&L.r, pl));
		if (l > 0) CDR_TRY(alloc(&L.ci, pl * 8));
		// packed y couplings on levels with y-lines of at most 1024 points
		const bool ypk = l + 1 < nl && L.ny <= 1024 &&
		                 (s.relaxation == CDR_RELAX_LINE_Y || s.relaxation == CDR_RELAX_LINE_XY);
		if (l + 1 < nl) {
			CDR_TRY(alloc(&L.sor, pl * 2));
			if (lines) CDR_TRY(alloc(&L.sory, L.ysize() * nb));
			// FP64 sweeps only in FP64 batches (an FP32-refined batch cycles in FP32)
			if (ypk && !mixed() && !(s.line_flags & CDR_LINES_EXACT)) CDR_TRY(alloc(&L.yc, L.ypsize() * nb));
		}
		if (mixed() && !external32) {
			CDR_TRY(alloc(&L.so32, pl * L.ns));
			CDR_TRY(alloc(&L.x32, pl));
			CDR_TRY(alloc(&L.b32, pl));
			CDR_TRY(alloc(&L.r32, pl));
			if (l > 0) CDR_TRY(alloc(&L.ci32, pl * 8));
			if (l + 1 < nl) {
				CDR_TRY(alloc(&L.sor32, pl * 2));
				if (lines) CDR_TRY(alloc(&L.sory32, L.ysize() * nb));
				if (ypk) CDR_TRY(alloc(&L.yc32, L.ypsize() * nb));
			}
		}
	}
	lc[0] = pick_fused<double>();
	lc[1] = pick_fused<float>();
	const B2Level &Cg = lv.back();
	if ((size_t)Cg.nx * Cg.ny > 4096) {
		set_error(CDR_ERR_DIM, "coarsest grid %dx%d too large for the banded Cholesky", Cg.nx, Cg.ny);
		return CDR_ERR_DIM;
	}
	if (!external32) CDR_TRY(alloc(&abd, abd_size() * nb));
	CDR_TRY(alloc(&info, 2));
	return CDR_OK;
}

int Batch2::setup(bool check)
{
	const Sel all{0, 1, nb};
	CDR_CUDA_TRY(cudaMemsetAsync(info, 0, 2 * sizeof(int), st));
	for (int l = 0; l + 1 < L(); ++l) {
		B2Level &F = lv[l], &C = lv[l + 1];
		const Dims2 df = F.dims(all), dc = C.dims(all);
		CDR_TRY(setup_interp_2d(F.so, F.ns, C.ci, df, dc, st));
		CDR_TRY(galerkin_2d(F.so, F.ns, C.ci, C.so, df, dc, st));
		// smoother setup (multilevel::setup_relax_helper, include/cedar/multilevel.h:134-158)
		const int r = s.relaxation;
		if (r == CDR_RELAX_POINT) {
			CDR_TRY(setup_recip_2d<double>(F.so, F.sor, df, st, F.ns));
			if (mixed()) CDR_TRY(convert_f64_f32(F.sor, F.sor32, F.plane() * 2 * nb, st));
		}
		if (r == CDR_RELAX_LINE_X || r == CDR_RELAX_LINE_XY) {
			CDR_TRY(setup_lines_2d<double>(F.so, F.ns, F.sor, df, F.tpitch, CDR_DIR_X, info, st));
			if (mixed()) CDR_TRY(setup_lines_2d<float>(F.so, F.ns, F.sor32, df, F.tpitch, CDR_DIR_X, info, st));
		}
		if (r == CDR_RELAX_LINE_Y || r == CDR_RELAX_LINE_XY) {
			CDR_TRY(setup_lines_2d<double>(F.so, F.ns, F.sory, df, F.tpitch, CDR_DIR_Y, info, st));
			if (mixed()) CDR_TRY(setup_lines_2d<float>(F.so, F.ns, F.sory32, df, F.tpitch, CDR_DIR_Y, info, st));
			if (F.yc) CDR_TRY(pack_ylines_2d<double>(F.so, F.ns, F.yc, df, F.tpitch, st));
		}
	}
	B2Level &Cg = lv.back();
	CDR_TRY(setup_cg_2d(Cg.so, Cg.ns, Cg.dims(all), abd, info + 1, st));
	if (mixed()) {
		for (int l = 0; l < L(); ++l) {
			B2Level &F = lv[l];
			CDR_TRY(convert_f64_f32(F.so, F.so32, F.plane() * F.ns * nb, st));
			if (l > 0) CDR_TRY(convert_f64_f32(F.ci, F.ci32, F.plane() * 8 * nb, st));
			if (F.yc32) CDR_TRY(pack_ylines_2d<float>(F.so32, F.ns, F.yc32, F.dims(all), F.tpitch, st));
		}
	}
	return check ? check_info() : CDR_OK;
}

// Launch shapes of the line kernels on every non-fused smoothing level, timed
// on all problems at once (the level arrays are the cycle's scratch; level 0 is
// reloaded by each solve)
template <typename T>
int Batch2::tune_lines()
{
	if (s.line_flags & CDR_LINES_NOTUNE) return CDR_OK;
	if (sizeof(T) == 8 && (s.line_flags & CDR_LINES_EXACT)) return CDR_OK;
	const int r = s.relaxation;
	const bool lx = r == CDR_RELAX_LINE_X || r == CDR_RELAX_LINE_XY, ly = r == CDR_RELAX_LINE_Y || r == CDR_RELAX_LINE_XY;
	const int f = lc[sizeof(T) == 4 ? 1 : 0];
	const int stop = f >= 0 ? f : L() - 1;
	const Sel all{0, 1, nb};
	for (int l = 0; l < stop; ++l) {
		B2Level &F = lv[l];
		const Dims2 d = F.dims(all);
		if (lx)
			CDR_TRY(lines_autotune<T>(BA<T>::so(F), F.ns, BA<T>::x(F), BA<T>::b(F), BA<T>::sor(F), d, F.tpitch, CDR_DIR_X,
			                          st));
		if (ly)
			CDR_TRY(lines_autotune<T>(BA<T>::so(F), F.ns, BA<T>::x(F), BA<T>::b(F), BA<T>::sory(F), d, F.tpitch,
			                          CDR_DIR_Y, st, nullptr, BA<T>::yc(F)));
	}
	return CDR_OK;
}

int Batch2::check_info()
{
	int h[2] = {0, 0};
	CDR_CUDA_TRY(cudaMemcpyAsync(h, info, sizeof(h), cudaMemcpyDeviceToHost, st));
	CDR_CUDA_TRY(cudaStreamSynchronize(st));
	if (h[0]) {
		set_error(CDR_ERR_SETUP, "line factorization: non-positive pivot in line %d", h[0]);
		return CDR_ERR_SETUP;
	}
	if (h[1]) {
		set_error(CDR_ERR_SETUP, "coarse-grid Cholesky failed at column %d", h[1]);
		return CDR_ERR_SETUP;
	}
	return CDR_OK;
}

// multilevel::setup_relax_helper smoother closures (include/cedar/multilevel.h:160-222)
template <typename T>
int Batch2::smooth(int l, Sel sel, int updown, bool zero)
{
	B2Level &F = lv[l];
	const Dims2 d = F.dims(sel);
	const size_t f = sel.first, pl = F.plane();
	const T *so = BA<T>::so(F) + f * F.ns * pl;
	T *x = BA<T>::x(F) + f * pl;
	const T *b = BA<T>::b(F) + f * pl;
	const T *sx = BA<T>::sor(F) ? BA<T>::sor(F) + f * 2 * pl : nullptr;
	const T *sy = BA<T>::sory(F) ? BA<T>::sory(F) + f * F.ysize() : nullptr;
	const T *yc = BA<T>::yc(F) ? BA<T>::yc(F) + f * F.ypsize() : nullptr;  // packed y couplings
	const int flags = sizeof(T) == 8 ? s.line_flags : (s.line_flags & CDR_LINES_NOTUNE);
	const int n = updown == CDR_DOWN ? s.nrelax_pre : s.nrelax_post;
	if (zero && (n == 0 || s.relaxation == CDR_RELAX_POINT)) {  // only the line sweeps skip reading it
		CDR_CUDA_TRY(cudaMemset2DAsync(x, sel.step * pl * sizeof(T), 0, pl * sizeof(T), sel.count, st));
		zero = false;
	}
	for (int it = 0; it < n; ++it) {
		const int f = flags | (zero && it == 0 ? CDR_LINES_ZERO_START : 0);  // the first sweep of a zero iterate
		switch (s.relaxation) {
		case CDR_RELAX_POINT: CDR_TRY(relax_point_2d<T>(so, F.ns, x, b, sx, d, updown, st)); break;
		case CDR_RELAX_LINE_X: CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sx, d, F.tpitch, CDR_DIR_X, updown, f, st)); break;
		case CDR_RELAX_LINE_Y: CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sy, d, F.tpitch, CDR_DIR_Y, updown, f, st, nullptr, yc)); break;
		default:
			if (updown == CDR_DOWN) {
				CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sx, d, F.tpitch, CDR_DIR_X, updown, f, st));
				CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sy, d, F.tpitch, CDR_DIR_Y, updown, flags, st, nullptr, yc));
			} else {
				CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sy, d, F.tpitch, CDR_DIR_Y, updown, f, st, nullptr, yc));
				CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sx, d, F.tpitch, CDR_DIR_X, updown, flags, st));
			}
		}
	}
	return CDR_OK;
}

template <typename T>
int Batch2::ncycle(int l, Sel sel, bool zero)
{
	B2Level &F = lv[l], &C = lv[l + 1];
	const Dims2 df = F.dims(sel), dc = C.dims(sel);
	const size_t f = sel.first, fp = F.plane(), cp = C.plane();
	const T *so = BA<T>::so(F) + f * F.ns * fp;
	T *x = BA<T>::x(F) + f * fp;
	const T *b = BA<T>::b(F) + f * fp;
	T *r = BA<T>::r(F) + f * fp;
	const T *ci = BA<T>::ci(C) + f * 8 * cp;
	T *xc = BA<T>::x(C) + f * cp;
	T *bc = BA<T>::b(C) + f * cp;
	CDR_TRY(smooth<T>(l, sel, CDR_DOWN, zero));
	CDR_TRY(residual_2d<T>(so, F.ns, x, b, r, df, nullptr, nullptr, st));
	CDR_TRY(restrict_2d<T>(ci, r, bc, df, dc, st));
	// the selected coarse iterates are zero (include/cedar/cycle/vcycle.h:79):
	// cleared here (rows of cp elements, step*cp apart) for the direct coarse
	// solves, treated as zero without being read by a coarse cycle's first sweep
	const bool direct = l + 1 == L() - 1 || l + 1 == lc[sizeof(T) == 4];
	if (direct) CDR_CUDA_TRY(cudaMemset2DAsync(xc, sel.step * cp * sizeof(T), 0, cp * sizeof(T), sel.count, st));
	if (l + 1 == L() - 1) CDR_TRY(solve_cg_2d<T>(abd + f * abd_size(), xc, bc, dc, st));
	else if (l + 1 == lc[sizeof(T) == 4]) CDR_TRY(fused<T>(l + 1, sel));
	else CDR_TRY(ncycle<T>(l + 1, sel, true));
	CDR_TRY(interp_add_2d<T>(ci, xc, r, so, x, df, dc, st, F.ns));
	CDR_TRY(smooth<T>(l, sel, CDR_UP));
	return CDR_OK;
}

// First level (not the fine one) of the fused coarse cycle: both edges at most
// fuse_coarse and the level's shared-memory copy within the limit
template <typename T>
int Batch2::pick_fused()
{
	if (s.fuse_coarse <= 0) return -1;
	for (int l0 = 1; l0 + 1 < L(); ++l0) {
		if (lv[l0].nx > s.fuse_coarse || lv[l0].ny > s.fuse_coarse || L() - l0 > kMaxCoarseLevels) continue;
		CoarseCycle<T> cc;
		cc.nl = L() - l0;
		cc.relax = s.relaxation;
		for (int l = l0; l < L(); ++l) {
			CoarseLevel<T> &c = cc.lv[l - l0];
			c.nx = lv[l].nx;
			c.ny = lv[l].ny;
			c.ns = lv[l].ns;
		}
		if (coarse_cycle_bytes(cc) <= kCoarseSmemMax) return l0;
	}
	return -1;
}

// Levels l0..L-1 of the selected problems in one launch, one CTA per problem
template <typename T>
int Batch2::fused(int l0, Sel sel)
{
	CoarseCycle<T> cc;
	cc.nl = L() - l0;
	const size_t f = sel.first;
	for (int l = l0; l < L(); ++l) {
		B2Level &V = lv[l];
		CoarseLevel<T> &c = cc.lv[l - l0];
		const size_t pl = V.plane();
		c.so = BA<T>::so(V) + f * V.ns * pl;
		c.sor = BA<T>::sor(V) ? BA<T>::sor(V) + f * 2 * pl : nullptr;
		c.sory = BA<T>::sory(V) ? BA<T>::sory(V) + f * V.ysize() : nullptr;
		c.ci = BA<T>::ci(V) ? BA<T>::ci(V) + f * 8 * pl : nullptr;
		c.x = BA<T>::x(V) + f * pl;
		c.b = BA<T>::b(V) + f * pl;
		c.r = BA<T>::r(V) + f * pl;
		c.nx = V.nx;
		c.ny = V.ny;
		c.pitch = V.pitch;
		c.tpitch = V.tpitch;
		c.ns = V.ns;
	}
	cc.abd = abd + f * abd_size();
	cc.relax = s.relaxation;
	cc.npre = s.nrelax_pre;
	cc.npost = s.nrelax_post;
	cc.bstep = sel.step;
	return coarse_cycle<T>(cc, sel.count, st);
}

template <typename T>
int Batch2::cycle(Sel sel, bool zero)
{
	if (sel.count < 1) return CDR_OK;
	if (L() == 1) {
		B2Level &F = lv[0];
		const size_t f = sel.first, fp = F.plane();
		return solve_cg_2d<T>(abd + f * abd_size(), BA<T>::x(F) + f * fp, BA<T>::b(F) + f * fp, F.dims(sel), st);
	}
	return ncycle<T>(0, sel, zero);
}
template int Batch2::cycle<double>(Sel, bool);
template int Batch2::cycle<float>(Sel, bool);

}  // namespace cdrgpu

// ------------------------------------------------------------- C ABI: batches
namespace cdrgpu {
namespace {

// dst[p] = src[p] for the problems whose flag is set (grid z = problem)
__global__ void k_masked_copy(const double *__restrict__ src, double *__restrict__ dst, size_t per,
                              const int *__restrict__ flag)
{
	if (!flag[blockIdx.z]) return;
	const size_t o = (size_t)blockIdx.z * per;
	for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < per; e += (size_t)gridDim.x * blockDim.x)
		dst[o + e] = src[o + e];
}

}  // namespace
}  // namespace cdrgpu

using namespace cdrgpu;

struct cdr_gpu_batch2d {
	Batch2 B;
	cudaStream_t st = nullptr;
	bool own_stream = false;
	std::vector<void *> allocs;
	double *x64[2] = {nullptr, nullptr};  // FP64 iterates (ping-pong in the refinement loop)
	double *norm = nullptr, *partial = nullptr;
	int *active = nullptr;                // device: 1 while the problem iterates
	double *h_norm = nullptr;             // pinned host copy of the norms
	int *h_active = nullptr;              // pinned host copy of the flags
	cudaGraphExec_t gexec[2] = {nullptr, nullptr};
	long long glaunches[2] = {0, 0};
	std::vector<cudaEvent_t> ev;          // ev[0] start, ev[k] after iteration k
	float setup_ms = 0.f, solve_ms = 0.f;

	template <typename T>
	int alloc(T **p, size_t n)
	{
		void *q = nullptr;
		CDR_CUDA_TRY(cudaMalloc(&q, n * sizeof(T) + 256));
		CDR_CUDA_TRY(cudaMemsetAsync(q, 0, n * sizeof(T) + 256, st));
		allocs.push_back(q);
		*p = (T *)q;
		return CDR_OK;
	}

	int run_cycle(int prec)
	{
		const Sel all{0, 1, B.nb};
		// FP32: the refinement's correction, from zero
		auto body = [&]() -> int { return prec == 0 ? B.cycle<double>(all) : B.cycle<float>(all, true); };
		if (!B.s.use_graph) return body();
		if (!gexec[prec]) {
			cudaGraph_t g = nullptr;
			CDR_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
			const long long before = cdr_gpu_launch_count();
			int rc = body();
			glaunches[prec] = cdr_gpu_launch_count() - before;
			count_launches(-glaunches[prec]);
			cudaError_t e = cudaStreamEndCapture(st, &g);
			if (rc != CDR_OK) {
				if (g) cudaGraphDestroy(g);
				return rc;
			}
			if (e != cudaSuccess) {
				set_error(CDR_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
				return CDR_ERR_CUDA;
			}
			CDR_CUDA_TRY(cudaGraphInstantiate(&gexec[prec], g, 0));
			cudaGraphDestroy(g);
		}
		CDR_CUDA_TRY(cudaGraphLaunch(gexec[prec], st));
		count_launches(glaunches[prec]);
		return CDR_OK;
	}
};

extern "C" {

int cdr_gpu_batch2d_destroy(cdr_gpu_batch2d *h)
{
	if (!h) return CDR_ERR_HANDLE;
	if (h->st) cudaStreamSynchronize(h->st);
	for (auto &g : h->gexec)
		if (g) cudaGraphExecDestroy(g);
	for (auto &e : h->ev) cudaEventDestroy(e);
	for (void *p : h->allocs) cudaFree(p);
	if (h->h_norm) cudaFreeHost(h->h_norm);
	if (h->h_active) cudaFreeHost(h->h_active);
	cudaStream_t st = h->st;
	const bool own = h->own_stream;
	delete h;  // frees the batch arrays
	if (own && st) cudaStreamDestroy(st);
	return CDR_OK;
}

int cdr_gpu_batch2d_create(const cdr_gpu_settings *s, const double *so_dev, int ns, int nx, int ny, int pitch, int nb,
                           cudaStream_t stream, cdr_gpu_batch2d **out)
{
	if (!s || !so_dev || !out) { set_error(CDR_ERR_ARG, "null argument"); return CDR_ERR_ARG; }
	*out = nullptr;
	if (ns != 3 && ns != 5) { set_error(CDR_ERR_ARG, "nstencil must be 3 or 5"); return CDR_ERR_ARG; }
	if (nx < 1 || ny < 1 || pitch < nx + 2) {
		set_error(CDR_ERR_DIM, "bad grid %dx%d pitch %d", nx, ny, pitch);
		return CDR_ERR_DIM;
	}
	if (s->relaxation < CDR_RELAX_POINT || s->relaxation > CDR_RELAX_LINE_XY) {
		set_error(CDR_ERR_ARG, "invalid 2D relaxation %d", s->relaxation);
		return CDR_ERR_ARG;
	}
	if (s->precision != CDR_PREC_F64 && s->precision != CDR_PREC_F32_IR) {
		set_error(CDR_ERR_ARG, "invalid precision %d", s->precision);
		return CDR_ERR_ARG;
	}
	if (s->periodic) {
		set_error(CDR_ERR_UNSUPPORTED, "batched solves: periodic boundaries are implemented for single problems");
		return CDR_ERR_UNSUPPORTED;
	}
	if (s->krylov != CDR_KRYLOV_NONE || s->coarse_solve != CDR_COARSE_BANDED || s->fp32_levels != 0 ||
	    s->cycle != CDR_CYCLE_V) {
		set_error(CDR_ERR_UNSUPPORTED, "batched 2D solves: the Krylov outer iteration is implemented for the 2D solver only");
		return CDR_ERR_UNSUPPORTED;
	}
	if (s->maxiter < 1) { set_error(CDR_ERR_ARG, "max-iter must be positive"); return CDR_ERR_ARG; }
	cdr_gpu_batch2d *h = new cdr_gpu_batch2d();
	if (stream) h->st = stream;
	else {
		if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
			set_error(CDR_ERR_CUDA, "cannot create stream");
			delete h;
			return CDR_ERR_CUDA;
		}
		h->own_stream = true;
	}
	auto fail = [&](int rc) {
		cdr_gpu_batch2d_destroy(h);
		return rc;
	};
	int rc = lines_prepare();
	if (rc == CDR_OK) rc = h->B.init(*s, ns, nx, ny, nb, h->st);
	if (rc != CDR_OK) return fail(rc);
	B2Level &F = h->B.lv[0];
	const size_t pl = F.plane();
	const int per = norm_blocks(F.dims(Sel{0, 1, nb}));
	if ((rc = h->alloc(&h->x64[0], pl * nb)) || (rc = h->alloc(&h->x64[1], pl * nb)) ||
	    (rc = h->alloc(&h->norm, (size_t)nb)) || (rc = h->alloc(&h->partial, (size_t)per * nb)) ||
	    (rc = h->alloc(&h->active, (size_t)nb)))
		return fail(rc);
	if (cudaMallocHost(&h->h_norm, sizeof(double) * nb) != cudaSuccess ||
	    cudaMallocHost(&h->h_active, sizeof(int) * nb) != cudaSuccess) {
		set_error(CDR_ERR_CUDA, "cannot allocate pinned host buffers");
		return fail(CDR_ERR_CUDA);
	}
	h->ev.resize(s->maxiter + 2);
	for (auto &e : h->ev)
		if (cudaEventCreate(&e) != cudaSuccess) {
			e = nullptr;
			set_error(CDR_ERR_CUDA, "cannot create events");
			return fail(CDR_ERR_CUDA);
		}
	// fine operators (caller pitch) -> batch layout; rows of all problems are contiguous in both
	if (cudaMemcpy2DAsync(F.so, F.pitch * sizeof(double), so_dev, pitch * sizeof(double), (nx + 2) * sizeof(double),
	                      (size_t)(ny + 2) * ns * nb, cudaMemcpyDeviceToDevice, h->st) != cudaSuccess) {
		set_error(CDR_ERR_CUDA, "operator copy failed");
		return fail(CDR_ERR_CUDA);
	}
	if (cudaEventRecord(h->ev[0], h->st) != cudaSuccess) return fail(CDR_ERR_CUDA);
	rc = h->B.setup(true);
	if (rc != CDR_OK) return fail(rc);
	if (cudaEventRecord(h->ev[1], h->st) != cudaSuccess || cudaEventSynchronize(h->ev[1]) != cudaSuccess ||
	    cudaEventElapsedTime(&h->setup_ms, h->ev[0], h->ev[1]) != cudaSuccess) {
		set_error(CDR_ERR_CUDA, "setup timing events failed");
		return fail(CDR_ERR_CUDA);
	}
	rc = h->B.tune();
	if (rc != CDR_OK) return fail(rc);
	*out = h;
	return CDR_OK;
}

// multilevel::solve (include/cedar/multilevel.h:278-298) for every problem of the
// batch: each stops at its own relative tolerance (its iterate no longer changes
// after that), iters/rel/done_ms (host arrays of nb, done_ms may be null) report
// its cycles, final relative l2 residual and the time from the start of the
// solve to its last cycle.
int cdr_gpu_batch2d_solve_device(cdr_gpu_batch2d *h, const double *b_dev, double *x_dev, int pitch, int *iters,
                                 double *rel, float *done_ms)
{
	if (!h) { set_error(CDR_ERR_HANDLE, "null batch"); return CDR_ERR_HANDLE; }
	if (!b_dev || !x_dev || !iters || !rel) { set_error(CDR_ERR_ARG, "null argument"); return CDR_ERR_ARG; }
	Batch2 &B = h->B;
	B2Level &F = B.lv[0];
	if (pitch < F.nx + 2) { set_error(CDR_ERR_DIM, "pitch %d < nx+2", pitch); return CDR_ERR_DIM; }
	const int nb = B.nb;
	const cudaStream_t st = h->st;
	const Sel all{0, 1, nb};
	const Dims2 d = F.dims(all);
	const size_t pl = F.plane(), w = (F.nx + 2) * sizeof(double), rows = (size_t)(F.ny + 2) * nb;
	const bool mixed = B.mixed();
	std::vector<double> res0(nb);
	std::vector<int> last(nb, 0);
	for (int p = 0; p < nb; ++p) { iters[p] = 0; rel[p] = 1.0; h->h_active[p] = 1; }
	CDR_CUDA_TRY(cudaMemcpy2DAsync(F.b, F.pitch * sizeof(double), b_dev, pitch * sizeof(double), w, rows,
	                               cudaMemcpyDeviceToDevice, st));
	double *xw = mixed ? h->x64[0] : F.x;  // the iterate the cycles update
	CDR_CUDA_TRY(cudaMemcpy2DAsync(xw, F.pitch * sizeof(double), x_dev, pitch * sizeof(double), w, rows,
	                               cudaMemcpyDeviceToDevice, st));
	if (!mixed)
		CDR_CUDA_TRY(cudaMemcpyAsync(h->x64[0], F.x, sizeof(double) * pl * nb, cudaMemcpyDeviceToDevice, st));
	CDR_CUDA_TRY(cudaMemcpyAsync(h->active, h->h_active, sizeof(int) * nb, cudaMemcpyHostToDevice, st));
	CDR_CUDA_TRY(cudaEventRecord(h->ev[0], st));
	if (mixed) CDR_TRY(ir_residual_2d(F.so, F.ns, h->x64[0], F.x32, F.b, h->x64[1], F.b32, d, d, h->norm, h->partial, 0, st));
	else CDR_TRY(residual_2d<double>(F.so, F.ns, F.x, F.b, F.r, d, h->norm, h->partial, st));
	CDR_CUDA_TRY(cudaMemcpyAsync(h->h_norm, h->norm, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
	CDR_CUDA_TRY(cudaStreamSynchronize(st));
	for (int p = 0; p < nb; ++p) res0[p] = h->h_norm[p];
	int cur = 0, nactive = nb, it = 0, bad = 0;
	const dim3 cgrid(ceil_div((long)pl, 256) < 256 ? ceil_div((long)pl, 256) : 256, 1, nb);
	for (it = 0; it < B.s.maxiter && nactive > 0; ++it) {
		if (mixed) {
			CDR_TRY(h->run_cycle(1));  // the correction F.x32 from zero
			CDR_TRY(ir_residual_2d(F.so, F.ns, h->x64[cur], F.x32, F.b, h->x64[1 - cur], F.b32, d, d, h->norm,
			                       h->partial, 1, st, h->active));
			cur = 1 - cur;
		} else {
			CDR_TRY(h->run_cycle(0));
			CDR_TRY(residual_2d<double>(F.so, F.ns, F.x, F.b, F.r, d, h->norm, h->partial, st));
			// keep the iterate of every problem still iterating
			k_masked_copy<<<cgrid, 256, 0, st>>>(F.x, h->x64[0], pl, h->active);
			CDR_LAUNCH_CHECK();
		}
		CDR_CUDA_TRY(cudaEventRecord(h->ev[it + 1], st));
		CDR_CUDA_TRY(cudaMemcpyAsync(h->h_norm, h->norm, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
		CDR_CUDA_TRY(cudaStreamSynchronize(st));
		for (int p = 0; p < nb; ++p) {
			if (!h->h_active[p]) continue;
			const double r = h->h_norm[p] / res0[p];
			iters[p] = it + 1;
			rel[p] = r;
			last[p] = it + 1;
			if (!std::isfinite(r)) bad = 1;
			if (!(r >= B.s.tol)) {  // converged (or not finite): stop this problem
				h->h_active[p] = 0;
				--nactive;
			}
		}
		CDR_CUDA_TRY(cudaMemcpyAsync(h->active, h->h_active, sizeof(int) * nb, cudaMemcpyHostToDevice, st));
	}
	CDR_CUDA_TRY(cudaMemcpy2DAsync(x_dev, pitch * sizeof(double), mixed ? h->x64[cur] : h->x64[0],
	                               F.pitch * sizeof(double), w, rows, cudaMemcpyDeviceToDevice, st));
	CDR_CUDA_TRY(cudaStreamSynchronize(st));
	CDR_CUDA_TRY(cudaEventElapsedTime(&h->solve_ms, h->ev[0], h->ev[it > 0 ? it : 0]));
	if (done_ms)
		for (int p = 0; p < nb; ++p) {
			float t = 0.f;
			if (last[p] > 0) CDR_CUDA_TRY(cudaEventElapsedTime(&t, h->ev[0], h->ev[last[p]]));
			done_ms[p] = t;
		}
	if (bad) {
		set_error(CDR_ERR_NUMERIC, "non-finite residual norm in a problem of the batch");
		return CDR_ERR_NUMERIC;
	}
	return CDR_OK;
}

// New fine operators for the same batch (same sizes and settings): copied in
// and the whole hierarchy set up again (multilevel::setup,
// include/cedar/multilevel.h:243-265, per problem); the cycle graph and the
// line shapes stay.
int cdr_gpu_batch2d_resetup_device(cdr_gpu_batch2d *h, const double *so_dev, int pitch)
{
	if (!h) { set_error(CDR_ERR_HANDLE, "null batch"); return CDR_ERR_HANDLE; }
	if (!so_dev) { set_error(CDR_ERR_ARG, "null operator"); return CDR_ERR_ARG; }
	B2Level &F = h->B.lv[0];
	if (pitch < F.nx + 2) { set_error(CDR_ERR_DIM, "pitch %d < nx+2", pitch); return CDR_ERR_DIM; }
	CDR_CUDA_TRY(cudaMemcpy2DAsync(F.so, F.pitch * sizeof(double), so_dev, pitch * sizeof(double),
	                               (F.nx + 2) * sizeof(double), (size_t)(F.ny + 2) * F.ns * h->B.nb,
	                               cudaMemcpyDeviceToDevice, h->st));
	CDR_CUDA_TRY(cudaEventRecord(h->ev[0], h->st));
	CDR_TRY(h->B.setup(true));
	CDR_CUDA_TRY(cudaEventRecord(h->ev[1], h->st));
	CDR_CUDA_TRY(cudaEventSynchronize(h->ev[1]));
	CDR_CUDA_TRY(cudaEventElapsedTime(&h->setup_ms, h->ev[0], h->ev[1]));
	return CDR_OK;
}

int cdr_gpu_batch2d_timings(const cdr_gpu_batch2d *h, double *setup_ms, double *solve_ms)
{
	if (!h) return CDR_ERR_HANDLE;
	if (setup_ms) *setup_ms = h->setup_ms;
	if (solve_ms) *solve_ms = h->solve_ms;
	return CDR_OK;
}

int cdr_gpu_batch2d_nlevels(const cdr_gpu_batch2d *h) { return h ? h->B.L() : -1; }

}  // extern "C"
