// solver3d.cu -- 3D BoxMG multilevel solver on the device (27-point or
// seven-point fine operator, 27-point coarse operators; point Gauss-Seidel or
// plane relaxation).
//
// Host control mirrors cdr3::solver over Cedar's multilevel driver: setup builds
// interpolation, Galerkin operator and smoother level by level and factors the
// coarsest operator (multilevel::setup, include/cedar/multilevel.h:243-265); the
// cycle is cycle::vcycle::ncycle_helper (include/cedar/cycle/vcycle.h:57-115);
// the solve loop with its relative l2 stopping test is multilevel::solve
// (multilevel.h:278-298).  As in 2D the cycle is captured once as a CUDA graph
// and replayed; CDR_PREC_F32_IR runs FP32 cycles inside FP64 refinement.
//
// Plane relaxation (planes<rdir>, include/cedar/3d/relax_planes.h:35-234): every
// level but the coarsest keeps, per direction, one 2D hierarchy per plane (a
// Batch2 of all planes of the level).  A sweep relaxes the odd planes, then the
// even ones (reversed going up); each colour is one batched pass: gather the
// planes' x and right-hand sides (b plus the couplings to the neighbouring
// planes), one 2D V-cycle of line-xy smoothing on every plane of the colour, and
// scatter x back.  The planes of one colour couple only through planes of the
// other colour, so the batched pass equals the reference's plane-by-plane loop.
#include <memory>
#include <vector>
#include <cmath>

#include "batch2d.cuh"
#include "kernels3d.cuh"

using namespace cdrgpu;

namespace {

inline int round_up3(int v, int m) { return (v + m - 1) / m * m; }

struct Level3 {
	int nx = 0, ny = 0, nz = 0;
	int ns = 14;  // stencil planes: 14, or 4 for a seven-point fine operator
	Dims3 d{};
	std::unique_ptr<Batch2> pl[3];  // plane problems: xy, xz, yz
	double *so = nullptr, *x = nullptr, *b = nullptr, *r = nullptr, *sor = nullptr, *ci = nullptr;
	float *so32 = nullptr, *x32 = nullptr, *b32 = nullptr, *r32 = nullptr, *sor32 = nullptr, *ci32 = nullptr;
};

template <typename T> struct Arr3;
template <> struct Arr3<double> {
	static double *so(Level3 &L) { return L.so; }
	static double *x(Level3 &L) { return L.x; }
	static double *b(Level3 &L) { return L.b; }
	static double *r(Level3 &L) { return L.r; }
	static double *sor(Level3 &L) { return L.sor; }
	static double *ci(Level3 &L) { return L.ci; }
};
template <> struct Arr3<float> {
	static float *so(Level3 &L) { return L.so32; }
	static float *x(Level3 &L) { return L.x32; }
	static float *b(Level3 &L) { return L.b32; }
	static float *r(Level3 &L) { return L.r32; }
	static float *sor(Level3 &L) { return L.sor32; }
	static float *ci(Level3 &L) { return L.ci32; }
};

// The coarsest direct solve keeps its right-hand side in shared memory.
constexpr size_t kMaxCoarse3 = 6144;

}  // namespace

struct cdr_gpu_solver3 {
	cdr_gpu_settings s{};
	std::vector<Level3> lv;
	std::vector<void *> allocs;
	double *abd = nullptr;
	int *info = nullptr;
	double *norm = nullptr, *partial = nullptr;
	double *x64[2] = {nullptr, nullptr};
	double *h_norm = nullptr;
	cudaStream_t st = nullptr;
	bool own_stream = false;
	cudaGraphExec_t gexec[2] = {nullptr, nullptr};
	long long glaunches[2] = {0, 0};
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;
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
	bool mixed() const { return s.precision == CDR_PREC_F32_IR; }
	int L() const { return (int)lv.size(); }

	bool plane(int dir) const
	{
		const int r = s.relaxation;
		return r == CDR_RELAX_PLANE_XYZ || r == CDR_RELAX_PLANE_XY + dir;
	}

	// relax_planes (include/cedar/3d/relax_planes.h:35-70) for one direction
	template <typename T>
	int relax_planes(int l, int dir, T *x, const T *b, int updown)
	{
		Level3 &F = lv[l];
		Batch2 &P = *F.pl[dir];
		B2Level &P0 = P.lv[0];
		T *x2 = sizeof(T) == 8 ? (T *)P0.x : (T *)P0.x32;
		T *b2 = sizeof(T) == 8 ? (T *)P0.b : (T *)P0.b32;
		const int n = P.nb;
		for (int c = 0; c < 2; ++c) {
			// DOWN: odd planes (1, 3, ...) first; UP: even planes first
			const int beg = (updown == CDR_DOWN) == (c == 0) ? 1 : 2;
			if (beg > n) continue;
			const Sel sel{beg - 1, 2, (n - beg) / 2 + 1};
			CDR_TRY(plane_copy<T>(x, F.d, dir, sel.first, 2, sel.count, x2, P0.nx, P0.ny, P0.pitch, true, st));
			CDR_TRY(plane_rhs<T>(Arr3<T>::so(F), x, b, F.d, dir, sel.first, 2, sel.count, b2, P0.nx, P0.ny, P0.pitch,
			                     st, F.ns));
			CDR_TRY(P.cycle<T>(sel));
			CDR_TRY(plane_copy<T>(x, F.d, dir, sel.first, 2, sel.count, x2, P0.nx, P0.ny, P0.pitch, false, st));
		}
		return CDR_OK;
	}

	// multilevel::setup_relax_helper closures (include/cedar/multilevel.h:160-222):
	// plane-xyz runs xy, yz, xz going down and xz, yz, xy going up
	template <typename T>
	int smooth(int l, T *x, const T *b, int updown)
	{
		Level3 &F = lv[l];
		const int n = updown == CDR_DOWN ? s.nrelax_pre : s.nrelax_post;
		static const int down[3] = {0, 2, 1}, up[3] = {1, 2, 0};
		for (int it = 0; it < n; ++it) {
			if (s.relaxation == CDR_RELAX_POINT) {
				CDR_TRY(relax_point_3d<T>(Arr3<T>::so(F), x, b, Arr3<T>::sor(F), F.d, updown, st, F.ns));
				continue;
			}
			for (int q = 0; q < 3; ++q) {
				const int dir = updown == CDR_DOWN ? down[q] : up[q];
				if (plane(dir)) CDR_TRY(relax_planes<T>(l, dir, x, b, updown));
			}
		}
		return CDR_OK;
	}

	// cycle::vcycle::ncycle_helper (include/cedar/cycle/vcycle.h:57-115), n = 1
	template <typename T>
	int ncycle(int l, T *x, const T *b)
	{
		Level3 &F = lv[l], &C = lv[l + 1];
		CDR_TRY(smooth<T>(l, x, b, CDR_DOWN));
		CDR_TRY(residual_3d<T>(Arr3<T>::so(F), x, b, Arr3<T>::r(F), F.d, nullptr, nullptr, st, F.ns));
		CDR_TRY(restrict_3d<T>(Arr3<T>::ci(C), Arr3<T>::r(F), Arr3<T>::b(C), F.d, C.d, st));
		CDR_CUDA_TRY(cudaMemsetAsync(Arr3<T>::x(C), 0, sizeof(T) * C.d.plane(), st));
		if (l + 1 == L() - 1) CDR_TRY(solve_cg_3d<T>(abd, Arr3<T>::x(C), Arr3<T>::b(C), C.d, st));
		else CDR_TRY(ncycle<T>(l + 1, Arr3<T>::x(C), Arr3<T>::b(C)));
		CDR_TRY(interp_add_3d<T>(Arr3<T>::ci(C), Arr3<T>::x(C), Arr3<T>::r(F), Arr3<T>::so(F), x, F.d, C.d, st));
		CDR_TRY(smooth<T>(l, x, b, CDR_UP));
		return CDR_OK;
	}

	// cycle::fcycle::fmg_cycle / fmg_cycle_helper (include/cedar/cycle/fcycle.h:49-83):
	// restrict b, recurse (the coarsest level solved directly), then x = P x_c with
	// a zero residual term and one V-cycle on this level
	template <typename T>
	int fcycle(int l, T *x, const T *b)
	{
		if (l == L() - 1) return solve_cg_3d<T>(abd, x, b, lv[l].d, st);
		Level3 &F = lv[l], &C = lv[l + 1];
		CDR_TRY(restrict_3d<T>(Arr3<T>::ci(C), b, Arr3<T>::b(C), F.d, C.d, st));
		CDR_TRY(fcycle<T>(l + 1, Arr3<T>::x(C), Arr3<T>::b(C)));
		CDR_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(T) * F.d.plane(), st));
		CDR_CUDA_TRY(cudaMemsetAsync(Arr3<T>::r(F), 0, sizeof(T) * F.d.plane(), st));
		CDR_TRY(interp_add_3d<T>(Arr3<T>::ci(C), Arr3<T>::x(C), Arr3<T>::r(F), Arr3<T>::so(F), x, F.d, C.d, st));
		return ncycle<T>(l, x, b);
	}

	template <typename T>
	int cycle(T *x, const T *b)
	{
		if (L() == 1) return solve_cg_3d<T>(abd, x, b, lv[0].d, st);
		if (s.cycle == CDR_CYCLE_F) return fcycle<T>(0, x, b);
		return ncycle<T>(0, x, b);
	}

	int run_cycle(int prec)
	{
		auto body = [&]() -> int {
			if (prec == 0) return cycle<double>(lv[0].x, lv[0].b);
			return cycle<float>(lv[0].x32, lv[0].b32);
		};
		if (!s.use_graph) return body();
		if (!gexec[prec]) {
			cudaGraph_t g = nullptr;
			CDR_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
			const long long before = cdr_gpu_launch_count();
			int rc = body();
			glaunches[prec] = cdr_gpu_launch_count() - before;
			count_launches(-glaunches[prec]);  // captured, not launched
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

	// multilevel::setup (include/cedar/multilevel.h:243-265)
	int setup()
	{
		for (int l = 0; l + 1 < L(); ++l) {
			Level3 &F = lv[l], &C = lv[l + 1];
			CDR_TRY(setup_interp_3d(F.so, C.ci, F.d, C.d, st, F.ns));
			CDR_TRY(galerkin_3d(F.so, C.ci, C.so, F.d, C.d, st, F.ns));
			CDR_TRY(setup_recip_3d<double>(F.so, F.sor, F.d, st));
			// plane smoothers: 2D operators from the in-plane couplings, then the 2D setups
			for (int dir = 0; dir < 3; ++dir) {
				if (!F.pl[dir]) continue;
				Batch2 &P = *F.pl[dir];
				B2Level &P0 = P.lv[0];
				CDR_TRY(plane_coeff(F.so, F.d, dir, P0.so, P.nb, P0.nx, P0.ny, P0.pitch, st, F.ns));
				CDR_TRY(P.setup(false));
			}
		}
		for (int l = 0; l + 1 < L(); ++l)
			for (int dir = 0; dir < 3; ++dir)
				if (lv[l].pl[dir]) CDR_TRY(lv[l].pl[dir]->check_info());
		Level3 &Cg = lv[L() - 1];
		CDR_TRY(setup_cg_3d(Cg.so, Cg.d, abd, info, st, Cg.ns));
		if (mixed()) {
			for (int l = 0; l < L(); ++l) {
				Level3 &F = lv[l];
				CDR_TRY(convert_f64_f32(F.so, F.so32, F.d.plane() * F.ns, st));
				if (l > 0) CDR_TRY(convert_f64_f32(F.ci, F.ci32, F.d.plane() * 26, st));
				if (l + 1 < L()) CDR_TRY(convert_f64_f32(F.sor, F.sor32, F.d.plane(), st));
			}
		}
		int hinfo = 0;
		CDR_CUDA_TRY(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st));
		CDR_CUDA_TRY(cudaStreamSynchronize(st));
		if (hinfo) {
			set_error(CDR_ERR_SETUP, "coarse-grid Cholesky failed at column %d", hinfo);
			return CDR_ERR_SETUP;
		}
		return CDR_OK;
	}
};

// cdr3::solver::compute_num_levels (include/cedar/3d/solver.h:59-77)
static int num_levels3(int nx, int ny, int nz, int min_coarse)
{
	float a, b, c;
	int ng = 0;
	do {
		ng++;
		a = (float)((nx - 1) / (1 << ng) + 1);
		b = (float)((ny - 1) / (1 << ng) + 1);
		c = (float)((nz - 1) / (1 << ng) + 1);
	} while (std::fmin(std::fmin(a, b), c) >= min_coarse);
	return ng;
}

static int create3(cdr_gpu_solver3 *h, const double *so_src, int src_pitch, cudaMemcpyKind kind, int ns, int nx, int ny,
                   int nz)
{
	const cdr_gpu_settings &s = h->s;
	int nl = num_levels3(nx, ny, nz, s.min_coarse);
	if (s.num_levels > 0) {
		if (s.num_levels > nl) {
			set_error(CDR_ERR_ARG, "too many levels specified (%d > %d)", s.num_levels, nl);
			return CDR_ERR_ARG;
		}
		nl = s.num_levels;
	}
	h->lv.resize(nl);
	for (int l = 0; l < nl; ++l) {
		Level3 &L = h->lv[l];
		if (l == 0) { L.nx = nx; L.ny = ny; L.nz = nz; }
		else {
			const Level3 &P = h->lv[l - 1];
			L.nx = (int)((P.nx - 1) / 2. + 1);
			L.ny = (int)((P.ny - 1) / 2. + 1);
			L.nz = (int)((P.nz - 1) / 2. + 1);
		}
		L.d = Dims3{L.nx, L.ny, L.nz, round_up3(L.nx + 2, 8)};
		L.ns = l == 0 ? ns : 14;
		const size_t pl = L.d.plane();
		CDR_TRY(h->alloc(&L.so, pl * L.ns));
		CDR_TRY(h->alloc(&L.x, pl));
		CDR_TRY(h->alloc(&L.b, pl));
		CDR_TRY(h->alloc(&L.r, pl));
		if (l > 0) CDR_TRY(h->alloc(&L.ci, pl * 26));
		if (l + 1 < nl) CDR_TRY(h->alloc(&L.sor, pl));
		// plane problems of this level: the reference's plane config (line-xy,
		// max-iter 1, other keys at their defaults; src/kernel_params.cc:83-89);
		// five-point planes for a seven-point level (relax_planes.h:77-107)
		for (int dir = 0; dir < 3 && l + 1 < nl; ++dir) {
			if (!h->plane(dir)) continue;
			cdr_gpu_settings s2;
			cdr_gpu_settings_default(&s2);
			s2.relaxation = CDR_RELAX_LINE_XY;
			s2.maxiter = 1;
			s2.precision = s.precision;
			s2.line_flags = s.line_flags;
			s2.fuse_coarse = s.fuse_coarse;  // the planes' coarse levels fused as the caller asks
			const int np = dir == 0 ? L.nz : dir == 1 ? L.ny : L.nx;
			const int n1 = dir == 2 ? L.ny : L.nx, n2 = dir == 0 ? L.ny : L.nz;
			L.pl[dir].reset(new Batch2());
			CDR_TRY(L.pl[dir]->init(s2, L.ns == 4 ? 3 : 5, n1, n2, np, h->st));
		}
		if (h->mixed()) {
			CDR_TRY(h->alloc(&L.so32, pl * L.ns));
			CDR_TRY(h->alloc(&L.x32, pl));
			CDR_TRY(h->alloc(&L.b32, pl));
			CDR_TRY(h->alloc(&L.r32, pl));
			if (l > 0) CDR_TRY(h->alloc(&L.ci32, pl * 26));
			if (l + 1 < nl) CDR_TRY(h->alloc(&L.sor32, pl));
		}
	}
	Level3 &Cg = h->lv[nl - 1];
	const size_t ncg = (size_t)Cg.nx * Cg.ny * Cg.nz;
	if (ncg > kMaxCoarse3) {
		set_error(CDR_ERR_DIM, "coarsest grid %dx%dx%d too large for the banded Cholesky (%zu > %zu unknowns)", Cg.nx,
		          Cg.ny, Cg.nz, ncg, kMaxCoarse3);
		return CDR_ERR_DIM;
	}
	CDR_TRY(h->alloc(&h->abd, (size_t)cg3_ldab(Cg.d) * ncg));
	CDR_TRY(h->alloc(&h->info, 2));
	CDR_TRY(h->alloc(&h->norm, 4));
	CDR_TRY(h->alloc(&h->partial, kNormScratchBytes / sizeof(double)));
	if (h->mixed()) {
		CDR_TRY(h->alloc(&h->x64[0], h->lv[0].d.plane()));
		CDR_TRY(h->alloc(&h->x64[1], h->lv[0].d.plane()));
	}
	CDR_CUDA_TRY(cudaMallocHost(&h->h_norm, 4 * sizeof(double)));
	// fine operator (source pitch) -> device pitch: every row of every k-slice and plane
	Level3 &F = h->lv[0];
	CDR_CUDA_TRY(cudaMemcpy2DAsync(F.so, F.d.pitch * sizeof(double), so_src, src_pitch * sizeof(double),
	                               (nx + 2) * sizeof(double), (size_t)(ny + 2) * (nz + 2) * ns, kind, h->st));
	CDR_CUDA_TRY(cudaEventRecord(h->ev0, h->st));
	CDR_TRY(h->setup());
	CDR_CUDA_TRY(cudaEventRecord(h->ev1, h->st));
	CDR_CUDA_TRY(cudaEventSynchronize(h->ev1));
	CDR_CUDA_TRY(cudaEventElapsedTime(&h->setup_ms, h->ev0, h->ev1));
	return CDR_OK;
}

// multilevel::solve (include/cedar/multilevel.h:278-298) on the level-0 buffers.
static int solve3_loaded(cdr_gpu_solver3 *h, int *iters, double *hist, int maxhist)
{
	Level3 &F = h->lv[0];
	cudaStream_t st = h->st;
	double res0 = 0;
	int it = 0;
	auto fetch = [&]() -> int {
		CDR_CUDA_TRY(cudaMemcpyAsync(h->h_norm, h->norm, sizeof(double), cudaMemcpyDeviceToHost, st));
		CDR_CUDA_TRY(cudaStreamSynchronize(st));
		return CDR_OK;
	};
	CDR_CUDA_TRY(cudaEventRecord(h->ev0, st));
	int cur = 0;
	if (!h->mixed()) {
		CDR_TRY(residual_3d<double>(F.so, F.x, F.b, F.r, F.d, h->norm, h->partial, st, F.ns));
	} else {
		CDR_CUDA_TRY(cudaMemcpyAsync(h->x64[0], F.x, sizeof(double) * F.d.plane(), cudaMemcpyDeviceToDevice, st));
		CDR_TRY(ir_residual_3d(F.so, h->x64[0], F.x32, F.b, h->x64[1], F.b32, F.d, F.d, h->norm, h->partial, 0, st,
		                       F.ns));
	}
	CDR_TRY(fetch());
	res0 = h->h_norm[0];
	for (it = 0; it < h->s.maxiter;) {
		if (!h->mixed()) {
			CDR_TRY(h->run_cycle(0));
			CDR_TRY(residual_3d<double>(F.so, F.x, F.b, F.r, F.d, h->norm, h->partial, st, F.ns));
		} else {
			CDR_CUDA_TRY(cudaMemsetAsync(F.x32, 0, sizeof(float) * F.d.plane(), st));
			CDR_TRY(h->run_cycle(1));
			CDR_TRY(ir_residual_3d(F.so, h->x64[cur], F.x32, F.b, h->x64[1 - cur], F.b32, F.d, F.d, h->norm,
			                       h->partial, 1, st, F.ns));
			cur = 1 - cur;
		}
		CDR_TRY(fetch());
		const double rel = h->h_norm[0] / res0;
		if (hist && it < maxhist) hist[it] = rel;
		++it;
		if (!std::isfinite(rel)) {
			set_error(CDR_ERR_NUMERIC, "non-finite residual norm at iteration %d", it - 1);
			return CDR_ERR_NUMERIC;
		}
		if (rel < h->s.tol) break;
	}
	if (h->mixed())
		CDR_CUDA_TRY(cudaMemcpyAsync(F.x, h->x64[cur], sizeof(double) * F.d.plane(), cudaMemcpyDeviceToDevice, st));
	CDR_CUDA_TRY(cudaEventRecord(h->ev1, st));
	CDR_CUDA_TRY(cudaEventSynchronize(h->ev1));
	CDR_CUDA_TRY(cudaEventElapsedTime(&h->solve_ms, h->ev0, h->ev1));
	if (iters) *iters = it;
	return CDR_OK;
}

extern "C" {

int cdr_gpu_solver3_destroy(cdr_gpu_solver3 *h)
{
	if (!h) return CDR_ERR_HANDLE;
	if (h->st) cudaStreamSynchronize(h->st);
	for (auto &g : h->gexec)
		if (g) cudaGraphExecDestroy(g);
	for (auto &L : h->lv)  // plane batches before the stream they use
		for (auto &p : L.pl) p.reset();
	for (void *p : h->allocs) cudaFree(p);
	if (h->h_norm) cudaFreeHost(h->h_norm);
	if (h->ev0) cudaEventDestroy(h->ev0);
	if (h->ev1) cudaEventDestroy(h->ev1);
	if (h->own_stream && h->st) cudaStreamDestroy(h->st);
	delete h;
	return CDR_OK;
}

static int create3_any(const cdr_gpu_settings *s, const double *so_src, int src_pitch, cudaMemcpyKind kind, int ns,
                       int nx, int ny, int nz, cudaStream_t stream, cdr_gpu_solver3 **out)
{
	if (!s || !so_src || !out) { set_error(CDR_ERR_ARG, "null argument"); return CDR_ERR_ARG; }
	*out = nullptr;
	if (ns != 4 && ns != 14) {
		set_error(CDR_ERR_ARG, "nstencil %d: 3D operators have 4 (seven-point) or 14 (27-point) planes", ns);
		return CDR_ERR_ARG;
	}
	if (nx < 1 || ny < 1 || nz < 1) { set_error(CDR_ERR_DIM, "bad grid %dx%dx%d", nx, ny, nz); return CDR_ERR_DIM; }
	if (s->relaxation != CDR_RELAX_POINT && (s->relaxation < CDR_RELAX_PLANE_XY || s->relaxation > CDR_RELAX_PLANE_XYZ)) {
		set_error(CDR_ERR_UNSUPPORTED, "3D solver: point or plane relaxation (got %d)", s->relaxation);
		return CDR_ERR_UNSUPPORTED;
	}
	if (s->precision != CDR_PREC_F64 && s->precision != CDR_PREC_F32_IR) {
		set_error(CDR_ERR_ARG, "invalid precision %d", s->precision);
		return CDR_ERR_ARG;
	}
	if (s->cycle != CDR_CYCLE_V && s->cycle != CDR_CYCLE_F) {
		set_error(CDR_ERR_ARG, "invalid cycle type %d", s->cycle);
		return CDR_ERR_ARG;
	}
	if (s->krylov != CDR_KRYLOV_NONE || s->coarse_solve != CDR_COARSE_BANDED || s->fp32_levels != 0) {
		set_error(CDR_ERR_UNSUPPORTED, "3D solver: the Krylov outer iteration is implemented for the 2D solver only");
		return CDR_ERR_UNSUPPORTED;
	}
	if (s->periodic) {
		set_error(CDR_ERR_UNSUPPORTED, "3D solver: periodic boundaries are implemented for the 2D solver only");
		return CDR_ERR_UNSUPPORTED;
	}
	cdr_gpu_solver3 *h = new cdr_gpu_solver3();
	h->s = *s;
	if (stream) h->st = stream;
	else {
		if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
			set_error(CDR_ERR_CUDA, "cannot create stream");
			delete h;
			return CDR_ERR_CUDA;
		}
		h->own_stream = true;
	}
	cudaEventCreate(&h->ev0);
	cudaEventCreate(&h->ev1);
	int rc = lines_prepare();  // the plane problems' line and fused kernels
	if (rc == CDR_OK) rc = create3(h, so_src, src_pitch, kind, ns, nx, ny, nz);
	if (rc != CDR_OK) {
		cdr_gpu_solver3_destroy(h);
		return rc;
	}
	*out = h;
	return CDR_OK;
}

int cdr_gpu_solver3_create(const cdr_gpu_settings *s, const double *so_host, int nstencil, int nx, int ny, int nz,
                           cudaStream_t stream, cdr_gpu_solver3 **out)
{
	return create3_any(s, so_host, nx + 2, cudaMemcpyHostToDevice, nstencil, nx, ny, nz, stream, out);
}

int cdr_gpu_solver3_create_device(const cdr_gpu_settings *s, const double *so_dev, int nstencil, int nx, int ny,
                                  int nz, int pitch, cudaStream_t stream, cdr_gpu_solver3 **out)
{
	if (pitch < nx + 2) { set_error(CDR_ERR_DIM, "pitch %d < nx+2", pitch); return CDR_ERR_DIM; }
	return create3_any(s, so_dev, pitch, cudaMemcpyDeviceToDevice, nstencil, nx, ny, nz, stream, out);
}

static int copy3(void *dst, int dpitch, const void *src, int spitch, int nx, int ny, int nz, cudaMemcpyKind kind,
                 cudaStream_t st)
{
	const size_t w = (nx + 2) * sizeof(double);
	CDR_CUDA_TRY(cudaMemcpy2DAsync(dst, dpitch * sizeof(double), src, spitch * sizeof(double), w,
	                               (size_t)(ny + 2) * (nz + 2), kind, st));
	return CDR_OK;
}

int cdr_gpu_solver3_solve(cdr_gpu_solver3 *h, const double *b_host, double *x_host, int *iters, double *hist,
                          int maxhist)
{
	if (!h) { set_error(CDR_ERR_HANDLE, "null solver"); return CDR_ERR_HANDLE; }
	if (!b_host || !x_host) { set_error(CDR_ERR_ARG, "null buffer"); return CDR_ERR_ARG; }
	Level3 &F = h->lv[0];
	CDR_TRY(copy3(F.b, F.d.pitch, b_host, F.nx + 2, F.nx, F.ny, F.nz, cudaMemcpyHostToDevice, h->st));
	CDR_TRY(copy3(F.x, F.d.pitch, x_host, F.nx + 2, F.nx, F.ny, F.nz, cudaMemcpyHostToDevice, h->st));
	CDR_TRY(solve3_loaded(h, iters, hist, maxhist));
	CDR_TRY(copy3(x_host, F.nx + 2, F.x, F.d.pitch, F.nx, F.ny, F.nz, cudaMemcpyDeviceToHost, h->st));
	CDR_CUDA_TRY(cudaStreamSynchronize(h->st));
	return CDR_OK;
}

int cdr_gpu_solver3_solve_device(cdr_gpu_solver3 *h, const double *b_dev, double *x_dev, int pitch, int *iters,
                                 double *hist, int maxhist)
{
	if (!h) { set_error(CDR_ERR_HANDLE, "null solver"); return CDR_ERR_HANDLE; }
	if (!b_dev || !x_dev) { set_error(CDR_ERR_ARG, "null buffer"); return CDR_ERR_ARG; }
	Level3 &F = h->lv[0];
	if (pitch < F.nx + 2) { set_error(CDR_ERR_DIM, "pitch %d < nx+2", pitch); return CDR_ERR_DIM; }
	CDR_TRY(copy3(F.b, F.d.pitch, b_dev, pitch, F.nx, F.ny, F.nz, cudaMemcpyDeviceToDevice, h->st));
	CDR_TRY(copy3(F.x, F.d.pitch, x_dev, pitch, F.nx, F.ny, F.nz, cudaMemcpyDeviceToDevice, h->st));
	CDR_TRY(solve3_loaded(h, iters, hist, maxhist));
	CDR_TRY(copy3(x_dev, pitch, F.x, F.d.pitch, F.nx, F.ny, F.nz, cudaMemcpyDeviceToDevice, h->st));
	CDR_CUDA_TRY(cudaStreamSynchronize(h->st));
	return CDR_OK;
}

int cdr_gpu_solver3_nlevels(const cdr_gpu_solver3 *h) { return h ? (int)h->lv.size() : -1; }

int cdr_gpu_solver3_level(const cdr_gpu_solver3 *h, int level, int which, void **ptr, int *nx, int *ny, int *nz,
                          int *pitch)
{
	if (!h) { set_error(CDR_ERR_HANDLE, "null solver"); return CDR_ERR_HANDLE; }
	if (level < 0 || level >= (int)h->lv.size()) { set_error(CDR_ERR_ARG, "bad level %d", level); return CDR_ERR_ARG; }
	const Level3 &L = h->lv[level];
	void *p = nullptr;
	switch (which) {
	case 0: p = L.so; break;
	case 1: p = L.x; break;
	case 2: p = L.b; break;
	case 3: p = L.r; break;
	case 4: p = L.sor; break;
	case 6: p = L.ci; break;
	case 16: p = L.so32; break;
	case 17: p = L.x32; break;
	case 18: p = L.b32; break;
	case 19: p = L.r32; break;
	case 20: p = L.sor32; break;
	case 22: p = L.ci32; break;
	case 100: p = h->abd; break;
	default: set_error(CDR_ERR_ARG, "bad array id %d", which); return CDR_ERR_ARG;
	}
	if (ptr) *ptr = p;
	if (nx) *nx = L.nx;
	if (ny) *ny = L.ny;
	if (nz) *nz = L.nz;
	if (pitch) *pitch = L.d.pitch;
	return CDR_OK;
}

int cdr_gpu_solver3_level_get(const cdr_gpu_solver3 *h, int level, int which, void *host, size_t bytes)
{
	void *p = nullptr;
	int nx, ny, nz, pitch;
	CDR_TRY(cdr_gpu_solver3_level(h, level, which, &p, &nx, &ny, &nz, &pitch));
	if (!p) { set_error(CDR_ERR_ARG, "array %d not allocated on level %d", which, level); return CDR_ERR_ARG; }
	const int w = which & 15;
	const size_t elem = which >= 16 && which < 100 ? sizeof(float) : sizeof(double);
	size_t n;
	if (which == 100) n = (size_t)cg3_ldab(h->lv.back().d) * h->lv.back().nx * h->lv.back().ny * h->lv.back().nz;
	else n = (size_t)(w == 0 ? h->lv[level].ns : w == 6 ? 26 : 1) * h->lv[level].d.plane();
	if (!host || bytes < n * elem) {
		set_error(CDR_ERR_ARG, "host buffer too small (%zu < %zu)", bytes, n * elem);
		return CDR_ERR_ARG;
	}
	CDR_CUDA_TRY(cudaMemcpyAsync(host, p, n * elem, cudaMemcpyDeviceToHost, h->st));
	CDR_CUDA_TRY(cudaStreamSynchronize(h->st));
	return CDR_OK;
}

int cdr_gpu_solver3_timings(const cdr_gpu_solver3 *h, double *setup_ms, double *solve_ms)
{
	if (!h) return CDR_ERR_HANDLE;
	if (setup_ms) *setup_ms = h->setup_ms;
	if (solve_ms) *solve_ms = h->solve_ms;
	return CDR_OK;
}

}  // extern "C"
