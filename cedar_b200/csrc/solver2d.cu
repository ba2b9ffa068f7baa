// solver2d.cu -- 2D BoxMG multilevel solver on the device.
//
// Host control mirrors Cedar's multilevel driver: setup builds the hierarchy
// level by level (interpolation, Galerkin operator, smoother) and factors the
// coarsest operator (multilevel::setup, include/cedar/multilevel.h:243-265);
// the V-cycle recursion is cycle::vcycle::ncycle_helper
// (include/cedar/cycle/vcycle.h:57-115); the solve loop with its relative l2
// stopping test is multilevel::solve (multilevel.h:278-298).  Every step is a
// stream-ordered kernel launch; the whole cycle is captured once as a CUDA
// graph and replayed, and only the per-iteration residual norm comes back to
// the host.
//
// Two solve forms:
//   CDR_PREC_F64     plain FP64 cycles (the drop-in path);
//   CDR_PREC_F32_IR  FP64 iterative refinement: r = b - A x in FP64, one FP32
//                    V-cycle on r (FP32 copies of every operator, interpolation
//                    and line factor; FP64 coarsest Cholesky), x += e in FP64.
// With settings.krylov = CDR_KRYLOV_FCG either cycle instead preconditions
// flexible CG (k2_krylov.cu); the iteration (cycle + three FCG kernels) is one
// CUDA graph.
#include <algorithm>
#include <vector>
#include <cstring>
#include <cmath>

#include "kernels2d.cuh"

using namespace cdrgpu;

namespace {

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

struct Level {
	int nx = 0, ny = 0, ns = 5;
	Dims2 d{};      // pitch for grid arrays
	int tpitch = 0; // pitch of the transposed y-line factors
	// FP64
	double *so = nullptr, *x = nullptr, *b = nullptr, *r = nullptr, *sor = nullptr, *sory = nullptr, *ci = nullptr;
	// FP32 preconditioner copies
	float *so32 = nullptr, *x32 = nullptr, *b32 = nullptr, *r32 = nullptr, *sor32 = nullptr, *sory32 = nullptr,
	      *ci32 = nullptr;
	// fine level of the FP32 preconditioner (settings.fp64_fine_iterate): the
	// iterate from the interpolate-add on, in FP64, and the row-sum excess of
	// the operator (the difference form of its residual)
	double *xw = nullptr;
	bool ypk = false;  // the y-line factor arrays carry the packed couplings
	size_t ysize() const { return 2 * (size_t)tpitch * (nx + 2); }  // the two y factor planes
	float *dg32 = nullptr;
};

}  // namespace

struct cdr_gpu_solver {
	cdr_gpu_settings s{};
	std::vector<Level> lv;
	std::vector<void *> allocs;
	double *abd = nullptr;
	int *info = nullptr;
	double *norm = nullptr;     // device scalars
	double *partial = nullptr;  // norm scratch
	double *x64[2] = {nullptr, nullptr};
	// flexible CG: b, x, r, p (two buffers), q on the fine grid (FP64) and the scalars
	double *kb = nullptr, *kx[2] = {nullptr, nullptr}, *kr = nullptr, *kp[2] = {nullptr, nullptr}, *kq = nullptr;
	FcgScalars *ks = nullptr;
	double *kpart = nullptr;  // partial sums of the FCG kernels
	unsigned *ysync = nullptr;  // tickets and flags of the one-launch y-line sweeps (k2_lines.cu)
	double *ainv = nullptr;   // CDR_COARSE_INVERSE: inverse of the coarsest operator
	float *ainv32 = nullptr;
	// FCG iteration graphs: [0] FP64, [1] FP32 cycle; [.][0] residual updated, [.][1] formed
	cudaGraphExec_t kexec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
	long long klaunches[2][2] = {{0, 0}, {0, 0}};
	double *h_norm = nullptr;   // pinned host copy of the norm
	cudaStream_t st = nullptr;
	bool own_stream = false;
	int lc[2] = {-1, -1};  // first level of the fused coarse cycle, [0] FP64, [1] FP32 (-1: none)
	int per = 0;           // periodic directions (settings.periodic): bit 0 x, bit 1 y
	cudaGraphExec_t gexec[2] = {nullptr, nullptr};  // cycle graphs: [0] FP64, [1] FP32
	long long glaunches[2] = {0, 0};                 // kernel launches per replay
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;
	float setup_ms = 0.f, solve_ms = 0.f;
	bool wide = false;  // inside an FCG iteration with a widened fine-level iterate (lv[0].xw)
	// y-line factor arrays carry the packed couplings (pack_ylines_2d): y-line
	// relaxation without periodic directions, on levels whose y-lines have at
	// most 1024 points (K = 8 chunks; there the strided coupling loads, not
	// DRAM, bound the sweep; the longer lines of a fine level stream from DRAM
	// either way and run as fast unpacked)
	bool ypack = false;

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
	// the exact (sequential) line substitution applies to the FP64 cycle only;
	// CDR_LINES_NOTUNE to both
	template <typename T>
	int lflags() const
	{
		return sizeof(T) == 8 ? s.line_flags : (s.line_flags & (CDR_LINES_NOTUNE | CDR_LINES_STREAM));
	}
	int L() const { return (int)lv.size(); }

	// -------------------------------------------------------------- smoothing
	// zero: x is zero on entry (its interior may hold anything; the ghost ring
	// is zero): line sweeps start with CDR_LINES_ZERO_START, others clear x
	template <typename T>
	int smooth(int l, T *x, const T *b, int updown, bool zero = false);
	template <typename T>
	int ncycle(int l, T *x, const T *b, bool zero = false);
	template <typename T>
	int fused(int l0);
	template <typename T>
	int cycle(T *x, const T *b, bool zero = false);
	template <typename T>
	int coarse_solve(T *x, const T *b);
	template <typename T>
	int fcycle(int l, T *x, const T *b);
	template <typename T>
	int restrict_to(int l, T *rf);
	template <typename T>
	int interp_from(int l, T *x);
	int run_cycle(int prec);
	template <typename T>
	int fcg_iteration(bool formed);
	int run_fcg(int prec, bool formed);
	template <typename T>
	int tune_lines();
	int setup();
};

namespace {
template <typename T> struct Arr;
template <> struct Arr<double> {
	static double *so(Level &L) { return L.so; }
	static double *x(Level &L) { return L.x; }
	static double *b(Level &L) { return L.b; }
	static double *r(Level &L) { return L.r; }
	static double *sor(Level &L) { return L.sor; }
	static double *sory(Level &L) { return L.sory; }
	static double *ci(Level &L) { return L.ci; }
};
template <> struct Arr<float> {
	static float *so(Level &L) { return L.so32; }
	static float *x(Level &L) { return L.x32; }
	static float *b(Level &L) { return L.b32; }
	static float *r(Level &L) { return L.r32; }
	static float *sor(Level &L) { return L.sor32; }
	static float *sory(Level &L) { return L.sory32; }
	static float *ci(Level &L) { return L.ci32; }
};
}  // namespace

// multilevel::setup_relax_helper smoother closures (include/cedar/multilevel.h:160-222)
template <typename T>
int cdr_gpu_solver::smooth(int l, T *x, const T *b, int updown, bool zero)
{
	Level &L = lv[l];
	const int n = updown == CDR_DOWN ? s.nrelax_pre : s.nrelax_post;
	const T *so = Arr<T>::so(L), *sor = Arr<T>::sor(L), *sory = Arr<T>::sory(L);
	const bool lines = s.relaxation == CDR_RELAX_LINE_X || s.relaxation == CDR_RELAX_LINE_Y ||
	                   s.relaxation == CDR_RELAX_LINE_XY;
	if (zero && (n == 0 || !lines || per)) {  // only the line sweeps skip reading a zero iterate
		CDR_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(T) * L.d.plane(), st));
		zero = false;
	}
	const int yf = L.ypk ? CDR_LINES_YPACKED : 0;  // the packed couplings follow the y factors
	for (int it = 0; it < n; ++it) {
		// the first sweep of a zero iterate does not read it
		const int f = lflags<T>() | (zero && it == 0 ? CDR_LINES_ZERO_START : 0);
		switch (s.relaxation) {
		case CDR_RELAX_POINT: CDR_TRY(relax_point_2d<T>(so, L.ns, x, b, sor, L.d, updown, st, per)); break;
		case CDR_RELAX_LINE_X:
			CDR_TRY(relax_lines_2d<T>(so, L.ns, x, b, sor, L.d, L.tpitch, CDR_DIR_X, updown, f, st));
			break;
		case CDR_RELAX_LINE_Y:
			CDR_TRY(relax_lines_2d<T>(so, L.ns, x, b, sory, L.d, L.tpitch, CDR_DIR_Y, updown, f | yf, st, ysync));
			break;
		case CDR_RELAX_LINE_XY:
			if (updown == CDR_DOWN) {
				CDR_TRY(relax_lines_2d<T>(so, L.ns, x, b, sor, L.d, L.tpitch, CDR_DIR_X, updown, f, st));
				CDR_TRY(relax_lines_2d<T>(so, L.ns, x, b, sory, L.d, L.tpitch, CDR_DIR_Y, updown, lflags<T>() | yf, st,
				                          ysync));
			} else {
				CDR_TRY(relax_lines_2d<T>(so, L.ns, x, b, sory, L.d, L.tpitch, CDR_DIR_Y, updown, f | yf, st, ysync));
				CDR_TRY(relax_lines_2d<T>(so, L.ns, x, b, sor, L.d, L.tpitch, CDR_DIR_X, updown, lflags<T>(), st));
			}
			break;
		default: set_error(CDR_ERR_ARG, "unknown relaxation %d", s.relaxation); return CDR_ERR_ARG;
		}
	}
	return CDR_OK;
}

// cycle::vcycle::ncycle_helper (include/cedar/cycle/vcycle.h:57-115), n = 1
template <typename T>
int cdr_gpu_solver::ncycle(int l, T *x, const T *b, bool zero)
{
	Level &F = lv[l], &C = lv[l + 1];
	CDR_TRY(smooth<T>(l, x, b, CDR_DOWN, zero));
	CDR_TRY(residual_2d<T>(Arr<T>::so(F), F.ns, x, b, Arr<T>::r(F), F.d, nullptr, nullptr, st));
	if constexpr (sizeof(T) == 4) {
		if (l + 1 == s.fp32_levels) {  // FP32 -> FP64 hand-over: the coarse sub-cycle in FP64
			CDR_TRY(restrict_2d_mixed(C.ci, F.r32, C.b, F.d, C.d, st));
			CDR_CUDA_TRY(cudaMemsetAsync(C.x, 0, sizeof(double) * C.d.plane(), st));
			if (l + 1 == L() - 1) CDR_TRY(coarse_solve<double>(C.x, C.b));
			else if (l + 1 == lc[0]) CDR_TRY(fused<double>(l + 1));
			else CDR_TRY(ncycle<double>(l + 1, C.x, C.b));
			CDR_TRY(interp_add_2d_mixed(C.ci, C.x, F.r32, F.so32, x, F.d, C.d, st, F.ns));
			return smooth<T>(l, x, b, CDR_UP);
		}
	}
	CDR_TRY(restrict_to<T>(l, Arr<T>::r(F)));
	// coarse_x.set(0.0) (include/cedar/cycle/vcycle.h:79): the coarse cycle's
	// first sweep treats its iterate as zero without reading it
	const bool direct = l + 1 == L() - 1 || l + 1 == lc[sizeof(T) == 4];
	if (direct) CDR_CUDA_TRY(cudaMemsetAsync(Arr<T>::x(C), 0, sizeof(T) * C.d.plane(), st));
	if (l + 1 == L() - 1) CDR_TRY(coarse_solve<T>(Arr<T>::x(C), Arr<T>::b(C)));
	else if (l + 1 == lc[sizeof(T) == 4]) CDR_TRY(fused<T>(l + 1));
	else CDR_TRY(ncycle<T>(l + 1, Arr<T>::x(C), Arr<T>::b(C), true));
	if constexpr (sizeof(T) == 4) {
		if (l == 0 && wide) {
			// the fine level's iterate goes on in FP64, xw = x + P x_c + r/c; the
			// post-smoothing runs in FP32 on the correction from zero, with the
			// right-hand side b - A xw formed in FP64 over the difference form;
			// the cycle's output is xw + x (read by the FCG step as two parts)
			CDR_TRY(interp_add_2d_wide(C.ci32, C.x32, F.r32, F.so32, x, F.xw, F.d, C.d, st, F.ns));
			CDR_TRY(residual_2d_wide(F.so32, F.dg32, F.ns, F.xw, b, F.r32, nullptr, F.d, st));
			return smooth<T>(l, x, F.r32, CDR_UP, true);
		}
	}
	CDR_TRY(interp_from<T>(l, x));
	CDR_TRY(smooth<T>(l, x, b, CDR_UP));
	return CDR_OK;
}

// Restriction of a level-l grid function to level l+1's right-hand side.  The
// periodic branch (BMG2_SymStd_restrict.f90:94-130) first refreshes, in place,
// the ghost lines of each periodic direction whose fine size is even (the
// coarse grid then has Nf/2 + 1 points with its ghosts).
template <typename T>
int cdr_gpu_solver::restrict_to(int l, T *rf)
{
	Level &F = lv[l], &C = lv[l + 1];
	if (per) {
		const int xm = (per & 1) && F.nx % 2 == 0 ? 2 : 0, ym = (per & 2) && F.ny % 2 == 0 ? 1 : 0;
		CDR_TRY(ghost_copy_2d<T>(rf, F.d, 1, xm, ym, -1, st));
	}
	return restrict_2d<T>(Arr<T>::ci(C), rf, Arr<T>::b(C), F.d, C.d, st);
}

// x(l) += P x(l+1), then (periodic, BMG2_SymStd_interp_add.f90:139-156) the
// fine ghost lines.
template <typename T>
int cdr_gpu_solver::interp_from(int l, T *x)
{
	Level &F = lv[l], &C = lv[l + 1];
	CDR_TRY(interp_add_2d<T>(Arr<T>::ci(C), Arr<T>::x(C), Arr<T>::r(F), Arr<T>::so(F), x, F.d, C.d, st, F.ns));
	if (per) CDR_TRY(ghost_copy_2d<T>(x, F.d, 1, per & 1 ? 2 : 0, per & 2 ? 1 : 0, -1, st));
	return CDR_OK;
}

// Levels l0..L-1 in one launch (k2_coarse.cu); same operations as ncycle with
// the sequential line substitutions.
template <typename T>
CoarseCycle<T> coarse_desc(std::vector<Level> &lv, int l0, const cdr_gpu_settings &s);

template <typename T>
int cdr_gpu_solver::fused(int l0)
{
	CoarseCycle<T> cc = coarse_desc<T>(lv, l0, s);
	cc.abd = abd;
	return coarse_cycle<T>(cc, 1, st);
}

// Descriptor of the fused coarse cycle over levels l0..L-1
template <typename T>
CoarseCycle<T> coarse_desc(std::vector<Level> &lv, int l0, const cdr_gpu_settings &s)
{
	const int L = (int)lv.size();
	CoarseCycle<T> cc;
	cc.nl = L - l0;
	for (int l = l0; l < L; ++l) {
		Level &V = lv[l];
		CoarseLevel<T> &c = cc.lv[l - l0];
		c.so = Arr<T>::so(V);
		c.sor = Arr<T>::sor(V);
		c.sory = Arr<T>::sory(V);
		c.ci = Arr<T>::ci(V);
		c.x = Arr<T>::x(V);
		c.b = Arr<T>::b(V);
		c.r = Arr<T>::r(V);
		c.nx = V.nx;
		c.ny = V.ny;
		c.pitch = V.d.pitch;
		c.tpitch = V.tpitch;
		c.ns = V.ns;
	}
	cc.relax = s.relaxation;
	cc.npre = s.nrelax_pre;
	cc.npost = s.nrelax_post;
	return cc;
}

// First level (not the fine one) from which the fused coarse cycle runs: both
// edges at most fuse_coarse and the level's shared-memory copy within the limit.
template <typename T>
int pick_fused_level(std::vector<Level> &lv, const cdr_gpu_settings &s)
{
	const int L = (int)lv.size();
	if (s.fuse_coarse <= 0) return -1;
	for (int l = 1; l + 1 < L; ++l) {
		if (lv[l].nx > s.fuse_coarse || lv[l].ny > s.fuse_coarse || L - l > kMaxCoarseLevels) continue;
		if (coarse_cycle_bytes(coarse_desc<T>(lv, l, s)) <= kCoarseSmemMax) return l;
	}
	return -1;
}

template <typename T>
int cdr_gpu_solver::coarse_solve(T *x, const T *b)
{
	const Dims2 d = lv.back().d;
	if (per) {
		if constexpr (sizeof(T) == 8) return solve_cg_per_2d(abd, x, b, d, per, st);
		set_error(CDR_ERR_UNSUPPORTED, "periodic coarse solve in FP32");
		return CDR_ERR_UNSUPPORTED;
	}
	if (s.coarse_solve == CDR_COARSE_INVERSE) {
		if constexpr (sizeof(T) == 4) return solve_cg_inv_2d<float>(ainv32, x, b, d, st);
		else return solve_cg_inv_2d<double>(ainv, x, b, d, st);
	}
	return solve_cg_2d<T>(abd, x, b, d, st);
}

// cycle::fcycle::fmg_cycle / fmg_cycle_helper (include/cedar/cycle/fcycle.h:49-83)
template <typename T>
int cdr_gpu_solver::fcycle(int l, T *x, const T *b)
{
	if (l == L() - 1) return coarse_solve<T>(x, b);
	Level &F = lv[l], &C = lv[l + 1];
	// b is a level array (the solver's copy of the caller's right-hand side on
	// level 0): the periodic restriction refreshes its ghosts in place, as the
	// reference does
	CDR_TRY(restrict_to<T>(l, const_cast<T *>(b)));
	CDR_TRY(fcycle<T>(l + 1, Arr<T>::x(C), Arr<T>::b(C)));
	CDR_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(T) * F.d.plane(), st));
	CDR_CUDA_TRY(cudaMemsetAsync(Arr<T>::r(F), 0, sizeof(T) * F.d.plane(), st));
	CDR_TRY(interp_from<T>(l, x));
	return ncycle<T>(l, x, b);
}

template <typename T>
int cdr_gpu_solver::cycle(T *x, const T *b, bool zero)
{
	if (L() == 1) return coarse_solve<T>(x, b);
	if (s.cycle == CDR_CYCLE_F) return fcycle<T>(0, x, b);  // discards x
	return ncycle<T>(0, x, b, zero);
}

// One cycle on the level-0 work buffers, replayed from a CUDA graph when enabled.
int cdr_gpu_solver::run_cycle(int prec)
{
	auto body = [&]() -> int {
		if (prec == 0) return cycle<double>(lv[0].x, lv[0].b);
		return cycle<float>(lv[0].x32, lv[0].b32, true);  // the refinement's correction starts at zero
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

// One FCG iteration: the cycle on the preconditioner input (zero initial
// guess) and the three FCG kernels.
template <typename T>
int cdr_gpu_solver::fcg_iteration(bool formed)
{
	Level &F = lv[0];
	T *z = Arr<T>::x(F), *rin = Arr<T>::b(F);
	if constexpr (sizeof(T) == 4) {
		// every cycle starts from z = 0 without reading z (its first sweep treats
		// the iterate as zero), so the step leaves z as it is
		if (F.xw) {  // the cycle's output is F.xw + z
			wide = true;
			const int rc = cycle<T>(z, rin, true);
			wide = false;
			CDR_TRY(rc);
			return fcg_step<double, float>(F.so, F.ns, F.xw, z, rin, (float *)nullptr, kx[0], kx[1], kb, kr, kp[0],
			                               kp[1], kq, F.d, kpart, ks, st, formed);
		}
	}
	CDR_TRY(cycle<T>(z, rin, true));
	return fcg_step<T, T>(F.so, F.ns, z, nullptr, rin, (T *)nullptr, kx[0], kx[1], kb, kr, kp[0], kp[1], kq, F.d, kpart,
	                      ks, st, formed);
}

int cdr_gpu_solver::run_fcg(int prec, bool formed)
{
	auto body = [&]() -> int { return prec == 0 ? fcg_iteration<double>(formed) : fcg_iteration<float>(formed); };
	if (!s.use_graph) return body();
	cudaGraphExec_t &exec = kexec[prec][formed ? 1 : 0];
	long long &launches = klaunches[prec][formed ? 1 : 0];
	if (!exec) {
		cudaGraph_t g = nullptr;
		CDR_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
		const long long before = cdr_gpu_launch_count();
		int rc = body();
		launches = cdr_gpu_launch_count() - before;
		count_launches(-launches);  // captured, not launched
		cudaError_t e = cudaStreamEndCapture(st, &g);
		if (rc != CDR_OK) {
			if (g) cudaGraphDestroy(g);
			return rc;
		}
		if (e != cudaSuccess) {
			set_error(CDR_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
			return CDR_ERR_CUDA;
		}
		CDR_CUDA_TRY(cudaGraphInstantiate(&exec, g, 0));
		cudaGraphDestroy(g);
	}
	CDR_CUDA_TRY(cudaGraphLaunch(exec, st));
	count_launches(launches);
	return CDR_OK;
}

// Launch shapes of the line kernels of every level the cycle sweeps with them
// (all but the coarsest and the fused ones), timed on the levels' arrays.
template <typename T>
int cdr_gpu_solver::tune_lines()
{
	if (s.line_flags & CDR_LINES_NOTUNE) return CDR_OK;
	if (sizeof(T) == 8 && (s.line_flags & CDR_LINES_EXACT)) return CDR_OK;
	const bool lx = s.relaxation == CDR_RELAX_LINE_X || s.relaxation == CDR_RELAX_LINE_XY;
	const bool ly = s.relaxation == CDR_RELAX_LINE_Y || s.relaxation == CDR_RELAX_LINE_XY;
	const int f = lc[sizeof(T) == 4 ? 1 : 0];
	int lo = 0, stop = f >= 0 ? f : L() - 1;
	if (mixed() && s.fp32_levels > 0) {  // FP32 on the finest fp32_levels levels, FP64 below
		if (sizeof(T) == 4) stop = std::min(stop, s.fp32_levels);
		else lo = s.fp32_levels;
	}
	for (int l = lo; l < stop; ++l) {
		Level &F = lv[l];
		if (lx)
			CDR_TRY(lines_autotune<T>(Arr<T>::so(F), F.ns, Arr<T>::x(F), Arr<T>::b(F), Arr<T>::sor(F), F.d, F.tpitch,
			                          CDR_DIR_X, st));
		if (ly)
			CDR_TRY(lines_autotune<T>(Arr<T>::so(F), F.ns, Arr<T>::x(F), Arr<T>::b(F), Arr<T>::sory(F), F.d, F.tpitch,
			                          CDR_DIR_Y, st, ysync, F.ypk ? Arr<T>::sory(F) + F.ysize() : nullptr));
	}
	return CDR_OK;
}

// multilevel::setup (include/cedar/multilevel.h:243-265) on the device.
int cdr_gpu_solver::setup()
{
	for (int l = 0; l + 1 < L(); ++l) {
		Level &F = lv[l], &C = lv[l + 1];
		if (per) {
			// periodic branches: the interpolation's own walk, then the definite
			// product and the coarse operator's ghost lines
			// (BMG2_SymStd_SETUP_ITLI_ex.f90:216-247, 333-363)
			CDR_TRY(setup_interp_per_2d(F.so, F.ns, C.ci, F.d, C.d, per, st));
			CDR_TRY(galerkin_2d(F.so, F.ns, C.ci, C.so, F.d, C.d, st));
			CDR_TRY(ghost_copy_2d<double>(C.so, C.d, 5, per & 1 ? 2 : 0, per & 2 ? 1 : 0, -1, st));
		} else {
			CDR_TRY(setup_interp_2d(F.so, F.ns, C.ci, F.d, C.d, st));
			CDR_TRY(galerkin_2d(F.so, F.ns, C.ci, C.so, F.d, C.d, st));
		}
		// smoother setup (multilevel::setup_relax_helper, multilevel.h:134-158)
		switch (s.relaxation) {
		case CDR_RELAX_POINT: CDR_TRY(setup_recip_2d<double>(F.so, F.sor, F.d, st)); break;
		case CDR_RELAX_LINE_X:
			CDR_TRY(setup_lines_2d<double>(F.so, F.ns, F.sor, F.d, F.tpitch, CDR_DIR_X, info, st));
			break;
		case CDR_RELAX_LINE_Y:
			CDR_TRY(setup_lines_2d<double>(F.so, F.ns, F.sory, F.d, F.tpitch, CDR_DIR_Y, info, st));
			break;
		case CDR_RELAX_LINE_XY:
			CDR_TRY(setup_lines_2d<double>(F.so, F.ns, F.sor, F.d, F.tpitch, CDR_DIR_X, info, st));
			CDR_TRY(setup_lines_2d<double>(F.so, F.ns, F.sory, F.d, F.tpitch, CDR_DIR_Y, info, st));
			break;
		}
		if (F.ypk) CDR_TRY(pack_ylines_2d<double>(F.so, F.ns, F.sory + F.ysize(), F.d, F.tpitch, st));
	}
	Level &Cg = lv[L() - 1];
	if (per) CDR_TRY(setup_cg_per_2d(Cg.so, Cg.ns, Cg.d, abd, info + 1, per, st));
	else CDR_TRY(setup_cg_2d(Cg.so, Cg.ns, Cg.d, abd, info + 1, st));
	if (s.coarse_solve == CDR_COARSE_INVERSE) {
		CDR_TRY(cg_inverse_2d(abd, Cg.d, ainv, st));
		if (mixed()) CDR_TRY(convert_f64_f32(ainv, ainv32, (size_t)Cg.nx * Cg.ny * Cg.nx * Cg.ny, st));
	}
	if (mixed()) {
		for (int l = 0; l < L(); ++l) {
			Level &F = lv[l];
			CDR_TRY(convert_f64_f32(F.so, F.so32, F.d.plane() * F.ns, st));
			if (F.dg32) CDR_TRY(rowsum_excess_2d(F.so, F.ns, F.dg32, F.d, st));
			if (l > 0) CDR_TRY(convert_f64_f32(F.ci, F.ci32, F.d.plane() * 8, st));
			if (l + 1 == L()) continue;
			switch (s.relaxation) {
			case CDR_RELAX_POINT: CDR_TRY(convert_f64_f32(F.sor, F.sor32, F.d.plane(), st)); break;
			case CDR_RELAX_LINE_X:
				CDR_TRY(setup_lines_2d<float>(F.so, F.ns, F.sor32, F.d, F.tpitch, CDR_DIR_X, info, st));
				break;
			case CDR_RELAX_LINE_Y:
				CDR_TRY(setup_lines_2d<float>(F.so, F.ns, F.sory32, F.d, F.tpitch, CDR_DIR_Y, info, st));
				break;
			case CDR_RELAX_LINE_XY:
				CDR_TRY(setup_lines_2d<float>(F.so, F.ns, F.sor32, F.d, F.tpitch, CDR_DIR_X, info, st));
				CDR_TRY(setup_lines_2d<float>(F.so, F.ns, F.sory32, F.d, F.tpitch, CDR_DIR_Y, info, st));
				break;
			}
			if (F.ypk) CDR_TRY(pack_ylines_2d<float>(F.so32, F.ns, F.sory32 + F.ysize(), F.d, F.tpitch, st));
		}
	}
	int hinfo[2] = {0, 0};
	CDR_CUDA_TRY(cudaMemcpyAsync(hinfo, info, sizeof(hinfo), cudaMemcpyDeviceToHost, st));
	CDR_CUDA_TRY(cudaStreamSynchronize(st));
	if (hinfo[0]) {
		set_error(CDR_ERR_SETUP, "line factorization: non-positive pivot in line %d", hinfo[0]);
		return CDR_ERR_SETUP;
	}
	if (hinfo[1]) {
		set_error(CDR_ERR_SETUP, "coarse-grid Cholesky failed at column %d", hinfo[1]);
		return CDR_ERR_SETUP;
	}
	return CDR_OK;
}

// cdr2::solver::compute_num_levels (include/cedar/2d/solver.h:63-79)
static int num_levels(int nx, int ny, int min_coarse)
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

extern "C" {

int cdr_gpu_settings_default(cdr_gpu_settings *s)
{
	if (!s) return CDR_ERR_ARG;
	// defaults of ml_settings::init (src/multilevel_settings.cc:15-61)
	s->relaxation = CDR_RELAX_POINT;
	s->nrelax_pre = 2;
	s->nrelax_post = 1;
	s->num_levels = -1;
	s->maxiter = 10;
	s->tol = 1e-8;
	s->min_coarse = 3;
	s->precision = CDR_PREC_F64;
	s->use_graph = 1;
	s->line_flags = 0;
	s->fuse_coarse = 32;
	s->krylov = CDR_KRYLOV_NONE;
	s->coarse_solve = CDR_COARSE_BANDED;
	s->fp32_levels = 0;
	s->cycle = CDR_CYCLE_V;
	s->krylov_replace = 1;
	s->periodic = 0;
	s->fp64_fine_iterate = 1;
	return CDR_OK;
}

int cdr_gpu_solver_destroy(cdr_gpu_solver *h)
{
	if (!h) return CDR_ERR_HANDLE;
	if (h->st) cudaStreamSynchronize(h->st);
	for (auto &g : h->gexec)
		if (g) cudaGraphExecDestroy(g);
	for (auto &gp : h->kexec)
		for (auto &g : gp)
			if (g) cudaGraphExecDestroy(g);
	for (void *p : h->allocs) cudaFree(p);
	if (h->h_norm) cudaFreeHost(h->h_norm);
	if (h->ev0) cudaEventDestroy(h->ev0);
	if (h->ev1) cudaEventDestroy(h->ev1);
	if (h->own_stream && h->st) cudaStreamDestroy(h->st);
	delete h;
	return CDR_OK;
}

static int load_and_setup(cdr_gpu_solver *h, const double *so, int src_pitch, cudaMemcpyKind kind)
{
	Level &F = h->lv[0];
	CDR_CUDA_TRY(cudaMemcpy2DAsync(F.so, F.d.pitch * sizeof(double), so, src_pitch * sizeof(double),
	                               (F.nx + 2) * sizeof(double), (size_t)(F.ny + 2) * F.ns, kind, h->st));
	CDR_CUDA_TRY(cudaEventRecord(h->ev0, h->st));
	CDR_TRY(h->setup());
	CDR_CUDA_TRY(cudaEventRecord(h->ev1, h->st));
	CDR_CUDA_TRY(cudaEventSynchronize(h->ev1));
	CDR_CUDA_TRY(cudaEventElapsedTime(&h->setup_ms, h->ev0, h->ev1));
	// launch shapes of the line kernels (once per shape and process; the sweeps
	// run on the level arrays, which the solve reloads or overwrites)
	if (!h->mixed()) return h->tune_lines<double>();
	CDR_TRY(h->tune_lines<float>());
	return h->s.fp32_levels > 0 ? h->tune_lines<double>() : CDR_OK;
}

static int create_impl(cdr_gpu_solver *h, const double *so_src, int ns, int nx, int ny, int src_pitch,
                       cudaMemcpyKind kind)
{
	const cdr_gpu_settings &s = h->s;
	int nl = num_levels(nx, ny, s.min_coarse);
	if (s.num_levels > 0) {
		if (s.num_levels > nl) {
			set_error(CDR_ERR_ARG, "too many levels specified (%d > %d)", s.num_levels, nl);
			return CDR_ERR_ARG;
		}
		nl = s.num_levels;
	}
	h->lv.resize(nl);
	h->ypack = (s.relaxation == CDR_RELAX_LINE_Y || s.relaxation == CDR_RELAX_LINE_XY) && s.periodic == 0;
	for (int l = 0; l < nl; ++l) {
		Level &L = h->lv[l];
		if (l == 0) { L.nx = nx; L.ny = ny; L.ns = ns; }
		else {
			// cdr2::solver::setup_space (include/cedar/2d/solver.h:93-94)
			L.nx = (int)((h->lv[l - 1].nx - 1) / 2. + 1);
			L.ny = (int)((h->lv[l - 1].ny - 1) / 2. + 1);
			L.ns = 5;
		}
		L.d = Dims2{L.nx, L.ny, round_up(L.nx + 2, 32)};
		L.tpitch = round_up(L.ny + 2, 32);
		const size_t pl = L.d.plane();
		const size_t tpl = (size_t)L.tpitch * (L.nx + 2);
		CDR_TRY(h->alloc(&L.so, pl * L.ns));
		CDR_TRY(h->alloc(&L.x, pl));
		CDR_TRY(h->alloc(&L.b, pl));
		CDR_TRY(h->alloc(&L.r, pl));
		if (l > 0) CDR_TRY(h->alloc(&L.ci, pl * 8));
		L.ypk = h->ypack && l + 1 < nl && L.ny <= 1024;
		const int ypl = 2 + (L.ypk ? ypack_planes(L.ns) : 0);  // factors [+ packed couplings]
		if (l + 1 < nl) {
			CDR_TRY(h->alloc(&L.sor, pl * 2));
			CDR_TRY(h->alloc(&L.sory, tpl * ypl));
		}
		if (h->mixed()) {
			CDR_TRY(h->alloc(&L.so32, pl * L.ns));
			CDR_TRY(h->alloc(&L.x32, pl));
			CDR_TRY(h->alloc(&L.b32, pl));
			CDR_TRY(h->alloc(&L.r32, pl));
			if (l > 0) CDR_TRY(h->alloc(&L.ci32, pl * 8));
			if (l + 1 < nl) {
				CDR_TRY(h->alloc(&L.sor32, pl * 2));
				CDR_TRY(h->alloc(&L.sory32, tpl * ypl));
			}
		}
	}
	// the fused coarse cycle takes over from the first level that fits (not the
	// fine level, whose arrays the caller may pass), when it spans two levels or more
	h->per = s.periodic;
	// the fused coarse cycle has no periodic branches
	h->lc[0] = h->per ? -1 : pick_fused_level<double>(h->lv, s);
	h->lc[1] = h->per ? -1 : pick_fused_level<float>(h->lv, s);
	// FCG around the FP32 cycle: the fine level's iterate from the
	// interpolate-add on in FP64 (the preconditioner's output), when level 1 is
	// an FP32 level
	{
		Level &F0 = h->lv[0];
		if (h->mixed() && s.krylov == CDR_KRYLOV_FCG && s.fp64_fine_iterate && !h->per && nl >= 2 &&
		    s.fp32_levels != 1) {
			CDR_TRY(h->alloc(&F0.xw, F0.d.plane()));
			CDR_TRY(h->alloc(&F0.dg32, F0.d.plane()));
		}
	}
	Level &Cg = h->lv[nl - 1];
	if ((size_t)Cg.nx * Cg.ny > 4096) {
		set_error(CDR_ERR_DIM, "coarsest grid %dx%d too large for the %s Cholesky", Cg.nx, Cg.ny,
		          h->per ? "dense" : "banded");
		return CDR_ERR_DIM;
	}
	// periodic: a dense N x N factor (include/cedar/2d/solver.h:118-121)
	const size_t ncg = (size_t)Cg.nx * Cg.ny;
	CDR_TRY(h->alloc(&h->abd, h->per ? ncg * ncg : (size_t)(Cg.nx + 2) * ncg));
	if (s.coarse_solve == CDR_COARSE_INVERSE) {
		const size_t nn = (size_t)Cg.nx * Cg.ny * Cg.nx * Cg.ny;
		CDR_TRY(h->alloc(&h->ainv, nn));
		if (h->mixed()) CDR_TRY(h->alloc(&h->ainv32, nn));
	}
	CDR_TRY(h->alloc(&h->info, 2));
	CDR_TRY(h->alloc(&h->norm, 4));
	CDR_TRY(h->alloc(&h->ysync, lines_sync_words(h->lv[0].d)));
	CDR_TRY(h->alloc(&h->partial, kNormScratchBytes / sizeof(double)));
	if (h->mixed()) {
		CDR_TRY(h->alloc(&h->x64[0], h->lv[0].d.plane()));
		CDR_TRY(h->alloc(&h->x64[1], h->lv[0].d.plane()));
	}
	if (s.krylov == CDR_KRYLOV_FCG) {
		const size_t pl = h->lv[0].d.plane();
		for (double **p : {&h->kb, &h->kx[0], &h->kx[1], &h->kr, &h->kp[0], &h->kp[1], &h->kq}) CDR_TRY(h->alloc(p, pl));
		CDR_TRY(h->alloc(&h->ks, 1));
		CDR_TRY(h->alloc(&h->kpart, fcg_scratch_doubles(h->lv[0].d)));
	}
	CDR_CUDA_TRY(cudaMallocHost(&h->h_norm, 4 * sizeof(double)));
	// fine operator (source pitch) -> device pitch, then the device setup
	return load_and_setup(h, so_src, src_pitch, kind);
}

static int create_any(const cdr_gpu_settings *s, const double *so_src, int ns, int nx, int ny, int src_pitch,
                      cudaMemcpyKind kind, cudaStream_t stream, cdr_gpu_solver **out)
{
	if (!s || !so_src || !out) { set_error(CDR_ERR_ARG, "null argument"); return CDR_ERR_ARG; }
	if (ns != 3 && ns != 5) { set_error(CDR_ERR_ARG, "nstencil must be 3 or 5"); return CDR_ERR_ARG; }
	if (nx < 1 || ny < 1) { set_error(CDR_ERR_DIM, "bad grid %dx%d", nx, ny); return CDR_ERR_DIM; }
	if (s->relaxation < CDR_RELAX_POINT || s->relaxation > CDR_RELAX_LINE_XY) {
		set_error(CDR_ERR_ARG, "invalid relaxation %d", s->relaxation);
		return CDR_ERR_ARG;
	}
	if (s->precision != CDR_PREC_F64 && s->precision != CDR_PREC_F32_IR) {
		set_error(CDR_ERR_ARG, "invalid precision %d", s->precision);
		return CDR_ERR_ARG;
	}
	if (s->krylov != CDR_KRYLOV_NONE && s->krylov != CDR_KRYLOV_FCG) {
		set_error(CDR_ERR_ARG, "invalid krylov %d", s->krylov);
		return CDR_ERR_ARG;
	}
	if (s->coarse_solve != CDR_COARSE_BANDED && s->coarse_solve != CDR_COARSE_INVERSE) {
		set_error(CDR_ERR_ARG, "invalid coarse_solve %d", s->coarse_solve);
		return CDR_ERR_ARG;
	}
	if (s->fp32_levels < 0) {
		set_error(CDR_ERR_ARG, "invalid fp32_levels %d", s->fp32_levels);
		return CDR_ERR_ARG;
	}
	if (s->cycle != CDR_CYCLE_V && s->cycle != CDR_CYCLE_F) {
		set_error(CDR_ERR_ARG, "invalid cycle type %d", s->cycle);
		return CDR_ERR_ARG;
	}
	if (s->krylov_replace < 0) {
		set_error(CDR_ERR_ARG, "invalid krylov_replace %d", s->krylov_replace);
		return CDR_ERR_ARG;
	}
	if (s->fp64_fine_iterate != 0 && s->fp64_fine_iterate != 1) {
		set_error(CDR_ERR_ARG, "invalid fp64_fine_iterate %d (0 or 1)", s->fp64_fine_iterate);
		return CDR_ERR_ARG;
	}
	if (s->periodic & ~3) {
		set_error(CDR_ERR_ARG, "invalid periodic mask %d (bit 0 x, bit 1 y)", s->periodic);
		return CDR_ERR_ARG;
	}
	if (s->periodic && (s->relaxation != CDR_RELAX_POINT || s->precision != CDR_PREC_F64 ||
	                    s->krylov != CDR_KRYLOV_NONE || s->coarse_solve != CDR_COARSE_BANDED)) {
		set_error(CDR_ERR_UNSUPPORTED, "periodic boundaries: FP64 point relaxation and the direct coarse solve only");
		return CDR_ERR_UNSUPPORTED;
	}
	*out = nullptr;
	cdr_gpu_solver *h = new cdr_gpu_solver();
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
	int rc = lines_prepare();
	if (rc == CDR_OK) rc = create_impl(h, so_src, ns, nx, ny, src_pitch, kind);
	if (rc != CDR_OK) {
		cdr_gpu_solver_destroy(h);
		return rc;
	}
	*out = h;
	return CDR_OK;
}

int cdr_gpu_solver_create_2d(const cdr_gpu_settings *s, const double *so_host, int ns, int nx, int ny,
                             cudaStream_t stream, cdr_gpu_solver **out)
{
	return create_any(s, so_host, ns, nx, ny, nx + 2, cudaMemcpyHostToDevice, stream, out);
}

int cdr_gpu_solver_create_2d_device(const cdr_gpu_settings *s, const double *so_dev, int ns, int nx, int ny,
                                    int pitch, cudaStream_t stream, cdr_gpu_solver **out)
{
	if (pitch < nx + 2) { set_error(CDR_ERR_DIM, "pitch %d < nx+2", pitch); return CDR_ERR_DIM; }
	return create_any(s, so_dev, ns, nx, ny, pitch, cudaMemcpyDeviceToDevice, stream, out);
}

int cdr_gpu_solver_resetup_device(cdr_gpu_solver *h, const double *so_dev, int pitch)
{
	if (!h) { set_error(CDR_ERR_HANDLE, "null solver"); return CDR_ERR_HANDLE; }
	if (!so_dev) { set_error(CDR_ERR_ARG, "null operator"); return CDR_ERR_ARG; }
	if (pitch < h->lv[0].nx + 2) { set_error(CDR_ERR_DIM, "pitch %d < nx+2", pitch); return CDR_ERR_DIM; }
	return load_and_setup(h, so_dev, pitch, cudaMemcpyDeviceToDevice);
}

// Flexible CG on the level-0 buffers (x in F.x, b in F.b on entry, x out in
// F.x); the residual of every iteration is the true one, so the stopping test
// is the reference's (|b - A x| / |b - A x0| < tol).
static int solve_fcg(cdr_gpu_solver *h, int *iters, double *hist, int maxhist)
{
	Level &F = h->lv[0];
	cudaStream_t st = h->st;
	const int prec = h->mixed() ? 1 : 0;
	const size_t bytes = sizeof(double) * F.d.plane();
	CDR_CUDA_TRY(cudaMemcpyAsync(h->kb, F.b, bytes, cudaMemcpyDeviceToDevice, st));
	CDR_CUDA_TRY(cudaMemcpyAsync(h->kx[0], F.x, bytes, cudaMemcpyDeviceToDevice, st));
	CDR_TRY(residual_2d<double>(F.so, F.ns, h->kx[0], h->kb, h->kr, F.d, h->norm, h->partial, st));
	CDR_CUDA_TRY(cudaMemcpyAsync(h->h_norm, h->norm, sizeof(double), cudaMemcpyDeviceToHost, st));
	CDR_CUDA_TRY(cudaStreamSynchronize(st));
	const double res0 = h->h_norm[0];
	int it = 0;
	if (res0 > 0) {
		if (prec) CDR_TRY(fcg_load<float>(h->kr, F.b32, F.x32, F.d, h->ks, st));
		else CDR_TRY(fcg_load<double>(h->kr, F.b, F.x, F.d, h->ks, st));
		// the residual is formed (b - A x) every m-th iteration, updated in between
		const int m = h->s.krylov_replace > 1 ? h->s.krylov_replace : 1;
		while (it < h->s.maxiter) {
			const bool formed = (it + 1) % m == 0;
			CDR_TRY(h->run_fcg(prec, formed));
			CDR_CUDA_TRY(cudaMemcpyAsync(h->h_norm, &h->ks->rr, sizeof(double), cudaMemcpyDeviceToHost, st));
			CDR_CUDA_TRY(cudaStreamSynchronize(st));
			double rel = std::sqrt(h->h_norm[0]) / res0;
			++it;
			if (std::isfinite(rel) && rel < h->s.tol && !formed) {
				// an updated residual met the tolerance: form b - A x of the iterate
				// (in kx[it & 1]); stop only if that meets it too, else go on from it
				CDR_TRY(residual_2d<double>(F.so, F.ns, h->kx[it & 1], h->kb, h->kr, F.d, h->norm, h->partial, st));
				CDR_CUDA_TRY(cudaMemcpyAsync(h->h_norm, h->norm, sizeof(double), cudaMemcpyDeviceToHost, st));
				CDR_CUDA_TRY(cudaStreamSynchronize(st));
				rel = h->h_norm[0] / res0;
				if (rel >= h->s.tol && std::isfinite(rel)) {
					if (prec) CDR_TRY(fcg_load<float>(h->kr, F.b32, F.x32, F.d, h->ks, st, false));
					else CDR_TRY(fcg_load<double>(h->kr, F.b, F.x, F.d, h->ks, st, false));
				}
			}
			if (hist && it - 1 < maxhist) hist[it - 1] = rel;
			if (!std::isfinite(rel)) {
				set_error(CDR_ERR_NUMERIC, "non-finite residual norm at iteration %d", it - 1);
				return CDR_ERR_NUMERIC;
			}
			if (rel < h->s.tol) break;
		}
	}
	// iterate of step it is in kx[it & 1] (FcgScalars::iter counts the same steps)
	CDR_CUDA_TRY(cudaMemcpyAsync(F.x, h->kx[it & 1], bytes, cudaMemcpyDeviceToDevice, st));
	if (iters) *iters = it;
	return CDR_OK;
}

// multilevel::solve (include/cedar/multilevel.h:278-298) on the level-0 buffers.
static int solve_loaded(cdr_gpu_solver *h, int *iters, double *hist, int maxhist)
{
	Level &F = h->lv[0];
	cudaStream_t st = h->st;
	double res0 = 0;
	int it = 0;
	CDR_CUDA_TRY(cudaEventRecord(h->ev0, st));
	if (h->s.krylov == CDR_KRYLOV_FCG) {
		CDR_TRY(solve_fcg(h, &it, hist, maxhist));
	} else if (!h->mixed()) {
		CDR_TRY(residual_2d<double>(F.so, F.ns, F.x, F.b, F.r, F.d, h->norm, h->partial, st));
		CDR_CUDA_TRY(cudaMemcpyAsync(h->h_norm, h->norm, sizeof(double), cudaMemcpyDeviceToHost, st));
		CDR_CUDA_TRY(cudaStreamSynchronize(st));
		res0 = h->h_norm[0];
		for (it = 0; it < h->s.maxiter;) {
			CDR_TRY(h->run_cycle(0));
			CDR_TRY(residual_2d<double>(F.so, F.ns, F.x, F.b, F.r, F.d, h->norm, h->partial, st));
			CDR_CUDA_TRY(cudaMemcpyAsync(h->h_norm, h->norm, sizeof(double), cudaMemcpyDeviceToHost, st));
			CDR_CUDA_TRY(cudaStreamSynchronize(st));
			double rel = h->h_norm[0] / res0;
			if (hist && it < maxhist) hist[it] = rel;
			++it;
			if (!std::isfinite(rel)) {
				set_error(CDR_ERR_NUMERIC, "non-finite residual norm at iteration %d", it - 1);
				return CDR_ERR_NUMERIC;
			}
			if (rel < h->s.tol) break;
		}
	} else {
		// x64[0] = x; r = b - A x (FP64), r32 -> level-0 FP32 right-hand side
		int cur = 0;
		CDR_CUDA_TRY(cudaMemcpyAsync(h->x64[0], F.x, sizeof(double) * F.d.plane(), cudaMemcpyDeviceToDevice, st));
		CDR_TRY(ir_residual_2d(F.so, F.ns, h->x64[0], F.x32, F.b, h->x64[1], F.b32, F.d, F.d, h->norm, h->partial, 0,
		                       st));
		CDR_CUDA_TRY(cudaMemcpyAsync(h->h_norm, h->norm, sizeof(double), cudaMemcpyDeviceToHost, st));
		CDR_CUDA_TRY(cudaStreamSynchronize(st));
		res0 = h->h_norm[0];
		for (it = 0; it < h->s.maxiter;) {
			CDR_TRY(h->run_cycle(1));  // the correction F.x32 from zero
			CDR_TRY(ir_residual_2d(F.so, F.ns, h->x64[cur], F.x32, F.b, h->x64[1 - cur], F.b32, F.d, F.d, h->norm,
			                       h->partial, 1, st));
			cur = 1 - cur;
			CDR_CUDA_TRY(cudaMemcpyAsync(h->h_norm, h->norm, sizeof(double), cudaMemcpyDeviceToHost, st));
			CDR_CUDA_TRY(cudaStreamSynchronize(st));
			double rel = h->h_norm[0] / res0;
			if (hist && it < maxhist) hist[it] = rel;
			++it;
			if (!std::isfinite(rel)) {
				set_error(CDR_ERR_NUMERIC, "non-finite residual norm at iteration %d", it - 1);
				return CDR_ERR_NUMERIC;
			}
			if (rel < h->s.tol) break;
		}
		CDR_CUDA_TRY(cudaMemcpyAsync(F.x, h->x64[cur], sizeof(double) * F.d.plane(), cudaMemcpyDeviceToDevice, st));
	}
	CDR_CUDA_TRY(cudaEventRecord(h->ev1, st));
	CDR_CUDA_TRY(cudaEventSynchronize(h->ev1));
	CDR_CUDA_TRY(cudaEventElapsedTime(&h->solve_ms, h->ev0, h->ev1));
	if (iters) *iters = it;
	// both give-up counts are read (and reset) before either is reported
	unsigned to_lines = 0, to_inv = 0;
	CDR_TRY(lines_stream_timeouts(st, &to_lines));
	if (h->s.coarse_solve == CDR_COARSE_INVERSE) CDR_TRY(cg_inv_timeouts(st, &to_inv));
	if (to_lines || to_inv) {
		// a y-line block that gave up left its flags set: clear them for the next solve
		CDR_CUDA_TRY(cudaMemsetAsync(h->ysync, 0, sizeof(unsigned) * lines_sync_words(F.d), st));
		CDR_CUDA_TRY(cudaStreamSynchronize(st));
		set_error(CDR_ERR_NUMERIC, "%u line-sweep CTAs and %u inverse-product CTAs gave up waiting for their rows",
		          to_lines, to_inv);
		return CDR_ERR_NUMERIC;
	}
	return CDR_OK;
}

int cdr_gpu_solver_solve(cdr_gpu_solver *h, const double *b_host, double *x_host, int *iters, double *hist,
                         int maxhist)
{
	if (!h) { set_error(CDR_ERR_HANDLE, "null solver"); return CDR_ERR_HANDLE; }
	if (!b_host || !x_host) { set_error(CDR_ERR_ARG, "null buffer"); return CDR_ERR_ARG; }
	Level &F = h->lv[0];
	const size_t w = (F.nx + 2) * sizeof(double);
	CDR_CUDA_TRY(cudaMemcpy2DAsync(F.b, F.d.pitch * sizeof(double), b_host, w, w, F.ny + 2, cudaMemcpyHostToDevice,
	                               h->st));
	CDR_CUDA_TRY(cudaMemcpy2DAsync(F.x, F.d.pitch * sizeof(double), x_host, w, w, F.ny + 2, cudaMemcpyHostToDevice,
	                               h->st));
	CDR_TRY(solve_loaded(h, iters, hist, maxhist));
	CDR_CUDA_TRY(cudaMemcpy2DAsync(x_host, w, F.x, F.d.pitch * sizeof(double), w, F.ny + 2, cudaMemcpyDeviceToHost,
	                               h->st));
	CDR_CUDA_TRY(cudaStreamSynchronize(h->st));
	return CDR_OK;
}

int cdr_gpu_solver_solve_device(cdr_gpu_solver *h, const double *b_dev, double *x_dev, int pitch, int *iters,
                                double *hist, int maxhist)
{
	if (!h) { set_error(CDR_ERR_HANDLE, "null solver"); return CDR_ERR_HANDLE; }
	if (!b_dev || !x_dev) { set_error(CDR_ERR_ARG, "null buffer"); return CDR_ERR_ARG; }
	Level &F = h->lv[0];
	if (pitch < F.nx + 2) { set_error(CDR_ERR_DIM, "pitch %d < nx+2", pitch); return CDR_ERR_DIM; }
	const size_t w = (F.nx + 2) * sizeof(double);
	CDR_CUDA_TRY(cudaMemcpy2DAsync(F.b, F.d.pitch * sizeof(double), b_dev, pitch * sizeof(double), w, F.ny + 2,
	                               cudaMemcpyDeviceToDevice, h->st));
	CDR_CUDA_TRY(cudaMemcpy2DAsync(F.x, F.d.pitch * sizeof(double), x_dev, pitch * sizeof(double), w, F.ny + 2,
	                               cudaMemcpyDeviceToDevice, h->st));
	CDR_TRY(solve_loaded(h, iters, hist, maxhist));
	CDR_CUDA_TRY(cudaMemcpy2DAsync(x_dev, pitch * sizeof(double), F.x, F.d.pitch * sizeof(double), w, F.ny + 2,
	                               cudaMemcpyDeviceToDevice, h->st));
	CDR_CUDA_TRY(cudaStreamSynchronize(h->st));
	return CDR_OK;
}

int cdr_gpu_solver_vcycle_device(cdr_gpu_solver *h, const double *b_dev, double *x_dev, int pitch)
{
	if (!h) { set_error(CDR_ERR_HANDLE, "null solver"); return CDR_ERR_HANDLE; }
	if (!b_dev || !x_dev) { set_error(CDR_ERR_ARG, "null buffer"); return CDR_ERR_ARG; }
	Level &F = h->lv[0];
	if (pitch < F.nx + 2) { set_error(CDR_ERR_DIM, "pitch %d < nx+2", pitch); return CDR_ERR_DIM; }
	const size_t w = (F.nx + 2) * sizeof(double);
	CDR_CUDA_TRY(cudaMemcpy2DAsync(F.b, F.d.pitch * sizeof(double), b_dev, pitch * sizeof(double), w, F.ny + 2,
	                               cudaMemcpyDeviceToDevice, h->st));
	CDR_CUDA_TRY(cudaMemcpy2DAsync(F.x, F.d.pitch * sizeof(double), x_dev, pitch * sizeof(double), w, F.ny + 2,
	                               cudaMemcpyDeviceToDevice, h->st));
	CDR_TRY(h->run_cycle(0));
	CDR_CUDA_TRY(cudaMemcpy2DAsync(x_dev, pitch * sizeof(double), F.x, F.d.pitch * sizeof(double), w, F.ny + 2,
	                               cudaMemcpyDeviceToDevice, h->st));
	CDR_CUDA_TRY(cudaStreamSynchronize(h->st));
	return CDR_OK;
}

int cdr_gpu_solver_nlevels(const cdr_gpu_solver *h) { return h ? (int)h->lv.size() : -1; }

int cdr_gpu_solver_level(const cdr_gpu_solver *h, int level, int which, void **ptr, int *nx, int *ny, int *pitch,
                         int *tpitch, int *nstencil)
{
	if (!h) { set_error(CDR_ERR_HANDLE, "null solver"); return CDR_ERR_HANDLE; }
	if (level < 0 || level >= (int)h->lv.size()) { set_error(CDR_ERR_ARG, "bad level %d", level); return CDR_ERR_ARG; }
	const Level &L = h->lv[level];
	void *p = nullptr;
	switch (which) {
	case 0: p = L.so; break;
	case 1: p = L.x; break;
	case 2: p = L.b; break;
	case 3: p = L.r; break;
	case 4: p = L.sor; break;
	case 5: p = L.sory; break;
	case 6: p = L.ci; break;
	case 16: p = L.so32; break;
	case 17: p = L.x32; break;
	case 18: p = L.b32; break;
	case 19: p = L.r32; break;
	case 20: p = L.sor32; break;
	case 21: p = L.sory32; break;
	case 22: p = L.ci32; break;
	case 100: p = h->abd; break;
	default: set_error(CDR_ERR_ARG, "bad array id %d", which); return CDR_ERR_ARG;
	}
	if (ptr) *ptr = p;
	if (nx) *nx = L.nx;
	if (ny) *ny = L.ny;
	if (pitch) *pitch = L.d.pitch;
	if (tpitch) *tpitch = L.tpitch;
	if (nstencil) *nstencil = L.ns;
	return CDR_OK;
}

int cdr_gpu_solver_level_get(const cdr_gpu_solver *h, int level, int which, void *host, size_t bytes)
{
	void *p = nullptr;
	int nx, ny, pitch, tpitch, ns;
	CDR_TRY(cdr_gpu_solver_level(h, level, which, &p, &nx, &ny, &pitch, &tpitch, &ns));
	if (!p) { set_error(CDR_ERR_ARG, "array %d not allocated on level %d", which, level); return CDR_ERR_ARG; }
	const int w = which & 15;
	const size_t elem = which >= 16 && which < 100 ? sizeof(float) : sizeof(double);
	size_t n;
	if (which == 100) n = (size_t)(nx + 2) * nx * ny;
	else if (w == 5) n = (size_t)2 * tpitch * (nx + 2);
	else n = (size_t)(w == 0 ? ns : w == 4 ? 2 : w == 6 ? 8 : 1) * pitch * (ny + 2);
	if (!host || bytes < n * elem) { set_error(CDR_ERR_ARG, "host buffer too small (%zu < %zu)", bytes, n * elem); return CDR_ERR_ARG; }
	CDR_CUDA_TRY(cudaMemcpyAsync(host, p, n * elem, cudaMemcpyDeviceToHost, h->st));
	CDR_CUDA_TRY(cudaStreamSynchronize(h->st));
	return CDR_OK;
}

int cdr_gpu_solver_timings(const cdr_gpu_solver *h, double *setup_ms, double *solve_ms)
{
	if (!h) return CDR_ERR_HANDLE;
	if (setup_ms) *setup_ms = h->setup_ms;
	if (solve_ms) *solve_ms = h->solve_ms;
	return CDR_OK;
}

}  // extern "C"
