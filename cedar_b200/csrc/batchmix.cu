// batchmix.cu -- independent 2D problems of several grid sizes solved together.
//
// The reference solves one problem per cdr2::solver (include/cedar/2d/solver.h:
// 45-129); each problem here keeps that solve's semantics (its own hierarchy,
// FP32 V-cycles refined in FP64 to its own relative tolerance).  What is shared
// is the work: every level of every problem with the same grid size lives in
// one FP32 array, the problems back to back, so that one launch of each step
// of the V-cycle (a colour of lines, a residual, a restriction, ...) covers
// that level of all problems at once, whatever their fine size.  The cycle
// walks the sizes from the largest down and back up; the sizes at and below
// the common fused coarse level run as one k_coarse_cycle launch over all
// problems.  A problem's own steps still come in its own V-cycle order (the
// levels of one problem have distinct sizes), so each problem gets exactly the
// operations of its single-size batch.  The whole cycle is one CUDA graph on
// one stream.
//
// The FP64 parts stay per size class (one Batch2 each): the fine operators,
// the hierarchy's setup (operator-induced interpolation, Galerkin operators,
// line factors, coarsest factor, all written into the shared FP32 arrays) and
// the outer refinement step.
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <numeric>
#include <vector>

#include "batch2d.cuh"

namespace cdrgpu {

namespace {

// The FP32 arrays of one grid size: every problem's level of that size,
// problems back to back (entries), for the FP32 cycle
struct USize {
	int nx = 0, ny = 0, ns = 5, pitch = 0, tpitch = 0;
	int entries = 0;
	bool coarsest = false;   // the coarsest level of every problem that has it
	bool smoothed = false;   // a smoothing level (not the coarsest) of its problems
	float *so32 = nullptr, *x32 = nullptr, *b32 = nullptr, *r32 = nullptr, *ci32 = nullptr, *sor32 = nullptr,
	      *sory32 = nullptr;
	float *yc32 = nullptr;  // packed y-line couplings (y-lines of at most 1024 points)
	double *abd = nullptr;
	int child = -1;      // index of the next coarser size
	int child_off = 0;   // entry of this size's first problem among the child's entries
	size_t plane() const { return (size_t)pitch * (ny + 2); }
	size_t ysize() const { return 2 * (size_t)tpitch * (nx + 2); }
	size_t ypsize() const { return (size_t)ypack_planes(ns) * tpitch * (nx + 2); }
	size_t abd_size() const { return (size_t)(nx + 2) * nx * ny; }
	Dims2 dims(int count) const
	{
		Dims2 d{nx, ny, pitch};
		d.nb = count;
		d.bstep = 1;
		return d;
	}
};

// One size class: nb problems of one fine size (a Batch2 of its own for the
// FP64 parts) and where its levels sit among the shared sizes
struct Cls {
	std::unique_ptr<Batch2> B;
	int nb = 0, caller = 0;  // problems, the class's index in the caller's arrays
	std::vector<int> size;   // shared size of each level
	std::vector<int> off;    // entry of the class's first problem at that size
	double *x64[2] = {nullptr, nullptr}, *norm = nullptr, *partial = nullptr;
	int *active = nullptr;
	double *h_norm = nullptr;
	int *h_active = nullptr;
};

__global__ void k_zero_f32(float *__restrict__ p, size_t n)
{
	for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
		p[e] = 0.f;
}

}  // namespace
}  // namespace cdrgpu

using namespace cdrgpu;

struct cdr_gpu_batchmix {
	cdr_gpu_settings s{};
	cudaStream_t st = nullptr;
	bool own_stream = false;
	std::vector<Cls> cls;        // by fine size, largest first
	std::vector<USize> sz;       // shared sizes, largest first
	int fused = -1;              // size from which the coarse cycle runs in one launch (-1: none)
	int nfused_levels = 0;
	std::vector<void *> allocs;
	cudaGraphExec_t gexec = nullptr;
	long long glaunches = 0;
	std::vector<cudaEvent_t> ev;
	float setup_ms = 0.f, solve_ms = 0.f;
	int total = 0;               // problems

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

	// zero: every entry's iterate is zero on entry (its interior is not read)
	int smooth(USize &U, int updown, bool zero = false)
	{
		const Dims2 d = U.dims(U.entries);
		const int flags = s.line_flags & CDR_LINES_NOTUNE;
		const int n = updown == CDR_DOWN ? s.nrelax_pre : s.nrelax_post;
		if (zero && (n == 0 || s.relaxation == CDR_RELAX_POINT)) {  // only the line sweeps skip reading it
			CDR_CUDA_TRY(cudaMemsetAsync(U.x32, 0, sizeof(float) * U.plane() * U.entries, st));
			zero = false;
		}
		for (int it = 0; it < n; ++it) {
			const int f = flags | (zero && it == 0 ? CDR_LINES_ZERO_START : 0);
			switch (s.relaxation) {
			case CDR_RELAX_POINT: CDR_TRY(relax_point_2d<float>(U.so32, U.ns, U.x32, U.b32, U.sor32, d, updown, st)); break;
			case CDR_RELAX_LINE_X:
				CDR_TRY(relax_lines_2d<float>(U.so32, U.ns, U.x32, U.b32, U.sor32, d, U.tpitch, CDR_DIR_X, updown, f, st));
				break;
			case CDR_RELAX_LINE_Y:
				CDR_TRY(relax_lines_2d<float>(U.so32, U.ns, U.x32, U.b32, U.sory32, d, U.tpitch, CDR_DIR_Y, updown, f, st, nullptr, U.yc32));
				break;
			default:
				if (updown == CDR_DOWN) {
					CDR_TRY(relax_lines_2d<float>(U.so32, U.ns, U.x32, U.b32, U.sor32, d, U.tpitch, CDR_DIR_X, updown, f, st));
					CDR_TRY(relax_lines_2d<float>(U.so32, U.ns, U.x32, U.b32, U.sory32, d, U.tpitch, CDR_DIR_Y, updown, flags, st, nullptr, U.yc32));
				} else {
					CDR_TRY(relax_lines_2d<float>(U.so32, U.ns, U.x32, U.b32, U.sory32, d, U.tpitch, CDR_DIR_Y, updown, f, st, nullptr, U.yc32));
					CDR_TRY(relax_lines_2d<float>(U.so32, U.ns, U.x32, U.b32, U.sor32, d, U.tpitch, CDR_DIR_X, updown, flags, st));
				}
			}
		}
		return CDR_OK;
	}

	// sizes [0, smoothed_sizes()) are smoothed by the cycle's separate launches
	int smoothed_sizes() const { return fused >= 0 ? fused : (int)sz.size() - 1; }

	// One FP32 V-cycle of every problem on its fine-level x32 and b32
	// (cycle::vcycle::ncycle_helper, include/cedar/cycle/vcycle.h:57-115, per
	// problem): down the sizes, the coarse end, up the sizes.  Every problem's
	// iterate is zero when its first smoothing starts (the refinement's
	// correction on its fine level, coarse_x.set(0.0) below it): the sizes the
	// cycle smooths start with sweeps that treat it as zero without reading it,
	// the coarse end's iterates are cleared.
	int cycle()
	{
		const int ns = (int)sz.size();
		const int stop = smoothed_sizes();
		for (int k = 0; k < stop; ++k) {
			USize &F = sz[k], &C = sz[F.child];
			const Dims2 df = F.dims(F.entries), dc = C.dims(F.entries);
			CDR_TRY(smooth(F, CDR_DOWN, true));
			CDR_TRY(residual_2d<float>(F.so32, F.ns, F.x32, F.b32, F.r32, df, nullptr, nullptr, st));
			const size_t co = (size_t)F.child_off;
			CDR_TRY(restrict_2d<float>(C.ci32 + co * 8 * C.plane(), F.r32, C.b32 + co * C.plane(), df, dc, st));
			if (F.child >= stop)
				CDR_CUDA_TRY(cudaMemsetAsync(C.x32 + co * C.plane(), 0, sizeof(float) * C.plane() * F.entries, st));
		}
		if (fused >= 0) {
			CoarseCycle<float> cc;
			cc.nl = nfused_levels;
			int k = fused;
			for (int l = 0; l < nfused_levels; ++l, k = sz[k].child) {
				USize &V = sz[k];
				CoarseLevel<float> &c = cc.lv[l];
				c.so = V.so32;
				c.sor = V.sor32;
				c.sory = V.sory32;
				c.ci = l > 0 ? V.ci32 : nullptr;
				c.x = V.x32;
				c.b = V.b32;
				c.r = V.r32;
				c.nx = V.nx;
				c.ny = V.ny;
				c.pitch = V.pitch;
				c.tpitch = V.tpitch;
				c.ns = V.ns;
				if (l + 1 == nfused_levels) cc.abd = V.abd;
			}
			cc.relax = s.relaxation;
			cc.npre = s.nrelax_pre;
			cc.npost = s.nrelax_post;
			cc.bstep = 1;
			CDR_TRY(coarse_cycle<float>(cc, sz[fused].entries, st));
		} else {
			USize &Cg = sz[ns - 1];
			CDR_TRY(solve_cg_2d<float>(Cg.abd, Cg.x32, Cg.b32, Cg.dims(Cg.entries), st));
		}
		for (int k = stop - 1; k >= 0; --k) {
			USize &F = sz[k], &C = sz[F.child];
			const Dims2 df = F.dims(F.entries), dc = C.dims(F.entries);
			const size_t co = (size_t)F.child_off;
			CDR_TRY(interp_add_2d<float>(C.ci32 + co * 8 * C.plane(), C.x32 + co * C.plane(), F.r32, F.so32, F.x32, df,
			                             dc, st, F.ns));
			CDR_TRY(smooth(F, CDR_UP));
		}
		return CDR_OK;
	}

	int run_cycle()
	{
		if (!s.use_graph) return cycle();
		if (!gexec) {
			cudaGraph_t g = nullptr;
			CDR_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
			const long long before = cdr_gpu_launch_count();
			int rc = cycle();
			glaunches = cdr_gpu_launch_count() - before;
			count_launches(-glaunches);
			cudaError_t e = cudaStreamEndCapture(st, &g);
			if (rc != CDR_OK) {
				if (g) cudaGraphDestroy(g);
				return rc;
			}
			if (e != cudaSuccess) {
				set_error(CDR_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
				return CDR_ERR_CUDA;
			}
			CDR_CUDA_TRY(cudaGraphInstantiate(&gexec, g, 0));
			cudaGraphDestroy(g);
		}
		CDR_CUDA_TRY(cudaGraphLaunch(gexec, st));
		count_launches(glaunches);
		return CDR_OK;
	}
};

namespace {

// The shared sizes of the classes' hierarchies and each level's entry range;
// the classes' levels of one size are back to back in class order, and the
// problems of a size map onto one contiguous block of its child size.
int build_sizes(cdr_gpu_batchmix *h)
{
	std::map<std::pair<int, int>, int> index;  // (nx, ny) -> provisional id
	std::vector<USize> tmp;
	for (Cls &c : h->cls) {
		Batch2 &B = *c.B;
		c.size.resize(B.L());
		c.off.resize(B.L());
		for (int l = 0; l < B.L(); ++l) {
			const B2Level &L = B.lv[l];
			auto key = std::make_pair(L.nx, L.ny);
			auto it = index.find(key);
			if (it == index.end()) {
				USize U;
				U.nx = L.nx;
				U.ny = L.ny;
				U.ns = L.ns;
				U.pitch = L.pitch;
				U.tpitch = L.tpitch;
				U.coarsest = l + 1 == B.L();
				U.smoothed = l + 1 < B.L();
				it = index.emplace(key, (int)tmp.size()).first;
				tmp.push_back(U);
			}
			USize &U = tmp[it->second];
			if (U.ns != L.ns || U.coarsest != (l + 1 == B.L()) || U.smoothed != (l + 1 < B.L())) {
				set_error(CDR_ERR_UNSUPPORTED,
				          "mixed batch: the %dx%d levels of the classes differ (stencil planes or coarsest)", L.nx, L.ny);
				return CDR_ERR_UNSUPPORTED;
			}
			c.size[l] = it->second;
			c.off[l] = U.entries;
			U.entries += c.nb;
		}
	}
	// order the sizes largest first (a level's child is always smaller)
	std::vector<int> order(tmp.size());
	std::iota(order.begin(), order.end(), 0);
	std::sort(order.begin(), order.end(), [&](int a, int b) {
		return (long)tmp[a].nx * tmp[a].ny > (long)tmp[b].nx * tmp[b].ny ||
		       ((long)tmp[a].nx * tmp[a].ny == (long)tmp[b].nx * tmp[b].ny && tmp[a].nx > tmp[b].nx);
	});
	std::vector<int> rank(tmp.size());
	for (size_t k = 0; k < order.size(); ++k) rank[order[k]] = (int)k;
	h->sz.clear();
	for (int id : order) h->sz.push_back(tmp[id]);
	for (Cls &c : h->cls)
		for (int &sid : c.size) sid = rank[sid];
	// children and the contiguity of each size's problems within its child
	for (size_t k = 0; k < h->sz.size(); ++k) {
		USize &U = h->sz[k];
		if (U.coarsest) continue;
		int child = -1, first = -1, next = 0;
		for (Cls &c : h->cls)
			for (size_t l = 0; l + 1 < c.size.size(); ++l) {
				if (c.size[l] != (int)k) continue;
				const int cs = c.size[l + 1], co = c.off[l + 1];
				if (child < 0) {
					child = cs;
					first = co;
					next = co;
				}
				// classes appear in order: each continues the block in the child
				if (cs != child || co != next || c.off[l] != next - first) {
					set_error(CDR_ERR_UNSUPPORTED, "mixed batch: the %dx%d levels do not map onto one block of the next size",
					          U.nx, U.ny);
					return CDR_ERR_UNSUPPORTED;
				}
				next = co + c.nb;
			}
		U.child = child;
		U.child_off = first;
	}
	return CDR_OK;
}

}  // namespace

extern "C" {

int cdr_gpu_batchmix_destroy(cdr_gpu_batchmix *h)
{
	if (!h) return CDR_ERR_HANDLE;
	if (h->st) cudaStreamSynchronize(h->st);
	if (h->gexec) cudaGraphExecDestroy(h->gexec);
	for (auto &e : h->ev)
		if (e) cudaEventDestroy(e);
	for (Cls &c : h->cls) {
		if (c.h_norm) cudaFreeHost(c.h_norm);
		if (c.h_active) cudaFreeHost(c.h_active);
	}
	for (void *p : h->allocs) cudaFree(p);
	cudaStream_t st = h->st;
	const bool own = h->own_stream;
	delete h;  // the classes' batches free their arrays
	if (own && st) cudaStreamDestroy(st);
	return CDR_OK;
}

int cdr_gpu_batchmix_create(const cdr_gpu_settings *s, int nclass, const double *const *so_dev, const int *ns,
                            const int *nx, const int *ny, const int *pitch, const int *nb, cudaStream_t stream,
                            cdr_gpu_batchmix **out)
{
	if (!s || !so_dev || !ns || !nx || !ny || !pitch || !nb || !out) {
		set_error(CDR_ERR_ARG, "null argument");
		return CDR_ERR_ARG;
	}
	*out = nullptr;
	if (nclass < 1 || nclass > 64) {
		set_error(CDR_ERR_ARG, "mixed batch of %d size classes (1..64)", nclass);
		return CDR_ERR_ARG;
	}
	if (s->precision != CDR_PREC_F32_IR) {
		set_error(CDR_ERR_UNSUPPORTED, "mixed batch: FP32 cycles with FP64 refinement only (precision fp32-ir)");
		return CDR_ERR_UNSUPPORTED;
	}
	if (s->relaxation < CDR_RELAX_POINT || s->relaxation > CDR_RELAX_LINE_XY) {
		set_error(CDR_ERR_ARG, "invalid 2D relaxation %d", s->relaxation);
		return CDR_ERR_ARG;
	}
	if (s->krylov != CDR_KRYLOV_NONE || s->coarse_solve != CDR_COARSE_BANDED || s->fp32_levels != 0 ||
	    s->cycle != CDR_CYCLE_V || s->periodic) {
		set_error(CDR_ERR_UNSUPPORTED, "mixed batch: V-cycles with the banded coarsest solve, no Krylov iteration");
		return CDR_ERR_UNSUPPORTED;
	}
	if (s->maxiter < 1) { set_error(CDR_ERR_ARG, "max-iter must be positive"); return CDR_ERR_ARG; }
	for (int c = 0; c < nclass; ++c) {
		if (!so_dev[c] || (ns[c] != 3 && ns[c] != 5) || nx[c] < 1 || ny[c] < 1 || pitch[c] < nx[c] + 2 || nb[c] < 1) {
			set_error(CDR_ERR_ARG, "size class %d: bad operator, grid %dx%d, pitch %d or %d problems", c, nx[c], ny[c],
			          pitch[c], nb[c]);
			return CDR_ERR_ARG;
		}
	}
	cdr_gpu_batchmix *h = new cdr_gpu_batchmix();
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
	auto fail = [&](int rc) {
		cdr_gpu_batchmix_destroy(h);
		return rc;
	};
	int rc = lines_prepare();
	if (rc != CDR_OK) return fail(rc);
	// classes largest fine grid first
	std::vector<int> order(nclass);
	std::iota(order.begin(), order.end(), 0);
	std::stable_sort(order.begin(), order.end(),
	                 [&](int a, int b) { return (long)nx[a] * ny[a] > (long)nx[b] * ny[b]; });
	h->cls.resize(nclass);
	for (int k = 0; k < nclass; ++k) {
		const int c = order[k];
		Cls &C = h->cls[k];
		C.caller = c;
		C.nb = nb[c];
		C.B.reset(new Batch2());
		if ((rc = C.B->init(*s, ns[c], nx[c], ny[c], nb[c], h->st, true)) != CDR_OK) return fail(rc);
		h->total += nb[c];
	}
	if ((rc = build_sizes(h)) != CDR_OK) return fail(rc);
	const bool lines = s->relaxation != CDR_RELAX_POINT;
	for (USize &U : h->sz) {
		const size_t pl = U.plane() * U.entries;
		if ((rc = h->alloc(&U.so32, pl * U.ns)) || (rc = h->alloc(&U.x32, pl)) || (rc = h->alloc(&U.b32, pl)) ||
		    (rc = h->alloc(&U.r32, pl)) || (rc = h->alloc(&U.ci32, pl * 8)))
			return fail(rc);
		if (U.smoothed) {
			if ((rc = h->alloc(&U.sor32, pl * 2))) return fail(rc);
			if (lines && (rc = h->alloc(&U.sory32, U.ysize() * U.entries))) return fail(rc);
			const bool ly = s->relaxation == CDR_RELAX_LINE_Y || s->relaxation == CDR_RELAX_LINE_XY;
			if (ly && U.ny <= 1024 && (rc = h->alloc(&U.yc32, U.ypsize() * U.entries))) return fail(rc);
		}
		if (U.coarsest && (rc = h->alloc(&U.abd, U.abd_size() * U.entries))) return fail(rc);
	}
	// each class's FP32 levels and coarsest factor inside the shared arrays
	for (Cls &C : h->cls) {
		Batch2 &B = *C.B;
		for (int l = 0; l < B.L(); ++l) {
			USize &U = h->sz[C.size[l]];
			B2Level &L = B.lv[l];
			const size_t o = (size_t)C.off[l], pl = U.plane();
			L.so32 = U.so32 + o * U.ns * pl;
			L.x32 = U.x32 + o * pl;
			L.b32 = U.b32 + o * pl;
			L.r32 = U.r32 + o * pl;
			L.ci32 = l > 0 ? U.ci32 + o * 8 * pl : nullptr;
			L.sor32 = U.sor32 ? U.sor32 + o * 2 * pl : nullptr;
			L.sory32 = U.sory32 ? U.sory32 + o * U.ysize() : nullptr;
			L.yc32 = U.yc32 ? U.yc32 + o * U.ypsize() : nullptr;
			if (l + 1 == B.L()) B.abd = U.abd + o * U.abd_size();
		}
		const B2Level &F = B.lv[0];
		const size_t fpl = F.plane();
		if ((rc = h->alloc(&C.x64[0], fpl * C.nb)) || (rc = h->alloc(&C.x64[1], fpl * C.nb)) ||
		    (rc = h->alloc(&C.norm, (size_t)C.nb)) ||
		    (rc = h->alloc(&C.partial, (size_t)norm_blocks(F.dims(Sel{0, 1, C.nb})) * C.nb)) ||
		    (rc = h->alloc(&C.active, (size_t)C.nb)))
			return fail(rc);
		if (cudaMallocHost(&C.h_norm, sizeof(double) * C.nb) != cudaSuccess ||
		    cudaMallocHost(&C.h_active, sizeof(int) * C.nb) != cudaSuccess) {
			set_error(CDR_ERR_CUDA, "cannot allocate pinned host buffers");
			return fail(CDR_ERR_CUDA);
		}
	}
	// the fused coarse cycle: from a size every class fuses from (the classes'
	// own choice), else none
	{
		int f = -2;
		for (Cls &C : h->cls) {
			const int lc = C.B->lc[1];
			const int sid = lc >= 0 ? C.size[lc] : -1;
			if (f == -2) f = sid;
			else if (f != sid) f = -1;
		}
		h->fused = f >= 0 ? f : -1;
		if (h->fused >= 0) {
			// every size of the chain holds all problems in the same order
			int n = 0;
			for (int k = h->fused; k >= 0; k = h->sz[k].child) {
				if (h->sz[k].entries != h->total || (!h->sz[k].coarsest && h->sz[k].child_off != 0)) {
					h->fused = -1;
					break;
				}
				++n;
			}
			h->nfused_levels = h->fused >= 0 ? n : 0;
			if (n > kMaxCoarseLevels) h->fused = -1;
		}
	}
	if (h->fused < 0)
		for (size_t k = 0; k + 1 < h->sz.size(); ++k)
			if (h->sz[k].coarsest || h->sz[k].child < 0) {
				set_error(CDR_ERR_UNSUPPORTED, "mixed batch: the classes' coarsest grids differ");
				return fail(CDR_ERR_UNSUPPORTED);
			}
	h->ev.resize(s->maxiter + 2);
	for (auto &e : h->ev)
		if (cudaEventCreate(&e) != cudaSuccess) {
			e = nullptr;
			set_error(CDR_ERR_CUDA, "cannot create events");
			return fail(CDR_ERR_CUDA);
		}
	// fine operators (caller pitch) -> class layout, then each class's setup
	for (Cls &C : h->cls) {
		B2Level &F = C.B->lv[0];
		const int c = C.caller;
		if (cudaMemcpy2DAsync(F.so, F.pitch * sizeof(double), so_dev[c], pitch[c] * sizeof(double),
		                      (nx[c] + 2) * sizeof(double), (size_t)(ny[c] + 2) * ns[c] * nb[c],
		                      cudaMemcpyDeviceToDevice, h->st) != cudaSuccess) {
			set_error(CDR_ERR_CUDA, "operator copy failed");
			return fail(CDR_ERR_CUDA);
		}
	}
	if (cudaEventRecord(h->ev[0], h->st) != cudaSuccess) return fail(CDR_ERR_CUDA);
	for (Cls &C : h->cls)
		if ((rc = C.B->setup(true)) != CDR_OK) return fail(rc);
	if (cudaEventRecord(h->ev[1], h->st) != cudaSuccess || cudaEventSynchronize(h->ev[1]) != cudaSuccess ||
	    cudaEventElapsedTime(&h->setup_ms, h->ev[0], h->ev[1]) != cudaSuccess) {
		set_error(CDR_ERR_CUDA, "setup timing events failed");
		return fail(CDR_ERR_CUDA);
	}
	// line kernels' launch shapes on the shared sizes (sweeps on the shared
	// arrays: the solve zeroes the iterates it starts from)
	if (lines && !(s->line_flags & CDR_LINES_NOTUNE)) {
		const bool lx = s->relaxation == CDR_RELAX_LINE_X || s->relaxation == CDR_RELAX_LINE_XY;
		const bool ly = s->relaxation == CDR_RELAX_LINE_Y || s->relaxation == CDR_RELAX_LINE_XY;
		const int stop = h->fused >= 0 ? h->fused : (int)h->sz.size() - 1;
		for (int k = 0; k < stop; ++k) {
			USize &U = h->sz[k];
			const Dims2 d = U.dims(U.entries);
			if (lx && (rc = lines_autotune<float>(U.so32, U.ns, U.x32, U.b32, U.sor32, d, U.tpitch, CDR_DIR_X, h->st)))
				return fail(rc);
			if (ly && (rc = lines_autotune<float>(U.so32, U.ns, U.x32, U.b32, U.sory32, d, U.tpitch, CDR_DIR_Y, h->st,
			                                      nullptr, U.yc32)))
				return fail(rc);
		}
	}
	*out = h;
	return CDR_OK;
}

// multilevel::solve (include/cedar/multilevel.h:278-298) for every problem:
// FP32 V-cycles of all problems together, each problem's FP64 refinement step
// and stopping test its own (its iterate no longer changes once it has met the
// tolerance).  b_dev[c] / x_dev[c]: class c's problems back to back at the
// create call's pitch; iters, rel, done_ms: per problem, classes in the
// caller's order (done_ms may be null).
int cdr_gpu_batchmix_solve_device(cdr_gpu_batchmix *h, const double *const *b_dev, double *const *x_dev,
                                  const int *pitch, int *iters, double *rel, float *done_ms)
{
	if (!h) { set_error(CDR_ERR_HANDLE, "null batch"); return CDR_ERR_HANDLE; }
	if (!b_dev || !x_dev || !pitch || !iters || !rel) { set_error(CDR_ERR_ARG, "null argument"); return CDR_ERR_ARG; }
	const cudaStream_t st = h->st;
	const int nclass = (int)h->cls.size();
	std::vector<int> first(nclass + 1, 0);  // problem index of caller class c
	{
		std::vector<int> nbc(nclass);
		for (Cls &C : h->cls) nbc[C.caller] = C.nb;
		for (int c = 0; c < nclass; ++c) first[c + 1] = first[c] + nbc[c];
	}
	std::vector<std::vector<double>> res0(nclass);
	std::vector<int> last(h->total, 0);
	int nactive = 0;
	for (Cls &C : h->cls) {
		B2Level &F = C.B->lv[0];
		const int c = C.caller;
		if (pitch[c] < F.nx + 2 || !b_dev[c] || !x_dev[c]) {
			set_error(CDR_ERR_ARG, "size class %d: bad buffer or pitch %d", c, pitch[c]);
			return CDR_ERR_ARG;
		}
		const size_t w = (F.nx + 2) * sizeof(double), rows = (size_t)(F.ny + 2) * C.nb;
		CDR_CUDA_TRY(cudaMemcpy2DAsync(F.b, F.pitch * sizeof(double), b_dev[c], pitch[c] * sizeof(double), w, rows,
		                               cudaMemcpyDeviceToDevice, st));
		CDR_CUDA_TRY(cudaMemcpy2DAsync(C.x64[0], F.pitch * sizeof(double), x_dev[c], pitch[c] * sizeof(double), w, rows,
		                               cudaMemcpyDeviceToDevice, st));
		for (int p = 0; p < C.nb; ++p) {
			iters[first[c] + p] = 0;
			rel[first[c] + p] = 1.0;
			C.h_active[p] = 1;
		}
		nactive += C.nb;
		CDR_CUDA_TRY(cudaMemcpyAsync(C.active, C.h_active, sizeof(int) * C.nb, cudaMemcpyHostToDevice, st));
	}
	CDR_CUDA_TRY(cudaEventRecord(h->ev[0], st));
	for (Cls &C : h->cls) {
		B2Level &F = C.B->lv[0];
		const Dims2 d = F.dims(Sel{0, 1, C.nb});
		CDR_TRY(ir_residual_2d(F.so, F.ns, C.x64[0], F.x32, F.b, C.x64[1], F.b32, d, d, C.norm, C.partial, 0, st));
		CDR_CUDA_TRY(cudaMemcpyAsync(C.h_norm, C.norm, sizeof(double) * C.nb, cudaMemcpyDeviceToHost, st));
	}
	CDR_CUDA_TRY(cudaStreamSynchronize(st));
	for (Cls &C : h->cls) res0[C.caller].assign(C.h_norm, C.h_norm + C.nb);
	int cur = 0, it = 0, bad = 0;
	for (it = 0; it < h->s.maxiter && nactive > 0; ++it) {
		for (Cls &C : h->cls) {
			if (C.size[0] < h->smoothed_sizes()) continue;  // the cycle's first sweep treats it as zero
			B2Level &F = C.B->lv[0];
			const size_t n = F.plane() * C.nb;
			k_zero_f32<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0, st>>>(F.x32, n);
			CDR_LAUNCH_CHECK();
		}
		CDR_TRY(h->run_cycle());
		for (Cls &C : h->cls) {
			B2Level &F = C.B->lv[0];
			const Dims2 d = F.dims(Sel{0, 1, C.nb});
			CDR_TRY(ir_residual_2d(F.so, F.ns, C.x64[cur], F.x32, F.b, C.x64[1 - cur], F.b32, d, d, C.norm, C.partial,
			                       1, st, C.active));
			CDR_CUDA_TRY(cudaMemcpyAsync(C.h_norm, C.norm, sizeof(double) * C.nb, cudaMemcpyDeviceToHost, st));
		}
		cur = 1 - cur;
		CDR_CUDA_TRY(cudaEventRecord(h->ev[it + 1], st));
		CDR_CUDA_TRY(cudaStreamSynchronize(st));
		for (Cls &C : h->cls) {
			const int c = C.caller;
			for (int p = 0; p < C.nb; ++p) {
				if (!C.h_active[p]) continue;
				const double r = C.h_norm[p] / res0[c][p];
				iters[first[c] + p] = it + 1;
				rel[first[c] + p] = r;
				last[first[c] + p] = it + 1;
				if (!std::isfinite(r)) bad = 1;
				if (!(r >= h->s.tol)) {
					C.h_active[p] = 0;
					--nactive;
				}
			}
			CDR_CUDA_TRY(cudaMemcpyAsync(C.active, C.h_active, sizeof(int) * C.nb, cudaMemcpyHostToDevice, st));
		}
	}
	for (Cls &C : h->cls) {
		B2Level &F = C.B->lv[0];
		const int c = C.caller;
		const size_t w = (F.nx + 2) * sizeof(double), rows = (size_t)(F.ny + 2) * C.nb;
		CDR_CUDA_TRY(cudaMemcpy2DAsync(x_dev[c], pitch[c] * sizeof(double), C.x64[cur], F.pitch * sizeof(double), w,
		                               rows, cudaMemcpyDeviceToDevice, st));
	}
	CDR_CUDA_TRY(cudaStreamSynchronize(st));
	CDR_CUDA_TRY(cudaEventElapsedTime(&h->solve_ms, h->ev[0], h->ev[it > 0 ? it : 0]));
	if (done_ms)
		for (int p = 0; p < h->total; ++p) {
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

int cdr_gpu_batchmix_timings(const cdr_gpu_batchmix *h, double *setup_ms, double *solve_ms)
{
	if (!h) return CDR_ERR_HANDLE;
	if (setup_ms) *setup_ms = h->setup_ms;
	if (solve_ms) *solve_ms = h->solve_ms;
	return CDR_OK;
}

int cdr_gpu_batchmix_sizes(const cdr_gpu_batchmix *h) { return h ? (int)h->sz.size() : -1; }

long long cdr_gpu_batchmix_cycle_launches(const cdr_gpu_batchmix *h) { return h ? h->glaunches : -1; }

}  // extern "C"
