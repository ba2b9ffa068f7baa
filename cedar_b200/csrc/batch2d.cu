// batch2d.cu -- batched 2D BoxMG hierarchies (see batch2d.cuh).
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
	static double *ci(B2Level &L) { return L.ci; }
};
template <> struct BA<float> {
	static float *so(B2Level &L) { return L.so32; }
	static float *x(B2Level &L) { return L.x32; }
	static float *b(B2Level &L) { return L.b32; }
	static float *r(B2Level &L) { return L.r32; }
	static float *sor(B2Level &L) { return L.sor32; }
	static float *sory(B2Level &L) { return L.sory32; }
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

int Batch2::init(const cdr_gpu_settings &settings, int ns, int nx, int ny, int nbatch, cudaStream_t stream)
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
		if (l + 1 < nl) {
			CDR_TRY(alloc(&L.sor, pl * 2));
			if (lines) CDR_TRY(alloc(&L.sory, L.ysize() * nb));
		}
		if (mixed()) {
			CDR_TRY(alloc(&L.so32, pl * L.ns));
			CDR_TRY(alloc(&L.x32, pl));
			CDR_TRY(alloc(&L.b32, pl));
			CDR_TRY(alloc(&L.r32, pl));
			if (l > 0) CDR_TRY(alloc(&L.ci32, pl * 8));
			if (l + 1 < nl) {
				CDR_TRY(alloc(&L.sor32, pl * 2));
				if (lines) CDR_TRY(alloc(&L.sory32, L.ysize() * nb));
			}
		}
	}
	const B2Level &Cg = lv.back();
	if ((size_t)Cg.nx * Cg.ny > 4096) {
		set_error(CDR_ERR_DIM, "coarsest grid %dx%d too large for the banded Cholesky", Cg.nx, Cg.ny);
		return CDR_ERR_DIM;
	}
	CDR_TRY(alloc(&abd, abd_size() * nb));
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
		}
	}
	B2Level &Cg = lv.back();
	CDR_TRY(setup_cg_2d(Cg.so, Cg.ns, Cg.dims(all), abd, info + 1, st));
	if (mixed()) {
		for (int l = 0; l < L(); ++l) {
			B2Level &F = lv[l];
			CDR_TRY(convert_f64_f32(F.so, F.so32, F.plane() * F.ns * nb, st));
			if (l > 0) CDR_TRY(convert_f64_f32(F.ci, F.ci32, F.plane() * 8 * nb, st));
		}
	}
	return check ? check_info() : CDR_OK;
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
int Batch2::smooth(int l, Sel sel, int updown)
{
	B2Level &F = lv[l];
	const Dims2 d = F.dims(sel);
	const size_t f = sel.first, pl = F.plane();
	const T *so = BA<T>::so(F) + f * F.ns * pl;
	T *x = BA<T>::x(F) + f * pl;
	const T *b = BA<T>::b(F) + f * pl;
	const T *sx = BA<T>::sor(F) ? BA<T>::sor(F) + f * 2 * pl : nullptr;
	const T *sy = BA<T>::sory(F) ? BA<T>::sory(F) + f * F.ysize() : nullptr;
	const int flags = sizeof(T) == 8 ? s.line_flags : 0;
	const int n = updown == CDR_DOWN ? s.nrelax_pre : s.nrelax_post;
	for (int it = 0; it < n; ++it) {
		switch (s.relaxation) {
		case CDR_RELAX_POINT: CDR_TRY(relax_point_2d<T>(so, F.ns, x, b, sx, d, updown, st)); break;
		case CDR_RELAX_LINE_X: CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sx, d, F.tpitch, CDR_DIR_X, updown, flags, st)); break;
		case CDR_RELAX_LINE_Y: CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sy, d, F.tpitch, CDR_DIR_Y, updown, flags, st)); break;
		default:
			if (updown == CDR_DOWN) {
				CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sx, d, F.tpitch, CDR_DIR_X, updown, flags, st));
				CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sy, d, F.tpitch, CDR_DIR_Y, updown, flags, st));
			} else {
				CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sy, d, F.tpitch, CDR_DIR_Y, updown, flags, st));
				CDR_TRY(relax_lines_2d<T>(so, F.ns, x, b, sx, d, F.tpitch, CDR_DIR_X, updown, flags, st));
			}
		}
	}
	return CDR_OK;
}

template <typename T>
int Batch2::ncycle(int l, Sel sel)
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
	CDR_TRY(smooth<T>(l, sel, CDR_DOWN));
	CDR_TRY(residual_2d<T>(so, F.ns, x, b, r, df, nullptr, nullptr, st));
	CDR_TRY(restrict_2d<T>(ci, r, bc, df, dc, st));
	// zero the selected coarse iterates: rows of cp elements, step*cp apart
	CDR_CUDA_TRY(cudaMemset2DAsync(xc, sel.step * cp * sizeof(T), 0, cp * sizeof(T), sel.count, st));
	if (l + 1 == L() - 1) CDR_TRY(solve_cg_2d<T>(abd + f * abd_size(), xc, bc, dc, st));
	else CDR_TRY(ncycle<T>(l + 1, sel));
	CDR_TRY(interp_add_2d<T>(ci, xc, r, so, x, df, dc, st, F.ns));
	CDR_TRY(smooth<T>(l, sel, CDR_UP));
	return CDR_OK;
}

template <typename T>
int Batch2::cycle(Sel sel)
{
	if (sel.count < 1) return CDR_OK;
	if (L() == 1) {
		B2Level &F = lv[0];
		const size_t f = sel.first, fp = F.plane();
		return solve_cg_2d<T>(abd + f * abd_size(), BA<T>::x(F) + f * fp, BA<T>::b(F) + f * fp, F.dims(sel), st);
	}
	return ncycle<T>(0, sel);
}
template int Batch2::cycle<double>(Sel);
template int Batch2::cycle<float>(Sel);

}  // namespace cdrgpu
