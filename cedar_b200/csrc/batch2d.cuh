// batch2d.cuh -- a batch of independent 2D BoxMG hierarchies of one grid size.
//
// Every level array holds the problems back to back (problem p of an array of
// P planes starts at p*P*plane()), so one launch of a 2D kernel covers a whole
// selection of problems (grid z, Dims2::nb / bstep).  Used for the plane
// smoothers of the 3D solver (one 2D solver per plane, as
// planes<rdir>::setup_impl in include/cedar/3d/relax_planes.h:171-222 builds
// them) and for batches of independent 2D solves.
#pragma once
#include <vector>

#include "kernels2d.cuh"

namespace cdrgpu {

// Problems first, first + step, ... (count of them).
struct Sel {
	int first = 0, step = 1, count = 1;
};

struct B2Level {
	int nx = 0, ny = 0, ns = 5, pitch = 0, tpitch = 0;
	double *so = nullptr, *x = nullptr, *b = nullptr, *r = nullptr, *sor = nullptr, *sory = nullptr, *ci = nullptr;
	float *so32 = nullptr, *x32 = nullptr, *b32 = nullptr, *r32 = nullptr, *sor32 = nullptr, *sory32 = nullptr,
	      *ci32 = nullptr;
	// packed y-line couplings (pack_ylines_2d) of levels whose y-lines have at
	// most 1024 points, ypsize() per problem; null elsewhere
	double *yc = nullptr;
	float *yc32 = nullptr;
	size_t plane() const { return (size_t)pitch * (ny + 2); }
	size_t ysize() const { return 2 * (size_t)tpitch * (nx + 2); }  // y-line factors of one problem
	size_t ypsize() const { return (size_t)ypack_planes(ns) * tpitch * (nx + 2); }
	Dims2 dims(Sel s) const
	{
		Dims2 d{nx, ny, pitch};
		d.nb = s.count;
		d.bstep = s.step;
		return d;
	}
};

class Batch2 {
public:
	cdr_gpu_settings s{};
	int nb = 0;
	std::vector<B2Level> lv;
	double *abd = nullptr;
	int *info = nullptr;  // [0] line factorizations, [1] coarse Cholesky
	int lc[2] = {-1, -1}; // first level of the fused coarse cycle, [0] FP64, [1] FP32 (-1: none)
	cudaStream_t st = nullptr;

	Batch2() = default;
	Batch2(const Batch2 &) = delete;
	Batch2 &operator=(const Batch2 &) = delete;
	~Batch2();

	// Allocate nb hierarchies for an nx x ny fine grid with ns-plane fine
	// operators (the fine operators are then written into lv[0].so).  With
	// external32 the FP32 level arrays and the coarsest factor (abd) are not
	// allocated: the owner points them into its own storage before setup.
	int init(const cdr_gpu_settings &settings, int ns, int nx, int ny, int nb, cudaStream_t stream,
	         bool external32 = false);
	// multilevel::setup (include/cedar/multilevel.h:243-265) for all problems;
	// checks the factorizations (synchronises the stream) when check is set.
	int setup(bool check);
	// Times the line kernels' launch shapes of every smoothing level (once per
	// shape and process); runs sweeps on the level arrays.
	int tune() { return mixed() ? tune_lines<float>() : tune_lines<double>(); }
	int check_info();
	// One V-cycle of the selected problems on their level-0 x and b
	// (cycle::vcycle::ncycle_helper, include/cedar/cycle/vcycle.h:57-115).
	template <typename T>
	int cycle(Sel sel, bool zero = false);  // zero: the level-0 iterate is zero on entry (not read)
	bool mixed() const { return s.precision == CDR_PREC_F32_IR; }
	int L() const { return (int)lv.size(); }
	size_t ldab() const { return (size_t)lv.back().nx + 2; }
	size_t abd_size() const { return ldab() * lv.back().nx * lv.back().ny; }

private:
	std::vector<void *> allocs_;
	template <typename T>
	int alloc(T **p, size_t n);
	template <typename T>
	int smooth(int l, Sel sel, int updown, bool zero = false);
	template <typename T>
	int ncycle(int l, Sel sel, bool zero = false);
	template <typename T>
	int fused(int l0, Sel sel);
	template <typename T>
	int pick_fused();
	template <typename T>
	int tune_lines();
};

// cdr2::solver::compute_num_levels (include/cedar/2d/solver.h:63-79)
int num_levels_2d(int nx, int ny, int min_coarse);

}  // namespace cdrgpu
