// kernels2d.cuh -- host-side launchers of the 2D kernels (internal C++ API).
#pragma once
#include "cdr_common.cuh"

namespace cdrgpu {

template <typename T>
int residual_2d(const T *so, int nstencil, const T *x, const T *b, T *r, Dims2 d, double *norm_out,
                double *partial, cudaStream_t st);
template <typename T>
int setup_recip_2d(const T *so, T *sor, Dims2 d, cudaStream_t st, int nstencil = 5);
// per: periodic directions (bit 0 x, bit 1 y; single problems only)
template <typename T>
int relax_point_2d(const T *so, int nstencil, T *x, const T *b, const T *sor, Dims2 d, int updown, cudaStream_t st,
                   int per = 0);
template <typename TS>
int setup_lines_2d(const double *so, int nstencil, TS *sor, Dims2 d, int tpitch, int dir, int *info, cudaStream_t st);
int lines_prepare();
// ysync (device, lines_sync_words(d) words, zero before the first use and
// between uses): y-lines of a single problem sweep both colours in one launch
// (k_ylines_pair, bit-identical to the two one-colour launches); one buffer
// per stream, since concurrent sweeps on it would race.
template <typename T>
int relax_lines_2d(const T *so, int nstencil, T *x, const T *b, const T *sor, Dims2 d, int tpitch, int dir,
                   int updown, int flags, cudaStream_t st, unsigned *ysync = nullptr, const T *ycpl = nullptr);
size_t lines_sync_words(Dims2 d);
// Launch shape of the line kernel (K elements per thread, y-line CTA cap) and
// the setup-time autotuner that picks it per level (k2_lines.cu).  The tuner
// runs line sweeps on the arrays it is given (x changes unless x = 0 and b = 0).
struct LineShape {
	int K = 8, cap = 1024;
	int stream = 0;  // x-lines: rows streamed into shared memory (k_lines_xstream)
	int pair = 0;    // y-lines of a single problem with a sync buffer: 1 both colours in one launch
	                 // (k_ylines_pair), 0 one launch per colour (the same bits)
};
// bounded waits of the streamed x-line kernel that gave up since the last call
// (read and reset into *count; 0 in a healthy run); CDR_ERR_CUDA if they
// cannot be read
int lines_stream_timeouts(cudaStream_t st, unsigned *count);
// the same for the streamed explicit-inverse product (k2_cginv.cu)
int cg_inv_timeouts(cudaStream_t st, unsigned *count);
// Test hooks (current device): add to a give-up count from the host, and set
// the limit of the streamed kernels' first wait on a stage (ns; 0: one
// non-blocking test)
int lines_stream_add_timeouts(unsigned n);
int cg_inv_add_timeouts(unsigned n);
int lines_stream_set_wait(unsigned long long ns);
constexpr unsigned long long kStreamWaitDefaultNs = 200000000ull;  // kWaitLimitNs of k2_bulk.cuh
int cg_inv_set_wait(unsigned long long ns);
// The packed y-line couplings of a level: ypack_planes(nstencil) planes of
// tpitch * (nx+2) per problem (d.nb problems, bstep apart), line-contiguous;
// relax_lines_2d's y sweeps read them when given the array (ycpl).
template <typename T>
int pack_ylines_2d(const T *so, int nstencil, T *yc, Dims2 d, int tpitch, cudaStream_t st);
inline int ypack_planes(int nstencil) { return nstencil == 5 ? 6 : 2; }
template <typename T>
int lines_autotune(const T *so, int nstencil, T *x, const T *b, const T *sor, Dims2 d, int tpitch, int dir,
                   cudaStream_t st, unsigned *ysync = nullptr, const T *ycpl = nullptr);
bool lines_shape(int dir, int tsize, int ns, int n, int nl, int nb, LineShape *out);
// pin a shape for a line geometry (the autotuner then leaves it); false if the
// shape cannot run lines of length n
bool lines_set_shape(int dir, int tsize, int ns, int n, int nl, int nb, LineShape sh);
template <typename T>
int restrict_2d(const T *ci, const T *rf, T *bc, Dims2 f, Dims2 c, cudaStream_t st);
template <typename T>
int interp_add_2d(const T *ci, const T *xc, const T *rf, const T *sof, T *xf, Dims2 f, Dims2 c, cudaStream_t st,
                  int nstencil_fine = 5);
// Hand-over from an FP32 fine level to an FP64 coarse one (mixed cycles)
int restrict_2d_mixed(const double *ci, const float *rf, double *bc, Dims2 f, Dims2 c, cudaStream_t st);
// The FP32 cycle's fine level with a widened (FP64) iterate: the row-sum
// excess dg of the operator (FP64, rounded), the residual r = b - dg x -
// sum a (x - x_nb) of the FP64 iterate in FP64 arithmetic over the FP32 data
// (zeroing `zero`, the post-smoothing's initial guess), and the interpolate-add
// xout (FP64) = xin + P xc + r/c in FP64
int rowsum_excess_2d(const double *so, int ns, float *dg, Dims2 d, cudaStream_t st);
int residual_2d_wide(const float *so, const float *dg, int ns, const double *x, const float *b, float *r, float *zero,
                     Dims2 d, cudaStream_t st);
int interp_add_2d_wide(const float *ci, const float *xc, const float *rf, const float *sof, const float *xin,
                       double *xout, Dims2 f, Dims2 c, cudaStream_t st, int nsf);
int interp_add_2d_mixed(const double *ci, const double *xc, const float *rf, const float *sof, float *xf, Dims2 f,
                        Dims2 c, cudaStream_t st, int nsf_fine = 5);
int setup_interp_2d(const double *so, int nstencil, double *ci, Dims2 f, Dims2 c, cudaStream_t st);
// Periodic boundary conditions (k2_periodic.cu); per: bit 0 x, bit 1 y.
// Ghost-line copies of `planes` planes: xmode 1 x ghosts of interior rows (of
// parity jpar when jpar >= 0), 2 of all rows; ymode 1 the y ghost rows.
template <typename T>
int ghost_copy_2d(T *q, Dims2 d, int planes, int xmode, int ymode, int jpar, cudaStream_t st);
int setup_interp_per_2d(const double *so, int nstencil, double *ci, Dims2 f, Dims2 c, int per, cudaStream_t st);
// dense N x N factor (N = nx*ny) of the coarsest operator; info as setup_cg_2d
int setup_cg_per_2d(const double *so, int nstencil, Dims2 d, double *abd, int *info, int per, cudaStream_t st);
int solve_cg_per_2d(const double *abd, double *x, const double *b, Dims2 d, int per, cudaStream_t st);
int galerkin_2d(const double *so, int nstencil, const double *ci, double *soc, Dims2 f, Dims2 c, cudaStream_t st);
int setup_cg_2d(const double *so, int nstencil, Dims2 d, double *abd, int *info, cudaStream_t st);
template <typename T>
int solve_cg_2d(const double *abd, T *x, const T *b, Dims2 d, cudaStream_t st);
// Explicit inverse of the coarsest operator from its banded factor (n x n,
// FP64, n = nx*ny) and its application (k2_cginv.cu)
int cg_inverse_2d(const double *abd, Dims2 d, double *ainv, cudaStream_t st);
template <typename T>
int solve_cg_inv_2d(const T *ainv, T *x, const T *b, Dims2 d, cudaStream_t st);
int convert_f64_f32(const double *in, float *out, size_t n, cudaStream_t st);
int ir_residual_2d(const double *so, int nstencil, const double *x, const float *e, const double *b, double *xo,
                   float *r32, Dims2 d, Dims2 d32, double *norm_out, double *partial, int apply, cudaStream_t st,
                   const int *active = nullptr);
// partial-sum blocks per problem of a residual norm (partial holds nb times that)
int norm_blocks(Dims2 d);

// Device scalars of a flexible-CG solve (k2_krylov.cu); its kernels' partial
// sums need fcg_scratch_doubles(d) doubles of scratch.
struct FcgScalars {
	double zq, pq, beta, alpha, rr;
	int first, iter;
	unsigned ticket[3];
};
// r -> preconditioner input rin (zero ghost ring), z = 0, restart the recurrences
size_t fcg_scratch_doubles(Dims2 d);
template <typename TZ>
int fcg_load(const double *r, TZ *rin, TZ *z, Dims2 d, FcgScalars *S, cudaStream_t st, bool restart = true);
// One FCG iteration after the preconditioner wrote its output, z (+ zf when
// zf is not null: an FP64 part and an FP32 part), 3 launches; leaves the next
// preconditioner input in rin, zz = 0 (the cycle's initial guess; zz null:
// left as it is, for a cycle that starts from zero without reading it) and
// |r|^2 in S->rr.  x alternates between x0 and x1: after the step the iterate is in
// x[S->iter & 1].
template <typename TZ, typename TR>
int fcg_step(const double *so, int ns, const TZ *z, const float *zf, TR *rin, TR *zz, double *x0, double *x1,
             const double *b, double *r, double *p0, double *p1, double *q, Dims2 d, double *partial, FcgScalars *S,
             cudaStream_t st, bool formed = true);

constexpr size_t kNormScratchBytes = 2048 * sizeof(double);

// Levels of a fused coarse cycle (k2_coarse.cu): level 0 holds the restricted
// right-hand side and a zero iterate on entry; the last level is the coarsest
// (banded Cholesky factor abd).  Arrays of a batch lie back to back (problem
// blockIdx.x * bstep; the pointers are those of the first problem).
constexpr int kMaxCoarseLevels = 12;
template <typename T>
struct CoarseLevel {
	const T *so = nullptr, *sor = nullptr, *sory = nullptr, *ci = nullptr;
	T *x = nullptr, *b = nullptr, *r = nullptr;
	int nx = 0, ny = 0, pitch = 0, tpitch = 0, ns = 5;
};
template <typename T>
struct CoarseCycle {
	CoarseLevel<T> lv[kMaxCoarseLevels];
	int nl = 0;
	const double *abd = nullptr;
	int relax = CDR_RELAX_POINT, npre = 2, npost = 1, bstep = 1;
};
// shared memory of the fused kernel (bytes) and its limit
constexpr size_t kCoarseSmemMax = 220 * 1024;
template <typename T>
size_t coarse_cycle_bytes(const CoarseCycle<T> &cc);
template <typename T>
int coarse_cycle(const CoarseCycle<T> &cc, int nproblems, cudaStream_t st);
int coarse_prepare();

}  // namespace cdrgpu
