/*
 * cdr_gpu.h -- C ABI of cedar_b200, the B200 (sm_100a) BoxMG kernels and solver.
 *
 * Every entry point is extern "C", takes plain pointers and sizes and returns
 * an int status (CDR_OK = 0).  Kernel entry points take DEVICE pointers and a
 * cudaStream_t and are stream ordered; they replace the Fortran BIND(C)
 * routines that Cedar's serial C++ kernels call (the call each one replaces is
 * cited beside it, as path:line in cedar-framework/cedar).
 *
 * 2D array layout (Cedar's, include/cedar/stencil_op_nd.h:41-78): one ghost
 * ring, i fastest, one plane per stencil direction.  A grid of nx*ny interior
 * points has (nx+2)*(ny+2) entries per plane; "pitch" is the number of
 * elements between row starts (pitch >= nx+2; Cedar's own host arrays have
 * pitch = nx+2) and planes are pitch*(ny+2) elements apart.  Stencil planes:
 * five_pt {c, w, s} (nstencil = 3), nine_pt {c, w, s, sw, nw} (nstencil = 5)
 * (include/cedar/2d/stencil_op.h:9-10).  Interpolation weights: 8 planes
 * {L, R, A, B, SW, NW, NE, SE} on the coarse grid (include/cedar/2d/prolong_op.h:14).
 */
#ifndef CDR_GPU_H
#define CDR_GPU_H

#include <stddef.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (modelled on include/cedar/capi.h:12-24). */
#define CDR_OK              0
#define CDR_ERR_ARG         1  /* bad argument (null pointer, bad enum)        */
#define CDR_ERR_DIM         2  /* dimension / pitch mismatch                   */
#define CDR_ERR_CUDA        3  /* CUDA runtime error (launch, copy, alloc)     */
#define CDR_ERR_SETUP       4  /* factorization failed (non-positive pivot)    */
#define CDR_ERR_HANDLE      5  /* invalid solver handle                        */
#define CDR_ERR_NUMERIC     6  /* NaN or Inf met in a residual norm            */
#define CDR_ERR_UNSUPPORTED 7  /* option not implemented                       */
#define CDR_ERR_TIMEOUT     8  /* bounded device wait gave up                  */

/* cycle::Dir (include/cedar/cycle/types.h); BMG_DOWN=0, BMG_UP=1 (BMG_parameters_c.h:240-244) */
#define CDR_DOWN 0
#define CDR_UP   1

/* ml_settings::relax_type (include/cedar/multilevel_settings.h:30-31) */
#define CDR_RELAX_POINT   0
#define CDR_RELAX_LINE_X  1
#define CDR_RELAX_LINE_Y  2
#define CDR_RELAX_LINE_XY 3
#define CDR_RELAX_PLANE_XY  4  /* 3D: plane relaxation (include/cedar/3d/relax_planes.h) */
#define CDR_RELAX_PLANE_XZ  5
#define CDR_RELAX_PLANE_YZ  6
#define CDR_RELAX_PLANE_XYZ 7

/* Precision of the solve. */
#define CDR_PREC_F64    0  /* plain FP64 V-cycles: the drop-in path                    */
#define CDR_PREC_F32_IR 1  /* FP32 V-cycle preconditioner in an FP64 refinement loop  */

/* Outer iteration of the 2D solve (settings.krylov).  CDR_KRYLOV_NONE repeats
 * the cycle (plain FP64) or the refinement step (FP32-IR), as the reference's
 * solve loop does.  CDR_KRYLOV_FCG (no counterpart in the reference) uses the
 * cycle, in the solve's precision, as the preconditioner of flexible conjugate
 * gradients (Notay's FCG(1)) with FP64 recurrences; for a symmetric
 * preconditioner choose nrelax_pre == nrelax_post.  The residual is formed
 * as b - A x every settings.krylov_replace iterations (default: every one)
 * and updated as r - alpha A p in between; when an updated residual meets the
 * tolerance the solve forms b - A x and stops only if that meets it too
 * (otherwise it continues from the formed residual).  The history's final
 * entry is always a formed residual b - A x. */
#define CDR_KRYLOV_NONE 0
#define CDR_KRYLOV_FCG  1

/* Coarsest-level solve of the 2D solver (settings.coarse_solve).
 * CDR_COARSE_BANDED: DPBTRS with the banded Cholesky factor, as the reference
 * (bit-identical).  CDR_COARSE_INVERSE (no counterpart in the reference): the
 * setup forms the inverse from that factor and every cycle multiplies by it —
 * equal to rounding, and fast when the coarsest level has thousands of
 * unknowns (solver.num-levels set so that it stops at e.g. 63^2). */
#define CDR_COARSE_BANDED  0
#define CDR_COARSE_INVERSE 1

/* Cycle type (ml_settings::cycle_type, include/cedar/multilevel_settings.h:32):
 * CDR_CYCLE_F runs cycle::fcycle (include/cedar/cycle/fcycle.h:49-83): the
 * right-hand side restricted level by level, the coarsest solved, and on the
 * way up x = P x_coarse followed by a V-cycle at each level.  As in the
 * reference, the F-cycle starts from zero whatever x the solve loop holds. */
#define CDR_CYCLE_V 0
#define CDR_CYCLE_F 1

/* Line direction */
#define CDR_DIR_X 0
#define CDR_DIR_Y 1

/* Text of the last error raised on the calling host thread. */
const char *cdr_gpu_last_error(void);
int cdr_gpu_version(void);
/* Kernel launches issued by this library so far in this process (a replayed
 * cycle graph counts the launches it holds). */
long long cdr_gpu_launch_count(void);
/* Launch shape the line-kernel autotuner chose for lines of length n, nlines
 * lines, direction dir (CDR_DIR_*), FP32 (fp32 = 1) or FP64 sweeps, nstencil 3
 * or 5, a single problem (batch = 0) or a batch (batch = 1): elements per
 * thread *K and the CTA thread cap *cap (x-lines: the CTA size, at most 256,
 * or 0: x-lines streamed through shared memory, CDR_LINES_STREAM; y-lines:
 * lines per CTA = cap / threads per line, at most 4).  K is fixed by the line
 * length (8 up to 2048 points, 16 up to 4096 for FP32), so every shape gives
 * the same bits.  Returns CDR_ERR_ARG when no solver of this process has tuned
 * that shape.  No counterpart in the reference. */
int cdr_gpu_lines_shape(int dir, int fp32, int nstencil, int n, int nlines, int batch, int *K, int *cap);
/* Pin the launch shape (K: the fixed one above; CTA thread cap 32..1024,
 * x-lines at most 256; cap 0: streamed FP32 x-lines) for that geometry in this
 * process; solvers created afterwards use it and the autotuner leaves it.
 * CDR_ERR_ARG if the shape cannot run lines of length n.  No counterpart in
 * the reference. */
int cdr_gpu_lines_set_shape(int dir, int fp32, int nstencil, int n, int nlines, int batch, int K, int cap);

/* ------------------------------------------------------------------------
 * 2D kernels.  T = double (_f64) or float (_f32).
 * ------------------------------------------------------------------------ */

/* r = b - A x on interior points; replaces kernels::residual::run
 * (include/cedar/kernels/residual.h:19-26) -> BMG2_SymStd_residual
 * (include/cedar/2d/residual.h:9-10, src/2d/ftn/BMG2_SymStd_residual.f90:85-119).
 * If norm_out (device, one double) is non-null it receives ||r||_2 over the
 * interior (grid_func::lp_norm<2>, include/cedar/2d/grid_func.h:43-54), summed
 * in FP64 in a fixed order; scratch (device) must then hold
 * cdr_gpu_norm_scratch_bytes() bytes. */
size_t cdr_gpu_norm_scratch_bytes(void);
int cdr_gpu_residual_2d_f64(const double *so, int nstencil, const double *x, const double *b, double *r,
                            int nx, int ny, int pitch, double *norm_out, void *scratch, cudaStream_t stream);
int cdr_gpu_residual_2d_f32(const float *so, int nstencil, const float *x, const float *b, float *r,
                            int nx, int ny, int pitch, double *norm_out, void *scratch, cudaStream_t stream);

/* The same residual and ||r||_2 without any device allocation and without
 * caller scratch, for callers that cannot allocate device memory when they call
 * the library (a plugin inside an application that owns every device allocation
 * and forbids cudaMalloc/cudaFree during a run).  No counterpart in the
 * reference.  The partial sums live in a fixed 512 KiB array of device memory
 * (65536 slots, one per 32x8 tile), reserved on every GPU that loads the library
 * until the process exits; grids of more than 65536 tiles (e.g. beyond
 * 4096x4096 points) are rejected with CDR_ERR_DIM.  The first call on a device
 * looks the array up (once per device, device current): make it before any
 * stream capture.  The looked-up address is kept for the process: after a
 * cudaDeviceReset of that device it is stale, so do not call this entry point
 * on a device that has been reset.  All calls share the array: calls that
 * overlap on the GPU race.  norm_out (device, one double) is required. */
int cdr_gpu_residual_2d_f64_noalloc(const double *so, int nstencil, const double *x, const double *b, double *r,
                                   int nx, int ny, int pitch, double *norm_out, cudaStream_t stream);

/* sor = 1/c; replaces point_relax::setup (include/cedar/kernels/point_relax.h:31-46)
 * -> BMG2_SymStd_SETUP_recip (src/2d/relax.cc:23-33, src/2d/ftn/BMG2_SymStd_SETUP_recip.f90:63-67).
 * sor is one plane (Cedar keeps it in plane 2 of a 2-plane relax_stencil). */
int cdr_gpu_setup_recip_2d_f64(const double *so, double *sor, int nx, int ny, int pitch, cudaStream_t stream);
int cdr_gpu_setup_recip_2d_f32(const float *so, float *sor, int nx, int ny, int pitch, cudaStream_t stream);

/* One red-black (5-pt) / four-colour (9-pt) Gauss-Seidel sweep; replaces
 * point_relax::run (include/cedar/kernels/point_relax.h:48-71) -> BMG2_SymStd_relax_GS
 * (src/2d/relax.cc:38-68, src/2d/ftn/BMG2_SymStd_relax_GS.f90:78-137). */
int cdr_gpu_relax_point_2d_f64(const double *so, int nstencil, double *x, const double *b, const double *sor,
                               int nx, int ny, int pitch, int updown, cudaStream_t stream);
int cdr_gpu_relax_point_2d_f32(const float *so, int nstencil, float *x, const float *b, const float *sor,
                               int nx, int ny, int pitch, int updown, cudaStream_t stream);

/* Line smoother setup: L*D*L^T factors of every line's tridiagonal, plane 0 = D,
 * plane 1 = multipliers (LAPACK DPTTRF storage).  Replaces line_relax::setup
 * (include/cedar/kernels/line_relax.h:22-30) -> BMG2_SymStd_SETUP_lines_{x,y}
 * (src/2d/relax.cc:79-95, src/2d/ftn/BMG2_SymStd_SETUP_lines_x.f90:68-87,
 * BMG2_SymStd_SETUP_lines_y.f90:69-88).  dir = CDR_DIR_X: sor has the grid's layout.
 * dir = CDR_DIR_Y: sor is stored transposed as Cedar does (SOR(JJ,II,2)): element
 * (j, i) at i*tpitch + j with tpitch >= ny+2, planes tpitch*(nx+2) apart.
 * The factorization is always done in FP64; the f32 variant rounds the factors and
 * stores the reciprocal pivots 1/d in plane 0 (its sweeps multiply by them). */
int cdr_gpu_setup_lines_2d_f64(const double *so, int nstencil, double *sor, int nx, int ny, int pitch,
                               int tpitch, int dir, int *info_dev, cudaStream_t stream);
int cdr_gpu_setup_lines_2d_f32(const double *so, int nstencil, float *sor, int nx, int ny, int pitch,
                               int tpitch, int dir, int *info_dev, cudaStream_t stream);

/* One zebra line Gauss-Seidel sweep (both colours); replaces line_relax::run
 * (include/cedar/kernels/line_relax.h:31-39) -> BMG2_SymStd_relax_lines_{x,y}
 * (src/2d/relax.cc:98-133, src/2d/ftn/BMG2_SymStd_relax_lines_x.f90:74-131,
 * BMG2_SymStd_relax_lines_y.f90:74-129).  flags = 0: the per-line DPTTRS
 * substitutions run as a parallel affine scan (fast; each element gets the
 * DPTTS2 update of its inputs, chunk-entry values may differ by rounding);
 * flags = CDR_LINES_EXACT: sequential substitutions, bit-identical to DPTTRS.
 * The parallel kernel's launch shape is the one a solver of this process tuned
 * for this line length and count (cdr_gpu_lines_shape), else the default;
 * CDR_LINES_NOTUNE forces the default. */
#define CDR_LINES_EXACT 1
/* Solver settings.line_flags / kernel flags: keep the default launch shape of
 * the line kernel instead of timing the candidates at setup (the autotuner,
 * whose choice is kept for the process). */
#define CDR_LINES_NOTUNE 2
/* Kernel flags: FP32 x-lines of a single problem (256 <= nx <= 2048) by the
 * streamed kernel: persistent CTAs (two per SM) whose line rows arrive in
 * shared memory by bulk asynchronous copies; each CTA takes its chunks into
 * registers and requests the next line before running the scans.  Same
 * arithmetic as the register-chunk kernel (bit-identical results); the default
 * for FP32 x-lines longer than 1024 points, an autotuner candidate elsewhere
 * (other lines take the register-chunk kernel). */
#define CDR_LINES_STREAM 4
/* Kernel flags: x is zero on entry and its interior is not read (its ghost
 * ring must be zero).  The first colour's right-hand sides are then b alone
 * (b + a*0 for every coupling a, equal up to the sign of an exact zero), so the
 * sweep neither clears x nor reads the couplings to the other colour for it:
 * the first pre-smoothing sweep of a coarse level after restriction
 * (coarse_x.set(0.0), include/cedar/cycle/vcycle.h:79). */
#define CDR_LINES_ZERO_START 8
/* Kernel flags, y-lines through cdr_gpu_relax_lines_2d_sync_*: both colours in
 * one launch (blocks of column pairs, a bounded flag wait between neighbouring
 * blocks) whatever shape the autotuner chose; the same bits as two launches. */
#define CDR_LINES_YPAIR 16
/* Kernel flags, y-lines of a single problem: the factor array sor carries,
 * after its two factor planes, the packed couplings that
 * cdr_gpu_pack_ylines_2d_* wrote; the sweep reads those (the same values, the
 * same bits) with vector loads of each line's own segment. */
#define CDR_LINES_YPACKED 32
/* Status of the streamed x-line kernel since the last call, read on stream s
 * (synchronises it): CDR_ERR_NUMERIC if a CTA gave up waiting for its staged
 * rows (a bounded wait; the sweep's result is then incomplete), else CDR_OK.
 * The 2D solver checks it after every solve; kernel-level callers that use
 * CDR_LINES_STREAM or a streamed pinned shape call it themselves. */
int cdr_gpu_lines_stream_status(cudaStream_t s);
/* Test hooks for the bounded waits of the two streamed kernels (the x-line
 * sweep above and the 2D solver's explicit-inverse coarsest product); no
 * counterpart in the reference.  cdr_gpu_set_wait_limit_ns sets, for the
 * current device, how long a CTA waits for its staged rows before it gives up
 * (ns of the global timer; 0: give up at once, without waiting; negative: the
 * default, 0.2 s).  A CTA that gives up counts itself, waits (at most 1 s) for
 * the copies it still has in flight and leaves its rows unsolved; the status
 * calls and the solver's solve then return CDR_ERR_NUMERIC.
 * cdr_gpu_inject_timeouts adds to the two give-up counts from the host (the
 * host side of that reporting path, without any device wait). */
int cdr_gpu_set_wait_limit_ns(long long ns);
int cdr_gpu_inject_timeouts(unsigned lines, unsigned inverse);
int cdr_gpu_relax_lines_2d_f64(const double *so, int nstencil, double *x, const double *b, const double *sor,
                               int nx, int ny, int pitch, int tpitch, int dir, int updown, int flags,
                               cudaStream_t stream);
int cdr_gpu_relax_lines_2d_f32(const float *so, int nstencil, float *x, const float *b, const float *sor,
                               int nx, int ny, int pitch, int tpitch, int dir, int updown, int flags,
                               cudaStream_t stream);
/* The same sweep with a caller-owned sync buffer (device, cdr_gpu_lines_sync_words(nx)
 * unsigned words, zeroed before its first use; a sweep leaves it zeroed):
 * y-lines (scan mode, 16-byte aligned rows and factor lines) may then run both
 * colours in one launch, where the autotuner chose it for the level or flags
 * hold CDR_LINES_YPAIR.  Blocks of column pairs draw their order from a
 * ticket; each solves its first-colour lines, raises a flag, waits (bounded,
 * as the streamed x-line kernel; a give-up is reported by
 * cdr_gpu_lines_stream_status) for the flag of the block before it and solves
 * its second-colour lines.  The result is bit-identical to the two-launch
 * sweep.  One buffer per stream: sweeps that run concurrently on one buffer
 * race.  x-lines and the other cases run as cdr_gpu_relax_lines_2d_*.  No
 * counterpart in the reference. */
/* Pack a level's y-line couplings after the two factor planes of its y-line
 * factor array sor (transposed layout, tpitch): planes of tpitch*(nx+2)
 * entries, line i's position j at i*tpitch + j, holding w(i,j), w(i+1,j) and
 * for nine-point operators sw(i,j), nw(i+1,j), nw(i,j+1), sw(i+1,j+1) -- the
 * couplings of relax_lines_y.f90:102-106.  sor must hold 2 + 2 (nstencil 3) or
 * 2 + 6 (nstencil 5) planes.  A single problem.  No counterpart in the
 * reference (its sweep reads the operator in place). */
int cdr_gpu_pack_ylines_2d_f64(const double *so, int nstencil, double *sor, int nx, int ny, int pitch, int tpitch,
                               cudaStream_t stream);
int cdr_gpu_pack_ylines_2d_f32(const float *so, int nstencil, float *sor, int nx, int ny, int pitch, int tpitch,
                               cudaStream_t stream);
size_t cdr_gpu_lines_sync_words(int nx);
int cdr_gpu_relax_lines_2d_sync_f64(const double *so, int nstencil, double *x, const double *b, const double *sor,
                                    int nx, int ny, int pitch, int tpitch, int dir, int updown, int flags,
                                    unsigned *sync, cudaStream_t stream);
int cdr_gpu_relax_lines_2d_sync_f32(const float *so, int nstencil, float *x, const float *b, const float *sor,
                                    int nx, int ny, int pitch, int tpitch, int dir, int updown, int flags,
                                    unsigned *sync, cudaStream_t stream);

/* The FP32 preconditioner's fine level with its iterate kept in FP64
 * (settings.fp64_fine_iterate); no counterpart in the reference (its cycle is
 * FP64 throughout).  cdr_gpu_rowsum_excess_2d: dg = c - (sum of the point's
 * 4 or 8 couplings) of an FP64 operator, formed in FP64 and rounded to FP32
 * (interior points).  cdr_gpu_residual_2d_wide: r = b - dg x - sum a (x - x_nb)
 * for an FP64 iterate x over the FP32 couplings a (so32, plane 0 unused) and dg,
 * in FP64 arithmetic, r rounded to FP32; it also zeroes `zero` on the interior
 * (the post-smoothing's initial guess).  Rows 16-byte aligned, pitch a multiple
 * of 4.  cdr_gpu_interp_add_2d_wide: x_out (FP64) = x_in + P x_c + r/c over
 * FP32 weights, coarse iterate, residual and operator diagonal, in FP64
 * arithmetic (interp_add::run, BMG2_SymStd_interp_add.f90:101-137, with the
 * fine iterate widened). */
int cdr_gpu_rowsum_excess_2d(const double *so, int nstencil, float *dg, int nx, int ny, int pitch,
                             cudaStream_t stream);
int cdr_gpu_residual_2d_wide(const float *so, const float *dg, int nstencil, const double *x, const float *b,
                             float *r, float *zero, int nx, int ny, int pitch, cudaStream_t stream);
int cdr_gpu_interp_add_2d_wide(const float *ci, const float *x_coarse, const float *r_fine, const float *so_fine,
                               int nstencil_fine, const float *x_in, double *x_out, int nxf, int nyf, int pf,
                               int nxc, int nyc, int pc, cudaStream_t stream);

/* b_coarse = P^T r_fine; replaces restriction::run (include/cedar/kernels/restrict.h:17-19)
 * -> BMG2_SymStd_restrict (src/2d/restrict.cc:14-29, src/2d/ftn/BMG2_SymStd_restrict.f90:72-92). */
int cdr_gpu_restrict_2d_f64(const double *ci, const double *r_fine, double *b_coarse,
                            int nxf, int nyf, int pitchf, int nxc, int nyc, int pitchc, cudaStream_t stream);
int cdr_gpu_restrict_2d_f32(const float *ci, const float *r_fine, float *b_coarse,
                            int nxf, int nyf, int pitchf, int nxc, int nyc, int pitchc, cudaStream_t stream);

/* x_fine += P x_coarse + r/c at fine-only points; replaces interp_add::run
 * (include/cedar/kernels/interp_add.h:17-20) -> BMG2_SymStd_interp_add (src/2d/interp.cc:20-46,
 * src/2d/ftn/BMG2_SymStd_interp_add.f90:89-137).  so_fine is the fine operator
 * (only its c plane is read).  Unlike the reference, res_fine is not overwritten
 * by res/c (no later step reads it). */
int cdr_gpu_interp_add_2d_f64(const double *ci, const double *x_coarse, const double *res_fine,
                              const double *so_fine, double *x_fine,
                              int nxf, int nyf, int pitchf, int nxc, int nyc, int pitchc, cudaStream_t stream);
int cdr_gpu_interp_add_2d_f32(const float *ci, const float *x_coarse, const float *res_fine,
                              const float *so_fine, float *x_fine,
                              int nxf, int nyf, int pitchf, int nxc, int nyc, int pitchc, cudaStream_t stream);

/* Operator-induced interpolation weights; replaces setup_interp::run
 * (include/cedar/kernels/setup_interp.h:30-47) -> BMG2_SymStd_SETUP_interp_OI
 * (src/2d/interp.cc:49-106, src/2d/ftn/BMG2_SymStd_SETUP_interp_OI.f90:85-257). */
int cdr_gpu_setup_interp_2d_f64(const double *so_fine, int nstencil, double *ci,
                                int nxf, int nyf, int pitchf, int nxc, int nyc, int pitchc, cudaStream_t stream);

/* Galerkin coarse operator so_coarse = P^T A P (5 planes); replaces coarsen_op::run
 * (include/cedar/kernels/coarsen_op.h:23-40) -> BMG2_SymStd_SETUP_ITLI_ex
 * (include/cedar/2d/coarsen.h:34-61, src/2d/ftn/BMG2_SymStd_SETUP_ITLI_ex.f90:94-331). */
int cdr_gpu_galerkin_2d_f64(const double *so_fine, int nstencil, const double *ci, double *so_coarse,
                            int nxf, int nyf, int pitchf, int nxc, int nyc, int pitchc, cudaStream_t stream);

/* Coarsest-grid banded Cholesky, LAPACK upper band storage ABD(nx+2, nx*ny)
 * (column-major, ldab = nx+2, KD = nx+1); replaces solve_cg::setup/run
 * (include/cedar/kernels/solve_cg.h:20-28) -> BMG2_SymStd_SETUP_cg_LU + DPBTRF
 * (include/cedar/2d/solve_cg.h:32-55, src/2d/ftn/BMG2_SymStd_SETUP_cg_LU.f90:92-118,229-255)
 * and BMG2_SymStd_SOLVE_cg + DPBTRS (src/2d/solve_cg.cc:13-28,
 * src/2d/ftn/BMG2_SymStd_SOLVE_cg.f90:93-123).  The solve is FP64 for both variants. */
int cdr_gpu_setup_cg_2d_f64(const double *so, int nstencil, int nx, int ny, int pitch, double *abd,
                            int *info_dev, cudaStream_t stream);
int cdr_gpu_solve_cg_2d_f64(const double *abd, double *x, const double *b, int nx, int ny, int pitch,
                            cudaStream_t stream);
int cdr_gpu_solve_cg_2d_f32(const double *abd, float *x, const float *b, int nx, int ny, int pitch,
                            cudaStream_t stream);

/* ------------------------------------------------------------------------
 * Bilinear finite elements of -div(K grad u), K = diag(kx, ky) per cell, on
 * the unit square with Dirichlet zero boundary (the reference's gallery has
 * only constant-coefficient operators, src/2d/gallery.cc:7-113).  Cells form an
 * (ny+1) x (nx+1) array with row pitch cell_pitch >= nx+1; cell (cj, ci) has
 * corner nodes (ci..ci+1, cj..cj+1) in the ghost-inclusive node index.
 * ------------------------------------------------------------------------ */
/* so (nine_pt, 5 planes) = assembled operator. */
int cdr_gpu_fe_assemble_2d_f64(const double *kx, const double *ky, int cell_pitch, double *so, int nx, int ny,
                               int pitch, cudaStream_t stream);
/* Per-cell dL/dkx = -lam_e^T Ex u_e and dL/dky = -lam_e^T Ey u_e, where u solves
 * A u = f and lam solves A lam = dL/du (A symmetric). */
int cdr_gpu_fe_grad_2d_f64(const double *u, const double *lam, int nx, int ny, int pitch, double *gkx,
                           double *gky, int cell_pitch, cudaStream_t stream);

/* Trilinear elements in 3D: 27-point operator (14 planes) of -div(k grad u), k
 * scalar per cell of an (nz+1) x (ny+1) x (nx+1) cell array (row pitch
 * cell_pitch >= nx+1, k-slices cell_slice >= cell_pitch*(ny+1) apart), cube
 * cells of side 1/(nx+1), Dirichlet zero boundary. */
int cdr_gpu_fe_assemble_3d_f64(const double *k, int cell_pitch, int cell_slice, double *so, int nx, int ny, int nz,
                               int pitch, cudaStream_t stream);

/* ------------------------------------------------------------------------
 * 2D multilevel solver: setup in create (multilevel::setup,
 * include/cedar/multilevel.h:243-265), solve (multilevel::solve, :278-298),
 * vcycle (multilevel::vcycle, :80-84).
 * ------------------------------------------------------------------------ */

/* Mirrors ml_settings (include/cedar/multilevel_settings.h:28-50) plus the GPU options. */
typedef struct cdr_gpu_settings {
	int relaxation;   /* CDR_RELAX_*            "solver.relaxation"   (default point)  */
	int nrelax_pre;   /* "solver.cycle.nrelax-pre"  (default 2)                        */
	int nrelax_post;  /* "solver.cycle.nrelax-post" (default 1)                        */
	int num_levels;   /* "solver.num-levels"  (-1 = from min_coarse)                   */
	int maxiter;      /* "solver.max-iter"    (default 10)                             */
	double tol;       /* "solver.tol"         (default 1e-8)                           */
	int min_coarse;   /* "solver.min_coarse"  (default 3)                              */
	int precision;    /* CDR_PREC_F64 (default) or CDR_PREC_F32_IR                     */
	int use_graph;    /* replay the cycle as a CUDA graph (default 1)                  */
	int line_flags;   /* CDR_LINES_EXACT: sequential line substitutions; CDR_LINES_NOTUNE (default 0) */
	int fuse_coarse;  /* levels with both edges <= this run as one fused kernel (default 32, 0 = off) */
	int krylov;       /* CDR_KRYLOV_NONE (default) or CDR_KRYLOV_FCG; 2D solver only    */
	int coarse_solve; /* CDR_COARSE_BANDED (default) or CDR_COARSE_INVERSE; 2D solver only */
	int fp32_levels;  /* CDR_PREC_F32_IR, 2D solver: the FP32 cycle runs this many finest levels in FP32 and
	                     the coarser ones in FP64 (latency-bound there, so FP64 costs little); 0 = all (default) */
	int cycle;        /* "solver.cycle.type": CDR_CYCLE_V (default) or CDR_CYCLE_F; 2D and 3D solvers (not batched) */
	int krylov_replace; /* CDR_KRYLOV_FCG: form the residual as b - A x every this many iterations and to
	                       confirm convergence, the iterations between update it as r - alpha A p (one pass
	                       over the operator fewer); 0 or 1 (default): every iteration */
	int periodic;     /* "grid.periodic" as a mask: bit 0 x, bit 1 y (default 0).  2D solver with FP64
	                     point relaxation (V or F cycle) and the direct coarse solve; the operator and b
	                     hold the wrap-around couplings and copies of the opposite interior lines in
	                     their ghost lines (examples/basic-2d-ser/periodic.cc) */
	int fp64_fine_iterate; /* CDR_PREC_F32_IR with CDR_KRYLOV_FCG, 2D solver: 1 (default) keeps the FP32
	                          cycle's fine-level iterate in FP64 from the interpolate-add on: the post-smoothing
	                          runs in FP32 on a correction from zero whose right-hand side is the residual of the
	                          FP64 iterate, formed in FP64 arithmetic over the FP32 operator in difference form,
	                          and the preconditioner's output is the FP64 iterate plus that correction.  The
	                          output then carries no FP32 rounding of the iterate itself (of relative size
	                          eps32 |A||x| in the residual, large on high-contrast operators); 0: FP32
	                          throughout */
} cdr_gpu_settings;

typedef struct cdr_gpu_solver cdr_gpu_solver;

int cdr_gpu_settings_default(cdr_gpu_settings *s);

/* Set up the hierarchy from a host fine operator in Cedar's layout
 * (pitch nx+2, nstencil planes).  stream may be 0 (the library creates its own). */
int cdr_gpu_solver_create_2d(const cdr_gpu_settings *s, const double *so_host, int nstencil, int nx, int ny,
                             cudaStream_t stream, cdr_gpu_solver **out);
/* Same from a DEVICE fine operator of the given pitch. */
int cdr_gpu_solver_create_2d_device(const cdr_gpu_settings *s, const double *so_dev, int nstencil, int nx, int ny,
                                    int pitch, cudaStream_t stream, cdr_gpu_solver **out);
/* Replace the fine operator (same size and stencil) and rerun the whole setup
 * on the existing allocations; the captured cycle graphs stay valid. */
int cdr_gpu_solver_resetup_device(cdr_gpu_solver *h, const double *so_dev, int pitch);
int cdr_gpu_solver_destroy(cdr_gpu_solver *h);

/* Solve with HOST buffers in Cedar's layout ((nx+2)*(ny+2) doubles).  x holds the
 * initial guess on entry (Cedar's solve(b) starts from zero: pass zeros).
 * iters (may be null) receives the number of cycles run, hist (may be null) the
 * relative l2 residual after each cycle. */
int cdr_gpu_solver_solve(cdr_gpu_solver *h, const double *b_host, double *x_host, int *iters,
                         double *hist, int maxhist);
/* Same with DEVICE buffers of the given pitch. */
int cdr_gpu_solver_solve_device(cdr_gpu_solver *h, const double *b_dev, double *x_dev, int pitch,
                                int *iters, double *hist, int maxhist);
/* One cycle x <- x + B(b - A x) on DEVICE buffers (multilevel::vcycle). */
int cdr_gpu_solver_vcycle_device(cdr_gpu_solver *h, const double *b_dev, double *x_dev, int pitch);

int cdr_gpu_solver_nlevels(const cdr_gpu_solver *h);
/* Level geometry and device arrays, for tests and tooling.  which: 0 so, 1 x,
 * 2 b, 3 res, 4 sor (point: 1/c; lines: x factors), 5 y factors, 6 ci.  For the
 * FP32 preconditioner arrays add 16 to which. */
int cdr_gpu_solver_level(const cdr_gpu_solver *h, int level, int which, void **ptr, int *nx, int *ny,
                         int *pitch, int *tpitch, int *nstencil);
/* Copy a level array (as returned by cdr_gpu_solver_level, all planes, padded
 * rows) into a host buffer of at least `bytes` bytes. */
int cdr_gpu_solver_level_get(const cdr_gpu_solver *h, int level, int which, void *host, size_t bytes);
/* Setup and solve timings of the last calls (ms, from CUDA events). */
int cdr_gpu_solver_timings(const cdr_gpu_solver *h, double *setup_ms, double *solve_ms);

/* ------------------------------------------------------------------------
 * 3D kernels.  Operators have nstencil planes in the order of
 * include/cedar/3d/base_types.h: 14 for 27-point operators (xxvii_pt: p pw ps b
 * psw pnw bw bnw bn bne be bse bs bsw), 4 for seven-point ones (seven_pt: p pw
 * ps b).  Coarse (Galerkin) operators are always 27-point.
 * A grid of nx*ny*nz interior points has (nx+2)*(ny+2)*(nz+2) entries per
 * plane: rows of `pitch` elements (pitch >= nx+2), k-slices pitch*(ny+2)
 * elements apart, planes pitch*(ny+2)*(nz+2) apart.  Interpolation weights: 26
 * planes on the coarse grid (include/cedar/3d/prolong_op.h).
 * ------------------------------------------------------------------------ */

/* r = b - A x (BMG3_SymStd_residual via include/cedar/3d/residual.h:58); the
 * optional norm is as in the 2D call (scratch of cdr_gpu_norm_scratch_bytes()). */
int cdr_gpu_residual_3d_f64(const double *so, int nstencil, const double *x, const double *b, double *r, int nx,
                            int ny, int nz, int pitch, double *norm_out, void *scratch, cudaStream_t stream);
int cdr_gpu_residual_3d_f32(const float *so, int nstencil, const float *x, const float *b, float *r, int nx, int ny,
                            int nz, int pitch, double *norm_out, void *scratch, cudaStream_t stream);
/* sor = 1/c (BMG3_SymStd_SETUP_recip via include/cedar/3d/relax.h:62). */
int cdr_gpu_setup_recip_3d_f64(const double *so, double *sor, int nx, int ny, int nz, int pitch,
                               cudaStream_t stream);
/* One Gauss-Seidel sweep (BMG3_SymStd_relax_GS via include/cedar/3d/relax.h:96):
 * 27-point: 8 colours, updown CDR_DOWN runs the colours 8..1, CDR_UP 1..8;
 * seven-point: red-black, CDR_UP the points with i+j+k even first, CDR_DOWN
 * the odd ones first (1-based indices). */
int cdr_gpu_relax_point_3d_f64(const double *so, int nstencil, double *x, const double *b, const double *sor, int nx,
                               int ny, int nz, int pitch, int updown, cudaStream_t stream);
int cdr_gpu_relax_point_3d_f32(const float *so, int nstencil, float *x, const float *b, const float *sor, int nx,
                               int ny, int nz, int pitch, int updown, cudaStream_t stream);
/* b_coarse = P^T r_fine (BMG3_SymStd_restrict via src/3d/restrict.cc:29).  The
 * coarse grid must be ((nxf-1)/2+1, (nyf-1)/2+1, (nzf-1)/2+1). */
int cdr_gpu_restrict_3d_f64(const double *ci, const double *r_fine, double *b_coarse, int nxf, int nyf, int nzf,
                            int pitch_f, int nxc, int nyc, int nzc, int pitch_c, cudaStream_t stream);
/* x_fine += P x_coarse + r/c on fine-only points (BMG3_SymStd_interp_add via
 * src/3d/interp.cc:41); so_fine is the fine operator (its p plane is read),
 * res_fine the fine residual (not modified). */
int cdr_gpu_interp_add_3d_f64(const double *ci, const double *x_coarse, const double *res_fine,
                              const double *so_fine, double *x_fine, int nxf, int nyf, int nzf, int pitch_f,
                              int nxc, int nyc, int nzc, int pitch_c, cudaStream_t stream);
/* Operator-induced interpolation weights (BMG3_SymStd_SETUP_interp_OI via
 * include/cedar/3d/interp.h:68), its 27-point or seven-point branch. */
int cdr_gpu_setup_interp_3d_f64(const double *so_fine, int nstencil, double *ci, int nxf, int nyf, int nzf,
                                int pitch_f, int nxc, int nyc, int nzc, int pitch_c, cudaStream_t stream);
/* Galerkin coarse operator P^T A P, 14 planes (BMG3_SymStd_SETUP_ITLI27_ex, or
 * ITLI07_ex for a seven-point fine operator, via include/cedar/3d/coarsen.h:46-58). */
int cdr_gpu_galerkin_3d_f64(const double *so_fine, int nstencil, const double *ci, double *so_coarse, int nxf,
                            int nyf, int nzf, int pitch_f, int nxc, int nyc, int nzc, int pitch_c,
                            cudaStream_t stream);
/* Banded Cholesky of the coarsest operator (BMG3_SymStd_SETUP_cg_LU via
 * include/cedar/3d/solve_cg.h:43): abd holds (nx*(ny+1)+2) * nx*ny*nz doubles;
 * info (device int, may be null) receives the failing column or 0. */
int cdr_gpu_setup_cg_3d_f64(const double *so, int nstencil, int nx, int ny, int nz, int pitch, double *abd,
                            int *info, cudaStream_t stream);
/* x = A^{-1} b with that factor (BMG3_SymStd_SOLVE_cg via src/3d/solve_cg.cc:28). */
int cdr_gpu_solve_cg_3d_f64(const double *abd, double *x, const double *b, int nx, int ny, int nz, int pitch,
                            cudaStream_t stream);

/* ------------------------------------------------------------------------
 * 3D multilevel solver (cdr3::solver, include/cedar/3d/solver.h), 27-point or
 * seven-point fine operator (nstencil 14 or 4).  Same settings struct as 2D; relaxation CDR_RELAX_POINT (8-colour
 * Gauss-Seidel) or CDR_RELAX_PLANE_* (one 2D line-xy V-cycle per plane, red-black
 * over planes; line_flags applies to those 2D cycles).
 * ------------------------------------------------------------------------ */
typedef struct cdr_gpu_solver3 cdr_gpu_solver3;

/* Host fine operator in Cedar's layout (pitch nx+2, nstencil planes). */
int cdr_gpu_solver3_create(const cdr_gpu_settings *s, const double *so_host, int nstencil, int nx, int ny, int nz,
                           cudaStream_t stream, cdr_gpu_solver3 **out);
/* Same from a DEVICE fine operator of the given pitch. */
int cdr_gpu_solver3_create_device(const cdr_gpu_settings *s, const double *so_dev, int nstencil, int nx, int ny,
                                  int nz, int pitch, cudaStream_t stream, cdr_gpu_solver3 **out);
int cdr_gpu_solver3_destroy(cdr_gpu_solver3 *h);
/* Host buffers of (nx+2)*(ny+2)*(nz+2) doubles; as cdr_gpu_solver_solve. */
int cdr_gpu_solver3_solve(cdr_gpu_solver3 *h, const double *b_host, double *x_host, int *iters, double *hist,
                          int maxhist);
/* Device buffers of the given pitch (k-slices pitch*(ny+2) apart). */
int cdr_gpu_solver3_solve_device(cdr_gpu_solver3 *h, const double *b_dev, double *x_dev, int pitch, int *iters,
                                 double *hist, int maxhist);
int cdr_gpu_solver3_nlevels(const cdr_gpu_solver3 *h);
/* which: 0 so, 1 x, 2 b, 3 res, 4 sor, 6 ci (+16: FP32 copies), 100 coarse factor. */
int cdr_gpu_solver3_level(const cdr_gpu_solver3 *h, int level, int which, void **ptr, int *nx, int *ny, int *nz,
                          int *pitch);
int cdr_gpu_solver3_level_get(const cdr_gpu_solver3 *h, int level, int which, void *host, size_t bytes);
int cdr_gpu_solver3_timings(const cdr_gpu_solver3 *h, double *setup_ms, double *solve_ms);

/* ------------------------------------------------------------------------
 * Batches of independent 2D problems of one grid size, solved together (every
 * kernel launch covers the whole batch).  The reference solves such problems
 * one cdr2::solver at a time (include/cedar/2d/solver.h:45-129); each problem
 * here follows multilevel::solve (include/cedar/multilevel.h:278-298) with its
 * own stopping test.  Arrays hold the nb problems back to back: operators nb x
 * nstencil planes, grid functions nb planes, each plane pitch*(ny+2) elements.
 * ------------------------------------------------------------------------ */
typedef struct cdr_gpu_batch2d cdr_gpu_batch2d;

/* Set up nb hierarchies (2D relaxations only) from DEVICE fine operators. */
int cdr_gpu_batch2d_create(const cdr_gpu_settings *s, const double *so_dev, int nstencil, int nx, int ny, int pitch,
                           int nb, cudaStream_t stream, cdr_gpu_batch2d **out);
int cdr_gpu_batch2d_destroy(cdr_gpu_batch2d *h);
/* Solve all problems from the initial guesses in x_dev.  Host arrays of nb:
 * iters receives each problem's cycle count, rel its final relative l2
 * residual, done_ms (may be null) the time from the start of the solve to that
 * problem's last cycle.  A problem's iterate is final once it has met the
 * tolerance; the others keep cycling. */
int cdr_gpu_batch2d_solve_device(cdr_gpu_batch2d *h, const double *b_dev, double *x_dev, int pitch, int *iters,
                                 double *rel, float *done_ms);
int cdr_gpu_batch2d_nlevels(const cdr_gpu_batch2d *h);
int cdr_gpu_batch2d_timings(const cdr_gpu_batch2d *h, double *setup_ms, double *solve_ms);
/* New fine operators (device, the create call's layout at pitch) for the same
 * batch: the hierarchy is set up again (multilevel::setup per problem). */
int cdr_gpu_batch2d_resetup_device(cdr_gpu_batch2d *h, const double *so_dev, int pitch);

/* Independent 2D problems of several grid sizes solved together: nclass size
 * classes, class c holding nb[c] problems of nx[c] x ny[c] points (fine
 * operators so_dev[c], nstencil ns[c], back to back at pitch[c]).  No single
 * reference call: each problem keeps the semantics of its own cdr2::solver
 * (include/cedar/2d/solver.h:45-129), FP32 V-cycles refined in FP64 to its own
 * relative tolerance (settings.precision CDR_PREC_F32_IR, V-cycles, banded
 * coarsest solve).  Every hierarchy level of every problem with the same grid
 * size shares one FP32 array (problems back to back), so one launch of each
 * cycle step covers that level of all problems; the sizes at and below the
 * classes' common fused coarse level run as one launch over all problems (when
 * the classes fuse from different sizes, every level runs with its own
 * launches); the cycle is one CUDA graph on one stream.  Solve: b_dev[c] / x_dev[c] per class
 * at pitch[c] (x holds the initial guesses); iters, rel, done_ms per problem,
 * classes in the caller's order (done_ms may be null). */
typedef struct cdr_gpu_batchmix cdr_gpu_batchmix;
int cdr_gpu_batchmix_create(const cdr_gpu_settings *s, int nclass, const double *const *so_dev, const int *ns,
                            const int *nx, const int *ny, const int *pitch, const int *nb, cudaStream_t stream,
                            cdr_gpu_batchmix **out);
int cdr_gpu_batchmix_destroy(cdr_gpu_batchmix *h);
int cdr_gpu_batchmix_solve_device(cdr_gpu_batchmix *h, const double *const *b_dev, double *const *x_dev,
                                  const int *pitch, int *iters, double *rel, float *done_ms);
int cdr_gpu_batchmix_timings(const cdr_gpu_batchmix *h, double *setup_ms, double *solve_ms);
/* grid sizes shared by the classes' levels; kernel launches of one cycle (its graph) */
int cdr_gpu_batchmix_sizes(const cdr_gpu_batchmix *h);
long long cdr_gpu_batchmix_cycle_launches(const cdr_gpu_batchmix *h);

#ifdef __cplusplus
}
#endif
#endif
