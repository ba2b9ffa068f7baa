/*
 * cedar_capi.h -- Cedar's C interface (include/cedar/capi.h of
 * cedar-framework/cedar) over the B200 solvers of libcdrgpu.so.
 *
 * The names, handle types, handle encoding, error codes and argument meaning
 * are the reference's, so that a C or Fortran caller of Cedar links against
 * libcdrgpu.so instead.  Differences, all forced by running one problem on one
 * GPU without MPI:
 *   - a topology is a single-rank grid: nprocx (nprocy, nprocz) must be 1 and
 *     the communicator argument is an opaque value that is kept, not used;
 *   - vectors live in host memory (cedar_vec_baseptr gives the ghost-inclusive
 *     array, i fastest, as in the reference); the solver copies them to the
 *     device and back;
 *   - the solver is the GPU hierarchy of cdr_gpu.h, configured from the same
 *     JSON keys (solver.*, plus the GPU options under "gpu"); the level count
 *     follows cdr2::solver / cdr3::solver (solver.num-levels to override);
 *   - cedar_vec_free accepts vector handles (the reference compares them with
 *     the topology kind and refuses every vector).
 * Each handle is an int: the object kind in the top four bits, the object's
 * 1-based slot below (include/cedar/interface/object.h).  Calls are not
 * thread-safe, as in the reference.
 */
#ifndef CEDAR_CAPI_H
#define CEDAR_CAPI_H

#ifdef __cplusplus
extern "C" {
#endif

/* include/cedar/capi.h:12-24 */
#define CEDAR_SUCCESS     0
#define CEDAR_ERR_TOPO    1
#define CEDAR_ERR_KIND    2
#define CEDAR_ERR_HANDLE  3
#define CEDAR_ERR_MAT     4
#define CEDAR_ERR_VEC     5
#define CEDAR_ERR_DIM     6
#define CEDAR_ERR_STENCIL 7
#define CEDAR_ERR_SOLVER  8
#define CEDAR_ERR_CONFIG  9
#define CEDAR_ERR_FNAME   10
#define CEDAR_ERR_CONFIG_PATH 11
#define CEDAR_ERR_OTHER   12

typedef double cedar_real;        /* include/cedar/ctypes.h */
typedef unsigned int cedar_len;

typedef int cedar_config;
typedef int cedar_topo;
typedef int cedar_mat;
typedef int cedar_vec;
typedef int cedar_solver;
/* the caller's communicator (MPI_Comm cast to a pointer-sized integer, or 0) */
typedef long cedar_comm;

/* include/cedar/capi.h:32-36 */
#define CEDAR_TOPO_NULL ((cedar_topo) 0x10000000)
#define CEDAR_MAT_NULL ((cedar_mat) 0x30000000)
#define CEDAR_SOLVER_NULL ((cedar_solver) 0x20000000)
#define CEDAR_VEC_NULL ((cedar_vec) 0x40000000)
#define CEDAR_CONFIG_NULL ((cedar_config) 0x50000000)

/* stencil directions (include/cedar/2d/base_types.h, include/cedar/3d/base_types.h) */
typedef enum {
	BMG2_C = 0, BMG2_W = 1, BMG2_S = 2, BMG2_SW = 3, BMG2_NW = 4,
	BMG2_SE = 5, BMG2_N = 6, BMG2_NE = 7, BMG2_E = 8
} bmg2_dir;

typedef struct {
	unsigned int i;  /* 0-based global interior index */
	unsigned int j;
	bmg2_dir dir;
} cedar_coord_2d;

typedef struct {
	unsigned int i;
	unsigned int j;
	unsigned int k;
	int dir;         /* storage plane of the 3D stencil (seven_pt 0-3, xxvii_pt 0-13) */
} cedar_coord_3d;

typedef enum { CEDAR_STENCIL_FIVE_PT, CEDAR_STENCIL_NINE_PT } cedar_stencil_2d;
typedef enum { CEDAR_STENCIL_SEVEN_PT, CEDAR_STENCIL_XXVII_PT } cedar_stencil_3d;

/* Logging (include/cedar/capi.h:47): accepted; messages go to cdr_gpu_last_error. */
int cedar_log_init(cedar_config conf);

/* Config from a JSON file (include/cedar/capi.h:59-84). */
int cedar_config_create(const char *fname, cedar_config *newconfig);
int cedar_config_get_int(cedar_config conf, const char *confpath, int *val);
int cedar_config_free(cedar_config *conf);

/* Grid topology (include/cedar/capi.h:100-142): ngx x ngy (x ngz) interior
 * points; lnx[0] (lny[0], lnz[0]) must equal them (one rank). */
int cedar_topo_create2d(cedar_comm comm, unsigned int ngx, unsigned int ngy, unsigned int lnx[], unsigned int lny[],
                        int nprocx, int nprocy, cedar_topo *newtopo);
int cedar_topo_create3d(cedar_comm comm, unsigned int ngx, unsigned int ngy, unsigned int ngz, unsigned int lnx[],
                        unsigned int lny[], unsigned int lnz[], int nprocx, int nprocy, int nprocz,
                        cedar_topo *newtopo);
int cedar_topo_free(cedar_topo *topo);

/* Vectors (grid functions, include/cedar/capi.h:153-233). */
int cedar_vec_create2d(cedar_topo topo, cedar_vec *vec);
int cedar_vec_create3d(cedar_topo topo, cedar_vec *vec);
int cedar_vec_baseptr(cedar_vec vec, cedar_real **base);
int cedar_vec_len2d(cedar_vec vec, cedar_len *ilen, cedar_len *jlen);
int cedar_vec_len3d(cedar_vec vec, cedar_len *ilen, cedar_len *jlen, cedar_len *klen);
int cedar_vec_getdim(cedar_vec vec, int *nd);
int cedar_vec_free(cedar_vec *vec);

/* Matrices (stencil operators, include/cedar/capi.h:276-367).  cedar_mat_set2d
 * takes vertex-based entries A[(i,j), neighbour in dir] and stores them in
 * BoxMG's symmetric form (negated off-diagonals; E, N, NE, SE, NW moved to
 * the neighbour's W, S, SW, NW planes; five-point operators refuse the
 * diagonal directions with CEDAR_ERR_STENCIL). */
int cedar_mat_create2d(cedar_config conf, cedar_topo topo, cedar_stencil_2d sten_type, cedar_mat *mat);
int cedar_mat_create3d(cedar_config conf, cedar_topo topo, cedar_stencil_3d sten_type, cedar_mat *mat);
int cedar_mat_set2d(cedar_mat mat, unsigned int nvals, cedar_coord_2d coords[], cedar_real vals[]);
int cedar_mat_set3d(cedar_mat mat, unsigned int nvals, cedar_coord_3d coords[], cedar_real vals[]);
/* y = mat * x (on the GPU) */
int cedar_matvec(cedar_mat mat, cedar_vec x, cedar_vec y);
int cedar_mat_gettopo(cedar_mat mat, cedar_topo *topo);
/* text dump of the operator: op-0-0.txt (2D, the reference's row format) or so-0.0.0 (3D) */
int cedar_mat_dump(cedar_mat mat);
int cedar_mat_free(cedar_mat *mat);

/* Solver (include/cedar/capi.h:380-403): setup on the GPU from the matrix and
 * its config; run solves mat x = b from the initial guess in x. */
int cedar_solver_create(cedar_mat mat, cedar_solver *solver);
int cedar_solver_run(cedar_solver solver, cedar_vec x, cedar_vec b);
int cedar_solver_destroy(cedar_solver *solver);
/* the reference implements destroy under this name (src/2d/interface/c/solver.cc) */
int cedar_solver_free(cedar_solver *solver);

#ifdef __cplusplus
}
#endif
#endif
