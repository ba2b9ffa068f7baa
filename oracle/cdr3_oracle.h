/* cdr3_oracle.h -- CPU restatement of Cedar's serial 3D BoxMG path.
 * TEST INFRASTRUCTURE ONLY (parity oracle); see cdr3_oracle.c. */
#ifndef CDR3_ORACLE_H
#define CDR3_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif
/* relax: O3_RELAX_POINT or one of the plane relaxations (ml_settings::relax_type,
 * include/cedar/multilevel_settings.h:30-31) */
enum { O3_RELAX_POINT = 0, O3_RELAX_PLANE_XY = 4, O3_RELAX_PLANE_XZ = 5, O3_RELAX_PLANE_YZ = 6, O3_RELAX_PLANE_XYZ = 7 };
enum { O3_XY = 0, O3_XZ = 1, O3_YZ = 2 };
typedef struct {
	int nrelax_pre, nrelax_post, num_levels, maxiter;
	double tol;
	int min_coarse;
	int relax;
	int cycle; /* 0: V-cycle, 1: F-cycle (cycle::fcycle) */
} o3_settings;
typedef struct o3_solver o3_solver;
void o3_residual(const double *so, const double *qf, const double *q, double *res, int II, int JJ, int KK);
void o3_setup_recip(const double *so, double *sor, int II, int JJ, int KK);
void o3_relax_gs(const double *so, const double *qf, double *q, const double *sor, int II, int JJ, int KK, int updown);
void o3_restrict(const double *ci, const double *q, double *qc, int Nx, int Ny, int Nz, int Nxc, int Nyc, int Nzc);
void o3_interp_add(double *q, const double *qc, double *res, const double *so_kp, const double *ci, int iic, int jjc,
                   int kkc, int iif, int jjf, int kkf);
void o3_setup_interp(const double *so, double *ci, int iif, int jjf, int kkf, int iic, int jjc, int kkc);
void o3_galerkin(const double *so, double *soc, const double *ci, int II, int JJ, int KK, int iic, int jjc, int kkc);
int o3_setup_cg(const double *so, int II, int JJ, int KK, double *abd, int nabd1);
void o3_solve_cg(double *q, const double *qf, int II, int JJ, int KK, const double *abd, double *bbd, int nabd1);
double o3_l2norm(const double *r, int II, int JJ, int KK);
int o3_num_levels(int nx, int ny, int nz, int min_coarse);
o3_solver *o3_create(const o3_settings *s, const double *so_fine, int nstncl, int nx, int ny, int nz);
void o3_residual7(const double *so, const double *qf, const double *q, double *res, int II, int JJ, int KK);
void o3_relax_gs7(const double *so, const double *qf, double *q, const double *sor, int II, int JJ, int KK, int updown);
void o3_setup_interp7(const double *so, double *ci, int iif, int jjf, int kkf, int iic, int jjc, int kkc);
void o3_destroy(o3_solver *h);
void o3_vcycle(o3_solver *h, double *x, const double *b);
/* the cycle of the settings (V or F) */
void o3_cycle(o3_solver *h, double *x, const double *b);
int o3_solve(o3_solver *h, const double *b, double *x, double *hist, int maxhist);
int o3_nlevels(const o3_solver *h);
int o3_cg_info(const o3_solver *h);
void o3_level_dims(const o3_solver *h, int l, int *d);
double *o3_level_array(o3_solver *h, int l, int which);
/* one plane-relaxation sweep of direction dir on level l of h (x, b: that level's
 * ghost-inclusive arrays) */
void o3_relax_planes(o3_solver *h, int l, int dir, double *x, const double *b, int updown);
/* the 2D operator of plane ipl (1-based) of direction dir of level l, five planes */
const double *o3_plane_op(o3_solver *h, int l, int dir, int ipl, int *n1, int *n2);
#ifdef __cplusplus
}
#endif
#endif
