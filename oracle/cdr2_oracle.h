/*
 * cdr2_oracle.h -- CPU restatement of Cedar's serial 2D BoxMG path.
 * TEST INFRASTRUCTURE ONLY (parity oracle); see cdr2_oracle.c.
 */
#ifndef CDR2_ORACLE_H
#define CDR2_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { O2_RELAX_POINT = 0, O2_RELAX_LINE_X = 1, O2_RELAX_LINE_Y = 2, O2_RELAX_LINE_XY = 3 };
enum { O2_ARR_SO = 0, O2_ARR_X, O2_ARR_B, O2_ARR_RES, O2_ARR_SOR0, O2_ARR_SOR1, O2_ARR_CI, O2_ARR_ABD };

/* mirrors ml_settings, include/cedar/multilevel_settings.h:28-50 */
typedef struct {
	int relax;
	int nrelax_pre;
	int nrelax_post;
	int num_levels;
	int maxiter;
	double tol;
	int min_coarse;
	int cycle; /* 0: V-cycle, 1: F-cycle (ml_settings::cycle_type) */
	int bc;    /* boundary-condition code (BMG_get_bc of the periodic mask): 0 definite, 2 periodic x,
	              1 periodic y, 3 both; periodic codes need point relaxation */
} o2_settings;

typedef struct o2_solver o2_solver;

int o_dpttrf(int n, double *d, double *e);
void o_dpttrs(int n, const double *d, const double *e, double *b);
int o_dpbtrf_u(int n, int kd, double *ab, int ldab);
void o_dpbtrs_u(int n, int kd, const double *ab, int ldab, double *x);

void o2_residual(const double *so, const double *qf, const double *q, double *res, int II, int JJ, int ifd);
void o2_setup_recip(const double *so, double *sor, int II, int JJ);
void o2_relax_gs(const double *so, const double *qf, double *q, const double *sor, int II, int JJ, int ifd, int updown);
int o2_setup_lines_x(const double *so, double *sor, int Nx, int Ny);
int o2_setup_lines_y(const double *so, double *sor, int Nx, int Ny);
void o2_relax_lines_x(const double *so, const double *qf, double *q, const double *sor, int II, int JJ, int ifd, int updown);
void o2_relax_lines_y(const double *so, const double *qf, double *q, const double *sor, int II, int JJ, int ifd, int updown);
void o2_restrict(const double *ci, const double *q, double *qc, int Nx, int Ny, int Nxc, int Nyc);
void o2_interp_add(double *q, const double *qc, double *res, const double *so_ko, const double *ci,
                   int IIC, int JJC, int IIF, int JJF);
void o2_setup_interp(const double *so, double *ci, int IIF, int JJF, int IIC, int JJC, int ifd);
void o2_setup_galerkin(const double *so, double *soc, const double *ci, int IIF, int JJF, int IIC, int JJC, int ifd);
int o2_setup_cg(const double *so, int II, int JJ, int nstncl, double *abd, int nabd1);
void o2_solve_cg(double *q, const double *qf, int II, int JJ, const double *abd, double *bbd, int nabd1);
double o2_l2norm(const double *r, int II, int JJ);
double o2_inf_norm(const double *r, int II, int JJ);

int o2_num_levels(int nx, int ny, int min_coarse);
o2_solver *o2_create(const o2_settings *s, const double *so_fine, int nstncl, int nx, int ny);
void o2_destroy(o2_solver *h);
void o2_vcycle(o2_solver *h, double *x, const double *b);
void o2_cycle(o2_solver *h, double *x, const double *b);
void o2_cycle(o2_solver *h, double *x, const double *b);
int o2_solve(o2_solver *h, const double *b, double *x, double *hist, int maxhist);
/* Flexible CG preconditioned by one cycle (residual formed every `replace`
 * iterations and to confirm convergence); returns the iterations run. */
int o2_solve_fcg(o2_solver *h, const double *b, double *x, int replace, double *hist, int maxhist);
int o_num_threads(void);
/* periodic branches (cdr2_periodic.c) */
int o2_bc_code(int per_mask);
void o2_relax_gs_per(const double *so, const double *qf, double *q, const double *sor, int II, int JJ, int ifd,
                     int updown, int ipn);
void o2_restrict_per(const double *ci, double *q, double *qc, int Nx, int Ny, int Nxc, int Nyc, int ipn);
void o2_interp_add_per(double *q, const double *qc, double *res, const double *so_ko, const double *ci, int IIC,
                       int JJC, int IIF, int JJF, int ipn);
void o2_setup_galerkin_per(const double *so, double *soc, const double *ci, int IIF, int JJF, int IIC, int JJC,
                           int ifd, int ipn);
void o2_setup_interp_per(const double *so, double *ci, int IIF, int JJF, int IIC, int JJC, int ifd, int ipn);
int o_dpotf2_u(int n, double *a, int lda);
void o_dpotrs_u(int n, const double *a, int lda, double *b);
int o2_setup_cg_per(const double *so, int II, int JJ, int nstncl, double *abd, int ipn);
void o2_solve_cg_per(double *q, const double *qf, int II, int JJ, const double *abd, double *bbd, int ipn);
void o_set_threads(int n);
int o2_nlevels(const o2_solver *h);
int o2_info(const o2_solver *h, int which);
void o2_level_dims(const o2_solver *h, int l, int *dims);
double *o2_level_array(o2_solver *h, int l, int which);
void o2_abd_dims(const o2_solver *h, int *dims);

#ifdef __cplusplus
}
#endif
#endif
