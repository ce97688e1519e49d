/*
 * leq_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of MFIX 2016-1's linear-equation path (SOLVE_LIN_EQ ->
 * LEQ_BICGS -> LEQ_MATVEC / LEQ_MSOLVE / DGTSV / DOT_PRODUCT_PAR), used as the
 * parity checker for the CUDA library and as the timed CPU baseline.  Only the
 * tests, the smoke check and the benchmark's CPU-baseline leg may load it; the
 * product library never links or calls it.
 *
 * Parity pinning: the reference publishes no golden vectors for this path and
 * cannot be compiled here (Fortran).  The DGTSV restatement is pinned
 * bit-for-bit against LAPACK's dgtsv (scipy), and the solver against
 * known-answer systems built with the recipe of model/test_lin_eq.f:63-117.
 *
 * Geometry follows a serial, non-cyclic MFIX box: cells carry the one-cell wall
 * layer (model/set_max2.f:48-66), the linear index puts J fastest
 * (model/include/functions.inc:37-42, model/dmp_modules/gridmap_mod.f:553-556)
 * and neighbour offsets clamp at the array edge (model/set_increments.f:80-109).
 * The seven diagonals are stored the way Fortran stores A_M(DIMENSION_3,-3:3):
 * diagonal d (d = -3..3) of cell ijk sits at a[(d+3)*n + ijk].
 */
#ifndef LEQ_ORACLE_H
#define LEQ_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int imax2, jmax2, kmax2; /* cell extents including the wall layer */
    int do_k;                /* 0: two-dimensional (kmax2 == 1) */
    int64_t n;               /* DIMENSION_3 */
    int cyclic;              /* 1 CYCLIC_X, 2 CYCLIC_Y, 4 CYCLIC_Z: the interior cells' neighbours wrap */
    int pad;
} orc_geom;

typedef struct {
    int ier;          /* IER as LEQ_BICGS0 leaves it */
    int iterations;   /* value of the reference's ITER counter at exit */
    int iter_tot_add; /* what the call adds to ITER_TOT(VNO) */
    int exit_kind;    /* 0 converged-by-Rnorm, 1 Snorm<=TOLMIN, 2 rho==0, 3 itmax, 4 singular row, -1 error */
    int line_info_skips; /* IKSWEEP/ISWEEP lines left unchanged because DGTSV INFO != 0 */
    double rnorm0, rnorm;
} orc_stats;

/* rows: MATVEC, dot, DGTSV, sweeps */
void orc_matvec(const orc_geom *g, const double *a, const double *x, double *y);
double orc_dot(const double *x, const double *y, int64_t n);
int orc_dgtsv(int n, double *dl, double *d, double *du, double *b);
int orc_iksweep(const orc_geom *g, int i, int k, double *var, const double *a, const double *b);
int orc_isweep(const orc_geom *g, int i, double *var, const double *a, const double *b);
int orc_jksweep(const orc_geom *g, int j, int k, double *var, const double *a, const double *b);
int orc_ijsweep(const orc_geom *g, int i, int j, double *var, const double *a, const double *b);
int orc_msolve(const orc_geom *g, const double *b, const double *a, double *var, const char *sweep,
               int *skips);
void orc_msolve1(const orc_geom *g, const double *b, const double *a, double *var);
int orc_scale(const orc_geom *g, double *a, double *b);
void orc_scale_diag(const orc_geom *g, double *a, double *b);

/* Rtilde's random stream: counter-based splitmix64, the same on CPU and GPU */
double orc_uniform(uint64_t seed, uint64_t tag, uint64_t idx);

/* LEQ_BICGS(VNAME,VNO,VAR,A_M,B_M,CMETHOD,TOL,PC,ITMAX,IER) on one phase slice */
int orc_leq_bicgs(const orc_geom *g, double *var, double *a, double *b, const char *sweep,
                  double tol, const char *pc, int itmax, uint64_t rt_seed, orc_stats *st);

/* MINIMIZE_DOTPRODUCTS = .TRUE. with ICHECK_BICGS = icheck (model/leq_bicgs.f:372,411,439):
 * no Snorm exit, the Rnorm test every icheck-th iteration. */
int orc_leq_bicgs_icheck(const orc_geom *g, double *var, double *a, double *b, const char *sweep, double tol,
                         const char *pc, int itmax, uint64_t rt_seed, int icheck, orc_stats *st);

/* Same algorithm with a cap on the number of iterations actually executed (timing samples). */
int orc_leq_bicgs_sample(const orc_geom *g, double *var, double *a, double *b, const char *sweep,
                         double tol, const char *pc, int itmax, uint64_t rt_seed, int max_exec,
                         orc_stats *st);

/* LEQ_CG(VNAME,VNO,VAR,A_M,B_M,CMETHOD,TOL,PC,ITMAX,IER) on one phase slice (METHOD 5) */
int orc_leq_cg(const orc_geom *g, double *var, double *a, double *b, const char *sweep, double tol,
               const char *pc, int itmax, orc_stats *st);

/* LEQ_GMRES (METHOD 3, one restart cycle of ITMAX steps, left-preconditioned by
 * LEQ_MSOLVE with the sweep letters; A and B are not scaled).  IER 0 or 1. */
int orc_leq_gmres(const orc_geom *g, double *var, const double *a, const double *b, const char *sweep, double tol,
                  int itmax, orc_stats *st);

/* LEQ_SOR (METHOD 1): one point-Jacobi step after scaling each row by 1/A(0);
 * st->iter_tot_add is the value ITER_TOT(VNO) is set to (ITMAX + 1). */
int orc_leq_sor(const orc_geom *g, double *var, double *a, double *b, int itmax, orc_stats *st);

/* true residual ||b - A x||_2 in long double */
double orc_true_resid(const orc_geom *g, const double *a, const double *b, const double *x);

/* FP64 "truth" solve: BiCGSTAB + LINE/RSRS restarted on the true residual until
 * ||b-Ax|| <= rtol * ||b-A x0|| (long-double residuals). Returns restarts used or -1. */
int orc_truth_solve(const orc_geom *g, const double *a, const double *b, double *x, double rtol,
                    int max_iter, uint64_t rt_seed, double *final_rel);
/* The same refinement from the guess in x, stopping at ||b-Ax|| <= rtol * r0 for a
 * given r0 (e.g. ||b|| for the system's zero initial guess). */
int orc_truth_refine(const orc_geom *g, const double *a, const double *b, double *x, double r0, double rtol,
                     int max_iter, uint64_t rt_seed, double *final_rel);

/* Pressure-correction system of the gas phase, A_M(:,:,0) / B_M(:,0) / B_MMAX(:,0),
 * as CONV_PP_G (model/conv_pp_g.f:33-182) and SOURCE_PP_G (model/source_pp_g.f:18-214)
 * build it for an incompressible run (RO_G0 defined) on a Cartesian grid without
 * shear: face coefficients from the face densities and areas, the continuity
 * residual and its largest term, the D_E/D_N/D_T factors, the solids phases
 * that are not close packed, the centre coefficient, identity rows outside the
 * fluid, the links to pressure-flow cells cut, and the reference cell IJK_P_G.
 * Phase arrays are column-major: D_E(DIMENSION_3, 0:MMAX) and ROP_SE(DIMENSION_3,
 * 1:MMAX) with phase m at offset m*n and (m-1)*n.  ijk_p_g is 1-based, <= 0 when
 * undefined.  a is A_M(DIMENSION_3,-3:3), b and bmmax have n entries. */
typedef struct {
    const int *flag;
    const double *rop_ge, *rop_gn, *rop_gt, *ayz, *axz, *axy, *u_g, *v_g, *w_g;
    const double *rop_g, *rop_go, *vol, *sum_r_g, *d_e, *d_n, *d_t;
    int mmax;
    const int *close_packed;
    const double *rop_se, *rop_sn, *rop_st, *u_s, *v_s, *w_s, *rop_s, *rop_so, *sum_r_s;
    double odt;
    long long ijk_p_g;
} orc_pp_fields;
void orc_conv_source_pp_g(const orc_geom *g, const orc_pp_fields *f, double *a, double *b, double *bmmax);

/* CALC_RESID_PP (model/calc_resid.f:391-534), serial: RESID of B over the fluid
 * cells (|B| summed in cell order) with normalization `norm`. */
double orc_calc_resid_pp(const orc_geom *g, const int *flag, const double *b, double norm);

/* DO_TRANSPOSE: LEQ_MSOLVEt (model/leq_bicgst.f:978-1177) on the same A_M values,
 * and LEQ_BICGSt's solve: LEQ_BICGS0's iteration with LEQ_MSOLVEt, A scaled in a
 * copy (a is left as given), B scaled in place. */
int orc_msolve_t(const orc_geom *g, const double *b, const double *a, double *var, const char *sweep, int *skips);
int orc_leq_bicgst(const orc_geom *g, double *var, const double *a, double *b, const char *sweep, double tol,
                   const char *pc, int itmax, uint64_t rt_seed, int minimize, orc_stats *st);

int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
