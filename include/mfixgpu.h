/*
 * mfixgpu.h -- C ABI of the B200 replacement for MFIX's linear-equation hot
 * path, SOLVE_LIN_EQ -> LEQ_BICGS (MFIX 2016-1).
 *
 * A Fortran host binds these through ISO_C_BINDING (fortran/mfixgpu_mod.f90)
 * or, for mfixgpu_solve_lin_eq_, through gfortran's implicit calling
 * convention.  Arrays are passed the way the reference passes them: A_M is the
 * whole A_M(DIMENSION_3,-3:3,0:DIMENSION_M) array in Fortran (column-major)
 * order and M selects the phase, B_M is B_M(DIMENSION_3,0:DIMENSION_M).
 * Plain pointers and sizes only; no exceptions cross the boundary.
 *
 * Error convention: the reference's IER values (0 converged, -1 not converged
 * but below 0.2*Rnorm0, -2 breakdown / singular row, model/leq_bicgs.f:189-233,
 * 485-495) plus the codes below, all <= -10, where the reference would stop
 * the run through MFIX_EXIT.
 */
#ifndef MFIXGPU_H
#define MFIXGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MFIXGPU_ERR_UNSUPPORTED (-10) /* METHOD/PC/SWEEP/geometry not served (the reference: MFIX_EXIT) */
#define MFIXGPU_ERR_NOMEM (-11)       /* device memory */
#define MFIXGPU_ERR_DGTSV (-12)       /* DGTSV INFO != 0 in a JK/IJ sweep (model/leqsol_mod.f:991-996) */
#define MFIXGPU_ERR_CUDA (-13)        /* CUDA runtime error */
#define MFIXGPU_ERR_ARGS (-14)        /* inconsistent arguments */
#define MFIXGPU_ERR_INCOMPLETE (-15)  /* solve stopped without a verdict */
#define MFIXGPU_ERR_NOGEOM (-16)      /* mfixgpu_init_geometry was not called */
#define MFIXGPU_ERR_CANCELLED (-17)   /* serving: the request was withdrawn before it was admitted */

/* ---------------------------------------------------------------- drop-in */

/* Registers the box geometry that SOLVE_LIN_EQ reads from modules: IMAX2,
 * JMAX2, KMAX2 (model/set_max2.f:48-135), DO_K, DIMENSION_3
 * (model/set_param.f:98) and DIMENSION_M.  Call once after SET_INCREMENTS.
 * Only the serial, non-cut-cell box is served: neighbour offsets clamp at the
 * array edge as in model/set_increments.f:80-109, or wrap along the cyclic axes
 * registered by mfixgpu_init_cyclic.  Returns 0 or MFIXGPU_ERR_ARGS. */
int mfixgpu_init_geometry(const int *imax2, const int *jmax2, const int *kmax2, const int *do_k,
                          const int64_t *dimension_3, const int *dimension_m);

/* CYCLIC_X, CYCLIC_Y, CYCLIC_Z (nonzero = .TRUE.) of a serial run, registered
 * after mfixgpu_init_geometry (which resets them): the neighbour increments of
 * the interior cells wrap along those axes as SET_INCREMENTS builds them
 * (model/set_increments.f:73-113 with IMAP_C(IMAX2) = IMIN1, IMAP_C(IMIN2) = IMAX1,
 * model/dmp_modules/gridmap_mod.f:496-503), in LEQ_MATVEC and in the
 * right-hand sides of the line sweeps; the lines themselves stay open
 * tridiagonals, as LEQ_IKSWEEP solves them (model/leqsol_mod.f:907-909).  CYCLIC_Z
 * is ignored in 2-D.  Returns 0, MFIXGPU_ERR_ARGS or MFIXGPU_ERR_NOGEOM. */
int mfixgpu_init_cyclic(const int *cyclic_x, const int *cyclic_y, const int *cyclic_z);

/* SOLVE_LIN_EQ(VNAME, VNO, VAR, A_M, B_M, M, ITMAX, METHOD, SWEEP, TOL1, PC, IER),
 * model/solve_lin_eq.f:17-78, in gfortran's convention: every argument by
 * reference, CHARACTER lengths appended by value.  Served: METHOD 1 (LEQ_SOR,
 * :133-135, model/leq_sor.f: rows scaled by 1/A(0), one point-Jacobi step,
 * ITER_TOT(VNO) set to ITMAX+1, IER left as passed); METHOD 2 (BiCGSTAB,
 * :137-153); METHOD 3 (GMRES, :156-158, model/leq_gmres.f: one restart cycle of
 * ITMAX steps, left-preconditioned by the sweeps, PC ignored, A/B not scaled,
 * IER 0 or 1, FP64); METHOD 4 (:161-171: BiCGSTAB, and on IER -2 GMRES from its
 * result with IER reset to 0); METHOD 5 (CG, :173-176, model/leq_cg.f, FP64).
 * "precision" applies to the BiCGSTAB solves only.  Other values return
 * MFIXGPU_ERR_UNSUPPORTED (the reference stops in MFIX_EXIT).
 * As in model/leq_bicgs.f:194-233 (BiCGSTAB: rows divided by max|A(ijk,:)|) and
 * model/leq_cg.f:197-211 (CG: rows divided by A(ijk,0)), A_M(:,:,M) and B_M(:,M)
 * come back unit-scaled (option "write_back_ab"). */
void mfixgpu_solve_lin_eq_(const char *vname, const int *vno, double *var, double *a_m, double *b_m,
                           const int *m, const int *itmax, const int *method, const char *sweep,
                           const double *tol1, const char *pc, int *ier, size_t vname_len, size_t sweep_len,
                           size_t pc_len);

/* The same call with values and explicit lengths, for a BIND(C) interface. */
void mfixgpu_solve_lin_eq(const char *vname, int vname_len, int vno, double *var, double *a_m, double *b_m,
                          int m, int itmax, int method, const char *sweep, int sweep_len, double tol1,
                          const char *pc, int pc_len, int *ier);

/* Batching the SIMPLE loop's independent SOLVE_LIN_EQ calls (no reference
 * counterpart).  The per-phase calls of one transport equation solve
 * independent slices A_M(:,:,M) / B_M(:,M) back to back (for example the U_g and
 * U_s(M) calls of model/solve_vel_star.f:308-331); a caller that replaces them by
 * mfixgpu_solve_lin_eq_defer_ (the same dummy list and convention as
 * mfixgpu_solve_lin_eq_) and then calls mfixgpu_solve_lin_eq_flush solves them
 * as one batch, each with the result it gets alone.  A deferred call is checked
 * at once (a failing check sets its IER at once); a METHOD 2 call with red/black
 * sweeps is queued with IER = MFIXGPU_ERR_INCOMPLETE, any other call is solved at
 * once.  Until the flush the arrays and IER must stay in place and untouched.
 * The flush solves the queue, one batch per (PC, SWEEP), writes every IER, adds
 * to ITER_TOT, and returns 0 or the first error code (also written to the IER of
 * every call of the batch that failed). */
void mfixgpu_solve_lin_eq_defer_(const char *vname, const int *vno, double *var, double *a_m, double *b_m,
                                 const int *m, const int *itmax, const int *method, const char *sweep,
                                 const double *tol1, const char *pc, int *ier, size_t vname_len, size_t sweep_len,
                                 size_t pc_len);
int mfixgpu_solve_lin_eq_flush(void);
int mfixgpu_solve_lin_eq_pending(void); /* calls queued */

/* ITER_TOT(VNO) of MODULE leqsol (model/leqsol_mod.f:17), 1-based VNO in
 * 1..10 (DIM_EQS, model/param_mod.f:97); the accounting of
 * model/leq_bicgs.f:458,491. */
int mfixgpu_iter_tot(int vno);
void mfixgpu_reset_iter_tot(void);

typedef struct {
    int ier;
    int iterations;     /* the reference's ITER at exit (mixed form: inner iterations) */
    int iter_tot_add;
    int exit_kind;      /* 0 Rnorm test, 1 Snorm<=TOLMIN, 2 rho=0, 3 ITMAX, 4 singular row, 5 error */
    int line_skips;     /* J-lines left unchanged on DGTSV INFO != 0 (model/leqsol_mod.f:910-914) */
    int line_fallbacks; /* J-lines solved by the sequential pivoting DGTSV path */
    int outer_steps;    /* mixed form: FP64 refinement steps */
    int pad;
    double rnorm0, rnorm;
    double seconds;     /* wall time of the call, copies included */
    double device_ms;   /* device time of the solve (CUDA events), copies excluded */
    double jline_ms;    /* summed J-line sweep kernel time (option "time_kernels") */
    int jline_launches; /* J-line sweep launches timed */
    int fp64_fallback;  /* mixed form: 1 when the FP32 iteration stalled and the FP64 drop-in re-solved;
                           after mfixgpu_batch_solve, the number of such systems */
    long long kernel_launches; /* kernels of this library launched by the solve */
    int mixed_iterations; /* mixed form: FP32 iterations spent before an FP64 re-solve */
    int deflated;       /* mixed form: 1 when the near-null mode was deflated (option "deflate");
                           after mfixgpu_batch_solve, the number of deflated systems */
} mfixgpu_stats;

int mfixgpu_last_stats(mfixgpu_stats *out);

/* With option "time_kernels" set: the summed launch durations (ms, CUDA events)
 * and launch counts of the last solve or batch per kernel class, in this order:
 * 0 J-line half-sweeps (LINE preconditioner), 1 P update, 2 V = A*Phat with
 * alpha, 3 S update with Snorm, 4 T = A*Shat with omega, 5 X/R update with
 * Rnorm and rho, 6 mixed form's FP64 reliable update, 7 copies / DIAG /
 * sequential line sweeps.  Fills up to max_classes entries of each non-NULL
 * array and returns the number of classes (8). */
int mfixgpu_last_kernel_times(double *ms, long long *launches, int max_classes);
const char *mfixgpu_last_error(void);

/* Options (no reference counterpart; defaults reproduce the reference):
 *   "precision"      0 FP64 drop-in (default), 1 FP32 BiCGSTAB with FP64 solution accumulation,
 *                    FP64 dot products and FP64 reliable residual updates; a system whose FP32
 *                    iteration diverges or stalls is re-solved by the FP64 drop-in
 *   "mixed_growth"   mixed form: hand over to FP64 when a true residual exceeds this multiple of
 *                    the best one seen (default 10)
 *   "mixed_stalls"   mixed form: hand over after this many reliable updates without a 10% gain (default 6)
 *   "mixed_min_margin" mixed form: a system whose smallest diagonal-dominance margin,
 *                    min over rows of |sum of A's row| / |A(0)|, is below this (pressure correction)
 *                    is deflated, or with "deflate" 0 solved by the FP64 drop-in from the start
 *                    (default 1e-4; 0 never)
 *   "deflate"        mixed form, systems below mixed_min_margin: 1 (default) the FP32 inner iteration's
 *                    preconditioner also solves the constant mode over the coupled rows exactly
 *                    (Phat = M^{-1} P + c z, z = 1 on rows with a nonzero neighbour coefficient,
 *                    c = z^T P / z^T A z), which keeps it converging on near-singular operators;
 *                    0: such systems go to the FP64 drop-in
 *   "do_transpose"   0 (default) / 1: the reference's DO_TRANSPOSE keyword (model/solve_lin_eq.f:139-150):
 *                    METHOD 2 runs LEQ_BICGSt (model/leq_bicgst.f), i.e. LEQ_BICGS0's iteration on a
 *                    transposed copy of A_M: A_M comes back unscaled and B_M scaled, and LEQ_MSOLVEt's
 *                    letters apply (2-D: I only; 3-D: R, I, K; an odd IMAX2 with R returns
 *                    MFIXGPU_ERR_UNSUPPORTED)
 *   "replace_every"  mixed form, deflated systems: the FP32 residual is replaced by the FP64 true
 *                    residual at least every this many inner iterations (default 20; 0: only after
 *                    the inner_tol drop)
 *   "minimize_dotproducts" 0 (default) / 1: the reference's MINIMIZE_DOTPRODUCTS for METHOD 2 in
 *                    FP64 (model/leq_bicgs.f:372,411,439): no Snorm exit, Rnorm formed and tested
 *                    every "icheck_bicgs" iterations (every fifth with do_transpose); the mixed
 *                    form decides convergence on its FP64 residual and ignores it
 *   "icheck_bicgs"   ICHECK_BICGS, >= 1 (default 1)
 *   "restart_growth" mixed form, deflated systems: when a true residual exceeds this multiple of the
 *                    best one, the FP32 Krylov process restarts from the true residual (default 100;
 *                    0: never)
 *   "staged_matvec"  mixed form: 2 (default) the FP32 matvecs stream their operands into shared memory
 *                    by bulk copies, x's i/k neighbours read through L2; 1: x's i/k neighbour lines
 *                    staged too; 0: per-thread register loads (all three give the same products and
 *                    sums)
 *   "write_back_ab"  1 (default) copy the scaled A_M/B_M slices back
 *   "rtilde_seed"    seed of the Rtilde random stream (replaces RANDOM_NUMBER, model/leq_bicgs.f:298)
 *   "inner_tol"      mixed form: drop of the FP32 residual between FP64 reliable updates (default 1e-2)
 *   "check_every"    iterations between host polls of convergence (default 4)
 *   "use_graph"      1 (default) replay the iteration body as a CUDA graph
 *   "time_kernels"   1: time every J-line sweep launch with CUDA events (no graph replay)
 *   "autotune"       1 (default): lanes per J-line picked by measurement for the new line lengths of a
 *                    solve or batch (one lanes-per-line value timed on all their lines at once)
 *   "line_lanes"     0 (default) automatic, else lanes per J-line (1..32, rounded down to a power of two)
 * Returns 0, or MFIXGPU_ERR_ARGS for an unknown name. */
int mfixgpu_set_option(const char *name, double value);
double mfixgpu_get_option(const char *name);

/* Autotuner of the J-line kernel (no reference counterpart): its choices,
 * keyed by precision and line length, are read from and written to the JSON
 * file at `path` (NULL or "" keeps them in memory only). */
int mfixgpu_autotune_cache(const char *path);
/* Copies up to max_entries (element bytes, line length, lanes per line) triples
 * into out[3*i..3*i+2]; returns the number of entries recorded. */
int mfixgpu_autotune_table(int *out, int max_entries);

/* Releases device memory and the per-device engine. */
void mfixgpu_finalize(void);

/* ---------------------------------------------------------------- single routines on device arrays */

typedef struct {
    int imax2, jmax2, kmax2, do_k;
    int64_t dimension_3;
    int cyclic;  /* 1 CYCLIC_X | 2 CYCLIC_Y | 4 CYCLIC_Z (0: the clamped box) */
    int pad;
} mfixgpu_geom;

/* LEQ_MATVEC(VNAME, VAR, A_M, AVAR), model/leqsol_mod.f:103-265: avar = A*var. */
int mfixgpu_leq_matvec(const mfixgpu_geom *g, const double *a_dev, const double *var_dev, double *avar_dev);

/* LEQ_MSOLVE / LEQ_MSOLVE1 / LEQ_MSOLVE0 (model/leqsol_mod.f:286-749) chosen by
 * PC as in model/leq_bicgs.f:74-87: var = M^{-1} b.  sweep and pc are 4
 * characters, blank padded. */
int mfixgpu_leq_msolve(const mfixgpu_geom *g, const double *b_dev, const double *a_dev, double *var_dev,
                       const char *sweep, const char *pc);

/* DOT_PRODUCT_PAR(R1, R2), model/leqsol_mod.f:1094-1201, serial semantics
 * (the whole array): *out = sum r1*r2, reduced in a fixed order. */
int mfixgpu_dot_product_par(const double *r1_dev, const double *r2_dev, int64_t n, double *out);

/* No counterpart in the reference.  The dot product of DOT_PRODUCT_PAR for
 * callers that cannot allocate device memory: hosts whose own pool owns all
 * device memory or that run under a hard device-memory budget, and timing-
 * critical loops that cannot take the implicit synchronization of
 * cudaMalloc/cudaFree.  *out_dev (device memory) = sum r1*r2, reduced in a fixed
 * order, enqueued on `stream` (a cudaStream_t; NULL: the default stream).  Its
 * scratch is a fixed array inside this library, one per device, kept until the
 * process exits and shared by every call: calls whose work overlaps on the GPU
 * race.  n may not exceed MFIXGPU_NOALLOC_MAX_N (MFIXGPU_ERR_ARGS otherwise).
 * The first call on a device looks up the array's address; make it before any
 * stream capture. */
#define MFIXGPU_NOALLOC_MAX_N (268435456LL) /* 2^28 elements */
int mfixgpu_dot_product_par_noalloc(const double *r1_dev, const double *r2_dev, int64_t n, double *out_dev,
                                    void *stream);

/* ---------------------------------------------------------------- pressure correction on the device */

/* The fields SOLVE_PP_G assembles the gas pressure-correction system from
 * (CONV_PP_G, model/conv_pp_g.f:33-182; SOURCE_PP_G, model/source_pp_g.f:18-214),
 * in MFIX's own layouts: cell arrays of DIMENSION_3; D_E/D_N/D_T(DIMENSION_3,
 * 0:DIMENSION_M) with phase m at m*DIMENSION_3; the solids arrays (DIMENSION_3,
 * DIMENSION_M) with phase m at (m-1)*DIMENSION_3.  Served: an incompressible run
 * (RO_G0 defined, so COMPRESSIBLE_PP_G is not called) on a Cartesian grid without
 * cut cells, shear, point sources or user sources.  With on_device set every
 * array pointer except close_packed is device memory; otherwise host memory,
 * copied in. */
typedef struct {
    const int *flag;                          /* FLAG: 1 fluid, 10/11 pressure inflow/outflow */
    const double *rop_ge, *rop_gn, *rop_gt;   /* gas face densities (CONV_ROP_G) */
    const double *ayz, *axz, *axy;            /* face areas */
    const double *u_g, *v_g, *w_g;            /* gas velocities */
    const double *rop_g, *rop_go, *vol, *sum_r_g;
    const double *d_e, *d_n, *d_t;            /* pressure-correction coefficients, phases 0..MMAX */
    int mmax;                                 /* solids phases */
    int ro_g0_defined;                        /* 1: incompressible gas (RO_G0 defined); 0 is not served */
    const int *close_packed;                  /* CLOSE_PACKED(1:MMAX), nonzero = .TRUE. (host memory) */
    const double *rop_se, *rop_sn, *rop_st;   /* solids face densities, phases 1..MMAX */
    const double *u_s, *v_s, *w_s, *rop_s, *rop_so, *sum_r_s;
    double odt;                               /* ODT = 1/DT */
    long long ijk_p_g;                        /* IJK_P_G (1-based), <= 0 when undefined */
    int on_device;
    int pad;
} mfixgpu_pp_fields;

/* CONV_PP_G followed by SOURCE_PP_G on the device: A_M(:,:,0) (7*DIMENSION_3),
 * B_M(:,0) and B_MMAX(:,0), the largest term of each cell's continuity residual
 * (zero outside the fluid), written to the given arrays (host memory unless
 * on_device).  Bit for bit the reference's arithmetic without fused
 * multiply-adds.  Returns 0, MFIXGPU_ERR_NOGEOM, MFIXGPU_ERR_ARGS,
 * MFIXGPU_ERR_UNSUPPORTED (a compressible run) or MFIXGPU_ERR_CUDA. */
int mfixgpu_conv_source_pp_g(const mfixgpu_pp_fields *f, double *a_m, double *b_m, double *b_mmax);

/* SOLVE_PP_G(NORMG, RESG, IER) (model/solve_pp_g.f:10-118) with the LEQ settings
 * of equation 1 passed in (LEQ_IT(1), LEQ_METHOD(1), LEQ_SWEEP(1), LEQ_TOL(1),
 * LEQ_PC(1)), gfortran convention: PP_G = 0, the system assembled on the
 * device, RESG from CALC_RESID_PP (normalized by RESID(B_MMAX)/10 when NORMG
 * = 0, model/solve_pp_g.f:94-104), then SOLVE_LIN_EQ('Pp_g', 1, PP_G, A_M, B_M, 0,
 * ...).  Only the fields and PP_G cross the host link (none when on_device);
 * A_M and B_M exist on the device only. */
void mfixgpu_solve_pp_g_(const mfixgpu_pp_fields *f, const double *normg, double *pp_g, double *resg,
                         const int *itmax, const int *method, const char *sweep, const double *tol, const char *pc,
                         int *ier, size_t sweep_len, size_t pc_len);

/* ---------------------------------------------------------------- batches */

typedef struct {
    int imax2, jmax2, kmax2, do_k;
    int64_t dimension_3;
    double *a_m;  /* 7*DIMENSION_3, the phase slice A_M(:,:,M) */
    double *b_m;  /* DIMENSION_3 */
    double *var;  /* DIMENSION_3, initial guess in, solution out */
    double tol;
    int itmax;
    /* results */
    int ier;
    int iterations;
    int outer_steps;
    int exit_kind;
    int fp64_fallback;
    double rnorm0, rnorm;
} mfixgpu_system;

/* Solves independent systems of uneven sizes together: every kernel launch of
 * an iteration covers all of them (the SIMPLE loop's back-to-back calls, e.g.
 * model/solve_vel_star.f:315-331).  Each system follows the drop-in's
 * algorithm; results are bit-identical to solving it alone.  precision 0/1 as
 * the "precision" option; on_device 1: the pointers are device memory, solved
 * in place.  sweep letters R and S only (other letters: single solves). */
int mfixgpu_batch_solve(mfixgpu_system *systems, int nsys, const char *sweep, const char *pc, int precision,
                        int on_device);
/* mfixgpu_last_stats after a batch: seconds, device_ms, jline_*, kernel_launches of the whole batch. */

/* ---------------------------------------------------------------- serving (no reference counterpart)
 *
 * A request loop for solves that arrive from concurrent cases.  A worker
 * thread owns the device: it admits requests in arrival order while their
 * device memory fits the HBM budget and a slot is free, copies their arrays
 * in on a copy stream, and joins them to a live batch between iterations, so
 * requests that arrive while others are on the GPU share every kernel launch
 * with them (continuous batching).  Each request runs the drop-in's algorithm
 * (LEQ_BICGS, model/leq_bicgs.f:107-509) exactly as when solved alone, and
 * its result is bit-identical to a solve of it alone with the same options.
 * In the mixed form a request whose FP32 iteration gives up moves to an FP64
 * live batch and is solved again from its initial guess. */

typedef struct {
    int precision;          /* 1 (default): FP32 inner / FP64 outer with FP64 hand-over; 0: FP64 drop-in */
    int max_systems;        /* slots of each live batch (default 256) */
    int check_every;        /* iterations between reads of the batch state (default 8) */
    int device;             /* CUDA device (default 0) */
    double hbm_budget;      /* bytes of device memory the requests may hold (0: 85% of free memory) */
    double inner_tol;       /* mixed form: as the "inner_tol" option (0: 1e-2) */
    char sweep[4];          /* "RSRS" when blank; letters R and S only */
    char pc[4];             /* "LINE", "DIAG" or "NONE"; "LINE" when blank */
} mfixgpu_server_config;

/* submit flags */
#define MFIXGPU_REQ_ZERO_GUESS 1   /* the initial guess is zero: var is output only */
#define MFIXGPU_REQ_WRITE_AB 2     /* copy the unit-scaled A_M/B_M back (model/leq_bicgs.f:202-203) */
#define MFIXGPU_REQ_ON_DEVICE 4    /* a_m/b_m/var are device memory, solved in place */

typedef struct {
    int status;             /* 0 queued, 1 copying in, 2 in a batch, 3 copying out, 4 done */
    int ier;
    int iterations;         /* the reference's ITER at exit (mixed form: inner iterations) */
    int iter_tot_add;
    int exit_kind;
    int outer_steps;
    int fp64_fallback;
    int mixed_iterations;
    double rnorm0, rnorm;
    double t_submit, t_admit, t_start, t_done; /* seconds on the server's clock */
} mfixgpu_request;

typedef struct {
    long long submitted, completed, queued, copying, running;
    long long commits;          /* membership changes applied to the live batches */
    long long iterations;       /* iteration bodies launched, summed over the live batches */
    long long kernel_launches;  /* kernels of this library launched by the server */
    long long fp64_fallbacks;
    long long max_running;      /* most requests in the live batches at once */
    double reserved_bytes, peak_reserved_bytes, budget_bytes;
    double seconds;             /* server clock now */
    double busy_ms[2];          /* device time of the form's live batch and of the FP64 hand-over batch */
} mfixgpu_server_counters;

/* Starts a server (its worker thread, streams, live batches).  cfg may be NULL
 * for the defaults.  Returns 0 and *server, or an error code. */
int mfixgpu_server_create(const mfixgpu_server_config *cfg, void **server);
/* Queues one solve.  a_m (7*DIMENSION_3), b_m and var belong to the caller and
 * stay valid and untouched until the request is done; tol and itmax come from
 * sys, results go to the request record (sys's result fields are not
 * written).  Returns a ticket >= 0, or MFIXGPU_ERR_ARGS, MFIXGPU_ERR_NOMEM
 * (larger than the whole budget) or MFIXGPU_ERR_CUDA (the server failed). */
long long mfixgpu_server_submit(void *server, const mfixgpu_system *sys, int flags);
/* 1: done, *out filled and the ticket released; 0: not done (*out holds its
 * status and times so far); MFIXGPU_ERR_ARGS for an unknown ticket. */
int mfixgpu_server_poll(void *server, long long ticket, mfixgpu_request *out);
/* Waits up to timeout_s seconds (< 0: no limit) for the ticket; returns as poll. */
int mfixgpu_server_wait(void *server, long long ticket, double timeout_s, mfixgpu_request *out);
/* Waits up to timeout_s for any request to finish that nobody has collected:
 * 1 with *ticket and *out (released), 0 on timeout. */
int mfixgpu_server_wait_any(void *server, double timeout_s, long long *ticket, mfixgpu_request *out);
int mfixgpu_server_counters_get(void *server, mfixgpu_server_counters *out);
/* Withdraws every request not yet admitted (copied in): they finish with IER
 * MFIXGPU_ERR_CANCELLED.  Requests already admitted run to the end. */
int mfixgpu_server_cancel_queued(void *server);
/* Finishes every submitted request, stops the worker and frees the server. */
int mfixgpu_server_destroy(void *server);

#ifdef __cplusplus
}
#endif
#endif /* MFIXGPU_H */
