/*
 * shakti_oracle.h -- CPU restatement of Shakti.jl's per-timestep head solve and field updates.
 *
 * TEST INFRASTRUCTURE ONLY.  This header and oracle/shakti_oracle.c are the test oracle of
 * the CUDA library: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may link or
 * call them.  The product path (libshakti_b200.so) never does.
 *
 * Parity pinning: the reference (Julia) cannot run in this environment, and the reference holds no
 * stored golden vectors.  The restatement is pinned against every fixture and known-answer property
 * of the reference's own test suite (test/linear_solver_test.jl, test/parabolic_solver_test.jl,
 * test/sliding_law_test.jl) -- see tests/test_oracle_reference_suite.py -- and against a sparse
 * direct solve (SciPy SuperLU standing in for CHOLMOD).  Field-level parity with a reference *run*
 * is therefore pinned only through those properties, not through reference-generated outputs.
 *
 * Layout: every field is Float64, column-major (ix fastest), exactly as the reference's State
 * (src/state.jl:13-57): centre fields (nx,ny), x-face fields (nx+1,ny), y-face fields (nx,ny+1).
 * Index (ix,iy) 0-based here; the reference is 1-based, so reference index i maps to ix = i-1.
 */
#ifndef SHAKTI_ORACLE_H
#define SHAKTI_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ModelParameters (src/model_parameters.jl:9-29). */
typedef struct {
    double rho_w, rho_sw, rho_i, g, nu, n, omega, L, br, lr, ct, cw, p_atm, b_min, b_max, e_v;
} orc_params;

/* Sliding laws (src/sliding_law.jl).  kind:
 *   0 RegularizedCoulombSlidingLaw(C)              (:33-35, kernel :213-249)
 *   1 RegularizedCoulombFieldSlidingLaw(Cx,Cy)      (:270-273, kernel :340-382)
 *   2 RegularizedCoulombV0SlidingLaw(Cx,Cy,v0)      (:412-416, kernel :488-522)
 *   3 LinearSlidingLaw(Cx2,Cy2)                     (:61-64, kernel :588-600)
 *   4 PrescribedSlidingLaw                          (:45, no-op)
 * Cx/Cy are face arrays already staggered (and squared for kind 3) as the reference's
 * constructors do. */
typedef struct {
    int kind;
    double C;
    double v0;
    const double *Cx, *Cy;
} orc_sliding;

/* State (src/state.jl:13-57) plus the grid spacing (src/grid.jl:26-35). */
typedef struct {
    int nx, ny;
    double dx, dy;
    /* centre (nx,ny) */
    double *h, *pw, *po, *b, *beta, *abs_ub, *mdot, *shear, *potential, *sensible, *Re, *K, *G,
        *zb, *zs, *H, *ieb, *lambda, *A_visc, *N, *mask;
    /* x-face (nx+1,ny) */
    double *dhdx, *q_x, *Re_x, *b_x, *ub_x, *taub_x, *dpwdx, *valid_x;
    /* y-face (nx,ny+1) */
    double *dhdy, *q_y, *Re_y, *b_y, *ub_y, *taub_y, *dpwdy, *valid_y;
} orc_state;

/* CG options: precond 0 = Jacobi (Diagonal(aP)), 1 = ChebyshevPreconditioner.
 * stop_rule 0 = Krylov.jl cg! default: sqrt(r'z) <= atol + rtol*sqrt(r0'z0) (z = M^-1 r).
 * stop_rule 1 = unpreconditioned relative residual ||r||_2 <= rtol*||b_G||_2 (atol ignored), b_G the
 *               GROUNDED rows of b when a mask is given (orc_cg_masked and the Picard drivers).
 * itmax <= 0 means Krylov's default 2*n. */
typedef struct {
    int precond, cheb_degree, cheb_nsteps, stop_rule;
    double atol, rtol;
    long itmax;
} orc_cg_opts;

typedef struct {
    long niter;
    int status; /* 0 solved, 1 itmax reached, 2 zero curvature / breakdown */
    double rnorm0, rnorm;
} orc_cg_stats;

/* Chebyshev preconditioner persistent state: the (lambda_min, lambda_max) pair that survives
 * across solves (src/preconditioner.jl:160-186), starting at the (1,1) placeholder. */
typedef struct {
    double lambda_min, lambda_max;
    int last_estimate_valid;
} orc_cheb_state;

int  orc_num_threads(void);
void orc_set_num_threads(int n);

/* mask.jl:62-105 */
void orc_compute_face_masks(orc_state *s);
void orc_apply_mask_to_sliding(orc_state *s);

/* set_initial_conditions! (src/initial_conditions.jl:14-125) after the caller copied the raw input
 * fields (mask, A_visc, zb, zs, b, G, ub_x, ub_y, ieb, taub_x, taub_y) into the state. */
void orc_set_initial_conditions(orc_state *s, const orc_params *p, const orc_sliding *sl);

/* Individual field kernels (for the reference-suite ports). */
void orc_compute_H(orc_state *s);
void orc_compute_po(orc_state *s, const orc_params *p);
void orc_compute_h(orc_state *s, const orc_params *p);
void orc_compute_abs_ub(orc_state *s);
void orc_compute_pw(orc_state *s, const orc_params *p);
void orc_compute_N(orc_state *s);
void orc_compute_dhdxy(orc_state *s);
void orc_compute_dpwdxy(orc_state *s);
void orc_compute_q_xy_lagged(orc_state *s, const orc_params *p);
void orc_compute_Re_xy_lagged(orc_state *s, const orc_params *p);
void orc_compute_q_and_Re_xy(orc_state *s, const orc_params *p);
void orc_compute_Re(orc_state *s);
void orc_compute_taub_xy(orc_state *s, const orc_params *p, const orc_sliding *sl);
void orc_compute_mdot(orc_state *s, const orc_params *p);
void orc_compute_K(orc_state *s, const orc_params *p);
void orc_compute_beta(orc_state *s, const orc_params *p);
void orc_compute_b_xy(orc_state *s);

/* update_MFLS! / update_MFLS_parabolic! (src/linear_solver.jl:438-610).  kfs 0 Arithmetic, 1 Harmonic. */
void orc_assemble_mfls(const orc_state *s, const orc_params *p, int kfs, int parabolic, double dt,
                       double *aP, double *aE, double *aW, double *aN, double *aS, double *rhs);
/* update_SALS! / update_SALS_parabolic! (src/linear_solver.jl:226-430): diagonal and the four
 * signed off-diagonal bands of the sparse matrix (sign baked in), plus rhs. */
void orc_assemble_sals(const orc_state *s, const orc_params *p, int kfs, int parabolic, double dt,
                       double *dP, double *oE, double *oW, double *oN, double *oS, double *rhs);

/* stencil_matvec_kernel! (src/linear_solver.jl:616-633) */
void orc_matvec(int nx, int ny, const double *aP, const double *aE, const double *aW,
                const double *aN, const double *aS, const double *x, double *y);

/* estimate_eigenvalue_bounds + update_chebyshev_bounds! (src/preconditioner.jl:89-233).
 * Returns 1 when the estimate was adopted, 0 when the previous bounds were kept. */
int orc_update_chebyshev_bounds(int nx, int ny, const double *aP, const double *aE, const double *aW,
                                const double *aN, const double *aS, const double *rhs, int nsteps,
                                orc_cheb_state *cs, double *est_out /* [2] raw estimate, may be NULL */);
/* ChebyshevPreconditioner ldiv! (src/preconditioner.jl:239-267) */
void orc_chebyshev_apply(int nx, int ny, const double *aP, const double *aE, const double *aW,
                         const double *aN, const double *aS, int degree, const orc_cheb_state *cs,
                         const double *x, double *y);

/* Krylov.jl cg! with warm start x0 (call sites src/linear_solver.jl:881,902,921,941). x holds x0
 * on entry and the solution on exit. */
int orc_cg(int nx, int ny, const double *aP, const double *aE, const double *aW, const double *aN,
           const double *aS, const double *rhs, double *x, const orc_cg_opts *o, orc_cheb_state *cs,
           orc_cg_stats *st);
/* orc_cg with the relative-residual rule (stop_rule 1) measured against the GROUNDED rows of rhs
 * only: ||rhs - A x||_2 (every row) <= rtol * ||rhs restricted to mask == GROUNDED||_2.  mask NULL:
 * every row counts, as in orc_cg.  The Picard and parabolic drivers pass State.mask. */
int orc_cg_masked(int nx, int ny, const double *aP, const double *aE, const double *aW, const double *aN,
                  const double *aS, const double *rhs, const double *mask, double *x, const orc_cg_opts *o,
                  orc_cheb_state *cs, orc_cg_stats *st);

/* Picard / parabolic / gap / melt input / run loop */
typedef struct {
    int iters, check_every;
    double tol;
    double alpha; /* under-relaxation; NaN or <= 0 => NoHeadRelaxation */
} orc_picard_opts;

typedef struct {
    int converged, last_iter;
    long cg_iters_total;
    int cg_solves;
    int cg_breakdowns;
} orc_picard_stats;

/* Melt input (src/melt_input.jl).  kind 0 Constant, 1 Seasonal (uniform fill), 2 Seasonal plus a
 * fixed spatial field `base` (nx*ny, m/s; the library's SeasonalBaseMeltInput extension: ieb =
 * seasonal value + base, e.g. point moulins). */
typedef struct {
    int kind;
    double t_start, period, omega, amplitude, offset, i_min, seconds_per_year;
    const double *base;
} orc_melt;

void orc_update_ieb(orc_state *s, const orc_melt *mi, double t);

/* One Picard_iteration! (src/elliptic_solver.jl:187-208) including the linear solve. */
int orc_picard_iteration(orc_state *s, const orc_params *p, const orc_sliding *sl, int kfs,
                         const orc_cg_opts *cg, orc_cheb_state *cs, double alpha, const double *h_prev,
                         orc_cg_stats *cst);
/* Picard_loop! (src/elliptic_solver.jl:138-176) */
int orc_picard_loop(orc_state *s, const orc_params *p, const orc_sliding *sl, int kfs,
                    const orc_cg_opts *cg, orc_cheb_state *cs, const orc_picard_opts *po,
                    orc_picard_stats *pst);
/* parabolic_solver! (src/parabolic_solver.jl:16-38) */
int orc_parabolic_step(orc_state *s, const orc_params *p, const orc_sliding *sl, int kfs,
                       const orc_cg_opts *cg, orc_cheb_state *cs, double dt, orc_cg_stats *cst);
/* The shared field-update tail (pw..K) of Picard_iteration! / parabolic_solver!. */
void orc_picard_tail(orc_state *s, const orc_params *p, const orc_sliding *sl);
/* step_b! (src/run.jl:154-164): gap 0 explicit, 1 implicit. */
void orc_step_b(orc_state *s, const orc_params *p, int gap_scheme, double dt);

/* run! loop body (src/run.jl:82-88) for tsteps steps, starting at total_time *t. */
typedef struct {
    int head_scheme; /* 0 elliptic (Picard), 1 parabolic */
    int gap_scheme;  /* 0 explicit, 1 implicit */
    int kfs;
    double dt;
} orc_sim;

int orc_run(orc_state *s, const orc_params *p, const orc_sliding *sl, const orc_melt *mi,
            const orc_sim *sim, const orc_cg_opts *cg, orc_cheb_state *cs, const orc_picard_opts *po,
            int tsteps, double *total_time, orc_picard_stats *per_step /* tsteps entries or NULL */);

/* Bounded run session: the orc_run loop, resumable between CG iterations (see the .c file). */
typedef struct {
    int steps_done;          /* completed timesteps                                        */
    long picard_iters;       /* completed linear solves (Picard iterations) in total       */
    long cg_iters;           /* CG iterations in total (including the solve in progress)   */
    int cg_breakdowns;
    int pic_iter_now;        /* Picard iteration in progress (0 between timesteps)         */
    long cg_iter_now;        /* CG iterations of the solve in progress                     */
    double elapsed;          /* wall seconds spent inside orc_session_advance              */
    double completed_s;      /* wall seconds of the completed timesteps                    */
    double step_s_now;       /* wall seconds spent on the timestep in progress             */
    double last_step_s;      /* the last completed timestep: seconds, Picard, CG, converged */
    int last_picard;
    long last_cg;
    int last_converged;
    int all_converged;
    double total_time;
} orc_session_progress;

typedef struct orc_session orc_session;
orc_session *orc_session_create(orc_state *s, const orc_params *p, const orc_sliding *sl, const orc_melt *mi,
                                const orc_sim *sim, const orc_cg_opts *cg, orc_cheb_state *cs,
                                const orc_picard_opts *po, double total_time);
int orc_session_advance(orc_session *S, double seconds, int max_steps, orc_session_progress *out);
void orc_session_destroy(orc_session *S);

#ifdef __cplusplus
}
#endif
#endif
