/*
 * shakti_b200.h -- C ABI of libshakti_b200.so, the sm_100a implementation of Shakti.jl's
 * per-timestep head solve and field updates.
 *
 * Conventions
 *  - Plain C types only: device pointers, sizes, a cudaStream_t passed as void*.
 *  - Every State array is caller-owned device memory, Float64, column-major with ix fastest,
 *    exactly the reference's State layout (src/state.jl:13-57): centre fields nx*ny, x-face fields
 *    (nx+1)*ny, y-face fields nx*(ny+1).  A Julia CuArray's pointer() can be passed with no copy.
 *  - The library owns its scratch (linear-system coefficients, Krylov vectors, reduction buffers),
 *    allocated in shk_create and freed in shk_destroy.  One context per stream; a context is not
 *    re-entrant.
 *  - Every entry point returns an int status (shk_status).  Non-convergence is a status, not an
 *    error, as in the reference (src/elliptic_solver.jl:143-174); shk_last_error() gives a message.
 *
 * Each entry point cites the reference interface it replaces (file:line in Shakti.jl).
 */
#ifndef SHAKTI_B200_H
#define SHAKTI_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SHK_API __attribute__((visibility("default")))
#else
#define SHK_API
#endif

typedef enum {
    SHK_OK = 0,
    SHK_NOT_CONVERGED = 1, /* Picard or CG hit its iteration cap                          */
    SHK_BREAKDOWN = 2,     /* CG zero curvature |p'Ap| <= eps*||p||^2, or a NaN reduction  */
    SHK_BAD_ARG = 3,
    SHK_CUDA_ERROR = 4,
    SHK_NOT_BOUND = 5      /* state / parameters not set before a solve                   */
} shk_status;

/* Mask codes (src/mask.jl:21-41); the State's mask stays Float64 0.0/1.0/2.0/3.0. */
enum { SHK_GROUNDED = 0, SHK_OCEAN = 1, SHK_LAND = 2, SHK_OTHER_BASIN = 3 };

/* ModelParameters (src/model_parameters.jl:9-29). n, n-1 and 1/n are derived inside. */
typedef struct {
    double rho_w, rho_sw, rho_i, g, nu, n, omega, L, br, lr, ct, cw, p_atm, b_min, b_max, e_v;
} shk_params;

/* State (src/state.jl:13-57): device pointers, Float64, column-major. */
typedef struct {
    double *h, *pw, *po, *b, *beta, *abs_ub, *mdot, *shear, *potential, *sensible, *Re, *K, *G, *zb,
        *zs, *H, *ieb, *lambda, *A_visc, *N, *mask;                              /* (nx, ny)   */
    double *dhdx, *q_x, *Re_x, *b_x, *ub_x, *taub_x, *dpwdx, *valid_x;          /* (nx+1, ny) */
    double *dhdy, *q_y, *Re_y, *b_y, *ub_y, *taub_y, *dpwdy, *valid_y;          /* (nx, ny+1) */
} shk_state;

/* AbstractKFaceScheme (src/k_face_scheme.jl:1-33) */
enum { SHK_KFACE_ARITHMETIC = 0, SHK_KFACE_HARMONIC = 1 };
/* AbstractGapScheme (src/simulation.jl:42-56) */
enum { SHK_GAP_EXPLICIT = 0, SHK_GAP_IMPLICIT = 1 };
/* AbstractHeadScheme (src/simulation.jl:9-33) */
enum { SHK_HEAD_ELLIPTIC = 0, SHK_HEAD_PARABOLIC = 1 };

/* AbstractSlidingLaw (src/sliding_law.jl:18-64, 270-273, 412-416).  Cx/Cy are caller-owned
 * device face arrays, already staggered (and squared for the linear law) as the reference's
 * constructors do. */
enum {
    SHK_SLIDING_REG_COULOMB = 0,       /* RegularizedCoulombSlidingLaw(C)          */
    SHK_SLIDING_REG_COULOMB_FIELD = 1, /* RegularizedCoulombFieldSlidingLaw(Cx,Cy) */
    SHK_SLIDING_REG_COULOMB_V0 = 2,    /* RegularizedCoulombV0SlidingLaw(Cx,Cy,v0) */
    SHK_SLIDING_LINEAR = 3,            /* LinearSlidingLaw(Cx2,Cy2)                */
    SHK_SLIDING_PRESCRIBED = 4         /* PrescribedSlidingLaw                     */
};
typedef struct {
    int kind;
    double C;
    double v0;
    const double *Cx, *Cy;
} shk_sliding_law;

/* AbstractMeltInput (src/melt_input.jl:1-94).  SHK_MELT_SEASONAL_BASE is this library's extension:
 * ieb = seasonal(t) * ones + base (a caller-owned device centre field, e.g. moulin point sources),
 * used by the 4096^2 seasonal + moulin workload that the reference's uniform SeasonalMeltInput
 * cannot express. */
enum { SHK_MELT_CONSTANT = 0, SHK_MELT_SEASONAL = 1, SHK_MELT_SEASONAL_BASE = 2 };
typedef struct {
    int kind;
    double t_start, period, omega, amplitude, offset, i_min, seconds_per_year;
    const double *base;
} shk_melt_input;

/* CGIterativeSolver(g, MatrixFreeLinearSystem; chebyshev_degree, chebyshev_nsteps_estimate)
 * (src/linear_solver.jl:832-843) plus the Krylov.jl cg! keywords the reference leaves at their
 * defaults.
 *   stop_rule SHK_STOP_KRYLOV: sqrt(r'z) <= atol + rtol*sqrt(r0'z0) (Krylov.jl default rule)
 *   stop_rule SHK_STOP_RELRES: ||b - A x||_2 <= rtol*||b_G||_2, the recursive residual over every
 *     row against the GROUNDED rows of b (b_G).  The OCEAN/LAND/OTHER_BASIN rows are identity
 *     rows holding a fixed head (~1e3 m), decoupled from the free heads; their residual is zero
 *     once h holds the fixed value, and counted in ||b|| they would dominate it.
 *   precision SHK_FP64: every vector and coefficient in Float64
 *   precision SHK_MIXED: Float32 stencil and CG inside Float64 iterative refinement; the outer
 *     residual, the refinement update and the stopping test stay Float64 (rel-res rule only).
 *     Each refinement replaces the Float32 residual by the Float64 true residual b - A h and
 *     continues the CG direction rather than restarting it. */
/* SHK_PRECOND_MULTIGRID: this library's extension, the GPU counterpart of the reference's
 * CPU-only AMGPreconditioner (src/preconditioner.jl:298-327): a Float32 aggregation-multigrid
 * V-cycle (2x2 aggregation, Galerkin coarse operators in Laplacian form) inside the Float64 CG.
 * Requires precision SHK_FP64 (the outer CG). */
enum { SHK_PRECOND_JACOBI = 0, SHK_PRECOND_CHEBYSHEV = 1, SHK_PRECOND_MULTIGRID = 2 };
enum { SHK_STOP_KRYLOV = 0, SHK_STOP_RELRES = 1 };
enum { SHK_FP64 = 0, SHK_MIXED = 1 };
typedef struct {
    int precond;
    int cheb_degree;
    int cheb_nsteps;
    int stop_rule;
    int precision;
    int max_refine;     /* mixed precision: cap on outer refinement steps (<=0: 200)         */
    double atol, rtol;  /* Krylov defaults: sqrt(eps(Float64)) both                          */
    double inner_rtol;  /* mixed precision: Float32 residual drop per refinement (<=0: 1e-2) */
    long itmax;         /* <= 0: 2*nx*ny, Krylov's default                                   */
    long inner_itmax;   /* mixed precision: cap on Float32 iterations between two Float64
                           residual replacements (<= 0: max(200, (nx+ny)/2))                   */
} shk_cg_opts;

typedef struct {
    long niter;          /* CG iterations (inner iterations summed for SHK_MIXED)            */
    int status;          /* shk_status of the solve                                          */
    int refinements;     /* outer refinement steps (SHK_MIXED)                               */
    double rnorm0, rnorm;
    double lambda_min, lambda_max; /* Chebyshev bounds in use after the solve                */
    int bounds_valid;    /* 1 if this solve's Lanczos estimate was adopted, 0 if it fell back */
} shk_cg_stats;

/* PicardSolver(iters, tol, ls, g; alpha, check_every) (src/elliptic_solver.jl:59-105).
 * alpha <= 0 or NaN selects NoHeadRelaxation. */
typedef struct {
    int iters, check_every;
    double tol, alpha;
} shk_picard_opts;

typedef struct {
    int converged, last_iter; /* ps.converged / ps.last_iter                                  */
    long cg_iters_total;
    int cg_solves, cg_breakdowns;
    double max_dh, max_h;     /* last convergence-check maxima                                */
} shk_picard_stats;

/* ---------------------------------------------------------------------------------------------
 * Context
 * ------------------------------------------------------------------------------------------- */
SHK_API int shk_version(void);
SHK_API const char *shk_status_string(int status);

/* Grid(nx, ny, lx, ly) (src/grid.jl:26-35) + CGIterativeSolver workspace allocation
 * (src/linear_solver.jl:832-843).  dx = lx/(nx-1), dy = ly/(ny-1).  stream may be NULL. */
SHK_API int shk_create(int nx, int ny, double lx, double ly, void *stream, void **ctx_out);
SHK_API int shk_destroy(void *ctx);
SHK_API const char *shk_last_error(const void *ctx);
SHK_API int shk_set_stream(void *ctx, void *stream);

SHK_API int shk_set_params(void *ctx, const shk_params *p);                 /* ModelParameters      */
SHK_API int shk_set_sliding_law(void *ctx, const shk_sliding_law *sl);      /* AbstractSlidingLaw   */
SHK_API int shk_set_schemes(void *ctx, int kface_scheme, int gap_scheme);   /* Simulation ctor      */
SHK_API int shk_bind_state(void *ctx, const shk_state *s);                  /* State pointers       */

/* ---------------------------------------------------------------------------------------------
 * Set-up
 * ------------------------------------------------------------------------------------------- */
/* set_initial_conditions! (src/initial_conditions.jl:14-125), after the caller has copied the raw
 * inputs (mask, A_visc, zb, zs, b, G, ub_x, ub_y, ieb, and taub_x/taub_y for the prescribed law)
 * into the bound State.  Also rebuilds the library's compact copy of the mask: call it again after
 * any change to State.mask (compute_face_masks!, src/mask.jl:62-105). */
SHK_API int shk_set_initial_conditions(void *ctx);

/* ---------------------------------------------------------------------------------------------
 * Linear algebra seams
 * ------------------------------------------------------------------------------------------- */
/* update_MFLS! / update_MFLS_parabolic! (src/linear_solver.jl:438-610). */
SHK_API int shk_assemble(void *ctx, int parabolic, double dt);
/* Writes the five coefficient arrays and rhs of the assembled MatrixFreeLinearSystem
 * (src/linear_solver.jl:91-98) into caller device buffers of nx*ny doubles each. */
SHK_API int shk_export_mfls(void *ctx, double *aP, double *aE, double *aW, double *aN, double *aS,
                            double *rhs);
/* LinearAlgebra.mul!(y, ::StencilOperator, x) (src/linear_solver.jl:664-669); device buffers. */
SHK_API int shk_matvec(void *ctx, const double *x, double *y);
/* update_chebyshev_bounds!(P, rhs) (src/preconditioner.jl:197-233) on the assembled operator.
 * rhs == NULL uses the assembled rhs.  est_out (2 doubles, host, may be NULL) receives the raw
 * estimate; *adopted (host, may be NULL) is 1 if it passed the validity check. */
SHK_API int shk_update_chebyshev_bounds(void *ctx, int nsteps, const double *rhs, double *est_out,
                                        int *adopted);
SHK_API int shk_get_chebyshev_bounds(void *ctx, double *lambda_min, double *lambda_max);
SHK_API int shk_set_chebyshev_bounds(void *ctx, double lambda_min, double lambda_max);
/* ldiv!(y, ::ChebyshevPreconditioner, x) (src/preconditioner.jl:239-267); device buffers. */
SHK_API int shk_chebyshev_apply(void *ctx, int degree, const double *x, double *y);
/* _cg_precond! + cg!(ws, StencilOperator, rhs, vec(h); M, ldiv=true) + s.h .= x
 * (src/linear_solver.jl:918-923) on the already-assembled system. */
SHK_API int shk_cg_solve(void *ctx, const shk_cg_opts *o, shk_cg_stats *st);
/* solve_elliptic_linear_system!(::CGIterativeSolver{<:MatrixFreeLinearSystem}, ...)
 * (src/linear_solver.jl:915-925) */
SHK_API int shk_solve_elliptic(void *ctx, const shk_cg_opts *o, shk_cg_stats *st);
/* solve_parabolic_linear_system!(::CGIterativeSolver{<:MatrixFreeLinearSystem}, ..., dt)
 * (src/linear_solver.jl:935-945) */
SHK_API int shk_solve_parabolic(void *ctx, double dt, const shk_cg_opts *o, shk_cg_stats *st);

/* ---------------------------------------------------------------------------------------------
 * Field updates and drivers
 * ------------------------------------------------------------------------------------------- */
/* The field-update tail of Picard_iteration! / parabolic_solver!: compute_dhdxy!, compute_pw!,
 * compute_dpwdxy!, compute_N!, compute_q_and_Re_xy!, compute_Re!, compute_taub_xy!,
 * compute_mdot!, compute_K! (src/elliptic_solver.jl:193-206), fused into one pass. */
SHK_API int shk_picard_tail(void *ctx);
/* relax_h!(UnderHeadRelaxation(alpha), state, h_prev) (src/elliptic_solver.jl:42-46) with h_prev
 * the caller's device buffer. */
SHK_API int shk_relax_h(void *ctx, double alpha, const double *h_prev);
/* Picard_loop! (src/elliptic_solver.jl:138-176) including every Picard_iteration! (:187-208). */
SHK_API int shk_picard_solve(void *ctx, const shk_picard_opts *po, const shk_cg_opts *o,
                             shk_picard_stats *st);
/* parabolic_solver! (src/parabolic_solver.jl:16-38) */
SHK_API int shk_parabolic_step(void *ctx, double dt, const shk_cg_opts *o, shk_cg_stats *st);
/* step_b! (src/run.jl:154-164): compute_b! (implicit/explicit) + compute_beta! + compute_b_x!/y!. */
SHK_API int shk_step_b(void *ctx, double dt);
/* update_ieb!(mi, state, t) (src/melt_input.jl:30, 86-94) */
SHK_API int shk_update_ieb(void *ctx, const shk_melt_input *mi, double t);
/* step!(sim) (src/run.jl:82-88): update_ieb!, step_h!, step_b!.  st may be NULL. */
SHK_API int shk_step(void *ctx, int head_scheme, double dt, double total_time,
                     const shk_melt_input *mi, const shk_picard_opts *po, const shk_cg_opts *o,
                     shk_picard_stats *st);
/* The time loop of run!(sim) (src/run.jl:37-43) without observers: tsteps calls of step!,
 * advancing *total_time by dt each.  per_step (host, tsteps entries) may be NULL. */
SHK_API int shk_run(void *ctx, int head_scheme, double dt, int tsteps, double *total_time,
                    const shk_melt_input *mi, const shk_picard_opts *po, const shk_cg_opts *o,
                    shk_picard_stats *per_step);

/* Launch accounting: number of kernels this context has enqueued since creation. */
SHK_API long shk_kernel_launches(const void *ctx);

/* ---------------------------------------------------------------------------------------------
 * Ensembles.  The reference advances one Simulation at a time; a caller with many independent
 * simulations (parameter sweeps, uncertainty ensembles) loops run! over them
 * (src/run.jl:21-63).  These calls advance N instances together on one GPU: each batched kernel is
 * one launch over every instance, and each timestep is one CUDA graph launch whose Picard and CG
 * loops run on the device (instances that have converged skip the remaining iterations).
 *
 * Each instance is an ordinary context (shk_create ... shk_set_initial_conditions), of any grid
 * size; all on the same device.  The ensemble runs the elliptic head scheme with Float64 Jacobi
 * CG, no head relaxation, and a constant melt input (update_ieb! is then a no-op), and gives each
 * instance the same fields as its own shk_step would, up to the rounding of the reductions'
 * block counts.
 * --------------------------------------------------------------------------------------------- */
typedef struct {
    long long steps, steps_converged;   /* timesteps run / with a converged Picard loop */
    long long picard_iters, cg_iters;   /* totals over those timesteps */
    int last_picard_iters, last_converged;
    int march_th;                       /* row-marching tile height in use (autotuned) */
    int pad;
    double max_dh, max_h;               /* last Picard check of the last timestep */
} shk_ensemble_stats;

/* N contexts -> one ensemble (the contexts stay owned by the caller and must outlive it). */
SHK_API int shk_ensemble_create(int n, void *const *ctxs, void *stream, void **ens_out);
SHK_API int shk_ensemble_destroy(void *ens);
SHK_API const char *shk_ensemble_last_error(const void *ens);
/* Measured choice of the CG stencil kernel's tile height per grid size; th_out (n) may be NULL. */
SHK_API int shk_ensemble_autotune(void *ens, int iters, int *th_out);
/* tsteps timesteps of dt for every instance (step!, src/run.jl:82-88).  per_instance (n entries)
 * may be NULL.  Returns SHK_NOT_CONVERGED if any instance's Picard loop did not converge. */
SHK_API int shk_ensemble_run(void *ens, double dt, int tsteps, const shk_picard_opts *po,
                             const shk_cg_opts *o, shk_ensemble_stats *per_instance);
/* Per-instance device buffers (n pointers, nx*ny doubles each; NULL entries: none) that receive h
 * after each timestep's first Picard iteration (training data for the learned warm start). */
SHK_API int shk_ensemble_set_snapshots(void *ens, double *const *bufs);
/* Blocks per launch of each batched kernel family (stencil, row-marching, streaming, flat). */
SHK_API int shk_ensemble_launch_counts(const void *ens, int *stencil, int *march, int *stream,
                                       int *flat);

/* ---------------------------------------------------------------------------------------------
 * Learned warm start: BF16 tensor-core kernels of a small convolutional encoder-decoder that
 * predicts the head increment of the coming timestep.  No counterpart in the reference, which
 * seeds each solve with the current head (cg! x0 = vec(h), src/linear_solver.jl:876-881); the
 * prediction only seeds Picard/CG, which still converge to their tolerances.
 *
 * Tensors are device pointers in NHWC order (channels innermost).  BF16 tensors are passed as
 * void*; Float32 tensors as float*.  Weights: [9][Cout][Cin] (3x3 taps row-major), BF16 for the
 * tensor cores, Float32 master copies for the optimiser.  stream may be NULL.
 * --------------------------------------------------------------------------------------------- */
/* Y = act(conv3x3(X, W) + bias) with zero padding; Y (BF16) and/or Yf (Float32) may be NULL.
 * Cin % 16 == 0, Cout % 8 == 0.  flip = 1 negates the tap offsets: with the per-tap transposed
 * weights [9][Cin][Cout] this is the input gradient of the forward convolution. */
SHK_API int shk_nn_conv3x3(const void *X, const void *Wt, const float *bias, void *Y, float *Yf, int N,
                           int H, int W, int Cin, int Cout, int relu, int flip, void *stream);
/* dW[tap][co][ci] += sum_p dY[p][co] X[p + off(tap)][ci]   (Cout % 16 == 0, Cin % 8 == 0) */
/* The tensor-core convolution's fault word on the current device: 1 when one of its bounded waits
 * ran out since the last call (its results are then invalid); read and cleared.  No counterpart in
 * the reference. */
SHK_API int shk_nn_conv_fault(int *fault);
SHK_API int shk_nn_conv3x3_wgrad(const void *X, const void *dY, float *dW, int N, int H, int W, int Cin,
                                 int Cout, void *stream);
/* dYm = dY * (Y > 0) (relu = 0: dY) as BF16; db[c] += sum over the P pixels (db may be NULL) */
SHK_API int shk_nn_relu_grad(const float *dY, const void *Y, void *dYm, float *db, long long P, int C,
                             int relu, void *stream);
/* 2x2 average pooling (H, W: input size) and its gradient (acc = 1 adds into dX) */
SHK_API int shk_nn_pool2(const void *X, void *Y, int N, int H, int W, int C, void *stream);
SHK_API int shk_nn_pool2_grad(const float *dY, float *dX, int N, int H, int W, int C, int acc,
                              void *stream);
/* Y = nearest 2x upsampling of X plus S (S may be NULL; H, W: output size), and the upsampling's
 * gradient (H, W: the coarse size) */
SHK_API int shk_nn_up2_add(const void *X, const void *S, void *Y, int N, int H, int W, int C,
                           void *stream);
SHK_API int shk_nn_up2_grad(const float *dY, float *dX, int N, int H, int W, int C, void *stream);
/* y = x (acc = 0) or y += x (acc = 1), Float32 */
SHK_API int shk_nn_axpy(const float *x, float *y, long long n, int acc, void *stream);
/* mean squared error of channel 0 of Yf (C channels per pixel) against T (weights wgt, may be
 * NULL); writes the gradient dY and adds the loss (already scaled by inv_count) to *loss */
SHK_API int shk_nn_mse(const float *Yf, const float *T, const float *wgt, float *dY, float *loss,
                       long long P, int C, float inv_count, void *stream);
/* one Adam step (bias-corrected at `step` >= 1) on Float32 weights w with gradient g; refreshes the
 * BF16 copy wb and the per-tap transposed copy wt when given (both may be NULL) */
SHK_API int shk_nn_adam(float *w, const float *g, float *m, float *v, void *wb, void *wt, long long n,
                        int Cout, int Cin, float lr, float b1, float b2, float eps, int step,
                        void *stream);
SHK_API int shk_nn_wcast(const float *w, void *wb, void *wt, long long n, int Cout, int Cin,
                         void *stream);
SHK_API int shk_nn_zero(float *p, long long n, void *stream);
/* the network input from a State: channels h, b, N, zb, zs, ieb, mask as (v - norm[2c]) *
 * norm[2c+1] (norm: 14 floats on the device), zero-padded to 16 channels and Hp x Wp pixels */
SHK_API int shk_nn_pack_state(const shk_state *st, int nx, int ny, int Hp, int Wp, const float *norm,
                              void *X, void *stream);
/* out = h + dh_scale * Yf[channel 0] on GROUNDED cells (mask 0), h elsewhere */
SHK_API int shk_nn_apply_increment(const float *Yf, int C, int nx, int ny, int Wp, double dh_scale,
                                   const double *h, const double *mask, double *out, void *stream);
/* ||rhs - A h||_2 (every row) and ||rhs||_2 (GROUNDED rows) of the elliptic system assembled at the
 * context's current h (the initial residual a Picard iteration would start from); assembles into
 * the context's workspace. */
SHK_API int shk_initial_residual(void *ctx, double *rnorm, double *bnorm);
/* ||rhs - A x||_2 (every row; and ||rhs||_2 over the GROUNDED rows) of the system last assembled in
 * the context, for a device vector x of nx*ny doubles. */
SHK_API int shk_residual_of(void *ctx, const double *x, double *rnorm, double *bnorm);
/* `sweeps` damped Jacobi sweeps x <- x + omega (rhs - A x) / aP on the system last assembled in the
 * context (x and tmp: nx*ny doubles, device): removes the rough part of an initial guess's error. */
SHK_API int shk_smooth_guess(void *ctx, double *x, double *tmp, int sweeps, double omega);
/* A one-shot initial guess (nx*ny doubles, device, caller-owned until the solve) for the next
 * Float64 CG solve of the context in place of the current head (cg! x0, src/linear_solver.jl:
 * 876-881); the solve's result still replaces h.  NULL clears it. */
SHK_API int shk_set_cg_warm_start(void *ctx, const double *x0);

/* ---------------------------------------------------------------------------------------------
 * Allocation-free solve.  No counterpart in the reference: it exists for callers that cannot
 * allocate device memory when they solve -- an application whose device memory all belongs to its
 * own pool allocator, a real-time loop that cannot afford the device-wide synchronisation of
 * cudaMalloc/cudaFree, or a plugin host that forbids allocation after start-up.
 *
 * Float64 Jacobi-preconditioned CG (Krylov.jl cg! semantics, as shk_cg_solve) on a caller-owned
 * operator in this library's matrix-free form: aP, aE, aN (nx*ny doubles each; the west/south
 * couplings are the neighbours' east/north entries, exactly what shk_export_mfls writes), rhs,
 * and x (warm start in, solution out).  Only o->precond = SHK_PRECOND_JACOBI, o->precision =
 * SHK_FP64 are accepted.  stream may be NULL.  The operator carries no mask, so with
 * SHK_STOP_RELRES ||rhs|| counts every row.
 *
 * Scratch (Krylov vectors, reduction partials, scalars) lives in one file-scope device array of
 * about 2.8 MB that every GPU loading the library holds until the process exits; nothing is
 * allocated.  Limit: nx*ny <= 65536 cells (e.g. 256 x 256); larger grids return SHK_BAD_ARG with a
 * message on stderr.  The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current: make that first call before any stream
 * capture.  All calls share the array and it keeps the last call's contents, so calls that overlap
 * on the GPU (different streams or host threads) race: serialise them.  The call waits on
 * `stream` between batches of iterations (it reads the stopping flag back to the host), so it
 * returns with the solve complete.  Returns the solve's status (SHK_OK, SHK_NOT_CONVERGED,
 * SHK_BREAKDOWN) or an error code; *st is filled in either case. */
SHK_API int shk_cg_solve_static(int nx, int ny, const double *aP, const double *aE, const double *aN,
                                const double *rhs, double *x, const shk_cg_opts *o, shk_cg_stats *st,
                                void *stream);

#ifdef __cplusplus
}
#endif
#endif
