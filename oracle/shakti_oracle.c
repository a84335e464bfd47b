/*
 * shakti_oracle.c -- CPU restatement (FP64, OpenMP) of Shakti.jl's per-timestep head solve and
 * field updates.  TEST INFRASTRUCTURE: the test oracle and the reported CPU baseline, never the product.
 *
 * Every function restates one reference kernel or driver, cited by file:line.  Each kernel is its
 * own loop (no fusion) and every arithmetic expression keeps the reference's evaluation order
 * (Julia folds `a+b+c` and `a*b*c` left to right and never contracts to FMA; this file is compiled
 * with -ffp-contract=off).  Known, unavoidable differences from a reference run:
 *   - dot products: the reference's Krylov.jl calls BLAS ddot (OpenBLAS summation order); here an
 *     OpenMP reduction.  Everything downstream of a reduction therefore agrees to rounding, not bits.
 *   - the 15x15 symmetric tridiagonal eigensolve (LinearAlgebra.eigvals -> LAPACK) is restated as
 *     Sturm-sequence bisection for the two extreme eigenvalues (the only ones used).
 *   - x^(1/n) calls the C library pow (the reference calls Julia's own Float64 pow).
 * Krylov.jl 0.10.8's cg! is a third-party dependency not present in the reference tree; its
 * published algorithm (Hestenes-Stiefel CG with warm start, preconditioned-norm stopping test,
 * atol = rtol = sqrt(eps), itmax = 2n) is restated in orc_cg below.
 */
#include "shakti_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define GROUNDED 0.0
#define OCEAN 1.0
#define LAND 2.0
#define OTHER_BASIN 3.0

#define CI(ix, iy) ((size_t)(ix) + (size_t)(iy) * (size_t)nx)        /* centre (nx,ny)     */
#define XI(ix, iy) ((size_t)(ix) + (size_t)(iy) * (size_t)(nx + 1))  /* x-face (nx+1,ny)   */
#define YI(ix, iy) ((size_t)(ix) + (size_t)(iy) * (size_t)nx)        /* y-face (nx,ny+1)   */

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ---------------------------------------------------------------------------------------------
 * Scalar helpers
 * ------------------------------------------------------------------------------------------- */

/* Julia's x^n for Float64 x and Integer n (Base.pow_body): n==3 is x*x*x; otherwise a compensated
 * power-by-squaring.  For n == 2 this reduces to fl(x*x). */
static double jl_powi(double x, long n) {
    if (n == 0) return 1.0;
    if (n == 3) return x * x * x;
    if (n < 0) return 1.0 / jl_powi(x, -n); /* not reached for Glen exponents used here */
    double y = 1.0, xnlo = 0.0, ynlo = 0.0;
    while (n > 1) {
        if (n & 1) {
            double err = fma(y, xnlo, x * ynlo);
            double hi = x * y;
            double lo = fma(x, y, -hi);
            y = hi;
            ynlo = lo + err;
        }
        double err = x * 2.0 * xnlo;
        double hi = x * x;
        double lo = fma(x, x, -hi);
        x = hi;
        xnlo = lo + err;
        n >>= 1;
    }
    double err = fma(y, xnlo, x * ynlo);
    if (isfinite(x) && isfinite(err)) return fma(x, y, fma(y, xnlo, x * ynlo));
    return x * y;
}

/* pow(x, e) dispatching like the reference's canonical_exponent/pow (model_parameters.jl:122-134):
 * an integer-valued exponent takes the integer path, otherwise the float power. */
static double jl_pow(double x, double e) {
    if (e == floor(e) && fabs(e) < 1e9) return jl_powi(x, (long)e);
    return pow(x, e);
}

/* Julia max/min propagate NaN. */
static double jl_max(double a, double b) {
    if (isnan(a) || isnan(b)) return NAN;
    return a > b ? a : b;
}

static double jl_min(double a, double b) {
    if (isnan(a) || isnan(b)) return NAN;
    return a < b ? a : b;
}

/* Julia sign(x): -1, 0 (signed), +1, NaN. */
static double jl_sign(double x) {
    if (x > 0) return 1.0;
    if (x < 0) return -1.0;
    return x;
}

/* Julia clamp(x, lo, hi) */
static double jl_clamp(double x, double lo, double hi) { return x > hi ? hi : (x < lo ? lo : x); }

/* Bool * Float in Julia: true*y = y, false*y = copysign(0, y). */
static double jl_boolmul(int b, double y) { return b ? y : copysign(0.0, y); }

static double dot(size_t n, const double *a, const double *b) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long i = 0; i < (long)n; i++) s += a[i] * b[i];
    return s;
}

/* ---------------------------------------------------------------------------------------------
 * mask.jl
 * ------------------------------------------------------------------------------------------- */

/* compute_valid_x_kernel!/compute_valid_y_kernel! (src/mask.jl:62-84) */
void orc_compute_face_masks(orc_state *s) {
    const int nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < ny; iy++)
        for (int f = 0; f <= nx; f++) {
            double v = 1.0;
            if (f > 0 && f < nx) {
                int valid = (s->mask[CI(f - 1, iy)] != OTHER_BASIN) && (s->mask[CI(f, iy)] != OTHER_BASIN);
                v = valid ? 1.0 : 0.0;
            }
            s->valid_x[XI(f, iy)] = v;
        }
#pragma omp parallel for schedule(static)
    for (int f = 0; f <= ny; f++)
        for (int ix = 0; ix < nx; ix++) {
            double v = 1.0;
            if (f > 0 && f < ny) {
                int valid = (s->mask[CI(ix, f - 1)] != OTHER_BASIN) && (s->mask[CI(ix, f)] != OTHER_BASIN);
                v = valid ? 1.0 : 0.0;
            }
            s->valid_y[YI(ix, f)] = v;
        }
}

/* apply_mask_to_sliding_x/y_kernel! (src/mask.jl:117-136) */
void orc_apply_mask_to_sliding(orc_state *s) {
    const int nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < ny; iy++)
        for (int f = 0; f <= nx; f++)
            if (f == 0 || f == nx || !(s->mask[CI(f - 1, iy)] == GROUNDED && s->mask[CI(f, iy)] == GROUNDED))
                s->ub_x[XI(f, iy)] = 0.0;
#pragma omp parallel for schedule(static)
    for (int f = 0; f <= ny; f++)
        for (int ix = 0; ix < nx; ix++)
            if (f == 0 || f == ny || !(s->mask[CI(ix, f - 1)] == GROUNDED && s->mask[CI(ix, f)] == GROUNDED))
                s->ub_y[YI(ix, f)] = 0.0;
}

/* ---------------------------------------------------------------------------------------------
 * static_fields.jl / pressure.jl
 * ------------------------------------------------------------------------------------------- */

/* compute_H_kernel! (src/static_fields.jl:8-13) */
void orc_compute_H(orc_state *s) {
    const size_t n = (size_t)s->nx * s->ny;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) s->H[i] = s->zs[i] - (s->zb[i] + s->b[i]);
}

/* compute_po_kernel! (src/static_fields.jl:22-27) */
void orc_compute_po(orc_state *s, const orc_params *p) {
    const size_t n = (size_t)s->nx * s->ny;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) s->po[i] = p->rho_i * p->g * s->H[i];
}

/* compute_h_kernel! (src/static_fields.jl:39-44) */
void orc_compute_h(orc_state *s, const orc_params *p) {
    const size_t n = (size_t)s->nx * s->ny;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) s->h[i] = s->pw[i] / (p->rho_w * p->g) + s->zb[i];
}

/* compute_abs_ub_kernel! (src/static_fields.jl:59-66) */
void orc_compute_abs_ub(orc_state *s) {
    const int nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++) {
            double ubx_c = (s->ub_x[XI(ix, iy)] + s->ub_x[XI(ix + 1, iy)]) / 2;
            double uby_c = (s->ub_y[YI(ix, iy)] + s->ub_y[YI(ix, iy + 1)]) / 2;
            s->abs_ub[CI(ix, iy)] = sqrt(ubx_c * ubx_c + uby_c * uby_c);
        }
}

/* compute_pw_kernel! (src/pressure.jl:1-6) */
void orc_compute_pw(orc_state *s, const orc_params *p) {
    const size_t n = (size_t)s->nx * s->ny;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) s->pw[i] = p->rho_w * p->g * (s->h[i] - s->zb[i]);
}

/* compute_N_kernel! (src/pressure.jl:15-21) */
void orc_compute_N(orc_state *s) {
    const size_t n = (size_t)s->nx * s->ny;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) s->N[i] = jl_boolmul(s->mask[i] == GROUNDED, s->po[i] - s->pw[i]);
}

/* ---------------------------------------------------------------------------------------------
 * field_gradients.jl -- interior faces only; edge faces never written.
 * ------------------------------------------------------------------------------------------- */

static void grad_xy(int nx, int ny, double dx, double dy, const double *f, const double *valid_x,
                    const double *valid_y, double *dfdx, double *dfdy) {
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < ny; iy++)
        for (int fx = 1; fx < nx; fx++)
            dfdx[XI(fx, iy)] = ((f[CI(fx, iy)] - f[CI(fx - 1, iy)]) / dx) * valid_x[XI(fx, iy)];
#pragma omp parallel for schedule(static)
    for (int fy = 1; fy < ny; fy++)
        for (int ix = 0; ix < nx; ix++)
            dfdy[YI(ix, fy)] = ((f[CI(ix, fy)] - f[CI(ix, fy - 1)]) / dy) * valid_y[YI(ix, fy)];
}

/* compute_dhdxy_kernel! (src/field_gradients.jl:95-103) */
void orc_compute_dhdxy(orc_state *s) {
    grad_xy(s->nx, s->ny, s->dx, s->dy, s->h, s->valid_x, s->valid_y, s->dhdx, s->dhdy);
}

/* compute_dpwdxy_kernel! (src/field_gradients.jl:112-120) */
void orc_compute_dpwdxy(orc_state *s) {
    grad_xy(s->nx, s->ny, s->dx, s->dy, s->pw, s->valid_x, s->valid_y, s->dpwdx, s->dpwdy);
}

/* ---------------------------------------------------------------------------------------------
 * water_flux.jl
 * ------------------------------------------------------------------------------------------- */

/* compute_q_xy_kernel! (lagged, src/water_flux.jl:46-54): q = -(b^3 g dhdx) / (12 nu (1 + omega Re)) */
void orc_compute_q_xy_lagged(orc_state *s, const orc_params *p) {
    const int nx = s->nx, ny = s->ny;
    const size_t nxf = (size_t)(nx + 1) * ny, nyf = (size_t)nx * (ny + 1);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nxf; i++) {
        double bb = s->b_x[i];
        s->q_x[i] = -(bb * bb * bb * p->g * s->dhdx[i]) / (12 * p->nu * (1 + p->omega * s->Re_x[i]));
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nyf; i++) {
        double bb = s->b_y[i];
        s->q_y[i] = -(bb * bb * bb * p->g * s->dhdy[i]) / (12 * p->nu * (1 + p->omega * s->Re_y[i]));
    }
}

/* compute_Re_xy_kernel! (lagged, src/water_flux.jl:90-98): Re = |q| / nu */
void orc_compute_Re_xy_lagged(orc_state *s, const orc_params *p) {
    const int nx = s->nx, ny = s->ny;
    const size_t nxf = (size_t)(nx + 1) * ny, nyf = (size_t)nx * (ny + 1);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nxf; i++) s->Re_x[i] = fabs(s->q_x[i]) / p->nu;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nyf; i++) s->Re_y[i] = fabs(s->q_y[i]) / p->nu;
}

static void q_re_face(double bf, double grad, const orc_params *p, double *q, double *re) {
    double G = fabs(grad);
    double D = (bf * bf * bf * p->g * G) / (12 * (p->nu * p->nu));
    double R = 2 * D / (1 + sqrt(1 + 4 * p->omega * D));
    *re = R;
    *q = -jl_sign(grad) * p->nu * R;
}

/* compute_q_and_Re_xy_kernel! (lag-free, src/water_flux.jl:192-208):
 * D = b^3 g |dh| / (12 nu^2);  Re = 2D / (1 + sqrt(1 + 4 omega D));  q = -sign(dh) nu Re */
void orc_compute_q_and_Re_xy(orc_state *s, const orc_params *p) {
    const int nx = s->nx, ny = s->ny;
    const size_t nxf = (size_t)(nx + 1) * ny, nyf = (size_t)nx * (ny + 1);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nxf; i++) q_re_face(s->b_x[i], s->dhdx[i], p, &s->q_x[i], &s->Re_x[i]);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nyf; i++) q_re_face(s->b_y[i], s->dhdy[i], p, &s->q_y[i], &s->Re_y[i]);
}

/* compute_Re_kernel! (src/water_flux.jl:107-112) */
void orc_compute_Re(orc_state *s) {
    const int nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++)
            s->Re[CI(ix, iy)] = (s->Re_x[XI(ix, iy)] + s->Re_x[XI(ix + 1, iy)] + s->Re_y[YI(ix, iy)] +
                                 s->Re_y[YI(ix, iy + 1)]) / 4;
}

/* compute_K_kernel! (src/water_flux.jl:221-226): K = b^3 g / (12 nu (1 + omega Re)) */
void orc_compute_K(orc_state *s, const orc_params *p) {
    const size_t n = (size_t)s->nx * s->ny;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) {
        double bb = s->b[i];
        s->K[i] = (bb * bb * bb * p->g) / (12 * p->nu * (1 + p->omega * s->Re[i]));
    }
}

/* ---------------------------------------------------------------------------------------------
 * sliding_law.jl -- all five laws.
 * ------------------------------------------------------------------------------------------- */

/* One face of the regularized-Coulomb family (src/sliding_law.jl:213-249, :340-382, :488-522):
 * taub = Nf*C*pow(|v|/(|v| + denom), 1/n)*(ub/|v|) if |v| > 0 else 0,
 * denom = |Nf|^n * lambda_f (Coulomb, Field) or v0 (V0). */
static double taub_coulomb(double Nf, double Cf, double abs_v, double lf, double ub, const orc_params *p,
                           int v0law, double v0) {
    if (!(abs_v > 0)) return 0.0;
    double denom = v0law ? v0 : jl_pow(fabs(Nf), p->n) * lf;
    return Nf * Cf * jl_pow(abs_v / (abs_v + denom), 1.0 / p->n) * (ub / abs_v);
}

void orc_compute_taub_xy(orc_state *s, const orc_params *p, const orc_sliding *sl) {
    const int nx = s->nx, ny = s->ny;
    if (sl->kind == 4) return; /* PrescribedSlidingLaw: no-op (src/sliding_law.jl:115-131) */
    const int v0law = sl->kind == 2;
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < ny; iy++)
        for (int f = 0; f <= nx; f++) {
            int a = f == 0 ? 0 : (f == nx ? nx - 1 : -1);
            double Nf, lf, abs_v;
            if (a >= 0) {
                Nf = s->N[CI(a, iy)];
                lf = s->lambda[CI(a, iy)];
                abs_v = s->abs_ub[CI(a, iy)];
            } else {
                Nf = (s->N[CI(f, iy)] + s->N[CI(f - 1, iy)]) / 2;
                lf = (s->lambda[CI(f, iy)] + s->lambda[CI(f - 1, iy)]) / 2;
                abs_v = (s->abs_ub[CI(f, iy)] + s->abs_ub[CI(f - 1, iy)]) / 2;
            }
            double ub = s->ub_x[XI(f, iy)];
            double t;
            if (sl->kind == 3) t = sl->Cx[XI(f, iy)] * Nf * ub; /* LinearSlidingLaw (:588-600) */
            else t = taub_coulomb(Nf, sl->kind == 0 ? sl->C : sl->Cx[XI(f, iy)], abs_v, lf, ub, p, v0law, sl->v0);
            s->taub_x[XI(f, iy)] = t;
        }
#pragma omp parallel for schedule(static)
    for (int f = 0; f <= ny; f++)
        for (int ix = 0; ix < nx; ix++) {
            int a = f == 0 ? 0 : (f == ny ? ny - 1 : -1);
            double Nf, lf, abs_v;
            if (a >= 0) {
                Nf = s->N[CI(ix, a)];
                lf = s->lambda[CI(ix, a)];
                abs_v = s->abs_ub[CI(ix, a)];
            } else {
                Nf = (s->N[CI(ix, f)] + s->N[CI(ix, f - 1)]) / 2;
                lf = (s->lambda[CI(ix, f)] + s->lambda[CI(ix, f - 1)]) / 2;
                abs_v = (s->abs_ub[CI(ix, f)] + s->abs_ub[CI(ix, f - 1)]) / 2;
            }
            double ub = s->ub_y[YI(ix, f)];
            double t;
            if (sl->kind == 3) t = sl->Cy[YI(ix, f)] * Nf * ub;
            else t = taub_coulomb(Nf, sl->kind == 0 ? sl->C : sl->Cy[YI(ix, f)], abs_v, lf, ub, p, v0law, sl->v0);
            s->taub_y[YI(ix, f)] = t;
        }
}

/* ---------------------------------------------------------------------------------------------
 * melt_rate.jl -- fused compute_mdot_kernel! (src/melt_rate.jl:106-137), both schemes.
 * Sensible heat is on iff ct*cw != 0 (src/simulation.jl:132).
 * ------------------------------------------------------------------------------------------- */
void orc_compute_mdot(orc_state *s, const orc_params *p) {
    const int nx = s->nx, ny = s->ny;
    const int with_sens = !(p->ct == 0.0 || p->cw == 0.0);
    const double Linv = 1 / p->L;
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++) {
            size_t xe = XI(ix + 1, iy), xw = XI(ix, iy), yn = YI(ix, iy + 1), ys = YI(ix, iy);
            double sh = fabs((s->ub_x[xe] * s->taub_x[xe] + s->ub_x[xw] * s->taub_x[xw]) / 2 +
                             (s->ub_y[yn] * s->taub_y[yn] + s->ub_y[ys] * s->taub_y[ys]) / 2);
            double pot = fabs((s->q_x[xe] * s->dhdx[xe] + s->q_x[xw] * s->dhdx[xw]) / 2 +
                              (s->q_y[yn] * s->dhdy[yn] + s->q_y[ys] * s->dhdy[ys]) / 2);
            size_t c = CI(ix, iy);
            s->shear[c] = sh;
            s->potential[c] = pot;
            if (with_sens) {
                double sens = (s->q_x[xe] * s->dpwdx[xe] + s->q_x[xw] * s->dpwdx[xw]) / 2 +
                              (s->q_y[yn] * s->dpwdy[yn] + s->q_y[ys] * s->dpwdy[ys]) / 2;
                s->sensible[c] = sens;
                s->mdot[c] = Linv * (s->G[c] + sh + p->rho_w * p->g * pot + p->ct * p->cw * p->rho_w * sens);
            } else {
                s->mdot[c] = Linv * (s->G[c] + sh + p->rho_w * p->g * pot);
            }
        }
}

/* ---------------------------------------------------------------------------------------------
 * gap_height.jl
 * ------------------------------------------------------------------------------------------- */

/* compute_beta_kernel! (src/gap_height.jl:47-52); skipped entirely when br == 0 (:65-73). */
void orc_compute_beta(orc_state *s, const orc_params *p) {
    if (p->br == 0.0) return;
    const size_t n = (size_t)s->nx * s->ny;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) s->beta[i] = jl_max(0.0, (p->br - s->b[i]) / p->lr);
}

/* compute_b_x_kernel!/compute_b_y_kernel! (src/gap_height.jl:75-108) */
void orc_compute_b_xy(orc_state *s) {
    const int nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < ny; iy++)
        for (int f = 0; f <= nx; f++) {
            double v;
            if (f == 0) v = s->b[CI(0, iy)];
            else if (f == nx) v = s->b[CI(nx - 1, iy)];
            else v = (s->b[CI(f, iy)] + s->b[CI(f - 1, iy)]) / 2;
            s->b_x[XI(f, iy)] = v;
        }
#pragma omp parallel for schedule(static)
    for (int f = 0; f <= ny; f++)
        for (int ix = 0; ix < nx; ix++) {
            double v;
            if (f == 0) v = s->b[CI(ix, 0)];
            else if (f == ny) v = s->b[CI(ix, ny - 1)];
            else v = (s->b[CI(ix, f)] + s->b[CI(ix, f - 1)]) / 2;
            s->b_y[YI(ix, f)] = v;
        }
}

/* compute_b_implicit_kernel!/compute_b_explicit_kernel! (src/gap_height.jl:117-135) then
 * compute_beta!, compute_b_x!, compute_b_y! -- step_b! (src/run.jl:154-164). */
void orc_step_b(orc_state *s, const orc_params *p, int gap_scheme, double dt) {
    const size_t n = (size_t)s->nx * s->ny;
    const double nm1 = p->n - 1;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) {
        if (s->mask[i] != GROUNDED) continue;
        double Nn = jl_pow(fabs(s->N[i]), nm1);
        double bnew;
        if (gap_scheme == 1)
            bnew = (s->b[i] + dt * (s->mdot[i] / p->rho_i + s->beta[i] * s->abs_ub[i])) /
                   (1 + dt * s->A_visc[i] * Nn * s->N[i]);
        else
            bnew = s->b[i] + dt * (s->mdot[i] / p->rho_i + s->beta[i] * s->abs_ub[i] - s->A_visc[i] * Nn * s->N[i] * s->b[i]);
        s->b[i] = jl_clamp(bnew, p->b_min, p->b_max);
    }
    orc_compute_beta(s, p);
    orc_compute_b_xy(s);
}

/* ---------------------------------------------------------------------------------------------
 * initial_conditions.jl -- set_initial_conditions! (src/initial_conditions.jl:14-125), after the
 * raw inputs are in place.
 * ------------------------------------------------------------------------------------------- */
void orc_set_initial_conditions(orc_state *s, const orc_params *p, const orc_sliding *sl) {
    const size_t n = (size_t)s->nx * s->ny;
    orc_compute_face_masks(s);
    const double lambda_coeff = 1.5;
    for (size_t i = 0; i < n; i++) s->lambda[i] = lambda_coeff * s->A_visc[i];
    for (size_t i = 0; i < n; i++) s->b[i] = (s->mask[i] != GROUNDED) ? 0.0 : s->b[i];
    orc_compute_H(s);
    orc_compute_beta(s, p);
    orc_apply_mask_to_sliding(s);
    orc_compute_abs_ub(s);
    orc_compute_po(s, p);
    for (size_t i = 0; i < n; i++) s->pw[i] = s->po[i] / 2;
    for (size_t i = 0; i < n; i++) {
        double m = s->mask[i];
        if (m == OCEAN) s->pw[i] = p->p_atm - p->rho_sw * p->g * jl_min(s->zb[i], 0.0);
        else if (m == LAND || m == OTHER_BASIN) s->pw[i] = p->p_atm;
    }
    orc_compute_dpwdxy(s);
    orc_compute_N(s);
    orc_compute_h(s, p);
    orc_compute_dhdxy(s);
    orc_compute_b_xy(s);
    orc_compute_q_and_Re_xy(s, p);
    orc_compute_Re(s);
    orc_compute_taub_xy(s, p, sl);
    orc_compute_mdot(s, p);
    orc_compute_K(s, p);
}

/* ---------------------------------------------------------------------------------------------
 * linear_solver.jl -- assembly
 * ------------------------------------------------------------------------------------------- */

/* dirichlet_head (src/linear_solver.jl:13-27) */
static double dirichlet_head(double m, double zb, const orc_params *p) {
    if (m == OCEAN) {
        double pw_bc = p->p_atm - p->rho_sw * p->g * jl_min(zb, 0.0);
        return pw_bc / (p->rho_w * p->g) + zb;
    }
    return p->p_atm / (p->rho_w * p->g) + zb;
}

/* compute_K_face / boundary_K_face (src/k_face_scheme.jl:32-61) */
static double boundary_K_face(int kfs, const double *K, const double *mask, size_t c1, size_t c2) {
    double m2 = mask[c2];
    if (m2 == OTHER_BASIN) return 0.0;
    if (m2 == OCEAN || m2 == LAND) return K[c1];
    if (kfs == 1) return (2 * K[c1] * K[c2]) / (K[c1] + K[c2] + DBL_EPSILON);
    return (K[c1] + K[c2]) / 2;
}

/* Shared per-cell assembly for update_MFLS_kernel!/update_MFLS_parabolic_kernel!
 * (src/linear_solver.jl:438-501, 529-588) and their SALS twins (:226-307, :345-406).
 * Returns the row: diag, the four face conductances stored (0 where folded), rhs. */
static void assemble_cell(const orc_state *s, const orc_params *p, int kfs, int parabolic, double dt,
                          int ix, int iy, double *oP, double *oE, double *oW, double *oN, double *oS,
                          double *orhs) {
    const int nx = s->nx, ny = s->ny;
    const double dx2 = s->dx * s->dx, dy2 = s->dy * s->dy;
    size_t c = CI(ix, iy);
    double m = s->mask[c];
    *oE = *oW = *oN = *oS = 0.0;
    if (m == OCEAN || m == LAND) {
        *oP = 1;
        *orhs = dirichlet_head(m, s->zb[c], p);
        return;
    }
    if (m == OTHER_BASIN) {
        *oP = 1;
        *orhs = s->h[c];
        return;
    }
    double aE = (ix < nx - 1) ? boundary_K_face(kfs, s->K, s->mask, c, CI(ix + 1, iy)) / dx2 : 0.0;
    double aW = (ix > 0) ? boundary_K_face(kfs, s->K, s->mask, c, CI(ix - 1, iy)) / dx2 : 0.0;
    double aN = (iy < ny - 1) ? boundary_K_face(kfs, s->K, s->mask, c, CI(ix, iy + 1)) / dy2 : 0.0;
    double aS = (iy > 0) ? boundary_K_face(kfs, s->K, s->mask, c, CI(ix, iy - 1)) / dy2 : 0.0;
    const double Nn = jl_pow(fabs(s->N[c]), p->n - 1);
    if (parabolic)
        *oP = (aE + aW + aN + aS) + p->e_v / dt;
    else
        *oP = (aE + aW + aN + aS) + p->n * p->rho_w * p->g * s->A_visc[c] * Nn * s->b[c];
    double drhs = 0.0;
    if (ix < nx - 1) {
        size_t e = CI(ix + 1, iy);
        double mE = s->mask[e];
        if (mE == OCEAN || mE == LAND) drhs += aE * dirichlet_head(mE, s->zb[e], p);
        else *oE = aE;
    }
    if (ix > 0) {
        size_t w = CI(ix - 1, iy);
        double mW = s->mask[w];
        if (mW == OCEAN || mW == LAND) drhs += aW * dirichlet_head(mW, s->zb[w], p);
        else *oW = aW;
    }
    if (iy < ny - 1) {
        size_t no = CI(ix, iy + 1);
        double mN = s->mask[no];
        if (mN == OCEAN || mN == LAND) drhs += aN * dirichlet_head(mN, s->zb[no], p);
        else *oN = aN;
    }
    if (iy > 0) {
        size_t so = CI(ix, iy - 1);
        double mS = s->mask[so];
        if (mS == OCEAN || mS == LAND) drhs += aS * dirichlet_head(mS, s->zb[so], p);
        else *oS = aS;
    }
    if (parabolic)
        *orhs = s->mdot[c] * (1 / p->rho_w - 1 / p->rho_i) - s->beta[c] * s->abs_ub[c] +
                s->A_visc[c] * Nn * s->N[c] * s->b[c] + s->ieb[c] + (p->e_v / dt) * s->h[c] + drhs;
    else
        *orhs = s->mdot[c] * (1 / p->rho_w - 1 / p->rho_i) - s->beta[c] * s->abs_ub[c] +
                s->A_visc[c] * Nn * s->N[c] * s->b[c] +
                s->A_visc[c] * Nn * (p->n * p->rho_w * p->g * s->h[c]) * s->b[c] + s->ieb[c] + drhs;
}

void orc_assemble_mfls(const orc_state *s, const orc_params *p, int kfs, int parabolic, double dt,
                       double *aP, double *aE, double *aW, double *aN, double *aS, double *rhs) {
    const int nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++) {
            size_t c = CI(ix, iy);
            assemble_cell(s, p, kfs, parabolic, dt, ix, iy, &aP[c], &aE[c], &aW[c], &aN[c], &aS[c], &rhs[c]);
        }
}

/* SALS: nzval starts at 0 (fill!), the diagonal is `+= aP` (GROUNDED) or `= 1`, off-diagonals
 * `-= a`.  0 + aP == aP and 0 - a == -a exactly, so the bands are the MFLS values with the sign
 * baked in -- but they are produced by their own pass here, mirroring update_SALS_kernel!. */
void orc_assemble_sals(const orc_state *s, const orc_params *p, int kfs, int parabolic, double dt,
                       double *dP, double *oE, double *oW, double *oN, double *oS, double *rhs) {
    const int nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++) {
            size_t c = CI(ix, iy);
            double P, E, W, Nn, S, r;
            assemble_cell(s, p, kfs, parabolic, dt, ix, iy, &P, &E, &W, &Nn, &S, &r);
            double m = s->mask[c];
            dP[c] = (m == GROUNDED) ? 0.0 + P : P;
            oE[c] = 0.0 - E;
            oW[c] = 0.0 - W;
            oN[c] = 0.0 - Nn;
            oS[c] = 0.0 - S;
            rhs[c] = r;
        }
}

/* stencil_matvec_kernel! (src/linear_solver.jl:616-633) */
void orc_matvec(int nx, int ny, const double *aP, const double *aE, const double *aW, const double *aN,
                const double *aS, const double *x, double *y) {
#pragma omp parallel for schedule(static)
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++) {
            size_t c = CI(ix, iy);
            double yij = aP[c] * x[c];
            if (ix < nx - 1) yij -= aE[c] * x[c + 1];
            if (ix > 0) yij -= aW[c] * x[c - 1];
            if (iy < ny - 1) yij -= aN[c] * x[c + nx];
            if (iy > 0) yij -= aS[c] * x[c - nx];
            y[c] = yij;
        }
}

/* JacobiScaledOperator mul! (src/preconditioner.jl:66-70): y = (A p) ./ d, d = aP */
static void jacobi_scaled_matvec(int nx, int ny, const double *aP, const double *aE, const double *aW,
                                 const double *aN, const double *aS, const double *x, double *y) {
    orc_matvec(nx, ny, aP, aE, aW, aN, aS, x, y);
    const size_t n = (size_t)nx * ny;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) y[i] /= aP[i];
}

/* ---------------------------------------------------------------------------------------------
 * preconditioner.jl -- Chebyshev
 * ------------------------------------------------------------------------------------------- */

/* Number of eigenvalues of the symmetric tridiagonal (d, e) strictly below x (Sturm count). */
static int sturm_count(int m, const double *d, const double *e, double x) {
    int cnt = 0;
    double q = d[0] - x;
    if (q < 0) cnt++;
    for (int i = 1; i < m; i++) {
        if (q == 0) q = DBL_EPSILON * (fabs(e[i - 1]) + DBL_MIN);
        q = d[i] - x - e[i - 1] * e[i - 1] / q;
        if (q < 0) cnt++;
    }
    return cnt;
}

/* Extreme eigenvalues of SymTridiagonal(d, e) by bisection (stands in for LAPACK eigvals). */
static void tridiag_extreme_eigs(int m, const double *d, const double *e, double *lmin, double *lmax) {
    for (int i = 0; i < m; i++)
        if (!isfinite(d[i])) { *lmin = *lmax = NAN; return; }
    for (int i = 0; i + 1 < m; i++)
        if (!isfinite(e[i])) { *lmin = *lmax = NAN; return; }
    double lo = INFINITY, hi = -INFINITY;
    for (int i = 0; i < m; i++) {
        double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < m ? fabs(e[i]) : 0.0);
        if (d[i] - r < lo) lo = d[i] - r;
        if (d[i] + r > hi) hi = d[i] + r;
    }
    double span = fmax(fabs(lo), fabs(hi));
    lo -= DBL_EPSILON * span + DBL_MIN;
    hi += DBL_EPSILON * span + DBL_MIN;
    /* smallest: count(x) >= 1 */
    double a = lo, b = hi;
    for (int it = 0; it < 200; it++) {
        double mid = 0.5 * (a + b);
        if (mid == a || mid == b) break;
        if (sturm_count(m, d, e, mid) >= 1) b = mid; else a = mid;
    }
    *lmin = 0.5 * (a + b);
    a = lo; b = hi;
    for (int it = 0; it < 200; it++) {
        double mid = 0.5 * (a + b);
        if (mid == a || mid == b) break;
        if (sturm_count(m, d, e, mid) >= m) b = mid; else a = mid;
    }
    *lmax = 0.5 * (a + b);
}

/* estimate_eigenvalue_bounds (src/preconditioner.jl:89-134) + update_chebyshev_bounds!
 * validity check and fallback (:197-233). */
int orc_update_chebyshev_bounds(int nx, int ny, const double *aP, const double *aE, const double *aW,
                                const double *aN, const double *aS, const double *rhs, int nsteps,
                                orc_cheb_state *cs, double *est_out) {
    const size_t n = (size_t)nx * ny;
    double *r = malloc(n * sizeof(double)), *p = malloc(n * sizeof(double)), *Ap = malloc(n * sizeof(double));
    double *alphas = calloc(nsteps, sizeof(double)), *betas = calloc(nsteps > 1 ? nsteps - 1 : 1, sizeof(double));
    memcpy(r, rhs, n * sizeof(double));
    memcpy(p, r, n * sizeof(double));
    double gamma = dot(n, r, r);
    for (int k = 0; k < nsteps; k++) {
        jacobi_scaled_matvec(nx, ny, aP, aE, aW, aN, aS, p, Ap);
        double pAp = dot(n, p, Ap);
        alphas[k] = gamma / pAp;
        if (k < nsteps - 1) {
            const double ak = alphas[k];
#pragma omp parallel for schedule(static)
            for (long i = 0; i < (long)n; i++) r[i] -= ak * Ap[i];
            double gamma_next = dot(n, r, r);
            betas[k] = gamma_next / gamma;
            const double bk = betas[k];
#pragma omp parallel for schedule(static)
            for (long i = 0; i < (long)n; i++) p[i] = r[i] + bk * p[i];
            gamma = gamma_next;
        }
    }
    double *d = calloc(nsteps, sizeof(double)), *e = calloc(nsteps > 1 ? nsteps - 1 : 1, sizeof(double));
    d[0] = 1 / alphas[0];
    for (int k = 1; k < nsteps; k++) d[k] = 1 / alphas[k] + betas[k - 1] / alphas[k - 1];
    for (int k = 0; k < nsteps - 1; k++) e[k] = sqrt(betas[k]) / alphas[k];
    double rmin, rmax;
    tridiag_extreme_eigs(nsteps, d, e, &rmin, &rmax);
    double lmin = rmin * 0.9, lmax = rmax * 1.1;
    if (est_out) { est_out[0] = lmin; est_out[1] = lmax; }
    int ok = isfinite(lmin) && isfinite(lmax) && lmin > 0 && lmax > lmin;
    if (ok) { cs->lambda_min = lmin; cs->lambda_max = lmax; }
    cs->last_estimate_valid = ok;
    free(r); free(p); free(Ap); free(alphas); free(betas); free(d); free(e);
    return ok;
}

/* ChebyshevPreconditioner ldiv! (src/preconditioner.jl:239-267) with scratch allocated per call. */
static void cheb_apply_ws(int nx, int ny, const double *aP, const double *aE, const double *aW,
                          const double *aN, const double *aS, int degree, const orc_cheb_state *cs,
                          const double *x, double *y, double *r, double *p, double *Ap) {
    const size_t n = (size_t)nx * ny;
    const double d_mid = (cs->lambda_max + cs->lambda_min) / 2;
    const double c_rad = (cs->lambda_max - cs->lambda_min) / 2;
    double alpha = 1.0 / d_mid;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) {
        r[i] = x[i] / aP[i];
        p[i] = r[i];
        y[i] = 0.0 + alpha * p[i];
    }
    jacobi_scaled_matvec(nx, ny, aP, aE, aW, aN, aS, p, Ap);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) r[i] -= alpha * Ap[i];
    double alpha_prev = alpha;
    for (int k = 2; k <= degree; k++) {
        double t = c_rad * alpha_prev / 2;
        double beta = t * t;
        alpha = 1.0 / (d_mid - beta / alpha_prev);
        const double a = alpha;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; i++) {
            p[i] = r[i] + beta * p[i];
            y[i] += a * p[i];
        }
        jacobi_scaled_matvec(nx, ny, aP, aE, aW, aN, aS, p, Ap);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; i++) r[i] -= a * Ap[i];
        alpha_prev = alpha;
    }
}

void orc_chebyshev_apply(int nx, int ny, const double *aP, const double *aE, const double *aW,
                         const double *aN, const double *aS, int degree, const orc_cheb_state *cs,
                         const double *x, double *y) {
    const size_t n = (size_t)nx * ny;
    double *r = malloc(n * sizeof(double)), *p = malloc(n * sizeof(double)), *Ap = malloc(n * sizeof(double));
    cheb_apply_ws(nx, ny, aP, aE, aW, aN, aS, degree, cs, x, y, r, p, Ap);
    free(r); free(p); free(Ap);
}

/* ---------------------------------------------------------------------------------------------
 * Krylov.jl cg! (third-party, v0.10.8) restated: warm start x0 = Delta_x, x accumulates the
 * correction from 0 and Delta_x is added at the end.
 * ------------------------------------------------------------------------------------------- */
/* Squared norm of rhs over the GROUNDED rows (mask == 0): the rows whose unknown is a free head.
 * The OCEAN/LAND/OTHER_BASIN rows are identity rows (aP = 1, rhs = the fixed head), decoupled from
 * the rest; their residual is zero once h holds their fixed value, and their rhs (heads of order
 * 1e3 m) would otherwise dominate ||b||.  mask == NULL: every row. */
static double free_norm2(size_t n, const double *rhs, const double *mask) {
    if (!mask) return dot(n, rhs, rhs);
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long i = 0; i < (long)n; i++) s += (mask[i] == GROUNDED) ? rhs[i] * rhs[i] : 0.0;
    return s;
}

/* One Krylov.jl cg! solve as a resumable object: cg_begin (initial residual, preconditioner,
 * stopping scalars), cg_step (one iteration), cg_end (x = Delta_x + x accumulated, statistics).
 * orc_cg_masked runs them back to back; the bounded run session below interleaves them with
 * clock checks.  The arithmetic and its order are those of one uninterrupted solve. */
typedef struct {
    int nx, ny;
    size_t n;
    const double *aP, *aE, *aW, *aN, *aS, *rhs;
    double *x_io;
    orc_cg_opts o;
    orc_cheb_state *cs;
    double *x, *r, *z, *p, *Ap, *cr, *cp, *cAp;
    double gamma, rNorm, bNorm, rr, pNorm2, eps_stop, rnorm0;
    long iter, itmax;
    int solved, zero_curv, trivial;
} cg_work;

static void cg_apply_m(cg_work *w, double *dst, const double *src) {
    if (w->o.precond == 1) {
        cheb_apply_ws(w->nx, w->ny, w->aP, w->aE, w->aW, w->aN, w->aS, w->o.cheb_degree, w->cs, src, dst, w->cr, w->cp,
                      w->cAp);
    } else {
        const double *aP = w->aP;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)w->n; i++) dst[i] = src[i] / aP[i];
    }
}

static void cg_begin(cg_work *w, int nx, int ny, const double *aP, const double *aE, const double *aW,
                     const double *aN, const double *aS, const double *rhs, const double *mask, double *x_io,
                     const orc_cg_opts *o, orc_cheb_state *cs) {
    const size_t n = (size_t)nx * ny;
    memset(w, 0, sizeof(*w));
    w->nx = nx; w->ny = ny; w->n = n;
    w->aP = aP; w->aE = aE; w->aW = aW; w->aN = aN; w->aS = aS; w->rhs = rhs;
    w->x_io = x_io; w->o = *o; w->cs = cs;
    w->x = calloc(n, sizeof(double)); w->r = malloc(n * sizeof(double)); w->z = malloc(n * sizeof(double));
    w->p = malloc(n * sizeof(double)); w->Ap = malloc(n * sizeof(double));
    if (o->precond == 1) {
        w->cr = malloc(n * sizeof(double)); w->cp = malloc(n * sizeof(double)); w->cAp = malloc(n * sizeof(double));
        /* _cg_precond! refreshes the bounds from this solve's rhs (src/linear_solver.jl:853-856) */
        orc_update_chebyshev_bounds(nx, ny, aP, aE, aW, aN, aS, rhs, o->cheb_nsteps, cs, NULL);
    }
    double *r = w->r;
    /* r = b - A*Delta_x */
    orc_matvec(nx, ny, aP, aE, aW, aN, aS, x_io, r);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) r[i] = 1.0 * rhs[i] + (-1.0) * r[i];
    cg_apply_m(w, w->z, r);
    memcpy(w->p, w->z, n * sizeof(double));
    w->gamma = dot(n, r, w->z);
    w->rNorm = sqrt(w->gamma);
    w->bNorm = (o->stop_rule == 1) ? sqrt(free_norm2(n, rhs, mask)) : 0.0;
    w->rr = (o->stop_rule == 1) ? sqrt(dot(n, r, r)) : 0.0;
    w->rnorm0 = (o->stop_rule == 1) ? w->rr : w->rNorm;
    if (w->gamma == 0) {
        w->trivial = 1;
        return;
    }
    w->itmax = o->itmax > 0 ? o->itmax : 2 * (long)n;
    w->pNorm2 = w->gamma;
    w->eps_stop = o->atol + o->rtol * w->rNorm;
    w->solved = (o->stop_rule == 1) ? (w->rr <= o->rtol * w->bNorm) : (w->rNorm <= w->eps_stop);
}

static int cg_done(const cg_work *w) { return w->trivial || w->solved || w->iter >= w->itmax || w->zero_curv; }

/* One iteration (callers test cg_done first). */
static void cg_step(cg_work *w) {
    const size_t n = w->n;
    double *x = w->x, *r = w->r, *z = w->z, *p = w->p, *Ap = w->Ap;
    orc_matvec(w->nx, w->ny, w->aP, w->aE, w->aW, w->aN, w->aS, p, Ap);
    double pAp = dot(n, p, Ap);
    if (pAp <= DBL_EPSILON * w->pNorm2 && fabs(pAp) <= DBL_EPSILON * w->pNorm2) { w->zero_curv = 1; return; }
    if (isnan(pAp)) { w->zero_curv = 1; return; }
    double alpha = w->gamma / pAp;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) {
        x[i] += alpha * p[i];
        r[i] += (-alpha) * Ap[i];
    }
    cg_apply_m(w, z, r);
    double gamma_next = dot(n, r, z);
    w->rNorm = sqrt(gamma_next);
    if (w->o.stop_rule == 1) {
        w->rr = sqrt(dot(n, r, r));
        w->solved = w->rr <= w->o.rtol * w->bNorm;
    } else {
        w->solved = (w->rNorm <= w->eps_stop) || (w->rNorm + 1.0 <= 1.0);
    }
    if (!w->solved) {
        double beta = gamma_next / w->gamma;
        w->pNorm2 = gamma_next + beta * beta * w->pNorm2;
        w->gamma = gamma_next;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; i++) p[i] = 1.0 * z[i] + beta * p[i];
    }
    w->iter++;
}

static int cg_end(cg_work *w, orc_cg_stats *st) {
    const size_t n = w->n;
    double *x = w->x, *x_io = w->x_io;
    st->rnorm0 = w->rnorm0;
    if (w->trivial) {
        st->niter = 0;
        st->status = 0;
        st->rnorm = 0.0;
    } else {
        st->niter = w->iter;
        st->rnorm = (w->o.stop_rule == 1) ? w->rr : w->rNorm;
        st->status = w->zero_curv ? 2 : (w->solved ? 0 : 1);
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) x_io[i] = x[i] + x_io[i];
    free(w->x); free(w->r); free(w->z); free(w->p); free(w->Ap);
    free(w->cr); free(w->cp); free(w->cAp);
    return st->status;
}

int orc_cg(int nx, int ny, const double *aP, const double *aE, const double *aW, const double *aN,
           const double *aS, const double *rhs, double *x_io, const orc_cg_opts *o, orc_cheb_state *cs,
           orc_cg_stats *st) {
    return orc_cg_masked(nx, ny, aP, aE, aW, aN, aS, rhs, NULL, x_io, o, cs, st);
}

int orc_cg_masked(int nx, int ny, const double *aP, const double *aE, const double *aW, const double *aN,
                  const double *aS, const double *rhs, const double *mask, double *x_io, const orc_cg_opts *o,
                  orc_cheb_state *cs, orc_cg_stats *st) {
    cg_work w;
    cg_begin(&w, nx, ny, aP, aE, aW, aN, aS, rhs, mask, x_io, o, cs);
    while (!cg_done(&w)) cg_step(&w);
    return cg_end(&w, st);
}

/* ---------------------------------------------------------------------------------------------
 * elliptic_solver.jl / parabolic_solver.jl / run.jl
 * ------------------------------------------------------------------------------------------- */

/* Field-update tail shared by Picard_iteration! (src/elliptic_solver.jl:193-206) and
 * parabolic_solver! (src/parabolic_solver.jl:27-37). */
void orc_picard_tail(orc_state *s, const orc_params *p, const orc_sliding *sl) {
    orc_compute_dhdxy(s);
    orc_compute_pw(s, p);
    orc_compute_dpwdxy(s);
    orc_compute_N(s);
    orc_compute_q_and_Re_xy(s, p);
    orc_compute_Re(s);
    orc_compute_taub_xy(s, p, sl);
    orc_compute_mdot(s, p);
    orc_compute_K(s, p);
}

static int solve_linear(orc_state *s, const orc_params *p, int kfs, int parabolic, double dt,
                        const orc_cg_opts *cg, orc_cheb_state *cs, orc_cg_stats *cst) {
    const size_t n = (size_t)s->nx * s->ny;
    double *buf = malloc(6 * n * sizeof(double));
    double *aP = buf, *aE = buf + n, *aW = buf + 2 * n, *aN = buf + 3 * n, *aS = buf + 4 * n, *rhs = buf + 5 * n;
    orc_assemble_mfls(s, p, kfs, parabolic, dt, aP, aE, aW, aN, aS, rhs);
    int rc = orc_cg_masked(s->nx, s->ny, aP, aE, aW, aN, aS, rhs, s->mask, s->h, cg, cs, cst);
    free(buf);
    return rc;
}

/* Picard_iteration! (src/elliptic_solver.jl:187-208) */
int orc_picard_iteration(orc_state *s, const orc_params *p, const orc_sliding *sl, int kfs,
                         const orc_cg_opts *cg, orc_cheb_state *cs, double alpha, const double *h_prev,
                         orc_cg_stats *cst) {
    int rc = solve_linear(s, p, kfs, 0, 0.0, cg, cs, cst);
    if (alpha > 0) { /* relax_h! (src/elliptic_solver.jl:42-46) */
        const size_t n = (size_t)s->nx * s->ny;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; i++) s->h[i] = alpha * s->h[i] + (1 - alpha) * h_prev[i];
    }
    orc_picard_tail(s, p, sl);
    return rc;
}

/* Picard_loop! (src/elliptic_solver.jl:138-176) */
int orc_picard_loop(orc_state *s, const orc_params *p, const orc_sliding *sl, int kfs,
                    const orc_cg_opts *cg, orc_cheb_state *cs, const orc_picard_opts *po,
                    orc_picard_stats *pst) {
    const size_t n = (size_t)s->nx * s->ny;
    double *h_prev = malloc(n * sizeof(double));
    pst->converged = 0;
    pst->last_iter = 0;
    pst->cg_iters_total = 0;
    pst->cg_solves = 0;
    pst->cg_breakdowns = 0;
    const int check_every = po->check_every > 0 ? po->check_every : 1;
    for (int iter = 1; iter <= po->iters; iter++) {
        memcpy(h_prev, s->h, n * sizeof(double));
        orc_cg_stats cst;
        int rc = orc_picard_iteration(s, p, sl, kfs, cg, cs, po->alpha, h_prev, &cst);
        pst->cg_iters_total += cst.niter;
        pst->cg_solves++;
        if (rc == 2) pst->cg_breakdowns++;
        if (iter % check_every == 0 || iter == po->iters) {
            double dmax = 0.0, hmax = 0.0;
            for (size_t i = 0; i < n; i++) {
                dmax = jl_max(dmax, fabs(s->h[i] - h_prev[i]));
                hmax = jl_max(hmax, fabs(s->h[i]));
            }
            if (dmax / (hmax + DBL_EPSILON) < po->tol) {
                pst->converged = 1;
                pst->last_iter = iter;
                free(h_prev);
                return 0;
            }
        }
    }
    pst->last_iter = po->iters;
    free(h_prev);
    return 1;
}

/* parabolic_solver! (src/parabolic_solver.jl:16-38) */
int orc_parabolic_step(orc_state *s, const orc_params *p, const orc_sliding *sl, int kfs,
                       const orc_cg_opts *cg, orc_cheb_state *cs, double dt, orc_cg_stats *cst) {
    int rc = solve_linear(s, p, kfs, 1, dt, cg, cs, cst);
    orc_picard_tail(s, p, sl);
    return rc;
}

/* update_ieb! (src/melt_input.jl:30, :86-94) */
void orc_update_ieb(orc_state *s, const orc_melt *mi, double t) {
    if (mi->kind != 1 && mi->kind != 2) return;
    double yf = fmod(t / mi->seconds_per_year, 1.0);
    if (yf < 0) yf += 1.0;
    double i_ma = (mi->t_start <= yf && yf <= mi->t_start + mi->period)
                      ? (mi->offset - mi->amplitude * cos(mi->omega * (yf - mi->t_start)))
                      : mi->i_min;
    const double v = i_ma / mi->seconds_per_year;
    const size_t n = (size_t)s->nx * s->ny;
    if (mi->kind == 2 && mi->base) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; i++) s->ieb[i] = v + mi->base[i];
    } else {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; i++) s->ieb[i] = v;
    }
}

/* run! loop body (src/run.jl:37-43) over step! (:82-88). */
int orc_run(orc_state *s, const orc_params *p, const orc_sliding *sl, const orc_melt *mi,
            const orc_sim *sim, const orc_cg_opts *cg, orc_cheb_state *cs, const orc_picard_opts *po,
            int tsteps, double *total_time, orc_picard_stats *per_step) {
    int worst = 0;
    for (int t = 0; t < tsteps; t++) {
        orc_update_ieb(s, mi, *total_time);
        orc_picard_stats pst;
        memset(&pst, 0, sizeof(pst));
        if (sim->head_scheme == 0) {
            int rc = orc_picard_loop(s, p, sl, sim->kfs, cg, cs, po, &pst);
            if (rc > worst) worst = rc;
        } else {
            orc_cg_stats cst;
            int rc = orc_parabolic_step(s, p, sl, sim->kfs, cg, cs, sim->dt, &cst);
            pst.converged = -1;
            pst.last_iter = -1;
            pst.cg_iters_total = cst.niter;
            pst.cg_solves = 1;
            pst.cg_breakdowns = rc == 2;
        }
        orc_step_b(s, p, sim->gap_scheme, sim->dt);
        *total_time += sim->dt;
        if (per_step) per_step[t] = pst;
    }
    return worst;
}

/* ---------------------------------------------------------------------------------------------
 * Bounded run session: the run! loop above (update_ieb!, Picard_loop! or parabolic_solver!,
 * step_b!) executed as a resumable sequence, so that a caller can spend a fixed amount of wall
 * time on it, stop between two CG iterations, and continue later with nothing recomputed.  The
 * arithmetic is that of orc_run.  Used to time the CPU restatement on workloads whose timesteps
 * take longer than a benchmark can wait for.
 * ------------------------------------------------------------------------------------------- */
enum { SES_STEP_START = 0, SES_SOLVE_START = 1, SES_CG = 2, SES_STEP_END = 3 };

struct orc_session {
    orc_state *s;
    orc_params p;
    orc_sliding sl;
    orc_melt mi;
    orc_sim sim;
    orc_cg_opts cg;
    orc_picard_opts po;
    orc_cheb_state *cs;
    double total_time;
    double *sys;     /* aP, aE, aW, aN, aS, rhs */
    double *h_prev;
    cg_work w;
    int phase, pic_iter, step_converged;
    long step_cg;
    double step_s;   /* seconds spent on the timestep in progress */
    orc_session_progress pr;
};

static double wtime(void) {
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return (double)clock() / CLOCKS_PER_SEC;
#endif
}

orc_session *orc_session_create(orc_state *s, const orc_params *p, const orc_sliding *sl, const orc_melt *mi,
                                const orc_sim *sim, const orc_cg_opts *cg, orc_cheb_state *cs,
                                const orc_picard_opts *po, double total_time) {
    orc_session *S = calloc(1, sizeof(orc_session));
    const size_t n = (size_t)s->nx * s->ny;
    S->s = s; S->p = *p; S->sl = *sl; S->mi = *mi; S->sim = *sim; S->cg = *cg; S->po = *po; S->cs = cs;
    S->total_time = total_time;
    S->sys = malloc(6 * n * sizeof(double));
    S->h_prev = malloc(n * sizeof(double));
    S->phase = SES_STEP_START;
    S->pr.all_converged = 1;
    return S;
}

void orc_session_destroy(orc_session *S) {
    if (!S) return;
    if (S->phase == SES_CG) {
        orc_cg_stats st;
        cg_end(&S->w, &st);
    }
    free(S->sys);
    free(S->h_prev);
    free(S);
}

/* Advances the run by about `seconds` of wall time (it stops at the first CG-iteration, solve or
 * timestep boundary after the budget; max_steps > 0 also stops it after that many completed
 * timesteps in total).  Returns 1 while the run has more to do, 0 once max_steps are complete. */
int orc_session_advance(orc_session *S, double seconds, int max_steps, orc_session_progress *out) {
    orc_state *s = S->s;
    const size_t n = (size_t)s->nx * s->ny;
    const double t0 = wtime();
    double mark = t0;
    int more = 1;
    const int check_every = S->po.check_every > 0 ? S->po.check_every : 1;
    for (;;) {
        if (max_steps > 0 && S->pr.steps_done >= max_steps) { more = 0; break; }
        if (wtime() - t0 >= seconds) break;
        if (S->phase == SES_STEP_START) {
            orc_update_ieb(s, &S->mi, S->total_time);
            S->pic_iter = 0;
            S->step_cg = 0;
            S->step_converged = S->sim.head_scheme == 0 ? 0 : -1;
            S->phase = SES_SOLVE_START;
        } else if (S->phase == SES_SOLVE_START) {
            double *b = S->sys;
            const int parabolic = S->sim.head_scheme != 0;
            S->pic_iter++;
            if (!parabolic) memcpy(S->h_prev, s->h, n * sizeof(double));
            orc_assemble_mfls(s, &S->p, S->sim.kfs, parabolic, parabolic ? S->sim.dt : 0.0, b, b + n, b + 2 * n,
                              b + 3 * n, b + 4 * n, b + 5 * n);
            cg_begin(&S->w, s->nx, s->ny, b, b + n, b + 2 * n, b + 3 * n, b + 4 * n, b + 5 * n, s->mask, s->h,
                     &S->cg, S->cs);
            S->pr.cg_iter_now = 0;
            S->phase = SES_CG;
        } else if (S->phase == SES_CG) {
            if (!cg_done(&S->w)) {
                cg_step(&S->w);
                S->pr.cg_iters++;
                S->pr.cg_iter_now++;
                S->step_cg++;
                continue;
            }
            orc_cg_stats cst;
            cg_end(&S->w, &cst);
            if (cst.status == 2) S->pr.cg_breakdowns++;
            S->pr.picard_iters++;
            if (S->sim.head_scheme != 0) {
                orc_picard_tail(s, &S->p, &S->sl);
                S->phase = SES_STEP_END;
                continue;
            }
            const double alpha = S->po.alpha;
            if (alpha > 0) { /* relax_h! (src/elliptic_solver.jl:42-46) */
#pragma omp parallel for schedule(static)
                for (long i = 0; i < (long)n; i++) s->h[i] = alpha * s->h[i] + (1 - alpha) * S->h_prev[i];
            }
            orc_picard_tail(s, &S->p, &S->sl);
            int stop = S->pic_iter >= S->po.iters;
            if (S->pic_iter % check_every == 0 || S->pic_iter == S->po.iters) {
                double dmax = 0.0, hmax = 0.0;
                for (size_t i = 0; i < n; i++) {
                    dmax = jl_max(dmax, fabs(s->h[i] - S->h_prev[i]));
                    hmax = jl_max(hmax, fabs(s->h[i]));
                }
                if (dmax / (hmax + DBL_EPSILON) < S->po.tol) {
                    S->step_converged = 1;
                    stop = 1;
                }
            }
            S->phase = stop ? SES_STEP_END : SES_SOLVE_START;
        } else { /* SES_STEP_END */
            orc_step_b(s, &S->p, S->sim.gap_scheme, S->sim.dt);
            S->total_time += S->sim.dt;
            const double now = wtime();
            S->step_s += now - mark;
            mark = now;
            S->pr.steps_done++;
            S->pr.completed_s += S->step_s;
            S->pr.last_step_s = S->step_s;
            S->pr.last_picard = S->pic_iter;
            S->pr.last_cg = S->step_cg;
            S->pr.last_converged = S->step_converged;
            if (S->step_converged == 0) S->pr.all_converged = 0;
            S->step_s = 0.0;
            S->phase = SES_STEP_START;
        }
    }
    const double now = wtime();
    S->step_s += now - mark;
    S->pr.elapsed += now - t0;
    S->pr.pic_iter_now = S->phase == SES_STEP_START ? 0 : S->pic_iter;
    S->pr.step_s_now = S->step_s;
    S->pr.total_time = S->total_time;
    if (out) *out = S->pr;
    return more;
}
