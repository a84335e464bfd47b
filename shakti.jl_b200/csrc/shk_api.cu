// shk_api.cu -- the extern "C" boundary of libshakti_b200 and its host-side drivers
// (Picard_loop!, parabolic_solver!, step!, run!).  See include/shakti_b200.h for the contract.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cstdlib>
#include <new>
#include <string>

#include "shk_internal.cuh"

namespace shk {

int fail(Ctx *c, int status, const std::string &msg) {
    if (c) c->err = msg;
    return status;
}

int check_cuda(Ctx *c, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return SHK_OK;
    return fail(c, SHK_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

int check_launch(Ctx *c, const char *what) { return check_cuda(c, cudaGetLastError(), what); }

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static void derive_params(Ctx *c) {
    const shk_params &p = c->hp;
    Params &P = c->P;
    P.rho_w = p.rho_w; P.rho_sw = p.rho_sw; P.rho_i = p.rho_i; P.g = p.g; P.nu = p.nu; P.n = p.n;
    P.omega = p.omega; P.L = p.L; P.br = p.br; P.lr = p.lr; P.ct = p.ct; P.cw = p.cw; P.p_atm = p.p_atm;
    P.b_min = p.b_min; P.b_max = p.b_max; P.e_v = p.e_v;
    // canonical_exponent (src/model_parameters.jl:122-123): integral exponents take the integer path
    P.nm1 = p.n - 1;
    P.inv_n = 1 / p.n;
    P.n_int = (p.n == floor(p.n) && fabs(p.n) < 1e6) ? (int)p.n : -1;
    P.nm1_int = (P.nm1 == floor(P.nm1) && fabs(P.nm1) < 1e6) ? (int)P.nm1 : -1;
    if (P.n_int < 0) P.n_int = -1;
    if (P.nm1_int < 0) P.nm1_int = -1;
    P.with_sensible = !(p.ct == 0.0 || p.cw == 0.0); // src/simulation.jl:132
    P.root3 = p.n == 3.0;
    P.Linv = 1 / p.L;
    P.dx = c->dx;
    P.dy = c->dy;
    P.dx2 = c->dx * c->dx;
    P.dy2 = c->dy * c->dy;
}

static int ctx_alloc(Ctx *c) {
    const size_t n = (size_t)c->nx * c->ny;
    const size_t A = 256;
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes, A);
        return o;
    };
    const size_t dN = n * sizeof(double), fN = n * sizeof(float);
    size_t o_mask8 = carve(n);
    size_t o_aP = carve(dN), o_aE = carve(dN), o_aN = carve(dN), o_rhs = carve(dN);
    size_t o_x = carve(dN), o_r = carve(dN), o_z = carve(dN), o_p0 = carve(dN), o_p1 = carve(dN), o_Ap = carve(dN);
    size_t o_hprev = carve(dN), o_r2 = carve(dN);
    size_t o_cr0 = carve(dN), o_cr1 = carve(dN), o_cp0 = carve(dN), o_cp1 = carve(dN);
    size_t o_f[16];
    for (int i = 0; i < 16; i++) o_f[i] = carve(fN);
    // multigrid hierarchy: level 0 aliases the Float32 operator; levels >= 1 own their arrays
    int dims[2 * kMgMaxLevels];
    c->mg_levels = mg_levels_for(c->nx, c->ny, dims, kMgMaxLevels);
    if (c->mg_levels < 1) return fail(c, SHK_BAD_ARG, "grid too large for the multigrid hierarchy");
    size_t o_act0 = carve(n);
    size_t o_mg[kMgMaxLevels][10];
    for (int l = 1; l < c->mg_levels; l++) {
        const size_t m = (size_t)dims[2 * l] * dims[2 * l + 1];
        for (int k = 0; k < 3; k++) o_mg[l][k] = carve(m * sizeof(double));
        for (int k = 3; k < 9; k++) o_mg[l][k] = carve(m * sizeof(float)); // aE, aN, dP, wD, x0, x1
        o_mg[l][9] = carve(m * sizeof(float) + m);                       // b, then act bytes
    }
    size_t o_part = carve((size_t)kMaxRedValues * c->max_blocks * sizeof(double));
    size_t o_cnt = carve(64);
    size_t o_dev = carve(sizeof(DevScalars));
    c->arena_bytes = off;
    cudaError_t e = cudaMalloc(&c->arena, off);
    if (e != cudaSuccess) return check_cuda(c, e, "cudaMalloc(workspace)");
    char *b = (char *)c->arena;
    c->mask8 = (uint8_t *)(b + o_mask8);
    c->aP = (double *)(b + o_aP); c->aE = (double *)(b + o_aE); c->aN = (double *)(b + o_aN);
    c->rhs = (double *)(b + o_rhs);
    c->x = (double *)(b + o_x); c->r = (double *)(b + o_r); c->z = (double *)(b + o_z);
    c->p[0] = (double *)(b + o_p0); c->p[1] = (double *)(b + o_p1); c->Ap = (double *)(b + o_Ap);
    c->h_prev = (double *)(b + o_hprev);
    c->r2 = (double *)(b + o_r2);
    c->cr[0] = (double *)(b + o_cr0); c->cr[1] = (double *)(b + o_cr1);
    c->cp[0] = (double *)(b + o_cp0); c->cp[1] = (double *)(b + o_cp1);
    float **fl[16] = {&c->aP32, &c->aE32, &c->aN32, &c->b32, &c->x32, &c->r32, &c->z32, &c->p32[0], &c->p32[1],
                      &c->Ap32, &c->cr32[0], &c->cr32[1], &c->cp32[0], &c->cp32[1], &c->dP32, &c->wD32};
    for (int i = 0; i < 16; i++) *fl[i] = (float *)(b + o_f[i]);
    for (int l = 0; l < c->mg_levels; l++) {
        MgLevel &m = c->mg[l];
        m.nx = dims[2 * l];
        m.ny = dims[2 * l + 1];
        if (l == 0) {
            m.aE = c->aE32; m.aN = c->aN32; m.dP = c->dP32; m.wD = c->wD32;
            m.act = (uint8_t *)(b + o_act0);
            m.x[0] = c->cr32[0]; m.x[1] = c->cr32[1];
            m.b = nullptr;
            continue;
        }
        const size_t cnt = (size_t)m.nx * m.ny;
        m.aE64 = (double *)(b + o_mg[l][0]); m.aN64 = (double *)(b + o_mg[l][1]); m.dP64 = (double *)(b + o_mg[l][2]);
        m.aE = (float *)(b + o_mg[l][3]); m.aN = (float *)(b + o_mg[l][4]); m.dP = (float *)(b + o_mg[l][5]);
        m.wD = (float *)(b + o_mg[l][6]); m.x[0] = (float *)(b + o_mg[l][7]); m.x[1] = (float *)(b + o_mg[l][8]);
        m.b = (float *)(b + o_mg[l][9]);
        m.act = (uint8_t *)(b + o_mg[l][9] + cnt * sizeof(float));
    }
    c->partials = (double *)(b + o_part);
    c->counter = (unsigned int *)(b + o_cnt);
    c->dev = (DevScalars *)(b + o_dev);
    e = cudaMemsetAsync(c->arena, 0, off, c->stream);
    if (e != cudaSuccess) return check_cuda(c, e, "cudaMemset(workspace)");
    e = cudaHostAlloc(&c->host_dev, sizeof(DevScalars), cudaHostAllocMapped);
    if (e != cudaSuccess) return check_cuda(c, e, "cudaHostAlloc");
    if (cudaHostGetDevicePointer((void **)&c->host_dev_d, c->host_dev, 0) != cudaSuccess) {
        cudaGetLastError();
        c->host_dev_d = nullptr;  // control scalars then move by cudaMemcpyAsync
    }
    memset(c->host_dev, 0, sizeof(DevScalars));
    // ChebyshevPreconditioner placeholder bounds (1, 1) (src/preconditioner.jl:179-186)
    c->host_dev->cheb.lam_min = 1.0;
    c->host_dev->cheb.lam_max = 1.0;
    e = cudaMemcpyAsync(&c->dev->cheb, &c->host_dev->cheb, sizeof(ChebDev), cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return check_cuda(c, e, "upload chebyshev state");
    return check_cuda(c, cudaStreamSynchronize(c->stream), "workspace init");
}

} // namespace shk

using namespace shk;

static Ctx *as_ctx(void *p) { return reinterpret_cast<Ctx *>(p); }
static const Ctx *as_ctx(const void *p) { return reinterpret_cast<const Ctx *>(p); }

#define REQUIRE_CTX(c)                                                                                    \
    if (!(c)) return SHK_BAD_ARG;

static int require_ready(Ctx *c) {
    if (!c->params_set) return fail(c, SHK_NOT_BOUND, "shk_set_params has not been called");
    if (!c->state_bound) return fail(c, SHK_NOT_BOUND, "shk_bind_state has not been called");
    if (!c->sliding_set) return fail(c, SHK_NOT_BOUND, "shk_set_sliding_law has not been called");
    return SHK_OK;
}

extern "C" {

SHK_API int shk_version(void) { return 1; }

SHK_API const char *shk_status_string(int s) {
    switch (s) {
    case SHK_OK: return "ok";
    case SHK_NOT_CONVERGED: return "not converged";
    case SHK_BREAKDOWN: return "breakdown";
    case SHK_BAD_ARG: return "bad argument";
    case SHK_CUDA_ERROR: return "cuda error";
    case SHK_NOT_BOUND: return "not bound";
    default: return "unknown";
    }
}

// The multigrid cycle's smoothing weights and coarse-correction scaling omega_c by grid size.
// Piecewise-constant (unsmoothed) aggregation under-corrects the smooth error, so every coarse
// correction is scaled by omega_c inside (0, 2), where the symmetric cycle stays a positive definite
// preconditioner; the deeper the hierarchy, the smaller the best scaling.  The two sweeps on each
// side take either one damping omega (damped Jacobi) or the degree-2 Chebyshev pair of weights.
// Measured outer CG iterations over 10 timesteps of the seasonal workloads (Picard re-solves):
//   damped Jacobi (0.8, 1.6) / (0.9, 1.3) / (0.9, 1.45), Chebyshev pair with the size's omega_c:
//   4096^2: 3182 / 2163 / 2309 (at 1.4) / 2003;   2048^2: 2089 / 1729 / 1788 / 1623;
//   1024^2: 1600 / 1520 / 1448 / 1310;   the ragged 128^2-1024^2 ensemble (20 steps, Jacobi only):
//   266059 / 320142 / 279021.  Undamped Jacobi (omega = 1) leaves the highest frequencies: 9626 at
//   4096^2.  Grids of at most 512 cells a side keep damped Jacobi (0.8, 1.6).
static void mg_chebyshev_weights(Ctx *c) {
    // the reciprocals of the two roots of the degree-2 Chebyshev polynomial for the interval
    // [0.45, 1.8] of the spectrum of D^-1 A; the smaller weight first before the coarse correction
    // and last after it
    const double lo = 0.45, hi = 1.8, mid = 0.5 * (hi + lo), half = 0.5 * (hi - lo) * std::sqrt(0.5);
    const double tau1 = 1.0 / (mid + half), tau2 = 1.0 / (mid - half);
    c->mg_omega = (float)tau1;
    c->mg_s2 = (float)(tau2 / tau1);
}

static void mg_default_weights(Ctx *c) {
    const int n = std::max(c->nx, c->ny);
    c->mg_omega_c = n > 1024 ? 1.3f : (n > 512 ? 1.45f : 1.6f);
    if (n > 512) {
        mg_chebyshev_weights(c);
    } else {
        c->mg_omega = 0.8f;
        c->mg_s2 = 1.0f;
    }
}

SHK_API int shk_create(int nx, int ny, double lx, double ly, void *stream, void **ctx_out) {
    if (!ctx_out) return SHK_BAD_ARG;
    *ctx_out = nullptr;
    if (nx < 2 || ny < 2) return SHK_BAD_ARG; // dx = lx/(nx-1) needs nx >= 2
    if ((long long)nx * ny > (1LL << 30)) return SHK_BAD_ARG;
    if (!(lx > 0) || !(ly > 0)) return SHK_BAD_ARG;
    Ctx *c = new (std::nothrow) Ctx();
    if (!c) return SHK_CUDA_ERROR;
    c->nx = nx;
    c->ny = ny;
    c->lx = lx;
    c->ly = ly;
    c->dx = lx / (nx - 1); // Grid (src/grid.jl:26-35)
    c->dy = ly / (ny - 1);
    c->stream = (cudaStream_t)stream;
    int rc = check_cuda(c, cudaGetDevice(&c->device), "cudaGetDevice");
    if (!rc) rc = check_cuda(c, cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device),
                             "cudaDeviceGetAttribute");
    if (rc) {
        delete c;
        return rc;
    }
    const long long tiles = (long long)((nx + kTX - 1) / kTX) * ((ny + kTY - 1) / kTY);
    long long g = (long long)c->num_sms * 6;
    if (g > tiles) g = tiles;
    if (g < 1) g = 1;
    c->grid_stencil = (int)g;
    // Row-marching tiles: kMarchX columns by march_th rows; the height is chosen so that the grid
    // offers about 12 blocks per SM (one resident wave), between 8 and 64 rows.
    {
        const long long tiles_x = (nx + kMarchX - 1) / kMarchX;
        long long th = (long long)ny * tiles_x / ((long long)c->num_sms * 12);
        if (th > 64) th = 64;
        if (th < 8) th = 8;
        c->march_th = (int)th;
        c->march_blocks = (int)(tiles_x * ((ny + th - 1) / th));
    }
    mg_default_weights(c);
    if (const char *v = getenv("SHK_MG_NU")) c->mg_nu = std::max(1, atoi(v));
    // SHK_MG_CHEB=1: the Chebyshev pair on every grid size; 0: damped Jacobi (omega 0.9 above 512
    // cells a side, 0.8 below)
    if (const char *v = getenv("SHK_MG_CHEB")) {
        if (atoi(v) != 0) {
            mg_chebyshev_weights(c);
        } else {
            c->mg_omega = std::max(c->nx, c->ny) > 512 ? 0.9f : 0.8f;
            c->mg_s2 = 1.0f;
        }
    }
    // SHK_MG_OMEGA: damped Jacobi with this damping
    if (const char *v = getenv("SHK_MG_OMEGA")) {
        c->mg_omega = (float)atof(v);
        c->mg_s2 = 1.0f;
    }
    if (const char *v = getenv("SHK_MG_OMEGA_C")) c->mg_omega_c = (float)atof(v);
    if (const char *v = getenv("SHK_MG_FUSED")) c->mg_fused = std::min(2, std::max(0, atoi(v)));
    if (const char *v = getenv("SHK_MG_TMA")) c->mg_tma = atoi(v) != 0;
    // SHK_MG_CLUSTER=1: the coarse levels from the finest one whose row slabs fit eight CTAs' shared
    // memory run on one thread-block cluster (default: tile kernels down to the one-block bottom)
    if (const char *v = getenv("SHK_MG_CLUSTER")) c->mg_cluster = atoi(v) != 0;
    // SHK_MG_PAIR_X=0: the multigrid form's x updated in every iteration (the same x bit for bit)
    if (const char *v = getenv("SHK_MG_PAIR_X")) c->mg_pair_x = atoi(v) != 0;
    // SHK_CG_GRAPHS: 0 issues each CG iteration's kernels directly, 1 replays one CUDA graph per
    // iteration in host-sized batches, 2 (default) runs the whole iteration loop as one graph with a
    // device-side WHILE node
    if (const char *v = getenv("SHK_CG_GRAPHS")) {
        c->graph_mode = std::min(2, std::max(0, atoi(v)));
        c->graphs_disabled = c->graph_mode == 0;
    }
    c->max_blocks = c->grid_stencil > c->march_blocks ? c->grid_stencil : c->march_blocks;
    if (c->max_blocks < c->num_sms * 8) c->max_blocks = c->num_sms * 8;
    rc = mg_set_first_wait_polls();
    if (!rc) rc = ctx_alloc(c);
    if (rc) {
        if (c->arena) cudaFree(c->arena);
        if (c->host_dev) cudaFreeHost(c->host_dev);
        delete c;
        return rc;
    }
    *ctx_out = c;
    return SHK_OK;
}

SHK_API int shk_destroy(void *ctx) {
    Ctx *c = as_ctx(ctx);
    if (!c) return SHK_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    else cudaDeviceSynchronize();
    for (auto &g : c->graphs) cudaGraphExecDestroy(g.exec);
    c->graphs.clear();
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    mg_release(c);
    if (c->arena) cudaFree(c->arena);
    if (c->host_dev) cudaFreeHost(c->host_dev);
    delete c;
    return SHK_OK;
}

SHK_API const char *shk_last_error(const void *ctx) {
    const Ctx *c = as_ctx(ctx);
    return c ? c->err.c_str() : "null context";
}

SHK_API int shk_set_stream(void *ctx, void *stream) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    c->stream = (cudaStream_t)stream;
    return SHK_OK;
}

SHK_API int shk_set_params(void *ctx, const shk_params *p) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!p) return fail(c, SHK_BAD_ARG, "null params");
    if (!(p->L != 0.0) || !(p->nu > 0) || !(p->rho_w > 0) || !(p->g != 0.0) || !(p->n > 0))
        return fail(c, SHK_BAD_ARG, "invalid ModelParameters (need L != 0, nu > 0, rho_w > 0, g != 0, n > 0)");
    c->hp = *p;
    derive_params(c);
    c->params_set = true;
    return SHK_OK;
}

SHK_API int shk_set_sliding_law(void *ctx, const shk_sliding_law *sl) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!sl || sl->kind < 0 || sl->kind > SHK_SLIDING_PRESCRIBED) return fail(c, SHK_BAD_ARG, "invalid sliding law");
    if ((sl->kind == SHK_SLIDING_REG_COULOMB_FIELD || sl->kind == SHK_SLIDING_REG_COULOMB_V0 ||
         sl->kind == SHK_SLIDING_LINEAR) &&
        (!sl->Cx || !sl->Cy))
        return fail(c, SHK_BAD_ARG, "sliding law needs face coefficient arrays Cx/Cy");
    c->SL.kind = sl->kind;
    c->SL.C = sl->C;
    c->SL.v0 = sl->v0;
    c->SL.Cx = sl->Cx;
    c->SL.Cy = sl->Cy;
    c->sliding_set = true;
    return SHK_OK;
}

SHK_API int shk_set_schemes(void *ctx, int kface, int gap) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (kface != SHK_KFACE_ARITHMETIC && kface != SHK_KFACE_HARMONIC)
        return fail(c, SHK_BAD_ARG, "unknown k-face scheme (expected arithmetic or harmonic)");
    if (gap != SHK_GAP_EXPLICIT && gap != SHK_GAP_IMPLICIT)
        return fail(c, SHK_BAD_ARG, "unknown gap scheme (expected explicit or implicit)");
    c->kfs = kface;
    c->gap = gap;
    return SHK_OK;
}

SHK_API int shk_bind_state(void *ctx, const shk_state *s) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!s) return fail(c, SHK_BAD_ARG, "null state");
    const double *const *f = reinterpret_cast<const double *const *>(s);
    for (size_t i = 0; i < sizeof(shk_state) / sizeof(double *); i++)
        if (!f[i]) return fail(c, SHK_BAD_ARG, "state field " + std::to_string(i) + " is null");
    c->st = *s;
    c->state_bound = true;
    return SHK_OK;
}

SHK_API int shk_set_initial_conditions(void *ctx) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = require_ready(c);
    if (rc) return rc;
    rc = launch_initial_conditions(c);
    if (rc) return rc;
    c->initialized = true;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "set_initial_conditions");
}

SHK_API int shk_assemble(void *ctx, int parabolic, double dt) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = require_ready(c);
    if (rc) return rc;
    if (parabolic && !(dt != 0.0)) return fail(c, SHK_BAD_ARG, "parabolic assembly needs dt != 0");
    if (!c->initialized && (rc = build_mask8(c))) return rc;
    rc = launch_assemble(c, parabolic, dt, false);
    if (rc) return rc;
    c->assembled = true;
    c->assembled_parabolic = parabolic != 0;
    return SHK_OK;
}

SHK_API int shk_export_mfls(void *ctx, double *aP, double *aE, double *aW, double *aN, double *aS, double *rhs) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!c->assembled) return fail(c, SHK_NOT_BOUND, "system not assembled");
    int rc = launch_export_mfls(c, aP, aE, aW, aN, aS, rhs);
    if (rc) return rc;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "export mfls");
}

SHK_API int shk_matvec(void *ctx, const double *x, double *y) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!c->assembled) return fail(c, SHK_NOT_BOUND, "system not assembled");
    if (!x || !y) return fail(c, SHK_BAD_ARG, "null vector");
    int rc = launch_matvec(c, x, y);
    if (rc) return rc;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "matvec");
}

SHK_API int shk_update_chebyshev_bounds(void *ctx, int nsteps, const double *rhs, double *est_out, int *adopted) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!c->assembled) return fail(c, SHK_NOT_BOUND, "system not assembled");
    int rc = run_chebyshev_bounds(c, nsteps, rhs ? rhs : c->rhs);
    if (rc) return rc;
    if ((rc = read_scalars(c))) return rc;
    if (est_out) {
        est_out[0] = c->host_dev->cheb.est_min;
        est_out[1] = c->host_dev->cheb.est_max;
    }
    if (adopted) *adopted = c->host_dev->cheb.adopted;
    return SHK_OK;
}

SHK_API int shk_get_chebyshev_bounds(void *ctx, double *lmin, double *lmax) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = read_scalars(c);
    if (rc) return rc;
    if (lmin) *lmin = c->host_dev->cheb.lam_min;
    if (lmax) *lmax = c->host_dev->cheb.lam_max;
    return SHK_OK;
}

SHK_API int shk_set_chebyshev_bounds(void *ctx, double lmin, double lmax) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = cheb_set_bounds(c, lmin, lmax);
    if (rc) return rc;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "set chebyshev bounds");
}

SHK_API int shk_chebyshev_apply(void *ctx, int degree, const double *x, double *y) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!c->assembled) return fail(c, SHK_NOT_BOUND, "system not assembled");
    if (!x || !y) return fail(c, SHK_BAD_ARG, "null vector");
    int rc = launch_chebyshev_apply_standalone(c, degree, x, y);
    if (rc) return rc;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "chebyshev apply");
}

static int validate_cg(Ctx *c, const shk_cg_opts *o) {
    if (!o) return fail(c, SHK_BAD_ARG, "null cg options");
    if (o->precond == SHK_PRECOND_CHEBYSHEV) {
        if (o->cheb_degree < 1) return fail(c, SHK_BAD_ARG, "ChebyshevPreconditioner: degree must be >= 1");
        if (o->cheb_nsteps < 2) return fail(c, SHK_BAD_ARG, "ChebyshevPreconditioner: nsteps_estimate must be >= 2");
    } else if (o->precond == SHK_PRECOND_MULTIGRID) {
        if (o->precision != SHK_FP64)
            return fail(c, SHK_BAD_ARG, "the multigrid preconditioner runs inside the Float64 CG (precision SHK_FP64)");
    } else if (o->precond != SHK_PRECOND_JACOBI) {
        return fail(c, SHK_BAD_ARG, "unknown preconditioner");
    }
    if (o->stop_rule != SHK_STOP_KRYLOV && o->stop_rule != SHK_STOP_RELRES) return fail(c, SHK_BAD_ARG, "unknown stop rule");
    if (o->precision == SHK_MIXED && o->stop_rule != SHK_STOP_RELRES)
        return fail(c, SHK_BAD_ARG, "the mixed-precision form uses the relative-residual stop rule");
    if (o->precision != SHK_FP64 && o->precision != SHK_MIXED) return fail(c, SHK_BAD_ARG, "unknown precision");
    if (!(o->rtol >= 0) || !(o->atol >= 0)) return fail(c, SHK_BAD_ARG, "tolerances must be >= 0");
    return SHK_OK;
}

SHK_API int shk_cg_solve(void *ctx, const shk_cg_opts *o, shk_cg_stats *st) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = validate_cg(c, o);
    if (rc) return rc;
    if (!c->assembled) return fail(c, SHK_NOT_BOUND, "system not assembled");
    shk_cg_stats s;
    memset(&s, 0, sizeof(s));
    rc = run_cg(c, o, &s);
    if (st) *st = s;
    if (rc) return rc;
    return s.status;
}

SHK_API int shk_solve_elliptic(void *ctx, const shk_cg_opts *o, shk_cg_stats *st) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = shk_assemble(ctx, 0, 0.0);
    if (rc) return rc;
    return shk_cg_solve(ctx, o, st);
}

SHK_API int shk_solve_parabolic(void *ctx, double dt, const shk_cg_opts *o, shk_cg_stats *st) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = shk_assemble(ctx, 1, dt);
    if (rc) return rc;
    return shk_cg_solve(ctx, o, st);
}

SHK_API int shk_picard_tail(void *ctx) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = require_ready(c);
    if (rc) return rc;
    if (!c->initialized && (rc = build_mask8(c))) return rc;
    rc = launch_tail(c, false);
    if (rc) return rc;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "picard tail");
}

SHK_API int shk_relax_h(void *ctx, double alpha, const double *h_prev) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!c->state_bound || !h_prev) return fail(c, SHK_BAD_ARG, "state not bound or null h_prev");
    int rc = launch_relax(c, alpha, h_prev);
    if (rc) return rc;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "relax_h");
}

// Picard_loop! (src/elliptic_solver.jl:138-176)
SHK_API int shk_picard_solve(void *ctx, const shk_picard_opts *po, const shk_cg_opts *o, shk_picard_stats *st) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = require_ready(c);
    if (rc) return rc;
    if (!po || po->iters < 1) return fail(c, SHK_BAD_ARG, "PicardSolver needs iters >= 1");
    if ((rc = validate_cg(c, o))) return rc;
    if (!c->initialized && (rc = build_mask8(c))) return rc;
    shk_picard_stats s;
    memset(&s, 0, sizeof(s));
    const int check_every = po->check_every > 0 ? po->check_every : 1;
    const bool relax = po->alpha > 0; // NaN / <= 0: NoHeadRelaxation
    int status = SHK_NOT_CONVERGED;
    for (int iter = 1; iter <= po->iters; iter++) {
        // h_prev .= h is fused into the assembly pass (first step of the iteration)
        if ((rc = launch_assemble(c, 0, 0.0, true))) return rc;
        c->assembled = true;
        c->assembled_parabolic = false;
        shk_cg_stats cs;
        memset(&cs, 0, sizeof(cs));
        rc = run_cg(c, o, &cs);
        if (rc) return rc;
        s.cg_iters_total += cs.niter;
        s.cg_solves++;
        if (cs.status == SHK_BREAKDOWN) s.cg_breakdowns++;
        if (relax && (rc = launch_relax(c, po->alpha, c->h_prev))) return rc;
        const bool check = (iter % check_every == 0) || iter == po->iters;
        if ((rc = launch_tail(c, check))) return rc;
        if (check) {
            if ((rc = read_scalars(c))) return rc;
            s.max_dh = c->host_dev->pic.dmax;
            s.max_h = c->host_dev->pic.hmax;
            if (s.max_dh / (s.max_h + DBL_EPSILON) < po->tol) {
                s.converged = 1;
                s.last_iter = iter;
                status = SHK_OK;
                break;
            }
        }
        s.last_iter = iter;
    }
    if (!s.converged) s.last_iter = po->iters;
    if (st) *st = s;
    return status;
}

SHK_API int shk_initial_residual(void *ctx, double *rnorm, double *bnorm) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = require_ready(c);
    if (rc) return rc;
    if (!c->initialized && (rc = build_mask8(c))) return rc;
    if ((rc = launch_assemble(c, 0, 0.0, false))) return rc;
    c->assembled = true;
    c->assembled_parabolic = false;
    return residual_norms(c, nullptr, rnorm, bnorm);
}

SHK_API int shk_residual_of(void *ctx, const double *x, double *rnorm, double *bnorm) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!x) return fail(c, SHK_BAD_ARG, "null vector");
    if (!c->assembled) return fail(c, SHK_NOT_BOUND, "no assembled system: call shk_assemble or shk_initial_residual");
    return residual_norms(c, x, rnorm, bnorm);
}

SHK_API int shk_smooth_guess(void *ctx, double *x, double *tmp, int sweeps, double omega) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!x || !tmp || sweeps < 0) return fail(c, SHK_BAD_ARG, "bad smoothing arguments");
    if (!c->assembled) return fail(c, SHK_NOT_BOUND, "no assembled system: call shk_assemble or shk_initial_residual");
    return jacobi_smooth(c, x, tmp, sweeps, omega);
}

SHK_API int shk_set_cg_warm_start(void *ctx, const double *x0) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    c->ws_x0 = x0;
    return SHK_OK;
}

// parabolic_solver! (src/parabolic_solver.jl:16-38)
SHK_API int shk_parabolic_step(void *ctx, double dt, const shk_cg_opts *o, shk_cg_stats *st) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = require_ready(c);
    if (rc) return rc;
    if ((rc = validate_cg(c, o))) return rc;
    if (!c->initialized && (rc = build_mask8(c))) return rc;
    if ((rc = launch_assemble(c, 1, dt, false))) return rc;
    c->assembled = true;
    c->assembled_parabolic = true;
    shk_cg_stats cs;
    memset(&cs, 0, sizeof(cs));
    rc = run_cg(c, o, &cs);
    if (rc) return rc;
    if ((rc = launch_tail(c, false))) return rc;
    if ((rc = check_cuda(c, cudaStreamSynchronize(c->stream), "parabolic step"))) return rc;
    if (st) *st = cs;
    return cs.status;
}

SHK_API int shk_step_b(void *ctx, double dt) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc = require_ready(c);
    if (rc) return rc;
    if (!c->initialized && (rc = build_mask8(c))) return rc;
    rc = launch_step_b(c, dt);
    if (rc) return rc;
    return SHK_OK;
}

SHK_API int shk_update_ieb(void *ctx, const shk_melt_input *mi, double t) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!mi) return fail(c, SHK_BAD_ARG, "null melt input");
    if (mi->kind == SHK_MELT_CONSTANT) return SHK_OK; // no-op (src/melt_input.jl:30)
    if (!c->state_bound) return fail(c, SHK_NOT_BOUND, "state not bound");
    if (mi->kind != SHK_MELT_SEASONAL && mi->kind != SHK_MELT_SEASONAL_BASE)
        return fail(c, SHK_BAD_ARG, "unknown melt input");
    if (mi->kind == SHK_MELT_SEASONAL_BASE && !mi->base) return fail(c, SHK_BAD_ARG, "seasonal+base needs base");
    // update_ieb!(::SeasonalMeltInput) (src/melt_input.jl:86-94)
    double yf = fmod(t / mi->seconds_per_year, 1.0);
    if (yf < 0) yf += 1.0;
    const double i_ma = (mi->t_start <= yf && yf <= mi->t_start + mi->period)
                            ? (mi->offset - mi->amplitude * cos(mi->omega * (yf - mi->t_start)))
                            : mi->i_min;
    const double v = i_ma / mi->seconds_per_year;
    const size_t n = (size_t)c->nx * c->ny;
    if (mi->kind == SHK_MELT_SEASONAL) return launch_fill(c, c->st.ieb, v, n);
    return launch_fill_plus_base(c, c->st.ieb, v, mi->base, n);
}

// step!(sim) (src/run.jl:82-88)
SHK_API int shk_step(void *ctx, int head_scheme, double dt, double total_time, const shk_melt_input *mi,
                     const shk_picard_opts *po, const shk_cg_opts *o, shk_picard_stats *st) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    int rc;
    if (mi && (rc = shk_update_ieb(ctx, mi, total_time))) return rc;
    int status = SHK_OK;
    shk_picard_stats s;
    memset(&s, 0, sizeof(s));
    if (head_scheme == SHK_HEAD_ELLIPTIC) {
        status = shk_picard_solve(ctx, po, o, &s);
        if (status != SHK_OK && status != SHK_NOT_CONVERGED) return status;
    } else if (head_scheme == SHK_HEAD_PARABOLIC) {
        shk_cg_stats cs;
        memset(&cs, 0, sizeof(cs));
        status = shk_parabolic_step(ctx, dt, o, &cs);
        if (status != SHK_OK && status != SHK_NOT_CONVERGED && status != SHK_BREAKDOWN) return status;
        s.converged = -1;
        s.last_iter = -1;
        s.cg_iters_total = cs.niter;
        s.cg_solves = 1;
        s.cg_breakdowns = cs.status == SHK_BREAKDOWN;
        status = SHK_OK;
    } else {
        return fail(c, SHK_BAD_ARG, "unknown head scheme");
    }
    if ((rc = shk_step_b(ctx, dt))) return rc;
    if (st) *st = s;
    return status;
}

// run!(sim) time loop (src/run.jl:37-43), no observers.
SHK_API int shk_run(void *ctx, int head_scheme, double dt, int tsteps, double *total_time, const shk_melt_input *mi,
                    const shk_picard_opts *po, const shk_cg_opts *o, shk_picard_stats *per_step) {
    Ctx *c = as_ctx(ctx);
    REQUIRE_CTX(c);
    if (!total_time || tsteps < 0) return fail(c, SHK_BAD_ARG, "bad run arguments");
    int worst = SHK_OK;
    for (int t = 0; t < tsteps; t++) {
        shk_picard_stats s;
        int rc = shk_step(ctx, head_scheme, dt, *total_time, mi, po, o, &s);
        if (rc != SHK_OK && rc != SHK_NOT_CONVERGED) return rc;
        if (rc > worst) worst = rc;
        *total_time += dt;
        if (per_step) per_step[t] = s;
    }
    int rc = check_cuda(c, cudaStreamSynchronize(c->stream), "run");
    return rc ? rc : worst;
}

SHK_API long shk_kernel_launches(const void *ctx) {
    const Ctx *c = as_ctx(ctx);
    return c ? (long)c->launches : 0;
}

} // extern "C"
