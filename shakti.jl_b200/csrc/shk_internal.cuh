// shk_internal.cuh -- shared definitions of libshakti_b200 (sm_100a).
//
// Data layout in HBM
//   State arrays: caller-owned Float64, column-major (ix fastest), centre nx*ny, x-face (nx+1)*ny,
//   y-face nx*(ny+1) -- the reference's State layout (src/state.jl:13-57).
//   Library-owned:
//     mask8            uint8 copy of State.mask (codes 0..3, 4 = any other value)
//     aP, aE, aN, rhs  the assembled matrix-free system.  The operator is exactly symmetric
//                      (src/linear_solver.jl:468-471), so the reference's aW(i,j) equals aE(i-1,j)
//                      and aS(i,j) equals aN(i,j-1) bit for bit; only aE/aN are stored and the
//                      matvec reads the west/south couplings from the neighbour's entry.
//     x, r, z, p[2], Ap Krylov vectors (p double-buffered: the fused update+matvec reads p_old at
//                      the neighbours while writing p_new)
//     Float32 copies of the coefficients and vectors for the mixed-precision inner solve.
//   Device scalar block (CgDev / ChebDev / PicDev): every Krylov scalar (alpha, beta, gamma, the
//   stopping test) lives on the device; the host only reads a done flag between launch batches.
//
// Reductions: each block reduces its tiles, writes one partial per value, fences and bumps a
// counter; the last block to arrive sums the partials in a fixed order (deterministic for a fixed
// grid), finishes the scalar update and resets the counter.  No block ever waits on another.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/shakti_b200.h"

namespace shk {

constexpr int kTX = 32;             // tile width (cells along x, one warp)
constexpr int kTY = 8;              // tile height
constexpr int kThreads = kTX * kTY; // 256 threads per block
constexpr int kMaxRedValues = 4;
// Resident blocks per SM of the fused field tail (288 threads).  Five (40 registers, a few spills)
// measured fastest at 4096^2: 1310 us per call against 1376 with four, 1485 with six and 1616 with
// three (no spills): the tail needs warps in flight more than registers.
constexpr int kTailBlocksPerSm = 5;
// Resident blocks per SM of the assembly kernel (256 threads).  With every input loaded before the
// cell's first branch (64 registers), four measured fastest at 4096^2: 406 us per call against
// 419 with five (which spills); with the loads inside the branches, five had been fastest at
// 494-507 us (553 with four, 565 with six, 600 with seven, 605 with eight).
constexpr int kAsmBlocksPerSm = 4;
constexpr int kMarchX = 128;        // columns per block of the row-marching stencil kernels
constexpr int kUnrollB = 2;         // 16-byte vectors in flight per thread in streaming kernels
constexpr int kRingRows = 6;        // shared-memory ring depth of the row-marching kernels
constexpr int kMaxChebSteps = 64;   // chebyshev_nsteps_estimate cap
constexpr int kMaxChebDegree = 32;

enum : uint8_t { M_GROUNDED = 0, M_OCEAN = 1, M_LAND = 2, M_OTHER = 3, M_UNKNOWN = 4 };

struct CgDev {
    double gamma, pNorm2, eps_stop, alpha, beta, rnorm, rnorm0, bnorm, rr, pAp;
    double atol, rtol;
    double rz_last;  // last r'z computed (continuation across a residual replacement)
    long long iter, itmax;
    int done, status, first, stop_rule;
    int cont;        // init continues the previous search direction instead of restarting
    unsigned int trips;  // trips of the device-side iteration loop (bounded)
    int fault;           // set by a kernel whose bounded wait for a tile copy ran out
    // paired x updates of the multigrid form: alpha of the previous iteration, and which search
    // direction's x update is still to be applied (0 none, 1 + the p buffer's index)
    double alpha_prev;
    int x_pending;
};

struct ChebDev {
    double lam_min, lam_max;   // bounds in use (persist across solves; placeholder 1,1)
    double est_min, est_max;   // last raw estimate
    int adopted;               // last estimate adopted?
    int nsteps;
    double gamma;              // Lanczos-CG running gamma
    double alphas[kMaxChebSteps], betas[kMaxChebSteps];
    double calpha[kMaxChebDegree + 1], cbeta[kMaxChebDegree + 1]; // per-step coefficients, 1-based
};

struct PicDev {
    double dmax, hmax;
};

struct DevScalars {
    CgDev cg;        // outer (Float64) solve
    CgDev cg_in;     // inner (Float32) solve of the mixed-precision form
    ChebDev cheb;
    PicDev pic;
    double ref_rr, ref_bb; // mixed precision: outer residual norms
};

// One level of the multigrid hierarchy (level 0 aliases the Float32 operator of the mixed form).
struct MgLevel {
    int nx = 0, ny = 0;
    float *aE = nullptr, *aN = nullptr, *dP = nullptr;
    float *wD = nullptr;  // damped inverse diagonal of the smoother: omega/aP (active rows), 1/aP (identity rows)
    uint8_t *act = nullptr;
    float *x[2] = {nullptr, nullptr};
    float *b = nullptr;
    double *aE64 = nullptr, *aN64 = nullptr, *dP64 = nullptr;
};
constexpr int kMgMaxLevels = 24;

struct Params {
    double rho_w, rho_sw, rho_i, g, nu, n, omega, L, br, lr, ct, cw, p_atm, b_min, b_max, e_v;
    double nm1, inv_n;   // n-1, 1/n
    int n_int, nm1_int;  // integer-valued exponents (-1 if not integral)
    int with_sensible;   // ct*cw != 0
    int root3;           // n == 3: x^(1/n) as cbrt(x) (within an ulp of pow(x, 1/3.0))
    double Linv;         // 1/L
    double dx, dy, dx2, dy2;
};

struct Sliding {
    int kind;
    double C, v0;
    const double *Cx, *Cy;
};

struct Ctx {
    int nx, ny;
    double lx, ly, dx, dy;
    cudaStream_t stream = nullptr;
    int device = 0, num_sms = 148;
    shk_params hp{};
    bool params_set = false, state_bound = false, sliding_set = false, initialized = false;
    Params P{};
    Sliding SL{};
    int kfs = 0, gap = 1;
    shk_state st{};
    // library-owned device memory
    void *arena = nullptr;
    size_t arena_bytes = 0;
    uint8_t *mask8 = nullptr;
    double *aP = nullptr, *aE = nullptr, *aN = nullptr, *rhs = nullptr;
    double *x = nullptr, *r = nullptr, *z = nullptr, *p[2] = {nullptr, nullptr}, *Ap = nullptr;
    double *r2 = nullptr;  // second residual buffer: the multigrid form's fused x/r update alternates
    double *h_prev = nullptr;
    double *cr[2] = {nullptr, nullptr}, *cp[2] = {nullptr, nullptr}; // Chebyshev r/p buffers
    double *r64 = nullptr;                                            // mixed: outer residual
    float *aP32 = nullptr, *aE32 = nullptr, *aN32 = nullptr, *dP32 = nullptr, *wD32 = nullptr;
    float *b32 = nullptr, *x32 = nullptr, *r32 = nullptr, *z32 = nullptr, *p32[2] = {nullptr, nullptr}, *Ap32 = nullptr;
    float *cr32[2] = {nullptr, nullptr}, *cp32[2] = {nullptr, nullptr};
    double *partials = nullptr;  // kMaxRedValues * max_blocks
    unsigned int *counter = nullptr;
    DevScalars *dev = nullptr;
    DevScalars *host_dev = nullptr;  // pinned mirror for read-back
    DevScalars *host_dev_d = nullptr;  // its device alias (mapped pinned memory), or null
    MgLevel mg[kMgMaxLevels];
    int mg_levels = 0;
    int mg_nu = 2;           // damped-Jacobi sweeps before and after each coarse correction
    // Jacobi damping and coarse-correction scaling, set per grid size by mg_default_weights.
    float mg_omega = 0.8f;
    float mg_omega_c = 1.6f;
    // The weight of the two sweeps next to each coarse correction relative to mg_omega: 1 for
    // damped Jacobi; tau2/tau1 for the degree-2 Chebyshev pair (mg_omega = tau1).
    float mg_s2 = 1.0f;
    int mg_fused = 1;        // nu = 2 level kernels: 1 tile (default), 2 warp-marching, 0 per-sweep
    int mg_tma = 1;          // tile kernels stage through TMA copies where the level's pitch allows
    bool mg_cluster = false;  // the coarse levels on one thread-block cluster (measured slower; opt-in)
    bool mg_pair_x = true;    // the outer CG's x updated once per two iterations (bit-identical x)
    struct MgTma *mg_maps = nullptr;  // the levels' tensor maps (built on first use)
    struct CgTma *cg_maps = nullptr;  // the plain Jacobi CG's tensor maps (built before its first capture)
    int max_blocks = 0;
    int grid_stencil = 0;    // blocks for tile-stride kernels
    int march_th = 8;        // row-marching tile height
    int march_blocks = 1;    // row-marching grid (one block per kMarchX x march_th tile)
    long long launches = 0;
    // CUDA graphs of the CG iteration loop, keyed by precision, preconditioner, degree, p parity
    struct GraphSlot {
        long long key;
        cudaGraphExec_t exec;
        long long launches;  // kernels per replay (per trip for the device loop)
    };
    std::vector<GraphSlot> graphs;
    cudaStream_t cap_stream = nullptr;  // capture only; nothing executes on it
    int graph_mode = 2;                 // 0 direct launches, 1 one graph per iteration, 2 device-side loop
    bool graphs_disabled = false;       // set when capture fails: direct launches from then on
    bool loop_disabled = false;         // set when the device-loop graph cannot be built
    std::string err;
    bool assembled = false;
    bool assembled_parabolic = false;
    const double *ws_x0 = nullptr;  // one-shot CG warm start for the next Float64 solve (caller-owned)
};

// ---------------------------------------------------------------------------------------------
// Ensemble of independent instances (shk_ensemble.cu).  Each batched kernel runs one grid over
// every instance: the blocks of a kernel family are split into contiguous per-instance ranges
// (blk0, nblk), and a block-to-instance table maps a block to its instance.  An instance's state,
// workspace and device scalars are those of its own context.
// ---------------------------------------------------------------------------------------------
// Families, each with the grid its single-instance kernel uses, so that every reduction of an
// instance sums the same per-block partials in the same order as its own context would.
enum { EF_STENCIL = 0, EF_TAIL = 1, EF_MARCH = 2, EF_STREAM = 3, EF_FLAT = 4, EF_N = 5 };

struct alignas(8) EnsInst {
    int nx, ny, kfs, gap, march_th, size_class;
    int blk0[EF_N], nblk[EF_N];
    Params P;
    Sliding SL;
    shk_state st;
    const uint8_t *mask8;
    double *aP, *aE, *aN, *rhs, *x, *r, *p0, *p1, *Ap, *h_prev;
    double *z, *r2;  // multigrid form: preconditioned residual, the second residual buffer
    double *partials;
    unsigned int *counter;
    CgDev *cg;
    PicDev *pic;
    double *snap;  // optional copy of h after each timestep's first Picard iteration
    const struct EnsMg *mg;  // multigrid form: this instance's hierarchy and block ranges (else null)
    // loop control and statistics, written on the device
    int pic_active, pic_iter, pic_converged, cg_breakdowns;
    long long cg_iters, cg_solves;
    long long total_picard, total_cg, steps_converged, steps;
    double max_dh, max_h;
};

struct alignas(8) EnsCtl {
    int n;                      // instances
    int picard_iters, check_every, stop_rule;
    int precond;                // SHK_PRECOND_JACOBI or SHK_PRECOND_MULTIGRID
    double picard_tol, atol, rtol;
    long long itmax;            // 0: 2 n cells per instance
    unsigned int pic_trips, cg_trips;
    double dt;
};

// ---------------------------------------------------------------------------------------------
// Host helpers
// ---------------------------------------------------------------------------------------------
int fail(Ctx *c, int status, const std::string &msg);
int check_cuda(Ctx *c, cudaError_t e, const char *what);
int check_launch(Ctx *c, const char *what);

// shk_fields.cu
int build_mask8(Ctx *c);
int mg_set_first_wait_polls();
int launch_initial_conditions(Ctx *c);
int launch_assemble(Ctx *c, int parabolic, double dt, bool copy_h_prev);
int launch_export_mfls(Ctx *c, double *aP, double *aE, double *aW, double *aN, double *aS, double *rhs);
int launch_tail(Ctx *c, bool picard_check);
int launch_relax(Ctx *c, double alpha, const double *h_prev);
int launch_step_b(Ctx *c, double dt);
int launch_fill(Ctx *c, double *dst, double v, size_t n);
int launch_fill_plus_base(Ctx *c, double *dst, double v, const double *base, size_t n);

// shk_krylov.cu
int launch_matvec(Ctx *c, const double *x, double *y);
int run_chebyshev_bounds(Ctx *c, int nsteps, const double *rhs);
int cheb_set_bounds(Ctx *c, double lmin, double lmax);
int launch_chebyshev_apply_standalone(Ctx *c, int degree, const double *x, double *y);
int run_cg(Ctx *c, const shk_cg_opts *o, shk_cg_stats *st);
int read_scalars(Ctx *c);
int move_scalars(Ctx *c, void *dst, const void *src, size_t bytes, bool to_host);
int residual_norms(Ctx *c, const double *x, double *rnorm, double *bnorm);
int jacobi_smooth(Ctx *c, double *x, double *tmp, int sweeps, double omega);

// ensemble kernels: shk_fields.cu
void ens_assemble(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks);
void ens_tail(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks);
void ens_gap(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks, const EnsCtl *ctl);
// ensemble kernels: shk_krylov.cu
void ens_cg_reset(cudaStream_t s, EnsInst *E, EnsCtl *ctl, int n);
void ens_cg_init(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks);
void ens_cg_A(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks, int parity);
void ens_cg_B(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks, int parity);
void ens_cg_finish(cudaStream_t s, EnsInst *E, const EnsCtl *ctl, int n, const int *b2i, int nblocks);
void ens_cg_cond(cudaStream_t s, EnsInst *E, EnsCtl *ctl, int n, cudaGraphConditionalHandle h);

// ensemble multigrid form: shk_mg.cu.  Each instance's hierarchy, its bottom level and, per level
// depth, the instance's block range in the batched launch of that depth.
struct EnsMgPlan {
    int nlev, lb;                  // levels of the instance; its bottom level (the one-block kernel)
    int vc_blocks[kMgMaxLevels];   // blocks of the level-d tile kernels (the context's own grid)
    int set_blocks[kMgMaxLevels];  // blocks of the set-up kernel that produces level d
    size_t bottom_smem;
};
int ens_mg_plan(Ctx *c, EnsMgPlan *plan);
struct EnsMg *ens_mg_alloc(int n);  // device array of n descriptors
int ens_mg_upload(struct EnsMg *dM, int i, Ctx *c, const int *blk0_vc, const int *blk0_set);
void ens_mg_free(struct EnsMg *dM);
int ens_mg_kernel_attrs();
const struct EnsMg *ens_mg_at(const struct EnsMg *dM, int i);  // &dM[i]
void ens_mg_setup(cudaStream_t s, EnsInst *E, const struct EnsMg *M, const int *const *b2i_set, const int *nb_set,
                  int lmax);
void ens_mg_vcycle(cudaStream_t s, EnsInst *E, const struct EnsMg *M, const int *const *b2i_vc, const int *nb_vc,
                   int dmax, const int *b2i_bottom, int n, size_t bottom_smem, int mode, int parity);
void ens_cg_init_mg(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks);
void ens_cg_A_mg(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks, int parity);
enum { ENS_VC_INIT = 0, ENS_VC_ITER = 1 };

// shk_mg.cu
int mg_levels_for(int nx, int ny, int *dims, int maxl);
int mg_setup(Ctx *c);
void mg_release(Ctx *c);
int mg_apply(Ctx *c, const double *r, double *z, CgDev *cg, bool init);
bool mg_fuses_cg_update(const Ctx *c);
int cg_tma_prepare(Ctx *c);
int cg_jac_matvec(Ctx *c, int par, const double *r, const double *p_old, double *p_new, double *Ap, CgDev *cg,
                  double eps_curv, bool *launched);
int mg_cg_matvec(Ctx *c, int par, const double *aP, const double *aE, const double *aN, const double *z,
                 const double *p_old, double *p_new, double *Ap, CgDev *cg, double eps_curv, bool *launched);
int mg_apply_fused_update(Ctx *c, const double *r_in, double *r_out, double *x, const double *p, const double *Ap,
                          double *z, CgDev *cg, const double *p_prev = nullptr, int mode = 0, int pbuf = 0);
int mg_catch_up(Ctx *c, double *x, CgDev *cg);

} // namespace shk
