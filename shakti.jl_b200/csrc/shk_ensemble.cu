// shk_ensemble.cu -- batched ensembles of independent instances of uneven grid sizes.
//
// The reference advances one Simulation at a time (run!, src/run.jl:21-63; step!, :82-88, with
// Picard_loop!, src/elliptic_solver.jl:138-176, around the Jacobi-preconditioned cg!,
// src/linear_solver.jl:915-925).  Here N instances, each with its own context (state, workspace,
// device scalars, set up by the single-instance API), advance together:
//
//  * every kernel of the timestep is one launch over all instances: the blocks of a kernel family
//    are split into contiguous per-instance ranges, and a block-to-instance table maps a block to
//    its instance (the kernels are the single-instance kernels' bodies, so each instance computes
//    exactly what its own context would, up to the block count of its reductions);
//  * a timestep is one CUDA graph launch: a device-side WHILE node runs the Picard loop, whose body
//    (assembly, CG set-up, a nested WHILE node running two CG iterations per trip, h += x, the
//    fused tail with the convergence maxima, the per-instance Picard test) repeats while any
//    instance is still iterating; instances that have converged (or reached the iteration limit)
//    skip every kernel.  Both loops carry trip bounds, so they end whatever the flags say;
//  * the row-marching tile height of the CG stencil kernel is chosen per grid size by a measured
//    autotune over the candidates (shk_ensemble_autotune).
#include <cuda_runtime.h>
#include <float.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "shk_device.cuh"

namespace shk {

// Starts every instance's Picard loop of this timestep.
__global__ void k_ens_picard_begin(EnsInst *E, EnsCtl *ctl) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ctl->n; i += gridDim.x * blockDim.x) {
        E[i].pic_active = 1;
        E[i].pic_iter = 0;
        E[i].pic_converged = 0;
        E[i].cg_iters = 0;
        E[i].cg_solves = 0;
        E[i].cg_breakdowns = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->pic_trips = 0;
        ctl->cg_trips = 0;
    }
}

// After one Picard iteration: the convergence test of Picard_loop! (max|h - h_prev| /
// (max|h| + eps) < tol, checked every check_every iterations and at the last), then the loop
// condition: another trip while any instance is iterating, never more than picard_iters + 2 trips.
__global__ void k_ens_picard_cond(EnsInst *E, EnsCtl *ctl, cudaGraphConditionalHandle h) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    int mine = 0;
    for (int i = threadIdx.x; i < ctl->n; i += blockDim.x) {
        EnsInst &I = E[i];
        if (!I.pic_active) continue;
        I.pic_iter += 1;
        const int it = I.pic_iter;
        const bool check = (it % ctl->check_every == 0) || it == ctl->picard_iters;
        if (check) {
            I.max_dh = I.pic->dmax;
            I.max_h = I.pic->hmax;
            if (I.max_dh / (I.max_h + DBL_EPSILON) < ctl->picard_tol) {
                I.pic_converged = 1;
                I.pic_active = 0;
            }
        }
        if (I.pic_active && it >= ctl->picard_iters) I.pic_active = 0;
        if (!I.pic_active) {  // this instance's timestep is done: fold its counts into the totals
            I.total_picard += it;
            I.total_cg += I.cg_iters;
            I.steps += 1;
            I.steps_converged += I.pic_converged;
        }
        if (I.pic_active) mine = 1;
    }
    if (mine) atomicOr(&any, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int t = ++ctl->pic_trips;
        cudaGraphSetConditional(h, (any && t < (unsigned int)ctl->picard_iters + 2) ? 1u : 0u);
    }
}

// After the first Picard iteration of the timestep (before its Picard test), a copy of h for the
// instances that asked for one: the first Picard iterate, the learned warm start's target.
__global__ void __launch_bounds__(kThreads) k_ens_snapshot(EnsInst *E, const int *b2i) {
    __shared__ EnsInst I;
    const Blk B = ens_stage(I, E, b2i, EF_FLAT);
    if (!I.pic_active || !I.snap || I.pic_iter != 0) return;
    const long long n = (long long)I.nx * I.ny;
    for (long long i = (long long)B.id * blockDim.x + threadIdx.x; i < n; i += (long long)B.n * blockDim.x)
        I.snap[i] = I.st.h[i];
}

struct Ens {
    int n = 0, device = 0;
    std::vector<Ctx *> ctx;
    cudaStream_t stream = nullptr;
    cudaStream_t cap[3] = {nullptr, nullptr, nullptr};
    std::vector<EnsInst> hE;
    EnsInst *dE = nullptr;
    EnsCtl *dC = nullptr;
    EnsCtl hC{};
    int *b2i[EF_N] = {};
    int nb[EF_N] = {};
    cudaGraphExec_t step_exec = nullptr;
    int graph_precond = -1;  // the form step_exec was built for
    std::string err;
    // multigrid form (built at its first run): descriptors, per-depth tables
    EnsMg *dM = nullptr;
    int dmax = 0, lmax = 0;
    size_t bottom_smem = 0;
    int *b2i_vc[kMgMaxLevels] = {}, nb_vc[kMgMaxLevels] = {};
    int *b2i_set[kMgMaxLevels + 1] = {}, nb_set[kMgMaxLevels + 1] = {};
};

static int efail(Ens *e, int status, const std::string &msg) {
    if (e) e->err = msg;
    return status;
}
static int echeck(Ens *e, cudaError_t r, const char *what) {
    if (r == cudaSuccess) return SHK_OK;
    return efail(e, SHK_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(r));
}

static int tiles_of(int nx, int ny) { return ((nx + kTX - 1) / kTX) * ((ny + kTY - 1) / kTY); }
static int march_blocks_of(int nx, int ny, int th) { return ((nx + kMarchX - 1) / kMarchX) * ((ny + th - 1) / th); }

// Per-instance block counts of each family, the block -> instance tables, and the descriptors.
static int ens_layout(Ens *e) {
    std::vector<int> tab[EF_N];
    for (int i = 0; i < e->n; i++) {
        EnsInst &I = e->hE[i];
        const Ctx *c = e->ctx[i];
        const long long n = (long long)I.nx * I.ny;
        // the grids of the context's own launches (shk_api.cu, k_tail's launcher, stream_grid and
        // flat_grid in shk_krylov.cu)
        int nb[EF_N];
        nb[EF_STENCIL] = c->grid_stencil;
        nb[EF_TAIL] = std::max(1, std::min(tiles_of(I.nx, I.ny), c->num_sms * kTailBlocksPerSm));
        nb[EF_MARCH] = march_blocks_of(I.nx, I.ny, I.march_th);
        nb[EF_STREAM] = (int)std::max(1LL, std::min((long long)c->num_sms * 8, (n + 1023) / 1024));
        nb[EF_FLAT] = (int)std::max(1LL, std::min((long long)c->grid_stencil, (n + kThreads - 1) / kThreads));
        if (nb[EF_MARCH] > c->max_blocks) return efail(e, SHK_BAD_ARG, "march tile height too small for the workspace");
        for (int f = 0; f < EF_N; f++) {
            I.blk0[f] = (int)tab[f].size();
            I.nblk[f] = nb[f];
            tab[f].insert(tab[f].end(), nb[f], i);
        }
    }
    for (int f = 0; f < EF_N; f++) {
        if (e->b2i[f]) cudaFree(e->b2i[f]);
        e->b2i[f] = nullptr;
        e->nb[f] = (int)tab[f].size();
        int rc = echeck(e, cudaMalloc(&e->b2i[f], tab[f].size() * sizeof(int)), "cudaMalloc(ensemble tables)");
        if (rc) return rc;
        rc = echeck(e, cudaMemcpy(e->b2i[f], tab[f].data(), tab[f].size() * sizeof(int), cudaMemcpyHostToDevice),
                    "upload ensemble tables");
        if (rc) return rc;
    }
    return echeck(e, cudaMemcpy(e->dE, e->hE.data(), e->n * sizeof(EnsInst), cudaMemcpyHostToDevice),
                  "upload ensemble descriptors");
}

// The multigrid form's per-depth block tables and per-instance descriptors (each instance's blocks
// at depth d are the grid its own context launches for level d).
static int ens_mg_layout(Ens *e) {
    std::vector<EnsMgPlan> plan(e->n);
    e->dmax = 0;
    e->lmax = 0;
    e->bottom_smem = 0;
    for (int i = 0; i < e->n; i++) {
        Ctx *c = e->ctx[i];
        if (c->mg_levels >= kMgMaxLevels) return efail(e, SHK_BAD_ARG, "multigrid hierarchy too deep for the ensemble");
        if (ens_mg_plan(c, &plan[i])) return efail(e, SHK_BAD_ARG, c->err);
        e->dmax = std::max(e->dmax, plan[i].lb);
        e->lmax = std::max(e->lmax, plan[i].nlev);
        e->bottom_smem = std::max(e->bottom_smem, plan[i].bottom_smem);
    }
    std::vector<std::vector<int>> vc(kMgMaxLevels), set(kMgMaxLevels + 1);
    std::vector<std::vector<int>> b0vc(e->n, std::vector<int>(kMgMaxLevels, 0)),
        b0set(e->n, std::vector<int>(kMgMaxLevels + 1, 0));
    for (int i = 0; i < e->n; i++) {
        for (int d = 0; d < e->dmax; d++) {
            b0vc[i][d] = (int)vc[d].size();
            vc[d].insert(vc[d].end(), plan[i].vc_blocks[d], i);
        }
        for (int st = 1; st <= e->lmax; st++) {
            b0set[i][st] = (int)set[st].size();
            if (st <= plan[i].nlev) set[st].insert(set[st].end(), plan[i].set_blocks[st], i);
        }
    }
    auto upload = [&](std::vector<int> &t, int **dst, int *nb) -> int {
        if (*dst) cudaFree(*dst);
        *dst = nullptr;
        *nb = (int)t.size();
        if (t.empty()) return SHK_OK;
        int rc = echeck(e, cudaMalloc(dst, t.size() * sizeof(int)), "cudaMalloc(ensemble multigrid tables)");
        if (!rc) rc = echeck(e, cudaMemcpy(*dst, t.data(), t.size() * sizeof(int), cudaMemcpyHostToDevice),
                             "upload ensemble multigrid tables");
        return rc;
    };
    for (int d = 0; d < e->dmax; d++)
        if (int rc = upload(vc[d], &e->b2i_vc[d], &e->nb_vc[d])) return rc;
    for (int st = 1; st <= e->lmax; st++)
        if (int rc = upload(set[st], &e->b2i_set[st], &e->nb_set[st])) return rc;
    if (!e->dM && !(e->dM = ens_mg_alloc(e->n))) return efail(e, SHK_CUDA_ERROR, "cudaMalloc(ensemble multigrid)");
    for (int i = 0; i < e->n; i++) {
        int b0v[kMgMaxLevels], b0s[kMgMaxLevels];
        for (int d = 0; d < kMgMaxLevels; d++) {
            b0v[d] = b0vc[i][d];
            b0s[d] = b0set[i][d];
        }
        if (ens_mg_upload(e->dM, i, e->ctx[i], b0v, b0s)) return efail(e, SHK_CUDA_ERROR, "upload ensemble multigrid");
        e->hE[i].mg = ens_mg_at(e->dM, i);
    }
    if (ens_mg_kernel_attrs()) return efail(e, SHK_CUDA_ERROR, "ensemble multigrid bottom shared memory");
    return echeck(e, cudaMemcpy(e->dE, e->hE.data(), e->n * sizeof(EnsInst), cudaMemcpyHostToDevice),
                  "upload ensemble descriptors");
}

// A conditional handle (default 1, applied at each launch of the whole graph) on the graph being
// captured on stream s.
static cudaError_t capture_handle(cudaStream_t s, cudaGraphConditionalHandle *h) {
    cudaStreamCaptureStatus st;
    cudaGraph_t g;
    cudaError_t r = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, nullptr, nullptr);
    if (r != cudaSuccess) return r;
    if (st != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
    return cudaGraphConditionalHandleCreate(h, g, 1, cudaGraphCondAssignDefault);
}

// Adds a WHILE node on handle h after the work captured so far on stream s; returns its body.
static cudaError_t add_while(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraph_t *body) {
    cudaStreamCaptureStatus st;
    cudaGraph_t g;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaError_t r = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &ndeps);
    if (r != cudaSuccess) return r;
    if (st != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    r = cudaGraphAddNode(&node, g, deps, ndeps, &np);
    if (r != cudaSuccess) return r;
    *body = np.conditional.phGraph_out[0];
    return cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
}

// The timestep graph: Picard WHILE { assembly, CG set-up, CG WHILE { 2 iterations }, h += x,
// tail, Picard test }, then the gap update.
static int ens_build_graph(Ens *e) {
    if (e->step_exec) cudaGraphExecDestroy(e->step_exec);
    e->step_exec = nullptr;
    for (int k = 0; k < 3; k++)
        if (!e->cap[k]) {
            int rc = echeck(e, cudaStreamCreateWithFlags(&e->cap[k], cudaStreamNonBlocking), "capture stream");
            if (rc) return rc;
        }
    EnsInst *E = e->dE;
    EnsCtl *C = e->dC;
    cudaGraph_t graph = nullptr, body1 = nullptr, body2 = nullptr;
    cudaGraphConditionalHandle h1, h2;
    const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
    cudaError_t r = cudaStreamBeginCapture(e->cap[0], mode);
    if (r == cudaSuccess) {
        k_ens_picard_begin<<<(e->n + 255) / 256, 256, 0, e->cap[0]>>>(E, C);
        r = capture_handle(e->cap[0], &h1);  // top level: its default 1 starts every timestep's loop
        if (r == cudaSuccess) r = add_while(e->cap[0], h1, &body1);
        ens_gap(e->cap[0], E, e->b2i[EF_FLAT], e->nb[EF_FLAT], C);
        cudaError_t r2 = cudaStreamEndCapture(e->cap[0], &graph);
        if (r == cudaSuccess) r = r2;
    }
    const bool mg = e->hC.precond == SHK_PRECOND_MULTIGRID;
    if (r == cudaSuccess) r = cudaStreamBeginCaptureToGraph(e->cap[1], body1, nullptr, nullptr, 0, mode);
    if (r == cudaSuccess) {
        ens_assemble(e->cap[1], E, e->b2i[EF_STENCIL], e->nb[EF_STENCIL]);
        if (mg) ens_mg_setup(e->cap[1], E, e->dM, e->b2i_set, e->nb_set, e->lmax);
        ens_cg_reset(e->cap[1], E, C, e->n);
        if (mg) {
            ens_cg_init_mg(e->cap[1], E, e->b2i[EF_STENCIL], e->nb[EF_STENCIL]);
            ens_mg_vcycle(e->cap[1], E, e->dM, e->b2i_vc, e->nb_vc, e->dmax, nullptr, e->n, e->bottom_smem,
                          ENS_VC_INIT, 0);
        } else {
            ens_cg_init(e->cap[1], E, e->b2i[EF_STENCIL], e->nb[EF_STENCIL]);
        }
        // nested loop: a default value is applied once per graph launch, not at each start of the
        // loop, so each solve sets its own condition before the loop (any CG still running)
        r = capture_handle(e->cap[1], &h2);
        if (r == cudaSuccess) {
            ens_cg_cond(e->cap[1], E, C, e->n, h2);
            r = add_while(e->cap[1], h2, &body2);
        }
        ens_cg_finish(e->cap[1], E, C, e->n, e->b2i[EF_FLAT], e->nb[EF_FLAT]);
        k_ens_snapshot<<<e->nb[EF_FLAT], kThreads, 0, e->cap[1]>>>(E, e->b2i[EF_FLAT]);
        ens_tail(e->cap[1], E, e->b2i[EF_TAIL], e->nb[EF_TAIL]);
        k_ens_picard_cond<<<1, 256, 0, e->cap[1]>>>(E, C, h1);
        cudaGraph_t g = nullptr;
        cudaError_t r2 = cudaStreamEndCapture(e->cap[1], &g);
        if (r == cudaSuccess) r = r2;
    }
    if (r == cudaSuccess) r = cudaStreamBeginCaptureToGraph(e->cap[2], body2, nullptr, nullptr, 0, mode);
    if (r == cudaSuccess) {
        for (int par = 0; par < 2; par++) {
            if (mg) {
                ens_cg_A_mg(e->cap[2], E, e->b2i[EF_MARCH], e->nb[EF_MARCH], par);
                ens_mg_vcycle(e->cap[2], E, e->dM, e->b2i_vc, e->nb_vc, e->dmax, nullptr, e->n, e->bottom_smem,
                              ENS_VC_ITER, par);
            } else {
                ens_cg_A(e->cap[2], E, e->b2i[EF_MARCH], e->nb[EF_MARCH], par);
                ens_cg_B(e->cap[2], E, e->b2i[EF_STREAM], e->nb[EF_STREAM], par);
            }
        }
        ens_cg_cond(e->cap[2], E, C, e->n, h2);
        cudaGraph_t g = nullptr;
        cudaError_t r2 = cudaStreamEndCapture(e->cap[2], &g);
        if (r == cudaSuccess) r = r2;
    }
    if (r == cudaSuccess) r = cudaGraphInstantiate(&e->step_exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (r != cudaSuccess) {
        cudaGetLastError();
        e->step_exec = nullptr;
        return echeck(e, r, "ensemble timestep graph");
    }
    e->graph_precond = e->hC.precond;
    return SHK_OK;
}

static int ens_upload_ctl(Ens *e, double dt, const shk_picard_opts *po, const shk_cg_opts *o) {
    if (!po || po->iters < 1) return efail(e, SHK_BAD_ARG, "PicardSolver needs iters >= 1");
    if (po->alpha > 0) return efail(e, SHK_BAD_ARG, "the ensemble runs without head relaxation (alpha)");
    if (!o) return efail(e, SHK_BAD_ARG, "null cg options");
    if ((o->precond != SHK_PRECOND_JACOBI && o->precond != SHK_PRECOND_MULTIGRID) || o->precision != SHK_FP64)
        return efail(e, SHK_BAD_ARG, "the ensemble runs Float64 CG, Jacobi- or multigrid-preconditioned");
    if (o->precond == SHK_PRECOND_MULTIGRID && !e->dM) {
        int rc = ens_mg_layout(e);
        if (rc) return rc;
    }
    EnsCtl &C = e->hC;
    C.n = e->n;
    C.picard_iters = po->iters;
    C.check_every = po->check_every > 0 ? po->check_every : 1;
    C.picard_tol = po->tol;
    C.atol = o->atol;
    C.rtol = o->rtol;
    C.itmax = o->itmax;
    C.stop_rule = o->stop_rule;
    C.precond = o->precond;
    C.dt = dt;
    return echeck(e, cudaMemcpyAsync(e->dC, &C, sizeof(EnsCtl), cudaMemcpyHostToDevice, e->stream),
                  "upload ensemble control");
}

} // namespace shk

using namespace shk;

extern "C" {

SHK_API int shk_ensemble_create(int n, void *const *ctxs, void *stream, void **ens_out) {
    if (!ens_out) return SHK_BAD_ARG;
    *ens_out = nullptr;
    if (n < 1 || !ctxs) return SHK_BAD_ARG;
    Ens *e = new (std::nothrow) Ens();
    if (!e) return SHK_CUDA_ERROR;
    e->n = n;
    e->stream = (cudaStream_t)stream;
    e->hE.resize(n);
    int dev = -1;
    for (int i = 0; i < n; i++) {
        Ctx *c = reinterpret_cast<Ctx *>(ctxs[i]);
        if (!c) {
            delete e;
            return SHK_BAD_ARG;
        }
        if (!c->params_set || !c->state_bound || !c->sliding_set) {
            delete e;
            return SHK_NOT_BOUND;
        }
        if (!c->initialized) {  // the mask codes the kernels read, as the single-instance solves build them
            const int rc0 = build_mask8(c);
            if (rc0 == SHK_OK) cudaStreamSynchronize(c->stream);
            if (rc0) {
                delete e;
                return rc0;
            }
        }
        if (dev >= 0 && c->device != dev) {
            delete e;
            return SHK_BAD_ARG;
        }
        dev = c->device;
        e->ctx.push_back(c);
        EnsInst &I = e->hE[i];
        memset(&I, 0, sizeof(I));
        I.nx = c->nx;
        I.ny = c->ny;
        I.kfs = c->kfs;
        I.gap = c->gap;
        I.march_th = c->march_th;
        I.P = c->P;
        I.SL = c->SL;
        I.st = c->st;
        I.mask8 = c->mask8;
        I.aP = c->aP; I.aE = c->aE; I.aN = c->aN; I.rhs = c->rhs; I.x = c->x; I.r = c->r;
        I.p0 = c->p[0]; I.p1 = c->p[1]; I.Ap = c->Ap; I.h_prev = c->h_prev;
        I.z = c->z; I.r2 = c->r2;
        I.mg = nullptr;
        I.partials = c->partials;
        I.counter = c->counter;
        I.cg = &c->dev->cg;
        I.pic = &c->dev->pic;
    }
    e->device = dev;
    // size classes: instances of equal grid shape share an autotuned tile height
    std::map<std::pair<int, int>, int> cls;
    for (auto &I : e->hE) {
        auto key = std::make_pair(I.nx, I.ny);
        if (!cls.count(key)) {
            const int k = (int)cls.size();
            cls[key] = k;
        }
        I.size_class = cls[key];
    }
    int rc = echeck(e, cudaMalloc(&e->dE, n * sizeof(EnsInst)), "cudaMalloc(ensemble)");
    if (!rc) rc = echeck(e, cudaMalloc(&e->dC, sizeof(EnsCtl)), "cudaMalloc(ensemble control)");
    if (!rc) rc = ens_layout(e);
    if (rc) {
        fprintf(stderr, "shk_ensemble_create: %s\n", e->err.c_str());
        shk_ensemble_destroy(e);
        return rc;
    }
    *ens_out = e;
    return SHK_OK;
}

SHK_API int shk_ensemble_destroy(void *ens) {
    Ens *e = reinterpret_cast<Ens *>(ens);
    if (!e) return SHK_OK;
    if (e->stream) cudaStreamSynchronize(e->stream);
    else cudaDeviceSynchronize();
    if (e->step_exec) cudaGraphExecDestroy(e->step_exec);
    for (int k = 0; k < 3; k++)
        if (e->cap[k]) cudaStreamDestroy(e->cap[k]);
    for (int f = 0; f < EF_N; f++)
        if (e->b2i[f]) cudaFree(e->b2i[f]);
    for (int d = 0; d < kMgMaxLevels; d++)
        if (e->b2i_vc[d]) cudaFree(e->b2i_vc[d]);
    for (int d = 0; d <= kMgMaxLevels; d++)
        if (e->b2i_set[d]) cudaFree(e->b2i_set[d]);
    ens_mg_free(e->dM);
    if (e->dE) cudaFree(e->dE);
    if (e->dC) cudaFree(e->dC);
    delete e;
    return SHK_OK;
}

SHK_API const char *shk_ensemble_last_error(const void *ens) {
    const Ens *e = reinterpret_cast<const Ens *>(ens);
    return e ? e->err.c_str() : "null ensemble";
}

// Measured choice of the row-marching tile height per size class: on each instance's current
// state (assembled here), every candidate runs `iters` batched CG iterations of that class alone,
// timed with CUDA events; the fastest candidate is kept.  th_out (n entries, may be NULL) receives
// each instance's choice.
SHK_API int shk_ensemble_autotune(void *ens, int iters, int *th_out) {
    Ens *e = reinterpret_cast<Ens *>(ens);
    if (!e) return SHK_BAD_ARG;
    if (iters < 1) return efail(e, SHK_BAD_ARG, "autotune needs iters >= 1");
    static const int cand[] = {4, 8, 16, 32, 64};
    int nclass = 0;
    for (auto &I : e->hE) nclass = std::max(nclass, I.size_class + 1);
    shk_picard_opts po{1, 1, 1e-6, 0.0};
    shk_cg_opts o{SHK_PRECOND_JACOBI, 4, 15, SHK_STOP_RELRES, SHK_FP64, 0, 0.0, 0.0, 0.0, 0, 0};
    int rc = ens_upload_ctl(e, 0.0, &po, &o);
    if (rc) return rc;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    const std::vector<EnsInst> saved = e->hE;
    for (int k = 0; k < nclass; k++) {
        float best = 1e30f;
        int best_th = -1;
        for (int th : cand) {
            bool ok = true;
            for (int i = 0; i < e->n; i++) {
                EnsInst &I = e->hE[i];
                I.pic_active = I.size_class == k;
                if (I.size_class == k) {
                    if (march_blocks_of(I.nx, I.ny, th) > e->ctx[i]->max_blocks || th > std::max(I.ny, 4)) ok = false;
                    I.march_th = th;
                }
            }
            if (!ok) continue;
            if ((rc = ens_layout(e))) break;
            // assemble, start a solve that never meets its tolerance (rtol = 0), time the iterations
            ens_assemble(e->stream, e->dE, e->b2i[EF_STENCIL], e->nb[EF_STENCIL]);
            ens_cg_reset(e->stream, e->dE, e->dC, e->n);
            ens_cg_init(e->stream, e->dE, e->b2i[EF_STENCIL], e->nb[EF_STENCIL]);
            for (int w = 0; w < 2; w++) {
                ens_cg_A(e->stream, e->dE, e->b2i[EF_MARCH], e->nb[EF_MARCH], w & 1);
                ens_cg_B(e->stream, e->dE, e->b2i[EF_STREAM], e->nb[EF_STREAM], w & 1);
            }
            cudaEventRecord(t0, e->stream);
            for (int it = 0; it < 2 * iters; it++) {
                ens_cg_A(e->stream, e->dE, e->b2i[EF_MARCH], e->nb[EF_MARCH], it & 1);
                ens_cg_B(e->stream, e->dE, e->b2i[EF_STREAM], e->nb[EF_STREAM], it & 1);
            }
            cudaEventRecord(t1, e->stream);
            if ((rc = echeck(e, cudaEventSynchronize(t1), "autotune"))) break;
            float ms = 0;
            cudaEventElapsedTime(&ms, t0, t1);
            if (ms < best) {
                best = ms;
                best_th = th;
            }
        }
        if (rc) break;
        for (int i = 0; i < e->n; i++)
            if (saved[i].size_class == k && best_th > 0) e->hE[i].march_th = best_th;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    for (int i = 0; i < e->n; i++) {
        const int th = e->hE[i].march_th;
        e->hE[i] = saved[i];
        e->hE[i].march_th = th;
        if (th_out) th_out[i] = th;
    }
    if (!rc) rc = ens_layout(e);
    if (!rc && e->step_exec) {
        cudaGraphExecDestroy(e->step_exec);
        e->step_exec = nullptr;
    }
    return rc;
}

// tsteps timesteps of every instance (step! with a constant melt input: update_ieb! is a no-op),
// one graph launch each.  per_instance (n entries, may be NULL) receives each instance's totals.
SHK_API int shk_ensemble_run(void *ens, double dt, int tsteps, const shk_picard_opts *po, const shk_cg_opts *o,
                             shk_ensemble_stats *per_instance) {
    Ens *e = reinterpret_cast<Ens *>(ens);
    if (!e) return SHK_BAD_ARG;
    if (tsteps < 0) return efail(e, SHK_BAD_ARG, "tsteps must be >= 0");
    int rc = ens_upload_ctl(e, dt, po, o);
    if (rc) return rc;
    if (e->step_exec && e->graph_precond != e->hC.precond) {
        cudaGraphExecDestroy(e->step_exec);
        e->step_exec = nullptr;
    }
    if (!e->step_exec && (rc = ens_build_graph(e))) return rc;
    for (int k = 0; k < tsteps; k++)
        if ((rc = echeck(e, cudaGraphLaunch(e->step_exec, e->stream), "ensemble timestep"))) return rc;
    if ((rc = echeck(e, cudaStreamSynchronize(e->stream), "ensemble run"))) return rc;
    std::vector<EnsInst> out(e->n);
    if ((rc = echeck(e, cudaMemcpy(out.data(), e->dE, e->n * sizeof(EnsInst), cudaMemcpyDeviceToHost),
                     "read ensemble statistics")))
        return rc;
    int status = SHK_OK;
    for (int i = 0; i < e->n; i++) {
        const EnsInst &I = out[i];
        if (I.steps_converged < I.steps) status = SHK_NOT_CONVERGED;
        if (per_instance) {
            shk_ensemble_stats &s = per_instance[i];
            s.steps = I.steps;
            s.steps_converged = I.steps_converged;
            s.picard_iters = I.total_picard;
            s.cg_iters = I.total_cg;
            s.last_picard_iters = I.pic_iter;
            s.last_converged = I.pic_converged;
            s.march_th = e->hE[i].march_th;
            s.max_dh = I.max_dh;
            s.max_h = I.max_h;
        }
    }
    return status;
}

// Per-instance buffers (nx*ny doubles, device; NULL entries: none) that receive h after each
// timestep's first Picard iteration.
SHK_API int shk_ensemble_set_snapshots(void *ens, double *const *bufs) {
    Ens *e = reinterpret_cast<Ens *>(ens);
    if (!e) return SHK_BAD_ARG;
    for (int i = 0; i < e->n; i++) {
        e->hE[i].snap = bufs ? bufs[i] : nullptr;
        int rc = echeck(e, cudaMemcpy(&e->dE[i].snap, &e->hE[i].snap, sizeof(double *), cudaMemcpyHostToDevice),
                        "set snapshots");
        if (rc) return rc;
    }
    return SHK_OK;
}

SHK_API int shk_ensemble_launch_counts(const void *ens, int *stencil, int *march, int *stream, int *flat) {
    const Ens *e = reinterpret_cast<const Ens *>(ens);
    if (!e) return SHK_BAD_ARG;
    if (stencil) *stencil = e->nb[EF_STENCIL] + e->nb[EF_TAIL];
    if (march) *march = e->nb[EF_MARCH];
    if (stream) *stream = e->nb[EF_STREAM];
    if (flat) *flat = e->nb[EF_FLAT];
    return SHK_OK;
}

} // extern "C"
