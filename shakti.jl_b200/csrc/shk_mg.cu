// shk_mg.cu -- aggregation multigrid preconditioner (Float32 V-cycle inside Float64 CG).
//
// The GPU counterpart of the reference's AMGPreconditioner (src/preconditioner.jl:298-327, CPU
// only there): on the structured grid, 2x2 cell aggregation with piecewise-constant transfer P
// keeps every Galerkin coarse operator P'AP a 5-point stencil in Laplacian form,
//   (A x)_i = dP_i x_i + sum_j a_ij (x_i - x_j),
// with coarse conductances = sums of the fine face conductances crossing an aggregate boundary and
// coarse excess = sum of the fine excesses (internal faces cancel).  Operators are built in Float64
// and rounded once to Float32, so each stored value carries only a relative error; the V-cycle runs
// in Float32, the outer CG (residual, updates, stopping test) in Float64.
//
// Identity rows (OCEAN/LAND/OTHER_BASIN cells: aP = 1, no couplings) are not aggregated (their row
// of P is zero); the smoother solves them exactly.  The V-cycle is symmetric (the same sweep weights
// before and after the coarse correction; exact solve on the 1x1 coarsest level), so it is a valid
// CG preconditioner.  Per level: nu Jacobi sweeps before and after, with the stored damped inverse
// diagonal wD = omega/aP, the two sweeps next to the coarse correction scaled by Lv::s2 (1 for
// damped Jacobi, tau2/tau1 for the degree-2 Chebyshev pair), coarse correction scaled by omega_c;
// the levels that fit in one block's shared memory run as one kernel.
#include <cuda.h>
#include <cuda_runtime.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "shk_device.cuh"

namespace shk {

#define GSTRIDE(i, n) for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

// ---------------------------------------------------------------------------------------------
// Hierarchy construction
// ---------------------------------------------------------------------------------------------

// Level-0 activity flags (rows assembled by the GROUNDED branch: mask codes 0 and "other") and the
// smoother's damped inverse diagonal wD = omega/aP on active rows, 1/aP on identity rows, formed in
// Float64 and rounded once.
__global__ void k_mg_act0(int n, const uint8_t *m8, const double *aP, double omega, uint8_t *act, float *wD) {
    GSTRIDE(i, n) {
        const bool a = m8[i] == M_GROUNDED || m8[i] == M_UNKNOWN;
        act[i] = a ? 1 : 0;
        wD[i] = (float)((a ? omega : 1.0) / aP[i]);
    }
}

// Coarse operator of level l+1 from level l (Galerkin sums over 2x2 aggregates, Float64): the
// coarse excess dP is the sum of the active fine cells' excesses (dj outer, di inner); the coarse
// east (north) coupling the sum of the fine aE (aN) across the aggregate's east (north) boundary
// where both fine cells are active; inactive aggregates get dP = 1 and no couplings.
// Level 0 of a hierarchy of two or more levels in one pass: per fine cell the Float32 Laplacian-form
// operator (aE, aN, dP = aP - the four couplings) and the smoother's activity flag and damped
// inverse diagonal (the arrays k_to_float_lapl and k_mg_act0 write), and per 2x2 aggregate the
// level-1 Float64 operator (the sums above, dP computed from aP on the fly).  One thread per
// aggregate on a 2D grid, so a warp reads 64 consecutive fine cells of each of its two rows.
__device__ __forceinline__ void level0_aggregate(int I, int J, int nx, int ny, int nxc, const uint8_t *m8,
                                                 const double *aP, const double *aE, const double *aN,
                                                 double omega, float *fE, float *fN, float *fD, float *fW,
                                                 uint8_t *act0, double *aEc, double *aNc, double *dPc,
                                                 uint8_t *actc) {
    auto active = [&](size_t c) { return m8[c] == M_GROUNDED || m8[c] == M_UNKNOWN; };
    double dp[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    bool a[2][2] = {{false, false}, {false, false}};
    for (int dj = 0; dj < 2; dj++)
        for (int di = 0; di < 2; di++) {
            const int i = 2 * I + di, j = 2 * J + dj;
            if (i >= nx || j >= ny) continue;
            const size_t c = (size_t)i + (size_t)j * nx;
            const double e = aE[c], w = i > 0 ? aE[c - 1] : 0.0, no = aN[c], so = j > 0 ? aN[c - nx] : 0.0;
            const double p = aP[c], d = p - (e + w + no + so);
            const bool ac = active(c);
            fE[c] = (float)e;
            fN[c] = (float)no;
            fD[c] = (float)d;
            fW[c] = (float)((ac ? omega : 1.0) / p);
            act0[c] = ac ? 1 : 0;
            dp[dj][di] = d;
            a[dj][di] = ac;
        }
    double d = 0.0, e = 0.0, no = 0.0;
    int act = 0;
    for (int dj = 0; dj < 2; dj++)
        for (int di = 0; di < 2; di++) {
            if (!a[dj][di]) continue;  // out-of-range cells are inactive
            act = 1;
            d += dp[dj][di];
        }
    const int ie = 2 * I + 1;  // fine column on the west side of the east aggregate boundary
    if (ie + 1 < nx)
        for (int dj = 0; dj < 2; dj++) {
            const int j = 2 * J + dj;
            if (j >= ny) continue;
            const size_t c = (size_t)ie + (size_t)j * nx;
            if (a[dj][1] && active(c + 1)) e += aE[c];
        }
    const int jn = 2 * J + 1;
    if (jn + 1 < ny)
        for (int di = 0; di < 2; di++) {
            const int i = 2 * I + di;
            if (i >= nx) continue;
            const size_t c = (size_t)i + (size_t)jn * nx;
            if (a[1][di] && active(c + nx)) no += aN[c];
        }
    const size_t k = (size_t)I + (size_t)J * nxc;
    aEc[k] = act ? e : 0.0;
    aNc[k] = act ? no : 0.0;
    dPc[k] = act ? d : 1.0;
    actc[k] = (uint8_t)act;
}

__global__ void __launch_bounds__(256) k_mg_level0(int nx, int ny, int nxc, int nyc, const uint8_t *m8,
                                                   const double *aP, const double *aE, const double *aN,
                                                   double omega, float *fE, float *fN, float *fD, float *fW,
                                                   uint8_t *act0, double *aEc, double *aNc, double *dPc,
                                                   uint8_t *actc) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= nxc || J >= nyc) return;
    level0_aggregate(I, J, nx, ny, nxc, m8, aP, aE, aN, omega, fE, fN, fD, fW, act0, aEc, aNc, dPc, actc);
}

// The sums above and k_mg_finish_level's Float32 copies of coarse level l+1 (fine level l >= 1) in
// one pass.  The damped diagonal needs the coarse west and south couplings of the neighbouring
// aggregates; each thread recomputes them from the fine boundary they sum (same terms, same
// order), so they equal the values those aggregates store.
__device__ __forceinline__ void coarsen_finish_cell(int k, int nxf, int nyf, int nxc, const double *aEf,
                                                    const double *aNf, const double *dPf, const uint8_t *actf,
                                                    double omega, double *aEc, double *aNc, double *dPc,
                                                    uint8_t *actc, float *fE, float *fN, float *fD, float *fW) {
    {
        const int I = k % nxc, J = k / nxc;
        auto af = [&](int i, int j) { return i >= 0 && j >= 0 && i < nxf && j < nyf && actf[(size_t)i + (size_t)j * nxf]; };
        double d = 0.0, e = 0.0, no = 0.0;
        int act = 0;
        for (int dj = 0; dj < 2; dj++)
            for (int di = 0; di < 2; di++) {
                const int i = 2 * I + di, j = 2 * J + dj;
                if (!af(i, j)) continue;
                act = 1;
                d += dPf[(size_t)i + (size_t)j * nxf];
            }
        // east / north boundary sums of aggregate (A, B)
        auto east = [&](int A, int B) {
            double v = 0.0;
            const int ie = 2 * A + 1;
            if (ie + 1 < nxf)
                for (int dj = 0; dj < 2; dj++) {
                    const int j = 2 * B + dj;
                    if (j >= nyf) continue;
                    if (af(ie, j) && af(ie + 1, j)) v += aEf[(size_t)ie + (size_t)j * nxf];
                }
            return v;
        };
        auto north = [&](int A, int B) {
            double v = 0.0;
            const int jn = 2 * B + 1;
            if (jn + 1 < nyf)
                for (int di = 0; di < 2; di++) {
                    const int i = 2 * A + di;
                    if (i >= nxf) continue;
                    if (af(i, jn) && af(i, jn + 1)) v += aNf[(size_t)i + (size_t)jn * nxf];
                }
            return v;
        };
        auto any_active = [&](int A, int B) {
            return af(2 * A, 2 * B) || af(2 * A + 1, 2 * B) || af(2 * A, 2 * B + 1) || af(2 * A + 1, 2 * B + 1);
        };
        e = east(I, J);
        no = north(I, J);
        const double ae = act ? e : 0.0, an = act ? no : 0.0, dd = act ? d : 1.0;
        aEc[k] = ae;
        aNc[k] = an;
        dPc[k] = dd;
        actc[k] = (uint8_t)act;
        const double w = (I > 0 && any_active(I - 1, J)) ? east(I - 1, J) : 0.0;
        const double so = (J > 0 && any_active(I, J - 1)) ? north(I, J - 1) : 0.0;
        fE[k] = (float)ae;
        fN[k] = (float)an;
        fD[k] = (float)dd;
        fW[k] = act ? (float)(omega / (dd + (ae + w + an + so))) : 1.0f;
    }
}

__global__ void k_mg_coarsen_finish(int nxf, int nyf, int nxc, int nyc, const double *aEf, const double *aNf,
                                    const double *dPf, const uint8_t *actf, double omega, double *aEc,
                                    double *aNc, double *dPc, uint8_t *actc, float *fE, float *fN, float *fD,
                                    float *fW) {
    GSTRIDE(k, nxc * nyc)
    coarsen_finish_cell(k, nxf, nyf, nxc, aEf, aNf, dPf, actf, omega, aEc, aNc, dPc, actc, fE, fN, fD, fW);
}

// Float32 copies and the smoother's damped inverse diagonal wD = omega/aP with the Jacobi diagonal
// aP = dP + the four couplings (identity rows: aP = 1, wD = 1).
__device__ __forceinline__ void finish_level_cell(int k, int nx, const double *aE, const double *aN,
                                                  const double *dP, const uint8_t *act, double omega, float *fE,
                                                  float *fN, float *fD, float *fW) {
    const int ix = k % nx, iy = k / nx;
    const double w = ix > 0 ? aE[k - 1] : 0.0, s = iy > 0 ? aN[k - nx] : 0.0;
    fE[k] = (float)aE[k];
    fN[k] = (float)aN[k];
    fD[k] = (float)dP[k];
    fW[k] = act[k] ? (float)(omega / (dP[k] + (aE[k] + w + aN[k] + s))) : 1.0f;
}

__global__ void k_mg_finish_level(int nx, int ny, const double *aE, const double *aN, const double *dP,
                                  const uint8_t *act, double omega, float *fE, float *fN, float *fD, float *fW) {
    GSTRIDE(k, nx * ny) finish_level_cell(k, nx, aE, aN, dP, act, omega, fE, fN, fD, fW);
}

// ---------------------------------------------------------------------------------------------
// V-cycle kernels (Float32)
// ---------------------------------------------------------------------------------------------
struct Lv {
    int nx, ny;
    const float *aE, *aN, *dP, *wD;
    const uint8_t *act;
    const int *done;  // the outer CG's stop flag: V-cycles issued after the stop do no work
    // The weight of the two sweeps next to the coarse correction (the last one before it, the
    // first one after it) relative to wD: 1 for plain damped Jacobi; tau2/tau1 for the degree-2
    // Chebyshev pair (wD = tau1/aP).  The pre- and post-smoothers apply the same two factors, so the
    // cycle stays symmetric.
    float s2 = 1.0f;
};

// The outer CG's stop flag, read once per block (all threads must call it first).
__device__ __forceinline__ bool cg_finished(const int *done) { return block_cg_done(done); }

// (A x)_c in Laplacian form, with x given by a functor (so fused kernels can form x on the fly)
template <typename F>
__device__ __forceinline__ float lapl_apply(const Lv &L, int ix, int iy, size_t c, float xc, F x) {
    float y = L.dP[c] * xc;
    if (ix < L.nx - 1) y += L.aE[c] * (xc - x(c + 1));
    if (ix > 0) y += L.aE[c - 1] * (xc - x(c - 1));
    if (iy < L.ny - 1) y += L.aN[c] * (xc - x(c + L.nx));
    if (iy > 0) y += L.aN[c - L.nx] * (xc - x(c - L.nx));
    return y;
}

// The level kernels use a 2D grid of 32 x 8 blocks, one thread per cell (no div/mod per cell).
#define CELL2D()                                                                                      \
    if (cg_finished(L.done)) return;                                                                  \
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y; \
    const bool inside = ix < L.nx && iy < L.ny;                                                       \
    const size_t k = (size_t)ix + (size_t)iy * L.nx;

// First pre-smoothing sweep from x = 0: x = wD b (wD = omega/aP).  Level 0 reads b in Float64 (the
// outer residual).
template <typename TB>
__global__ void k_mg_pre0(Lv L, const TB *b, float *x) {
    CELL2D();
    if (inside) x[k] = L.wD[k] * (float)b[k];
}

// One damped-Jacobi sweep: xo = xi + (s wD) (b - A xi).
template <typename TB>
__global__ void k_mg_sweep(Lv L, const TB *b, const float *xi, float *xo, float s) {
    CELL2D();
    if (!inside) return;
    const float xc = xi[k];
    const float ax = lapl_apply(L, ix, iy, k, xc, [&](size_t q) { return xi[q]; });
    xo[k] = xc + __fmul_rn(L.wD[k], s) * ((float)b[k] - ax);
}

// Restriction of the residual: bc(C) = sum over the active fine cells of aggregate C of (b - A x).
// One thread per coarse cell (2D grid over the coarse level).
template <typename TB>
__global__ void k_mg_restrict(Lv L, const TB *b, const float *x, int nxc, int nyc, float *bc) {
    if (cg_finished(L.done)) return;
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= nxc || J >= nyc) return;
    float s = 0.0f;
#pragma unroll
    for (int dj = 0; dj < 2; dj++)
#pragma unroll
        for (int di = 0; di < 2; di++) {
            const int i = 2 * I + di, j = 2 * J + dj;
            if (i >= L.nx || j >= L.ny) continue;
            const size_t c = (size_t)i + (size_t)j * L.nx;
            if (!L.act[c]) continue;
            const float ax = lapl_apply(L, i, j, c, x[c], [&](size_t q) { return x[q]; });
            s += (float)b[c] - ax;
        }
    bc[(size_t)I + (size_t)J * nxc] = s;
}

// x + omega_c (P xc) at fine cell (i, j) = q
__device__ __forceinline__ float prolonged(const Lv &L, const float *xi, const float *xc, int nxc, float wc, int i,
                                           int j, size_t q) {
    float v = xi[q];
    if (L.act[q]) v += wc * xc[(size_t)(i >> 1) + (size_t)(j >> 1) * nxc];
    return v;
}

// Prolongation fused with the first post-smoothing sweep:
//   xt = xi + omega_c P xc,  xo = xt + (s wD) (b - A xt).
template <typename TB>
__global__ void k_mg_prolong_sweep(Lv L, const TB *b, const float *xi, const float *xc, int nxc, float wc,
                                   float *xo, float s) {
    CELL2D();
    if (!inside) return;
    const float xk = prolonged(L, xi, xc, nxc, wc, ix, iy, k);
    float y = L.dP[k] * xk;
    if (ix < L.nx - 1) y += L.aE[k] * (xk - prolonged(L, xi, xc, nxc, wc, ix + 1, iy, k + 1));
    if (ix > 0) y += L.aE[k - 1] * (xk - prolonged(L, xi, xc, nxc, wc, ix - 1, iy, k - 1));
    if (iy < L.ny - 1) y += L.aN[k] * (xk - prolonged(L, xi, xc, nxc, wc, ix, iy + 1, k + L.nx));
    if (iy > 0) y += L.aN[k - L.nx] * (xk - prolonged(L, xi, xc, nxc, wc, ix, iy - 1, k - L.nx));
    xo[k] = xk + __fmul_rn(L.wD[k], s) * ((float)b[k] - y);
}

// Last post-smoothing sweep on level 0, writing z in Float64 and finishing the outer CG's r'z:
// z = xt + wD (r - A xt) (xt = xi, plus the prolonged coarse correction when PROLONG);
// partials r'z, r'r -> init or iteration finish.  1D grid (the grid reduction is 1D).
template <bool PROLONG>
__global__ void __launch_bounds__(kThreads) k_mg_last(Lv L, const double *r, const float *xi, const float *xc, int nxc,
                                                      float wc, double *z, CgDev *cg, int init, double *partials,
                                                      unsigned int *counter) {
    if (block_cg_done(&cg->done)) return;
    double red[2] = {0.0, 0.0};
    GSTRIDE(kk, L.nx * L.ny) {
        const size_t k = (size_t)kk;
        const int ix = kk % L.nx, iy = kk / L.nx;
        auto xt = [&](int i, int j, size_t q) -> float {
            return PROLONG ? prolonged(L, xi, xc, nxc, wc, i, j, q) : xi[q];
        };
        const float xk = xt(ix, iy, k);
        float y = L.dP[k] * xk;
        if (ix < L.nx - 1) y += L.aE[k] * (xk - xt(ix + 1, iy, k + 1));
        if (ix > 0) y += L.aE[k - 1] * (xk - xt(ix - 1, iy, k - 1));
        if (iy < L.ny - 1) y += L.aN[k] * (xk - xt(ix, iy + 1, k + L.nx));
        if (iy > 0) y += L.aN[k - L.nx] * (xk - xt(ix, iy - 1, k - L.nx));
        const double rk = r[k];
        const double zk = (double)(xk + L.wD[k] * ((float)rk - y));
        z[k] = zk;
        red[0] += rk * zk;
        red[1] += rk * rk;
    }
    double out[2];
    if (grid_reduce<2, false>(red, partials, counter, out) && threadIdx.x == 0) {
        if (init) cg_init_finish(cg, out[0], cg->rr, cg->bnorm);
        else cg_iter_finish(cg, out[0], out[1]);
    }
}

// ---------------------------------------------------------------------------------------------
// Fused level kernels (nu = 2): the descending half of a level (first sweep from zero, second
// sweep, residual restriction) and the ascending half (prolongation, two sweeps) each run as one
// kernel over 32 x 16 tiles with a two-cell halo staged in shared memory, so the level's
// operator, right-hand side and iterates cross HBM once per half instead of once per sweep.  The
// arithmetic is the per-sweep kernels' expression for expression, so the results are identical.
// ---------------------------------------------------------------------------------------------
constexpr int kFW = 32, kFH = 16, kFR = 2;                  // tile and halo
constexpr int kFSW = kFW + 2 * kFR, kFSH = kFH + 2 * kFR;   // staged region (36 x 20)
constexpr int kFCells = kFSW * kFSH;

struct FusedSm {
    float b[kFSH][kFSW], wD[kFSH][kFSW], dP[kFSH][kFSW], aE[kFSH][kFSW], aN[kFSH][kFSW];
    float x0[kFSH][kFSW], x1[kFSH][kFSW];
    uint8_t act[kFSH][kFSW];
};

// (A X)_c at staged position (hx, hy), same operand order as lapl_apply.  No bounds tests: the
// couplings across the level's edge are zero in every assembled and coarsened operator (the
// east/north entries of the last column/row, and the staged zeros outside the level), so those
// terms add 0 * (finite) = 0.
// The tile kernels spell out every rounding (one multiply, then one fused multiply-add per
// coupling), so that their two staging forms -- these LDG ones and the TMA ones below, which work
// on packed pairs -- compute the same V-cycle bit for bit.
__device__ __forceinline__ float ax_sm(const FusedSm &S, const float (&X)[kFSH][kFSW], int hx, int hy) {
    const float xc = X[hy][hx];
    float y = __fmul_rn(S.dP[hy][hx], xc);
    y = __fmaf_rn(S.aE[hy][hx], __fsub_rn(xc, X[hy][hx + 1]), y);
    y = __fmaf_rn(S.aE[hy][hx - 1], __fsub_rn(xc, X[hy][hx - 1]), y);
    y = __fmaf_rn(S.aN[hy][hx], __fsub_rn(xc, X[hy + 1][hx]), y);
    y = __fmaf_rn(S.aN[hy - 1][hx], __fsub_rn(xc, X[hy - 1][hx]), y);
    return y;
}

// Stages the level's operator and rhs over the tile and its halo; cells outside the level are
// zeros (act = 0, wD = 0), so every sweep leaves them at 0.  (Flat loops over the staged region
// keep every lane busy; the divisions are by a compile-time constant.)
// X0 (the first iterate over the whole region) is formed in the same pass: DOWN, the first sweep
// from zero, wD b; UP, the fine iterate plus the prolonged coarse correction.
// FB (level 0 of an iteration): the outer CG's x/r update (k_cg_B's arithmetic, unfused) is done
// here: the staged rhs is r_new = r + (-alpha) Ap, and the tile's own cells write r_new to the
// other r buffer (never the one neighbouring blocks read) and x += alpha p.
// The outer CG's x/r update folded into the level-0 descending kernel.  mode 0: x += alpha p;
// mode 1 (first iteration of a pair): x untouched, the update recorded as pending; mode 2 (second):
// x = (x + alpha_prev p_prev) + alpha p -- the same two roundings as two single updates, so the
// pair gives x bit for bit, and one read and write of x per two iterations.
struct FusedB {
    const double *Ap, *p;
    double *x, *r_out;
    double alpha;
    const double *p_prev;
    int mode, pbuf;  // pbuf: index of the context's p buffer that p is (mode 1)
    double alpha_prev;
};

template <typename TB, bool UP, bool FB = false>
__device__ __forceinline__ void stage_level(FusedSm &S, const Lv &L, const TB *b, int x0, int y0, double *r64,
                                            const float *xi, const float *xc, int nxc, float wc,
                                            const FusedB *fb = nullptr) {
    for (int k = threadIdx.x; k < kFCells; k += blockDim.x) {
        const int hx = k % kFSW, hy = k / kFSW, gx = x0 - kFR + hx, gy = y0 - kFR + hy;
        if (gx >= 0 && gx < L.nx && gy >= 0 && gy < L.ny) {
            const size_t q = (size_t)gx + (size_t)gy * L.nx;
            TB bq = b[q];
            if constexpr (FB) {
                bq = __dadd_rn(bq, __dmul_rn(-fb->alpha, fb->Ap[q]));
                if (hx >= kFR && hx < kFR + kFW && hy >= kFR && hy < kFR + kFH) {
                    fb->r_out[q] = bq;
                    fb->x[q] = __dadd_rn(fb->x[q], __dmul_rn(fb->alpha, fb->p[q]));
                }
            }
            if (r64) r64[k] = (double)bq;
            const float bf = (float)bq, wd = L.wD[q];
            const uint8_t a = L.act[q];
            S.b[hy][hx] = bf;
            S.wD[hy][hx] = wd;
            S.dP[hy][hx] = L.dP[q];
            S.aE[hy][hx] = L.aE[q];
            S.aN[hy][hx] = L.aN[q];
            S.act[hy][hx] = a;
            if (UP) {
                float v = xi[q];
                if (a) v = __fmaf_rn(wc, xc[(size_t)(gx >> 1) + (size_t)(gy >> 1) * nxc], v);
                S.x0[hy][hx] = v;
            } else {
                S.x0[hy][hx] = __fmul_rn(wd, bf);
            }
        } else {
            if (r64) r64[k] = 0.0;
            S.b[hy][hx] = 0.0f;
            S.wD[hy][hx] = 0.0f;
            S.dP[hy][hx] = 0.0f;
            S.aE[hy][hx] = 0.0f;
            S.aN[hy][hx] = 0.0f;
            S.act[hy][hx] = 0;
            S.x0[hy][hx] = 0.0f;
        }
    }
}

// One damped-Jacobi sweep XO = XI + (s wD) (b - A XI) over the staged positions within distance 1
// of the tile.
__device__ __forceinline__ void sweep_sm(FusedSm &S, const float (&XI)[kFSH][kFSW], float (&XO)[kFSH][kFSW],
                                         float s) {
    constexpr int wdt = kFW + 2, hgt = kFH + 2;
    for (int k = threadIdx.x; k < wdt * hgt; k += blockDim.x) {
        const int hx = kFR - 1 + k % wdt, hy = kFR - 1 + k / wdt;
        XO[hy][hx] =
            __fmaf_rn(__fmul_rn(S.wD[hy][hx], s), __fsub_rn(S.b[hy][hx], ax_sm(S, XI, hx, hy)), XI[hy][hx]);
    }
}

// Descending half of level L: x1 = two sweeps from zero (written to xo), and the coarse rhs
// bc = restriction of b - A x1.  1D grid striding over 32 x 16 tiles.
template <typename TB, bool FB = false>
__device__ __forceinline__ void mg_down_body(Blk B, const Lv &L, const TB *b, float *xo, int nxc, int nyc, float *bc,
                                             FusedB fbv, const CgDev *cg) {
    if constexpr (FB) {
        const CgView cv = block_cg_view(cg);
        if (cv.done) return;
        fbv.alpha = cv.alpha;
    } else {
        if (cg_finished(L.done)) return;
    }
    __shared__ FusedSm S;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // output rows: 32 x 8 threads
    const int tiles_x = (L.nx + kFW - 1) / kFW, ntiles = tiles_x * ((L.ny + kFH - 1) / kFH);
    for (int t = B.id; t < ntiles; t += B.n) {
        const int x0 = (t % tiles_x) * kFW, y0 = (t / tiles_x) * kFH;
        stage_level<TB, false, FB>(S, L, b, x0, y0, nullptr, nullptr, nullptr, 0, 0.0f, &fbv);
        __syncthreads();
        sweep_sm(S, S.x0, S.x1, L.s2);
        __syncthreads();
        // x1 out, and each tile cell's residual (0 on inactive cells) into the x0 array, which
        // the restriction then sums per aggregate
        for (int r = ty; r < kFH; r += 8) {
            const int gx = x0 + tx, gy = y0 + r, hx = tx + kFR, hy = r + kFR;
            if (gx < L.nx && gy < L.ny) xo[(size_t)gx + (size_t)gy * L.nx] = S.x1[hy][hx];
            S.x0[hy][hx] = S.act[hy][hx] ? __fsub_rn(S.b[hy][hx], ax_sm(S, S.x1, hx, hy)) : 0.0f;
        }
        __syncthreads();
        // restriction: one thread per aggregate of the tile (16 x 8 aggregates, 128 threads), in the
        // per-sweep kernel's order (dj outer, di inner)
        if (threadIdx.x < (kFW / 2) * (kFH / 2)) {
            const int ai = threadIdx.x % (kFW / 2), aj = threadIdx.x / (kFW / 2);
            const int I = x0 / 2 + ai, J = y0 / 2 + aj;
            if (I < nxc && J < nyc) {
                const int hx = 2 * ai + kFR, hy = 2 * aj + kFR;
                float sres = 0.0f;
                sres += S.x0[hy][hx];
                sres += S.x0[hy][hx + 1];
                sres += S.x0[hy + 1][hx];
                sres += S.x0[hy + 1][hx + 1];
                bc[(size_t)I + (size_t)J * nxc] = sres;
            }
        }
        __syncthreads();  // the next tile reuses the staged arrays
    }
}

template <typename TB, bool FB = false>
__global__ void __launch_bounds__(256, 6) k_mg_down(Lv L, const TB *b, float *xo, int nxc, int nyc, float *bc,
                                                    FusedB fbv = FusedB{}, const CgDev *cg = nullptr) {
    mg_down_body<TB, FB>(grid_blk(), L, b, xo, nxc, nyc, bc, fbv, cg);
}

// Ascending half of level L: xt = xi + omega_c P xc, then two sweeps.  LAST (level 0): the second
// sweep writes z in Float64 and the outer CG's r'z, r'r finish the init or the iteration;
// otherwise it writes the level's result to xo.
template <typename TB, bool LAST>
__device__ __forceinline__ void mg_up_body(Blk B, const Lv &L, const TB *b, const float *xi, const float *xc, int nxc,
                                           float wc, float *xo, double *z, CgDev *cg, int init, double *partials,
                                           unsigned int *counter) {
    if (cg_finished(L.done)) return;
    __shared__ FusedSm S;
    __shared__ double r64[LAST ? kFCells : 1];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // output rows: 32 x 8 threads
    const int tiles_x = (L.nx + kFW - 1) / kFW, ntiles = tiles_x * ((L.ny + kFH - 1) / kFH);
    double red[2] = {0.0, 0.0};
    for (int t = B.id; t < ntiles; t += B.n) {
        const int x0 = (t % tiles_x) * kFW, y0 = (t / tiles_x) * kFH;
        stage_level<TB, true>(S, L, b, x0, y0, LAST ? r64 : nullptr, xi, xc, nxc, wc);
        __syncthreads();
        sweep_sm(S, S.x0, S.x1, L.s2);
        __syncthreads();
        for (int r = ty; r < kFH; r += 8) {
            const int gx = x0 + tx, gy = y0 + r;
            if (gx >= L.nx || gy >= L.ny) continue;
            const int hx = tx + kFR, hy = r + kFR;
            const float ax = ax_sm(S, S.x1, hx, hy);
            const size_t q = (size_t)gx + (size_t)gy * L.nx;
            if (LAST) {
                const double rk = r64[hy * kFSW + hx];
                const double zk = (double)__fmaf_rn(S.wD[hy][hx], __fsub_rn((float)rk, ax), S.x1[hy][hx]);
                z[q] = zk;
                red[0] += rk * zk;
                red[1] += rk * rk;
            } else {
                xo[q] = __fmaf_rn(S.wD[hy][hx], __fsub_rn(S.b[hy][hx], ax), S.x1[hy][hx]);
            }
        }
        __syncthreads();
    }
    if (LAST) {
        double out[2];
        if (grid_reduce<2, false>(B, red, partials, counter, out) && threadIdx.x == 0) {
            if (init) cg_init_finish(cg, out[0], cg->rr, cg->bnorm);
            else cg_iter_finish(cg, out[0], out[1]);
        }
    }
}

template <typename TB, bool LAST>
__global__ void __launch_bounds__(256, 6) k_mg_up(Lv L, const TB *b, const float *xi, const float *xc, int nxc, float wc,
                                                  float *xo, double *z, CgDev *cg, int init, double *partials,
                                                  unsigned int *counter) {
    mg_up_body<TB, LAST>(grid_blk(), L, b, xi, xc, nxc, wc, xo, z, cg, init, partials, counter);
}

// ---------------------------------------------------------------------------------------------
// TMA-staged tile kernels (the default where every array of the level has a 16-byte-multiple
// row pitch).  Same tiles, sweeps and expressions as the kernels above -- the same V-cycle bit
// for bit -- but a block's staged region arrives by 2D tensor copies (cp.async.bulk.tensor) into
// one of two shared-memory stages, completing on that stage's mbarrier: while the block smooths
// tile t, the copies of its next tile t + gridDim.x are in flight, so each SM keeps several tiles'
// bytes moving instead of stalling on every staging load.  Cells outside the level arrive as
// zeros (the copies' out-of-bounds fill), as the staging loops above write them.
// Box origins keep the innermost coordinate x 16-byte aligned: Float64 boxes start 2 columns
// left of the tile (36 wide), Float32 boxes 4 (40 wide), the uint8 activity box 16 (64 wide); the
// coarse iterate box covers the tile's aggregates from 4 coarse columns left (24 x 10).
// ---------------------------------------------------------------------------------------------
constexpr int kTFW = kFSW + 4, kTOff = 2;     // Float32 boxes: 40 wide, staged hx = 0 at column 2
constexpr int kTAW = 64, kTAOff = 14;         // activity box: 64 wide, staged hx = 0 at column 14
constexpr int kTCW = 24, kTCH = 10;           // coarse iterate box
constexpr long kTmaSpin = 1L << 22;           // try_wait polls before a wait gives up

struct TmaArgs {  // the launch's tensor maps (kernel parameters, one 128-byte descriptor each)
    CUtensorMap b, ap, wD, dP, aE, aN, act, xi, xc;
};

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_bar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(bar)) : "memory");
}

__device__ __forceinline__ void tma_expect(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(su32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(su32(bar))
        : "memory");
}

// Bounded wait for the stage's phase `parity`; false when the polls ran out.
// Polls allowed to the first tile wait of every TMA-staged launch: kTmaSpin, except in the test
// of the give-up path, which sets 0 (SHK_TEST_TMA_FIRST_WAIT, read at context creation) so that
// the first wait gives up at once while its copies still arrive and are drained.
__device__ long g_tma_first_spin = kTmaSpin;

__device__ __forceinline__ bool tma_wait(uint64_t *bar, uint32_t parity, long spin = kTmaSpin) {
    for (long i = 0; i < spin; i++) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(su32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Shared-memory layout of one launch: two stages of boxes, then the two iterates over the staged
// region, then the stages' mbarriers.  Box offsets are 128-byte aligned.
template <typename TB, bool UP, bool FB>
struct TLayout {
    static constexpr unsigned rnd(unsigned v) { return (v + 127u) & ~127u; }
    static constexpr int bW = sizeof(TB) == 8 ? kFSW : kTFW, bOff = sizeof(TB) == 8 ? 0 : kTOff;
    static constexpr unsigned bB = bW * kFSH * sizeof(TB), apB = FB ? kFSW * kFSH * 8 : 0;
    static constexpr unsigned fB = kTFW * kFSH * 4, actB = kTAW * kFSH;
    static constexpr unsigned xiB = UP ? fB : 0, xcB = UP ? kTCW * kTCH * 4 : 0;
    static constexpr unsigned o_b = 0, o_ap = rnd(o_b + bB), o_wD = rnd(o_ap + apB), o_dP = rnd(o_wD + fB),
                              o_aE = rnd(o_dP + fB), o_aN = rnd(o_aE + fB), o_act = rnd(o_aN + fB),
                              o_xi = rnd(o_act + actB), o_xc = rnd(o_xi + xiB), stage = rnd(o_xc + xcB);
    static constexpr unsigned tx = bB + apB + 4 * fB + actB + xiB + xcB;  // bytes per stage fill
    static constexpr unsigned o_x0 = 2 * stage, o_x1 = o_x0 + kFCells * 4, o_bar = rnd(o_x1 + kFCells * 4),
                              bytes = o_bar + 16;
};

// One stage's copies for the tile at (x0, y0) (issued by one thread).
template <typename Y, bool UP, bool FB>
__device__ __forceinline__ void tma_issue(const TmaArgs &M, unsigned char *st, uint64_t *bar, int x0, int y0) {
    tma_expect(bar, Y::tx);
    tma_load(st + Y::o_b, &M.b, bar, x0 - kFR - Y::bOff, y0 - kFR);
    if (FB) tma_load(st + Y::o_ap, &M.ap, bar, x0 - kFR, y0 - kFR);
    tma_load(st + Y::o_wD, &M.wD, bar, x0 - kFR - kTOff, y0 - kFR);
    tma_load(st + Y::o_dP, &M.dP, bar, x0 - kFR - kTOff, y0 - kFR);
    tma_load(st + Y::o_aE, &M.aE, bar, x0 - kFR - kTOff, y0 - kFR);
    tma_load(st + Y::o_aN, &M.aN, bar, x0 - kFR - kTOff, y0 - kFR);
    tma_load(st + Y::o_act, &M.act, bar, x0 - kFR - kTAOff, y0 - kFR);
    if (UP) {
        tma_load(st + Y::o_xi, &M.xi, bar, x0 - kFR - kTOff, y0 - kFR);
        tma_load(st + Y::o_xc, &M.xc, bar, x0 / 2 - 4, y0 / 2 - 1);
    }
}

// The staged operator of one stage (Float32 boxes pre-offset so that [hy * kTFW + hx] is staged
// position (hx, hy), as is [hy * kTAW + hx] of the activity box).
struct TOp {
    const float *wD, *dP, *aE, *aN;
    const uint8_t *act;
};

template <typename Y>
__device__ __forceinline__ TOp stage_op(const unsigned char *st) {
    return TOp{reinterpret_cast<const float *>(st + Y::o_wD) + kTOff,
               reinterpret_cast<const float *>(st + Y::o_dP) + kTOff,
               reinterpret_cast<const float *>(st + Y::o_aE) + kTOff,
               reinterpret_cast<const float *>(st + Y::o_aN) + kTOff,
               reinterpret_cast<const uint8_t *>(st + Y::o_act) + kTAOff};
}

// Work split of the TMA kernels: each thread owns horizontal pairs of staged cells (hx even) and
// keeps their operator and rhs in registers across the prolongation, both sweeps and the residual;
// only the iterates go through shared memory, as 64-bit words.  The arithmetic runs on packed
// Float32 pairs (Blackwell's two-wide FMUL/FADD/FFMA), element for element the roundings of
// ax_sm and sweep_sm.  Slot 0 of thread t is tile pair t (row 2 + t / 16, pair 1 + t % 16: a warp
// holds one row of aggregates, so the restriction is a shuffle); slot 1 of threads t < 104 is one
// of the 104 pairs of the two-cell ring around the tile.
struct Pair {
    int k, fo, ao;   // staged index of the first cell (row pitch kFSW), its Float32 and activity box index
    bool sweep;      // in the sweeps' rows (1 .. kFH + 2); pairs at hx = 0 and 34 also compute their
                     // outer cell, whose result nothing reads
    float2 B, W, D, E, Ew, N, Ns;
    bool a0, a1;     // activity of the two cells
};

__device__ __forceinline__ void pair_at(Pair &P, int row, int pr) {
    P.k = row * kFSW + 2 * pr;
    P.fo = row * kTFW + 2 * pr;
    P.ao = row * kTAW + 2 * pr;
    P.sweep = row >= kFR - 1 && row <= kFR + kFH;
}

// Slot 1: ring pair i (0 <= i < 104): rows 0, 1, 18, 19 (18 pairs each), then the first and last
// pair of rows 2 .. 17.
__device__ __forceinline__ void ring_pair_at(Pair &P, int i) {
    constexpr int np = kFSW / 2;
    if (i < 4 * np) {
        const int r = i / np;
        pair_at(P, r < 2 ? r : kFSH - 4 + r, i % np);
    } else {
        const int j = i - 4 * np;
        pair_at(P, kFR + j / 2, (j % 2) * (np - 1));
    }
}
constexpr int kRingPairs = 4 * (kFSW / 2) + 2 * kFH;  // 104

__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void st2(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }

__device__ __forceinline__ void pair_load(Pair &P, const TOp &O) {
    P.W = ld2(O.wD + P.fo);
    P.D = ld2(O.dP + P.fo);
    P.E = ld2(O.aE + P.fo);
    P.Ew = make_float2(O.aE[P.fo - 1], P.E.x);
    P.N = ld2(O.aN + P.fo);
    P.Ns = P.sweep ? ld2(O.aN + P.fo - kTFW) : make_float2(0.0f, 0.0f);
    const uchar2 a = *reinterpret_cast<const uchar2 *>(O.act + P.ao);
    P.a0 = a.x != 0;
    P.a1 = a.y != 0;
}

// A X at the pair (ax_sm's roundings, elementwise).
__device__ __forceinline__ float2 pair_ax(const Pair &P, const float *X) {
    const float2 xc = ld2(X + P.k);
    float2 y = __fmul2_rn(P.D, xc);
    y = __ffma2_rn(P.E, sub2(xc, make_float2(xc.y, X[P.k + 2])), y);
    y = __ffma2_rn(P.Ew, sub2(xc, make_float2(X[P.k - 1], xc.x)), y);
    y = __ffma2_rn(P.N, sub2(xc, ld2(X + P.k + kFSW)), y);
    y = __ffma2_rn(P.Ns, sub2(xc, ld2(X + P.k - kFSW)), y);
    return y;
}

__device__ __forceinline__ void pair_sweep(const Pair &P, const float *XI, float *XO, float s) {
    const float2 w = __fmul2_rn(P.W, make_float2(s, s));
    st2(XO + P.k, __ffma2_rn(w, sub2(P.B, pair_ax(P, XI)), ld2(XI + P.k)));
}

// Records a failed wait (the solve stops and reports it).  Before the block returns, thread 0
// waits, with the normal bound, for every copy the block issued: the stage whose wait ran out
// (its copies may still be on their way) and, when pending, the other stage.  A block exits only
// after its staged copies have landed, so no copy writes shared memory a later block owns.
__device__ __forceinline__ void tma_give_up(CgDev *cg, uint64_t *cur, uint32_t cur_parity, bool cur_issued,
                                            uint64_t *other, uint32_t other_parity, bool other_pending) {
    if (threadIdx.x == 0) {
        if (cur_issued) tma_wait(cur, cur_parity);
        if (other_pending) tma_wait(other, other_parity);
        cg->fault = 1;
        atomicExch(&cg->done, 1);
    }
}

// Common frame of the two kernels: barrier set-up, the first tile's copies, and per tile the next
// tile's copies, PRE(tile origin) (work that needs no staged data), the wait, and BODY(stage, tile
// origin).
template <typename Y, typename Iss, typename Pre, typename Body>
__device__ __forceinline__ void tma_tiles(int nx, int ny, unsigned char *sm, CgDev *cg, Iss iss, Pre pre, Body body) {
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + Y::o_bar);
    const int tiles_x = (nx + kFW - 1) / kFW, ntiles = tiles_x * ((ny + kFH - 1) / kFH);
    if (su32(sm) & 127u) {  // the boxes' 128-byte alignment is not met: no copy is issued
        tma_give_up(cg, nullptr, 0, false, nullptr, 0, false);
        return;
    }
    if (threadIdx.x == 0) {
        tma_bar_init(&bar[0]);
        tma_bar_init(&bar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if ((int)blockIdx.x < ntiles)
            iss(sm, &bar[0], ((int)blockIdx.x % tiles_x) * kFW, ((int)blockIdx.x / tiles_x) * kFH);
    }
    __syncthreads();
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
        const int s = it & 1, tn = t + gridDim.x;
        if (threadIdx.x == 0 && tn < ntiles) {
            // the other stage was last read before the previous tile's closing barrier
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            iss(sm + (s ^ 1) * Y::stage, &bar[s ^ 1], (tn % tiles_x) * kFW, (tn / tiles_x) * kFH);
        }
        const int x0 = (t % tiles_x) * kFW, y0 = (t / tiles_x) * kFH;
        pre(x0, y0);
        const bool ok = tma_wait(&bar[s], (it >> 1) & 1, it == 0 ? g_tma_first_spin : kTmaSpin);
        if (__syncthreads_or(!ok)) {
            tma_give_up(cg, &bar[s], (it >> 1) & 1, true, &bar[s ^ 1], ((it + 1) >> 1) & 1, tn < ntiles);
            return;
        }
        body(sm + s * Y::stage, x0, y0);
        __syncthreads();  // the stage and the staged arrays are reused
    }
}

// The rhs pair at staged index k (Float64 boxes: pitch kFSW; Float32: kTFW, pre-offset).
template <typename Y>
__device__ __forceinline__ double2 rhs_pair(const double *SB, const Pair &P) {
    return *reinterpret_cast<const double2 *>(SB + P.k);
}
template <typename Y>
__device__ __forceinline__ double2 rhs_pair(const float *SB, const Pair &P) {
    const float2 v = ld2(SB + P.fo);
    return make_double2((double)v.x, (double)v.y);
}

// k_mg_down on TMA-staged tiles.  FB: x and p of the tile pair are read before the wait.
template <typename TB, bool FB>
__global__ void __launch_bounds__(256, 3) k_mg_down_t(const __grid_constant__ TmaArgs M, Lv L, float *xo, int nxc,
                                                      int nyc, float *bc, FusedB fbv, CgDev *cg) {
    if constexpr (FB) {
        const CgView cv = block_cg_view(cg);
        if (cv.done) return;
        fbv.alpha = cv.alpha;
        fbv.alpha_prev = cv.alpha_prev;
        if (fbv.mode && blockIdx.x == 0 && threadIdx.x == 0) cg->x_pending = fbv.mode == 1 ? 1 + fbv.pbuf : 0;
    } else {
        if (cg_finished(L.done)) return;
    }
    using Y = TLayout<TB, false, FB>;
    extern __shared__ __align__(128) unsigned char sm[];
    float *X0 = reinterpret_cast<float *>(sm + Y::o_x0);
    float *X1 = reinterpret_cast<float *>(sm + Y::o_x1);
    const int tid = threadIdx.x;
    Pair P0, P1;
    pair_at(P0, kFR + (tid >> 4), 1 + (tid & 15));
    const bool has1 = tid < kRingPairs;
    ring_pair_at(P1, has1 ? tid : 0);
    const int gx0 = -kFR + 2 * (1 + (tid & 15)), gy0 = (tid >> 4);  // tile pair's offset from (x0, y0)
    double2 xq = make_double2(0.0, 0.0), pq = xq;
    bool inside = false;
    size_t q = 0;
    tma_tiles<Y>(
        L.nx, L.ny, sm, cg,
        [&](unsigned char *st, uint64_t *b, int x0, int y0) { tma_issue<Y, false, FB>(M, st, b, x0, y0); },
        [&](int x0, int y0) {
            const int gx = x0 + gx0, gy = y0 + gy0;
            inside = gx < L.nx && gy < L.ny;  // nx is even: both cells of the pair, or neither
            q = (size_t)gx + (size_t)gy * L.nx;
            if constexpr (FB) {
                if (inside && fbv.mode != 1) {
                    xq = *reinterpret_cast<const double2 *>(fbv.x + q);
                    pq = *reinterpret_cast<const double2 *>(fbv.p + q);
                    if (fbv.mode == 2) {
                        const double2 pp = *reinterpret_cast<const double2 *>(fbv.p_prev + q);
                        xq = make_double2(__dadd_rn(xq.x, __dmul_rn(fbv.alpha_prev, pp.x)),
                                          __dadd_rn(xq.y, __dmul_rn(fbv.alpha_prev, pp.y)));
                    }
                }
            }
        },
        [&](unsigned char *st, int x0, int y0) {
            const TB *SB = reinterpret_cast<const TB *>(st + Y::o_b) + Y::bOff;
            const TOp O = stage_op<Y>(st);
            auto prep = [&](Pair &P, bool tile) {
                double2 bq = rhs_pair<Y>(SB, P);
                if constexpr (FB) {
                    const double2 ap = *reinterpret_cast<const double2 *>(
                        reinterpret_cast<const double *>(st + Y::o_ap) + P.k);
                    bq.x = __dadd_rn(bq.x, __dmul_rn(-fbv.alpha, ap.x));
                    bq.y = __dadd_rn(bq.y, __dmul_rn(-fbv.alpha, ap.y));
                    if (tile && inside) {
                        *reinterpret_cast<double2 *>(fbv.r_out + q) = bq;
                        if (fbv.mode != 1)
                            *reinterpret_cast<double2 *>(fbv.x + q) =
                                make_double2(__dadd_rn(xq.x, __dmul_rn(fbv.alpha, pq.x)),
                                             __dadd_rn(xq.y, __dmul_rn(fbv.alpha, pq.y)));
                    }
                }
                pair_load(P, O);
                P.B = make_float2((float)bq.x, (float)bq.y);
                st2(X0 + P.k, __fmul2_rn(P.W, P.B));
            };
            prep(P0, true);
            if (has1) prep(P1, false);
            __syncthreads();
            pair_sweep(P0, X0, X1, L.s2);
            if (has1 && P1.sweep) pair_sweep(P1, X0, X1, L.s2);
            __syncthreads();
            // residual of the tile pair (0 on inactive cells), x1 out, restriction by shuffle
            const float2 ax = pair_ax(P0, X1);
            const float2 x1 = ld2(X1 + P0.k);
            if (inside) *reinterpret_cast<float2 *>(xo + q) = x1;
            const float r0 = P0.a0 ? __fsub_rn(P0.B.x, ax.x) : 0.0f, r1 = P0.a1 ? __fsub_rn(P0.B.y, ax.y) : 0.0f;
            const float u0 = __shfl_down_sync(0xffffffffu, r0, 16), u1 = __shfl_down_sync(0xffffffffu, r1, 16);
            if ((tid & 16) == 0) {
                const int I = x0 / 2 + (tid & 15), J = y0 / 2 + (tid >> 5);
                if (I < nxc && J < nyc) {
                    float sres = 0.0f;
                    sres += r0;
                    sres += r1;
                    sres += u0;
                    sres += u1;
                    bc[(size_t)I + (size_t)J * nxc] = sres;
                }
            }
        });
}

// k_mg_up on TMA-staged tiles.
template <typename TB, bool LAST>
__global__ void __launch_bounds__(256, 4) k_mg_up_t(const __grid_constant__ TmaArgs M, Lv L, float wc, float *xo,
                                                    double *z, CgDev *cg, int init, double *partials,
                                                    unsigned int *counter) {
    if (cg_finished(L.done)) return;
    using Y = TLayout<TB, true, false>;
    extern __shared__ __align__(128) unsigned char sm[];
    float *X0 = reinterpret_cast<float *>(sm + Y::o_x0);
    float *X1 = reinterpret_cast<float *>(sm + Y::o_x1);
    const int tid = threadIdx.x;
    Pair P0, P1;
    pair_at(P0, kFR + (tid >> 4), 1 + (tid & 15));
    const bool has1 = tid < kRingPairs;
    ring_pair_at(P1, has1 ? tid : 0);
    const int gx0 = -kFR + 2 * (1 + (tid & 15)), gy0 = (tid >> 4);
    double red[2] = {0.0, 0.0};
    tma_tiles<Y>(
        L.nx, L.ny, sm, cg,
        [&](unsigned char *st, uint64_t *b, int x0, int y0) { tma_issue<Y, true, false>(M, st, b, x0, y0); },
        [&](int, int) {},
        [&](unsigned char *st, int x0, int y0) {
            const TB *SB = reinterpret_cast<const TB *>(st + Y::o_b) + Y::bOff;
            const TOp O = stage_op<Y>(st);
            const float *XI = reinterpret_cast<const float *>(st + Y::o_xi) + kTOff;
            const float *XC = reinterpret_cast<const float *>(st + Y::o_xc);
            auto prep = [&](Pair &P) {
                const double2 bq = rhs_pair<Y>(SB, P);
                pair_load(P, O);
                P.B = make_float2((float)bq.x, (float)bq.y);
                float2 v = ld2(XI + P.fo);
                // both cells of a pair prolong from the same coarse cell
                const int hx = P.k % kFSW, hy = P.k / kFSW;
                const float c = XC[(1 + ((hy - kFR) >> 1)) * kTCW + 4 + ((hx - kFR) >> 1)];
                if (P.a0) v.x = __fmaf_rn(wc, c, v.x);
                if (P.a1) v.y = __fmaf_rn(wc, c, v.y);
                st2(X0 + P.k, v);
            };
            prep(P0);
            if (has1) prep(P1);
            __syncthreads();
            pair_sweep(P0, X0, X1, L.s2);
            if (has1 && P1.sweep) pair_sweep(P1, X0, X1, L.s2);
            __syncthreads();
            const int gx = x0 + gx0, gy = y0 + gy0;
            if (gx < L.nx && gy < L.ny) {
                const float2 ax = pair_ax(P0, X1);
                const float2 x1 = ld2(X1 + P0.k);
                const size_t q = (size_t)gx + (size_t)gy * L.nx;
                if (LAST) {
                    const double2 rk = rhs_pair<Y>(SB, P0);
                    const double z0 = (double)__fmaf_rn(P0.W.x, __fsub_rn((float)rk.x, ax.x), x1.x);
                    const double z1 = (double)__fmaf_rn(P0.W.y, __fsub_rn((float)rk.y, ax.y), x1.y);
                    *reinterpret_cast<double2 *>(z + q) = make_double2(z0, z1);
                    red[0] += rk.x * z0;
                    red[0] += rk.y * z1;
                    red[1] += rk.x * rk.x;
                    red[1] += rk.y * rk.y;
                } else {
                    *reinterpret_cast<float2 *>(xo + q) = __ffma2_rn(P0.W, sub2(P0.B, ax), x1);
                }
            }
        });
    if (LAST) {
        double out[2];
        if (grid_reduce<2, false>(red, partials, counter, out) && threadIdx.x == 0) {
            if (init) cg_init_finish(cg, out[0], cg->rr, cg->bnorm);
            else cg_iter_finish(cg, out[0], out[1]);
        }
    }
}

// The outer CG's search-direction update and matvec of the multigrid form on TMA-staged tiles:
// p_new = z + beta p_old over the tile and a one-cell ring, then Ap = A p_new on the tile and
// p_new'Ap, with the Float64 roundings of k_cg_A (no fused multiply-adds: every product and sum is
// rounded, in k_cg_A's order, so the two kernels agree bit for bit up to the order of the grid
// sum).  Boxes: z and p_old over rows y0-1 .. y0+16 and columns x0-2 .. x0+33 (36 x 18), aP on
// the tile, aE from column x0-2 (34 x 16), aN from row y0-1 (32 x 17).
constexpr int kMvW = kFW + 4, kMvH = kFH + 2;  // staged p region (36 x 18)

struct MvArgs {
    CUtensorMap z, po, aP, aE, aN;
};

constexpr unsigned rnd128(unsigned v) { return (v + 127u) & ~127u; }

// JAC: the plain Jacobi-preconditioned CG's form -- z = r / aP is formed in the kernel, so aP is
// staged over the same 36 x 18 region as r and p_old.
template <bool JAC = false>
struct MvLayoutT {
    static constexpr unsigned pB = kMvW * kMvH * 8, apB = JAC ? pB : kFW * kFH * 8, aeB = (kFW + 2) * kFH * 8,
                              anB = kFW * (kFH + 1) * 8;
    static constexpr unsigned o_z = 0, o_po = rnd128(pB), o_aP = rnd128(o_po + pB), o_aE = rnd128(o_aP + apB),
                              o_aN = rnd128(o_aE + aeB), stage = rnd128(o_aN + anB);
    static constexpr unsigned o_p = 2 * stage, o_bar = rnd128(o_p + pB), bytes = o_bar + 16;
};
using MvLayout = MvLayoutT<false>;

template <bool JAC>
__global__ void __launch_bounds__(256, 4) k_cg_matvec_t(const __grid_constant__ MvArgs M, int nx, int ny,
                                                        double *p_new, double *Ap, CgDev *cg, double *partials,
                                                        unsigned int *counter, double eps_curv) {
    const CgView cv = block_cg_view(cg);
    if (cv.done) return;
    using Y = MvLayoutT<JAC>;
    extern __shared__ __align__(128) unsigned char sm[];
    double *P = reinterpret_cast<double *>(sm + Y::o_p);
    const bool first = cv.first != 0;
    const double beta = cv.beta;
    const int tid = threadIdx.x;
    const unsigned tx = Y::pB * (first ? 1 : 2) + Y::apB + Y::aeB + Y::anB;
    // p pairs: slot 0 = pair tid of the 324, slot 1 = pair 256 + tid (tid < 68)
    constexpr int np = kMvW / 2, npairs = np * kMvH;
    const int k0 = (tid / np) * kMvW + 2 * (tid % np), k1 = ((tid + 256) / np) * kMvW + 2 * ((tid + 256) % np);
    const bool has1 = tid + 256 < npairs;
    const int r = tid >> 4, pc = 2 * (tid & 15);  // the thread's output pair: tile row r, columns pc, pc + 1
    double acc = 0.0;
    tma_tiles<Y>(
        nx, ny, sm, cg,
        [&](unsigned char *st, uint64_t *b, int x0, int y0) {
            tma_expect(b, tx);
            tma_load(st + Y::o_z, &M.z, b, x0 - 2, y0 - 1);
            if (!first) tma_load(st + Y::o_po, &M.po, b, x0 - 2, y0 - 1);
            if (JAC) tma_load(st + Y::o_aP, &M.aP, b, x0 - 2, y0 - 1);
            else tma_load(st + Y::o_aP, &M.aP, b, x0, y0);
            tma_load(st + Y::o_aE, &M.aE, b, x0 - 2, y0);
            tma_load(st + Y::o_aN, &M.aN, b, x0, y0 - 1);
        },
        [&](int, int) {},
        [&](unsigned char *st, int x0, int y0) {
            const double *Z = reinterpret_cast<const double *>(st + Y::o_z);
            const double *PO = reinterpret_cast<const double *>(st + Y::o_po);
            const double *APh = reinterpret_cast<const double *>(st + Y::o_aP);
            auto form = [&](int k) {
                double2 z = *reinterpret_cast<const double2 *>(Z + k);  // JAC: r
                if (JAC) {  // outside the grid r = aP = 0 gives NaN there, a value no output reads
                    const double2 d = *reinterpret_cast<const double2 *>(APh + k);
                    z = make_double2(__ddiv_rn(z.x, d.x), __ddiv_rn(z.y, d.y));
                }
                double2 v = z;
                if (!first) {
                    const double2 po = *reinterpret_cast<const double2 *>(PO + k);
                    v = make_double2(__dadd_rn(z.x, __dmul_rn(beta, po.x)), __dadd_rn(z.y, __dmul_rn(beta, po.y)));
                }
                *reinterpret_cast<double2 *>(P + k) = v;
            };
            form(k0);
            if (has1) form(k1);
            __syncthreads();
            const double *AP = reinterpret_cast<const double *>(st + Y::o_aP);
            const double *AE = reinterpret_cast<const double *>(st + Y::o_aE);
            const double *AN = reinterpret_cast<const double *>(st + Y::o_aN);
            const int gy = y0 + r, gx = x0 + pc;
            if (gy < ny && gx < nx) {  // nx is even: both cells of the pair, or neither
                const int kp = (r + 1) * kMvW + pc + 2;  // staged index of the pair's first cell
                double y[2], pv[2];
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int k = kp + e, ix = gx + e;
                    const double pk = P[k];
                    double v = __dmul_rn(JAC ? AP[k] : AP[r * kFW + pc + e], pk);
                    if (ix < nx - 1) v = __dsub_rn(v, __dmul_rn(AE[r * (kFW + 2) + pc + e + 2], P[k + 1]));
                    if (ix > 0) v = __dsub_rn(v, __dmul_rn(AE[r * (kFW + 2) + pc + e + 1], P[k - 1]));
                    if (gy + 1 < ny) v = __dsub_rn(v, __dmul_rn(AN[(r + 1) * kFW + pc + e], P[k + kMvW]));
                    if (gy > 0) v = __dsub_rn(v, __dmul_rn(AN[r * kFW + pc + e], P[k - kMvW]));
                    y[e] = v;
                    pv[e] = pk;
                }
                const size_t q = (size_t)gx + (size_t)gy * nx;
                *reinterpret_cast<double2 *>(p_new + q) = make_double2(pv[0], pv[1]);
                *reinterpret_cast<double2 *>(Ap + q) = make_double2(y[0], y[1]);
                acc = __dadd_rn(acc, __dmul_rn(pv[0], y[0]));
                acc = __dadd_rn(acc, __dmul_rn(pv[1], y[1]));
            }
        });
    double red[1] = {acc}, out[1];
    if (grid_reduce<1, false>(red, partials, counter, out) && threadIdx.x == 0) {
        const double pAp = out[0];
        cg->pAp = pAp;
        const double lim = eps_curv * cg->pNorm2;
        if ((pAp <= lim && fabs(pAp) <= lim) || isnan(pAp)) {
            cg->done = 1;
            cg->status = SHK_BREAKDOWN;
        } else {
            cg->alpha_prev = cg->alpha;
            cg->alpha = __ddiv_rn(cg->gamma, pAp);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Warp-marching level kernels (SHK_MG_FUSED=2).  A warp owns a strip of 32 columns (lanes
// 2..29 are its 28 output columns; lanes 0, 1, 30, 31 the halo the two sweeps need) and marches
// down kMH rows plus two halo rows each side.  Each row is loaded once (coalesced), the two sweeps
// are pipelined two rows apart in registers, and the x +- 1 neighbours and the west coupling come
// from warp shuffles: no shared memory and no block barrier.  Cells outside the level load as
// zeros (act = 0, wD = 0), so every sweep leaves them at 0, and the couplings across the level's
// edge are zero in every operator, so no neighbour term needs a bounds test.
// ---------------------------------------------------------------------------------------------
constexpr int kMW = 28, kMH = 64;  // output columns and rows of a warp's strip

struct RowC {  // one row's coefficients at this lane's column
    float b, wD, dP, aE, aN;
    int act;
};

template <typename TB>
__device__ __forceinline__ RowC load_row(const Lv &L, const TB *b, int gx, int gy, bool inx, double *bd = nullptr) {
    RowC r;
    if (inx && gy >= 0 && gy < L.ny) {
        const size_t q = (size_t)gx + (size_t)gy * L.nx;
        const TB bq = b[q];
        if (bd) *bd = (double)bq;
        r.b = (float)bq;
        r.wD = L.wD[q];
        r.dP = L.dP[q];
        r.aE = L.aE[q];
        r.aN = L.aN[q];
        r.act = L.act[q];
    } else {
        if (bd) *bd = 0.0;
        r.b = r.wD = r.dP = r.aE = r.aN = 0.0f;
        r.act = 0;
    }
    return r;
}

// (A x) at row c: xs, xn the column's south/north values, aNs the south row's north coupling
__device__ __forceinline__ float ax_row(const RowC &c, float aNs, float x, float xs, float xn) {
    const float xe = __shfl_down_sync(0xffffffffu, x, 1), xw = __shfl_up_sync(0xffffffffu, x, 1);
    const float aW = __shfl_up_sync(0xffffffffu, c.aE, 1);
    float y = c.dP * x;
    y += c.aE * (x - xe);
    y += aW * (x - xw);
    y += c.aN * (x - xn);
    y += aNs * (x - xs);
    return y;
}

// Descending half: x1 = two sweeps from zero (to xo), coarse rhs bc = restriction of b - A x1.
template <typename TB>
__global__ void __launch_bounds__(128) k_mg_down_m(Lv L, const TB *b, float *xo, int nxc, int nyc, float *bc) {
    if (cg_finished(L.done)) return;
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const int sxn = (L.nx + kMW - 1) / kMW, nstrips = sxn * ((L.ny + kMH - 1) / kMH);
    for (int st = blockIdx.x * wpb + (threadIdx.x >> 5); st < nstrips; st += gridDim.x * wpb) {
        const int x0 = (st % sxn) * kMW, y0 = (st / sxn) * kMH;
        const int gx = x0 - 2 + lane;
        const bool inx = gx >= 0 && gx < L.nx, out_lane = lane >= 2 && lane < 2 + kMW && gx < L.nx;
        // pipeline registers: coefficients of rows j-1, j-2, j-3 (c1, c2, c3), x0 of rows j-1, j-2
        // (x0a, x0b), x1 of rows j-2, j-3 (x1a, x1b); row j is loaded at the top of the loop
        RowC c1 = load_row<TB>(L, b, gx, y0 - 3, inx), c2{}, c3{};
        RowC cj = load_row<TB>(L, b, gx, y0 - 2, inx);
        float x0a = cj.wD * cj.b, x0b = 0.0f, x0m = c1.wD * c1.b;  // rows y0-2, -, y0-3
        c3 = c2;
        c2 = c1;
        c1 = cj;
        x0b = x0m;
        float x1a = 0.0f, x1b = 0.0f, part = 0.0f;
        RowC nxt = load_row<TB>(L, b, gx, y0 - 1, inx);  // rows are fetched one iteration ahead
        for (int j = y0 - 1; j <= y0 + kMH + 1; j++) {
            cj = nxt;
            if (j + 1 <= y0 + kMH + 1) nxt = load_row<TB>(L, b, gx, j + 1, inx);
            const float x0j = cj.wD * cj.b;
            // x1 at row j-1 (c1, x0a) from x0 at rows j-2 (x0b), j-1, j
            const float ax0 = ax_row(c1, c2.aN, x0a, x0b, x0j);
            const float x1n = x0a + __fmul_rn(c1.wD, L.s2) * (c1.b - ax0);
            // residual at row j-2 (c2, x1a) from x1 at rows j-3 (x1b), j-2, j-1
            if (j - 2 >= y0) {
                const float ax1 = ax_row(c2, c3.aN, x1a, x1b, x1n);
                const float r = c2.act ? c2.b - ax1 : 0.0f;
                const float pr = r + __shfl_down_sync(0xffffffffu, r, 1);  // columns gx, gx + 1
                const int gy = j - 2;
                if ((gy & 1) == 0) {
                    part = pr;
                } else {
                    const int I = gx >> 1, J = gy >> 1;
                    if (out_lane && (lane & 1) == 0 && I < nxc && J < nyc) bc[(size_t)I + (size_t)J * nxc] = part + pr;
                }
            }
            if (j - 1 >= y0 && j - 1 < y0 + kMH && j - 1 < L.ny && out_lane)
                xo[(size_t)gx + (size_t)(j - 1) * L.nx] = x1n;
            // shift the pipeline
            c3 = c2;
            c2 = c1;
            c1 = cj;
            x0b = x0a;
            x0a = x0j;
            x1b = x1a;
            x1a = x1n;
        }
    }
}

// Ascending half: xt = xi + omega_c P xc, x2 = one sweep, then the second sweep; LAST (level 0)
// writes z in Float64 and finishes the outer CG's r'z, r'r; otherwise writes the result to xo.
template <typename TB, bool LAST>
__global__ void __launch_bounds__(128) k_mg_up_m(Lv L, const TB *b, const float *xi, const float *xc, int nxc,
                                                 float wc, float *xo, double *z, CgDev *cg, int init,
                                                 double *partials, unsigned int *counter) {
    if (cg_finished(L.done)) return;
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const int sxn = (L.nx + kMW - 1) / kMW, nstrips = sxn * ((L.ny + kMH - 1) / kMH);
    double red[2] = {0.0, 0.0};
    for (int st = blockIdx.x * wpb + (threadIdx.x >> 5); st < nstrips; st += gridDim.x * wpb) {
        const int x0 = (st % sxn) * kMW, y0 = (st / sxn) * kMH;
        const int gx = x0 - 2 + lane;
        const bool inx = gx >= 0 && gx < L.nx, out_lane = lane >= 2 && lane < 2 + kMW && gx < L.nx;
        // the fine iterate and the coarse value under this cell (0 outside the level)
        auto fetch_x = [&](int gy, float &fi, float &co) {
            fi = co = 0.0f;
            if (!inx || gy < 0 || gy >= L.ny) return;
            fi = xi[(size_t)gx + (size_t)gy * L.nx];
            co = xc[(size_t)(gx >> 1) + (size_t)(gy >> 1) * nxc];
        };
        auto xt_of = [&](const RowC &c, float fi, float co) -> float {  // the prolonged fine iterate
            float v = fi;
            if (c.act) v += wc * co;
            return v;
        };
        double bd = 0.0, bd1 = 0.0, bd2 = 0.0;  // Float64 rhs of rows j, j-1, j-2 (LAST)
        float fi, co;
        RowC c1 = load_row<TB>(L, b, gx, y0 - 3, inx, LAST ? &bd2 : nullptr), c2{}, c3{};
        fetch_x(y0 - 3, fi, co);
        float xtm = xt_of(c1, fi, co);
        RowC cj = load_row<TB>(L, b, gx, y0 - 2, inx, LAST ? &bd1 : nullptr);
        fetch_x(y0 - 2, fi, co);
        float xta = xt_of(cj, fi, co), xtb = xtm;
        c3 = c2;
        c2 = c1;
        c1 = cj;
        float x2a = 0.0f, x2b = 0.0f;
        double bdj1 = bd1, bdj2 = 0.0, bdn = 0.0;
        // rows are fetched one iteration ahead
        RowC nxt = load_row<TB>(L, b, gx, y0 - 1, inx, LAST ? &bdn : nullptr);
        float fin, con;
        fetch_x(y0 - 1, fin, con);
        for (int j = y0 - 1; j <= y0 + kMH + 1; j++) {
            cj = nxt;
            bd = bdn;
            fi = fin;
            co = con;
            if (j + 1 <= y0 + kMH + 1) {
                nxt = load_row<TB>(L, b, gx, j + 1, inx, LAST ? &bdn : nullptr);
                fetch_x(j + 1, fin, con);
            }
            const float xtj = xt_of(cj, fi, co);
            // x2 at row j-1 from xt at rows j-2, j-1, j
            const float axt = ax_row(c1, c2.aN, xta, xtb, xtj);
            const float x2n = xta + __fmul_rn(c1.wD, L.s2) * (c1.b - axt);
            // final sweep at row j-2 from x2 at rows j-3, j-2, j-1
            if (j - 2 >= y0) {
                const float ax2 = ax_row(c2, c3.aN, x2a, x2b, x2n);
                const int gy = j - 2;
                if (out_lane && gy < y0 + kMH && gy < L.ny) {
                    const size_t q = (size_t)gx + (size_t)gy * L.nx;
                    if (LAST) {
                        const double rk = bdj2;
                        const double zk = (double)(x2a + c2.wD * ((float)rk - ax2));
                        z[q] = zk;
                        red[0] += rk * zk;
                        red[1] += rk * rk;
                    } else {
                        xo[q] = x2a + c2.wD * (c2.b - ax2);
                    }
                }
            }
            c3 = c2;
            c2 = c1;
            c1 = cj;
            xtb = xta;
            xta = xtj;
            x2b = x2a;
            x2a = x2n;
            if (LAST) {
                bdj2 = bdj1;
                bdj1 = bd;
            }
        }
    }
    if (LAST) {
        double out[2];
        if (grid_reduce<2, false>(red, partials, counter, out) && threadIdx.x == 0) {
            if (init) cg_init_finish(cg, out[0], cg->rr, cg->bnorm);
            else cg_iter_finish(cg, out[0], out[1]);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Bottom of the V-cycle in one block: every level from `lb` down to the 1 x 1 coarsest level lives
// in shared memory (29 bytes per cell: aE, aN, dP, wD, x, scratch, b and the activity flag); the
// block runs the same pre-smoothing / restriction / exact solve / prolongation / post-smoothing
// sequence as the per-level kernels, separated by __syncthreads, and writes level lb's result to
// global memory.  This replaces five launches per small level with one launch per V-cycle.
// ---------------------------------------------------------------------------------------------
constexpr size_t kBottomBytesPerCell = 7 * sizeof(float) + 1;
constexpr size_t kBottomBytes = 200 * 1024;
// The one-block bottom kernel takes the levels of at most this many cells in all: with 1400 (the
// levels up to 32 x 32) one multigrid iteration at 4096^2 measured 590 us against 595 us with every
// level that fits its shared memory (up to 64 x 64), which the tile kernels then spread over all SMs.
constexpr long long kBottomMaxCells = 1400;

struct BottomLevel {
    int nx, ny, off;  // offset of this level's cells in the shared arrays
};
struct BottomPlan {
    int nlev, total;
    BottomLevel lv[kMgMaxLevels];
    const float *aE[kMgMaxLevels], *aN[kMgMaxLevels], *dP[kMgMaxLevels], *wD[kMgMaxLevels];
    const uint8_t *act[kMgMaxLevels];
    const int *done;
    float s2;  // Lv::s2
};

// Every loop over a level runs on a 2D thread map (32 columns x blockDim/32 rows), so no cell's
// coordinates need an integer division; the arithmetic per cell is unchanged.
__device__ __forceinline__ void mg_bottom_body(const BottomPlan &P, const float *b_top, float *x_top, int nu,
                                               float wc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (cg_finished(P.done)) return;
    const int T = P.total;
    float *sE = (float *)smem_raw, *sN = sE + T, *sD = sN + T, *sP = sD + T, *sX = sP + T, *sY = sX + T, *sB = sY + T;
    uint8_t *sA = (uint8_t *)(sB + T);
    const int tid = threadIdx.x, nt = blockDim.x, tx = tid & 31, ty = tid >> 5, nty = nt >> 5;
    for (int l = 0; l < P.nlev; l++) {
        const int n = P.lv[l].nx * P.lv[l].ny, o = P.lv[l].off;
        for (int i = tid; i < n; i += nt) {
            sE[o + i] = P.aE[l][i];
            sN[o + i] = P.aN[l][i];
            sD[o + i] = P.dP[l][i];
            sP[o + i] = P.wD[l][i];
            sA[o + i] = P.act[l][i];
            if (l == 0) sB[o + i] = b_top[i];
        }
    }
    __syncthreads();
    // (A X)_i on level l at (ix, iy), level-local index i
    auto Ax = [&](int l, const float *X, int ix, int iy, int i) -> float {
        const int nx = P.lv[l].nx, ny = P.lv[l].ny, o = P.lv[l].off;
        const float xc = X[o + i];
        float y = sD[o + i] * xc;
        if (ix < nx - 1) y += sE[o + i] * (xc - X[o + i + 1]);
        if (ix > 0) y += sE[o + i - 1] * (xc - X[o + i - 1]);
        if (iy < ny - 1) y += sN[o + i] * (xc - X[o + i + nx]);
        if (iy > 0) y += sN[o + i - nx] * (xc - X[o + i - nx]);
        return y;
    };
    // A level's iterate alternates between the two buffers, one damped-Jacobi sweep
    // XO = XI + wD (B - A XI) per swap (sP holds wD): the level's iterate is in Xb[cur].  The
    // descending half (the first sweep from zero into sX, nu - 1 more) leaves it in
    // Xb[(nu - 1) & 1]; the ascending half (nu sweeps from there) in Xb[(2 nu - 1) & 1] = sY;
    // the coarsest level's exact solve in sX.
    float *Xb[2] = {sX, sY};
    auto sweep = [&](int l, int cur, float w) {
        const int nx = P.lv[l].nx, ny = P.lv[l].ny, o = P.lv[l].off;
        const float *XI = Xb[cur];
        float *XO = Xb[cur ^ 1];
        for (int iy = ty; iy < ny; iy += nty)
            for (int ix = tx; ix < nx; ix += 32) {
                const int i = ix + iy * nx;
                XO[o + i] = XI[o + i] + __fmul_rn(sP[o + i], w) * (sB[o + i] - Ax(l, XI, ix, iy, i));
            }
        __syncthreads();
        return cur ^ 1;
    };
    // the last sweep before and the first after the coarse correction take the factor s2
    auto wpre = [&](int k) { return k == nu - 1 ? P.s2 : 1.0f; };
    auto wpost = [&](int k) { return k == 0 && nu > 1 ? P.s2 : 1.0f; };
    const int L = P.nlev;
    const int cur_down = (nu - 1) & 1, cur_up = 1;
    for (int l = 0; l < L - 1; l++) {  // descend
        const int n = P.lv[l].nx * P.lv[l].ny, o = P.lv[l].off;
        for (int i = tid; i < n; i += nt) sX[o + i] = sP[o + i] * sB[o + i];
        __syncthreads();
        int cur = 0;
        for (int s = 1; s < nu; s++) cur = sweep(l, cur, wpre(s));
        const float *XC = Xb[cur];
        const int nxf = P.lv[l].nx, nyf = P.lv[l].ny, nxc = P.lv[l + 1].nx, nyc = P.lv[l + 1].ny, oc = P.lv[l + 1].off;
        for (int J = ty; J < nyc; J += nty)
            for (int I = tx; I < nxc; I += 32) {
                float sres = 0.0f;
                for (int dj = 0; dj < 2; dj++)
                    for (int di = 0; di < 2; di++) {
                        const int i = 2 * I + di, j = 2 * J + dj;
                        if (i >= nxf || j >= nyf) continue;
                        const int f = i + j * nxf;
                        if (!sA[o + f]) continue;
                        sres += sB[o + f] - Ax(l, XC, i, j, f);
                    }
                sB[oc + I + J * nxc] = sres;
            }
        __syncthreads();
    }
    {  // coarsest level: exact solve
        const int l = L - 1, n = P.lv[l].nx * P.lv[l].ny, o = P.lv[l].off;
        for (int i = tid; i < n; i += nt) sX[o + i] = sA[o + i] ? sB[o + i] / sD[o + i] : sB[o + i];
        __syncthreads();
    }
    for (int l = L - 2; l >= 0; l--) {  // ascend
        const int nxf = P.lv[l].nx, nyf = P.lv[l].ny, o = P.lv[l].off, nxc = P.lv[l + 1].nx, oc = P.lv[l + 1].off;
        float *XF = Xb[cur_down];
        const float *XC = Xb[l + 1 == L - 1 ? 0 : cur_up];
        for (int j = ty; j < nyf; j += nty)
            for (int i = tx; i < nxf; i += 32) {
                const int f = i + j * nxf;
                if (sA[o + f]) XF[o + f] += wc * XC[oc + (i >> 1) + (j >> 1) * nxc];
            }
        __syncthreads();
        int cur = cur_down;
        for (int s = 0; s < nu; s++) cur = sweep(l, cur, wpost(s));
    }
    const float *X0 = Xb[L == 1 ? 0 : cur_up];
    for (int i = tid; i < P.lv[0].nx * P.lv[0].ny; i += nt) x_top[i] = X0[i];
}

__global__ void __launch_bounds__(1024) k_mg_bottom(BottomPlan P, const float *b_top, float *x_top, int nu,
                                                    float wc) {
    mg_bottom_body(P, b_top, x_top, nu, wc);
}

// ---------------------------------------------------------------------------------------------
// The coarse levels on one thread-block cluster (kClusterCtas CTAs of 1024 threads).  The levels
// from lc (the finest level whose slabs fit the CTAs' shared memory) down to the last one with more
// than kCta0Cells cells are "distributed": CTA k holds rows [rows0[k], rows0[k+1]) << (ndist - l) of
// level l in its shared memory (the partition of the first CTA-0 level doubled level by level, so a
// coarse row and the two fine rows it aggregates live in the same CTA) and reads the one row above
// and below its slab from the neighbouring CTAs' shared memory (ld.shared::cluster).  The levels
// from there on are small and live in CTA 0 alone, which runs the one-block bottom solve on them
// while the other CTAs wait.  The V-cycle and its arithmetic are mg_bottom_body's: first sweep from
// zero, nu - 1 more, residual restricted by 2 x 2 sums, exact coarsest solve, prolongation scaled by
// wc, nu sweeps -- so the cluster kernel and the one-block kernel produce the same V-cycle.
// Synchronisation between phases: the hardware cluster barrier (cl_sync), the same sequence of
// barriers in every CTA.  Measured at 4096^2 (one multigrid CG iteration): 584 us against 580 us
// for the tile kernels down to the one-block bottom kernel, so this form is opt-in
// (SHK_MG_CLUSTER=1); with barriers built on mbarriers (bounded polling) it took 597-609 us.
// ---------------------------------------------------------------------------------------------
constexpr int kClusterCtas = 8, kClusterThreads = 1024;
constexpr long long kCta0Cells = 1024;           // levels at most this size are solved by CTA 0
constexpr size_t kClusterBytes = 200 * 1024;     // dynamic shared memory per CTA
constexpr size_t kClusterBytesPerCell = 7 * sizeof(float) + 1;

struct ClusterPlan {
    int nlev, ndist, total;          // levels lc .. lc + nlev - 1 (kernel-local 0 .. nlev - 1)
    int rows0[kClusterCtas + 1];     // rows of level ndist per CTA (the distributed levels: doubled)
    int slot_rows[kMgMaxLevels];     // distributed level: rows of every CTA's slot (+ 1 south halo row)
    BottomLevel lv[kMgMaxLevels];    // nx, ny, off (the level's offset in every CTA's arrays)
    const float *aE[kMgMaxLevels], *aN[kMgMaxLevels], *dP[kMgMaxLevels], *wD[kMgMaxLevels];
    const uint8_t *act[kMgMaxLevels];
    const int *done;
    float s2;  // Lv::s2
};

__device__ __forceinline__ uint32_t cl_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cl_map(const void *p, uint32_t rank) {
    uint32_t a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(su32(p)), "r"(rank));
    return a;
}
__device__ __forceinline__ float cl_ld(const float *p, uint32_t rank) {
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(cl_map(p, rank)) : "memory");
    return v;
}
__device__ __forceinline__ void cl_st(float *p, uint32_t rank, float v) {
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(cl_map(p, rank)), "f"(v) : "memory");
}

// Cluster barrier: the hardware barrier.cluster (release/acquire at cluster scope for every thread's
// shared-memory stores and remote loads).  Like __syncthreads it waits for threads, not for a value
// in memory: the cluster's CTAs are resident together and all take the same barriers.
__device__ __forceinline__ void cl_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(kClusterThreads, 1) k_mg_cluster(ClusterPlan P, const float *b_top, float *x_top,
                                                                   int nu, float wc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t rank = cl_rank();
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5, nty = kClusterThreads >> 5;
    if (cg_finished(P.done)) return;  // the same flag in every CTA: all return, no remote access made
    const int T = P.total, L = P.nlev, ND = P.ndist;
    float *sE = (float *)smem_raw, *sN = sE + T, *sD = sN + T, *sP = sD + T, *sX = sP + T, *sY = sX + T, *sB = sY + T;
    uint8_t *sA = (uint8_t *)(sB + T);
    float *Xb[2] = {sX, sY};
    // rows of CTA k on distributed level l
    auto rows = [&](int l, int k, int &s, int &e) {
        const int sh = ND - l, ny = P.lv[l].ny;
        s = min(P.rows0[k] << sh, ny);
        e = min(P.rows0[k + 1] << sh, ny);
    };
    // the nearest CTAs below and above with rows (the same on every distributed level)
    int south = -1, north = -1;
    for (int k = (int)rank - 1; k >= 0 && south < 0; k--)
        if (P.rows0[k] < P.rows0[k + 1]) south = k;
    for (int k = (int)rank + 1; k < kClusterCtas && north < 0; k++)
        if (P.rows0[k] < P.rows0[k + 1]) north = k;
    // slot index of (ix, iy) on distributed level l in the arrays of a CTA whose rows start at s
    auto at = [&](int l, int s, int ix, int iy) { return P.lv[l].off + (iy - s + 1) * P.lv[l].nx + ix; };
    int s0, e0;
    rows(0, rank, s0, e0);
    // operators of this CTA's slabs (and the south halo row's north coupling), the top rhs
    for (int l = 0; l < ND; l++) {
        int s, e;
        rows(l, rank, s, e);
        const int nx = P.lv[l].nx, lo = s > 0 ? s - 1 : s;
        for (int iy = lo + ty; iy < e; iy += nty)
            for (int ix = tx; ix < nx; ix += 32) {
                const int g = ix + iy * nx, i = at(l, s, ix, iy);
                sN[i] = P.aN[l][g];
                if (iy < s) continue;
                sE[i] = P.aE[l][g];
                sD[i] = P.dP[l][g];
                sP[i] = P.wD[l][g];
                sA[i] = P.act[l][g];
                if (l == 0) sB[i] = b_top[g];
            }
    }
    if (rank == 0)
        for (int l = ND; l < L; l++) {
            const int n = P.lv[l].nx * P.lv[l].ny, o = P.lv[l].off;
            for (int i = tid; i < n; i += kClusterThreads) {
                sE[o + i] = P.aE[l][i];
                sN[o + i] = P.aN[l][i];
                sD[o + i] = P.dP[l][i];
                sP[o + i] = P.wD[l][i];
                sA[o + i] = P.act[l][i];
            }
        }
    __syncthreads();
    // (A X)_i on distributed level l at (ix, iy), slot index i, rows [s, e) of this CTA
    auto Axd = [&](int l, const float *X, int ix, int iy, int i, int s, int e) -> float {
        const int nx = P.lv[l].nx, ny = P.lv[l].ny;
        const float xc = X[i];
        float y = sD[i] * xc;
        if (ix < nx - 1) y += sE[i] * (xc - X[i + 1]);
        if (ix > 0) y += sE[i - 1] * (xc - X[i - 1]);
        if (iy < ny - 1) {
            float xn;
            if (iy + 1 < e) xn = X[i + nx];
            else {
                int sn, en;
                rows(l, north, sn, en);
                xn = cl_ld(X + at(l, sn, ix, iy + 1), north);
            }
            y += sN[i] * (xc - xn);
        }
        if (iy > 0) {
            float xs;
            if (iy - 1 >= s) xs = X[i - nx];
            else {
                int ss, es;
                rows(l, south, ss, es);
                xs = cl_ld(X + at(l, ss, ix, iy - 1), south);
            }
            y += sN[i - nx] * (xc - xs);
        }
        return y;
    };
    auto sweep_d = [&](int l, int cur, float w) {
        int s, e;
        rows(l, rank, s, e);
        const int nx = P.lv[l].nx;
        const float *XI = Xb[cur];
        float *XO = Xb[cur ^ 1];
        for (int iy = s + ty; iy < e; iy += nty)
            for (int ix = tx; ix < nx; ix += 32) {
                const int i = at(l, s, ix, iy);
                XO[i] = XI[i] + __fmul_rn(sP[i], w) * (sB[i] - Axd(l, XI, ix, iy, i, s, e));
            }
        cl_sync();
        return cur ^ 1;
    };
    // the last sweep before and the first after the coarse correction take the factor s2
    auto wpre = [&](int k) { return k == nu - 1 ? P.s2 : 1.0f; };
    auto wpost = [&](int k) { return k == 0 && nu > 1 ? P.s2 : 1.0f; };
    const int cur_down = (nu - 1) & 1, cur_up = 1;
    for (int l = 0; l < ND; l++) {  // descend on the distributed levels
        int s, e;
        rows(l, rank, s, e);
        const int nx = P.lv[l].nx, ny = P.lv[l].ny;
        for (int iy = s + ty; iy < e; iy += nty)
            for (int ix = tx; ix < nx; ix += 32) {
                const int i = at(l, s, ix, iy);
                sX[i] = sP[i] * sB[i];
            }
        cl_sync();
        int cur = 0;
        for (int k = 1; k < nu; k++) cur = sweep_d(l, cur, wpre(k));
        const float *XC = Xb[cur];
        const int nxc = P.lv[l + 1].nx, nyc = P.lv[l + 1].ny;
        int cs, ce;
        if (l + 1 < ND) rows(l + 1, rank, cs, ce);
        else {
            cs = P.rows0[rank];
            ce = P.rows0[rank + 1];
        }
        for (int J = cs + ty; J < ce; J += nty)
            for (int I = tx; I < nxc; I += 32) {
                float sres = 0.0f;
                for (int dj = 0; dj < 2; dj++)
                    for (int di = 0; di < 2; di++) {
                        const int i = 2 * I + di, j = 2 * J + dj;
                        if (i >= nx || j >= ny) continue;
                        const int f = at(l, s, i, j);
                        if (!sA[f]) continue;
                        sres += sB[f] - Axd(l, XC, i, j, f, s, e);
                    }
                if (l + 1 < ND) sB[at(l + 1, cs, I, J)] = sres;
                else if (rank == 0) sB[P.lv[l + 1].off + I + J * nxc] = sres;
                else cl_st(sB + P.lv[l + 1].off + I + J * nxc, 0, sres);
            }
        (void)nyc;
        if (l + 1 < ND) __syncthreads();
        else cl_sync();
    }
    if (rank == 0) {  // the small levels: the one-block bottom solve in CTA 0
        auto Ax = [&](int l, const float *X, int ix, int iy, int i) -> float {
            const int nx = P.lv[l].nx, ny = P.lv[l].ny, o = P.lv[l].off;
            const float xc = X[o + i];
            float y = sD[o + i] * xc;
            if (ix < nx - 1) y += sE[o + i] * (xc - X[o + i + 1]);
            if (ix > 0) y += sE[o + i - 1] * (xc - X[o + i - 1]);
            if (iy < ny - 1) y += sN[o + i] * (xc - X[o + i + nx]);
            if (iy > 0) y += sN[o + i - nx] * (xc - X[o + i - nx]);
            return y;
        };
        auto sweep = [&](int l, int cur, float w) {
            const int nx = P.lv[l].nx, ny = P.lv[l].ny, o = P.lv[l].off;
            const float *XI = Xb[cur];
            float *XO = Xb[cur ^ 1];
            for (int iy = ty; iy < ny; iy += nty)
                for (int ix = tx; ix < nx; ix += 32) {
                    const int i = ix + iy * nx;
                    XO[o + i] = XI[o + i] + __fmul_rn(sP[o + i], w) * (sB[o + i] - Ax(l, XI, ix, iy, i));
                }
            __syncthreads();
            return cur ^ 1;
        };
        for (int l = ND; l < L - 1; l++) {
            const int n = P.lv[l].nx * P.lv[l].ny, o = P.lv[l].off;
            for (int i = tid; i < n; i += kClusterThreads) sX[o + i] = sP[o + i] * sB[o + i];
            __syncthreads();
            int cur = 0;
            for (int k = 1; k < nu; k++) cur = sweep(l, cur, wpre(k));
            const float *XC = Xb[cur];
            const int nxf = P.lv[l].nx, nyf = P.lv[l].ny, nxc = P.lv[l + 1].nx, nyc = P.lv[l + 1].ny,
                      oc = P.lv[l + 1].off;
            for (int J = ty; J < nyc; J += nty)
                for (int I = tx; I < nxc; I += 32) {
                    float sres = 0.0f;
                    for (int dj = 0; dj < 2; dj++)
                        for (int di = 0; di < 2; di++) {
                            const int i = 2 * I + di, j = 2 * J + dj;
                            if (i >= nxf || j >= nyf) continue;
                            const int f = i + j * nxf;
                            if (!sA[o + f]) continue;
                            sres += sB[o + f] - Ax(l, XC, i, j, f);
                        }
                    sB[oc + I + J * nxc] = sres;
                }
            __syncthreads();
        }
        {  // coarsest level: exact solve
            const int l = L - 1, n = P.lv[l].nx * P.lv[l].ny, o = P.lv[l].off;
            for (int i = tid; i < n; i += kClusterThreads) sX[o + i] = sA[o + i] ? sB[o + i] / sD[o + i] : sB[o + i];
            __syncthreads();
        }
        for (int l = L - 2; l >= ND; l--) {
            const int nxf = P.lv[l].nx, nyf = P.lv[l].ny, o = P.lv[l].off, nxc = P.lv[l + 1].nx,
                      oc = P.lv[l + 1].off;
            float *XF = Xb[cur_down];
            const float *XC = Xb[l + 1 == L - 1 ? 0 : cur_up];
            for (int j = ty; j < nyf; j += nty)
                for (int i = tx; i < nxf; i += 32) {
                    const int f = i + j * nxf;
                    if (sA[o + f]) XF[o + f] += wc * XC[oc + (i >> 1) + (j >> 1) * nxc];
                }
            __syncthreads();
            int cur = cur_down;
            for (int k = 0; k < nu; k++) cur = sweep(l, cur, wpost(k));
        }
    }
    cl_sync();
    for (int l = ND - 1; l >= 0; l--) {  // ascend on the distributed levels
        int s, e;
        rows(l, rank, s, e);
        const int nx = P.lv[l].nx, nxc = P.lv[l + 1].nx;
        float *XF = Xb[cur_down];
        const float *XC = Xb[l + 1 == L - 1 ? 0 : cur_up];
        int cs, ce;
        if (l + 1 < ND) rows(l + 1, rank, cs, ce);
        for (int iy = s + ty; iy < e; iy += nty)
            for (int ix = tx; ix < nx; ix += 32) {
                const int f = at(l, s, ix, iy);
                if (!sA[f]) continue;
                float xc;
                if (l + 1 < ND) xc = XC[at(l + 1, cs, ix >> 1, iy >> 1)];
                else {
                    const float *q = XC + P.lv[l + 1].off + (ix >> 1) + (iy >> 1) * nxc;
                    xc = rank == 0 ? *q : cl_ld(q, 0);
                }
                XF[f] += wc * xc;
            }
        cl_sync();
        int cur = cur_down;
        for (int k = 0; k < nu; k++) cur = sweep_d(l, cur, wpost(k));
    }
    for (int iy = s0 + ty; iy < e0; iy += nty)
        for (int ix = tx; ix < P.lv[0].nx; ix += 32) x_top[ix + iy * P.lv[0].nx] = Xb[cur_up][at(0, s0, ix, iy)];
}

// ---------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------
static int mg_grid(Ctx *c, long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    long long cap = (long long)c->num_sms * 8;
    return (int)std::max(1LL, std::min(b, cap));
}

static const dim3 kBlock2d(32, 8);
static dim3 grid2d(int nx, int ny) { return dim3((unsigned)((nx + 31) / 32), (unsigned)((ny + 7) / 8)); }

static Lv level_view(const Ctx *c, const MgLevel &m, const int *done) {
    return Lv{m.nx, m.ny, m.aE, m.aN, m.dP, m.wD, m.act, done, c->mg_s2};
}
// Per-sweep kernels: the weight factor of pre-sweep s (1 .. nu - 1; sweep 0 is k_mg_pre0) and of
// post-sweep s (0 .. nu - 1), as the fused kernels apply it.
static float sweep_pre(const Ctx *c, int s) { return s == c->mg_nu - 1 ? c->mg_s2 : 1.0f; }
static float sweep_post(const Ctx *c, int s) { return s == 0 && c->mg_nu > 1 ? c->mg_s2 : 1.0f; }

// The fused two-sweep level kernels serve nu = 2 (the default); other nu use the per-sweep kernels.
// Among the fused kernels, the tile ones are the default (SHK_MG_FUSED=1); the warp-marching ones
// (SHK_MG_FUSED=2) are the alternative (at 4096^2 one V-cycle-preconditioned CG iteration takes
// 959 us with the tile kernels, 1044 us with the marching ones).
static bool fused(const Ctx *c) { return c->mg_fused && c->mg_nu == 2; }
static bool marching(const Ctx *c) { return fused(c) && c->mg_fused == 2; }
static int march_grid(const Ctx *c, const MgLevel &m) {
    const long long strips = (long long)((m.nx + kMW - 1) / kMW) * ((m.ny + kMH - 1) / kMH);
    return (int)std::max(1LL, std::min((strips + 3) / 4, (long long)c->max_blocks));
}
static int fused_grid(const Ctx *c, const MgLevel &m) {
    const long long tiles = (long long)((m.nx + kFW - 1) / kFW) * ((m.ny + kFH - 1) / kFH);
    // one resident wave (six 256-thread blocks per SM), striding over the tiles
    return (int)std::max(1LL, std::min({tiles, (long long)c->max_blocks, (long long)c->num_sms * 6}));
}

// First level >= 1 from which the rest of the hierarchy fits the bottom kernel's shared memory and
// holds at most kBottomMaxCells cells.
static int bottom_level(const Ctx *c) {
    long long rest = 0;
    int lb = c->mg_levels - 1;
    for (int l = c->mg_levels - 1; l >= 1; l--) {
        rest += (long long)c->mg[l].nx * c->mg[l].ny;
        if ((size_t)rest * kBottomBytesPerCell > kBottomBytes || rest > kBottomMaxCells) break;
        lb = l;
    }
    return lb;
}

static size_t bottom_plan(const Ctx *c, int lb, BottomPlan *P) {
    P->nlev = c->mg_levels - lb;
    int off = 0;
    for (int k = 0; k < P->nlev; k++) {
        const MgLevel &m = c->mg[lb + k];
        P->lv[k] = BottomLevel{m.nx, m.ny, off};
        P->aE[k] = m.aE; P->aN[k] = m.aN; P->dP[k] = m.dP; P->wD[k] = m.wD; P->act[k] = m.act;
        off += m.nx * m.ny;
    }
    P->total = off;
    P->s2 = c->mg_s2;
    return (size_t)off * kBottomBytesPerCell;
}

// The cluster kernel's levels: lc = the finest level >= 1 whose slabs fit kClusterBytes, the CTA-0
// levels from the first one with at most kCta0Cells cells.  False when the hierarchy has no level
// to distribute (small grids: the one-block bottom kernel serves them).
static bool cluster_plan(const Ctx *c, int *lc_out, ClusterPlan *P, size_t *bytes) {
    const int nl = c->mg_levels;
    int ld = -1;
    for (int l = 2; l < nl && ld < 0; l++)
        if ((long long)c->mg[l].nx * c->mg[l].ny <= kCta0Cells) ld = l;
    if (ld < 2) return false;
    int rows0[kClusterCtas + 1];
    for (int k = 0; k <= kClusterCtas; k++) rows0[k] = (int)((long long)k * c->mg[ld].ny / kClusterCtas);
    auto slab_rows = [&](int l) {  // the most rows any CTA holds on distributed level l
        const int sh = ld - l, ny = c->mg[l].ny;
        int r = 0;
        for (int k = 0; k < kClusterCtas; k++)
            r = std::max(r, std::min(rows0[k + 1] << sh, ny) - std::min(rows0[k] << sh, ny));
        return r;
    };
    long long small = 0;
    for (int l = ld; l < nl; l++) small += (long long)c->mg[l].nx * c->mg[l].ny;
    for (int lc = 1; lc < ld; lc++) {
        long long cells = small;
        for (int l = lc; l < ld; l++) cells += (long long)(slab_rows(l) + 1) * c->mg[l].nx;
        if ((size_t)cells * kClusterBytesPerCell > kClusterBytes) continue;
        memset(P, 0, sizeof(*P));
        P->nlev = nl - lc;
        P->ndist = ld - lc;
        P->total = (int)cells;
        for (int k = 0; k <= kClusterCtas; k++) P->rows0[k] = rows0[k];
        int off = 0;
        for (int k = 0; k < P->nlev; k++) {
            const MgLevel &m = c->mg[lc + k];
            P->lv[k] = BottomLevel{m.nx, m.ny, off};
            P->aE[k] = m.aE; P->aN[k] = m.aN; P->dP[k] = m.dP; P->wD[k] = m.wD; P->act[k] = m.act;
            P->slot_rows[k] = k < P->ndist ? slab_rows(lc + k) + 1 : m.ny;
            off += P->slot_rows[k] * m.nx;
        }
        P->s2 = c->mg_s2;
        *lc_out = lc;
        *bytes = (size_t)cells * kClusterBytesPerCell;
        return true;
    }
    return false;
}

// Per device: 0 not yet checked, 1 the cluster kernel can run, -1 it cannot (no cluster of
// kClusterCtas CTAs with its shared memory fits).  Checked in mg_setup, outside any stream capture.
static int g_cluster_ok[128] = {};

static int cluster_check(Ctx *c) {
    if (c->device < 0 || c->device >= 128) return fail(c, SHK_BAD_ARG, "device ordinal out of range");
    if (g_cluster_ok[c->device]) return SHK_OK;
    cudaError_t e = cudaFuncSetAttribute(k_mg_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClusterBytes);
    int n = 0;
    if (e == cudaSuccess) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kClusterCtas);
        cfg.blockDim = dim3(kClusterThreads);
        cfg.dynamicSmemBytes = kClusterBytes;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = kClusterCtas;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        e = cudaOccupancyMaxActiveClusters(&n, k_mg_cluster, &cfg);
    }
    if (e != cudaSuccess) cudaGetLastError();
    g_cluster_ok[c->device] = (e == cudaSuccess && n > 0) ? 1 : -1;
    return SHK_OK;
}

// The first level of the cluster kernel, or -1 when the one-block bottom kernel serves (also where
// the bottom kernel alone already starts at or above that level: small grids).
static int cluster_start(const Ctx *c, ClusterPlan *P, size_t *bytes) {
    if (!c->mg_cluster || c->device < 0 || c->device >= 128 || g_cluster_ok[c->device] != 1) return -1;
    int lc = -1;
    if (!cluster_plan(c, &lc, P, bytes) || lc >= bottom_level(c)) return -1;
    return lc;
}

struct MgTma;
static MgTma *tma_maps(Ctx *c, int *rc);

// Rebuilds every level's operator from the assembled Float64 system (after k_to_float_lapl).
int mg_setup(Ctx *c) {
    if (c->mg_levels < 1) return fail(c, SHK_CUDA_ERROR, "multigrid hierarchy not allocated");
    if (grid2d(c->nx, c->ny).y > 65535u) return fail(c, SHK_BAD_ARG, "multigrid needs ny <= 524280");
    MgLevel *lv = c->mg;
    const int n0 = c->nx * c->ny;
    if (c->mg_levels == 1) {  // level 0 alone (k_to_float_lapl has written its Float32 operator)
        k_mg_act0<<<mg_grid(c, n0), kThreads, 0, c->stream>>>(n0, c->mask8, c->aP, (double)c->mg_omega,
                                                               lv[0].act, lv[0].wD);
        c->launches++;
    }
    for (int l = 0; l + 1 < c->mg_levels; l++) {
        const MgLevel &f = lv[l];
        MgLevel &g = lv[l + 1];
        if (l > 0) {  // coarsening and the coarse level's Float32 copies in one pass
            k_mg_coarsen_finish<<<mg_grid(c, (long long)g.nx * g.ny), kThreads, 0, c->stream>>>(
                f.nx, f.ny, g.nx, g.ny, f.aE64, f.aN64, f.dP64, f.act, (double)c->mg_omega, g.aE64, g.aN64, g.dP64,
                g.act, (float *)g.aE, (float *)g.aN, (float *)g.dP, (float *)g.wD);
            c->launches++;
            continue;
        }
        k_mg_level0<<<grid2d(g.nx, g.ny), kBlock2d, 0, c->stream>>>(
            f.nx, f.ny, g.nx, g.ny, c->mask8, c->aP, c->aE, c->aN, (double)c->mg_omega, (float *)f.aE,
            (float *)f.aN, (float *)f.dP, (float *)f.wD, f.act, g.aE64, g.aN64, g.dP64, g.act);
        k_mg_finish_level<<<mg_grid(c, (long long)g.nx * g.ny), kThreads, 0, c->stream>>>(
            g.nx, g.ny, g.aE64, g.aN64, g.dP64, g.act, (double)c->mg_omega, (float *)g.aE, (float *)g.aN,
            (float *)g.dP, (float *)g.wD);
        c->launches += 2;
    }
    if (c->mg_levels > 1) {
        // the bottom kernel's dynamic shared memory limit, once per device
        static bool attr_set[128] = {};
        if (c->device < 0 || c->device >= 128) return fail(c, SHK_BAD_ARG, "device ordinal out of range");
        if (!attr_set[c->device]) {
            cudaError_t e = cudaFuncSetAttribute(k_mg_bottom, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)kBottomBytes);
            if (e != cudaSuccess) return check_cuda(c, e, "multigrid bottom shared memory");
            attr_set[c->device] = true;
        }
        if (c->mg_cluster) {
            const int rc = cluster_check(c);
            if (rc) return rc;
        }
        if (fused(c) && !marching(c)) {  // tensor maps and kernel attributes, outside any capture
            int rc = SHK_OK;
            tma_maps(c, &rc);
            if (rc) return rc;
        }
    }
    return check_launch(c, "multigrid setup");
}

// Tensor maps of the TMA-staged tile kernels, built once per context at the first multigrid set-up
// (outside any stream capture; the arrays live in the context's arena for its lifetime).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

struct MgTma {
    bool ok[kMgMaxLevels] = {};  // level l's tile kernels stage through TMA
    CUtensorMap wD[kMgMaxLevels], dP[kMgMaxLevels], aE[kMgMaxLevels], aN[kMgMaxLevels], act[kMgMaxLevels];
    CUtensorMap b[kMgMaxLevels], xi[kMgMaxLevels];
    CUtensorMap xc[kMgMaxLevels][2];  // level l's two iterates as coarse boxes (read by level l - 1)
    CUtensorMap r, r2, Ap;            // level 0's Float64 vectors
    bool mv_ok = false;               // the outer CG's matvec stages through TMA
    CUtensorMap mv_z, mv_p[2], mv_aP, mv_aE, mv_aN;
    int grid[6] = {};                 // per kernel: blocks of one resident wave
};

enum { TK_DOWN0, TK_DOWN0_FB, TK_DOWN, TK_UP0, TK_UP, TK_MV };

static bool encode(EncodeTiledFn fn, CUtensorMap *m, CUtensorMapDataType dt, size_t esz, const void *base, int nx,
                   int ny, int bw, int bh) {
    if (!base || (uintptr_t)base % 16 || ((size_t)nx * esz) % 16) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)ny};
    const cuuint64_t strides[1] = {(cuuint64_t)nx * esz};
    const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh}, es[2] = {1, 1};
    return fn(m, dt, 2, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename K>
static int tma_kernel_bps(Ctx *c, K kernel, unsigned smem, int *blocks_per_sm) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return check_cuda(c, e, "multigrid TMA kernel shared memory");
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kernel, 256, smem);
    if (e != cudaSuccess) return check_cuda(c, e, "multigrid TMA kernel occupancy");
    return SHK_OK;
}

void mg_release(Ctx *c) {
    delete c->mg_maps;
    c->mg_maps = nullptr;
    delete c->cg_maps;
    c->cg_maps = nullptr;
}

// The maps, or nullptr when the TMA kernels are off or no level qualifies.
static MgTma *tma_maps(Ctx *c, int *rc) {
    *rc = SHK_OK;
    if (!c->mg_tma || c->mg_levels < 2) return nullptr;
    if (c->mg_maps) return c->mg_maps;
    void *fp = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fp, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fp) {
        cudaGetLastError();
        c->mg_tma = 0;  // no driver entry point: the LDG-staged tile kernels serve every level
        return nullptr;
    }
    const EncodeTiledFn fn = (EncodeTiledFn)fp;
    MgTma *T = new MgTma();
    const CUtensorMapDataType F32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32, F64 = CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                              U8 = CU_TENSOR_MAP_DATA_TYPE_UINT8;
    const int lb = bottom_level(c);
    bool any = false;
    for (int l = 0; l < lb; l++) {
        const MgLevel &m = c->mg[l], &g = c->mg[l + 1];
        if (m.nx % 16 || g.nx % 4) continue;
        bool ok = encode(fn, &T->wD[l], F32, 4, m.wD, m.nx, m.ny, kTFW, kFSH) &&
                  encode(fn, &T->dP[l], F32, 4, m.dP, m.nx, m.ny, kTFW, kFSH) &&
                  encode(fn, &T->aE[l], F32, 4, m.aE, m.nx, m.ny, kTFW, kFSH) &&
                  encode(fn, &T->aN[l], F32, 4, m.aN, m.nx, m.ny, kTFW, kFSH) &&
                  encode(fn, &T->act[l], U8, 1, m.act, m.nx, m.ny, kTAW, kFSH) &&
                  encode(fn, &T->xi[l], F32, 4, m.x[0], m.nx, m.ny, kTFW, kFSH) &&
                  encode(fn, &T->xc[l + 1][0], F32, 4, g.x[0], g.nx, g.ny, kTCW, kTCH) &&
                  encode(fn, &T->xc[l + 1][1], F32, 4, g.x[1], g.nx, g.ny, kTCW, kTCH);
        if (l == 0)
            ok = ok && encode(fn, &T->r, F64, 8, c->r, m.nx, m.ny, kFSW, kFSH) &&
                 encode(fn, &T->r2, F64, 8, c->r2, m.nx, m.ny, kFSW, kFSH) &&
                 encode(fn, &T->Ap, F64, 8, c->Ap, m.nx, m.ny, kFSW, kFSH);
        else
            ok = ok && encode(fn, &T->b[l], F32, 4, m.b, m.nx, m.ny, kTFW, kFSH);
        T->ok[l] = ok;
        any = any || ok;
    }
    if (!any) {
        delete T;
        c->mg_tma = 0;
        return nullptr;
    }
    if (T->ok[0]) {
        const MgLevel &m = c->mg[0];
        T->mv_ok = encode(fn, &T->mv_z, F64, 8, c->z, m.nx, m.ny, kMvW, kMvH) &&
                   encode(fn, &T->mv_p[0], F64, 8, c->p[0], m.nx, m.ny, kMvW, kMvH) &&
                   encode(fn, &T->mv_p[1], F64, 8, c->p[1], m.nx, m.ny, kMvW, kMvH) &&
                   encode(fn, &T->mv_aP, F64, 8, c->aP, m.nx, m.ny, kFW, kFH) &&
                   encode(fn, &T->mv_aE, F64, 8, c->aE, m.nx, m.ny, kFW + 2, kFH) &&
                   encode(fn, &T->mv_aN, F64, 8, c->aN, m.nx, m.ny, kFW, kFH + 1);
    }
    int bps[6] = {};
    int e = tma_kernel_bps(c, k_mg_down_t<double, false>, TLayout<double, false, false>::bytes, &bps[TK_DOWN0]);
    if (!e) e = tma_kernel_bps(c, k_mg_down_t<double, true>, TLayout<double, false, true>::bytes, &bps[TK_DOWN0_FB]);
    if (!e) e = tma_kernel_bps(c, k_mg_down_t<float, false>, TLayout<float, false, false>::bytes, &bps[TK_DOWN]);
    if (!e) e = tma_kernel_bps(c, k_mg_up_t<double, true>, TLayout<double, true, false>::bytes, &bps[TK_UP0]);
    if (!e) e = tma_kernel_bps(c, k_mg_up_t<float, false>, TLayout<float, true, false>::bytes, &bps[TK_UP]);
    if (!e) e = tma_kernel_bps(c, k_cg_matvec_t<false>, MvLayout::bytes, &bps[TK_MV]);
    if (e) {
        delete T;
        *rc = e;
        return nullptr;
    }
    for (int k = 0; k < 6; k++) {
        if (bps[k] < 1) {
            delete T;
            *rc = fail(c, SHK_CUDA_ERROR, "multigrid TMA kernel does not fit on an SM");
            return nullptr;
        }
        T->grid[k] = c->num_sms * bps[k];
    }
    c->mg_maps = T;
    return T;
}

static int tma_grid(const Ctx *c, const MgTma *T, int kind, const MgLevel &m) {
    const long long tiles = (long long)((m.nx + kFW - 1) / kFW) * ((m.ny + kFH - 1) / kFH);
    return (int)std::max(1LL, std::min({tiles, (long long)c->max_blocks, (long long)T->grid[kind]}));
}

static TmaArgs tma_args(const MgTma *T, int l, const CUtensorMap &b, const CUtensorMap *ap, const CUtensorMap *xc) {
    TmaArgs a;
    memset(&a, 0, sizeof(a));
    a.b = b;
    if (ap) a.ap = *ap;
    a.wD = T->wD[l];
    a.dP = T->dP[l];
    a.aE = T->aE[l];
    a.aN = T->aN[l];
    a.act = T->act[l];
    a.xi = T->xi[l];
    if (xc) a.xc = *xc;
    return a;
}

// Level 0's residual map for a CG residual buffer (nullptr: not one of the context's buffers).
static const CUtensorMap *r_map(const Ctx *c, const MgTma *T, const double *r) {
    return r == c->r ? &T->r : r == c->r2 ? &T->r2 : nullptr;
}

// Recursive V-cycle on level l >= 1 with rhs lv[l].b; the solution ends in lv[l].x[*res].
static int vcycle(Ctx *c, int l, CgDev *cg, int *res) {
    MgLevel &m = c->mg[l];
    const int *done = &cg->done;
    const Lv L = level_view(c, m, done);
    const float wc = c->mg_omega_c;
    {
        ClusterPlan CP;
        size_t bytes = 0;
        if (l == cluster_start(c, &CP, &bytes)) {
            CP.done = done;
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(kClusterCtas);
            cfg.blockDim = dim3(kClusterThreads);
            cfg.dynamicSmemBytes = bytes;
            cfg.stream = c->stream;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = kClusterCtas;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            const cudaError_t e = cudaLaunchKernelEx(&cfg, k_mg_cluster, CP, (const float *)m.b, m.x[0], c->mg_nu, wc);
            if (e != cudaSuccess) return check_cuda(c, e, "multigrid cluster kernel launch");
            c->launches++;
            *res = 0;
            return SHK_OK;
        }
    }
    if (l == bottom_level(c)) {
        BottomPlan P;
        const size_t smem = bottom_plan(c, l, &P);
        P.done = done;
        k_mg_bottom<<<1, 1024, smem, c->stream>>>(P, m.b, m.x[0], c->mg_nu, wc);
        c->launches++;
        *res = 0;
        return SHK_OK;
    }
    MgLevel &g = c->mg[l + 1];
    if (marching(c)) {
        const int gm = march_grid(c, m);
        k_mg_down_m<float><<<gm, 128, 0, c->stream>>>(L, m.b, m.x[0], g.nx, g.ny, g.b);
        c->launches++;
        int gres = 0;
        int rc = vcycle(c, l + 1, cg, &gres);
        if (rc) return rc;
        k_mg_up_m<float, false><<<gm, 128, 0, c->stream>>>(L, m.b, m.x[0], g.x[gres], g.nx, wc, m.x[1], nullptr,
                                                           nullptr, 0, nullptr, nullptr);
        c->launches++;
        *res = 1;
        return SHK_OK;
    }
    int trc = SHK_OK;
    const MgTma *T = fused(c) ? tma_maps(c, &trc) : nullptr;
    if (trc) return trc;
    if (T && T->ok[l]) {
        const int gd = tma_grid(c, T, TK_DOWN, m), gu = tma_grid(c, T, TK_UP, m);
        k_mg_down_t<float, false><<<gd, 256, TLayout<float, false, false>::bytes, c->stream>>>(
            tma_args(T, l, T->b[l], nullptr, nullptr), L, m.x[0], g.nx, g.ny, g.b, FusedB{}, cg);
        c->launches++;
        int gres = 0;
        int rc = vcycle(c, l + 1, cg, &gres);
        if (rc) return rc;
        k_mg_up_t<float, false><<<gu, 256, TLayout<float, true, false>::bytes, c->stream>>>(
            tma_args(T, l, T->b[l], nullptr, &T->xc[l + 1][gres]), L, wc, m.x[1], nullptr, cg, 0, nullptr, nullptr);
        c->launches++;
        *res = 1;
        return SHK_OK;
    }
    if (fused(c)) {
        const int gt = fused_grid(c, m);
        k_mg_down<float><<<gt, 256, 0, c->stream>>>(L, m.b, m.x[0], g.nx, g.ny, g.b);
        c->launches++;
        int gres = 0;
        int rc = vcycle(c, l + 1, cg, &gres);
        if (rc) return rc;
        k_mg_up<float, false><<<gt, 256, 0, c->stream>>>(L, m.b, m.x[0], g.x[gres], g.nx, wc, m.x[1], nullptr,
                                                         nullptr, 0, nullptr, nullptr);
        c->launches++;
        *res = 1;
        return SHK_OK;
    }
    const dim3 gf = grid2d(m.nx, m.ny), gc = grid2d(g.nx, g.ny);
    k_mg_pre0<float><<<gf, kBlock2d, 0, c->stream>>>(L, m.b, m.x[0]);
    int cur = 0;
    for (int s = 1; s < c->mg_nu; s++, cur ^= 1)
        k_mg_sweep<float><<<gf, kBlock2d, 0, c->stream>>>(L, m.b, m.x[cur], m.x[cur ^ 1], sweep_pre(c, s));
    k_mg_restrict<float><<<gc, kBlock2d, 0, c->stream>>>(L, m.b, m.x[cur], g.nx, g.ny, g.b);
    c->launches += 1 + c->mg_nu;
    int gres = 0;
    int rc = vcycle(c, l + 1, cg, &gres);
    if (rc) return rc;
    k_mg_prolong_sweep<float><<<gf, kBlock2d, 0, c->stream>>>(L, m.b, m.x[cur], g.x[gres], g.nx, wc,
                                                              m.x[cur ^ 1], sweep_post(c, 0));
    cur ^= 1;
    for (int s = 1; s < c->mg_nu; s++, cur ^= 1)
        k_mg_sweep<float><<<gf, kBlock2d, 0, c->stream>>>(L, m.b, m.x[cur], m.x[cur ^ 1], sweep_post(c, s));
    c->launches += c->mg_nu;
    *res = cur;
    return SHK_OK;
}

// z = M^-1 r on level 0 (r Float64), then the outer CG's r'z (init or iteration finish).
int mg_apply(Ctx *c, const double *r, double *z, CgDev *cg, bool init) {
    MgLevel &m = c->mg[0];
    const Lv L = level_view(c, m, &cg->done);
    const int n = m.nx * m.ny;
    const float wc = c->mg_omega_c;
    const int gl = std::min(c->max_blocks, std::max(1, std::min(c->num_sms * 8, (n + kThreads - 1) / kThreads)));
    if (c->mg_levels == 1) {
        k_mg_last<false><<<gl, kThreads, 0, c->stream>>>(L, r, m.x[0], nullptr, 1, wc, z, cg, init, c->partials,
                                                         c->counter);
        c->launches++;
        return check_launch(c, "multigrid apply");
    }
    MgLevel &g = c->mg[1];
    if (marching(c)) {
        const int gm = march_grid(c, m);
        k_mg_down_m<double><<<gm, 128, 0, c->stream>>>(L, r, m.x[0], g.nx, g.ny, g.b);
        c->launches++;
        int gres = 0;
        int rc = vcycle(c, 1, cg, &gres);
        if (rc) return rc;
        k_mg_up_m<double, true><<<gm, 128, 0, c->stream>>>(L, r, m.x[0], g.x[gres], g.nx, wc, nullptr, z, cg, init,
                                                           c->partials, c->counter);
        c->launches++;
        return check_launch(c, "multigrid apply");
    }
    int trc = SHK_OK;
    const MgTma *T = fused(c) ? tma_maps(c, &trc) : nullptr;
    if (trc) return trc;
    if (T && T->ok[0] && r_map(c, T, r)) {
        const int gd = tma_grid(c, T, TK_DOWN0, m), gu = tma_grid(c, T, TK_UP0, m);
        k_mg_down_t<double, false><<<gd, 256, TLayout<double, false, false>::bytes, c->stream>>>(
            tma_args(T, 0, *r_map(c, T, r), nullptr, nullptr), L, m.x[0], g.nx, g.ny, g.b, FusedB{}, cg);
        c->launches++;
        int gres = 0;
        int rc = vcycle(c, 1, cg, &gres);
        if (rc) return rc;
        k_mg_up_t<double, true><<<gu, 256, TLayout<double, true, false>::bytes, c->stream>>>(
            tma_args(T, 0, *r_map(c, T, r), nullptr, &T->xc[1][gres]), L, wc, nullptr, z, cg, init, c->partials,
            c->counter);
        c->launches++;
        return check_launch(c, "multigrid apply");
    }
    if (fused(c)) {
        const int gt = fused_grid(c, m);
        k_mg_down<double><<<gt, 256, 0, c->stream>>>(L, r, m.x[0], g.nx, g.ny, g.b);
        c->launches++;
        int gres = 0;
        int rc = vcycle(c, 1, cg, &gres);
        if (rc) return rc;
        k_mg_up<double, true><<<gt, 256, 0, c->stream>>>(L, r, m.x[0], g.x[gres], g.nx, wc, nullptr, z, cg, init,
                                                         c->partials, c->counter);
        c->launches++;
        return check_launch(c, "multigrid apply");
    }
    const dim3 gf = grid2d(m.nx, m.ny), gc = grid2d(g.nx, g.ny);
    k_mg_pre0<double><<<gf, kBlock2d, 0, c->stream>>>(L, r, m.x[0]);
    int cur = 0;
    for (int s = 1; s < c->mg_nu; s++, cur ^= 1)
        k_mg_sweep<double><<<gf, kBlock2d, 0, c->stream>>>(L, r, m.x[cur], m.x[cur ^ 1], sweep_pre(c, s));
    k_mg_restrict<double><<<gc, kBlock2d, 0, c->stream>>>(L, r, m.x[cur], g.nx, g.ny, g.b);
    c->launches += 1 + c->mg_nu;
    int gres = 0;
    int rc = vcycle(c, 1, cg, &gres);
    if (rc) return rc;
    if (c->mg_nu == 1) {
        k_mg_last<true><<<gl, kThreads, 0, c->stream>>>(L, r, m.x[cur], g.x[gres], g.nx, wc, z, cg, init,
                                                        c->partials, c->counter);
        c->launches++;
    } else {
        k_mg_prolong_sweep<double><<<gf, kBlock2d, 0, c->stream>>>(L, r, m.x[cur], g.x[gres], g.nx, wc,
                                                                   m.x[cur ^ 1], sweep_post(c, 0));
        cur ^= 1;
        for (int s = 2; s < c->mg_nu; s++, cur ^= 1)
            k_mg_sweep<double><<<gf, kBlock2d, 0, c->stream>>>(L, r, m.x[cur], m.x[cur ^ 1], 1.0f);
        k_mg_last<false><<<gl, kThreads, 0, c->stream>>>(L, r, m.x[cur], nullptr, 1, wc, z, cg, init, c->partials,
                                                         c->counter);
        c->launches += c->mg_nu;
    }
    return check_launch(c, "multigrid apply");
}

// The outer CG's p update and matvec on TMA-staged tiles, where the context's maps cover these
// buffers; *launched says whether it ran (otherwise k_cg_A serves).
int mg_cg_matvec(Ctx *c, int par, const double *aP, const double *aE, const double *aN, const double *z,
                 const double *p_old, double *p_new, double *Ap, CgDev *cg, double eps_curv, bool *launched) {
    *launched = false;
    const MgTma *T = c->mg_maps;
    if (!T || !T->mv_ok || aP != c->aP || aE != c->aE || aN != c->aN || z != c->z || p_old != c->p[par] ||
        p_new != c->p[par ^ 1] || Ap != c->Ap)
        return SHK_OK;
    const MgLevel &m = c->mg[0];
    const MvArgs a{T->mv_z, T->mv_p[par], T->mv_aP, T->mv_aE, T->mv_aN};
    k_cg_matvec_t<false><<<tma_grid(c, T, TK_MV, m), 256, MvLayout::bytes, c->stream>>>(
        a, m.nx, m.ny, p_new, Ap, cg, c->partials, c->counter, eps_curv);
    *launched = true;
    return check_launch(c, "cg matvec");
}

// The plain Jacobi-preconditioned Float64 CG's p update and matvec on the same TMA-staged tiles
// (k_cg_matvec_t<true>: z = r / aP formed in the kernel; the roundings of k_cg_A<double, true>).
// Maps of the context's r, p[0], p[1], aP, aE, aN, built once per context before any capture.
struct CgTma {
    bool ok = false;
    CUtensorMap r, p[2], aP, aE, aN;
    int grid = 0;  // blocks of one resident wave
};

int cg_tma_prepare(Ctx *c) {
    if (c->cg_maps || !c->mg_tma) return SHK_OK;
    CgTma *T = new CgTma();
    c->cg_maps = T;
    void *fp = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fp, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fp) {
        cudaGetLastError();
        return SHK_OK;  // k_cg_A serves
    }
    const EncodeTiledFn fn = (EncodeTiledFn)fp;
    const CUtensorMapDataType F64 = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const int nx = c->nx, ny = c->ny;
    const bool maps = encode(fn, &T->r, F64, 8, c->r, nx, ny, kMvW, kMvH) &&
                      encode(fn, &T->p[0], F64, 8, c->p[0], nx, ny, kMvW, kMvH) &&
                      encode(fn, &T->p[1], F64, 8, c->p[1], nx, ny, kMvW, kMvH) &&
                      encode(fn, &T->aP, F64, 8, c->aP, nx, ny, kMvW, kMvH) &&
                      encode(fn, &T->aE, F64, 8, c->aE, nx, ny, kFW + 2, kFH) &&
                      encode(fn, &T->aN, F64, 8, c->aN, nx, ny, kFW, kFH + 1);
    if (!maps) return SHK_OK;
    int bps = 0;
    if (int e = tma_kernel_bps(c, k_cg_matvec_t<true>, MvLayoutT<true>::bytes, &bps)) return e;
    if (bps < 1) return SHK_OK;
    T->grid = c->num_sms * bps;
    T->ok = true;
    return SHK_OK;
}

int cg_jac_matvec(Ctx *c, int par, const double *r, const double *p_old, double *p_new, double *Ap, CgDev *cg,
                  double eps_curv, bool *launched) {
    *launched = false;
    const CgTma *T = c->cg_maps;
    if (!T || !T->ok || r != c->r || p_old != c->p[par] || p_new != c->p[par ^ 1] || Ap != c->Ap) return SHK_OK;
    const long long tiles = (long long)((c->nx + kFW - 1) / kFW) * ((c->ny + kFH - 1) / kFH);
    const int grid = (int)std::max(1LL, std::min({tiles, (long long)c->max_blocks, (long long)T->grid}));
    const MvArgs a{T->r, T->p[par], T->aP, T->aE, T->aN};
    k_cg_matvec_t<true><<<grid, 256, MvLayoutT<true>::bytes, c->stream>>>(a, c->nx, c->ny, p_new, Ap, cg,
                                                                           c->partials, c->counter, eps_curv);
    *launched = true;
    return check_launch(c, "cg matvec (Jacobi)");
}

// One iteration's x/r update fused into the V-cycle's first level-0 kernel (tile form, nu = 2):
// r_new = r_in - alpha Ap into r_out, x += alpha p, then z = M^-1 r_new and the CG's r'z, r'r.
bool mg_fuses_cg_update(const Ctx *c) { return marching(c) ? false : fused(c) && c->mg_levels > 1; }

// After a solve whose last iteration was the first of a pair: x += alpha p for the pending p (the
// rounding of the single update).  Returns at once when nothing is pending.
__global__ void k_cg_catchup(long long n, double *x, const double *p0, const double *p1, const CgDev *cg) {
    const int pend = cg->x_pending;
    if (!pend) return;
    const double *p = pend == 1 ? p0 : p1;
    const double a = cg->alpha;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = __dadd_rn(x[i], __dmul_rn(a, p[i]));
}

int mg_catch_up(Ctx *c, double *x, CgDev *cg) {
    k_cg_catchup<<<c->num_sms * 8, 256, 0, c->stream>>>((long long)c->nx * c->ny, x, c->p[0], c->p[1], cg);
    c->launches++;
    return check_launch(c, "cg pending x update");
}

// mode / p_prev / pbuf: the paired x update of FusedB (mode 0: x updated every iteration); the
// pairing needs the TMA-staged kernel, whose matvec records alpha_prev.
int mg_apply_fused_update(Ctx *c, const double *r_in, double *r_out, double *x, const double *p, const double *Ap,
                          double *z, CgDev *cg, const double *p_prev, int mode, int pbuf) {
    MgLevel &m = c->mg[0];
    const Lv L = level_view(c, m, &cg->done);
    MgLevel &g = c->mg[1];
    const float wc = c->mg_omega_c;
    int trc = SHK_OK;
    const MgTma *T = tma_maps(c, &trc);
    if (trc) return trc;
    if (T && T->ok[0] && r_map(c, T, r_in) && r_map(c, T, r_out) && Ap == c->Ap) {
        const int gd = tma_grid(c, T, TK_DOWN0_FB, m), gu = tma_grid(c, T, TK_UP0, m);
        k_mg_down_t<double, true><<<gd, 256, TLayout<double, false, true>::bytes, c->stream>>>(
            tma_args(T, 0, *r_map(c, T, r_in), &T->Ap, nullptr), L, m.x[0], g.nx, g.ny, g.b,
            FusedB{Ap, p, x, r_out, 0.0, p_prev, mode, pbuf, 0.0}, cg);
        c->launches++;
        int gres = 0;
        int rc = vcycle(c, 1, cg, &gres);
        if (rc) return rc;
        k_mg_up_t<double, true><<<gu, 256, TLayout<double, true, false>::bytes, c->stream>>>(
            tma_args(T, 0, *r_map(c, T, r_out), nullptr, &T->xc[1][gres]), L, wc, nullptr, z, cg, 0, c->partials,
            c->counter);
        c->launches++;
        return check_launch(c, "multigrid apply");
    }
    if (mode) return fail(c, SHK_CUDA_ERROR, "paired x updates need the TMA-staged level-0 kernel");
    const int gt = fused_grid(c, m);
    k_mg_down<double, true><<<gt, 256, 0, c->stream>>>(L, r_in, m.x[0], g.nx, g.ny, g.b,
                                                        FusedB{Ap, p, x, r_out, 0.0}, cg);
    c->launches++;
    int gres = 0;
    int rc = vcycle(c, 1, cg, &gres);
    if (rc) return rc;
    k_mg_up<double, true><<<gt, 256, 0, c->stream>>>(L, r_out, m.x[0], g.x[gres], g.nx, wc, nullptr, z, cg, 0,
                                                     c->partials, c->counter);
    c->launches++;
    return check_launch(c, "multigrid apply");
}

// Number of levels and their sizes: 2x2 aggregation down to a single cell.
int mg_levels_for(int nx, int ny, int *dims, int maxl) {
    int l = 0;
    int a = nx, b = ny;
    for (;;) {
        if (l >= maxl) return -1;
        dims[2 * l] = a;
        dims[2 * l + 1] = b;
        l++;
        if (a == 1 && b == 1) break;
        a = (a + 1) / 2;
        b = (b + 1) / 2;
    }
    return l;
}

// ---------------------------------------------------------------------------------------------
// Ensemble multigrid form: the V-cycle and its set-up batched over instances of uneven size.
//
// Each batched launch runs one level depth d of every instance that has it: the instance's blocks
// form a contiguous range (its block -> instance table and range start per depth), and each block
// runs the single-instance body on that instance's level with the instance's own block count, so
// the descending halves, the bottom solve and the ascending halves run in the order the instance's
// own V-cycle would: every instance's descending kernels depth by depth, then every instance's
// bottom kernel (one block each, whatever its bottom level), then the ascending kernels from the
// deepest depth up.  Instances between depths simply have no blocks in a launch.  The tile
// kernels are the LDG-staged ones (a launch's TMA tensor maps describe one array, not one per
// instance); the outer CG's x/r update is fused into the level-0 descending kernel as in the
// single-instance LDG path, alternating the two residual buffers with the iteration parity.
// ---------------------------------------------------------------------------------------------
struct EnsMg {
    int nlev, lb;
    int blk0_vc[kMgMaxLevels], nblk_vc[kMgMaxLevels];
    int blk0_set[kMgMaxLevels], nblk_set[kMgMaxLevels];
    MgLevel lv[kMgMaxLevels];
    BottomPlan bp;
    float wc;
    int nu;
    double omega;
    float s2;  // Lv::s2
};

// block -> (instance, position in its range) for table `tab` of depth d
struct EnsMgBlk {
    int i;
    Blk B;
};
__device__ __forceinline__ EnsMgBlk ens_mg_blk(const int *b2i, const EnsMg *M, bool vc, int d) {
    const int i = b2i[blockIdx.x];
    const EnsMg &G = M[i];
    const int b0 = vc ? G.blk0_vc[d] : G.blk0_set[d], nb = vc ? G.nblk_vc[d] : G.nblk_set[d];
    return EnsMgBlk{i, Blk{(int)blockIdx.x - b0, nb}};
}

// set-up of level d: d == 1 the level-0 pass (Float32 level 0 + level-1 sums), d == 2 level 1's
// Float32 copies, d >= 3 the coarsening of level d - 2 into level d - 1 (stage numbers, not levels:
// see ens_mg_setup)
__global__ void __launch_bounds__(256) k_ens_mg_setup(EnsInst *E, const EnsMg *M, const int *b2i, int stage) {
    const EnsMgBlk q = ens_mg_blk(b2i, M, false, stage);
    if (!E[q.i].pic_active) return;
    const EnsMg &G = M[q.i];
    const int tid = q.B.id * blockDim.x + threadIdx.x, nth = q.B.n * blockDim.x;
    if (stage == 1) {
        const EnsInst &I = E[q.i];
        const MgLevel &f = G.lv[0], &g = G.lv[1];
        for (int k = tid; k < g.nx * g.ny; k += nth)
            level0_aggregate(k % g.nx, k / g.nx, f.nx, f.ny, g.nx, I.mask8, I.aP, I.aE, I.aN, G.omega, (float *)f.aE,
                             (float *)f.aN, (float *)f.dP, (float *)f.wD, f.act, g.aE64, g.aN64, g.dP64, g.act);
    } else if (stage == 2) {
        const MgLevel &g = G.lv[1];
        for (int k = tid; k < g.nx * g.ny; k += nth)
            finish_level_cell(k, g.nx, g.aE64, g.aN64, g.dP64, g.act, G.omega, (float *)g.aE, (float *)g.aN,
                              (float *)g.dP, (float *)g.wD);
    } else {
        const MgLevel &f = G.lv[stage - 2], &g = G.lv[stage - 1];
        for (int k = tid; k < g.nx * g.ny; k += nth)
            coarsen_finish_cell(k, f.nx, f.ny, g.nx, f.aE64, f.aN64, f.dP64, f.act, G.omega, g.aE64, g.aN64, g.dP64,
                                g.act, (float *)g.aE, (float *)g.aN, (float *)g.dP, (float *)g.wD);
    }
}

// level 0 descending half: INIT stages r; an iteration applies the CG's x/r update (FB)
template <bool FB>
__global__ void __launch_bounds__(256, 6) k_ens_mg_down0(EnsInst *E, const EnsMg *M, const int *b2i, int parity) {
    const EnsMgBlk q = ens_mg_blk(b2i, M, true, 0);
    const EnsInst &I = E[q.i];
    if (!I.pic_active) return;
    const EnsMg &G = M[q.i];
    const MgLevel &m = G.lv[0], &g = G.lv[1];
    const Lv L{m.nx, m.ny, m.aE, m.aN, m.dP, m.wD, m.act, &I.cg->done, G.s2};
    if constexpr (FB) {
        const double *r_in = parity ? I.r2 : I.r;
        double *r_out = parity ? I.r : I.r2;
        const double *p_new = parity ? I.p0 : I.p1;
        mg_down_body<double, true>(q.B, L, r_in, m.x[0], g.nx, g.ny, g.b, FusedB{I.Ap, p_new, I.x, r_out, 0.0}, I.cg);
    } else {
        mg_down_body<double, false>(q.B, L, I.r, m.x[0], g.nx, g.ny, g.b, FusedB{}, nullptr);
    }
}

__global__ void __launch_bounds__(256, 6) k_ens_mg_down(EnsInst *E, const EnsMg *M, const int *b2i, int d) {
    const EnsMgBlk q = ens_mg_blk(b2i, M, true, d);
    const EnsInst &I = E[q.i];
    if (!I.pic_active) return;
    const EnsMg &G = M[q.i];
    const MgLevel &m = G.lv[d], &g = G.lv[d + 1];
    const Lv L{m.nx, m.ny, m.aE, m.aN, m.dP, m.wD, m.act, &I.cg->done, G.s2};
    mg_down_body<float, false>(q.B, L, m.b, m.x[0], g.nx, g.ny, g.b, FusedB{}, nullptr);
}

// every instance's bottom solve, one block each (block i = instance i)
__global__ void __launch_bounds__(1024) k_ens_mg_bottom(EnsInst *E, const EnsMg *M) {
    const EnsInst &I = E[blockIdx.x];
    if (!I.pic_active) return;
    const EnsMg &G = M[blockIdx.x];
    const MgLevel &m = G.lv[G.lb];
    mg_bottom_body(G.bp, m.b, m.x[0], G.nu, G.wc);
}

__global__ void __launch_bounds__(256, 6) k_ens_mg_up(EnsInst *E, const EnsMg *M, const int *b2i, int d) {
    const EnsMgBlk q = ens_mg_blk(b2i, M, true, d);
    const EnsInst &I = E[q.i];
    if (!I.pic_active) return;
    const EnsMg &G = M[q.i];
    const MgLevel &m = G.lv[d], &g = G.lv[d + 1];
    const Lv L{m.nx, m.ny, m.aE, m.aN, m.dP, m.wD, m.act, &I.cg->done, G.s2};
    const float *xc = g.x[d + 1 == G.lb ? 0 : 1];
    mg_up_body<float, false>(q.B, L, m.b, m.x[0], xc, g.nx, G.wc, m.x[1], nullptr, nullptr, 0, nullptr, nullptr);
}

// level 0 ascending half: z and the CG's r'z, r'r (init or iteration finish) over the instance's
// own reduction buffers
__global__ void __launch_bounds__(256, 6) k_ens_mg_up0(EnsInst *E, const EnsMg *M, const int *b2i, int init,
                                                       int parity) {
    const EnsMgBlk q = ens_mg_blk(b2i, M, true, 0);
    const EnsInst &I = E[q.i];
    if (!I.pic_active) return;
    const EnsMg &G = M[q.i];
    const MgLevel &m = G.lv[0], &g = G.lv[1];
    const Lv L{m.nx, m.ny, m.aE, m.aN, m.dP, m.wD, m.act, &I.cg->done, G.s2};
    const double *r = init ? I.r : (parity ? I.r : I.r2);  // the iteration's new residual buffer
    const float *xc = g.x[1 == G.lb ? 0 : 1];
    mg_up_body<double, true>(q.B, L, r, m.x[0], xc, g.nx, G.wc, nullptr, I.z, I.cg, init, I.partials, I.counter);
}

int ens_mg_plan(Ctx *c, EnsMgPlan *plan) {
    if (c->mg_levels < 2) return fail(c, SHK_BAD_ARG, "the ensemble's multigrid form needs two or more levels");
    if (!(c->mg_fused && c->mg_nu == 2)) return fail(c, SHK_BAD_ARG, "the ensemble's multigrid form runs nu = 2");
    plan->nlev = c->mg_levels;
    plan->lb = bottom_level(c);
    for (int l = 0; l < kMgMaxLevels; l++) plan->vc_blocks[l] = plan->set_blocks[l] = 0;
    for (int l = 0; l < plan->lb; l++) plan->vc_blocks[l] = fused_grid(c, c->mg[l]);
    // set-up stages 1 .. nlev: 1 and 2 produce level 1, s >= 3 level s - 1
    for (int st = 1; st <= plan->nlev; st++) {
        const MgLevel &g = c->mg[st <= 2 ? 1 : st - 1];
        plan->set_blocks[st] = st - 1 < plan->nlev ? mg_grid(c, (long long)g.nx * g.ny) : 0;
    }
    BottomPlan P;
    plan->bottom_smem = bottom_plan(c, plan->lb, &P);
    return SHK_OK;
}

EnsMg *ens_mg_alloc(int n) {
    EnsMg *d = nullptr;
    if (cudaMalloc(&d, (size_t)n * sizeof(EnsMg)) != cudaSuccess) return nullptr;
    return d;
}
const EnsMg *ens_mg_at(const EnsMg *dM, int i) { return dM + i; }
void ens_mg_free(EnsMg *dM) {
    if (dM) cudaFree(dM);
}

int ens_mg_upload(EnsMg *dM, int i, Ctx *c, const int *blk0_vc, const int *blk0_set) {
    EnsMgPlan plan;
    int rc = ens_mg_plan(c, &plan);
    if (rc) return rc;
    EnsMg G;
    memset(&G, 0, sizeof(G));
    G.nlev = plan.nlev;
    G.lb = plan.lb;
    for (int l = 0; l < kMgMaxLevels; l++) {
        G.blk0_vc[l] = blk0_vc[l];
        G.nblk_vc[l] = plan.vc_blocks[l];
        G.blk0_set[l] = blk0_set[l];
        G.nblk_set[l] = plan.set_blocks[l];
    }
    for (int l = 0; l < G.nlev; l++) G.lv[l] = c->mg[l];
    bottom_plan(c, plan.lb, &G.bp);
    G.bp.done = &c->dev->cg.done;
    G.wc = c->mg_omega_c;
    G.nu = c->mg_nu;
    G.omega = (double)c->mg_omega;
    G.s2 = c->mg_s2;
    return cudaMemcpy(dM + i, &G, sizeof(G), cudaMemcpyHostToDevice) == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

// The set-up of every instance's hierarchy after its assembly (mg_setup's sequence, stage by stage).
void ens_mg_setup(cudaStream_t s, EnsInst *E, const EnsMg *M, const int *const *b2i_set, const int *nb_set,
                  int lmax) {
    for (int st = 1; st <= lmax; st++)
        if (nb_set[st] > 0) k_ens_mg_setup<<<nb_set[st], 256, 0, s>>>(E, M, b2i_set[st], st);
}

// One V-cycle of every instance: INIT on r (the CG's set-up), ITER with the CG's x/r update of
// iteration `parity` fused into level 0.
void ens_mg_vcycle(cudaStream_t s, EnsInst *E, const EnsMg *M, const int *const *b2i_vc, const int *nb_vc, int dmax,
                   const int *b2i_bottom, int n, size_t bottom_smem, int mode, int parity) {
    (void)b2i_bottom;
    if (mode == ENS_VC_INIT) k_ens_mg_down0<false><<<nb_vc[0], 256, 0, s>>>(E, M, b2i_vc[0], parity);
    else k_ens_mg_down0<true><<<nb_vc[0], 256, 0, s>>>(E, M, b2i_vc[0], parity);
    for (int d = 1; d < dmax; d++)
        if (nb_vc[d] > 0) k_ens_mg_down<<<nb_vc[d], 256, 0, s>>>(E, M, b2i_vc[d], d);
    k_ens_mg_bottom<<<n, 1024, bottom_smem, s>>>(E, M);
    for (int d = dmax - 1; d >= 1; d--)
        if (nb_vc[d] > 0) k_ens_mg_up<<<nb_vc[d], 256, 0, s>>>(E, M, b2i_vc[d], d);
    k_ens_mg_up0<<<nb_vc[0], 256, 0, s>>>(E, M, b2i_vc[0], mode == ENS_VC_INIT ? 1 : 0, parity);
}

// The ensemble bottom kernel's dynamic shared memory limit on the current device.
int ens_mg_kernel_attrs() {
    return cudaFuncSetAttribute(k_ens_mg_bottom, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBottomBytes) ==
                   cudaSuccess
               ? SHK_OK
               : SHK_CUDA_ERROR;
}

// The first-wait poll count of the TMA-staged kernels on the current device: kTmaSpin, or the
// value of SHK_TEST_TMA_FIRST_WAIT (the give-up path's test).  Called at context creation.
int mg_set_first_wait_polls() {
    long v = kTmaSpin;
    if (const char *e = getenv("SHK_TEST_TMA_FIRST_WAIT")) v = std::max(0L, atol(e));
    return cudaMemcpyToSymbol(g_tma_first_spin, &v, sizeof(v)) == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

} // namespace shk
