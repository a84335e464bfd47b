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
// of P is zero); the smoother solves them exactly.  The V-cycle is symmetric (the same damped-Jacobi
// sweeps before and after the coarse correction; exact solve on the 1x1 coarsest level), so it is
// a valid CG preconditioner.  Per level: nu damped-Jacobi sweeps (omega = 2/3) before and after,
// coarse correction scaled by omega_c.
#include <cuda_runtime.h>
#include <float.h>
#include <string.h>

#include <algorithm>

#include "shk_device.cuh"

namespace shk {

#define GSTRIDE(i, n) for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

// ---------------------------------------------------------------------------------------------
// Hierarchy construction
// ---------------------------------------------------------------------------------------------

// Level-0 activity flags: rows assembled by the GROUNDED branch (mask codes 0 and "other").
__global__ void k_mg_act0(int n, const uint8_t *m8, uint8_t *act) {
    GSTRIDE(i, n) act[i] = (m8[i] == M_GROUNDED || m8[i] == M_UNKNOWN) ? 1 : 0;
}

// Fine excess dP = aP - (aE + aW + aN + aS) at level 0 (Float64 operator, 3-array storage).
__device__ __forceinline__ double dP0(const double *aP, const double *aE, const double *aN, int nx, int ix, int iy,
                                      size_t c) {
    const double w = ix > 0 ? aE[c - 1] : 0.0, s = iy > 0 ? aN[c - nx] : 0.0;
    return aP[c] - (aE[c] + w + aN[c] + s);
}

// Coarse operator of level l+1 from level l.  Fine inputs in Float64: aE, aN and either dP (fine
// level >= 1) or aP (fine level 0, dP computed on the fly).
__global__ void k_mg_coarsen(int nxf, int nyf, int nxc, int nyc, const double *aEf, const double *aNf,
                             const double *dPf, const double *aPf, const uint8_t *actf, double *aEc, double *aNc,
                             double *dPc, uint8_t *actc) {
    GSTRIDE(k, nxc * nyc) {
        const int I = k % nxc, J = k / nxc;
        double d = 0.0, e = 0.0, no = 0.0;
        int act = 0;
        for (int dj = 0; dj < 2; dj++)
            for (int di = 0; di < 2; di++) {
                const int i = 2 * I + di, j = 2 * J + dj;
                if (i >= nxf || j >= nyf) continue;
                const size_t c = (size_t)i + (size_t)j * nxf;
                if (!actf[c]) continue;
                act = 1;
                d += dPf ? dPf[c] : dP0(aPf, aEf, aNf, nxf, i, j, c);
            }
        const int ie = 2 * I + 1;  // fine column on the west side of the east aggregate boundary
        if (ie + 1 < nxf)
            for (int dj = 0; dj < 2; dj++) {
                const int j = 2 * J + dj;
                if (j >= nyf) continue;
                const size_t c = (size_t)ie + (size_t)j * nxf;
                if (actf[c] && actf[c + 1]) e += aEf[c];
            }
        const int jn = 2 * J + 1;
        if (jn + 1 < nyf)
            for (int di = 0; di < 2; di++) {
                const int i = 2 * I + di;
                if (i >= nxf) continue;
                const size_t c = (size_t)i + (size_t)jn * nxf;
                if (actf[c] && actf[c + nxf]) no += aNf[c];
            }
        aEc[k] = act ? e : 0.0;
        aNc[k] = act ? no : 0.0;
        dPc[k] = act ? d : 1.0;
        actc[k] = (uint8_t)act;
    }
}

// Float32 copies and the Jacobi diagonal aP = dP + sum of the four couplings.
__global__ void k_mg_finish_level(int nx, int ny, const double *aE, const double *aN, const double *dP,
                                  const uint8_t *act, float *fE, float *fN, float *fD, float *fP) {
    GSTRIDE(k, nx * ny) {
        const int ix = k % nx, iy = k / nx;
        const double w = ix > 0 ? aE[k - 1] : 0.0, s = iy > 0 ? aN[k - nx] : 0.0;
        fE[k] = (float)aE[k];
        fN[k] = (float)aN[k];
        fD[k] = (float)dP[k];
        fP[k] = act[k] ? (float)(dP[k] + (aE[k] + w + aN[k] + s)) : 1.0f;
    }
}

// ---------------------------------------------------------------------------------------------
// V-cycle kernels (Float32)
// ---------------------------------------------------------------------------------------------
struct Lv {
    int nx, ny;
    const float *aE, *aN, *dP, *aP;
    const uint8_t *act;
};

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

__device__ __forceinline__ float omega_of(const Lv &L, size_t c, float w) { return L.act[c] ? w : 1.0f; }

// First pre-smoothing sweep from x = 0: x = omega b / aP.  Level 0 reads b in Float64 (the outer
// residual).
template <typename TB>
__global__ void k_mg_pre0(Lv L, const TB *b, float *x, float w) {
    GSTRIDE(k, L.nx * L.ny) x[k] = omega_of(L, k, w) * (float)b[k] / L.aP[k];
}

// One damped-Jacobi sweep: xo = xi + omega (b - A xi) / aP.
template <typename TB>
__global__ void k_mg_sweep(Lv L, const TB *b, const float *xi, float *xo, float w) {
    GSTRIDE(k, L.nx * L.ny) {
        const int ix = k % L.nx, iy = k / L.nx;
        const float xc = xi[k];
        const float ax = lapl_apply(L, ix, iy, k, xc, [&](size_t q) { return xi[q]; });
        xo[k] = xc + omega_of(L, k, w) * ((float)b[k] - ax) / L.aP[k];
    }
}

// Restriction of the residual: bc(C) = sum over the active fine cells of aggregate C of (b - A x).
template <typename TB>
__global__ void k_mg_restrict(Lv L, const TB *b, const float *x, int nxc, int nyc, float *bc) {
    GSTRIDE(k, nxc * nyc) {
        const int I = k % nxc, J = k / nxc;
        float s = 0.0f;
        for (int dj = 0; dj < 2; dj++)
            for (int di = 0; di < 2; di++) {
                const int i = 2 * I + di, j = 2 * J + dj;
                if (i >= L.nx || j >= L.ny) continue;
                const size_t c = (size_t)i + (size_t)j * L.nx;
                if (!L.act[c]) continue;
                const float ax = lapl_apply(L, i, j, c, x[c], [&](size_t q) { return x[q]; });
                s += (float)b[c] - ax;
            }
        bc[k] = s;
    }
}

// Coarsest level (1 x 1): exact solve.
__global__ void k_mg_coarsest(Lv L, const float *b, float *x) {
    GSTRIDE(k, L.nx * L.ny) x[k] = L.act[k] ? b[k] / L.dP[k] : b[k];
}

// Prolongation fused with the first post-smoothing sweep:
//   xt = xi + omega_c P xc,  xo = xt + omega (b - A xt) / aP.
template <typename TB>
__global__ void k_mg_prolong_sweep(Lv L, const TB *b, const float *xi, const float *xc, int nxc, float wc, float w,
                                   float *xo) {
    GSTRIDE(k, L.nx * L.ny) {
        const int ix = k % L.nx, iy = k / L.nx;
        auto xt = [&](size_t q) -> float {
            const int qi = (int)(q % L.nx), qj = (int)(q / L.nx);
            float v = xi[q];
            if (L.act[q]) v += wc * xc[(size_t)(qi >> 1) + (size_t)(qj >> 1) * nxc];
            return v;
        };
        const float xk = xt(k);
        const float ax = lapl_apply(L, ix, iy, k, xk, xt);
        xo[k] = xk + omega_of(L, k, w) * ((float)b[k] - ax) / L.aP[k];
    }
}

// Last post-smoothing sweep on level 0, writing z in Float64 and finishing the outer CG's r'z:
// z = xi + omega (r - A xi)/aP; partials r'z, r'r -> init or iteration finish.
template <bool PROLONG>
__global__ void __launch_bounds__(kThreads) k_mg_last(Lv L, const double *r, const float *xi, const float *xc, int nxc,
                                                      float wc, float w, double *z, CgDev *cg, int init,
                                                      double *partials, unsigned int *counter) {
    if (*(volatile int *)&cg->done) return;
    double red[2] = {0.0, 0.0};
    GSTRIDE(k, L.nx * L.ny) {
        const int ix = k % L.nx, iy = k / L.nx;
        auto xt = [&](size_t q) -> float {
            float v = xi[q];
            if (PROLONG && L.act[q]) {
                const int qi = (int)(q % L.nx), qj = (int)(q / L.nx);
                v += wc * xc[(size_t)(qi >> 1) + (size_t)(qj >> 1) * nxc];
            }
            return v;
        };
        const float xk = xt(k);
        const float ax = lapl_apply(L, ix, iy, k, xk, xt);
        const double rk = r[k];
        const double zk = (double)(xk + omega_of(L, k, w) * ((float)rk - ax) / L.aP[k]);
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
// Host side
// ---------------------------------------------------------------------------------------------
static int mg_grid(Ctx *c, long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    long long cap = (long long)c->num_sms * 8;
    return (int)std::max(1LL, std::min(b, cap));
}

static Lv level_view(const MgLevel &m) { return Lv{m.nx, m.ny, m.aE, m.aN, m.dP, m.aP, m.act}; }

// Rebuilds every level's operator from the assembled Float64 system (after k_to_float_lapl).
int mg_setup(Ctx *c) {
    if (c->mg_levels < 1) return fail(c, SHK_CUDA_ERROR, "multigrid hierarchy not allocated");
    MgLevel *lv = c->mg;
    const int n0 = c->nx * c->ny;
    k_mg_act0<<<mg_grid(c, n0), kThreads, 0, c->stream>>>(n0, c->mask8, lv[0].act);
    c->launches++;
    for (int l = 0; l + 1 < c->mg_levels; l++) {
        const MgLevel &f = lv[l];
        MgLevel &g = lv[l + 1];
        const double *aEf = l == 0 ? c->aE : f.aE64, *aNf = l == 0 ? c->aN : f.aN64;
        const double *dPf = l == 0 ? nullptr : f.dP64;
        k_mg_coarsen<<<mg_grid(c, (long long)g.nx * g.ny), kThreads, 0, c->stream>>>(
            f.nx, f.ny, g.nx, g.ny, aEf, aNf, dPf, c->aP, f.act, g.aE64, g.aN64, g.dP64, g.act);
        k_mg_finish_level<<<mg_grid(c, (long long)g.nx * g.ny), kThreads, 0, c->stream>>>(
            g.nx, g.ny, g.aE64, g.aN64, g.dP64, g.act, (float *)g.aE, (float *)g.aN, (float *)g.dP, (float *)g.aP);
        c->launches += 2;
    }
    return check_launch(c, "multigrid setup");
}

// Recursive V-cycle on level l >= 1 with rhs lv[l].b, solution into lv[l].x[0].
static void vcycle(Ctx *c, int l) {
    MgLevel &m = c->mg[l];
    Lv L = level_view(m);
    const int n = m.nx * m.ny;
    const float w = c->mg_omega, wc = c->mg_omega_c;
    if (l == c->mg_levels - 1) {
        k_mg_coarsest<<<mg_grid(c, n), kThreads, 0, c->stream>>>(L, m.b, m.x[0]);
        c->launches++;
        return;
    }
    MgLevel &g = c->mg[l + 1];
    k_mg_pre0<float><<<mg_grid(c, n), kThreads, 0, c->stream>>>(L, m.b, m.x[0], w);
    int cur = 0;
    for (int s = 1; s < c->mg_nu; s++, cur ^= 1)
        k_mg_sweep<float><<<mg_grid(c, n), kThreads, 0, c->stream>>>(L, m.b, m.x[cur], m.x[cur ^ 1], w);
    k_mg_restrict<float><<<mg_grid(c, (long long)g.nx * g.ny), kThreads, 0, c->stream>>>(L, m.b, m.x[cur], g.nx, g.ny,
                                                                                        g.b);
    c->launches += 1 + c->mg_nu;
    vcycle(c, l + 1);
    k_mg_prolong_sweep<float><<<mg_grid(c, n), kThreads, 0, c->stream>>>(L, m.b, m.x[cur], g.x[0], g.nx, wc, w,
                                                                         m.x[cur ^ 1]);
    cur ^= 1;
    for (int s = 1; s < c->mg_nu; s++, cur ^= 1)
        k_mg_sweep<float><<<mg_grid(c, n), kThreads, 0, c->stream>>>(L, m.b, m.x[cur], m.x[cur ^ 1], w);
    c->launches += c->mg_nu;
    if (cur != 0) {  // leave the result in x[0]
        cudaMemcpyAsync(m.x[0], m.x[1], (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, c->stream);
    }
}

// z = M^-1 r on level 0 (r Float64), then the outer CG's r'z (init or iteration finish).
int mg_apply(Ctx *c, const double *r, double *z, CgDev *cg, bool init) {
    MgLevel &m = c->mg[0];
    Lv L = level_view(m);
    const int n = m.nx * m.ny;
    const float w = c->mg_omega, wc = c->mg_omega_c;
    if (c->mg_levels == 1) {
        k_mg_last<false><<<c->grid_stencil, kThreads, 0, c->stream>>>(L, r, m.x[0], nullptr, 1, wc, w, z, cg, init,
                                                                      c->partials, c->counter);
        c->launches++;
        return check_launch(c, "multigrid apply");
    }
    MgLevel &g = c->mg[1];
    k_mg_pre0<double><<<mg_grid(c, n), kThreads, 0, c->stream>>>(L, r, m.x[0], w);
    int cur = 0;
    for (int s = 1; s < c->mg_nu; s++, cur ^= 1)
        k_mg_sweep<double><<<mg_grid(c, n), kThreads, 0, c->stream>>>(L, r, m.x[cur], m.x[cur ^ 1], w);
    k_mg_restrict<double><<<mg_grid(c, (long long)g.nx * g.ny), kThreads, 0, c->stream>>>(L, r, m.x[cur], g.nx, g.ny,
                                                                                         g.b);
    c->launches += 1 + c->mg_nu;
    vcycle(c, 1);
    if (c->mg_nu == 1) {
        k_mg_last<true><<<c->grid_stencil, kThreads, 0, c->stream>>>(L, r, m.x[cur], g.x[0], g.nx, wc, w, z, cg, init,
                                                                     c->partials, c->counter);
        c->launches++;
    } else {
        k_mg_prolong_sweep<double><<<mg_grid(c, n), kThreads, 0, c->stream>>>(L, r, m.x[cur], g.x[0], g.nx, wc, w,
                                                                              m.x[cur ^ 1]);
        cur ^= 1;
        for (int s = 2; s < c->mg_nu; s++, cur ^= 1)
            k_mg_sweep<double><<<mg_grid(c, n), kThreads, 0, c->stream>>>(L, r, m.x[cur], m.x[cur ^ 1], w);
        k_mg_last<false><<<c->grid_stencil, kThreads, 0, c->stream>>>(L, r, m.x[cur], nullptr, 1, wc, w, z, cg, init,
                                                                      c->partials, c->counter);
        c->launches += c->mg_nu;
    }
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

} // namespace shk
