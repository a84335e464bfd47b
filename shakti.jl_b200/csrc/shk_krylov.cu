// shk_krylov.cu -- matrix-free operator, preconditioned CG, Chebyshev preconditioner, and the
// mixed-precision iterative-refinement form.
//
// CG follows Krylov.jl's cg! (v0.10.8, the reference's dependency; call site
// src/linear_solver.jl:921): warm start x0 = h, x accumulates the correction from zero, r = b - A x0,
// z = M^-1 r, p = z, gamma = r'z; per iteration Ap = A p, alpha = gamma/p'Ap, x += alpha p,
// r -= alpha Ap, z = M^-1 r, stop on sqrt(r'z) <= atol + rtol*sqrt(r0'z0), beta = gamma'/gamma,
// p = z + beta p; finally h = x + h.  All scalars stay on the device.
//
// One CG iteration is two kernels over the grid (Jacobi):
//   A: p_new = z + beta p_old (z = r/aP recomputed, also at the 4 neighbours), Ap = A p_new,
//      partial p'Ap  -> last block: alpha (or zero-curvature breakdown)
//   B: x += alpha p, r -= alpha Ap, z = r/aP, partial r'z and r'r -> last block: stop test, beta
// Algorithmic traffic per cell and iteration: A reads r, aP, p_old, aE, aN and writes p, Ap;
// B reads x, p, r, Ap, aP and writes x, r: 14 words (112 B in Float64, 56 B in Float32).
#include <algorithm>
#include <functional>
#include <cstdlib>
#include <type_traits>

#include <cuda_pipeline.h>
#include <cuda_runtime.h>
#include <float.h>
#include <stdio.h>
#include <string.h>

#include "shk_device.cuh"

namespace shk {

// ---------------------------------------------------------------------------------------------
// Stencil: stencil_matvec_kernel! (src/linear_solver.jl:616-633), subtraction order E, W, N, S.
// West/south couplings are the neighbour's east/north entries (exact symmetry of the assembly).
// ---------------------------------------------------------------------------------------------
template <typename T, typename F>
__device__ __forceinline__ T stencil_apply(const T *__restrict__ aP, const T *__restrict__ aE,
                                           const T *__restrict__ aN, int nx, int ny, int ix, int iy,
                                           size_t c, T xc, F val) {
    T y = aP[c] * xc;
    if (ix < nx - 1) y -= aE[c] * val(c + 1);
    if (ix > 0) y -= aE[c - 1] * val(c - 1);
    if (iy < ny - 1) y -= aN[c] * val(c + nx);
    if (iy > 0) y -= aN[c - nx] * val(c - nx);
    return y;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_matvec(int nx, int ny, const T *aP, const T *aE, const T *aN,
                                                     const T *x, T *y) {
    Tiles Tl(nx, ny);
    for (int t = blockIdx.x; t < Tl.ntiles; t += gridDim.x) {
        int ix, iy;
        Tl.cell(t, ix, iy);
        if (ix >= nx || iy >= ny) continue;
        size_t c = (size_t)ix + (size_t)iy * nx;
        y[c] = stencil_apply(aP, aE, aN, nx, ny, ix, iy, c, x[c], [&](size_t k) { return x[k]; });
    }
}

// ---------------------------------------------------------------------------------------------
// CG kernels.  T = double (plain form) or float (inner solve of the mixed form).
// ---------------------------------------------------------------------------------------------

// r = b - A x0 (x0 == nullptr: r = b), x = 0; JAC: partials r'z, r'r, b'b -> init finish;
// otherwise partials r'r, b'b are parked for the Chebyshev init pass.
// b'b is summed over the GROUNDED rows only when fmask (the uint8 mask) is given: the relative-
// residual rule measures ||b - A x|| (every row) against the rows whose unknown is a free head.  The
// OCEAN/LAND/OTHER_BASIN rows are identity rows holding a fixed head (of order 1e3 m), decoupled
// from the rest; counted in ||b|| they would loosen "1e-8" to about 1e-3 on the free rows.
template <typename T, bool JAC>
__device__ __forceinline__ void cg_init_body(Blk B, int nx, int ny, const T *aP, const T *aE, const T *aN,
                                             const double *x0, const T *b, T *r, T *x, CgDev *cg, double *partials,
                                             unsigned int *counter, const uint8_t *fmask) {
    Tiles Tl(nx, ny);
    double red[3] = {0.0, 0.0, 0.0};
    for (int t = B.id; t < Tl.ntiles; t += B.n) {
        int ix, iy;
        Tl.cell(t, ix, iy);
        if (ix >= nx || iy >= ny) continue;
        size_t c = (size_t)ix + (size_t)iy * nx;
        T bc = b[c];
        T rc;
        if (x0) {
            T ax = stencil_apply(aP, aE, aN, nx, ny, ix, iy, c, (T)x0[c], [&](size_t k) { return (T)x0[k]; });
            rc = (T)1 * bc + (T)(-1) * ax;
        } else {
            rc = bc;
        }
        r[c] = rc;
        x[c] = (T)0;
        if (JAC) {
            T zc = rc / aP[c];
            red[0] += (double)rc * (double)zc;
        }
        red[1] += (double)rc * (double)rc;
        if (!fmask || fmask[c] == M_GROUNDED) red[2] += (double)bc * (double)bc;
    }
    double out[3];
    if (grid_reduce<3, false>(B, red, partials, counter, out) && threadIdx.x == 0) {
        if (JAC) cg_init_finish(cg, out[0], out[1], out[2]);
        else {
            cg->rr = out[1];    // parked: squared norms, consumed by the Chebyshev init pass
            cg->bnorm = out[2];
        }
    }
}

template <typename T, bool JAC>
__global__ void __launch_bounds__(kThreads) k_cg_init(int nx, int ny, const T *aP, const T *aE, const T *aN,
                                                      const double *x0, const T *b, T *r, T *x, CgDev *cg,
                                                      double *partials, unsigned int *counter, const uint8_t *fmask) {
    cg_init_body<T, JAC>(grid_blk(), nx, ny, aP, aE, aN, x0, b, r, x, cg, partials, counter, fmask);
}

// A: p_new = z + beta*p_old (p_new = z on the first iteration), Ap = A p_new, partial p'Ap.
//
// One block owns a tile of kMarchX columns x TH rows and marches up the rows.  Input rows (r or
// z, aP, p_old, aE, aN, plus one halo column each side) stream into a shared-memory ring with
// cp.async, kRingRows - 2 rows ahead of use, so DRAM latency overlaps the arithmetic of earlier
// rows.  For input row k each thread forms p_k once (z = r/aP: one divide per cell) and the block
// then emits output row k-1, whose five stencil terms are all at hand: p at rows k-2, k-1, k in
// registers, p at columns x+-1 of row k-1 in a double-buffered shared row, and aE(x-1) in the ring.
// Subtraction order E, W, N, S as in stencil_matvec_kernel!.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src) {
    __pipeline_memcpy_async(dst, src, sizeof(T));
}

// LAPL (Float32 operator of the mixed form): the matvec is applied in Laplacian form
// y = dP p + aE (p - pE) + aW (p - pW) + aN (p - pN) + aS (p - pS), with dP = aP - (aE+aW+aN+aS)
// the diagonal excess computed in Float64 and rounded once.  Storing edge conductances and the
// excess (rather than aP and the couplings) keeps the rounded operator accurate entry by entry
// for this nearly singular M-matrix, whatever its condition number.
template <typename T, bool JAC, bool LAPL>
__device__ __forceinline__ void cg_A_body(Blk B, int nx, int ny, int TH, const T *__restrict__ aP,
                                          const T *__restrict__ aE, const T *__restrict__ aN,
                                          const T *__restrict__ r, const T *__restrict__ zbuf,
                                          const T *__restrict__ p_old, T *__restrict__ p_new, T *__restrict__ Ap,
                                          CgDev *cg, double *partials, unsigned int *counter, double eps_curv,
                                          const T *__restrict__ dP) {
    const CgView cv = block_cg_view(cg);
    if (cv.done) return;
    constexpr int R = kRingRows, W = kMarchX + 2;
    enum { IR = 0, IP = 1, IO = 2, IE = 3, IN = 4, ID = 5, NA = LAPL ? 6 : 5 };
    __shared__ __align__(16) T ring[R][NA][W];
    __shared__ T prow[2][W];
    const bool first = cv.first != 0;
    const T beta = (T)cv.beta;
    const int tiles_x = (nx + kMarchX - 1) / kMarchX;
    const int x0 = (B.id % tiles_x) * kMarchX, y0 = (B.id / tiles_x) * TH;
    const int tid = threadIdx.x, ix = x0 + tid;
    const bool inx = ix < nx;
    const int y1 = min(y0 + TH, ny);
    const int kfirst = y0 - 1, klast = y1;            // input rows kfirst..klast (clipped below)
    const T *src_r = JAC ? r : zbuf;
    // issue the copies of input row q into its ring slot (empty group when out of range)
    auto issue = [&](int q) {
        if (q >= 0 && q < ny && q <= klast) {
            const int slot = (q - kfirst) % R;
            const size_t rowoff = (size_t)q * nx;
            if (inx) {
                const size_t c = rowoff + ix;
                cp_async_elem(&ring[slot][IR][tid + 1], src_r + c);
                cp_async_elem(&ring[slot][IP][tid + 1], aP + c);
                if (!first) cp_async_elem(&ring[slot][IO][tid + 1], p_old + c);
                cp_async_elem(&ring[slot][IE][tid + 1], aE + c);
                cp_async_elem(&ring[slot][IN][tid + 1], aN + c);
                if (LAPL) cp_async_elem(&ring[slot][ID][tid + 1], dP + c);
            }
            if (tid == 0 && x0 > 0) {
                const size_t c = rowoff + x0 - 1;
                cp_async_elem(&ring[slot][IR][0], src_r + c);
                if (JAC) cp_async_elem(&ring[slot][IP][0], aP + c);
                if (!first) cp_async_elem(&ring[slot][IO][0], p_old + c);
                cp_async_elem(&ring[slot][IE][0], aE + c);
            }
            if (tid == kMarchX - 1 && x0 + kMarchX < nx) {
                const size_t c = rowoff + x0 + kMarchX;
                cp_async_elem(&ring[slot][IR][W - 1], src_r + c);
                if (JAC) cp_async_elem(&ring[slot][IP][W - 1], aP + c);
                if (!first) cp_async_elem(&ring[slot][IO][W - 1], p_old + c);
            }
        }
        __pipeline_commit();
    };
    auto pform = [&](int slot, int j) -> T {
        T z = JAC ? ring[slot][IR][j] / ring[slot][IP][j] : ring[slot][IR][j];
        return first ? z : z + beta * ring[slot][IO][j];
    };
    for (int q = kfirst; q < kfirst + R - 2; q++) issue(q);
    T p_m2 = (T)0, p_m1 = (T)0, aN_m2 = (T)0, aN_m1 = (T)0, aP_m1 = (T)0, aE_m1 = (T)0, dP_m1 = (T)0;
    double acc = 0.0;
    for (int k = kfirst; k <= klast; k++) {
        __pipeline_wait_prior(R - 3);
        __syncthreads();
        issue(k + R - 2);  // the slot of row k-2 is free: every thread finished row k-2 before the barrier
        const bool valid_k = k >= 0 && k < ny;
        const int slot = (k - kfirst) % R;
        T p_k = (T)0, aN_k = (T)0, aP_k = (T)0, aE_k = (T)0, dP_k = (T)0;
        T *pr = prow[k & 1];
        if (valid_k) {
            if (inx) {
                p_k = pform(slot, tid + 1);
                aP_k = ring[slot][IP][tid + 1];
                aE_k = ring[slot][IE][tid + 1];
                aN_k = ring[slot][IN][tid + 1];
                if (LAPL) dP_k = ring[slot][ID][tid + 1];
            }
            pr[tid + 1] = p_k;
            if (tid == 0) pr[0] = x0 > 0 ? pform(slot, 0) : (T)0;
            if (tid == kMarchX - 1) pr[W - 1] = (x0 + kMarchX < nx) ? pform(slot, W - 1) : (T)0;
        }
        // Output row k-1 reads only data published before this iteration's barrier (its p row and
        // its ring slot were written in earlier iterations), so no second barrier is needed here.
        const int iy = k - 1;  // output row
        if (iy >= y0 && iy < y1 && inx) {
            const T *pm = prow[iy & 1];
            const int sm1 = (iy - kfirst) % R;
            T y;
            if (LAPL) {
                y = dP_m1 * p_m1;
                if (ix < nx - 1) y += aE_m1 * (p_m1 - pm[tid + 2]);
                if (ix > 0) y += ring[sm1][IE][tid] * (p_m1 - pm[tid]);
                if (iy + 1 < ny) y += aN_m1 * (p_m1 - p_k);
                if (iy > 0) y += aN_m2 * (p_m1 - p_m2);
            } else {
                y = aP_m1 * p_m1;
                if (ix < nx - 1) y -= aE_m1 * pm[tid + 2];
                if (ix > 0) y -= ring[sm1][IE][tid] * pm[tid];
                if (iy + 1 < ny) y -= aN_m1 * p_k;
                if (iy > 0) y -= aN_m2 * p_m2;
            }
            const size_t c = (size_t)iy * nx + ix;
            p_new[c] = p_m1;
            Ap[c] = y;
            acc += (double)p_m1 * (double)y;
        }
        p_m2 = p_m1;
        p_m1 = p_k;
        aN_m2 = aN_m1;
        aN_m1 = aN_k;
        aP_m1 = aP_k;
        aE_m1 = aE_k;
        dP_m1 = dP_k;
    }
    __pipeline_wait_prior(0);
    double red[1] = {acc}, out[1];
    if (grid_reduce<1, false>(B, red, partials, counter, out) && threadIdx.x == 0) {
        const double pAp = out[0];
        cg->pAp = pAp;
        const double lim = eps_curv * cg->pNorm2;
        if ((pAp <= lim && fabs(pAp) <= lim) || isnan(pAp)) {
            cg->done = 1;
            cg->status = SHK_BREAKDOWN;
        } else {
            cg->alpha = cg->gamma / pAp;
        }
    }
}

template <typename T, bool JAC, bool LAPL = false>
__global__ void __launch_bounds__(kMarchX, 6) k_cg_A(int nx, int ny, int TH, const T *__restrict__ aP,
                                                  const T *__restrict__ aE, const T *__restrict__ aN,
                                                  const T *__restrict__ r, const T *__restrict__ zbuf,
                                                  const T *__restrict__ p_old, T *__restrict__ p_new,
                                                  T *__restrict__ Ap, CgDev *cg, double *partials,
                                                  unsigned int *counter, double eps_curv,
                                                  const T *__restrict__ dP = nullptr) {
    cg_A_body<T, JAC, LAPL>(grid_blk(), nx, ny, TH, aP, aE, aN, r, zbuf, p_old, p_new, Ap, cg, partials, counter,
                            eps_curv, dP);
}

// 16-byte vectors for the streaming kernels.
template <typename T> struct Vec16;
template <> struct Vec16<double> {
    using V = double2;
    static constexpr int W = 2;
    __device__ static inline double get(const V &v, int k) { return k == 0 ? v.x : v.y; }
    __device__ static inline void set(V &v, int k, double a) { if (k == 0) v.x = a; else v.y = a; }
};
template <> struct Vec16<float> {
    using V = float4;
    static constexpr int W = 4;
    __device__ static inline float get(const V &v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }
    __device__ static inline void set(V &v, int k, float a) {
        if (k == 0) v.x = a; else if (k == 1) v.y = a; else if (k == 2) v.z = a; else v.w = a;
    }
};

// B: x += alpha p, r -= alpha Ap; JAC: z = r/aP, partials r'z, r'r -> stop test.
// 16-byte loads, kUnrollB vectors in flight per thread; scalar tail for n not a multiple of the
// vector width.
template <typename T, bool JAC>
__device__ __forceinline__ void cg_B_body(Blk B, int n, const T *__restrict__ aP, const T *__restrict__ p,
                                          const T *__restrict__ Ap, T *__restrict__ x, T *__restrict__ r, CgDev *cg,
                                          double *partials, unsigned int *counter) {
    const CgView cv = block_cg_view(cg);
    if (cv.done) return;
    using VT = Vec16<T>;
    using V = typename VT::V;
    constexpr int W = VT::W;
    const T alpha = (T)cv.alpha;
    double rz = 0.0, rr = 0.0;
    const int nv = n / W;
    const V *aPv = reinterpret_cast<const V *>(aP), *pv = reinterpret_cast<const V *>(p),
            *Apv = reinterpret_cast<const V *>(Ap);
    V *xv = reinterpret_cast<V *>(x), *rv = reinterpret_cast<V *>(r);
    const int stride = B.n * blockDim.x;
    for (int base = B.id * blockDim.x + threadIdx.x; base < nv; base += stride * kUnrollB) {
        V X[kUnrollB], P[kUnrollB], R[kUnrollB], AP[kUnrollB], D[kUnrollB];
#pragma unroll
        for (int u = 0; u < kUnrollB; u++) {
            int i = base + u * stride;
            if (i < nv) {
                X[u] = xv[i];
                P[u] = pv[i];
                R[u] = rv[i];
                AP[u] = Apv[i];
                if (JAC) D[u] = aPv[i];
            }
        }
#pragma unroll
        for (int u = 0; u < kUnrollB; u++) {
            int i = base + u * stride;
            if (i < nv) {
#pragma unroll
                for (int k = 0; k < W; k++) {
                    T xi = VT::get(X[u], k) + alpha * VT::get(P[u], k);
                    T ri = VT::get(R[u], k) + (-alpha) * VT::get(AP[u], k);
                    VT::set(X[u], k, xi);
                    VT::set(R[u], k, ri);
                    if (JAC) {
                        T zi = ri / VT::get(D[u], k);
                        rz += (double)ri * (double)zi;
                        rr += (double)ri * (double)ri;
                    }
                }
                xv[i] = X[u];
                rv[i] = R[u];
            }
        }
    }
    for (int i = nv * W + B.id * blockDim.x + threadIdx.x; i < n; i += stride) {
        T xi = x[i] + alpha * p[i];
        T ri = r[i] + (-alpha) * Ap[i];
        x[i] = xi;
        r[i] = ri;
        if (JAC) {
            T zi = ri / aP[i];
            rz += (double)ri * (double)zi;
            rr += (double)ri * (double)ri;
        }
    }
    if (JAC) {
        double red[2] = {rz, rr}, out[2];
        if (grid_reduce<2, false>(B, red, partials, counter, out) && threadIdx.x == 0)
            cg_iter_finish(cg, out[0], out[1]);
    }
}

template <typename T, bool JAC>
__global__ void __launch_bounds__(kThreads) k_cg_B(int n, const T *__restrict__ aP, const T *__restrict__ p,
                                                   const T *__restrict__ Ap, T *__restrict__ x, T *__restrict__ r,
                                                   CgDev *cg, double *partials, unsigned int *counter) {
    cg_B_body<T, JAC>(grid_blk(), n, aP, p, Ap, x, r, cg, partials, counter);
}

// h = x + h (Krylov adds the warm start back at the end; then s.h .= x).
__device__ __forceinline__ void cg_finish_body(Blk B, int n, const double *x, double *h) {
    for (int i = B.id * blockDim.x + threadIdx.x; i < n; i += B.n * blockDim.x) h[i] = x[i] + h[i];
}
__global__ void k_cg_finish(int n, const double *x, double *h) { cg_finish_body(grid_blk(), n, x, h); }
// h = x + x0 for a warm start x0 other than h
__global__ void k_cg_finish_from(int n, const double *x, const double *x0, double *h) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) h[i] = x[i] + x0[i];
}

// One damped Jacobi sweep on the assembled system: xo = xi + omega (b - A xi) / aP
__global__ void __launch_bounds__(kThreads) k_jacobi_sweep(int nx, int ny, const double *aP, const double *aE,
                                                           const double *aN, const double *b, const double *xi,
                                                           double *xo, double omega) {
    Tiles Tl(nx, ny);
    for (int t = blockIdx.x; t < Tl.ntiles; t += gridDim.x) {
        int ix, iy;
        Tl.cell(t, ix, iy);
        if (ix >= nx || iy >= ny) continue;
        size_t c = (size_t)ix + (size_t)iy * nx;
        double ax = stencil_apply(aP, aE, aN, nx, ny, ix, iy, c, xi[c], [&](size_t k) { return xi[k]; });
        xo[c] = xi[c] + omega * (b[c] - ax) / aP[c];
    }
}

int jacobi_smooth(Ctx *c, double *x, double *tmp, int sweeps, double omega) {
    for (int k = 0; k < sweeps; k++) {
        const double *xi = (k & 1) ? tmp : x;
        double *xo = (k & 1) ? x : tmp;
        k_jacobi_sweep<<<c->grid_stencil, kThreads, 0, c->stream>>>(c->nx, c->ny, c->aP, c->aE, c->aN, c->rhs, xi, xo,
                                                                    omega);
        c->launches++;
    }
    if (sweeps & 1)
        cudaMemcpyAsync(x, tmp, (size_t)c->nx * c->ny * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    return check_launch(c, "jacobi smoothing");
}

// ||rhs - A x||^2 (every row) and ||rhs||^2 over the GROUNDED rows of the assembled system for a
// given x (Float64)
__global__ void __launch_bounds__(kThreads) k_residual_of(int nx, int ny, const double *aP, const double *aE,
                                                          const double *aN, const double *x, const double *b,
                                                          DevScalars *dv, double *partials, unsigned int *counter,
                                                          const uint8_t *fmask) {
    Tiles Tl(nx, ny);
    double red[2] = {0.0, 0.0};
    for (int t = blockIdx.x; t < Tl.ntiles; t += gridDim.x) {
        int ix, iy;
        Tl.cell(t, ix, iy);
        if (ix >= nx || iy >= ny) continue;
        size_t c = (size_t)ix + (size_t)iy * nx;
        double ax = stencil_apply(aP, aE, aN, nx, ny, ix, iy, c, x[c], [&](size_t k) { return x[k]; });
        double rc = b[c] - ax;
        red[0] += rc * rc;
        if (!fmask || fmask[c] == M_GROUNDED) red[1] += b[c] * b[c];
    }
    double out[2];
    if (grid_reduce<2, false>(red, partials, counter, out) && threadIdx.x == 0) {
        dv->ref_rr = out[0];
        dv->ref_bb = out[1];
    }
}

// ---------------------------------------------------------------------------------------------
// Chebyshev preconditioner ldiv! (src/preconditioner.jl:239-267): y ~ A^-1 x by the degree-d
// Chebyshev semi-iteration on D^-1 A.  The reference's final matvec and residual update do not
// reach y, so they are skipped (degree-1 matvecs per application, identical y).
//   FIRST: pc = x/aP (and at neighbours), y = 0 + a1 pc, rc = pc - a1 (A pc)/aP
//   MID  : pc' = rc + b_k pc, y += a_k pc', rc' = rc - a_k (A pc')/aP
//   LAST : pc' = rc + b_k pc, y += a_k pc'  (+ CG dot r'z and stop test when inside CG)
//   ONLY : degree 1: y = 0 + a1 x/aP
// ---------------------------------------------------------------------------------------------
enum ChebMode { CH_FIRST = 0, CH_MID = 1, CH_LAST = 2, CH_ONLY = 3 };
enum ChebCg { CG_NONE = 0, CG_INIT = 1, CG_ITER = 2 };

template <typename T, int MODE, int CGM>
__global__ void __launch_bounds__(kThreads) k_cheb(int nx, int ny, const T *__restrict__ aP,
                                                   const T *__restrict__ aE, const T *__restrict__ aN,
                                                   const T *__restrict__ xin, const T *__restrict__ rc_old,
                                                   const T *__restrict__ pc_old, T *__restrict__ rc_new,
                                                   T *__restrict__ pc_new, T *__restrict__ y, int k,
                                                   const ChebDev *ch, CgDev *cg, double *partials,
                                                   unsigned int *counter) {
    if (CGM != CG_NONE && block_cg_done(&cg->done)) return;
    const T a = (T)ch->calpha[k];
    const T bt = (T)ch->cbeta[k];
    Tiles Tl(nx, ny);
    double red[2] = {0.0, 0.0};
    for (int t = blockIdx.x; t < Tl.ntiles; t += gridDim.x) {
        int ix, iy;
        Tl.cell(t, ix, iy);
        if (ix >= nx || iy >= ny) continue;
        size_t c = (size_t)ix + (size_t)iy * nx;
        T yc;
        if (MODE == CH_FIRST) {
            auto pv = [&](size_t q) -> T { return xin[q] / aP[q]; };
            T pc = pv(c);
            yc = (T)0 + a * pc;
            T apc = stencil_apply(aP, aE, aN, nx, ny, ix, iy, c, pc, pv) / aP[c];
            pc_new[c] = pc;
            rc_new[c] = pc - a * apc;
            y[c] = yc;
        } else if (MODE == CH_MID) {
            auto pv = [&](size_t q) -> T { return rc_old[q] + bt * pc_old[q]; };
            T pc = pv(c);
            yc = y[c] + a * pc;
            T apc = stencil_apply(aP, aE, aN, nx, ny, ix, iy, c, pc, pv) / aP[c];
            pc_new[c] = pc;
            rc_new[c] = rc_old[c] - a * apc;
            y[c] = yc;
        } else if (MODE == CH_LAST) {
            T pc = rc_old[c] + bt * pc_old[c];
            yc = y[c] + a * pc;
            y[c] = yc;
        } else {
            yc = (T)0 + a * (xin[c] / aP[c]);
            y[c] = yc;
        }
        if (CGM != CG_NONE && (MODE == CH_LAST || MODE == CH_ONLY)) {
            T rcv = xin[c];
            red[0] += (double)rcv * (double)yc;
            red[1] += (double)rcv * (double)rcv;
        }
    }
    if (CGM != CG_NONE && (MODE == CH_LAST || MODE == CH_ONLY)) {
        double out[2];
        if (grid_reduce<2, false>(red, partials, counter, out) && threadIdx.x == 0) {
            if (CGM == CG_INIT) cg_init_finish(cg, out[0], cg->rr, cg->bnorm);
            else cg_iter_finish(cg, out[0], out[1]);
        }
    }
}

// Chebyshev per-step coefficients from the bounds (src/preconditioner.jl:241-263).
__device__ void cheb_tables(ChebDev *ch) {
    const double d_mid = (ch->lam_max + ch->lam_min) / 2;
    const double c_rad = (ch->lam_max - ch->lam_min) / 2;
    double alpha = 1.0 / d_mid;
    ch->calpha[1] = alpha;
    ch->cbeta[1] = 0.0;
    double alpha_prev = alpha;
    for (int k = 2; k <= kMaxChebDegree; k++) {
        double t = c_rad * alpha_prev / 2;
        double beta = t * t;
        alpha = 1.0 / (d_mid - beta / alpha_prev);
        ch->calpha[k] = alpha;
        ch->cbeta[k] = beta;
        alpha_prev = alpha;
    }
}

__global__ void k_cheb_set_bounds(ChebDev *ch, double lmin, double lmax) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        ch->lam_min = lmin;
        ch->lam_max = lmax;
        cheb_tables(ch);
    }
}

// Sturm count of eigenvalues below x for SymTridiagonal(d, e).
__device__ int sturm(int m, const double *d, const double *e, double x) {
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

// estimate_eigenvalue_bounds tail + update_chebyshev_bounds! validity/fallback
// (src/preconditioner.jl:115-133, 219-230).  LAPACK's eigvals(SymTridiagonal) is replaced by
// bisection on the Sturm count for the two extreme eigenvalues (the only ones used).
__device__ void cheb_finish_estimate(ChebDev *ch, int m) {
    double d[kMaxChebSteps], e[kMaxChebSteps];
    d[0] = 1 / ch->alphas[0];
    for (int k = 1; k < m; k++) d[k] = 1 / ch->alphas[k] + ch->betas[k - 1] / ch->alphas[k - 1];
    for (int k = 0; k < m - 1; k++) e[k] = sqrt(ch->betas[k]) / ch->alphas[k];
    bool finite = true;
    for (int k = 0; k < m; k++) finite = finite && isfinite(d[k]);
    for (int k = 0; k < m - 1; k++) finite = finite && isfinite(e[k]);
    double lmin = __longlong_as_double(0x7ff8000000000000LL), lmax = lmin;
    if (finite) {
        double lo = INFINITY, hi = -INFINITY;
        for (int i = 0; i < m; i++) {
            double rad = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < m ? fabs(e[i]) : 0.0);
            lo = fmin(lo, d[i] - rad);
            hi = fmax(hi, d[i] + rad);
        }
        double span = fmax(fabs(lo), fabs(hi));
        lo -= DBL_EPSILON * span + DBL_MIN;
        hi += DBL_EPSILON * span + DBL_MIN;
        double a = lo, b = hi;
        for (int it = 0; it < 200; it++) {
            double mid = 0.5 * (a + b);
            if (mid == a || mid == b) break;
            if (sturm(m, d, e, mid) >= 1) b = mid; else a = mid;
        }
        double rmin = 0.5 * (a + b);
        a = lo;
        b = hi;
        for (int it = 0; it < 200; it++) {
            double mid = 0.5 * (a + b);
            if (mid == a || mid == b) break;
            if (sturm(m, d, e, mid) >= m) b = mid; else a = mid;
        }
        double rmax = 0.5 * (a + b);
        lmin = rmin * 0.9;
        lmax = rmax * 1.1;
    }
    ch->est_min = lmin;
    ch->est_max = lmax;
    const bool ok = isfinite(lmin) && isfinite(lmax) && lmin > 0 && lmax > lmin;
    ch->adopted = ok;
    if (ok) {
        ch->lam_min = lmin;
        ch->lam_max = lmax;
    }
    cheb_tables(ch);
}

// Lanczos-from-CG estimate (src/preconditioner.jl:89-113), step k of nsteps:
// A: p = rhs (k == 0) or r + beta_{k-1} p_old; Ap = (A p)/aP; alpha_k = gamma/p'Ap.
template <bool FIRST>
__global__ void __launch_bounds__(kThreads) k_est_A(int nx, int ny, const double *aP, const double *aE,
                                                    const double *aN, const double *rhs, const double *r,
                                                    const double *p_old, double *p_new, double *Ap, int k,
                                                    int nsteps, ChebDev *ch, double *partials,
                                                    unsigned int *counter) {
    const double beta = FIRST ? 0.0 : ch->betas[k - 1];
    auto pv = [&](size_t q) -> double { return FIRST ? rhs[q] : r[q] + beta * p_old[q]; };
    Tiles Tl(nx, ny);
    double red[2] = {0.0, 0.0};
    for (int t = blockIdx.x; t < Tl.ntiles; t += gridDim.x) {
        int ix, iy;
        Tl.cell(t, ix, iy);
        if (ix >= nx || iy >= ny) continue;
        size_t c = (size_t)ix + (size_t)iy * nx;
        double pc = pv(c);
        double apc = stencil_apply(aP, aE, aN, nx, ny, ix, iy, c, pc, pv) / aP[c];
        p_new[c] = pc;
        Ap[c] = apc;
        red[0] += pc * apc;
        if (FIRST) red[1] += pc * pc;
    }
    double out[2];
    if (grid_reduce<2, false>(red, partials, counter, out) && threadIdx.x == 0) {
        if (FIRST) ch->gamma = out[1];
        ch->alphas[k] = ch->gamma / out[0];
        if (k == nsteps - 1) cheb_finish_estimate(ch, nsteps);
    }
}

// B: r = (rhs on k == 0) r - alpha_k Ap; beta_k = r'r/gamma.
template <bool FIRST>
__global__ void __launch_bounds__(kThreads) k_est_B(int n, const double *rhs, double *r, const double *Ap, int k,
                                                    ChebDev *ch, double *partials, unsigned int *counter) {
    const double a = ch->alphas[k];
    double red[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ri = (FIRST ? rhs[i] : r[i]) - a * Ap[i];
        r[i] = ri;
        red[0] += ri * ri;
    }
    double out[1];
    if (grid_reduce<1, false>(red, partials, counter, out) && threadIdx.x == 0) {
        ch->betas[k] = out[0] / ch->gamma;
        ch->gamma = out[0];
    }
}

// ---------------------------------------------------------------------------------------------
// Mixed precision helpers
// ---------------------------------------------------------------------------------------------
// Float32 operator of the mixed form: aP (Jacobi scaling), aE, aN and the diagonal excess
// dP = aP - (aE + aW + aN + aS) evaluated in Float64 before rounding.
__global__ void k_to_float_lapl(int nx, int ny, const double *aP, const double *aE, const double *aN, float *fP,
                                float *fE, float *fN, float *fD) {
    const int n = nx * ny;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int ix = i % nx, iy = i / nx;
        const double e = aE[i], w = ix > 0 ? aE[i - 1] : 0.0, no = aN[i], so = iy > 0 ? aN[i - nx] : 0.0;
        fP[i] = (float)aP[i];
        fE[i] = (float)e;
        fN[i] = (float)no;
        fD[i] = (float)(aP[i] - (e + w + no + so));
    }
}

// r32 = float(b - A h) with Float64 operator; partials ||r||^2 (every row), ||b||^2 (GROUNDED
// rows) of the outer residual.
__global__ void __launch_bounds__(kThreads) k_outer_residual(int nx, int ny, const double *aP, const double *aE,
                                                             const double *aN, const double *h, const double *b,
                                                             float *r32, DevScalars *dv, double *partials,
                                                             unsigned int *counter, const uint8_t *fmask) {
    Tiles Tl(nx, ny);
    double red[2] = {0.0, 0.0};
    for (int t = blockIdx.x; t < Tl.ntiles; t += gridDim.x) {
        int ix, iy;
        Tl.cell(t, ix, iy);
        if (ix >= nx || iy >= ny) continue;
        size_t c = (size_t)ix + (size_t)iy * nx;
        double ax = stencil_apply(aP, aE, aN, nx, ny, ix, iy, c, h[c], [&](size_t k) { return h[k]; });
        double rc = b[c] - ax;
        r32[c] = (float)rc;
        red[0] += rc * rc;
        if (!fmask || fmask[c] == M_GROUNDED) red[1] += b[c] * b[c];
    }
    double out[2];
    if (grid_reduce<2, false>(red, partials, counter, out) && threadIdx.x == 0) {
        dv->ref_rr = out[0];
        dv->ref_bb = out[1];
    }
}

__global__ void k_refine_update(int n, const float *d, double *h) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) h[i] += (double)d[i];
}

// ---------------------------------------------------------------------------------------------
// Host drivers
// ---------------------------------------------------------------------------------------------
static int flat_grid(Ctx *c, long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    long long cap = (long long)c->grid_stencil;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// Blocks for the 16-byte-vector streaming kernels: enough for kUnrollB vectors per thread, at
// most the resident capacity (148 SMs x 8 blocks of 256 threads).
static int stream_grid(Ctx *c, long long n, size_t elem) {
    long long vec = (long long)(16 / elem);
    long long per_block = (long long)kThreads * kUnrollB * vec;
    long long b = (n + per_block - 1) / per_block;
    long long cap = (long long)c->num_sms * 8;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// ||rhs - A x||_2 and ||rhs||_2 of the assembled system (x: the current h when null; Float64).
int residual_norms(Ctx *c, const double *x, double *rnorm, double *bnorm) {
    k_residual_of<<<c->grid_stencil, kThreads, 0, c->stream>>>(c->nx, c->ny, c->aP, c->aE, c->aN, x ? x : c->st.h,
                                                              c->rhs, c->dev, c->partials, c->counter, c->mask8);
    c->launches++;
    int rc = check_launch(c, "residual norm");
    if (rc) return rc;
    if ((rc = read_scalars(c))) return rc;
    if (rnorm) *rnorm = sqrt(c->host_dev->ref_rr);
    if (bnorm) *bnorm = sqrt(c->host_dev->ref_bb);
    return SHK_OK;
}

// Control scalars move between the device scalar block and its pinned host mirror through a
// one-block kernel that reads or writes the mapped host memory, not through a copy engine: a large
// transfer the caller has queued on a copy engine (a field on its way to the host while the solve
// runs) would otherwise hold every small control copy -- and the host loop waiting on it -- behind
// it.  Falls back to cudaMemcpyAsync for host memory outside the mirror.
__global__ void k_words(const unsigned long long *src, unsigned long long *dst, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

int move_scalars(Ctx *c, void *dst, const void *src, size_t bytes, bool to_host) {
    const char *h0 = (const char *)c->host_dev, *hp = (const char *)(to_host ? dst : src);
    const bool mirrored = c->host_dev_d && hp >= h0 && hp + bytes <= h0 + sizeof(DevScalars) && bytes % 8 == 0 &&
                          ((uintptr_t)dst % 8) == 0 && ((uintptr_t)src % 8) == 0;
    if (mirrored) {
        void *alias = (char *)c->host_dev_d + (hp - h0);
        const void *s = to_host ? src : alias;
        void *d = to_host ? alias : dst;
        k_words<<<1, 64, 0, c->stream>>>((const unsigned long long *)s, (unsigned long long *)d, (int)(bytes / 8));
        c->launches++;
        return check_launch(c, "control scalars");
    }
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, to_host ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice,
                                    c->stream);
    return e == cudaSuccess ? SHK_OK : check_cuda(c, e, "control scalars");
}

int read_scalars(Ctx *c) {
    if (int rc = move_scalars(c, c->host_dev, c->dev, sizeof(DevScalars), true)) return rc;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "stream sync");
}

static int read_cg_flags(Ctx *c, CgDev *dst, const CgDev *src) {
    if (int rc = move_scalars(c, dst, src, sizeof(CgDev), true)) return rc;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "stream sync");
}

int launch_matvec(Ctx *c, const double *x, double *y) {
    k_matvec<double><<<c->grid_stencil, kThreads, 0, c->stream>>>(c->nx, c->ny, c->aP, c->aE, c->aN, x, y);
    c->launches++;
    return check_launch(c, "k_matvec");
}

int run_chebyshev_bounds(Ctx *c, int nsteps, const double *rhs) {
    if (nsteps < 2 || nsteps > kMaxChebSteps) return fail(c, SHK_BAD_ARG, "chebyshev nsteps must be in [2, 64]");
    const int nx = c->nx, ny = c->ny, n = nx * ny;
    ChebDev *ch = &c->dev->cheb;
    for (int k = 0; k < nsteps; k++) {
        double *p_old = c->p[k & 1], *p_new = c->p[(k + 1) & 1];
        if (k == 0)
            k_est_A<true><<<c->grid_stencil, kThreads, 0, c->stream>>>(nx, ny, c->aP, c->aE, c->aN, rhs, c->r, p_old,
                                                                       p_new, c->Ap, k, nsteps, ch, c->partials,
                                                                       c->counter);
        else
            k_est_A<false><<<c->grid_stencil, kThreads, 0, c->stream>>>(nx, ny, c->aP, c->aE, c->aN, rhs, c->r, p_old,
                                                                        p_new, c->Ap, k, nsteps, ch, c->partials,
                                                                        c->counter);
        c->launches++;
        if (k < nsteps - 1) {
            if (k == 0)
                k_est_B<true><<<flat_grid(c, n), kThreads, 0, c->stream>>>(n, rhs, c->r, c->Ap, k, ch, c->partials,
                                                                            c->counter);
            else
                k_est_B<false><<<flat_grid(c, n), kThreads, 0, c->stream>>>(n, rhs, c->r, c->Ap, k, ch, c->partials,
                                                                             c->counter);
            c->launches++;
        }
    }
    return check_launch(c, "chebyshev bounds");
}

// Enqueue one Chebyshev application y = M^-1 xin (degree deg) in precision T.
template <typename T, int CGM>
static void enqueue_cheb(Ctx *c, int deg, const T *aP, const T *aE, const T *aN, const T *xin, T **cr, T **cp, T *y,
                         CgDev *cg) {
    const int nx = c->nx, ny = c->ny;
    const ChebDev *ch = &c->dev->cheb;
    if (deg == 1) {
        k_cheb<T, CH_ONLY, CGM><<<c->grid_stencil, kThreads, 0, c->stream>>>(
            nx, ny, aP, aE, aN, xin, nullptr, nullptr, nullptr, nullptr, y, 1, ch, cg, c->partials, c->counter);
        c->launches++;
        return;
    }
    k_cheb<T, CH_FIRST, CG_NONE == CGM ? CG_NONE : CGM><<<c->grid_stencil, kThreads, 0, c->stream>>>(
        nx, ny, aP, aE, aN, xin, nullptr, nullptr, cr[0], cp[0], y, 1, ch, cg, c->partials, c->counter);
    c->launches++;
    int cur = 0;
    for (int k = 2; k < deg; k++) {
        k_cheb<T, CH_MID, CGM><<<c->grid_stencil, kThreads, 0, c->stream>>>(
            nx, ny, aP, aE, aN, xin, cr[cur], cp[cur], cr[cur ^ 1], cp[cur ^ 1], y, k, ch, cg, c->partials, c->counter);
        c->launches++;
        cur ^= 1;
    }
    k_cheb<T, CH_LAST, CGM><<<c->grid_stencil, kThreads, 0, c->stream>>>(
        nx, ny, aP, aE, aN, xin, cr[cur], cp[cur], nullptr, nullptr, y, deg, ch, cg, c->partials, c->counter);
    c->launches++;
}

int cheb_set_bounds(Ctx *c, double lmin, double lmax) {
    k_cheb_set_bounds<<<1, 32, 0, c->stream>>>(&c->dev->cheb, lmin, lmax);
    c->launches++;
    return check_launch(c, "set chebyshev bounds");
}

int launch_chebyshev_apply_standalone(Ctx *c, int degree, const double *x, double *y) {
    if (degree < 1 || degree > kMaxChebDegree) return fail(c, SHK_BAD_ARG, "chebyshev degree must be in [1, 32]");
    enqueue_cheb<double, CG_NONE>(c, degree, c->aP, c->aE, c->aN, x, c->cr, c->cp, y, nullptr);
    return check_launch(c, "chebyshev apply");
}

// Condition of the device-side CG loop: another trip (two iterations) while the solve has not
// stopped, and never more than itmax/2 + 8 trips, so the loop ends whatever the flags say.
__global__ void k_cg_loop_cond(CgDev *cg, cudaGraphConditionalHandle h) {
    const unsigned int t = ++cg->trips;
    const bool more = !*(volatile int *)&cg->done && 2LL * (long long)t < cg->itmax + 16;
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

static CgDev make_cg_init(const shk_cg_opts *o, long long n, bool inner, double inner_rtol) {
    CgDev g;
    memset(&g, 0, sizeof(g));
    g.atol = inner ? 0.0 : o->atol;
    g.rtol = inner ? inner_rtol : o->rtol;
    g.itmax = o->itmax > 0 ? o->itmax : 2 * n;
    g.stop_rule = inner ? SHK_STOP_RELRES : o->stop_rule;
    g.done = 0;
    g.status = SHK_OK;
    g.first = 1;
    return g;
}

// One preconditioned CG solve in precision T on system (aP, aE, aN), b -> x (correction from x0).
// x0 (Float64, may be null) is the warm start used only for the initial residual.
template <typename T>
static int cg_core(Ctx *c, const shk_cg_opts *o, CgDev *cgd, CgDev *cgh, const T *aP, const T *aE, const T *aN,
                   const double *x0, const T *b, T *x, T *r, T *z, T **p, T *Ap, T **cr, T **cp, long *iters_out,
                   int p_parity = 0, const T *lapl = nullptr) {
    const int nx = c->nx, ny = c->ny, n = nx * ny;
    const bool jac = o->precond == SHK_PRECOND_JACOBI;
    const bool mg = o->precond == SHK_PRECOND_MULTIGRID;
    const int deg = o->cheb_degree;
    // z = M^-1 r for the non-Jacobi preconditioners (with the CG dot r'z fused into the last pass)
    auto apply_precond = [&](bool init) -> int {
        if constexpr (std::is_same<T, double>::value) {
            if (mg) return mg_apply(c, r, z, cgd, init);
        }
        if (init) enqueue_cheb<T, CG_INIT>(c, deg, aP, aE, aN, r, cr, cp, z, cgd);
        else enqueue_cheb<T, CG_ITER>(c, deg, aP, aE, aN, r, cr, cp, z, cgd);
        return SHK_OK;
    };
    const double eps_curv = sizeof(T) == 8 ? DBL_EPSILON : (double)FLT_EPSILON;
    if constexpr (std::is_same<T, double>::value) {
        if (jac && !lapl)  // tensor maps of the tile form, before any capture below
            if (int rc0 = cg_tma_prepare(c)) return rc0;
    }
    cgh->trips = 0;
    if (int rc0 = move_scalars(c, cgd, cgh, sizeof(CgDev), false)) return rc0;
    cudaError_t e = cudaSuccess;
    if (jac) {
        k_cg_init<T, true><<<c->grid_stencil, kThreads, 0, c->stream>>>(nx, ny, aP, aE, aN, x0, b, r, x, cgd, c->partials,
                                                                       c->counter, c->mask8);
        c->launches++;
    } else {
        k_cg_init<T, false><<<c->grid_stencil, kThreads, 0, c->stream>>>(nx, ny, aP, aE, aN, x0, b, r, x, cgd,
                                                                        c->partials, c->counter, c->mask8);
        c->launches++;
        int prc = apply_precond(true);
        if (prc) return prc;
    }
    int rc = check_launch(c, "cg init");
    if (rc) return rc;

    // One CG iteration: stencil + p update + p'Ap (k_cg_A), x/r update (k_cg_B), preconditioner.
    // Every kernel returns at once when the device-side stop flag is set.
    // Multigrid (tile form): k_cg_B's x/r update runs inside the V-cycle's first kernel, which
    // writes the new residual to the other of two buffers (r and r2 alternate with the p parity).
    bool fuse_update = false;
    if constexpr (std::is_same<T, double>::value) fuse_update = mg && mg_fuses_cg_update(c);
    auto enqueue_iteration = [&](int par) -> int {
        T *p_old = p[par], *p_new = p[par ^ 1];
        if constexpr (std::is_same<T, double>::value) {
            if (fuse_update && !jac && !lapl) {
                bool launched = false;
                int rc = mg_cg_matvec(c, par, aP, aE, aN, z, p_old, p_new, Ap, cgd, eps_curv, &launched);
                if (rc) return rc;
                if (launched) {
                    T *rb[2] = {r, c->r2};
                    c->launches += 1;
                    // x updated once per two iterations: the first of a pair (par == p_parity)
                    // leaves it pending, the second applies both directions' updates
                    return mg_apply_fused_update(c, rb[par], rb[par ^ 1], x, p_new, Ap, z, cgd, p_old,
                                                 !c->mg_pair_x ? 0 : (par == p_parity ? 1 : 2), par ^ 1);
                }
            }
        }
        if (jac && lapl) {
            k_cg_A<T, true, true><<<c->march_blocks, kMarchX, 0, c->stream>>>(
                nx, ny, c->march_th, aP, aE, aN, r, nullptr, p_old, p_new, Ap, cgd, c->partials, c->counter, eps_curv,
                lapl);
        } else if (jac) {
            bool launched = false;  // the TMA-staged tile form where the context's maps cover the buffers
            if constexpr (std::is_same<T, double>::value) {
                if (aP == c->aP && aE == c->aE && aN == c->aN) {
                    const int rc = cg_jac_matvec(c, par, r, p_old, p_new, Ap, cgd, eps_curv, &launched);
                    if (rc) return rc;
                }
            }
            if (!launched)
                k_cg_A<T, true><<<c->march_blocks, kMarchX, 0, c->stream>>>(nx, ny, c->march_th, aP, aE, aN, r,
                                                                           nullptr, p_old, p_new, Ap, cgd,
                                                                           c->partials, c->counter, eps_curv);
        } else if (lapl) {
            k_cg_A<T, false, true><<<c->march_blocks, kMarchX, 0, c->stream>>>(
                nx, ny, c->march_th, aP, aE, aN, r, z, p_old, p_new, Ap, cgd, c->partials, c->counter, eps_curv, lapl);
        } else {
            k_cg_A<T, false><<<c->march_blocks, kMarchX, 0, c->stream>>>(nx, ny, c->march_th, aP, aE, aN, r, z, p_old,
                                                                        p_new, Ap, cgd, c->partials, c->counter,
                                                                        eps_curv);
        }
        if constexpr (std::is_same<T, double>::value) {
            if (fuse_update) {
                T *rb[2] = {r, c->r2};
                c->launches += 1;
                return mg_apply_fused_update(c, rb[par], rb[par ^ 1], x, p_new, Ap, z, cgd);
            }
        }
        if (jac)
            k_cg_B<T, true><<<stream_grid(c, n, sizeof(T)), kThreads, 0, c->stream>>>(n, aP, p_new, Ap, x, r, cgd,
                                                                                      c->partials, c->counter);
        else
            k_cg_B<T, false><<<stream_grid(c, n, sizeof(T)), kThreads, 0, c->stream>>>(n, aP, p_new, Ap, x, r, cgd,
                                                                                       c->partials, c->counter);
        c->launches += 2;
        if (!jac) return apply_precond(false);
        return SHK_OK;
    };

    // a pending x update of the paired form, applied after the last iteration
    auto catch_up = [&]() -> int {
        if constexpr (std::is_same<T, double>::value) {
            if (fuse_update && !jac && !lapl) return mg_catch_up(c, x, cgd);
        }
        return SHK_OK;
    };
    // Graphs are keyed by everything that their kernel arguments depend on within one context.
    const long long key_base = ((long long)(lapl != nullptr) << 41) | ((long long)(sizeof(T) == 4) << 40) |
                               ((long long)o->precond << 32) | ((long long)deg << 8);
    // Records enqueue() on the context's private capture stream (the caller's stream may be the
    // legacy default stream, which cannot be captured), into *graph when `into`, else into a new
    // graph returned in *graph.  Nothing executes.  Returns the launches recorded, or -1.
    auto capture = [&](cudaGraph_t *graph, bool into, const std::function<int()> &enqueue) -> long long {
        cudaError_t ce = cudaSuccess;
        if (!c->cap_stream) ce = cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking);
        if (ce != cudaSuccess) return -1;
        ce = into ? cudaStreamBeginCaptureToGraph(c->cap_stream, *graph, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal)
                  : cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
        if (ce != cudaSuccess) return -1;
        const long long before = c->launches;
        cudaStream_t user = c->stream;
        c->stream = c->cap_stream;
        const int irc = enqueue();
        c->stream = user;
        cudaGraph_t g = nullptr;
        ce = cudaStreamEndCapture(c->cap_stream, &g);
        const long long recorded = c->launches - before;
        c->launches = before;
        if (ce != cudaSuccess || irc != SHK_OK) {
            if (g && !into) cudaGraphDestroy(g);
            cudaGetLastError();
            return -1;
        }
        if (!into) *graph = g;
        return recorded;
    };

    // Mode 2: the whole iteration loop as one graph.  A WHILE node runs a body of two iterations (the
    // search-direction buffers alternate within the body) and k_cg_loop_cond, which clears the
    // loop condition once the solve stops (or at the trip bound).  The host waits once per solve,
    // and no iteration is issued past the stop.
    if (c->graph_mode == 2 && !c->loop_disabled) {
        const long long key = key_base | (1LL << 42) | p_parity;
        Ctx::GraphSlot *slot = nullptr;
        for (auto &g : c->graphs)
            if (g.key == key) slot = &g;
        if (!slot) {
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            long long per_trip = -1;
            cudaGraphConditionalHandle handle;
            bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess &&
                      cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
            if (ok) {
                cudaGraphNodeParams np = {};
                np.type = cudaGraphNodeTypeConditional;
                np.conditional.handle = handle;
                np.conditional.type = cudaGraphCondTypeWhile;
                np.conditional.size = 1;
                cudaGraphNode_t node;
                ok = cudaGraphAddNode(&node, graph, nullptr, 0, &np) == cudaSuccess;
                if (ok) {
                    cudaGraph_t body = np.conditional.phGraph_out[0];
                    per_trip = capture(&body, true, [&]() -> int {
                        int rc2 = enqueue_iteration(p_parity);
                        if (!rc2) rc2 = enqueue_iteration(p_parity ^ 1);
                        if (rc2) return rc2;
                        k_cg_loop_cond<<<1, 1, 0, c->stream>>>(cgd, handle);
                        c->launches++;
                        return check_launch(c, "cg loop condition");
                    });
                    ok = per_trip > 0 && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
                }
            }
            if (graph) cudaGraphDestroy(graph);
            if (!ok) {
                cudaGetLastError();
                if (exec) cudaGraphExecDestroy(exec);
                c->loop_disabled = true;  // per-iteration graphs from now on
            } else {
                c->graphs.push_back({key, exec, per_trip});
                slot = &c->graphs.back();
            }
        }
        if (slot) {
            if ((rc = read_cg_flags(c, cgh, cgd))) return rc;
            if (!cgh->done) {
                e = cudaGraphLaunch(slot->exec, c->stream);
                if (e != cudaSuccess) return check_cuda(c, e, "cg loop graph launch");
                if ((rc = read_cg_flags(c, cgh, cgd))) return rc;
                c->launches += slot->launches * (long long)cgh->trips;
                if (!cgh->done) return fail(c, SHK_CUDA_ERROR, "cg device loop reached its trip bound before stopping");
            }
            if ((rc = catch_up())) return rc;
            if (iters_out) *iters_out = (long)cgh->iter;
            return SHK_OK;
        }
    }

    // Modes 0 and 1: batches of iterations issued by the host (8, 16, ... 256), the stop flag read
    // between batches; in mode 1 each iteration is one replay of a captured graph.
    long long enq = 0;
    int batch = 8;
    const int batch_max = 256;
    for (;;) {
        if ((rc = read_cg_flags(c, cgh, cgd))) return rc;
        if (cgh->done) break;
        for (int b2 = 0; b2 < batch; b2++, enq++) {
            const int par = (int)((enq + p_parity) & 1);
            if (c->graph_mode >= 1 && !c->graphs_disabled) {
                const long long key = key_base | par;
                cudaGraphExec_t exec = nullptr;
                for (auto &g : c->graphs)
                    if (g.key == key) {
                        exec = g.exec;
                        c->launches += g.launches;
                    }
                if (!exec) {
                    cudaGraph_t graph = nullptr;
                    const long long rec = capture(&graph, false, [&]() { return enqueue_iteration(par); });
                    if (rec < 0 || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
                        cudaGetLastError();
                        c->graphs_disabled = true;  // direct launches from now on
                        exec = nullptr;
                    } else {
                        c->graphs.push_back({key, exec, rec});
                        c->launches += rec;
                    }
                    if (graph) cudaGraphDestroy(graph);
                }
                if (exec) {
                    e = cudaGraphLaunch(exec, c->stream);
                    if (e != cudaSuccess) return check_cuda(c, e, "cg iteration graph launch");
                    continue;
                }
            }
            if ((rc = enqueue_iteration(par))) return rc;
        }
        if ((rc = check_launch(c, "cg iterations"))) return rc;
        if (batch < batch_max) batch *= 2;
        // The device stops at itmax; launches beyond it are no-ops.  If the device-side counters
        // ever stopped advancing, this bound still ends the loop.
        if (cgh->iter > cgh->itmax + 4 || enq > cgh->itmax + 2LL * batch_max + 8)
            return fail(c, SHK_CUDA_ERROR, "cg iteration accounting overran itmax");
    }
    if ((rc = catch_up())) return rc;
    if (iters_out) *iters_out = (long)cgh->iter;
    return SHK_OK;
}

int run_cg(Ctx *c, const shk_cg_opts *o, shk_cg_stats *st) {
    const int nx = c->nx, ny = c->ny, n = nx * ny;
    const double *ws = c->ws_x0;  // consumed by this solve (Float64 forms; ignored by the mixed form)
    c->ws_x0 = nullptr;
    if (o->precond != SHK_PRECOND_JACOBI && o->precond != SHK_PRECOND_CHEBYSHEV && o->precond != SHK_PRECOND_MULTIGRID)
        return fail(c, SHK_BAD_ARG, "unknown preconditioner");
    if (o->precond == SHK_PRECOND_MULTIGRID) {
        // the Float32 Laplacian-form operator of level 0 and the coarse levels (a hierarchy of two
        // or more levels builds level 0 inside its first coarsening pass)
        if (c->mg_levels <= 1) {
            k_to_float_lapl<<<flat_grid(c, n), kThreads, 0, c->stream>>>(nx, ny, c->aP, c->aE, c->aN, c->aP32,
                                                                         c->aE32, c->aN32, c->dP32);
            c->launches++;
        }
        int rc = mg_setup(c);
        if (rc) return rc;
    }
    if (o->precond == SHK_PRECOND_CHEBYSHEV) {
        if (o->cheb_degree < 1 || o->cheb_degree > kMaxChebDegree)
            return fail(c, SHK_BAD_ARG, "chebyshev_degree must be in [1, 32]");
        // _cg_precond! refreshes the bounds from this solve's rhs (src/linear_solver.jl:853-856)
        int rc = run_chebyshev_bounds(c, o->cheb_nsteps, c->rhs);
        if (rc) return rc;
    }
    shk_cg_stats s;
    memset(&s, 0, sizeof(s));
    if (o->precision == SHK_FP64) {
        CgDev *cgh = &c->host_dev->cg;
        *cgh = make_cg_init(o, n, false, 0.0);
        long it = 0;
        // warm start: the head, or a one-shot caller-provided guess (shk_set_cg_warm_start)
        const double *x0 = ws ? ws : c->st.h;
        int rc = cg_core<double>(c, o, &c->dev->cg, cgh, c->aP, c->aE, c->aN, x0, c->rhs, c->x, c->r, c->z, c->p,
                                 c->Ap, c->cr, c->cp, &it);
        if (rc) return rc;
        if (x0 == c->st.h)
            k_cg_finish<<<flat_grid(c, n), kThreads, 0, c->stream>>>(n, c->x, c->st.h);
        else
            k_cg_finish_from<<<flat_grid(c, n), kThreads, 0, c->stream>>>(n, c->x, x0, c->st.h);
        c->launches++;
        if ((rc = check_launch(c, "cg finish"))) return rc;
        if ((rc = read_scalars(c))) return rc;
        const CgDev &g = c->host_dev->cg;
        if (g.fault) return fail(c, SHK_CUDA_ERROR, "a TMA tile copy did not complete (bounded wait ran out)");
        s.niter = (long)g.iter;
        s.status = g.status;
        s.rnorm0 = g.rnorm0;
        s.rnorm = g.rnorm;
    } else if (o->precision == SHK_MIXED) {
        // Float32 stencil and CG with Float64 residual replacement.  The Float32 CG runs until its
        // recursive residual has dropped by inner_rtol; then its correction is folded into the
        // Float64 head (h += x32), the true residual b - A64 h is recomputed in Float64 and the CG
        // continues from it with the previous search direction.  Convergence is judged only on the
        // Float64 residual.  A Float32 zero-curvature event restarts the direction instead of
        // failing; three in a row, or no progress of the Float64 residual, end the solve.
        k_to_float_lapl<<<flat_grid(c, n), kThreads, 0, c->stream>>>(nx, ny, c->aP, c->aE, c->aN, c->aP32, c->aE32,
                                                                     c->aN32, c->dP32);
        c->launches++;
        const double inner_rtol = o->inner_rtol > 0 ? o->inner_rtol : 1e-2;
        const int max_refine = o->max_refine > 0 ? o->max_refine : 200;
        const long long itmax = o->itmax > 0 ? o->itmax : 2LL * n;
        const long long cycle_cap = o->inner_itmax > 0 ? o->inner_itmax : std::max(200LL, (long long)(nx + ny) / 2);
        const bool trace = getenv("SHK_VERBOSE") != nullptr;
        long total = 0;
        int refine = 0, restarts = 0, stalls = 0;
        double best = INFINITY;
        bool cont = false;
        int parity = 0;
        int status = SHK_NOT_CONVERGED;
        CgDev *cgh = &c->host_dev->cg_in;
        for (;;) {
            k_outer_residual<<<c->grid_stencil, kThreads, 0, c->stream>>>(nx, ny, c->aP, c->aE, c->aN, c->st.h, c->rhs,
                                                                         c->b32, c->dev, c->partials, c->counter,
                                                                         c->mask8);
            c->launches++;
            int rc = read_scalars(c);
            if (rc) return rc;
            const double rn = sqrt(c->host_dev->ref_rr), bn = sqrt(c->host_dev->ref_bb);
            if (trace)
                fprintf(stderr, "[shk mixed] cycle %d: ||r64||/||b|| = %.3e, inner iterations so far %ld, inner status %d\n",
                        refine, rn / bn, total, refine ? cgh->status : -1);
            if (refine == 0) s.rnorm0 = rn;
            s.rnorm = rn;
            if (isnan(rn)) {
                status = SHK_BREAKDOWN;
                break;
            }
            if (rn <= o->rtol * bn || rn == 0.0) {
                status = SHK_OK;
                break;
            }
            if (rn < 0.5 * best) {
                best = rn;
                stalls = 0;
            } else if (++stalls >= 8) {
                break;
            }
            if (refine >= max_refine || total >= itmax) break;
            if (cont) {
                // keep gamma / pNorm2 / rz_last of the previous inner solve, continue its direction
                cgh->done = 0;
                cgh->status = SHK_OK;
                cgh->iter = 0;
                cgh->cont = 1;
                cgh->itmax = std::min(itmax - total, cycle_cap);
                cgh->rtol = inner_rtol;
                cgh->atol = 0.0;
                cgh->stop_rule = SHK_STOP_RELRES;
            } else {
                *cgh = make_cg_init(o, n, true, inner_rtol);
                cgh->itmax = std::min(itmax - total, cycle_cap);
            }
            long it = 0;
            // the inner solve's "x" is the correction: x32 starts at 0 and r32 = b32; a continued
            // solve starts from the buffer holding the previous solve's last search direction
            rc = cg_core<float>(c, o, &c->dev->cg_in, cgh, c->aP32, c->aE32, c->aN32, nullptr, c->b32, c->x32, c->r32,
                                c->z32, c->p32, c->Ap32, c->cr32, c->cp32, &it, parity, c->dP32);
            if (rc) return rc;
            if ((rc = read_cg_flags(c, cgh, &c->dev->cg_in))) return rc;
            k_refine_update<<<flat_grid(c, n), kThreads, 0, c->stream>>>(n, c->x32, c->st.h);
            c->launches++;
            if ((rc = check_launch(c, "refine update"))) return rc;
            total += it;
            refine++;
            parity = (parity + (int)(cgh->iter & 1)) & 1;
            if (cgh->status == SHK_BREAKDOWN) {  // Float32 zero curvature: restart the direction
                cont = false;
                if (++restarts >= 3) {
                    status = SHK_BREAKDOWN;
                    break;
                }
            } else {
                restarts = 0;
                cont = true;
            }
        }
        s.niter = total;
        s.status = status;
        s.refinements = refine;
    } else {
        return fail(c, SHK_BAD_ARG, "unknown precision");
    }
    if ((o->precond == SHK_PRECOND_CHEBYSHEV)) {
        if (o->precision != SHK_FP64) {
            int rc = read_scalars(c);
            if (rc) return rc;
        }
        s.lambda_min = c->host_dev->cheb.lam_min;
        s.lambda_max = c->host_dev->cheb.lam_max;
        s.bounds_valid = c->host_dev->cheb.adopted;
    }
    if (st) *st = s;
    return SHK_OK;
}

} // namespace shk

// =============================================================================================
// Allocation-free Jacobi-PCG solve (shk_cg_solve_static).
//
// Some callers cannot allocate device memory at solve time: an application whose device memory
// is owned entirely by its own pool allocator, code running inside a real-time loop where the
// device-wide synchronisation of cudaMalloc/cudaFree is not acceptable, or a plugin host that
// forbids allocation after start-up.  This entry point serves them: its Krylov vectors, grid
// reduction partials and scalar block live in the file-scope array below, which every GPU that
// loads the library holds until the process exits.  The caller passes only inputs and outputs.
//
// Limits and sharing: at most kStaticMaxCells cells (a 256 x 256 grid); every call uses the same
// array and leaves its contents behind, so calls that overlap on the GPU (two streams, or two
// host threads) race and must be serialised by the caller.
// =============================================================================================
namespace shk {
namespace {
constexpr long long kStaticMaxCells = 65536;
constexpr int kStaticMaxBlocks = 4096;
constexpr size_t kStaticVecBytes = (size_t)kStaticMaxCells * sizeof(double);
constexpr size_t kStaticPartialBytes = (size_t)kMaxRedValues * kStaticMaxBlocks * sizeof(double);
constexpr size_t kStaticCgOffset = 5 * kStaticVecBytes + kStaticPartialBytes + 256;
constexpr size_t kStaticBytes = kStaticCgOffset + ((sizeof(CgDev) + 255) / 256) * 256;
} // namespace

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

// Writes the initial scalar block and clears the reduction counter (it must start at zero; an
// earlier call that stopped on an error could have left it non-zero).
__global__ void k_static_init(CgDev *cg, CgDev init, unsigned int *counter) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *cg = init;
        *counter = 0u;
    }
}

// Device address of g_static_scratch for each device, looked up once per device (with that device
// current) through cudaGetSymbolAddress: in host code the array's name is only a stand-in.
static void *g_static_addr[128];

static int static_scratch_address(int device, void **out) {
    if (device < 0 || device >= 128) return SHK_BAD_ARG;
    if (!g_static_addr[device]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess || !ptr) {
            fprintf(stderr, "shk_cg_solve_static: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return SHK_CUDA_ERROR;
        }
        g_static_addr[device] = ptr;
    }
    *out = g_static_addr[device];
    return SHK_OK;
}

// ---------------------------------------------------------------------------------------------
// Ensemble CG: the Jacobi-PCG bodies over every instance in one grid.  Instances whose Picard loop
// has finished, or whose CG has stopped, return at once.
// ---------------------------------------------------------------------------------------------

// Krylov state of a new solve for every instance still in its Picard loop (make_cg_init), and a
// fresh trip count for the solve's loop.
__global__ void k_ens_cg_reset(EnsInst *E, EnsCtl *ctl) {
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->cg_trips = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ctl->n; i += gridDim.x * blockDim.x) {
        if (!E[i].pic_active) continue;
        CgDev *g = E[i].cg;
        memset(g, 0, sizeof(CgDev));
        g->atol = ctl->atol;
        g->rtol = ctl->rtol;
        g->itmax = ctl->itmax > 0 ? ctl->itmax : 2LL * E[i].nx * E[i].ny;
        g->stop_rule = ctl->stop_rule;
        g->status = SHK_OK;
        g->first = 1;
    }
}

__global__ void __launch_bounds__(kThreads) k_ens_cg_init(EnsInst *E, const int *b2i) {
    __shared__ EnsInst I;
    const Blk B = ens_stage(I, E, b2i, EF_STENCIL);
    if (!I.pic_active) return;
    cg_init_body<double, true>(B, I.nx, I.ny, I.aP, I.aE, I.aN, I.st.h, I.rhs, I.r, I.x, I.cg, I.partials,
                               I.counter, I.mask8);
}

// Multigrid form: r = b - A h with r'r and the GROUNDED b'b parked for the V-cycle's finish.
__global__ void __launch_bounds__(kThreads) k_ens_cg_init_mg(EnsInst *E, const int *b2i) {
    __shared__ EnsInst I;
    const Blk B = ens_stage(I, E, b2i, EF_STENCIL);
    if (!I.pic_active) return;
    cg_init_body<double, false>(B, I.nx, I.ny, I.aP, I.aE, I.aN, I.st.h, I.rhs, I.r, I.x, I.cg, I.partials,
                                I.counter, I.mask8);
}

// Multigrid form: p = z + beta p, Ap, p'Ap (the V-cycle's z in place of r/aP).
__global__ void __launch_bounds__(kMarchX, 6) k_ens_cg_A_mg(EnsInst *E, const int *b2i, int parity) {
    __shared__ EnsInst I;
    const Blk B = ens_stage(I, E, b2i, EF_MARCH);
    if (!I.pic_active) return;
    const double *p_old = parity ? I.p1 : I.p0;
    double *p_new = parity ? I.p0 : I.p1;
    cg_A_body<double, false, false>(B, I.nx, I.ny, I.march_th, I.aP, I.aE, I.aN, I.r, I.z, p_old, p_new, I.Ap,
                                    I.cg, I.partials, I.counter, DBL_EPSILON, nullptr);
}

__global__ void __launch_bounds__(kMarchX, 6) k_ens_cg_A(EnsInst *E, const int *b2i, int parity) {
    __shared__ EnsInst I;
    const Blk B = ens_stage(I, E, b2i, EF_MARCH);
    if (!I.pic_active) return;
    const double *p_old = parity ? I.p1 : I.p0;
    double *p_new = parity ? I.p0 : I.p1;
    cg_A_body<double, true, false>(B, I.nx, I.ny, I.march_th, I.aP, I.aE, I.aN, I.r, nullptr, p_old, p_new, I.Ap,
                                   I.cg, I.partials, I.counter, DBL_EPSILON, nullptr);
}

__global__ void __launch_bounds__(kThreads) k_ens_cg_B(EnsInst *E, const int *b2i, int parity) {
    __shared__ EnsInst I;
    const Blk B = ens_stage(I, E, b2i, EF_STREAM);
    if (!I.pic_active) return;
    const double *p_new = parity ? I.p0 : I.p1;
    cg_B_body<double, true>(B, I.nx * I.ny, I.aP, p_new, I.Ap, I.x, I.r, I.cg, I.partials, I.counter);
}

// h = x + h, then (one thread per instance, after the solve) the solve's statistics
__global__ void __launch_bounds__(kThreads) k_ens_cg_finish(EnsInst *E, const int *b2i) {
    __shared__ EnsInst I;
    const Blk B = ens_stage(I, E, b2i, EF_FLAT);
    if (!I.pic_active) return;
    cg_finish_body(B, I.nx * I.ny, I.x, I.st.h);
}
__global__ void k_ens_cg_stats(EnsInst *E, const EnsCtl *ctl) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ctl->n; i += gridDim.x * blockDim.x) {
        if (!E[i].pic_active) continue;
        const CgDev *g = E[i].cg;
        E[i].cg_iters += g->iter;
        E[i].cg_solves += 1;
        if (g->status == SHK_BREAKDOWN) E[i].cg_breakdowns += 1;
    }
}

// Condition of the ensemble's CG loop (two iterations per trip): another trip while any instance
// in its Picard loop has a CG still running, and never more than the largest itmax/2 + 8 trips.
// Launched once before the loop as well: a conditional's default value is applied once per graph
// launch, not each time a nested loop starts, so every solve sets its loop's condition itself.
__global__ void k_ens_cg_cond(EnsInst *E, EnsCtl *ctl, cudaGraphConditionalHandle h) {
    __shared__ int any;
    __shared__ long long cap;
    if (threadIdx.x == 0) {
        any = 0;
        cap = 0;
    }
    __syncthreads();
    int mine = 0;
    long long mcap = 0;
    for (int i = threadIdx.x; i < ctl->n; i += blockDim.x) {
        const CgDev *g = E[i].cg;
        if (E[i].pic_active && !*(const volatile int *)&g->done) mine = 1;
        mcap = mcap > g->itmax ? mcap : g->itmax;
    }
    if (mine) atomicOr(&any, 1);
    atomicMax(reinterpret_cast<unsigned long long *>(&cap), (unsigned long long)mcap);
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int t = ++ctl->cg_trips;
        const bool more = any && 2LL * (long long)t < cap + 16;
        cudaGraphSetConditional(h, more ? 1u : 0u);
    }
}

void ens_cg_reset(cudaStream_t s, EnsInst *E, EnsCtl *ctl, int n) {
    k_ens_cg_reset<<<(n + 255) / 256, 256, 0, s>>>(E, ctl);
}
void ens_cg_init(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks) {
    k_ens_cg_init<<<nblocks, kThreads, 0, s>>>(E, b2i);
}
void ens_cg_init_mg(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks) {
    k_ens_cg_init_mg<<<nblocks, kThreads, 0, s>>>(E, b2i);
}
void ens_cg_A_mg(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks, int parity) {
    k_ens_cg_A_mg<<<nblocks, kMarchX, 0, s>>>(E, b2i, parity);
}
void ens_cg_A(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks, int parity) {
    k_ens_cg_A<<<nblocks, kMarchX, 0, s>>>(E, b2i, parity);
}
void ens_cg_B(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks, int parity) {
    k_ens_cg_B<<<nblocks, kThreads, 0, s>>>(E, b2i, parity);
}
void ens_cg_finish(cudaStream_t s, EnsInst *E, const EnsCtl *ctl, int n, const int *b2i, int nblocks) {
    k_ens_cg_finish<<<nblocks, kThreads, 0, s>>>(E, b2i);
    k_ens_cg_stats<<<(n + 255) / 256, 256, 0, s>>>(E, ctl);
}
void ens_cg_cond(cudaStream_t s, EnsInst *E, EnsCtl *ctl, int n, cudaGraphConditionalHandle h) {
    k_ens_cg_cond<<<1, 256, 0, s>>>(E, ctl, h);
}

} // namespace shk


extern "C" SHK_API int shk_cg_solve_static(int nx, int ny, const double *aP, const double *aE, const double *aN,
                                           const double *rhs, double *x, const shk_cg_opts *o, shk_cg_stats *st,
                                           void *stream) {
    using namespace shk;
    if (!o || !aP || !aE || !aN || !rhs || !x) return SHK_BAD_ARG;
    if (nx < 2 || ny < 2 || (long long)nx * ny > kStaticMaxCells) {
        fprintf(stderr, "shk_cg_solve_static: grid %d x %d exceeds the %lld-cell limit of the static scratch "
                        "(use shk_cg_solve with a context instead)\n", nx, ny, kStaticMaxCells);
        return SHK_BAD_ARG;
    }
    if (o->precond != SHK_PRECOND_JACOBI || o->precision != SHK_FP64 ||
        (o->stop_rule != SHK_STOP_KRYLOV && o->stop_rule != SHK_STOP_RELRES) || !(o->rtol >= 0) || !(o->atol >= 0)) {
        fprintf(stderr, "shk_cg_solve_static: only the Float64 Jacobi-preconditioned solve is available here\n");
        return SHK_BAD_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int device = 0, sms = 148;
    if (cudaGetDevice(&device) != cudaSuccess) return SHK_CUDA_ERROR;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return SHK_CUDA_ERROR;
    void *base = nullptr;
    int rc = static_scratch_address(device, &base);
    if (rc) return rc;
    const int n = nx * ny;
    // launch geometry, as a context computes it
    const long long tiles = (long long)((nx + kTX - 1) / kTX) * ((ny + kTY - 1) / kTY);
    const int grid_stencil = (int)std::max(1LL, std::min((long long)sms * 6, tiles));
    const long long tiles_x = (nx + kMarchX - 1) / kMarchX;
    const int march_th = (int)std::min(64LL, std::max(8LL, (long long)ny * tiles_x / ((long long)sms * 12)));
    const int march_blocks = (int)(tiles_x * ((ny + march_th - 1) / march_th));
    const int grid_b = (int)std::max(1LL, std::min((long long)sms * 8,
                                                   ((long long)n / 2 + (long long)kThreads * kUnrollB - 1) /
                                                       ((long long)kThreads * kUnrollB)));
    if (march_blocks > kStaticMaxBlocks || grid_stencil > kStaticMaxBlocks) return SHK_BAD_ARG;
    char *b = (char *)base;
    double *xc = (double *)(b), *r = (double *)(b + kStaticVecBytes);
    double *p[2] = {(double *)(b + 2 * kStaticVecBytes), (double *)(b + 3 * kStaticVecBytes)};
    double *Ap = (double *)(b + 4 * kStaticVecBytes);
    double *partials = (double *)(b + 5 * kStaticVecBytes);
    unsigned int *counter = (unsigned int *)(b + 5 * kStaticVecBytes + kStaticPartialBytes);
    CgDev *cg = (CgDev *)(b + kStaticCgOffset);
    CgDev init;
    memset(&init, 0, sizeof(init));
    init.atol = o->atol;
    init.rtol = o->rtol;
    init.itmax = o->itmax > 0 ? o->itmax : 2LL * n;
    init.stop_rule = o->stop_rule;
    init.first = 1;
    k_static_init<<<1, 32, 0, s>>>(cg, init, counter);
    k_cg_init<double, true><<<grid_stencil, kThreads, 0, s>>>(nx, ny, aP, aE, aN, x, rhs, r, xc, cg, partials, counter,
                                                              nullptr);
    if (cudaGetLastError() != cudaSuccess) return SHK_CUDA_ERROR;
    CgDev h;
    long long enq = 0;
    int batch = 8;
    for (;;) {
        if (cudaMemcpyAsync(&h, cg, sizeof(CgDev), cudaMemcpyDeviceToHost, s) != cudaSuccess) return SHK_CUDA_ERROR;
        if (cudaStreamSynchronize(s) != cudaSuccess) return SHK_CUDA_ERROR;
        if (h.done) break;
        if (h.iter > h.itmax + 4 || enq > h.itmax + 2LL * 256 + 8) {
            // The device loop ran past every bound it can reach: report what it reached.
            if (st) {
                memset(st, 0, sizeof(*st));
                st->niter = (long)h.iter;
                st->status = SHK_CUDA_ERROR;
                st->rnorm0 = h.rnorm0;
                st->rnorm = h.rnorm;
                st->lambda_min = st->lambda_max = 1.0;
            }
            return SHK_CUDA_ERROR;
        }
        for (int k = 0; k < batch; k++, enq++) {
            double *p_old = p[enq & 1], *p_new = p[(enq + 1) & 1];
            k_cg_A<double, true><<<march_blocks, kMarchX, 0, s>>>(nx, ny, march_th, aP, aE, aN, r, nullptr, p_old,
                                                                  p_new, Ap, cg, partials, counter, DBL_EPSILON);
            k_cg_B<double, true><<<grid_b, kThreads, 0, s>>>(n, aP, p_new, Ap, xc, r, cg, partials, counter);
        }
        if (cudaGetLastError() != cudaSuccess) return SHK_CUDA_ERROR;
        if (batch < 256) batch *= 2;
    }
    k_cg_finish<<<std::max(1, std::min(sms * 8, (n + kThreads - 1) / kThreads)), kThreads, 0, s>>>(n, xc, x);
    if (cudaGetLastError() != cudaSuccess) return SHK_CUDA_ERROR;
    if (cudaMemcpyAsync(&h, cg, sizeof(CgDev), cudaMemcpyDeviceToHost, s) != cudaSuccess) return SHK_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return SHK_CUDA_ERROR;
    if (st) {
        memset(st, 0, sizeof(*st));
        st->niter = (long)h.iter;
        st->status = h.status;
        st->rnorm0 = h.rnorm0;
        st->rnorm = h.rnorm;
        st->lambda_min = st->lambda_max = 1.0;
    }
    return h.status;
}
