// shk_device.cuh -- device helpers: Julia-faithful scalar functions, tile iteration and the
// deterministic last-block grid reduction.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "shk_internal.cuh"

namespace shk {

// ---- scalar semantics matching the reference (Julia) -----------------------------------------

// Julia x^n for Float64 and Integer n (Base.pow_body): n == 3 is x*x*x; n == 2 gives fl(x*x);
// other n use a compensated power-by-squaring.
__device__ __forceinline__ double jl_powi(double x, int n) {
    if (n == 0) return 1.0;
    if (n == 1) return x;
    if (n == 2) return x * x;
    if (n == 3) return x * x * x;
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

// pow with the reference's canonical_exponent dispatch (src/model_parameters.jl:122-134).
__device__ __forceinline__ double jl_pow(double x, double e, int e_int) {
    return e_int >= 0 ? jl_powi(x, e_int) : pow(x, e);
}

__device__ __forceinline__ double jl_max(double a, double b) {
    return (isnan(a) || isnan(b)) ? __longlong_as_double(0x7ff8000000000000LL) : (a > b ? a : b);
}
__device__ __forceinline__ double jl_min(double a, double b) {
    return (isnan(a) || isnan(b)) ? __longlong_as_double(0x7ff8000000000000LL) : (a < b ? a : b);
}
__device__ __forceinline__ double jl_sign(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : x); }
__device__ __forceinline__ double jl_clamp(double x, double lo, double hi) {
    return x > hi ? hi : (x < lo ? lo : x);
}

__device__ __forceinline__ bool is_dirichlet(uint8_t m) { return m == M_OCEAN || m == M_LAND; }

// ---- tiles -------------------------------------------------------------------------------------

struct Tiles {
    int nx, ny, tiles_x, ntiles;
    __device__ __forceinline__ Tiles(int nx_, int ny_) : nx(nx_), ny(ny_) {
        tiles_x = (nx + kTX - 1) / kTX;
        ntiles = tiles_x * ((ny + kTY - 1) / kTY);
    }
    __device__ __forceinline__ void cell(int t, int &ix, int &iy) const {
        int tx = t % tiles_x, ty = t / tiles_x;
        ix = tx * kTX + (int)(threadIdx.x % kTX);
        iy = ty * kTY + (int)(threadIdx.x / kTX);
    }
};

// ---- reductions -----------------------------------------------------------------------------

template <bool MAX>
__device__ __forceinline__ double red_op(double a, double b) {
    if (MAX) return jl_max(a, b);
    return a + b;
}

template <bool MAX>
__device__ __forceinline__ double warp_reduce(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = red_op<MAX>(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Block-reduce NV values; result valid in thread 0.  Deterministic order.
template <int NV, bool MAX>
__device__ __forceinline__ void block_reduce(double (&v)[NV]) {
    __shared__ double sh[NV][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_reduce<MAX>(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) sh[k][warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double t = lane < nwarps ? sh[k][lane] : 0.0;
            v[k] = warp_reduce<MAX>(t);
        }
    }
    __syncthreads();
}

// A block's place among the blocks that work on one instance: the single-instance kernels use
// their whole grid; the ensemble kernels give each instance a contiguous range of one grid.
struct Blk {
    int id, n;
};
__device__ __forceinline__ Blk grid_blk() { return Blk{(int)blockIdx.x, (int)gridDim.x}; }

// Grid reduction without inter-block waiting over the B.n blocks of one instance.  Returns true in
// exactly one block (the last to arrive); there, thread 0 holds the totals in out[] (other threads:
// unspecified).
template <int NV, bool MAX>
__device__ __forceinline__ bool grid_reduce(Blk B, double (&v)[NV], double *partials, unsigned int *counter,
                                            double (&out)[NV]) {
    __shared__ int am_last;
    block_reduce<NV, MAX>(v);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) partials[(size_t)k * B.n + B.id] = v[k];
        __threadfence();
        unsigned int prev = atomicAdd(counter, 1u);
        am_last = (prev == (unsigned int)B.n - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) {
        acc[k] = 0.0;
        for (int i = threadIdx.x; i < B.n; i += blockDim.x)
            acc[k] = red_op<MAX>(acc[k], __ldcg(&partials[(size_t)k * B.n + i]));
    }
    block_reduce<NV, MAX>(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) out[k] = acc[k];
        *counter = 0u;
        __threadfence();
    }
    return true;
}

template <int NV, bool MAX>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], double *partials, unsigned int *counter,
                                            double (&out)[NV]) {
    return grid_reduce<NV, MAX>(grid_blk(), v, partials, counter, out);
}

// ---------------------------------------------------------------------------------------------
// Per-block reads of the device-side CG scalars.  Thread (0,0) reads them and shares them through
// shared memory, so a launch sends one request per block to the scalars' L2 line instead of one
// per warp (a hot spot that cost more than the data traffic of the small level kernels).  Every
// thread of the block must call these, before any early return.
// ---------------------------------------------------------------------------------------------
struct CgView {
    int done, first;
    double alpha, beta, alpha_prev;
};

__device__ __forceinline__ CgView block_cg_view(const CgDev *cg) {
    __shared__ CgView v;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        v.done = *(const volatile int *)&cg->done;
        v.first = cg->first;
        v.alpha = cg->alpha;
        v.beta = cg->beta;
        v.alpha_prev = cg->alpha_prev;
    }
    __syncthreads();
    return v;
}

__device__ __forceinline__ bool block_cg_done(const int *done) {
    __shared__ int d;
    if (threadIdx.x == 0 && threadIdx.y == 0) d = done ? *(const volatile int *)done : 0;
    __syncthreads();
    return d != 0;
}

// ---------------------------------------------------------------------------------------------
// Ensemble kernels: the block's instance descriptor, copied to shared memory once per block, and
// the block's place among that instance's blocks of kernel family FAM.
// ---------------------------------------------------------------------------------------------
static_assert(sizeof(EnsInst) % 8 == 0, "EnsInst is copied in 8-byte words");
__device__ __forceinline__ Blk ens_stage(EnsInst &dst, const EnsInst *E, const int *b2i, int fam) {
    const long long *src = reinterpret_cast<const long long *>(&E[b2i[blockIdx.x]]);
    long long *d = reinterpret_cast<long long *>(&dst);
    for (int k = threadIdx.x; k < (int)(sizeof(EnsInst) / 8); k += blockDim.x) d[k] = src[k];
    __syncthreads();
    return Blk{(int)blockIdx.x - dst.blk0[fam], dst.nblk[fam]};
}

// ---------------------------------------------------------------------------------------------
// Scalar updates (run by thread 0 of the last block)
// ---------------------------------------------------------------------------------------------
static __device__ void cg_init_finish(CgDev *cg, double rz, double rr, double bb) {
    if (cg->cont) {
        // Residual replacement: keep the previous search direction, p = z + beta p with
        // beta = r'z (replaced residual) / r'z (last recursive residual).
        const double beta = rz / cg->rz_last;
        if (isfinite(beta) && beta >= 0) {
            cg->beta = beta;
            cg->pNorm2 = rz + beta * beta * cg->pNorm2;
            cg->first = 0;
        } else {
            cg->first = 1;
            cg->beta = 0.0;
            cg->pNorm2 = rz;
        }
    } else {
        cg->first = 1;
        cg->beta = 0.0;
        cg->pNorm2 = rz;
    }
    cg->gamma = rz;
    cg->rz_last = rz;
    const double rn = sqrt(rz);
    cg->rr = sqrt(rr);
    cg->bnorm = sqrt(bb);
    cg->rnorm0 = cg->stop_rule == SHK_STOP_KRYLOV ? rn : cg->rr;
    cg->rnorm = cg->rnorm0;
    cg->eps_stop = cg->atol + cg->rtol * rn;
    cg->iter = 0;
    if (isnan(rz) || isnan(rr)) {
        cg->done = 1;
        cg->status = SHK_BREAKDOWN;
    } else if (rz == 0.0) {
        cg->done = 1;
        cg->status = SHK_OK;
    } else {
        bool solved = cg->stop_rule == SHK_STOP_KRYLOV ? (rn <= cg->eps_stop) : (cg->rr <= cg->rtol * cg->bnorm);
        if (solved) {
            cg->done = 1;
            cg->status = SHK_OK;
        } else if (cg->iter >= cg->itmax) {
            cg->done = 1;
            cg->status = SHK_NOT_CONVERGED;
        } else {
            cg->done = 0;
        }
    }
}

static __device__ void cg_iter_finish(CgDev *cg, double rz, double rr) {
    const double rn = sqrt(rz), rrn = sqrt(rr);
    cg->rz_last = rz;
    cg->rr = rrn;
    bool solved;
    if (cg->stop_rule == SHK_STOP_KRYLOV) solved = (rn <= cg->eps_stop) || (rn + 1.0 <= 1.0);
    else solved = rrn <= cg->rtol * cg->bnorm;
    cg->rnorm = cg->stop_rule == SHK_STOP_KRYLOV ? rn : rrn;
    if (!solved) {
        double beta = rz / cg->gamma;
        cg->pNorm2 = rz + beta * beta * cg->pNorm2;
        cg->gamma = rz;
        cg->beta = beta;
        cg->first = 0;
    }
    cg->iter += 1;
    if (isnan(rz) || isnan(rr)) {
        cg->done = 1;
        cg->status = SHK_BREAKDOWN;
    } else if (solved) {
        cg->done = 1;
        cg->status = SHK_OK;
    } else if (cg->iter >= cg->itmax) {
        cg->done = 1;
        cg->status = SHK_NOT_CONVERGED;
    }
}

} // namespace shk
