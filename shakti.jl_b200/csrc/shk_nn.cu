// shk_nn.cu -- BF16 tensor-core kernels of the learned warm start (training and inference).
//
// No counterpart in the reference: the reference warm-starts each solve from the current head
// (cg! x0 = vec(h), src/linear_solver.jl:876-881).  Here a small convolutional encoder-decoder
// predicts the head increment of the coming timestep from the state; the prediction only seeds
// Picard/CG (the solve still runs to its tolerance) and is dropped when its initial residual is
// worse than the previous head's.
//
// Tensors are NHWC (channels innermost): activations BF16, gradients Float32, weights BF16 for the
// tensor cores with a Float32 master copy for the optimiser.  A 3x3 convolution is an implicit
// GEMM (BF16 inputs, Float32 accumulation) on the tcgen05 tensor cores -- by default reading its A
// operand straight out of TMA-loaded halo tiles, alternatively from per-tap gathered tiles -- or on
// mma.sync m16n8k16 (the comparison form):
//   forward      Y[p, co]  = sum_{tap, ci} X[p + off(tap), ci] W[tap, co, ci]        (+ bias, ReLU)
//   input grad   dX[p, ci] = sum_{tap, co} dY[p - off(tap), co] W[tap, co, ci]       (the forward
//                kernel on the per-tap transposed weights with the offsets negated)
//   weight grad  dW[tap, co, ci] = sum_p dY[p, co] X[p + off(tap), ci]                (split over
//                pixel chunks, Float32 atomics)
// with zero padding at each image's border.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <type_traits>

#include "../../include/shakti_b200.h"

namespace shk {
namespace nn {

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t ld_pair(const bf16 *p) { return *reinterpret_cast<const uint32_t *>(p); }
__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// ---------------------------------------------------------------------------------------------
// 3x3 convolution, forward form.  One block: 64 consecutive pixels (flattened n, y, x) x NT output
// channels; warp w owns pixels 16w..16w+15 of the block.  Lane (g = lane/4, t = lane%4) holds the
// A fragment rows g, g+8 (pixels) and columns 2t, 2t+1, 2t+8, 2t+9 (input channels), and the B
// fragment column g (output channel) rows 2t, 2t+1, 2t+8, 2t+9.  FLIP negates the tap offsets (the
// input-gradient form).  Cin % 16 == 0, Cout % NT == 0.
// ---------------------------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(128) k_conv3x3(const bf16 *__restrict__ X, const bf16 *__restrict__ Wt,
                                                 const float *__restrict__ bias, bf16 *__restrict__ Y,
                                                 float *__restrict__ Yf, int N, int H, int W, int Cin, int Cout,
                                                 int relu, int flip) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const long long P = (long long)N * H * W;
    const long long p0 = (long long)blockIdx.x * 64 + warp * 16;
    const int co0 = blockIdx.y * NT;
    const long long r0 = p0 + g, r1 = p0 + g + 8;
    int n0 = 0, y0 = 0, x0 = 0, n1 = 0, y1 = 0, x1 = 0;
    const bool v0 = r0 < P, v1 = r1 < P;
    if (v0) { n0 = (int)(r0 / ((long long)H * W)); const int q = (int)(r0 % ((long long)H * W)); y0 = q / W; x0 = q % W; }
    if (v1) { n1 = (int)(r1 / ((long long)H * W)); const int q = (int)(r1 % ((long long)H * W)); y1 = q / W; x1 = q % W; }
    float acc[NT / 8][4];
#pragma unroll
    for (int j = 0; j < NT / 8; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
    for (int tap = 0; tap < 9; tap++) {
        int dy = tap / 3 - 1, dx = tap % 3 - 1;
        if (flip) { dy = -dy; dx = -dx; }
        const int sy0 = y0 + dy, sx0 = x0 + dx, sy1 = y1 + dy, sx1 = x1 + dx;
        const bool ok0 = v0 && sy0 >= 0 && sy0 < H && sx0 >= 0 && sx0 < W;
        const bool ok1 = v1 && sy1 >= 0 && sy1 < H && sx1 >= 0 && sx1 < W;
        const bf16 *a0p = X + (((long long)n0 * H + (ok0 ? sy0 : 0)) * W + (ok0 ? sx0 : 0)) * Cin + 2 * t;
        const bf16 *a1p = X + (((long long)n1 * H + (ok1 ? sy1 : 0)) * W + (ok1 ? sx1 : 0)) * Cin + 2 * t;
        const bf16 *bp = Wt + ((long long)tap * Cout + co0 + g) * Cin + 2 * t;
        for (int c = 0; c < Cin; c += 16) {
            uint32_t a[4];
            a[0] = ok0 ? ld_pair(a0p + c) : 0u;
            a[1] = ok1 ? ld_pair(a1p + c) : 0u;
            a[2] = ok0 ? ld_pair(a0p + c + 8) : 0u;
            a[3] = ok1 ? ld_pair(a1p + c + 8) : 0u;
#pragma unroll
            for (int j = 0; j < NT / 8; j++) {
                const bf16 *q = bp + (long long)j * 8 * Cin + c;
                uint32_t b[2] = {ld_pair(q), ld_pair(q + 8)};
                mma_bf16(acc[j], a, b);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < NT / 8; j++) {
        const int co = co0 + j * 8 + 2 * t;
        const float b0 = bias ? bias[co] : 0.0f, b1 = bias ? bias[co + 1] : 0.0f;
        float o[4] = {acc[j][0] + b0, acc[j][1] + b1, acc[j][2] + b0, acc[j][3] + b1};
        if (relu)
#pragma unroll
            for (int k = 0; k < 4; k++) o[k] = o[k] > 0.0f ? o[k] : 0.0f;
        if (v0) {
            if (Y) *reinterpret_cast<uint32_t *>(Y + r0 * Cout + co) = pack2(__float2bfloat16(o[0]), __float2bfloat16(o[1]));
            if (Yf) { Yf[r0 * Cout + co] = o[0]; Yf[r0 * Cout + co + 1] = o[1]; }
        }
        if (v1) {
            if (Y) *reinterpret_cast<uint32_t *>(Y + r1 * Cout + co) = pack2(__float2bfloat16(o[2]), __float2bfloat16(o[3]));
            if (Yf) { Yf[r1 * Cout + co] = o[2]; Yf[r1 * Cout + co + 1] = o[3]; }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// 3x3 convolution on the 5th-generation tensor cores (tcgen05, sm_100a): the same implicit GEMM,
// D[pixel, co] = sum_{tap, ci} X[pixel + off(tap), ci] W[tap, co, ci], with a CTA tile of 128
// pixels (M) x NT output channels (N, Cout rounded up to a multiple of 16) and the Float32
// accumulator in tensor memory (TMEM, NT columns of 128 lanes).  K runs over (tap, 32- or
// 16-channel chunk); each chunk's A (128 x KC) and B (NT x KC) tiles are staged in shared memory in
// the canonical K-major layout without swizzle -- 8-row x 16-byte core matrices, the two 8-element
// K halves 128 B apart (LBO), 8-row groups 256 B apart (SBO) -- by all threads (zero fill outside
// the image and past Cout), then one thread issues the chunk's K = 16 MMAs and commits them to the
// stage's mbarrier.  Two stages: chunk c + 1 is staged while the tensor cores run chunk c.  The
// epilogue reads each warp's 32 TMEM lanes (its 32 pixels) 8 columns at a time (tcgen05.ld),
// adds the bias, applies ReLU and stores BF16 and/or Float32.  Every mbarrier wait is bounded; a
// wait that runs out sets *err, and the CTA still waits for its MMAs and frees its TMEM.
// ---------------------------------------------------------------------------------------------
constexpr long kTcSpin = 1L << 22;

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (sm_100 format): start address, LBO and SBO in 16-byte units,
// version 1 at bit 46, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: Float32 D (bit 4), BF16 A (bits 7-9) and B (bits 10-12),
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity) {
    for (long i = 0; i < kTcSpin; i++) {
        uint32_t ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok)
                     : "r"(su32(bar)), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}

constexpr int kTcM = 128, kTcKC = 32;  // pixels per CTA, largest channel chunk

// Shared memory per CTA: two stages, the two mbarriers and the TMEM address slot, padded so that
// the CTAs resident on an SM (228 KB of shared memory, 1 KB reserved per CTA) never ask for more
// than the 512 TMEM columns together.
template <int NT>
struct TcLayout {
    static constexpr uint32_t cols = NT < 32 ? 32 : NT;
    static constexpr uint32_t a = kTcM * kTcKC * 2, b = NT * kTcKC * 2, stage = a + b;
    static constexpr uint32_t bars = 2 * stage, slot = bars + 16, used = slot + 16;
    static constexpr uint32_t pad = 233472u / (512u / cols) - 2048u;
    static constexpr uint32_t bytes = used > pad ? used : pad;
};

template <int NT>
__global__ void __launch_bounds__(128) k_conv3x3_tc(const bf16 *__restrict__ X, const bf16 *__restrict__ Wt,
                                                    const float *__restrict__ bias, bf16 *__restrict__ Y,
                                                    float *__restrict__ Yf, int N, int H, int W, int Cin, int Cout,
                                                    int relu, int flip, int *err) {
    using Lay = TcLayout<NT>;
    constexpr uint32_t kCols = Lay::cols;
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + Lay::bars);
    uint32_t *slot = reinterpret_cast<uint32_t *>(sm + Lay::slot);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long P = (long long)N * H * W, p0 = (long long)blockIdx.x * kTcM;
    const int KC = (Cin % kTcKC == 0) ? kTcKC : 16, nk = KC / 16, per_tap = Cin / KC, nch = 9 * per_tap;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *slot;

    // Staging map, fixed for the CTA: thread tid stages 16-byte segment g8 = tid % spr (spr = KC/8
    // segments per row) of rows tid / spr + k * (128 / spr), k < spr, of A (pixels) and the same of
    // B (output channels), so the pixel coordinates are computed once, not per chunk.
    const int spr = KC / 8, g8 = tid % spr, r0 = tid / spr, rstep = kTcM / spr;
    const uint32_t soff = (uint32_t)((g8 >> 1) * (kTcM * 32) + (g8 & 1) * 128);  // A segment offset in a row group
    const uint32_t boff = (uint32_t)((g8 >> 1) * (NT * 32) + (g8 & 1) * 128);
    int py[4], px[4];
    long long pbase[4];  // element offset of the pixel's channel 0 (n, y, x unshifted), -1 past P
    for (int k = 0; k < spr; k++) {
        const long long p = p0 + r0 + k * rstep;
        py[k] = px[k] = 0;
        pbase[k] = -1;
        if (p < P) {
            const long long hw = (long long)H * W;
            const int n = (int)(p / hw), rem = (int)(p % hw);
            py[k] = rem / W;
            px[k] = rem % W;
            pbase[k] = (((long long)n * H + py[k]) * W + px[k]) * Cin;
        }
    }
    auto stage_chunk = [&](int c, int st) {
        const int tap = c / per_tap, c0 = (c % per_tap) * KC;
        int dy = tap / 3 - 1, dx = tap % 3 - 1;
        if (flip) { dy = -dy; dx = -dx; }
        const long long shift = ((long long)dy * W + dx) * Cin + c0 + g8 * 8;
        unsigned char *A = sm + st * Lay::stage, *B = A + Lay::a;
        for (int k = 0; k < spr; k++) {
            const int r = r0 + k * rstep, y = py[k] + dy, x = px[k] + dx;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (pbase[k] >= 0 && y >= 0 && y < H && x >= 0 && x < W)
                v = *reinterpret_cast<const uint4 *>(X + pbase[k] + shift);
            *reinterpret_cast<uint4 *>(A + soff + (r >> 3) * 256 + (r & 7) * 16) = v;
        }
        const bf16 *wrow = Wt + (long long)tap * Cout * Cin + c0 + g8 * 8;
        for (int r = r0; r < NT; r += rstep) {
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (r < Cout) v = *reinterpret_cast<const uint4 *>(wrow + (long long)r * Cin);
            *reinterpret_cast<uint4 *>(B + boff + (r >> 3) * 256 + (r & 7) * 16) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor-core reads
    };

    constexpr uint32_t idesc = umma_idesc_bf16(kTcM, NT);
    bool ok = true;
    stage_chunk(0, 0);
    __syncthreads();
    for (int c = 0; c < nch; c++) {
        const int st = c & 1;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t A = su32(sm + st * Lay::stage), B = A + Lay::a;
            for (int j = 0; j < nk; j++) {
                const uint64_t da = umma_desc(A + j * (kTcM * 32), 128, 256);
                const uint64_t db = umma_desc(B + j * (NT * 32), 128, 256);
                const uint32_t acc = (c > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t .reg .pred pacc;\n\t setp.ne.b32 pacc, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, pacc;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             su32(&bar[st]))
                         : "memory");
        }
        if (c + 1 < nch) {
            // stage st ^ 1 was last read by chunk c - 1's MMAs
            if (c >= 1) ok = ok && tc_wait(&bar[st ^ 1], ((c - 1) >> 1) & 1);
            ok = __syncthreads_and(ok) != 0;  // uniform: every thread leaves the loop together
            if (!ok) break;
            stage_chunk(c + 1, st ^ 1);
            __syncthreads();
        }
    }
    // the last commit covers every MMA this CTA issued
    const int last = ok ? nch - 1 : -1;
    bool done_all = true;
    if (last >= 0) done_all = tc_wait(&bar[last & 1], (last >> 1) & 1);
    else {  // gave up early: wait (bounded) for whatever was committed before freeing TMEM
        for (int st = 0; st < 2; st++) tc_wait(&bar[st], 0);
        done_all = false;
    }
    done_all = __syncthreads_and(done_all) != 0;  // uniform: tcgen05.ld below is warp-collective
    if (!done_all && tid == 0) atomicExch(err, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (done_all) {
        const long long p = p0 + warp * 32 + lane;
        for (int cb = 0; cb < NT; cb += 8) {
            uint32_t v[8];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (p >= P || cb >= Cout) continue;
            float o[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                o[k] = __uint_as_float(v[k]) + (bias ? bias[cb + k] : 0.0f);
                if (relu) o[k] = o[k] > 0.0f ? o[k] : 0.0f;
            }
            if (Y) {
                uint4 pk = make_uint4(pack2(__float2bfloat16(o[0]), __float2bfloat16(o[1])),
                                      pack2(__float2bfloat16(o[2]), __float2bfloat16(o[3])),
                                      pack2(__float2bfloat16(o[4]), __float2bfloat16(o[5])),
                                      pack2(__float2bfloat16(o[6]), __float2bfloat16(o[7])));
                *reinterpret_cast<uint4 *>(Y + p * Cout + cb) = pk;
            }
            if (Yf) {
                *reinterpret_cast<float4 *>(Yf + p * Cout + cb) = make_float4(o[0], o[1], o[2], o[3]);
                *reinterpret_cast<float4 *>(Yf + p * Cout + cb + 4) = make_float4(o[4], o[5], o[6], o[7]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

// ---------------------------------------------------------------------------------------------
// 3x3 convolution on halo tiles (tcgen05 + TMA; the default form).  A CTA computes super-tiles of
// MT x 128 pixels of one image -- 16 rows x 8 MT columns -- for NT output channels; M tile j
// (columns 8j .. 8j + 7) accumulates in TMEM columns [j NT, (j + 1) NT) of one of ACC buffers.
// K runs over 16-channel chunks.  A stage holds a chunk's input halo (18 rows x (8 MT + 2) columns,
// one TMA box per 8-channel group laid out [row][column][8 channels], 16 B per pixel, zero outside
// the image) and the chunk's weights for all nine taps (one box per group: [tap][co][8 channels]).
// The MMA of M tile j, tap (dy, dx) reads its A operand straight out of the halo: the descriptor
// starts at halo pixel (1 + dy, 8j + 1 + dx); a core matrix (8 rows x 16 B) is 8 consecutive pixels
// of one halo row, consecutive core matrices along M are consecutive rows (SBO = the halo row
// pitch) and along K the next channel group (LBO = one group's halo): no im2col gather, each input
// pixel crosses from memory once per super-tile.  B is the tap's NT x 16 slice of the staged
// weights (SBO = 8 rows, LBO = one group's weights).
// Warp 4's lane 0 issues the stages' TMA copies (S - 1 stages ahead) and the MMAs; tcgen05.commit
// frees a stage (empty[]) and, after a super-tile's last chunk, hands the accumulator to warps 0-3
// (accf[]), which read their 32 TMEM lanes (tcgen05.ld, 16 columns at a time), add the bias, apply
// ReLU, store BF16 and/or Float32, and give the buffer back (acce[]).  Every wait is bounded; one
// that runs out sets *err and the CTA winds down: no new copies or MMAs, the copies and MMAs in
// flight are waited for, TMEM is freed.
// ---------------------------------------------------------------------------------------------
constexpr int kHxRows = 16, kHxThreads = 160;
constexpr uint32_t kHxMaxSmem = 227u * 1024;  // dynamic shared memory a CTA may have on sm_100

template <int NT>
struct HxCfg {
    // M tiles per super-tile: each M tile's MMAs form one dependent accumulation chain and a chunk
    // rotates over the MT chains, so more tiles keep more MMAs in flight -- as many as still leave
    // room for two accumulator buffers (2 MT NT <= 512 TMEM columns), which lets the epilogue of one
    // super-tile overlap the next one's MMAs.  Measured at 2048^2: 8 tiles at N = 16/32 cut those
    // layers by 4-18 %; 8 at N = 64 and 4 at N = 128 (one buffer) made them 10-65 % slower.
    static constexpr int MT = NT <= 32 ? 8 : (NT == 64 ? 4 : 2);
    static constexpr int ACC = 2 * MT * NT <= 512 ? 2 : 1;       // accumulator buffers
    static constexpr int HW = 8 * MT + 2, HH = kHxRows + 2;      // halo columns, rows
    static constexpr uint32_t HB = HH * HW * 16;                 // bytes of one 8-channel halo box
    static constexpr uint32_t HG = (HB + 127) / 128 * 128;       // its pitch (TMA destinations 128-B aligned)
    static constexpr uint32_t WG = 9 * NT * 16;                  // one 8-channel group of the weights
    static constexpr uint32_t stage = 2 * HG + 2 * WG;
    static constexpr int S = 4 * stage <= 200u * 1024 ? 4 : (3 * stage <= 200u * 1024 ? 3 : 2);
    static constexpr uint32_t bars = S * stage;  // full[S], empty[S], accf[ACC], acce[ACC], the weights' barrier
    static constexpr uint32_t misc = bars + 8 * (2 * S + 2 * ACC + 1);  // TMEM address, abort flag
    static constexpr uint32_t used = misc + 16;
    // more than half of an SM's shared memory: one CTA per SM, which then owns all 512 TMEM columns
    static constexpr uint32_t bytes = used > 120u * 1024 ? used : 120u * 1024;
    // weights-resident form: all of a layer's weights loaded once per CTA after the halo stages,
    // the stages carry halo chunks only
    static constexpr uint32_t rstage = 2 * HG;
    static constexpr int RS = 4;
    static uint32_t __host__ __device__ res_bars(int Cin) { return (RS * rstage + (uint32_t)(Cin / 8) * WG + 127) / 128 * 128; }
    static uint32_t __host__ __device__ res_bytes(int Cin) {
        const uint32_t u = res_bars(Cin) + 8 * (2 * RS + 2 * ACC + 1) + 16;
        return u > 120u * 1024 ? u : 120u * 1024;
    }
};

__device__ __forceinline__ void hx_expect(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void hx_load4(void *dst, const CUtensorMap *map, uint64_t *bar, int c, int x, int y, int n) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(su32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c), "r"(x), "r"(y), "r"(n), "r"(su32(bar))
        : "memory");
}

__device__ __forceinline__ void hx_load3(void *dst, const CUtensorMap *map, uint64_t *bar, int c, int o, int t) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(su32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c), "r"(o), "r"(t), "r"(su32(bar))
        : "memory");
}

// Bounded wait that also gives up once the CTA's abort flag is set (abort == nullptr: only the bound).
__device__ __forceinline__ bool hx_wait(uint64_t *bar, uint32_t parity, volatile int *abort) {
    for (long i = 0; i < kTcSpin; i++) {
        uint32_t ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok)
                     : "r"(su32(bar)), "r"(parity)
                     : "memory");
        if (ok) return true;
        if ((i & 255) == 255 && abort && *abort) return false;
    }
    return false;
}

__device__ __forceinline__ void hx_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t .reg .pred pacc;\n\t setp.ne.b32 pacc, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, pacc;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void hx_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}

template <int NT, bool RES>
__global__ void __launch_bounds__(kHxThreads, 1) k_conv3x3_hx(const __grid_constant__ CUtensorMap mx,
                                                              const __grid_constant__ CUtensorMap mw,
                                                              const float *__restrict__ bias, bf16 *__restrict__ Y,
                                                              float *__restrict__ Yf, int N, int H, int W, int Cin,
                                                              int Cout, int relu, int flip, int *err) {
    using Cf = HxCfg<NT>;
    constexpr int MT = Cf::MT, ACC = Cf::ACC, S = RES ? Cf::RS : Cf::S;
    constexpr uint32_t STG = RES ? Cf::rstage : Cf::stage;  // bytes of one stage
    extern __shared__ __align__(1024) unsigned char sm[];
    const uint32_t bars_off = RES ? Cf::res_bars(Cin) : Cf::bars, misc_off = bars_off + 8 * (2 * S + 2 * ACC + 1);
    uint64_t *full = reinterpret_cast<uint64_t *>(sm + bars_off), *empty = full + S, *accf = empty + S,
             *acce = accf + ACC, *wbar = acce + ACC;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + misc_off);
    volatile int *abort = reinterpret_cast<volatile int *>(sm + misc_off + 4);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_x = (W + 8 * MT - 1) / (8 * MT), tiles_y = (H + kHxRows - 1) / kHxRows;
    const long long T = (long long)N * tiles_x * tiles_y;
    const long long G = gridDim.x, b0 = blockIdx.x;
    const long long my_tiles = b0 < T ? (T - b0 + G - 1) / G : 0;
    const int nc = Cin / 16;
    const long long total = my_tiles * nc;  // stages this CTA consumes

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(su32(tslot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 32) {
        for (int i = 0; i < S; i++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&full[i])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&empty[i])) : "memory");
        }
        for (int i = 0; i < ACC; i++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&accf[i])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(su32(&acce[i])) : "memory");
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(wbar)) : "memory");
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;

    auto tile_at = [&](long long ti, int &n, int &y0, int &x0) {
        const long long t = b0 + ti * G;
        const long long per = (long long)tiles_x * tiles_y;
        n = (int)(t / per);
        const int r = (int)(t % per);
        y0 = (r / tiles_x) * kHxRows;
        x0 = (r % tiles_x) * 8 * MT;
    };

    if (warp == 4) {
        if (lane == 0 && total > 0) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mx)) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mw)) : "memory");
            auto load = [&](long long q) {
                const int slot = (int)(q % S), kc = (int)(q % nc);
                int n, y0, x0;
                tile_at(q / nc, n, y0, x0);
                unsigned char *st = sm + slot * STG;
                hx_expect(&full[slot], RES ? 2 * Cf::HB : 2 * (Cf::HB + Cf::WG));
                for (int g = 0; g < 2; g++) {
                    hx_load4(st + g * Cf::HG, &mx, &full[slot], kc * 16 + g * 8, x0 - 1, y0 - 1, n);
                    if (!RES) hx_load3(st + 2 * Cf::HG + g * Cf::WG, &mw, &full[slot], kc * 16 + g * 8, 0, 0);
                }
            };
            unsigned char *wres = sm + S * STG;  // RES: the layer's weights, [group][tap][co][8 channels]
            if (RES) {
                hx_expect(wbar, (uint32_t)(Cin / 8) * Cf::WG);
                for (int g = 0; g < Cin / 8; g++) hx_load3(wres + g * Cf::WG, &mw, wbar, g * 8, 0, 0);
            }
            constexpr uint32_t idesc = umma_idesc_bf16(kTcM, NT);
            long long issued = 0, consumed = 0;
            bool ok = true;
            for (; issued < total && issued < S - 1; issued++) load(issued);
            bool wdone = !RES;
            if (RES) wdone = ok = hx_wait(wbar, 0, abort);
            for (long long q = 0; q < total && ok; q++) {
                const int slot = (int)(q % S), kc = (int)(q % nc);
                const long long ti = q / nc;
                const int buf = (int)(ti % ACC);
                ok = hx_wait(&full[slot], (uint32_t)((q / S) & 1), abort);
                if (ok && kc == 0 && ti >= ACC) ok = hx_wait(&acce[buf], (uint32_t)((ti / ACC - 1) & 1), abort);
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t st = su32(sm + slot * STG),
                               wt = RES ? su32(wres) + (uint32_t)(2 * kc) * Cf::WG : st + 2 * Cf::HG;
                // two base descriptors per chunk; a tap's and an M tile's operands are constant offsets
                // (in 16-byte units) added to the start-address field, which never carries out of it
                // (shared-memory addresses stay below 2^14 x 16 B)
                const uint64_t da0 = umma_desc(st, Cf::HG, Cf::HW * 16), db0 = umma_desc(wt, Cf::WG, 128);
                const uint32_t d0 = tmem + (uint32_t)(buf * MT * NT);
                auto issue = [&](auto flipc) {
                    constexpr bool F = decltype(flipc)::value;
#pragma unroll
                    for (int t = 0; t < 9; t++) {
                        const int dy = F ? 1 - t / 3 : t / 3 - 1, dx = F ? 1 - t % 3 : t % 3 - 1;
                        const uint64_t db = db0 + (uint64_t)(t * NT);  // t * NT * 16 bytes
                        const uint32_t acc = (kc > 0 || t > 0) ? 1u : 0u;
#pragma unroll
                        for (int j = 0; j < MT; j++)
                            hx_mma(d0 + (uint32_t)(j * NT), da0 + (uint64_t)((1 + dy) * Cf::HW + 8 * j + 1 + dx), db,
                                   idesc, acc);
                    }
                };
                if (flip) issue(std::true_type{});
                else issue(std::false_type{});
                hx_commit(&empty[slot]);
                if (kc == nc - 1) hx_commit(&accf[buf]);
                consumed = q + 1;
                // refill the stage that chunk q - 1 used, once its MMAs (queued before this chunk's) finish
                if (issued < total) {
                    const int rs = (int)(issued % S);
                    if (issued >= S) ok = hx_wait(&empty[rs], (uint32_t)((issued / S - 1) & 1), abort);
                    if (ok) load(issued++);
                }
            }
            if (!ok) {
                atomicExch(err, 1);
                *abort = 1;
            }
            // wind down: every copy issued has landed and every MMA committed has finished
            for (long long q = consumed; q < issued; q++) hx_wait(&full[q % S], (uint32_t)((q / S) & 1), nullptr);
            if (!wdone) hx_wait(wbar, 0, nullptr);
            if (consumed > 0) {
                const long long q = consumed - 1;
                if (!hx_wait(&empty[q % S], (uint32_t)((q / S) & 1), nullptr)) atomicExch(err, 1);
            }
        }
    } else {
        // epilogue: warp w holds TMEM lanes 32w .. 32w + 31, the super-tile rows 4w .. 4w + 3
        const int m = warp * 32 + lane, r = m >> 3, cpx = m & 7;
        for (long long ti = 0; ti < my_tiles; ti++) {
            const int buf = (int)(ti % ACC);
            const bool ok = hx_wait(&accf[buf], (uint32_t)((ti / ACC) & 1), abort);
            if (!__all_sync(0xffffffffu, ok)) {  // the warp leaves together (tcgen05.ld is warp-collective)
                if (lane == 0) {
                    atomicExch(err, 1);
                    *abort = 1;
                }
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            int n, y0, x0;
            tile_at(ti, n, y0, x0);
            const int y = y0 + r;
#pragma unroll 1
            for (int j = 0; j < MT; j++) {
                const int x = x0 + 8 * j + cpx;
                const bool valid = y < H && x < W;
                const long long p = ((long long)n * H + y) * W + x;
#pragma unroll 1
                for (int cb = 0; cb < NT; cb += 16) {
                    uint32_t v[16];
                    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((buf * MT + j) * NT + cb);
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                        "%12, %13, %14, %15}, [%16];"
                        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                          "=r"(v[14]), "=r"(v[15])
                        : "r"(taddr));
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    if (!valid || cb >= Cout) continue;
                    const int nv = Cout - cb >= 16 ? 16 : 8;  // Cout % 8 == 0
                    float o[16];
#pragma unroll
                    for (int k = 0; k < 16; k++) {
                        o[k] = __uint_as_float(v[k]) + (bias && k < nv ? bias[cb + k] : 0.0f);
                        if (relu) o[k] = o[k] > 0.0f ? o[k] : 0.0f;
                    }
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        if (h * 8 >= nv) break;
                        const float *q8 = o + 8 * h;
                        if (Y) {
                            const uint4 pk = make_uint4(pack2(__float2bfloat16(q8[0]), __float2bfloat16(q8[1])),
                                                        pack2(__float2bfloat16(q8[2]), __float2bfloat16(q8[3])),
                                                        pack2(__float2bfloat16(q8[4]), __float2bfloat16(q8[5])),
                                                        pack2(__float2bfloat16(q8[6]), __float2bfloat16(q8[7])));
                            *reinterpret_cast<uint4 *>(Y + p * Cout + cb + 8 * h) = pk;
                        }
                        if (Yf) {
                            *reinterpret_cast<float4 *>(Yf + p * Cout + cb + 8 * h) =
                                make_float4(q8[0], q8[1], q8[2], q8[3]);
                            *reinterpret_cast<float4 *>(Yf + p * Cout + cb + 8 * h + 4) =
                                make_float4(q8[4], q8[5], q8[6], q8[7]);
                        }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(&acce[buf])) : "memory");
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// ---------------------------------------------------------------------------------------------
// Weight gradient dW[tap, co, ci] += sum over a chunk of pixels of dY[p, co] X[p + off(tap), ci].
// GEMM M = co (16 per block), N = ci (64 per block, 16 per warp), K = pixels (16 per step).  The
// fragments gather pixel pairs (NHWC keeps channels, not pixels, contiguous), so they are built
// from 16-bit loads.  grid = (pixel chunks, Cout/16 * ceil(Cin/64), 9).
// ---------------------------------------------------------------------------------------------
constexpr int kWgChunk = 1024;

__global__ void __launch_bounds__(128) k_conv3x3_wgrad(const bf16 *__restrict__ X, const bf16 *__restrict__ dY,
                                                       float *__restrict__ dW, int N, int H, int W, int Cin,
                                                       int Cout) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int tap = blockIdx.z, dy = tap / 3 - 1, dx = tap % 3 - 1;
    const int ntile_ci = (Cin + 63) / 64;
    const int co0 = (blockIdx.y / ntile_ci) * 16, ci_blk = (blockIdx.y % ntile_ci) * 64;
    const int ciw = ci_blk + warp * 16;  // this warp's 16 input channels (two n-tiles of 8)
    if (ciw >= Cin) return;
    const long long P = (long long)N * H * W;
    const long long pbeg = (long long)blockIdx.x * kWgChunk, pend = min(P, pbeg + kWgChunk);
    float acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    const unsigned short *dYs = reinterpret_cast<const unsigned short *>(dY);
    const unsigned short *Xs = reinterpret_cast<const unsigned short *>(X);
    // source offset of pixel p shifted by the tap, or -1 outside the image
    auto src = [&](long long p) -> long long {
        if (p >= pend) return -1;
        const long long hw = (long long)H * W;
        const int n = (int)(p / hw), q = (int)(p % hw), y = q / W + dy, x = q % W + dx;
        if (y < 0 || y >= H || x < 0 || x >= W) return -1;
        return ((long long)n * H + y) * W + x;
    };
    for (long long k0 = pbeg; k0 < pend; k0 += 16) {
        const long long pk[4] = {k0 + 2 * t, k0 + 2 * t + 1, k0 + 2 * t + 8, k0 + 2 * t + 9};
        unsigned short av[2][4];  // A rows g and g+8 (co), k columns pk[]
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const bool in = pk[i] < pend;
            av[0][i] = in ? dYs[pk[i] * Cout + co0 + g] : (unsigned short)0;
            av[1][i] = in ? dYs[pk[i] * Cout + co0 + g + 8] : (unsigned short)0;
        }
        uint32_t a[4] = {(uint32_t)av[0][0] | ((uint32_t)av[0][1] << 16), (uint32_t)av[1][0] | ((uint32_t)av[1][1] << 16),
                         (uint32_t)av[0][2] | ((uint32_t)av[0][3] << 16), (uint32_t)av[1][2] | ((uint32_t)av[1][3] << 16)};
        long long s[4];
#pragma unroll
        for (int i = 0; i < 4; i++) s[i] = src(pk[i]);
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int ci = ciw + j * 8 + g;
            unsigned short bv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) bv[i] = (s[i] >= 0 && ci < Cin) ? Xs[s[i] * Cin + ci] : (unsigned short)0;
            uint32_t b[2] = {(uint32_t)bv[0] | ((uint32_t)bv[1] << 16), (uint32_t)bv[2] | ((uint32_t)bv[3] << 16)};
            mma_bf16(acc[j], a, b);
        }
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const int ci = ciw + j * 8 + 2 * t;
        if (ci >= Cin) continue;
        float *w0 = dW + ((long long)tap * Cout + co0 + g) * Cin + ci;
        float *w1 = dW + ((long long)tap * Cout + co0 + g + 8) * Cin + ci;
        atomicAdd(w0, acc[j][0]);
        atomicAdd(w0 + 1, acc[j][1]);
        atomicAdd(w1, acc[j][2]);
        atomicAdd(w1 + 1, acc[j][3]);
    }
}

// ---------------------------------------------------------------------------------------------
// Point-wise and resampling kernels
// ---------------------------------------------------------------------------------------------
#define NN_GSTRIDE(i, n) \
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// dYm = dY * (Y > 0) (ReLU; relu == 0: identity) in BF16; db[c] += sum of dYm over pixels.
__global__ void k_relu_grad(const float *__restrict__ dY, const bf16 *__restrict__ Y, bf16 *__restrict__ dYm,
                            float *__restrict__ db, long long P, int C, int relu) {
    extern __shared__ float sdb[];
    for (int c = threadIdx.x; c < C; c += blockDim.x) sdb[c] = 0.0f;
    __syncthreads();
    NN_GSTRIDE(i, P * C) {
        float v = dY[i];
        if (relu && !(__bfloat162float(Y[i]) > 0.0f)) v = 0.0f;
        dYm[i] = __float2bfloat16(v);
        if (db) atomicAdd(&sdb[i % C], v);
    }
    __syncthreads();
    if (db)
        for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(&db[c], sdb[c]);
}

// 2x2 average pooling (H, W even): Y[n, y, x, c] = mean of X[n, 2y+i, 2x+j, c]
__global__ void k_pool2(const bf16 *__restrict__ X, bf16 *__restrict__ Y, int N, int H, int W, int C) {
    const int h = H / 2, w = W / 2;
    NN_GSTRIDE(i, (long long)N * h * w * C) {
        const int c = (int)(i % C);
        long long q = i / C;
        const int x = (int)(q % w);
        q /= w;
        const int y = (int)(q % h);
        const int n = (int)(q / h);
        const long long b = (((long long)n * H + 2 * y) * W + 2 * x) * C + c;
        const float s = __bfloat162float(X[b]) + __bfloat162float(X[b + C]) + __bfloat162float(X[b + (long long)W * C]) +
                        __bfloat162float(X[b + (long long)W * C + C]);
        Y[i] = __float2bfloat16(0.25f * s);
    }
}
// dX[n, y, x, c] (+)= dY[n, y/2, x/2, c] / 4   (acc: add into dX)
__global__ void k_pool2_grad(const float *__restrict__ dY, float *__restrict__ dX, int N, int H, int W, int C, int acc) {
    NN_GSTRIDE(i, (long long)N * H * W * C) {
        const int c = (int)(i % C);
        long long q = i / C;
        const int x = (int)(q % W);
        q /= W;
        const int y = (int)(q % H);
        const int n = (int)(q / H);
        const float v = 0.25f * dY[(((long long)n * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c];
        dX[i] = acc ? dX[i] + v : v;
    }
}
// nearest 2x upsampling plus a skip tensor: Y[n, y, x, c] = X[n, y/2, x/2, c] + S[n, y, x, c]
// (S may be null), computed in Float32, stored BF16.  (H, W: output size)
__global__ void k_up2_add(const bf16 *__restrict__ X, const bf16 *__restrict__ S, bf16 *__restrict__ Y, int N, int H,
                          int W, int C) {
    NN_GSTRIDE(i, (long long)N * H * W * C) {
        const int c = (int)(i % C);
        long long q = i / C;
        const int x = (int)(q % W);
        q /= W;
        const int y = (int)(q % H);
        const int n = (int)(q / H);
        float v = __bfloat162float(X[(((long long)n * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c]);
        if (S) v += __bfloat162float(S[i]);
        Y[i] = __float2bfloat16(v);
    }
}
// dX[n, y, x, c] = sum over the 2x2 children of dY   (H, W: the coarse size)
__global__ void k_up2_grad(const float *__restrict__ dY, float *__restrict__ dX, int N, int H, int W, int C) {
    NN_GSTRIDE(i, (long long)N * H * W * C) {
        const int c = (int)(i % C);
        long long q = i / C;
        const int x = (int)(q % W);
        q /= W;
        const int y = (int)(q % H);
        const int n = (int)(q / H);
        const long long W2 = 2LL * W;
        const long long b = (((long long)n * 2 * H + 2 * y) * W2 + 2 * x) * C + c;
        dX[i] = dY[b] + dY[b + C] + dY[b + W2 * C] + dY[b + W2 * C + C];
    }
}
// y (+)= x (Float32)
__global__ void k_axpy(const float *__restrict__ x, float *__restrict__ y, long long n, int acc) {
    NN_GSTRIDE(i, n) y[i] = acc ? y[i] + x[i] : x[i];
}
// mean squared error of channel 0 of Yf (C channels) against T over `count` pixels (mask: weights,
// may be null); dY gets 2 (y - t) w / count in channel 0 and 0 elsewhere; *loss += the sum.
__global__ void k_mse(const float *__restrict__ Yf, const float *__restrict__ T, const float *__restrict__ wgt,
                      float *__restrict__ dY, float *__restrict__ loss, long long P, int C, float inv_count) {
    float s = 0.0f;
    NN_GSTRIDE(i, P) {
        const float w = wgt ? wgt[i] : 1.0f;
        const float d = (Yf[i * C] - T[i]) * w;
        s += d * (Yf[i * C] - T[i]);
        dY[i * C] = 2.0f * d * inv_count;
        for (int c = 1; c < C; c++) dY[i * C + c] = 0.0f;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * inv_count);
}
// Adam (bias-corrected), Float32 master weights; refreshes the BF16 copy and, when WT is given,
// the per-tap transposed copy used by the input-gradient convolution (layout [9][Cout][Cin] ->
// [9][Cin][Cout]).
__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       bf16 *__restrict__ wb, bf16 *__restrict__ wt, long long n, int Cout, int Cin, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
    NN_GSTRIDE(i, n) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.0f - b1) * gi;
        float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        const bf16 b = __float2bfloat16(wi);
        if (wb) wb[i] = b;
        if (wt) {
            const long long per = (long long)Cout * Cin;
            const long long tap = i / per, r = i % per;
            const int co = (int)(r / Cin), ci = (int)(r % Cin);
            wt[tap * per + (long long)ci * Cout + co] = b;
        }
    }
}
// BF16 copy and per-tap transpose of a weight tensor (no update)
__global__ void k_wcast(const float *__restrict__ w, bf16 *__restrict__ wb, bf16 *__restrict__ wt, long long n,
                        int Cout, int Cin) {
    NN_GSTRIDE(i, n) {
        const bf16 b = __float2bfloat16(w[i]);
        wb[i] = b;
        if (wt) {
            const long long per = (long long)Cout * Cin;
            const long long tap = i / per, r = i % per;
            const int co = (int)(r / Cin), ci = (int)(r % Cin);
            wt[tap * per + (long long)ci * Cout + co] = b;
        }
    }
}
__global__ void k_zero(float *p, long long n) { NN_GSTRIDE(i, n) p[i] = 0.0f; }

// Input stack of the network from a State (column-major, x fastest = NHWC row order): channels
// h, b, N, zb, zs, ieb, mask, each (v - shift_c) * scale_c, padded with zeros to 16 channels and
// to Hp x Wp pixels.
__global__ void k_pack_state(const shk_state s, int nx, int ny, int Hp, int Wp, const float *__restrict__ norm,
                             bf16 *__restrict__ X) {
    NN_GSTRIDE(i, (long long)Hp * Wp) {
        const int x = (int)(i % Wp), y = (int)(i / Wp);
        float v[16];
#pragma unroll
        for (int c = 0; c < 16; c++) v[c] = 0.0f;
        if (x < nx && y < ny) {
            const size_t k = (size_t)x + (size_t)y * nx;
            const double f[7] = {s.h[k], s.b[k], s.N[k], s.zb[k], s.zs[k], s.ieb[k], s.mask[k]};
#pragma unroll
            for (int c = 0; c < 7; c++) v[c] = (float)((f[c] - (double)norm[2 * c]) * (double)norm[2 * c + 1]);
        }
        uint32_t *o = reinterpret_cast<uint32_t *>(X + i * 16);
#pragma unroll
        for (int c = 0; c < 8; c++) o[c] = pack2(__float2bfloat16(v[2 * c]), __float2bfloat16(v[2 * c + 1]));
    }
}
// h_seed = h + dh_scale * Yf[ch 0] on GROUNDED cells (mask == 0), h elsewhere
__global__ void k_apply_increment(const float *__restrict__ Yf, int C, int nx, int ny, int Wp, double dh_scale,
                                  const double *__restrict__ h, const double *__restrict__ mask,
                                  double *__restrict__ out) {
    NN_GSTRIDE(i, (long long)nx * ny) {
        const int x = (int)(i % nx), y = (int)(i / nx);
        const double dh = (double)Yf[((long long)y * Wp + x) * C] * dh_scale;
        out[i] = mask[i] == 0.0 ? h[i] + dh : h[i];
    }
}

static int grid_for(long long n) {
    long long b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

} // namespace nn
} // namespace shk

using namespace shk::nn;

// Per device: the tensor-core convolution's fault word (set when one of its bounded waits runs out).
static int *g_tc_fault[64] = {};

static int tc_fault_word(int dev, int **out) {
    if (dev < 0 || dev >= 64) return SHK_BAD_ARG;
    if (!g_tc_fault[dev]) {
        int *p = nullptr;
        if (cudaMalloc(&p, sizeof(int)) != cudaSuccess || cudaMemset(p, 0, sizeof(int)) != cudaSuccess)
            return SHK_CUDA_ERROR;
        g_tc_fault[dev] = p;
    }
    *out = g_tc_fault[dev];
    return SHK_OK;
}

template <int NT>
static int launch_conv_tc(const bf16 *x, const bf16 *w, const float *bias, bf16 *y, float *Yf, int N, int H, int W,
                          int Cin, int Cout, int relu, int flip, cudaStream_t s) {
    static int attr_done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int *fault = nullptr;
    if (int rc = tc_fault_word(dev, &fault)) return rc;
    if (!attr_done[dev]) {
        if (cudaFuncSetAttribute(k_conv3x3_tc<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TcLayout<NT>::bytes) != cudaSuccess)
            return SHK_CUDA_ERROR;
        attr_done[dev] = 1;
    }
    const long long P = (long long)N * H * W;
    k_conv3x3_tc<NT><<<(unsigned)((P + kTcM - 1) / kTcM), 128, TcLayout<NT>::bytes, s>>>(
        x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip, fault);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

typedef CUresult (*HxEncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                               const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                               CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static HxEncodeFn hx_encoder() {
    static HxEncodeFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *fp = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fp, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess && fp)
            fn = (HxEncodeFn)fp;
        else
            cudaGetLastError();
    }
    return fn;
}

// The halo-tile form; *launched = false (and SHK_OK) when its tensor maps cannot be built here.
template <int NT>
static int launch_conv_hx(const bf16 *x, const bf16 *w, const float *bias, bf16 *y, float *Yf, int N, int H, int W,
                          int Cin, int Cout, int relu, int flip, cudaStream_t s, bool *launched) {
    using Cf = HxCfg<NT>;
    *launched = false;
    const HxEncodeFn fn = hx_encoder();
    if (!fn || (uintptr_t)x % 16 || (uintptr_t)w % 16) return SHK_OK;
    static int attr_done[64] = {}, sms[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return SHK_BAD_ARG;
    int *fault = nullptr;
    if (int rc = tc_fault_word(dev, &fault)) return rc;
    if (!attr_done[dev]) {
        if (cudaFuncSetAttribute(k_conv3x3_hx<NT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Cf::bytes) != cudaSuccess ||
            cudaFuncSetAttribute(k_conv3x3_hx<NT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kHxMaxSmem) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return SHK_CUDA_ERROR;
        attr_done[dev] = 1;
    }
    // the weights stay resident in each CTA where they fit beside the halo stages (SHK_NN_HX_STREAM=1:
    // always restage them with every chunk)
    const char *ev = getenv("SHK_NN_HX_STREAM");
    const bool res = !(ev && atoi(ev) != 0) && Cf::res_bytes(Cin) <= kHxMaxSmem;
    CUtensorMap mx, mw;
    const cuuint64_t xd[4] = {(cuuint64_t)Cin, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    const cuuint64_t xs[3] = {(cuuint64_t)Cin * 2, (cuuint64_t)W * Cin * 2, (cuuint64_t)H * W * Cin * 2};
    const cuuint32_t xb[4] = {8, (cuuint32_t)Cf::HW, (cuuint32_t)Cf::HH, 1}, e4[4] = {1, 1, 1, 1};
    const cuuint64_t wd[3] = {(cuuint64_t)Cin, (cuuint64_t)Cout, 9};
    const cuuint64_t ws[2] = {(cuuint64_t)Cin * 2, (cuuint64_t)Cout * Cin * 2};
    const cuuint32_t wb[3] = {8, (cuuint32_t)NT, 9};
    if (fn(&mx, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(x), xd, xs, xb, e4,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
        fn(&mw, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16 *>(w), wd, ws, wb, e4,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return SHK_OK;
    const long long tiles = (long long)N * ((W + 8 * Cf::MT - 1) / (8 * Cf::MT)) * ((H + kHxRows - 1) / kHxRows);
    const int grid = (int)(tiles < sms[dev] ? tiles : sms[dev]);
    if (res)
        k_conv3x3_hx<NT, true><<<grid, kHxThreads, Cf::res_bytes(Cin), s>>>(mx, mw, bias, y, Yf, N, H, W, Cin, Cout,
                                                                           relu, flip, fault);
    else
        k_conv3x3_hx<NT, false><<<grid, kHxThreads, Cf::bytes, s>>>(mx, mw, bias, y, Yf, N, H, W, Cin, Cout, relu,
                                                                    flip, fault);
    *launched = true;
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

// Forms: the halo-tile tcgen05 kernel (default); SHK_NN_TC_GATHER=1 the tcgen05 kernel that gathers
// each tap's A tile (also the form used when tensor maps are unavailable); SHK_NN_MMA_SYNC=1 the
// mma.sync kernel (kept as the comparison for the tensor-core forms' tests).  The variables are read
// at every call.  N tile = Cout rounded up to 16 (<= 256).
extern "C" {

SHK_API int shk_nn_conv3x3(const void *X, const void *Wt, const float *bias, void *Y, float *Yf, int N, int H, int W,
                           int Cin, int Cout, int relu, int flip, void *stream) {
    if (!X || !Wt || (!Y && !Yf) || N < 1 || H < 1 || W < 1 || Cin % 16 || Cout % 8) return SHK_BAD_ARG;
    const long long P = (long long)N * H * W;
    cudaStream_t s = (cudaStream_t)stream;
    const bf16 *x = (const bf16 *)X, *w = (const bf16 *)Wt;
    bf16 *y = (bf16 *)Y;
    const char *e1 = getenv("SHK_NN_MMA_SYNC"), *e2 = getenv("SHK_NN_TC_GATHER");
    const bool legacy = e1 && atoi(e1) != 0, gather = e2 && atoi(e2) != 0;
    if (!legacy && !gather && Cout <= 256) {
        const int nt = (Cout + 15) / 16 * 16;
        bool launched = false;
        int rc = SHK_OK;
        if (nt <= 16) rc = launch_conv_hx<16>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip, s, &launched);
        else if (nt <= 32) rc = launch_conv_hx<32>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip, s, &launched);
        else if (nt <= 64) rc = launch_conv_hx<64>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip, s, &launched);
        else if (nt <= 128) rc = launch_conv_hx<128>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip, s, &launched);
        else rc = launch_conv_hx<256>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip, s, &launched);
        if (rc || launched) return rc;
    }
    if (!legacy && Cout <= 256) {
        const int nt = (Cout + 15) / 16 * 16;
        if (nt <= 16) return launch_conv_tc<16>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip, s);
        if (nt <= 32) return launch_conv_tc<32>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip, s);
        if (nt <= 64) return launch_conv_tc<64>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip, s);
        if (nt <= 128) return launch_conv_tc<128>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip, s);
        return launch_conv_tc<256>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip, s);
    }
    const int NT = Cout % 64 == 0 ? 64 : (Cout % 32 == 0 ? 32 : 8);
    dim3 grid((unsigned)((P + 63) / 64), (unsigned)(Cout / NT));
    if (NT == 64) k_conv3x3<64><<<grid, 128, 0, s>>>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip);
    else if (NT == 32) k_conv3x3<32><<<grid, 128, 0, s>>>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip);
    else k_conv3x3<8><<<grid, 128, 0, s>>>(x, w, bias, y, Yf, N, H, W, Cin, Cout, relu, flip);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

// The tensor-core convolution's fault word on the current device (1 when one of its bounded waits
// ran out since the last call), read and cleared; synchronises the device.
SHK_API int shk_nn_conv_fault(int *fault) {
    if (!fault) return SHK_BAD_ARG;
    int dev = 0;
    cudaGetDevice(&dev);
    int *w = nullptr;
    if (int rc = tc_fault_word(dev, &w)) return rc;
    if (cudaMemcpy(fault, w, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SHK_CUDA_ERROR;
    return cudaMemset(w, 0, sizeof(int)) == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_conv3x3_wgrad(const void *X, const void *dY, float *dW, int N, int H, int W, int Cin, int Cout,
                                 void *stream) {
    if (!X || !dY || !dW || Cin % 8 || Cout % 16) return SHK_BAD_ARG;
    const long long P = (long long)N * H * W;
    dim3 grid((unsigned)((P + kWgChunk - 1) / kWgChunk), (unsigned)((Cout / 16) * ((Cin + 63) / 64)), 9);
    k_conv3x3_wgrad<<<grid, 128, 0, (cudaStream_t)stream>>>((const bf16 *)X, (const bf16 *)dY, dW, N, H, W, Cin,
                                                            Cout);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_relu_grad(const float *dY, const void *Y, void *dYm, float *db, long long P, int C, int relu,
                             void *stream) {
    if (C < 1 || C > 4096) return SHK_BAD_ARG;
    k_relu_grad<<<grid_for(P * C), 256, C * sizeof(float), (cudaStream_t)stream>>>(dY, (const bf16 *)Y, (bf16 *)dYm,
                                                                                   db, P, C, relu);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_pool2(const void *X, void *Y, int N, int H, int W, int C, void *stream) {
    if (H % 2 || W % 2) return SHK_BAD_ARG;
    k_pool2<<<grid_for((long long)N * H * W * C / 4), 256, 0, (cudaStream_t)stream>>>((const bf16 *)X, (bf16 *)Y, N,
                                                                                        H, W, C);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_pool2_grad(const float *dY, float *dX, int N, int H, int W, int C, int acc, void *stream) {
    k_pool2_grad<<<grid_for((long long)N * H * W * C), 256, 0, (cudaStream_t)stream>>>(dY, dX, N, H, W, C, acc);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_up2_add(const void *X, const void *S, void *Y, int N, int H, int W, int C, void *stream) {
    if (H % 2 || W % 2) return SHK_BAD_ARG;
    k_up2_add<<<grid_for((long long)N * H * W * C), 256, 0, (cudaStream_t)stream>>>((const bf16 *)X, (const bf16 *)S,
                                                                                      (bf16 *)Y, N, H, W, C);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_up2_grad(const float *dY, float *dX, int N, int H, int W, int C, void *stream) {
    k_up2_grad<<<grid_for((long long)N * H * W * C), 256, 0, (cudaStream_t)stream>>>(dY, dX, N, H, W, C);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_axpy(const float *x, float *y, long long n, int acc, void *stream) {
    k_axpy<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(x, y, n, acc);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_mse(const float *Yf, const float *T, const float *wgt, float *dY, float *loss, long long P, int C,
                       float inv_count, void *stream) {
    k_mse<<<grid_for(P), 256, 0, (cudaStream_t)stream>>>(Yf, T, wgt, dY, loss, P, C, inv_count);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_adam(float *w, const float *g, float *m, float *v, void *wb, void *wt, long long n, int Cout,
                        int Cin, float lr, float b1, float b2, float eps, int step, void *stream) {
    if (step < 1) return SHK_BAD_ARG;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, (bf16 *)wb, (bf16 *)wt, n, Cout, Cin, lr, b1, b2,
                                                          eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_wcast(const float *w, void *wb, void *wt, long long n, int Cout, int Cin, void *stream) {
    k_wcast<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, (bf16 *)wb, (bf16 *)wt, n, Cout, Cin);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_zero(float *p, long long n, void *stream) {
    k_zero<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(p, n);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_pack_state(const shk_state *st, int nx, int ny, int Hp, int Wp, const float *norm, void *X,
                              void *stream) {
    if (!st || Hp < ny || Wp < nx) return SHK_BAD_ARG;
    k_pack_state<<<grid_for((long long)Hp * Wp), 256, 0, (cudaStream_t)stream>>>(*st, nx, ny, Hp, Wp, norm, (bf16 *)X);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

SHK_API int shk_nn_apply_increment(const float *Yf, int C, int nx, int ny, int Wp, double dh_scale, const double *h,
                                   const double *mask, double *out, void *stream) {
    k_apply_increment<<<grid_for((long long)nx * ny), 256, 0, (cudaStream_t)stream>>>(Yf, C, nx, ny, Wp, dh_scale, h,
                                                                                     mask, out);
    return cudaGetLastError() == cudaSuccess ? SHK_OK : SHK_CUDA_ERROR;
}

} // extern "C"
