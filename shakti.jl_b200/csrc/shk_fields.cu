// shk_fields.cu -- point-wise and stencil field kernels of libshakti_b200:
//   set_initial_conditions!, update_MFLS! assembly, the fused Picard tail, relax_h!, step_b!.
//
// Every value is produced with the reference's formula and evaluation order (the library is
// compiled with --fmad=false, so no a*b+c is contracted), which makes these kernels bit-identical
// to the reference's unfused kernels except for x^(1/n) (cbrt for n = 3, pow otherwise), which may
// differ from Julia's x^(1/n) in the last bit.  Fusion never changes a value: a face quantity needed by two cells is
// computed once from the same operands and shared.
#include <cuda_runtime.h>
#include <float.h>

#include <algorithm>

#include "shk_device.cuh"

namespace shk {

#define CI(ix, iy) ((size_t)(ix) + (size_t)(iy) * (size_t)nx)
#define XI(ix, iy) ((size_t)(ix) + (size_t)(iy) * (size_t)(nx + 1))
#define YI(ix, iy) ((size_t)(ix) + (size_t)(iy) * (size_t)nx)

// ---------------------------------------------------------------------------------------------
// Mask
// ---------------------------------------------------------------------------------------------

__global__ void k_mask8(int n, const double *__restrict__ mask, uint8_t *__restrict__ m8) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double m = mask[i];
        uint8_t c = M_UNKNOWN;
        if (m == 0.0) c = M_GROUNDED;
        else if (m == 1.0) c = M_OCEAN;
        else if (m == 2.0) c = M_LAND;
        else if (m == 3.0) c = M_OTHER;
        m8[i] = c;
    }
}

// compute_valid_x/y_kernel! (src/mask.jl:62-84) and apply_mask_to_sliding_x/y_kernel!
// (src/mask.jl:117-136): one thread per face.
__global__ void k_face_masks_and_sliding(int nx, int ny, const uint8_t *__restrict__ m8,
                                         double *valid_x, double *valid_y, double *ub_x, double *ub_y) {
    const long long nxf = (long long)(nx + 1) * ny, nyf = (long long)nx * (ny + 1);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nxf + nyf;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < nxf) {
            int f = (int)(i % (nx + 1)), iy = (int)(i / (nx + 1));
            bool interior = f > 0 && f < nx;
            double v = 1.0;
            bool both_grounded = false;
            if (interior) {
                uint8_t a = m8[CI(f - 1, iy)], b = m8[CI(f, iy)];
                v = (a != M_OTHER && b != M_OTHER) ? 1.0 : 0.0;
                both_grounded = a == M_GROUNDED && b == M_GROUNDED;
            }
            valid_x[i] = v;
            if (!interior || !both_grounded) ub_x[i] = 0.0;
        } else {
            long long j = i - nxf;
            int ix = (int)(j % nx), f = (int)(j / nx);
            bool interior = f > 0 && f < ny;
            double v = 1.0;
            bool both_grounded = false;
            if (interior) {
                uint8_t a = m8[CI(ix, f - 1)], b = m8[CI(ix, f)];
                v = (a != M_OTHER && b != M_OTHER) ? 1.0 : 0.0;
                both_grounded = a == M_GROUNDED && b == M_GROUNDED;
            }
            valid_y[j] = v;
            if (!interior || !both_grounded) ub_y[j] = 0.0;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// set_initial_conditions! (src/initial_conditions.jl:14-125), centre steps in reference order.
// ---------------------------------------------------------------------------------------------
__global__ void k_init_center(int n, Params P, shk_state s, const uint8_t *__restrict__ m8) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint8_t m = m8[i];
        const double lambda_coeff = 1.5;
        s.lambda[i] = lambda_coeff * s.A_visc[i];
        double b = s.b[i];
        b = (s.mask[i] != 0.0) ? 0.0 : b; // ifelse(mask != GROUNDED, 0, b)
        s.b[i] = b;
        double H = s.zs[i] - (s.zb[i] + b); // compute_H!
        s.H[i] = H;
        if (P.br != 0.0) s.beta[i] = jl_max(0.0, (P.br - b) / P.lr); // compute_beta!
        double po = P.rho_i * P.g * H; // compute_po!
        s.po[i] = po;
        double pw = po / 2;
        if (m == M_OCEAN) pw = P.p_atm - P.rho_sw * P.g * jl_min(s.zb[i], 0.0);
        else if (m == M_LAND || m == M_OTHER) pw = P.p_atm;
        s.pw[i] = pw;
        // compute_N! then compute_h!
        double d = po - pw;
        s.N[i] = (m == M_GROUNDED) ? d : copysign(0.0, d);
        s.h[i] = pw / (P.rho_w * P.g) + s.zb[i];
    }
}

// compute_abs_ub! (src/static_fields.jl:59-66)
__global__ void k_abs_ub(int nx, int ny, shk_state s) {
    const int n = nx * ny;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int ix = i % nx, iy = i / nx;
        double ubx_c = (s.ub_x[XI(ix, iy)] + s.ub_x[XI(ix + 1, iy)]) / 2;
        double uby_c = (s.ub_y[YI(ix, iy)] + s.ub_y[YI(ix, iy + 1)]) / 2;
        s.abs_ub[i] = sqrt(ubx_c * ubx_c + uby_c * uby_c);
    }
}

// compute_dpwdx!/dpwdy!, compute_dhdx!/dhdy!, compute_b_x!/b_y! (initial-condition order; the
// gradient edge faces are never written).
__global__ void k_init_faces(int nx, int ny, Params P, shk_state s) {
    const long long nxf = (long long)(nx + 1) * ny, nyf = (long long)nx * (ny + 1);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nxf + nyf;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < nxf) {
            int f = (int)(i % (nx + 1)), iy = (int)(i / (nx + 1));
            if (f > 0 && f < nx) {
                size_t a = CI(f - 1, iy), b = CI(f, iy);
                s.dpwdx[i] = ((s.pw[b] - s.pw[a]) / P.dx) * s.valid_x[i];
                s.dhdx[i] = ((s.h[b] - s.h[a]) / P.dx) * s.valid_x[i];
                s.b_x[i] = (s.b[b] + s.b[a]) / 2;
            } else {
                s.b_x[i] = s.b[CI(f == 0 ? 0 : nx - 1, iy)];
            }
        } else {
            long long j = i - nxf;
            int ix = (int)(j % nx), f = (int)(j / nx);
            if (f > 0 && f < ny) {
                size_t a = CI(ix, f - 1), b = CI(ix, f);
                s.dpwdy[j] = ((s.pw[b] - s.pw[a]) / P.dy) * s.valid_y[j];
                s.dhdy[j] = ((s.h[b] - s.h[a]) / P.dy) * s.valid_y[j];
                s.b_y[j] = (s.b[b] + s.b[a]) / 2;
            } else {
                s.b_y[j] = s.b[CI(ix, f == 0 ? 0 : ny - 1)];
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Face physics shared by the tail: q/Re (src/water_flux.jl:192-208) and taub (src/sliding_law.jl)
// ---------------------------------------------------------------------------------------------
struct FaceOut {
    double dh, dpw, q, re, taub, ub;
};

__device__ __forceinline__ void q_re(const Params &P, double bf, double grad, double &q, double &re) {
    double G = fabs(grad);
    double D = (bf * bf * bf * P.g * G) / (12 * (P.nu * P.nu));
    double R = 2 * D / (1 + sqrt(1 + 4 * P.omega * D));
    re = R;
    q = -jl_sign(grad) * P.nu * R;
}

// One face of any sliding law.  Nf/lf/abs_v already staggered; Cf the face coefficient.
__device__ __forceinline__ double taub_face(const Params &P, const Sliding &L, double Nf, double lf,
                                            double abs_v, double ub, double Cf) {
    if (L.kind == SHK_SLIDING_LINEAR) return Cf * Nf * ub;
    if (!(abs_v > 0)) return 0.0;
    double denom = (L.kind == SHK_SLIDING_REG_COULOMB_V0) ? L.v0 : jl_pow(fabs(Nf), P.n, P.n_int) * lf;
    // x^(1/n): for n = 3, cbrt (a fraction of pow's cost; it differs from pow(x, 1/3.0) by at most
    // about an ulp, within the tolerance the parity tests hold the pow-dependent fields to)
    const double ratio = abs_v / (abs_v + denom);
    return Nf * Cf * (P.root3 ? cbrt(ratio) : jl_pow(ratio, P.inv_n, -1)) * (ub / abs_v);
}

// Cell-centred quantities needed by faces.
struct CellQ {
    double h, pw, N, lam, aub;
};

template <bool FROM_H>
__device__ __forceinline__ CellQ load_cell(const Params &P, const shk_state &s, const uint8_t *m8, size_t c) {
    CellQ q;
    if (FROM_H) {
        q.h = s.h[c];
        q.pw = P.rho_w * P.g * (q.h - s.zb[c]);
        double d = s.po[c] - q.pw;
        q.N = (m8[c] == M_GROUNDED) ? d : copysign(0.0, d);
    } else {
        q.h = s.h[c];
        q.pw = s.pw[c];
        q.N = s.N[c];
    }
    q.lam = s.lambda[c];
    q.aub = s.abs_ub[c];
    return q;
}

// x- (dir 0) or y-face (dir 1) between cells a (west/south) and b (east/north); a or b may be absent
// at the domain edge (edge face: gradients read from memory, taub uses the one adjacent cell).
template <bool FROM_H>
__device__ __forceinline__ FaceOut face(const Params &P, const Sliding &L, const shk_state &s, int dir,
                                        size_t fi, bool interior, const CellQ &a, const CellQ &b,
                                        const CellQ &edge_cell) {
    FaceOut o;
    const double *dhf = dir == 0 ? s.dhdx : s.dhdy;
    const double *dpwf = dir == 0 ? s.dpwdx : s.dpwdy;
    const double *valid = dir == 0 ? s.valid_x : s.valid_y;
    const double *bface = dir == 0 ? s.b_x : s.b_y;
    const double *ubf = dir == 0 ? s.ub_x : s.ub_y;
    const double dd = dir == 0 ? P.dx : P.dy;
    if (interior && FROM_H) {
        double v = valid[fi];
        o.dh = ((b.h - a.h) / dd) * v;
        o.dpw = ((b.pw - a.pw) / dd) * v;
    } else {
        o.dh = dhf[fi];
        o.dpw = dpwf[fi];
    }
    q_re(P, bface[fi], o.dh, o.q, o.re);
    o.ub = ubf[fi];
    if (L.kind == SHK_SLIDING_PRESCRIBED) {
        o.taub = (dir == 0 ? s.taub_x : s.taub_y)[fi];
    } else {
        double Nf, lf, av;
        if (interior) {
            Nf = (b.N + a.N) / 2;
            lf = (b.lam + a.lam) / 2;
            av = (b.aub + a.aub) / 2;
        } else {
            Nf = edge_cell.N;
            lf = edge_cell.lam;
            av = edge_cell.aub;
        }
        double Cf = (L.kind == SHK_SLIDING_REG_COULOMB) ? L.C : (dir == 0 ? L.Cx : L.Cy)[fi];
        o.taub = taub_face(P, L, Nf, lf, av, o.ub, Cf);
    }
    return o;
}

// ---------------------------------------------------------------------------------------------
// Fused tail: compute_dhdxy!, compute_pw!, compute_dpwdxy!, compute_N!, compute_q_and_Re_xy!,
// compute_Re!, compute_taub_xy!, compute_mdot!, compute_K! (src/elliptic_solver.jl:193-206),
// plus the Picard check maxima max|h - h_prev| and max|h| (src/elliptic_solver.jl:162-163).
// FROM_H = false is the initial-condition variant: pw, N and the gradients are taken as set.
//
// One 32 x 8 tile per block iteration, one thread per cell: (1) the tile's cells and a one-cell
// halo (no corners) are loaded to shared memory with pw and N formed from h; (2) each of the
// tile's 33 x 8 x-faces and 32 x 9 y-faces is computed once (q, Re, taub from the reference's
// face formulas), the faces the tile owns are written, and the products the cells need
// (Re, ub*taub, q*dh, q*dpw) stay in shared memory; (3) each cell sums its four faces.
// ---------------------------------------------------------------------------------------------
constexpr int kTailW = kTX, kTailH = kTY;           // cells per tile
// 288 threads: the tile's 552 faces take two rounds (with 256 threads the third round would keep
// only 40 threads busy while the rest waited at the barrier)
constexpr int kTailThreads = 288;
constexpr int kTailHW = kTailW + 2, kTailHH = kTailH + 2; // with the halo
constexpr int kTailXF = (kTailW + 1) * kTailH;      // x-faces of a tile
constexpr int kTailYF = kTailW * (kTailH + 1);      // y-faces of a tile

struct FaceSm {
    double re, ut, qd, qp;  // Re, ub*taub, q*dh, q*dpw
};

template <bool FROM_H, bool CHECK>
__device__ __forceinline__ void tail_body(Blk B, int nx, int ny, const Params &P, const Sliding &L,
                                          const shk_state &s, const uint8_t *__restrict__ m8,
                                          const double *__restrict__ h_prev, double *partials, unsigned int *counter,
                                          PicDev *pic) {
    __shared__ CellQ cq[kTailHH][kTailHW];
    __shared__ FaceSm fx[kTailXF], fy[kTailYF];
    const int tiles_x = (nx + kTailW - 1) / kTailW, ntiles = tiles_x * ((ny + kTailH - 1) / kTailH);
    const int tid = threadIdx.x, tx = tid % kTailW, ty = tid / kTailW;
    double red[2] = {0.0, 0.0};
    for (int t = B.id; t < ntiles; t += B.n) {
        const int x0 = (t % tiles_x) * kTailW, y0 = (t / tiles_x) * kTailH;
        // (1) cells of the tile and its halo
        for (int k = tid; k < kTailHH * kTailHW; k += kTailThreads) {
            const int hx = k % kTailHW, hy = k / kTailHW, ix = x0 - 1 + hx, iy = y0 - 1 + hy;
            const bool corner = (hx == 0 || hx == kTailHW - 1) && (hy == 0 || hy == kTailHH - 1);
            if (corner || ix < 0 || ix >= nx || iy < 0 || iy >= ny) continue;
            cq[hy][hx] = load_cell<FROM_H>(P, s, m8, CI(ix, iy));
        }
        __syncthreads();
        // (2) faces
        for (int k = tid; k < kTailXF + kTailYF; k += kTailThreads) {
            if (k < kTailXF) {
                const int fc = k % (kTailW + 1), row = k / (kTailW + 1), f = x0 + fc, iy = y0 + row;
                if (iy >= ny || f > nx) continue;
                const bool interior = f > 0 && f < nx;
                const CellQ &a = cq[row + 1][f > 0 ? fc : fc + 1];      // west cell (east cell at f = 0)
                const CellQ &b = cq[row + 1][f < nx ? fc + 1 : fc];     // east cell (west cell at f = nx)
                const size_t fi = XI(f, iy);
                const FaceOut o = face<FROM_H>(P, L, s, 0, fi, interior, a, b, f > 0 ? a : b);
                if ((fc < kTailW && f < nx) || f == nx) {
                    if (interior && FROM_H) {
                        s.dhdx[fi] = o.dh;
                        s.dpwdx[fi] = o.dpw;
                    }
                    s.q_x[fi] = o.q;
                    s.Re_x[fi] = o.re;
                    if (L.kind != SHK_SLIDING_PRESCRIBED) s.taub_x[fi] = o.taub;
                }
                fx[k] = FaceSm{o.re, o.ub * o.taub, o.q * o.dh, o.q * o.dpw};
            } else {
                const int kk = k - kTailXF, col = kk % kTailW, frow = kk / kTailW, ix = x0 + col, f = y0 + frow;
                if (ix >= nx || f > ny) continue;
                const bool interior = f > 0 && f < ny;
                const CellQ &a = cq[f > 0 ? frow : frow + 1][col + 1];  // south cell (north cell at f = 0)
                const CellQ &b = cq[f < ny ? frow + 1 : frow][col + 1]; // north cell (south cell at f = ny)
                const size_t fi = YI(ix, f);
                const FaceOut o = face<FROM_H>(P, L, s, 1, fi, interior, a, b, f > 0 ? a : b);
                if ((frow < kTailH && f < ny) || f == ny) {
                    if (interior && FROM_H) {
                        s.dhdy[fi] = o.dh;
                        s.dpwdy[fi] = o.dpw;
                    }
                    s.q_y[fi] = o.q;
                    s.Re_y[fi] = o.re;
                    if (L.kind != SHK_SLIDING_PRESCRIBED) s.taub_y[fi] = o.taub;
                }
                fy[kk] = FaceSm{o.re, o.ub * o.taub, o.q * o.dh, o.q * o.dpw};
            }
        }
        __syncthreads();
        // (3) cells
        const int ix = x0 + tx, iy = y0 + ty;
        if (tid < kTailW * kTailH && ix < nx && iy < ny) {
            const size_t c = CI(ix, iy);
            const CellQ &q0 = cq[ty + 1][tx + 1];
            const FaceSm &W = fx[ty * (kTailW + 1) + tx], &E = fx[ty * (kTailW + 1) + tx + 1];
            const FaceSm &S = fy[ty * kTailW + tx], &Nf = fy[(ty + 1) * kTailW + tx];
            if (FROM_H) {
                s.pw[c] = q0.pw;
                s.N[c] = q0.N;
            }
            // compute_Re! (src/water_flux.jl:107-112)
            const double Re_c = (W.re + E.re + S.re + Nf.re) / 4;
            s.Re[c] = Re_c;
            // compute_mdot! (src/melt_rate.jl:106-137)
            const double sh = fabs((E.ut + W.ut) / 2 + (Nf.ut + S.ut) / 2);
            const double pot = fabs((E.qd + W.qd) / 2 + (Nf.qd + S.qd) / 2);
            s.shear[c] = sh;
            s.potential[c] = pot;
            if (P.with_sensible) {
                const double sens = (E.qp + W.qp) / 2 + (Nf.qp + S.qp) / 2;
                s.sensible[c] = sens;
                s.mdot[c] = P.Linv * (s.G[c] + sh + P.rho_w * P.g * pot + P.ct * P.cw * P.rho_w * sens);
            } else {
                s.mdot[c] = P.Linv * (s.G[c] + sh + P.rho_w * P.g * pot);
            }
            // compute_K! (src/water_flux.jl:221-226)
            const double bb = s.b[c];
            s.K[c] = (bb * bb * bb * P.g) / (12 * P.nu * (1 + P.omega * Re_c));
            if (CHECK) {
                red[0] = jl_max(red[0], fabs(q0.h - h_prev[c]));
                red[1] = jl_max(red[1], fabs(q0.h));
            }
        }
        __syncthreads();  // the next tile reuses the shared arrays
    }
    if (CHECK) {
        double out[2];
        if (grid_reduce<2, true>(B, red, partials, counter, out) && threadIdx.x == 0) {
            pic->dmax = out[0];
            pic->hmax = out[1];
        }
    }
}

template <bool FROM_H, bool CHECK>
__global__ void __launch_bounds__(kTailThreads, kTailBlocksPerSm) k_tail(int nx, int ny, Params P, Sliding L, shk_state s,
                                                      const uint8_t *__restrict__ m8,
                                                      const double *__restrict__ h_prev, double *partials,
                                                      unsigned int *counter, PicDev *pic) {
    tail_body<FROM_H, CHECK>(grid_blk(), nx, ny, P, L, s, m8, h_prev, partials, counter, pic);
}

// ---------------------------------------------------------------------------------------------
// Assembly: update_MFLS_kernel! / update_MFLS_parabolic_kernel! (src/linear_solver.jl:438-588)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double dirichlet_head(const Params &P, uint8_t m, double zb) {
    if (m == M_OCEAN) {
        double pw_bc = P.p_atm - P.rho_sw * P.g * jl_min(zb, 0.0);
        return pw_bc / (P.rho_w * P.g) + zb;
    }
    return P.p_atm / (P.rho_w * P.g) + zb;
}

// boundary_K_face (src/k_face_scheme.jl:52-61)
__device__ __forceinline__ double bK(int kfs, double K1, double K2, uint8_t m2) {
    if (m2 == M_OTHER) return 0.0;
    if (m2 == M_OCEAN || m2 == M_LAND) return K1;
    if (kfs == SHK_KFACE_HARMONIC) return (2 * K1 * K2) / (K1 + K2 + DBL_EPSILON);
    return (K1 + K2) / 2;
}

template <bool PARABOLIC>
__device__ __forceinline__ void assemble_body(Blk B, int nx, int ny, const Params &P, int kfs, double dt,
                                              const shk_state &s, const uint8_t *__restrict__ m8,
                                              double *__restrict__ aP, double *__restrict__ aE,
                                              double *__restrict__ aN, double *__restrict__ rhs,
                                              double *__restrict__ h_prev) {
    Tiles T(nx, ny);
    for (int t = B.id; t < T.ntiles; t += B.n) {
        int ix, iy;
        T.cell(t, ix, iy);
        if (ix >= nx || iy >= ny) continue;
        const size_t c = CI(ix, iy);
        // every input is loaded before the first branch, so that the loads are in flight together
        // (the Dirichlet and OTHER_BASIN rows use few of them)
        const bool hE = ix < nx - 1, hW = ix > 0, hN = iy < ny - 1, hS = iy > 0;
        const uint8_t m = m8[c];
        const uint8_t mE = hE ? m8[c + 1] : 0, mW = hW ? m8[c - 1] : 0, mN = hN ? m8[c + nx] : 0,
                      mS = hS ? m8[c - nx] : 0;
        const double h = s.h[c], zb = s.zb[c], K = s.K[c];
        const double KE = hE ? s.K[c + 1] : 0.0, KW = hW ? s.K[c - 1] : 0.0, KN = hN ? s.K[c + nx] : 0.0,
                     KS = hS ? s.K[c - nx] : 0.0;
        const double Nc = s.N[c], A = s.A_visc[c], b = s.b[c], mdot = s.mdot[c], beta = s.beta[c],
                     aub = s.abs_ub[c], ieb = s.ieb[c];
        if (h_prev) h_prev[c] = h;
        double oP, oE = 0.0, oN = 0.0, orhs;
        if (is_dirichlet(m)) {
            oP = 1;
            orhs = dirichlet_head(P, m, zb);
        } else if (m == M_OTHER) {
            oP = 1;
            orhs = h;
        } else {
            double eE = 0.0, eW = 0.0, eN = 0.0, eS = 0.0;
            if (hE) eE = bK(kfs, K, KE, mE) / P.dx2;
            if (hW) eW = bK(kfs, K, KW, mW) / P.dx2;
            if (hN) eN = bK(kfs, K, KN, mN) / P.dy2;
            if (hS) eS = bK(kfs, K, KS, mS) / P.dy2;
            const double Nn = jl_pow(fabs(Nc), P.nm1, P.nm1_int);
            if (PARABOLIC) oP = (eE + eW + eN + eS) + P.e_v / dt;
            else oP = (eE + eW + eN + eS) + P.n * P.rho_w * P.g * A * Nn * b;
            double drhs = 0.0;
            if (ix < nx - 1) {
                if (is_dirichlet(mE)) drhs += eE * dirichlet_head(P, mE, s.zb[c + 1]);
                else oE = eE;
            }
            if (ix > 0 && is_dirichlet(mW)) drhs += eW * dirichlet_head(P, mW, s.zb[c - 1]);
            if (iy < ny - 1) {
                if (is_dirichlet(mN)) drhs += eN * dirichlet_head(P, mN, s.zb[c + nx]);
                else oN = eN;
            }
            if (iy > 0 && is_dirichlet(mS)) drhs += eS * dirichlet_head(P, mS, s.zb[c - nx]);
            if (PARABOLIC)
                orhs = mdot * (1 / P.rho_w - 1 / P.rho_i) - beta * aub + A * Nn * Nc * b + ieb + (P.e_v / dt) * h +
                       drhs;
            else
                orhs = mdot * (1 / P.rho_w - 1 / P.rho_i) - beta * aub + A * Nn * Nc * b +
                       A * Nn * (P.n * P.rho_w * P.g * h) * b + ieb + drhs;
        }
        aP[c] = oP;
        aE[c] = oE;
        aN[c] = oN;
        rhs[c] = orhs;
    }
}

template <bool PARABOLIC>
__global__ void __launch_bounds__(kThreads, kAsmBlocksPerSm) k_assemble(int nx, int ny, Params P, int kfs, double dt,
                                                       shk_state s, const uint8_t *__restrict__ m8,
                                                       double *__restrict__ aP, double *__restrict__ aE,
                                                       double *__restrict__ aN, double *__restrict__ rhs,
                                                       double *__restrict__ h_prev) {
    assemble_body<PARABOLIC>(grid_blk(), nx, ny, P, kfs, dt, s, m8, aP, aE, aN, rhs, h_prev);
}

__global__ void k_export_mfls(int nx, int ny, const double *aP, const double *aE, const double *aN,
                              const double *rhs, double *oP, double *oE, double *oW, double *oN, double *oS,
                              double *orhs) {
    const int n = nx * ny;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int ix = i % nx, iy = i / nx;
        if (oP) oP[i] = aP[i];
        if (oE) oE[i] = aE[i];
        if (oN) oN[i] = aN[i];
        if (oW) oW[i] = ix > 0 ? aE[i - 1] : 0.0;
        if (oS) oS[i] = iy > 0 ? aN[i - nx] : 0.0;
        if (orhs) orhs[i] = rhs[i];
    }
}

// relax_h! (src/elliptic_solver.jl:42-46)
__global__ void k_relax(int n, double alpha, double *h, const double *h_prev) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        h[i] = alpha * h[i] + (1 - alpha) * h_prev[i];
}

// compute_b_implicit/explicit_kernel! (src/gap_height.jl:117-135) then compute_beta! (:47-52).
template <bool IMPLICIT>
__device__ __forceinline__ void gap_b_body(Blk B, int n, const Params &P, double dt, const shk_state &s) {
    for (int i = B.id * blockDim.x + threadIdx.x; i < n; i += B.n * blockDim.x) {
        double b = s.b[i];
        if (s.mask[i] == 0.0) {
            const double Nc = s.N[i];
            const double Nn = jl_pow(fabs(Nc), P.nm1, P.nm1_int);
            double bnew;
            if (IMPLICIT)
                bnew = (b + dt * (s.mdot[i] / P.rho_i + s.beta[i] * s.abs_ub[i])) / (1 + dt * s.A_visc[i] * Nn * Nc);
            else
                bnew = b + dt * (s.mdot[i] / P.rho_i + s.beta[i] * s.abs_ub[i] - s.A_visc[i] * Nn * Nc * b);
            b = jl_clamp(bnew, P.b_min, P.b_max);
            s.b[i] = b;
        }
        if (P.br != 0.0) s.beta[i] = jl_max(0.0, (P.br - b) / P.lr);
    }
}

template <bool IMPLICIT>
__global__ void k_gap_b(int n, Params P, double dt, shk_state s, const uint8_t *__restrict__ m8) {
    gap_b_body<IMPLICIT>(grid_blk(), n, P, dt, s);
}

// compute_b_x!/compute_b_y! (src/gap_height.jl:75-108)
__device__ __forceinline__ void gap_faces_body(Blk B, int nx, int ny, const shk_state &s) {
    const long long nxf = (long long)(nx + 1) * ny, nyf = (long long)nx * (ny + 1);
    for (long long i = B.id * (long long)blockDim.x + threadIdx.x; i < nxf + nyf;
         i += (long long)B.n * blockDim.x) {
        if (i < nxf) {
            int f = (int)(i % (nx + 1)), iy = (int)(i / (nx + 1));
            double v;
            if (f == 0) v = s.b[CI(0, iy)];
            else if (f == nx) v = s.b[CI(nx - 1, iy)];
            else v = (s.b[CI(f, iy)] + s.b[CI(f - 1, iy)]) / 2;
            s.b_x[i] = v;
        } else {
            long long j = i - nxf;
            int ix = (int)(j % nx), f = (int)(j / nx);
            double v;
            if (f == 0) v = s.b[CI(ix, 0)];
            else if (f == ny) v = s.b[CI(ix, ny - 1)];
            else v = (s.b[CI(ix, f)] + s.b[CI(ix, f - 1)]) / 2;
            s.b_y[j] = v;
        }
    }
}
__global__ void k_gap_faces(int nx, int ny, shk_state s) { gap_faces_body(grid_blk(), nx, ny, s); }

__global__ void k_fill(size_t n, double *dst, double v, const double *base) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = base ? v + base[i] : v;
}

// ---------------------------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------------------------
static int flat_grid(Ctx *c, long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    long long cap = (long long)c->num_sms * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

int build_mask8(Ctx *c) {
    const int n = c->nx * c->ny;
    k_mask8<<<flat_grid(c, n), kThreads, 0, c->stream>>>(n, c->st.mask, c->mask8);
    c->launches++;
    return check_launch(c, "k_mask8");
}

// One resident wave of the tail (kTailBlocksPerSm blocks per SM), striding over the tiles.
static int tail_grid(const Ctx *c) {
    const long long tiles = (long long)((c->nx + kTailW - 1) / kTailW) * ((c->ny + kTailH - 1) / kTailH);
    return (int)std::max(1LL, std::min(tiles, (long long)c->num_sms * kTailBlocksPerSm));
}

int launch_initial_conditions(Ctx *c) {
    const int nx = c->nx, ny = c->ny, n = nx * ny;
    const long long nf = (long long)(nx + 1) * ny + (long long)nx * (ny + 1);
    int rc = build_mask8(c);
    if (rc) return rc;
    k_face_masks_and_sliding<<<flat_grid(c, nf), kThreads, 0, c->stream>>>(nx, ny, c->mask8, c->st.valid_x,
                                                                            c->st.valid_y, c->st.ub_x, c->st.ub_y);
    c->launches++;
    if ((rc = check_launch(c, "k_face_masks_and_sliding"))) return rc;
    k_init_center<<<flat_grid(c, n), kThreads, 0, c->stream>>>(n, c->P, c->st, c->mask8);
    c->launches++;
    if ((rc = check_launch(c, "k_init_center"))) return rc;
    k_abs_ub<<<flat_grid(c, n), kThreads, 0, c->stream>>>(nx, ny, c->st);
    c->launches++;
    if ((rc = check_launch(c, "k_abs_ub"))) return rc;
    k_init_faces<<<flat_grid(c, nf), kThreads, 0, c->stream>>>(nx, ny, c->P, c->st);
    c->launches++;
    if ((rc = check_launch(c, "k_init_faces"))) return rc;
    k_tail<false, false><<<tail_grid(c), kTailThreads, 0, c->stream>>>(nx, ny, c->P, c->SL, c->st, c->mask8, nullptr,
                                                                       c->partials, c->counter, nullptr);
    c->launches++;
    return check_launch(c, "k_tail<init>");
}

int launch_assemble(Ctx *c, int parabolic, double dt, bool copy_h_prev) {
    double *hp = copy_h_prev ? c->h_prev : nullptr;
    const long long tiles = (long long)((c->nx + kTX - 1) / kTX) * ((c->ny + kTY - 1) / kTY);
    const int grid = (int)std::max(1LL, std::min(tiles, (long long)c->num_sms * kAsmBlocksPerSm));
    if (parabolic)
        k_assemble<true><<<grid, kThreads, 0, c->stream>>>(c->nx, c->ny, c->P, c->kfs, dt, c->st, c->mask8,
                                                                      c->aP, c->aE, c->aN, c->rhs, hp);
    else
        k_assemble<false><<<grid, kThreads, 0, c->stream>>>(c->nx, c->ny, c->P, c->kfs, dt, c->st, c->mask8,
                                                                       c->aP, c->aE, c->aN, c->rhs, hp);
    c->launches++;
    return check_launch(c, "k_assemble");
}

int launch_export_mfls(Ctx *c, double *aP, double *aE, double *aW, double *aN, double *aS, double *rhs) {
    const int n = c->nx * c->ny;
    k_export_mfls<<<flat_grid(c, n), kThreads, 0, c->stream>>>(c->nx, c->ny, c->aP, c->aE, c->aN, c->rhs, aP, aE, aW,
                                                                aN, aS, rhs);
    c->launches++;
    return check_launch(c, "k_export_mfls");
}

int launch_tail(Ctx *c, bool picard_check) {
    if (picard_check)
        k_tail<true, true><<<tail_grid(c), kTailThreads, 0, c->stream>>>(c->nx, c->ny, c->P, c->SL, c->st, c->mask8,
                                                                        c->h_prev, c->partials, c->counter,
                                                                        &c->dev->pic);
    else
        k_tail<true, false><<<tail_grid(c), kTailThreads, 0, c->stream>>>(c->nx, c->ny, c->P, c->SL, c->st, c->mask8,
                                                                         nullptr, c->partials, c->counter, nullptr);
    c->launches++;
    return check_launch(c, "k_tail");
}

int launch_relax(Ctx *c, double alpha, const double *h_prev) {
    const int n = c->nx * c->ny;
    k_relax<<<flat_grid(c, n), kThreads, 0, c->stream>>>(n, alpha, c->st.h, h_prev);
    c->launches++;
    return check_launch(c, "k_relax");
}

int launch_step_b(Ctx *c, double dt) {
    const int nx = c->nx, ny = c->ny, n = nx * ny;
    const long long nf = (long long)(nx + 1) * ny + (long long)nx * (ny + 1);
    if (c->gap == SHK_GAP_IMPLICIT)
        k_gap_b<true><<<flat_grid(c, n), kThreads, 0, c->stream>>>(n, c->P, dt, c->st, c->mask8);
    else
        k_gap_b<false><<<flat_grid(c, n), kThreads, 0, c->stream>>>(n, c->P, dt, c->st, c->mask8);
    c->launches++;
    int rc = check_launch(c, "k_gap_b");
    if (rc) return rc;
    k_gap_faces<<<flat_grid(c, nf), kThreads, 0, c->stream>>>(nx, ny, c->st);
    c->launches++;
    return check_launch(c, "k_gap_faces");
}

int launch_fill(Ctx *c, double *dst, double v, size_t n) {
    k_fill<<<flat_grid(c, (long long)n), kThreads, 0, c->stream>>>(n, dst, v, nullptr);
    c->launches++;
    return check_launch(c, "k_fill");
}

int launch_fill_plus_base(Ctx *c, double *dst, double v, const double *base, size_t n) {
    k_fill<<<flat_grid(c, (long long)n), kThreads, 0, c->stream>>>(n, dst, v, base);
    c->launches++;
    return check_launch(c, "k_fill");
}

// ---------------------------------------------------------------------------------------------
// Ensemble: the same bodies over every instance in one grid (block -> instance table per family).
// Instances whose Picard loop has finished this timestep return at once.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_ens_assemble(EnsInst *E, const int *b2i) {
    __shared__ EnsInst I;
    const Blk B = ens_stage(I, E, b2i, EF_STENCIL);
    if (!I.pic_active) return;
    assemble_body<false>(B, I.nx, I.ny, I.P, I.kfs, 0.0, I.st, I.mask8, I.aP, I.aE, I.aN, I.rhs, I.h_prev);
}

__global__ void __launch_bounds__(kTailThreads, kTailBlocksPerSm) k_ens_tail(EnsInst *E, const int *b2i) {
    __shared__ EnsInst I;
    const Blk B = ens_stage(I, E, b2i, EF_TAIL);
    if (!I.pic_active) return;
    tail_body<true, true>(B, I.nx, I.ny, I.P, I.SL, I.st, I.mask8, I.h_prev, I.partials, I.counter, I.pic);
}

// step_b!: gap update of the cells, then the face averages (two launches: the faces read
// neighbouring cells' new b)
__global__ void __launch_bounds__(kThreads) k_ens_gap_cells(EnsInst *E, const int *b2i, const EnsCtl *ctl) {
    __shared__ EnsInst I;
    const Blk B = ens_stage(I, E, b2i, EF_FLAT);
    const double dt = ctl->dt;
    if (I.gap == SHK_GAP_IMPLICIT) gap_b_body<true>(B, I.nx * I.ny, I.P, dt, I.st);
    else gap_b_body<false>(B, I.nx * I.ny, I.P, dt, I.st);
}
__global__ void __launch_bounds__(kThreads) k_ens_gap_faces(EnsInst *E, const int *b2i) {
    __shared__ EnsInst I;
    const Blk B = ens_stage(I, E, b2i, EF_FLAT);
    gap_faces_body(B, I.nx, I.ny, I.st);
}

void ens_assemble(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks) {
    k_ens_assemble<<<nblocks, kThreads, 0, s>>>(E, b2i);
}
void ens_tail(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks) {
    k_ens_tail<<<nblocks, kTailThreads, 0, s>>>(E, b2i);
}
void ens_gap(cudaStream_t s, EnsInst *E, const int *b2i, int nblocks, const EnsCtl *ctl) {
    k_ens_gap_cells<<<nblocks, kThreads, 0, s>>>(E, b2i, ctl);
    k_ens_gap_faces<<<nblocks, kThreads, 0, s>>>(E, b2i);
}

} // namespace shk
