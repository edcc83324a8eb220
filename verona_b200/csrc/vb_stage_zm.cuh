// Z-marching 3D stage kernel ("2.5D" blocking), templated on the bulk type R.
//
// Same arithmetic, per cell, as the box-tile k_stage and as the reference
// (src/3dim/algos.jl:14-200 + src/3dim/structs.jl:218-628), organised for the
// hardware:
//   * a CTA owns TX x TY columns and walks one z-range of LZ cells; each
//     thread owns one (x, y) column;
//   * the z-stencil of a column (planes k-1 .. k+3, all five variables)
//     lives in registers and slides up one plane per step, so every z-face
//     is reconstructed once and the z-halo is read once per range;
//   * only the current plane k, with its 3-cell x/y halo (corners skipped),
//     is staged in shared memory for the x- and y-stencils;
//   * each cell is reconstructed once per axis: its right-face value goes to
//     shared memory, its left-face value stays in the thread, and one thread
//     per face computes the flux; the halo cells of the tile add TY (x) and
//     TX (y) extra reconstructions and faces per plane;
//   * all tile geometry is compile-time, so index arithmetic is shifts.
// The flux difference is accumulated in FP64 in the reference's order
// (x, y, z), then the RK combination, con2prim (guess = this stage's P) and
// the floors, as in k_stage.
#pragma once
#include "vb_ns.h"
#include <type_traits>

#include "vb_stage.cuh"

namespace VB_NS {

template <int TX, int TY> struct ZmGeom {
    static constexpr int NV = 5, NT = TX * TY;
    static constexpr int EX = TX + 6, EY = TY + 6;
    static constexpr int PLN = EX * EY;
    static constexpr int FXN = (TX + 1) * TY, FYN = TX * (TY + 1);
    static constexpr int FN = FXN > FYN ? FXN : FYN;
    static constexpr int QXN = TX > TY ? TX : TY;
    static constexpr int ZR = 5;        // z-window ring: planes k-1 .. k+3
    static constexpr int YHN = 2 * TX;  // y-halo face states: ql of row -1, qr of row TY
    template <typename R> static constexpr size_t smem_bytes() {
        return sizeof(R) * NV * (size_t)(PLN + 2 * FN + QXN + ZR * NT + YHN);
    }
};

// Flux-difference accumulator. FP64: the reference's order,
// U - dtdx*dFx - dtdy*dFy - dtdz*dFz in FP64. FP32 bulk: the divergence
// dtdx*dFx + dtdy*dFy + dtdz*dFz in FP32, subtracted from U in FP64.
template <typename R> struct DivAcc;
template <> struct DivAcc<double> {
    double a[5];
    __device__ __forceinline__ void init(const double* Us, long long vs, long long c) {
#pragma unroll
        for (int v = 0; v < 5; ++v) a[v] = Us[v * vs + c];
    }
    __device__ __forceinline__ void sub(int v, double coef, double fhi, double flo) { a[v] = a[v] - coef * (fhi - flo); }
    __device__ __forceinline__ double result(int v, const double*, long long, long long) const { return a[v]; }
};
template <> struct DivAcc<float> {
    float a[5];
    __device__ __forceinline__ void init(const double*, long long, long long) {
#pragma unroll
        for (int v = 0; v < 5; ++v) a[v] = 0.0f;
    }
    __device__ __forceinline__ void sub(int v, double coef, float fhi, float flo) { a[v] += (float)coef * (fhi - flo); }
    __device__ __forceinline__ double result(int v, const double* Us, long long vs, long long c) const {
        return Us[v * vs + c] - (double)a[v];
    }
};

template <int REC, typename R>
__device__ __forceinline__ void recon_floored(const R* q, int s, R fl, int v, R& qr, R& ql) {
    recon<REC>(q[-2 * s], q[-s], q[0], q[s], q[2 * s], qr, ql);
    if (v < 2) {  // face floor of rho and u (src/3dim/algos.jl:112-115)
        qr = jmax(fl, qr);
        ql = jmax(fl, ql);
    }
}

template <int REC, int RS, typename R, int TX, int TY, int LZ, int MINB, bool SPLIT>
__global__ void __launch_bounds__(TX * TY, MINB) k_stage_zm(StageParams p, StageBufs<R> b) {
    using G = ZmGeom<TX, TY>;
    constexpr int NV = 5, NT = G::NT, EX = G::EX, PLN = G::PLN, FN = G::FN, QXN = G::QXN;
    constexpr int FXR = TX + 1;  // x faces per row
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sPl = reinterpret_cast<R*>(smem_raw);  // [NV][EY][EX], plane k with x/y halo
    R* sQL = sPl + NV * PLN;                    // [NV][FN], left states of the faces
    R* sF = sQL + NV * FN;                      // [NV][FN], face fluxes
    R* sQX = sF + NV * FN;                      // [NV][QXN], right states of the last faces
    R* sZ = sQX + NV * QXN;                     // [ZR][NV][NT], this thread's z-window (private)
    constexpr int YHN = G::YHN;
    R* sYH = sZ + G::ZR * NV * NT;              // [NV][YHN], y-halo face states

    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int i0 = NG + blockIdx.x * TX, j0 = NG + blockIdx.y * TY;
    const int i = i0 + tx, j = j0 + ty;
    const int z0 = NG + blockIdx.z * LZ;
    const int zend = min(z0 + LZ, p.n[2] - NG);
    const long long sy = p.sy, sz = p.sz, vs = p.vs;
    const long long col = i + sy * j;
    const R fl = R(p.floor_);
    const R g = R(p.gamma);
    const double cx = p.dtdx[0], cy = p.dtdx[1], cz = p.dtdx[2];

    constexpr int ZR = G::ZR;
    // plane z of this column lives in ring slot z % ZR
    auto zslot = [&](int z, int v) -> R& { return sZ[((z % ZR) * NV + v) * NT + tid]; };
    auto zload = [&](int z) {
#pragma unroll
        for (int v = 0; v < NV; ++v) zslot(z, v) = b.Pin[v * vs + col + sz * z];
    };
    auto zrecon = [&](int zc, R* qr, R* ql) {  // reconstruct cell zc along z, floored
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            recon<REC>(zslot(zc - 2, v), zslot(zc - 1, v), zslot(zc, v), zslot(zc + 1, v), zslot(zc + 2, v), qr[v],
                       ql[v]);
            if (v < 2) {
                qr[v] = jmax(fl, qr[v]);
                ql[v] = jmax(fl, ql[v]);
            }
        }
    };
    R qlz[NV];  // left state of face k+1/2 (ql of cell k)
    R Fzm[NV];  // flux at face k-1/2
    // prologue: ql(z0-1), then qr/ql(z0), the flux at z0-1/2, and the window z0-1 .. z0+3
    for (int z = z0 - 3; z <= z0 + 1; ++z) zload(z);
    {
        R qr[NV], qlm[NV], qr0[NV];
        zrecon(z0 - 1, qr, qlm);
        zload(z0 + 2);
        zrecon(z0, qr0, qlz);
        face_flux<3, RS>(2, g, qlm, qr0, Fzm);
        zload(z0 + 3);
    }

    unsigned long long n_fail = 0, n_fb = 0, n_it = 0, n_cells = 0;
    for (int k = z0; k < zend; ++k) {
        const long long c = col + sz * k;
        DivAcc<R> acc;
        acc.init(b.Us, vs, c);

        // stage plane k: own value, then the x-halo (6 per row) and y-halo (6 per column)
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NV; ++v) sPl[v * PLN + (ty + 3) * EX + tx + 3] = zslot(k, v);
        constexpr int NXH = 6 * TY, NH = NXH + 6 * TX;
        for (int e = tid; e < NH; e += NT) {
            int hx, hy;
            if (e < NXH) {
                int s6 = e % 6;
                hy = e / 6;
                hx = s6 < 3 ? s6 - 3 : TX + s6 - 3;
            } else {
                int e2 = e - NXH, s6 = e2 / TX;
                hx = e2 % TX;
                hy = s6 < 3 ? s6 - 3 : TY + s6 - 3;
            }
            const long long gc = (i0 + hx) + sy * (j0 + hy) + sz * k;
#pragma unroll
            for (int v = 0; v < NV; ++v) sPl[v * PLN + (hy + 3) * EX + hx + 3] = b.Pin[v * vs + gc];
        }
        __syncthreads();

        // x: reconstruct own cell; halo cells -1 and TX of each row
        R qrx[NV];
        {
            const R* q = sPl + (ty + 3) * EX + tx + 3;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                R qr, ql;
                recon_floored<REC>(q + v * PLN, 1, fl, v, qr, ql);
                qrx[v] = qr;
                sQL[v * FN + ty * FXR + tx + 1] = ql;
            }
        }
        // the x halo as (cell, variable) items, on the last threads (the first
        // ones take the y halo): one variable's reconstruction each instead of
        // all five on a few threads while the rest wait at the barrier
        for (int e = NT - 1 - tid; e >= 0 && e < 2 * TY * NV; e += NT) {
            const int v = e / (2 * TY), rs = e - v * 2 * TY, r = rs >> 1, side = rs & 1;
            const R* q = sPl + (r + 3) * EX + (side ? TX : -1) + 3;
            R qr, ql;
            recon_floored<REC>(q + v * PLN, 1, fl, v, qr, ql);
            if (side)
                sQX[v * QXN + r] = qr;
            else
                sQL[v * FN + r * FXR] = ql;
        }
        __syncthreads();
        {
            R PL[NV], F[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) PL[v] = sQL[v * FN + ty * FXR + tx];
            face_flux<3, RS>(0, g, PL, qrx, F);
#pragma unroll
            for (int v = 0; v < NV; ++v) sF[v * FN + ty * FXR + tx] = F[v];
        }
        for (int e = NT - 1 - tid; e >= 0 && e < TY; e += NT) {
            R PL[NV], PR[NV], F[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                PL[v] = sQL[v * FN + e * FXR + TX];
                PR[v] = sQX[v * QXN + e];
            }
            face_flux<3, RS>(0, g, PL, PR, F);
#pragma unroll
            for (int v = 0; v < NV; ++v) sF[v * FN + e * FXR + TX] = F[v];
        }
        // the y halo as (cell, variable) items, in this phase: it needs only the
        // staged plane, and it fills the time the last threads spend on the
        // tile's x-edge faces; its face states go to sYH, since sQL and sQX
        // still hold the x states here
        for (int e = tid; e < 2 * TX * NV; e += NT) {
            const int v = e / (2 * TX), rs = e - v * 2 * TX, cx_ = rs % TX, side = rs / TX;
            const R* q = sPl + ((side ? TY : -1) + 3) * EX + cx_ + 3;
            R qr, ql;
            recon_floored<REC>(q + v * PLN, EX, fl, v, qr, ql);
            sYH[v * YHN + side * TX + cx_] = side ? qr : ql;
        }
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NV; ++v) acc.sub(v, cx, sF[v * FN + ty * FXR + tx + 1], sF[v * FN + ty * FXR + tx]);

        // y: reconstruct own cell; halo cells -1 and TY of each column
        R qry[NV];
        {
            const R* q = sPl + (ty + 3) * EX + tx + 3;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                R qr, ql;
                recon_floored<REC>(q + v * PLN, EX, fl, v, qr, ql);
                qry[v] = qr;
                sQL[v * FN + (ty + 1) * TX + tx] = ql;
            }
        }
        __syncthreads();
        {
            R PL[NV], F[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) PL[v] = ty == 0 ? sYH[v * YHN + tx] : sQL[v * FN + ty * TX + tx];
            face_flux<3, RS>(1, g, PL, qry, F);
#pragma unroll
            for (int v = 0; v < NV; ++v) sF[v * FN + ty * TX + tx] = F[v];
        }
        for (int e = NT - 1 - tid; e >= 0 && e < TX; e += NT) {
            R PL[NV], PR[NV], F[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                PL[v] = sQL[v * FN + TY * TX + e];
                PR[v] = sYH[v * YHN + TX + e];
            }
            face_flux<3, RS>(1, g, PL, PR, F);
#pragma unroll
            for (int v = 0; v < NV; ++v) sF[v * FN + TY * TX + e] = F[v];
        }
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NV; ++v) acc.sub(v, cy, sF[v * FN + (ty + 1) * TX + tx], sF[v * FN + ty * TX + tx]);

        // z: reconstruct cell k+1 from the window; flux at k+1/2
        R Pk[NV];
        {
            R qr1[NV], ql1[NV], Fzp[NV];
            zrecon(k + 1, qr1, ql1);
#pragma unroll
            for (int v = 0; v < NV; ++v) Pk[v] = zslot(k, v);
            face_flux<3, RS>(2, g, qlz, qr1, Fzp);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                acc.sub(v, cz, Fzp[v], Fzm[v]);
                Fzm[v] = Fzp[v];
                qlz[v] = ql1[v];
            }
        }
        // plane k+4 replaces plane k-1 in the ring; its latency overlaps con2prim
        R nxt[NV];
        const bool has_next = k + 4 < p.n[2];
#pragma unroll
        for (int v = 0; v < NV; ++v) nxt[v] = has_next ? b.Pin[v * vs + c + 4 * sz] : R(0);

        // RK combination, con2prim (guess = plane k of this stage's P), Limit;
        // in split mode only U is written here and k_c2p finishes the cell
        if (SPLIT) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                double u = acc.result(v, b.Us, vs, c);
                if (p.rk_a != 0.0) u = p.rk_a * b.U0[v * vs + c] + p.rk_b * u;
                b.Uo[v * vs + c] = u;
            }
        } else {
            double U[NV], P[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                double u = acc.result(v, b.Us, vs, c);
                if (p.rk_a != 0.0) u = p.rk_a * b.U0[v * vs + c] + p.rk_b * u;
                U[v] = u;
                b.Uo[v * vs + c] = u;
                P[v] = (double)Pk[v];
            }
            int fb;
            int r = solve_cell<3>(p, U, P, c, fb);
            n_fail += (r < 0);
            n_fb += fb;
            n_it += (r < 0 ? -r : r);
            n_cells += 1;
            P[0] = jmax(P[0], p.floor_);
            P[1] = jmax(P[1], p.floor_);
#pragma unroll
            for (int v = 0; v < NV; ++v) b.Pout[v * vs + c] = (R)P[v];
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) zslot(k + 4, v) = nxt[v];
    }

    if (n_fail) count_add(p.counters, CNT_C2P_FAIL, n_fail);
    if (p.stats) {
        for (int o = 16; o > 0; o >>= 1) {
            n_fb += __shfl_xor_sync(0xffffffffu, n_fb, o);
            n_it += __shfl_xor_sync(0xffffffffu, n_it, o);
            n_cells += __shfl_xor_sync(0xffffffffu, n_cells, o);
        }
        if ((tid & 31) == 0) {
            count_add(p.counters, CNT_C2P_FALLBACK, n_fb);
            count_add(p.counters, CNT_C2P_ITERS, n_it);
            count_add(p.counters, CNT_C2P_CELLS, n_cells);
        }
    } else if (n_fb) {
        count_add(p.counters, CNT_C2P_FALLBACK, n_fb);
    }
}

// Tile shape of the z-marching kernel per bulk type.
template <typename R> struct ZmCfg;
template <> struct ZmCfg<float> { static constexpr int TX = 32, TY = 8, LZ = 64, MINB = 3, MINB_SPLIT = 4; };
template <> struct ZmCfg<double> { static constexpr int TX = 32, TY = 8, LZ = 64, MINB = 2, MINB_SPLIT = 2; };

template <typename R> inline bool zm_fits(const StageParams& p) {
    using C = ZmCfg<R>;
    return (p.n[0] - 2 * NG) % C::TX == 0 && (p.n[1] - 2 * NG) % C::TY == 0 && p.n[2] - 2 * NG >= 1;
}

// Split-mode con2prim: one thread per interior cell, no barriers, no shared
// memory; reads the stage's U and the guess (the stage's input P, or the
// per-cell W guesses of p.w_guess), writes the floored P.
template <typename R, int MODE>
__global__ void __launch_bounds__(256) k_c2p(StageParams p, StageBufs<R> b) {
    constexpr int NV = 5;
    const int N0 = p.n[0] - 2 * NG, N1 = p.n[1] - 2 * NG, N2 = p.n[2] - 2 * NG;
    const long long tot = (long long)N0 * N1 * N2;  // < 2^32 (launch_c2p)
    CellMap cm;
    cm.init(N0, N1, p.sy, p.sz, NG);
    unsigned long long n_fail = 0, n_fb = 0, n_it = 0, n_cells = 0, n_64 = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const long long c = cm.padded((uint32_t)e);
        double U[NV], P[NV];
        const bool need_p = !(p.c2p_mode == C2P_GUESS_W && p.w_guess);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            U[v] = b.Uo[v * p.vs + c];
            P[v] = need_p ? (double)b.Pin[v * p.vs + c] : 0.0;
        }
        int fb, f64 = 1;
        int r = solve_cell<3, MODE>(p, U, P, c, fb, &f64);
        n_fail += (r < 0);
        n_fb += fb;
        n_it += (r < 0 ? -r : r);
        n_cells += 1;
        n_64 += f64;
        P[0] = jmax(P[0], p.floor_);
        P[1] = jmax(P[1], p.floor_);
#pragma unroll
        for (int v = 0; v < NV; ++v) b.Pout[v * p.vs + c] = (R)P[v];
    }
    if (n_fail) count_add(p.counters, CNT_C2P_FAIL, n_fail);
    if (p.stats) {
        for (int o = 16; o > 0; o >>= 1) {
            n_fb += __shfl_xor_sync(0xffffffffu, n_fb, o);
            n_it += __shfl_xor_sync(0xffffffffu, n_it, o);
            n_cells += __shfl_xor_sync(0xffffffffu, n_cells, o);
            n_64 += __shfl_xor_sync(0xffffffffu, n_64, o);
        }
        if ((threadIdx.x & 31) == 0) {
            count_add(p.counters, CNT_C2P_FALLBACK, n_fb);
            count_add(p.counters, CNT_C2P_ITERS, n_it);
            count_add(p.counters, CNT_C2P_CELLS, n_cells);
            count_add(p.counters, CNT_C2P_FP64, n_64);
        }
    } else if (n_fb) {
        count_add(p.counters, CNT_C2P_FALLBACK, n_fb);
    }
}

// the split con2prim alone (3D interior), e.g. after a kernel that wrote the W guesses
// The same for a 2D grid (padded extents (Nx + 6, Ny + 6, 1)): one thread per
// interior cell, the reference's 2D con2prim (solve_cell<2>) from the stage's
// input P, floors, P out; the statistics as the fused box kernel counts them.
template <typename R>
__global__ void __launch_bounds__(256) k_c2p_2d(StageParams p, StageBufs<R> b) {
    constexpr int NV = 4;
    const int N0 = p.n[0] - 2 * NG, N1 = p.n[1] - 2 * NG;
    const long long tot = (long long)N0 * N1;  // < 2^32 (launch_c2p)
    CellMap cm;
    cm.init(N0, N1, p.sy, p.sz, NG);
    unsigned long long n_fail = 0, n_fb = 0, n_it = 0, n_cells = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        // interior cell (i, j) -> (i + NG) + sy (j + NG); the z index stays 0
        const uint32_t j = cm.dx.div((uint32_t)e), i = (uint32_t)e - j * cm.n0;
        const long long c = (long long)(i + NG) + p.sy * (long long)(j + NG);
        double U[NV], P[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            U[v] = b.Uo[v * p.vs + c];
            P[v] = (double)b.Pin[v * p.vs + c];
        }
        int fb;
        int r;
        if (p.c2p_mode == C2P_GUESS_W) {
            // the previous state's W (VB_GUESS_PREVIOUS_W): the W Newton of the
            // 3D scheme on the state padded to three momenta (u^z = 0), with
            // the precision gate of the FP32-bulk form. It runs only here,
            // where 2D grids with this guess always split their stage, so the
            // fused box kernels keep their own register allocation.
            double U5[5] = {U[0], U[1], U[2], U[3], 0.0}, P5[5] = {P[0], P[1], P[2], P[3], 0.0};
            const double W0 = (P[0] + p.gamma * P[1]) * (sq(P[2]) + sq(P[3]) + 1.0);
            if (p.c2p_fp32) {
                int f64;
                r = c2p_w_gated(p.gamma, U5, (float)W0, p.w_rtol, p.w_max_newton, 4 * p.n_iter, true, P5, &fb, &f64);
            } else {
                r = c2p_w(p.gamma, U5, W0, p.w_rtol, p.w_max_newton, 4 * p.n_iter, P5, &fb);
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) P[v] = P5[v];
        } else {
            r = solve_cell<2>(p, U, P, c, fb);
        }
        n_fail += (r < 0);
        n_fb += fb;
        n_it += (r < 0 ? -r : r);
        n_cells += 1;
        P[0] = jmax(P[0], p.floor_);
        P[1] = jmax(P[1], p.floor_);
#pragma unroll
        for (int v = 0; v < NV; ++v) b.Pout[v * p.vs + c] = (R)P[v];
    }
    if (n_fail) count_add(p.counters, CNT_C2P_FAIL, n_fail);
    if (p.stats) {
        for (int o = 16; o > 0; o >>= 1) {
            n_fb += __shfl_xor_sync(0xffffffffu, n_fb, o);
            n_it += __shfl_xor_sync(0xffffffffu, n_it, o);
            n_cells += __shfl_xor_sync(0xffffffffu, n_cells, o);
        }
        if ((threadIdx.x & 31) == 0) {
            count_add(p.counters, CNT_C2P_FALLBACK, n_fb);
            count_add(p.counters, CNT_C2P_ITERS, n_it);
            count_add(p.counters, CNT_C2P_CELLS, n_cells);
        }
    } else if (n_fb) {
        count_add(p.counters, CNT_C2P_FALLBACK, n_fb);
    }
}

// split-mode con2prim of a 3D (k_c2p) or 2D (k_c2p_2d) grid
template <typename R> cudaError_t launch_c2p(const StageParams& p, const StageBufs<R>& b, cudaStream_t s) {
    if (p.n[2] == 1) {
        const long long cells = (long long)(p.n[0] - 2 * NG) * (p.n[1] - 2 * NG);
        if ((unsigned long long)cells > MAX_CELLS_U32) return cudaErrorInvalidValue;
        k_c2p_2d<R><<<grid_for(cells, 256), 256, 0, s>>>(p, b);
        return cudaGetLastError();
    }
    const long long cells = (long long)(p.n[0] - 2 * NG) * (p.n[1] - 2 * NG) * (p.n[2] - 2 * NG);
    if ((unsigned long long)cells > MAX_CELLS_U32) return cudaErrorInvalidValue;
    if (p.c2p_mode == C2P_GUESS_W)
        k_c2p<R, 2><<<grid_for(cells, 256), 256, 0, s>>>(p, b);
    else
        k_c2p<R, 1><<<grid_for(cells, 256), 256, 0, s>>>(p, b);
    return cudaGetLastError();
}

template <int REC, int RS, typename R, bool SPLIT>
cudaError_t launch_stage_zm_t(const StageParams& p, const StageBufs<R>& b, cudaStream_t s) {
    using C = ZmCfg<R>;
    using G = ZmGeom<C::TX, C::TY>;
    auto kern = k_stage_zm<REC, RS, R, C::TX, C::TY, C::LZ, SPLIT ? C::MINB_SPLIT : C::MINB, SPLIT>;
    const size_t smem = G::template smem_bytes<R>();
    static unsigned long long attr_set = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(attr_set >> (dev & 63) & 1ULL)) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        attr_set |= 1ULL << (dev & 63);
    }
    dim3 grid((p.n[0] - 2 * NG) / C::TX, (p.n[1] - 2 * NG) / C::TY, (p.n[2] - 2 * NG + C::LZ - 1) / C::LZ);
    kern<<<grid, C::TX * C::TY, smem, s>>>(p, b);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !SPLIT || p.skip_c2p) return e;
    const long long cells = (long long)(p.n[0] - 2 * NG) * (p.n[1] - 2 * NG) * (p.n[2] - 2 * NG);
    if ((unsigned long long)cells > MAX_CELLS_U32) return cudaErrorInvalidValue;
    if (p.c2p_mode == C2P_GUESS_W)
        k_c2p<R, 2><<<grid_for(cells, 256), 256, 0, s>>>(p, b);
    else
        k_c2p<R, 1><<<grid_for(cells, 256), 256, 0, s>>>(p, b);
    return cudaGetLastError();
}

template <int REC, int RS, typename R>
cudaError_t launch_stage_zm(const StageParams& p, const StageBufs<R>& b, cudaStream_t s) {
    return (p.split || p.skip_c2p) ? launch_stage_zm_t<REC, RS, R, true>(p, b, s)
                                   : launch_stage_zm_t<REC, RS, R, false>(p, b, s);
}

template <typename R> int stage_div_in_pout(int dims, int rec, int rs, const StageParams& p) {
    if (!std::is_same<R, float>::value || dims != 3 || p.force_box || !zm_fits<R>(p)) return 0;
    return p.pairs && zp_available(rec, rs) && p.skip_c2p && p.want_div ? 1 : 0;
}

// 1 when launch_stage with these arguments runs the stencil kernel and then
// k_c2p as a kernel of its own (a split 3D z-marching stage); the same two
// launches result from launch_stage with skip_c2p = 1, want_div = 0 followed
// by launch_c2p
template <typename R> int stage_split_c2p(int dims, const StageParams& p) {
    if (dims == 2) return p.split && !p.skip_c2p ? 1 : 0;
    return dims == 3 && !p.force_box && zm_fits<R>(p) && p.split && !p.skip_c2p ? 1 : 0;
}

template <typename R>
cudaError_t dispatch_stage_zm(int rec, int rs, const StageParams& p, const StageBufs<R>& b, cudaStream_t s) {
    if constexpr (std::is_same<R, float>::value) {
        if (p.pairs && zp_available(rec, rs)) return launch_stage_zp(rec, rs, p, b, s);
    }
#define VB_CASE(RC, RSC) \
    if (rec == RC && rs == RSC) return launch_stage_zm<RC, RSC, R>(p, b, s);
    VB_CASE(REC_MINMOD, RS_HLL)
    VB_CASE(REC_MINMOD, RS_HLLC)
    VB_CASE(REC_PPM, RS_HLL)
    VB_CASE(REC_PPM, RS_HLLC)
    VB_CASE(REC_WENOZ, RS_HLL)
    VB_CASE(REC_WENOZ, RS_HLLC)
#undef VB_CASE
    return cudaErrorInvalidValue;
}

}  // namespace vb
