// Fused RK-stage kernel and the small per-step kernels, templated on the
// bulk type R of the primitive arrays (double: plain FP64; float: the FP32
// bulk form, where U and con2prim stay FP64).
//
// Stage kernel (one launch per RK stage; replaces the reference's
// Fluxes x/y/z + Update + UtoP + Limit launches, src/3dim/algos.jl:279-293):
// a CTA owns a TX x TY x TZ tile of interior cells. For each axis it stages
// the tile plus a 3-cell halo along that axis in shared memory, reconstructs
// every cell ONCE (the reference evaluates WENOZ twice per face,
// src/3dim/algos.jl:78,105), floors the face states, computes the face
// fluxes in shared memory and accumulates the flux difference into per-cell
// FP64 registers. Face states and fluxes never reach HBM. It then applies the
// RK combination, solves con2prim with the cell's previous primitive state as
// the guess and writes U and the floored P. In 2D the tile with its halo
// along both axes can instead come as one TMA tile (TMA form of k_stage).
#pragma once
#include "vb_ns.h"
#include <cuda.h>  // CUtensorMap

#include "vb_con2prim.cuh"
#include "vb_index.cuh"
#include "vb_internal.h"
#include "vb_tc.cuh"
#include "vb_tmap.h"

namespace VB_NS {

template <int DIM> struct TileCfg;
template <> struct TileCfg<3> { static constexpr int TX = 32, TY = 4, TZ = 4, NT = 256; };
template <> struct TileCfg<2> { static constexpr int TX = 32, TY = 8, TZ = 1, NT = 256; };
template <> struct TileCfg<1> { static constexpr int TX = 256, TY = 1, TZ = 1, NT = 256; };

template <int DIM, int TX, int TY, int TZ> struct TileGeom {
    static constexpr int NV = 2 + DIM;
    static constexpr int TC = TX * TY * TZ;
    static constexpr int ext(int d) {
        return (TX + (d == 0 ? 6 : 0)) * (TY + (d == 1 ? 6 : 0)) * (TZ + (d == 2 ? 6 : 0));
    }
    static constexpr int faces(int d) {
        return (TX + (d == 0 ? 1 : 0)) * (TY + (d == 1 ? 1 : 0)) * (TZ + (d == 2 ? 1 : 0));
    }
    static constexpr int cmax(int a, int b) { return a > b ? a : b; }
    static constexpr int EXTMAX = cmax(ext(0), cmax(DIM > 1 ? ext(1) : 0, DIM > 2 ? ext(2) : 0));
    static constexpr int FACEMAX = cmax(faces(0), cmax(DIM > 1 ? faces(1) : 0, DIM > 2 ? faces(2) : 0));
    template <typename R> static constexpr size_t smem_bytes() {
        return sizeof(R) * NV * (size_t)(EXTMAX + 2 * FACEMAX);
    }
};

// TMA form of the 2D tile: one box of the tile with its 3-cell halo on both
// axes, every variable, [NV][TY + 6][BXW] (x fastest). The box starts at
// x = x0 - 3 = TX * blockIdx.x, 16-byte aligned when TX times the element
// size is a multiple of 16, and is TX + 6 cells rounded up to a 16-byte row
// wide.
template <typename R, int TX, int TY> struct TmaTile2 {
    static constexpr int NV = 4;
    static constexpr int BXW = (TX + 6 + 16 / (int)sizeof(R) - 1) / (16 / (int)sizeof(R)) * (16 / (int)sizeof(R));
    static constexpr int BY = TY + 6;
    static constexpr int BOXE = BXW * BY;  // elements per variable
    static constexpr int BOX_BYTES = (int)sizeof(R) * NV * BOXE;
    static constexpr int FACEMAX = (TX + 1) * TY > TX * (TY + 1) ? (TX + 1) * TY : TX * (TY + 1);
    static constexpr size_t smem_bytes() {
        return 128 + (size_t)(BOX_BYTES + 127) / 128 * 128 + sizeof(R) * NV * (size_t)(2 * FACEMAX) + 16;
    }
};
constexpr uint32_t TILE_MAX_POLLS = 1u << 22;  // bounded wait for the TMA tile
static_assert(TmaTile2<double, 32, 8>::BXW >= 32 + 6 && (TmaTile2<double, 32, 8>::BXW * 8) % 16 == 0, "box row");
static_assert(TmaTile2<float, 32, 8>::BXW >= 32 + 6 && (TmaTile2<float, 32, 8>::BXW * 4) % 16 == 0, "box row");

// tensor map of a 2D state array for the TMA form of k_stage: dims (x, y,
// variable) with byte strides (sy, vs) x element size; the box is TmaTile2's
template <typename R, int TX, int TY> bool encode_tile2_tmap(void* out, const R* P, const Grid& g) {
    using TT = TmaTile2<R, TX, TY>;
    if (g.dims != 2 || g.nv != TT::NV) return false;
    const cuuint64_t dim[3] = {(cuuint64_t)g.n[0], (cuuint64_t)g.n[1], (cuuint64_t)TT::NV};
    const cuuint64_t stride[2] = {(cuuint64_t)g.sy * sizeof(R), (cuuint64_t)g.vs * sizeof(R)};
    const cuuint32_t box[3] = {(cuuint32_t)TT::BXW, (cuuint32_t)TT::BY, (cuuint32_t)TT::NV};
    return encode_tmap(out, P, (int)sizeof(R), 3, dim, stride, box);
}

__device__ __forceinline__ void count_add(unsigned long long* c, int which, unsigned long long v) {
    if (c && v) atomicAdd(c + which, v);
}

// the learned guess's refinement of one cell (two-kernel learned form), out of
// line: kernels that run the reference cascade keep its registers out of theirs
static __device__ __noinline__ int solve_cell_learned(const StageParams& p, const double* U, double* P, float W0,
                                                      int* fallback, int* fp64) {
    return c2p_w_gated(p.gamma, U, W0, p.w_rtol, p.w_max_newton, 4 * p.n_iter, p.c2p_fp32 != 0, P, fallback, fp64);
}

// con2prim of one cell: per-dimension reference algorithm, or the W Newton
// from a supplied guess with the bracketed fallback.
// MODE: 0 reads p.c2p_mode at run time; 1 (reference) and 2 (W Newton) fix
// it at compile time, so a kernel of one mode carries no code of the other.
template <int DIM, int MODE = 0>
__device__ __forceinline__ int solve_cell(const StageParams& p, const double* U, double* P, long long gidx,
                                          int& fallback, int* fp64 = nullptr) {
    fallback = 0;
    if (DIM == 3 && MODE != 1 && (MODE == 2 || p.c2p_mode == C2P_GUESS_W)) {
        double W0;
        if (p.w_guess) {
            // the learned guess, with the precision gate of the FP32-bulk form
            int f64 = 1;
            const int it = solve_cell_learned(p, U, P, p.w_guess[gidx], &fallback, &f64);
            if (fp64) *fp64 = f64;
            return it;
        } else {
            // the previous state's W (VB_GUESS_PREVIOUS_W), with the same gate
            double gm2 = sq(P[2]) + sq(P[3]) + sq(P[4]) + 1.0;
            W0 = (P[0] + p.gamma * P[1]) * gm2;
            if (p.c2p_fp32) {
                int f64 = 1;
                const int it = solve_cell_learned(p, U, P, (float)W0, &fallback, &f64);
                if (fp64) *fp64 = f64;
                return it;
            }
        }
        int fb;
        int it = c2p_w(p.gamma, U, W0, p.w_rtol, p.w_max_newton, 4 * p.n_iter, P, &fb);
        fallback = fb;
        return it;
    }
    if (DIM == 1 || DIM == 2) {
        // The reference's 1D / 2D Newton has no failure signal: a cell that
        // diverges keeps a non-finite state (which then spreads); without
        // c2p_rescue (single grids) the reference's values are kept and the
        // cell is counted as a failure. With c2p_rescue (batched problems) a
        // reference result is accepted only if finite and reproducing U to
        // 1e-8 (its stop rule looks at the step, not the residual), the
        // bracketed W Newton on the conserved state padded to three momenta
        // is the other solver, and a cell neither solves keeps the stage's
        // input state (counted as failed). C2P_GUESS_W (FP32-bulk batches)
        // runs the W Newton first, from the input state's W; the reference
        // Newton, which also accepts negative-pressure roots that the floors
        // then lift, is its fallback.
        double Pin[2 + DIM];
#pragma unroll
        for (int v = 0; v < 2 + DIM; ++v) Pin[v] = P[v];
        auto ref_try = [&](int& r) -> bool {
#pragma unroll
            for (int v = 0; v < 2 + DIM; ++v) P[v] = Pin[v];
            r = DIM == 1 ? c2p_1d(p.gamma, p.n_iter, p.tol, U, P) : c2p_2d(p.gamma, p.n_iter, p.tol, U, P);
            bool finite = true;
#pragma unroll
            for (int v = 0; v < 2 + DIM; ++v) finite = finite && isfinite(P[v]);
            if (!(r >= 0 && finite)) return false;
            if (!p.c2p_rescue) return true;
            double Ur[2 + DIM];
            prim2con<DIM>(p.gamma, P, Ur);
            const double scale = fabs(U[0]) + fabs(U[1]);
            double res = 0.0;
#pragma unroll
            for (int v = 0; v < 2 + DIM; ++v) res = fmax(res, fabs(Ur[v] - U[v]));
            return res <= 1e-8 * scale;
        };
        auto w_try = [&](double W0, int& r) -> bool {
            double U5[5] = {U[0], U[1], U[2], DIM > 1 ? U[3] : 0.0, 0.0}, P5[5];
            int fb;
            r = c2p_w(p.gamma, U5, W0, p.w_rtol, p.w_max_newton, 4 * p.n_iter, P5, &fb);
            if (r < 0) return false;
#pragma unroll
            for (int v = 0; v < 2 + DIM; ++v) P[v] = P5[v];
            return true;
        };
        int r = 0;
        if (!p.c2p_rescue) {
            const bool ok = ref_try(r);
            return ok ? r : (r < 0 ? r : -(r + 1));
        }
        if (p.c2p_mode == C2P_GUESS_W) {
            const double gm2 = sq(Pin[2]) + (DIM > 1 ? sq(Pin[3]) : 0.0) + 1.0;
            if (w_try((Pin[0] + p.gamma * Pin[1]) * gm2, r)) return r;
            fallback = 1;
            if (ref_try(r)) return r;
        } else {
            if (ref_try(r)) return r;
            fallback = 1;
            if (w_try(U[0] - U[1], r)) return r;
        }
#pragma unroll
        for (int v = 0; v < 2 + DIM; ++v) P[v] = Pin[v];
        return r < 0 ? r : -(r + 1);
    }
    int r = c2p_3d(p.gamma, p.n_iter, p.tol, U, P);
    fallback = r > 1;
    return r;
}

// Loads of the stage inputs. CG: through L2 only (ld.global.cg), for a kernel
// that reads arrays written earlier in the same launch by other CTAs.
template <bool CG, typename T> __device__ __forceinline__ T ld_in(const T* p) {
    if (CG) return __ldcg(p);
    return *p;
}

// One TX x TY x TZ tile of a stage (tile coordinates bx, by, bz); the body of
// k_stage, shared with the batched kernel. smem_raw: TileGeom::smem_bytes<R>(),
// or TmaTile2::smem_bytes() for the TMA form (2D; tm: the tensor map of Pin,
// dims (x, y, variable)), which loads the tile once for both axes.
template <int DIM, int REC, int RS, typename R, int TX, int TY, int TZ, int NT, bool CG, bool TMA = false>
__device__ __forceinline__ void stage_tile(const StageParams& p, const StageBufs<R>& b, int bx, int by, int bz,
                                           unsigned char* smem_raw, const CUtensorMap* tm = nullptr) {
    using G = TileGeom<DIM, TX, TY, TZ>;
    using TT = TmaTile2<R, TX, TY>;
    static_assert(!TMA || (DIM == 2 && TZ == 1 && (TX * (int)sizeof(R)) % 16 == 0), "TMA tiles: 2D");
    constexpr int NV = G::NV;
    constexpr int TC = G::TC;
    constexpr int CPT = (TC + NT - 1) / NT;
    R* sP;
    uint64_t* sBar = nullptr;
    if constexpr (TMA)
        sP = reinterpret_cast<R*>(smem_raw + ((128u - (tc::smem_u32(smem_raw) & 127u)) & 127u));
    else
        sP = reinterpret_cast<R*>(smem_raw);
    R* sL = TMA ? sP + (TT::BOX_BYTES + 127) / 128 * 128 / (int)sizeof(R) : sP + NV * G::EXTMAX;
    R* sR = sL + NV * (TMA ? TT::FACEMAX : G::FACEMAX);
    if constexpr (TMA) sBar = reinterpret_cast<uint64_t*>(((uintptr_t)(sR + NV * TT::FACEMAX) + 7) & ~(uintptr_t)7);

    const int tid = threadIdx.x;
    const int T[3] = {TX, TY, TZ};
    const int org[3] = {NG + bx * TX, DIM > 1 ? NG + by * TY : 0, DIM > 2 ? NG + bz * TZ : 0};
    // valid cells of this (possibly partial) tile along each axis
    int vt[3];
    #pragma unroll
    for (int a = 0; a < 3; ++a) vt[a] = a < DIM ? min(T[a], p.n[a] - NG - org[a]) : 1;
    const long long vs = p.vs;
    const R fl = R(p.floor_);
    const R g = R(p.gamma);

    double acc[CPT][NV];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        int cell = tid + c * NT;
        int lx = cell % TX, ly = (cell / TX) % TY, lz = cell / (TX * TY);
        bool ok = cell < TC && lx < vt[0] && ly < vt[1] && lz < vt[2];
        long long gidx = (org[0] + lx) + p.sy * (org[1] + ly) + p.sz * (org[2] + lz);
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[c][v] = ok ? ld_in<CG>(b.Us + v * vs + gidx) : 0.0;
    }

    if constexpr (TMA) {
        // the tile with its halo on both axes, every variable, as one TMA box
        if (tid == 0) {
            tc::mbar_init(sBar, 1);
            tc::fence_mbar_init();
        }
        __syncthreads();
        if (tid == 0) {
            tc::mbar_arrive_expect_tx(sBar, TT::BOX_BYTES);
            tc::tma_load_3d(sP, tm, org[0] - NG, org[1] - NG, 0, sBar);
        }
        const bool ok = tc::mbar_wait(sBar, 0, nullptr, TILE_MAX_POLLS);
        if (__syncthreads_or(!ok)) {
            // the box may still be landing in this CTA's shared memory: thread 0
            // waits once more (bounded) before the CTA ends, so that the CTA
            // stays resident while the copy completes; if that wait runs out
            // too, the copy is still outstanding when the CTA exits
            if (tid == 0) {
                count_add(p.counters, CNT_TIMEOUT, 1);
                tc::mbar_wait(sBar, 0, nullptr, TILE_MAX_POLLS);
            }
            return;
        }
    }

#pragma unroll 1
    for (int d = 0; d < DIM; ++d) {
        // staged tile: EX x EY x EZ elements per variable; the TMA tile is the
        // same BXW x (TY + 6) box for both axes, the cell (0, 0) at (3, 3)
        const int EX = TMA ? TT::BXW : TX + (d == 0 ? 6 : 0), EY = TMA ? TT::BY : TY + (d == 1 ? 6 : 0),
                  EZ = TMA ? 1 : TZ + (d == 2 ? 6 : 0);
        const int EXT = EX * EY * EZ;
        const int ox = org[0] - (d == 0 ? NG : 0), oy = org[1] - (d == 1 ? NG : 0),
                  oz = org[2] - (d == 2 ? NG : 0);
        __syncthreads();
        // 1. stage the axis-extended tile of P
        if constexpr (!TMA) {
            for (int e = tid; e < NV * EXT; e += NT) {
                int v = e / EXT, r = e - v * EXT;
                int ex = r % EX, ey = (r / EX) % EY, ez = r / (EX * EY);
                int gi = ox + ex, gj = oy + ey, gk = oz + ez;
                R val = R(0);
                if (gi < p.n[0] && gj < p.n[1] && gk < p.n[2])
                    val = ld_in<CG>(b.Pin + v * vs + gi + p.sy * gj + p.sz * gk);
                sP[v * EXT + r] = val;
            }
            __syncthreads();
        }
        // 2. reconstruct each cell of the tile (plus one halo cell on each side
        //    along d) once; store its two face values, floored. The tile's own
        //    cells go one per thread with every variable; the two halo layers
        //    then go one (cell, variable) per thread, so that the phase takes
        //    1 + NV * halo / NT cell reconstructions per thread instead of two
        //    (with one cell per thread, the halo alone made a second round).
        const int FX = TX + (d == 0), FY = TY + (d == 1), FZ = TZ + (d == 2);
        const int NF = FX * FY * FZ;
        const int sd = d == 0 ? 1 : (d == 1 ? EX : EX * EY);
        const int vtd = d == 0 ? vt[0] : (d == 1 ? vt[1] : vt[2]);
        // cell c (tile coordinates, c_d in [-1, T_d]): staged base index, its
        // two faces and whether each is written; false if the cell is unused
        auto cell_at = [&](int c0, int c1, int c2, int& base, int& fR, int& fL, bool& wR, bool& wL) -> bool {
            const int c[3] = {c0, c1, c2};
            bool ok = true;
#pragma unroll
            for (int a = 0; a < 3; ++a)
                ok = ok && (a == d ? (c[a] >= -1 && c[a] <= vt[a]) : c[a] < vt[a]);
            if (!ok) return false;
            const int ex = c[0] + (d == 0 || TMA ? NG : 0), ey = c[1] + (d == 1 || TMA ? NG : 0),
                      ez = c[2] + (d == 2 ? NG : 0);
            base = ex + EX * (ey + EY * ez);
            fR = c[0] + FX * (c[1] + FY * c[2]);              // face c_d
            fL = fR + (d == 0 ? 1 : (d == 1 ? FX : FX * FY));  // face c_d + 1
            const int cd = d == 0 ? c[0] : (d == 1 ? c[1] : c[2]);
            wR = cd >= 0;
            wL = cd + 1 <= vtd;
            return true;
        };
        auto recon_var = [&](int v, int base, int fR, int fL, bool wR, bool wL) {
            const R* q = sP + v * EXT + base;
            R qr, ql;
            recon<REC>(q[-2 * sd], q[-sd], q[0], q[sd], q[2 * sd], qr, ql);
            if (v < 2) {
                qr = jmax(fl, qr);
                ql = jmax(fl, ql);
            }
            if (wR) sR[v * NF + fR] = qr;
            if (wL) sL[v * NF + fL] = ql;
        };
        for (int e = tid; e < TC; e += NT) {
            int base, fR, fL;
            bool wR, wL;
            if (!cell_at(e % TX, (e / TX) % TY, e / (TX * TY), base, fR, fL, wR, wL)) continue;
#pragma unroll
            for (int v = 0; v < NV; ++v) recon_var(v, base, fR, fL, wR, wL);
        }
        {
            // halo layers c_d = -1 and c_d = T_d: (cell, variable) items, variable-major
            const int td = d == 0 ? TX : (d == 1 ? TY : TZ);
            const int HL = TC / td;  // cells per layer
            for (int e = tid; e < 2 * HL * NV; e += NT) {
                const int v = e / (2 * HL), h = e - v * 2 * HL, side = h / HL, k = h - side * HL;
                // k enumerates the layer's cells over the two other axes, x fastest
                int c[3];
                const int o0 = d == 0 ? 1 : 0, o1 = d == 2 ? 1 : 2;  // the other axes, in order
                const int n0 = o0 == 0 ? TX : TY;
                c[d] = side ? td : -1;
                c[o0] = k % n0;
                c[o1] = k / n0;
                int base, fR, fL;
                bool wR, wL;
                if (cell_at(c[0], c[1], c[2], base, fR, fL, wR, wL)) recon_var(v, base, fR, fL, wR, wL);
            }
        }
        __syncthreads();
        // 3. face fluxes (overwrite the left states)
        for (int e = tid; e < NF; e += NT) {
            int f[3] = {e % FX, (e / FX) % FY, e / (FX * FY)};
            bool ok = true;
            #pragma unroll
            for (int a = 0; a < 3; ++a) ok = ok && (a == d ? f[a] <= vt[a] : f[a] < vt[a]);
            if (!ok) continue;
            R PL[NV], PR[NV], F[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                PL[v] = sL[v * NF + e];
                PR[v] = sR[v * NF + e];
            }
            face_flux<DIM, RS>(d, g, PL, PR, F);
#pragma unroll
            for (int v = 0; v < NV; ++v) sL[v * NF + e] = F[v];
        }
        __syncthreads();
        // 4. flux difference, in the reference's order x, y, z
        const double cdt = d == 0 ? p.dtdx[0] : (d == 1 ? p.dtdx[1] : p.dtdx[2]);
        const int fstep = d == 0 ? 1 : (d == 1 ? FX : FX * FY);
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            int cell = tid + c * NT;
            int lx = cell % TX, ly = (cell / TX) % TY, lz = cell / (TX * TY);
            if (!(cell < TC && lx < vt[0] && ly < vt[1] && lz < vt[2])) continue;
            int flo = lx + FX * (ly + FY * lz);
#pragma unroll
            for (int v = 0; v < NV; ++v)
                acc[c][v] = acc[c][v] - cdt * ((double)sL[v * NF + flo + fstep] - (double)sL[v * NF + flo]);
        }
    }

    // 5. RK combination, con2prim (guess = this stage's input P), Limit
    unsigned long long n_fail = 0, n_fb = 0, n_it = 0, n_cells = 0;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        int cell = tid + c * NT;
        int lx = cell % TX, ly = (cell / TX) % TY, lz = cell / (TX * TY);
        if (!(cell < TC && lx < vt[0] && ly < vt[1] && lz < vt[2])) continue;
        long long gidx = (org[0] + lx) + p.sy * (org[1] + ly) + p.sz * (org[2] + lz);
        double U[NV], P[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double u = acc[c][v];
            if (p.rk_a != 0.0) u = p.rk_a * ld_in<CG>(b.U0 + v * vs + gidx) + p.rk_b * u;
            U[v] = u;
            b.Uo[v * vs + gidx] = u;
            P[v] = (double)ld_in<CG>(b.Pin + v * vs + gidx);
        }
        if (p.skip_c2p) continue;  // con2prim runs in a separate kernel
        int fb;
        int r = solve_cell<DIM>(p, U, P, gidx, fb);
        n_fail += (r < 0);
        n_fb += fb;
        n_it += (r < 0 ? -r : r);
        n_cells += 1;
        P[0] = jmax(P[0], p.floor_);
        P[1] = jmax(P[1], p.floor_);
#pragma unroll
        for (int v = 0; v < NV; ++v) b.Pout[v * vs + gidx] = (R)P[v];
    }
    if (n_fail) count_add(p.counters, CNT_C2P_FAIL, n_fail);
    if (p.stats) {
        // warp-aggregate the statistics; every thread of the CTA reaches here
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

template <int DIM, int REC, int RS, typename R, int TX, int TY, int TZ, int NT, bool TMA>
__global__ void __launch_bounds__(NT) k_stage(StageParams p, StageBufs<R> b, const __grid_constant__ CUtensorMap tm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    stage_tile<DIM, REC, RS, R, TX, TY, TZ, NT, false, TMA>(p, b, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z,
                                                            smem_raw, &tm);
}

// TMA form where the caller encoded a tensor map of Pin (p.tmap_in; 2D)
template <int DIM, int REC, int RS, typename R, bool TMA>
cudaError_t launch_stage_tt(const StageParams& p, const StageBufs<R>& b, cudaStream_t s) {
    using C = TileCfg<DIM>;
    using G = TileGeom<DIM, C::TX, C::TY, C::TZ>;
    auto kern = k_stage<DIM, REC, RS, R, C::TX, C::TY, C::TZ, C::NT, TMA>;
    size_t smem;
    if constexpr (TMA)
        smem = TmaTile2<R, C::TX, C::TY>::smem_bytes();
    else
        smem = G::template smem_bytes<R>();
    static unsigned long long attr_set = 0;  // one bit per device, per instantiation
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(attr_set >> (dev & 63) & 1ULL)) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        attr_set |= 1ULL << (dev & 63);
    }
    dim3 grid((p.n[0] - 2 * NG + C::TX - 1) / C::TX, DIM > 1 ? (p.n[1] - 2 * NG + C::TY - 1) / C::TY : 1,
              DIM > 2 ? (p.n[2] - 2 * NG + C::TZ - 1) / C::TZ : 1);
    CUtensorMap tm;
    if (TMA)
        tm = *static_cast<const CUtensorMap*>(p.tmap_in);
    else
        memset(&tm, 0, sizeof tm);
    kern<<<grid, C::NT, smem, s>>>(p, b, tm);
    return cudaGetLastError();
}
template <int DIM, int REC, int RS, typename R>
cudaError_t launch_stage_t(const StageParams& p, const StageBufs<R>& b, cudaStream_t s) {
    if constexpr (DIM == 2) {
        if (p.tmap_in) return launch_stage_tt<DIM, REC, RS, R, true>(p, b, s);
    }
    return launch_stage_tt<DIM, REC, RS, R, false>(p, b, s);
}

template <int DIM, typename R>
cudaError_t dispatch_stage_dim(int rec, int rs, const StageParams& p, const StageBufs<R>& b, cudaStream_t s) {
#define VB_CASE(RC, RSC)                                                                      \
    if (rec == RC && rs == RSC) return launch_stage_t<DIM, RC, RSC, R>(p, b, s);
    VB_CASE(REC_MINMOD, RS_HLL)
    VB_CASE(REC_MINMOD, RS_HLLC)
    VB_CASE(REC_PPM, RS_HLL)
    VB_CASE(REC_PPM, RS_HLLC)
    VB_CASE(REC_WENOZ, RS_HLL)
    VB_CASE(REC_WENOZ, RS_HLLC)
#undef VB_CASE
    return cudaErrorInvalidValue;
}

template <typename R> inline bool zm_fits(const StageParams& p);
template <typename R>
cudaError_t dispatch_stage_zm(int rec, int rs, const StageParams& p, const StageBufs<R>& b, cudaStream_t s);

// 3D grids whose x/y interior extents are multiples of the z-marching tile
// use k_stage_zm; everything else (1D, 2D, ragged 3D) the box-tile k_stage.
// *kernels receives the number of kernels launched (2 for a split z-march
// stage, whose con2prim runs in k_c2p; else 1).
template <typename R>
cudaError_t launch_stage(int dims, int rec, int rs, const StageParams& p, const StageBufs<R>& b,
                         cudaStream_t s, int* kernels) {
    *kernels = 1;
    if (dims == 1) return dispatch_stage_dim<1, R>(rec, rs, p, b, s);
    if (dims == 2) {
        if (!p.split || p.skip_c2p) return dispatch_stage_dim<2, R>(rec, rs, p, b, s);
        // split: the box kernel writes U only, then k_c2p_2d
        StageParams q = p;
        q.skip_c2p = 1;
        const cudaError_t e = dispatch_stage_dim<2, R>(rec, rs, q, b, s);
        if (e != cudaSuccess) return e;
        *kernels = 2;
        return launch_c2p<R>(p, b, s);
    }
    if (dims == 3) {
        if (zm_fits<R>(p) && !p.force_box) {
            *kernels = p.split && !p.skip_c2p ? 2 : 1;
            return dispatch_stage_zm<R>(rec, rs, p, b, s);
        }
        return dispatch_stage_dim<3, R>(rec, rs, p, b, s);
    }
    return cudaErrorInvalidValue;
}

// ---- layout conversion -----------------------------------------------------
// One thread per cell; AoS reads of nv consecutive doubles, SoA writes are
// coalesced per variable.

// dense padded cell c (x fastest, rows of n[0] cells) -> index in the pitched SoA arrays
__host__ __device__ __forceinline__ long long soa_index(const Grid& g, long long c) {
    if (g.sy == g.n[0]) return c;
    const long long row = c / g.n[0];
    return (c - row * g.n[0]) + g.sy * row;  // sz == sy * n[1]: rows of every plane are consecutive
}

template <int DIM, typename R>
__global__ void k_load_prims(Grid g, const double* __restrict__ Pa, R* __restrict__ P, double* __restrict__ U0,
                             double gamma) {
    constexpr int NV = 2 + DIM;
    long long ncell = (long long)g.n[0] * g.n[1] * g.n[2];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x) {
        double q[NV], u[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) q[v] = Pa[c * NV + v];
        prim2con<DIM>(gamma, q, u);  // kernel_PtoU, src/3dim/structs.jl:66-81
        const long long s = soa_index(g, c);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            P[v * g.vs + s] = (R)q[v];
            U0[v * g.vs + s] = u[v];
        }
    }
}

template <int DIM, typename R>
__global__ void k_store_prims(Grid g, const R* __restrict__ P, double* __restrict__ Pa) {
    constexpr int NV = 2 + DIM;
    long long ncell = (long long)g.n[0] * g.n[1] * g.n[2];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const long long s = soa_index(g, c);
#pragma unroll
        for (int v = 0; v < NV; ++v) Pa[c * NV + v] = (double)P[v * g.vs + s];
    }
}

// ---- device initial conditions ----------------------------------------------
// splitmix64 (Steele, Lea, Flood 2014; constants of Vigna's reference
// implementation): a bijective 64-bit mixer, used as a counter-based stream.
__host__ __device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
// standard normal deviate of cell c in stream `seed` (Box-Muller on two words)
__device__ __forceinline__ double cell_normal(unsigned long long seed, unsigned long long c) {
    const unsigned long long h1 = splitmix64(seed ^ splitmix64(2 * c));
    const unsigned long long h2 = splitmix64(seed ^ splitmix64(2 * c + 1));
    const double u1 = (double)((h1 >> 11) + 1) * 0x1.0p-53;  // (0, 1]
    const double u2 = (double)(h2 >> 11) * 0x1.0p-53;        // [0, 1)
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

// The examples' initial conditions (examples/Jet3D/HARM_jet_breakout.jl:72-118,
// examples/Jet2D/HARM_jet_breakout.jl:37-72) or an ambient medium, on every
// padded cell; then the tail of k_load_prims.
template <int DIM, typename R>
__global__ void k_init_prims(Grid g, InitIC ic, R* __restrict__ P, double* __restrict__ U0, double gamma) {
    constexpr int NV = 2 + DIM;
    const long long ncell = (long long)g.n[0] * g.n[1] * g.n[2];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x) {
        double q[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) q[v] = 0.0;
        const double nz = ic.noise * cell_normal(ic.seed, (unsigned long long)c);
        if (ic.kind == 0) {
            q[0] = ic.rho * (1.0 + nz);
            q[1] = ic.u;
        } else {
            const int i = (int)(c % g.n[0]);
            const int j = (int)((c / g.n[0]) % g.n[1]);
            const int k = (int)(c / ((long long)g.n[0] * g.n[1]));
            const double X = (i + 1) * ic.dx[0];
            const double Y = (j + 1) * ic.dx[1] - ic.box[1];
            const double Z = DIM > 2 ? (k + 1) * ic.dx[2] - ic.box[2] : 0.0;
            const double R2 = DIM > 2 ? X * X + Y * Y + Z * Z : X * X + Y * Y;
            const double Rr = sqrt(R2);
            double rho;
            if (Rr < ic.r_max) {
                const double f = ic.r_max / (Rr < ic.r_eng ? ic.r_eng : Rr);
                rho = ic.rho0 * (f * f) * (1.0 + nz);
            } else {
                rho = ic.outer;
            }
            double u = rho * ic.temp;
            if (Rr < ic.r_eng) {
                const double s = DIM > 2 ? sqrt(X * X + Y * Y) : Y;
                const double ch = cosh(s / ic.r_eng);
                const double ch2 = ch * ch, ch4 = ch2 * ch2;
                const double v = 1.0 / (1.0 - 1.0 / (ic.gamma0 * ic.gamma0)) * (1.0 / (ch4 * ch4));
                q[2] = ic.gamma0 * v;
                rho = rho * ic.engine_rho;
                u = rho * ic.engine_temp;
            }
            q[0] = rho;
            q[1] = u;
        }
        double uc[NV];
        prim2con<DIM>(gamma, q, uc);
        const long long s = soa_index(g, c);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            P[v * g.vs + s] = (R)q[v];
            U0[v * g.vs + s] = uc[v];
        }
    }
}

inline int grid_for(long long n, int nt) {
    long long b = (n + nt - 1) / nt;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)(b < 1 ? 1 : b);
}

template <typename R>
cudaError_t launch_load_prims(const Grid& g, const double* Pa, R* P, double* U0, double gamma, cudaStream_t s) {
    long long ncell = (long long)g.n[0] * g.n[1] * g.n[2];
    int nb = grid_for(ncell, 256);
    if (g.dims == 1) k_load_prims<1, R><<<nb, 256, 0, s>>>(g, Pa, P, U0, gamma);
    else if (g.dims == 2) k_load_prims<2, R><<<nb, 256, 0, s>>>(g, Pa, P, U0, gamma);
    else k_load_prims<3, R><<<nb, 256, 0, s>>>(g, Pa, P, U0, gamma);
    return cudaGetLastError();
}

// Interior snapshot of a dump (src/3dim/saving.jl:57-146 copies
// P.arr[:, 4:end-3, 4:end-3, 4:end-3] to the host and rejects NaN): one
// thread per interior cell, x fastest; reads each variable array coalesced,
// writes the cell's nv consecutive doubles; NaN values counted per warp.
template <int DIM, typename R>
__global__ void k_pack_interior(Grid g, const R* __restrict__ P, double* __restrict__ out,
                                unsigned long long* __restrict__ nan_count) {
    constexpr int NV = 2 + DIM;
    const int N0 = g.n[0] - 2 * NG, N1 = DIM > 1 ? g.n[1] - 2 * NG : 1, N2 = DIM > 2 ? g.n[2] - 2 * NG : 1;
    const long long tot = (long long)N0 * N1 * N2;
    CellMap cm;
    cm.init(N0, N1, g.sy, g.sz, NG);
    const long long off = DIM == 1 ? 0 : (DIM == 2 ? -NG * g.sz : 0);  // 2D: no z ghosts
    unsigned int nans = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        long long c = cm.padded((uint32_t)e) + off;
        if (DIM == 1) c -= NG * (g.sy + g.sz);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double x = (double)P[v * g.vs + c];
            nans += isnan(x) ? 1u : 0u;
            out[e * NV + v] = x;
        }
    }
    nans = __reduce_add_sync(0xffffffffu, nans);
    if ((threadIdx.x & 31) == 0 && nans) atomicAdd(nan_count, (unsigned long long)nans);
}

template <typename R>
cudaError_t launch_pack_interior(const Grid& g, const R* P, double* out, unsigned long long* nan_count,
                                 cudaStream_t s) {
    const long long tot = (long long)(g.n[0] - 2 * NG) * (g.dims > 1 ? g.n[1] - 2 * NG : 1) *
                          (g.dims > 2 ? g.n[2] - 2 * NG : 1);
    if ((unsigned long long)tot > MAX_CELLS_U32) return cudaErrorInvalidValue;
    const int nb = grid_for(tot, 256);
    if (g.dims == 1) k_pack_interior<1, R><<<nb, 256, 0, s>>>(g, P, out, nan_count);
    else if (g.dims == 2) k_pack_interior<2, R><<<nb, 256, 0, s>>>(g, P, out, nan_count);
    else k_pack_interior<3, R><<<nb, 256, 0, s>>>(g, P, out, nan_count);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_init_prims(const Grid& g, const InitIC& ic, R* P, double* U0, double gamma, cudaStream_t s) {
    long long ncell = (long long)g.n[0] * g.n[1] * g.n[2];
    int nb = grid_for(ncell, 256);
    if (g.dims == 1) k_init_prims<1, R><<<nb, 256, 0, s>>>(g, ic, P, U0, gamma);
    else if (g.dims == 2) k_init_prims<2, R><<<nb, 256, 0, s>>>(g, ic, P, U0, gamma);
    else k_init_prims<3, R><<<nb, 256, 0, s>>>(g, ic, P, U0, gamma);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_store_prims(const Grid& g, const R* P, double* Pa, cudaStream_t s) {
    long long ncell = (long long)g.n[0] * g.n[1] * g.n[2];
    int nb = grid_for(ncell, 256);
    if (g.dims == 1) k_store_prims<1, R><<<nb, 256, 0, s>>>(g, P, Pa);
    else if (g.dims == 2) k_store_prims<2, R><<<nb, 256, 0, s>>>(g, P, Pa);
    else k_store_prims<3, R><<<nb, 256, 0, s>>>(g, P, Pa);
    return cudaGetLastError();
}

// ---- ghost cells -------------------------------------------------------------
// The ghost region is covered by disjoint slabs: x-lo/x-hi over all (j,k);
// y-lo/y-hi over interior i and all k; z-lo/z-hi over interior (i,j).
__device__ __forceinline__ bool ghost_slab_cell(const Grid& g, int slab, long long e, int& i, int& j, int& k) {
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int a = slab / 2, side = slab % 2;
    int ext[3];
    int lo[3];
    if (a == 0) {
        ext[0] = NG; ext[1] = n1; ext[2] = n2;
        lo[0] = side ? n0 - NG : 0; lo[1] = 0; lo[2] = 0;
    } else if (a == 1) {
        ext[0] = n0 - 2 * NG; ext[1] = NG; ext[2] = n2;
        lo[0] = NG; lo[1] = side ? n1 - NG : 0; lo[2] = 0;
    } else {
        ext[0] = n0 - 2 * NG; ext[1] = n1 - 2 * NG; ext[2] = NG;
        lo[0] = NG; lo[1] = NG; lo[2] = side ? n2 - NG : 0;
    }
    long long tot = (long long)ext[0] * ext[1] * ext[2];
    if (e >= tot) return false;
    i = lo[0] + (int)(e % ext[0]);
    j = lo[1] + (int)((e / ext[0]) % ext[1]);
    k = lo[2] + (int)(e / ((long long)ext[0] * ext[1]));
    return true;
}

template <typename R>
__global__ void k_ghost_limit(Grid g, const R* __restrict__ Pin, R* __restrict__ Pout, double floor_) {
    const int slab = blockIdx.y;
    const R fl = R(floor_);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;; e += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (!ghost_slab_cell(g, slab, e, i, j, k)) break;
        long long c = i + g.sy * j + g.sz * k;
        for (int v = 0; v < g.nv; ++v) {
            R x = Pin[v * g.vs + c];
            if (v < 2) x = jmax(x, fl);  // function_Limit, src/3dim/algos.jl:5-12
            Pout[v * g.vs + c] = x;
        }
    }
}

template <typename R>
cudaError_t launch_ghost_limit(const Grid& g, const R* Pin, R* Pout, double floor_, cudaStream_t s) {
    long long maxslab = (long long)NG * g.n[1] * g.n[2];
    if (g.dims > 1) maxslab = max(maxslab, (long long)NG * g.n[0] * g.n[2]);
    if (g.dims > 2) maxslab = max(maxslab, (long long)NG * g.n[0] * g.n[1]);
    dim3 grid(grid_for(maxslab, 256), 2 * g.dims);
    k_ghost_limit<R><<<grid, 256, 0, s>>>(g, Pin, Pout, floor_);
    return cudaGetLastError();
}

// Boundary fill of one face, the on-device replacement of the reference's
// host-side `fun_bound` broadcasts (examples/Jet3D/HARM_jet_breakout.jl:131-158):
// OUTFLOW copies the first interior cell into the 3 ghost layers over the
// full padded extent of the other axes; NOZZLE holds a fixed state inside a
// radius (cells, from a centre in the face plane) and is OUTFLOW outside.
// par: NOZZLE {radius, c1, c2, rho, u, u1, u2, u3}.
struct BCPar {
    double v[8];
};

template <typename R>
__global__ void k_bc_face(Grid g, R* __restrict__ P, int face, int kind, BCPar par) {
    const int a = face / 2, side = face % 2;
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    int ext[3] = {n0, n1, n2};
    ext[a] = NG;
    long long tot = (long long)ext[0] * ext[1] * ext[2];
    int b1 = (a + 1) % 3, b2 = (a + 2) % 3;
    if (b1 > b2) {
        int t = b1;
        b1 = b2;
        b2 = t;
    }
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        int idx[3] = {(int)(e % ext[0]), (int)((e / ext[0]) % ext[1]), (int)(e / ((long long)ext[0] * ext[1]))};
        if (side) idx[a] += g.n[a] - NG;
        long long c = idx[0] + g.sy * idx[1] + g.sz * idx[2];
        bool inside = false;
        if (kind == 2) {
            double y1 = (b1 < g.dims) ? (idx[b1] - NG + 0.5) - par.v[1] : 0.0;
            double y2 = (b2 < g.dims) ? (idx[b2] - NG + 0.5) - par.v[2] : 0.0;
            inside = y1 * y1 + y2 * y2 < par.v[0] * par.v[0];
        }
        if (inside) {
            P[c] = (R)par.v[3];
            P[g.vs + c] = (R)par.v[4];
            for (int m = 0; m < g.dims; ++m) P[(2 + m) * g.vs + c] = (R)par.v[5 + m];
        } else {
            int s[3] = {idx[0], idx[1], idx[2]};
            s[a] = side ? g.n[a] - NG - 1 : NG;
            long long cs = s[0] + g.sy * s[1] + g.sz * s[2];
            for (int v = 0; v < g.nv; ++v) P[v * g.vs + c] = P[v * g.vs + cs];
        }
    }
}

template <typename R>
cudaError_t launch_bc_face(const Grid& g, R* P, int face, int kind, const double* par, cudaStream_t s) {
    BCPar bp;
    for (int i = 0; i < 8; ++i) bp.v[i] = par ? par[i] : 0.0;
    int a = face / 2;
    long long tot = (long long)g.n[0] * g.n[1] * g.n[2] / g.n[a] * NG;
    k_bc_face<R><<<grid_for(tot, 256), 256, 0, s>>>(g, P, face, kind, bp);
    return cudaGetLastError();
}

// P[var, ghosts of face] *= factor (the engine decay of TurnOff,
// examples/Jet3D/HARM_jet_breakout.jl:132-135)
template <typename R>
__global__ void k_bc_decay(Grid g, R* __restrict__ P, int face, int var, double factor) {
    const int a = face / 2, side = face % 2;
    int ext[3] = {g.n[0], g.n[1], g.n[2]};
    ext[a] = NG;
    long long tot = (long long)ext[0] * ext[1] * ext[2];
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        int idx[3] = {(int)(e % ext[0]), (int)((e / ext[0]) % ext[1]), (int)(e / ((long long)ext[0] * ext[1]))};
        if (side) idx[a] += g.n[a] - NG;
        long long c = idx[0] + g.sy * idx[1] + g.sz * idx[2];
        P[var * g.vs + c] = (R)((double)P[var * g.vs + c] * factor);
    }
}

template <typename R>
cudaError_t launch_bc_decay(const Grid& g, R* P, int face, int var, double factor, cudaStream_t s) {
    int a = face / 2;
    long long tot = (long long)g.n[0] * g.n[1] * g.n[2] / g.n[a] * NG;
    k_bc_decay<R><<<grid_for(tot, 256), 256, 0, s>>>(g, P, face, var, factor);
    return cudaGetLastError();
}

// ---- CFL signal speed: per-thread max, warp-shuffle max, block max ----------
constexpr int MS_THREADS = 256;

__device__ __forceinline__ double warp_max(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

__device__ __forceinline__ double block_max(double x) {
    __shared__ double red[MS_THREADS / 32];
    x = warp_max(x);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
        x = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        x = warp_max(x);
    }
    return x;
}

template <int DIM, typename R>
__global__ void __launch_bounds__(MS_THREADS) k_max_speed(Grid g, const R* __restrict__ P, double gamma,
                                                          double* __restrict__ partial) {
    constexpr int NV = 2 + DIM;
    const int N0 = g.n[0] - 2 * NG;
    const int N1 = DIM > 1 ? g.n[1] - 2 * NG : 1;
    const int N2 = DIM > 2 ? g.n[2] - 2 * NG : 1;
    const long long tot = (long long)N0 * N1 * N2;
    double m = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        int i = (int)(e % N0) + NG;
        int j = DIM > 1 ? (int)((e / N0) % N1) + NG : 0;
        int k = DIM > 2 ? (int)(e / ((long long)N0 * N1)) + NG : 0;
        long long c = i + g.sy * j + g.sz * k;
        double q[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) q[v] = (double)P[v * g.vs + c];
        m = fmax(m, max_signal_speed<DIM>(gamma, q));
    }
    m = block_max(m);
    if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

static __global__ void __launch_bounds__(MS_THREADS) k_max_reduce(const double* __restrict__ partial, int n,
                                                           double* __restrict__ out) {
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, partial[i]);
    m = block_max(m);
    if (threadIdx.x == 0) *out = m;
}

template <typename R>
cudaError_t launch_max_speed(const Grid& g, const R* P, double gamma, double* partial, int max_partial,
                             double* out, cudaStream_t s) {
    int nb = min(max_speed_blocks(g), max_partial);
    if (nb < 1) return cudaErrorInvalidValue;
    if (g.dims == 1) k_max_speed<1, R><<<nb, MS_THREADS, 0, s>>>(g, P, gamma, partial);
    else if (g.dims == 2) k_max_speed<2, R><<<nb, MS_THREADS, 0, s>>>(g, P, gamma, partial);
    else k_max_speed<3, R><<<nb, MS_THREADS, 0, s>>>(g, P, gamma, partial);
    k_max_reduce<<<1, MS_THREADS, 0, s>>>(partial, nb, out);
    return cudaGetLastError();
}

// explicit instantiation of every launcher for one bulk type
#define VB_INSTANTIATE_LAUNCHERS(R)                                                                      \
    template cudaError_t launch_stage<R>(int, int, int, const StageParams&, const StageBufs<R>&,       \
                                         cudaStream_t, int*);                                         \
    template cudaError_t launch_load_prims<R>(const Grid&, const double*, R*, double*, double,        \
                                              cudaStream_t);                                          \
    template cudaError_t launch_store_prims<R>(const Grid&, const R*, double*, cudaStream_t);        \
    template cudaError_t launch_init_prims<R>(const Grid&, const InitIC&, R*, double*, double, cudaStream_t); \
    template cudaError_t launch_pack_interior<R>(const Grid&, const R*, double*, unsigned long long*, cudaStream_t); \
    template cudaError_t launch_ghost_limit<R>(const Grid&, const R*, R*, double, cudaStream_t);      \
    template cudaError_t launch_bc_face<R>(const Grid&, R*, int, int, const double*, cudaStream_t);  \
    template cudaError_t launch_bc_decay<R>(const Grid&, R*, int, int, double, cudaStream_t);        \
    template cudaError_t launch_max_speed<R>(const Grid&, const R*, double, double*, int, double*,   \
                                             cudaStream_t);                                          \
    template int stage_div_in_pout<R>(int, int, int, const StageParams&);                             \
    template int stage_split_c2p<R>(int, const StageParams&);

}  // namespace vb
