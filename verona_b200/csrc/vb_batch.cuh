// Batched independent problems in one persistent launch.
//
// A batch holds many 1D and 2D problems of uneven size (their own grid,
// reconstruction, cell widths and time step; shared gamma, Riemann solver,
// RK scheme and precision; outflow on every face). One launch advances every
// problem by nsteps time steps:
//
//   * The work of one RK stage of one problem is a set of tiles (TX2 x TY2
//     cells in 2D, pencils of L1 cells in 1D). Tickets enumerate
//     (step, stage, tile) stage-major -- within a stage the largest problems
//     first -- and each CTA of the persistent grid takes the next ticket with
//     one atomicAdd.
//   * A tile of global stage g of problem p may start once all tiles of stage
//     g - 1 of p are done: a per-problem completion counter, read with
//     acquire semantics in a bounded wait. Every ticket a tile waits for is
//     smaller than its own and is held by a CTA that is running, so the wait
//     always ends; a wait that runs out (a fault elsewhere, or a limit set
//     too small by vb_batch_set_wait_limit) counts CNT_TIMEOUT and stops the
//     CTA. The tiles that depend on the stopped one then run out in turn, so
//     the launch ends in bounded time; vb_batch_check reports it.
//   * The tile itself is the box-tile stage body (stage_tile, vb_stage.cuh)
//     with loads through L2, so data written earlier in the launch by other
//     SMs is seen.
//   * Ghost cells follow the single-grid solver exactly: at the first stage of
//     a step a tile on a domain edge copies the first interior cell into the
//     ghost layers it reads (outflow, src/3dim/sync_CUDA.jl semantics of the
//     examples' zero-gradient TurnOff) and writes the floored copy to the
//     stage output; later stages copy the floored ghosts of their input.
#pragma once
#include "vb_ns.h"
#include <type_traits>
#include "vb_batch.h"
#include "vb_stage.cuh"

namespace VB_NS {

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Ghost layers read by one tile: x-ghosts of its rows on an x edge, y-ghosts
// of its columns on a y edge. At the first stage of a step (first) they are
// filled as the single-grid solver fills them at the start of the step
// (vb_set_boundary kinds, launch_bc_face / launch_bc_decay): OUTFLOW copies
// the first interior cell, NOZZLE holds the inflow state inside the radius
// (cells measured from the centre along the face) and copies outside it,
// FIXED keeps the loaded ghosts and multiplies the decaying variable by its
// factor while t_on < t < t_off (t: the problem's time at the start of the
// step). The stage output gets the floored ghosts (k_ghost_limit); later
// stages copy the floored ghosts of their input.
template <typename R>
__device__ __forceinline__ void batch_ghosts(const StageParams& q, const BatchProb& pr, const R* Pin_c, R* Pout,
                                             int bx, int by, int TXc, int TYc, bool first, double t) {
    R* Pin = const_cast<R*>(Pin_c);
    const int dims = pr.dims, nv = 2 + dims;
    const R fl = R(q.floor_);
    const int n0 = q.n[0], n1 = q.n[1];
    const int ox = NG + bx * TXc, oy = dims > 1 ? NG + by * TYc : 0;
    const int vx = min(TXc, n0 - NG - ox), vy = dims > 1 ? min(TYc, n1 - NG - oy) : 1;
    // up to four edges: x-lo, x-hi (rows oy..oy+vy), y-lo, y-hi (columns ox..ox+vx)
    for (int edge = 0; edge < 4; ++edge) {
        const bool on =
            edge == 0 ? bx == 0 : edge == 1 ? bx == pr.ntx - 1 : dims > 1 && (edge == 2 ? by == 0 : by == pr.nty - 1);
        if (!on) continue;
        const int kind = pr.bc_kind[edge];
        const double* par = pr.bc_par[edge];
        const int dvar = first && kind == 1 && par[0] >= 0.0 && t > par[1] && t < par[2] ? (int)par[0] : -1;
        const int len = edge < 2 ? vy : vx;
        for (int e = threadIdx.x; e < NG * len; e += blockDim.x) {
            const int layer = e / len, r = e - layer * len;
            int gi, gj, si, sj;
            if (edge < 2) {
                gj = oy + r;
                sj = gj;
                gi = edge == 0 ? layer : n0 - NG + layer;
                si = edge == 0 ? NG : n0 - NG - 1;
            } else {
                gi = ox + r;
                si = gi;
                gj = edge == 2 ? layer : n1 - NG + layer;
                sj = edge == 2 ? NG : n1 - NG - 1;
            }
            bool inside = false;
            if (kind == 2) {
                const double y1 = dims > 1 ? ((edge < 2 ? gj : gi) - NG + 0.5) - par[1] : 0.0;
                inside = y1 * y1 < par[0] * par[0];
            }
            const long long c = gi + q.sy * gj, cs = si + q.sy * sj;
            for (int v = 0; v < nv; ++v) {
                R x;
                if (!first) {
                    x = __ldcg(Pin + v * q.vs + c);
                } else if (kind == 1) {
                    x = __ldcg(Pin + v * q.vs + c);
                    if (v == dvar) {
                        x = (R)((double)x * par[3]);
                        Pin[v * q.vs + c] = x;
                    }
                } else if (inside) {
                    x = (R)par[v < 2 ? 3 + v : 5 + (v - 2)];
                    Pin[v * q.vs + c] = x;
                } else {
                    x = __ldcg(Pin + v * q.vs + cs);
                    Pin[v * q.vs + c] = x;
                }
                if (v < 2) x = jmax(x, fl);
                Pout[v * q.vs + c] = x;
            }
        }
    }
}

template <typename R, int RS, int TX2, int TY2, int L1>
__global__ void __launch_bounds__(BATCH_NT) k_batch(BatchLaunch<R> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ long long s_ticket;
    __shared__ int s_ok;
    for (;;) {
        if (threadIdx.x == 0) s_ticket = (long long)atomicAdd(a.next, 1ULL);
        __syncthreads();
        const long long t = s_ticket;
        if (t >= a.total) break;
        const long long g = t / a.T;
        const BatchTile e = a.tiles[t - g * a.T];
        const BatchProb& pr = a.prob[e.p];
        if (threadIdx.x == 0) {
            const unsigned long long need = (unsigned long long)g * (unsigned long long)pr.ntiles;
            int ok = 1;
            for (unsigned it = 0; ld_acquire_u64(a.done + e.p) < need; ++it) {
                if (it >= a.max_polls) {
                    ok = 0;
                    atomicAdd(a.counters + CNT_TIMEOUT, 1ULL);
                    break;
                }
                __nanosleep(128);
            }
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) break;
        __threadfence();

        // stage of this ticket
        const int step = (int)(g / a.nstages), st = (int)(g - (long long)step * a.nstages);
        const int c = a.rk == 3 ? (a.cur0 ^ (step & 1)) : a.cur0;
        R* Pc = (c ? a.P1 : a.P0) + pr.offP;
        R* Pn = (c ? a.P0 : a.P1) + pr.offP;
        double* U0 = a.U0 + pr.offU;
        double* U1 = a.U1 + pr.offU;
        StageParams q{};
        q.n[0] = pr.n0;
        q.n[1] = pr.n1;
        q.n[2] = 1;
        q.sy = pr.n0;
        q.sz = (long long)pr.n0 * pr.n1;
        q.vs = pr.vs;
        q.gamma = a.gamma;
        q.floor_ = a.floor_;
        q.tol = a.tol;
        q.n_iter = a.n_iter;
        q.stats = a.stats;
        // FP64: the reference con2prim (parity with the single-grid solver);
        // FP32 bulk: the W Newton from the input state first (cheaper, no LU)
        q.c2p_mode = std::is_same<R, float>::value ? C2P_GUESS_W : C2P_REFERENCE;
        q.c2p_rescue = 1;
        q.w_rtol = 1e-12;
        q.w_max_newton = 8;
        q.counters = a.counters;
        const bool half = a.rk == 2 && st == 0;
        q.dtdx[0] = half ? pr.dtdx[1][0] : pr.dtdx[0][0];
        q.dtdx[1] = pr.dims > 1 ? (half ? pr.dtdx[1][1] : pr.dtdx[0][1]) : 0.0;
        q.dtdx[2] = 0.0;
        StageBufs<R> b;
        if (a.rk == 3) {
            // SSP-RK3: U1 = U - dt L(P); U2 = 3/4 U + 1/4 (U1 - dt L(P1)); U = 1/3 U + 2/3 (U2 - dt L(P2))
            q.rk_a = st == 0 ? 0.0 : (st == 1 ? 0.75 : 1.0 / 3.0);
            q.rk_b = st == 0 ? 1.0 : (st == 1 ? 0.25 : 2.0 / 3.0);
            b.Pin = (st & 1) ? Pn : Pc;
            b.Pout = (st & 1) ? Pc : Pn;
            b.Us = st == 0 ? U0 : U1;
            b.Uo = st == 2 ? U0 : U1;
        } else {
            // midpoint RK2: Uhalf = U - dt/2 L(P); U = U - dt L(Phalf)
            q.rk_a = 0.0;
            q.rk_b = 1.0;
            b.Pin = st ? Pn : Pc;
            b.Pout = st ? Pc : Pn;
            b.Us = U0;
            b.Uo = st ? U0 : U1;
        }
        b.U0 = U0;

        const int TXc = pr.dims == 1 ? L1 : TX2, TYc = pr.dims == 1 ? 1 : TY2;
        // the problem's time at the start of this step: its time at the start
        // of the launch plus dt once per earlier step (the host's additions)
        double tstep = a.time[e.p];
        for (int k = 0; k < step; ++k) tstep += pr.dt;
        batch_ghosts<R>(q, pr, b.Pin, b.Pout, e.x, e.y, TXc, TYc, st == 0, tstep);
        __threadfence_block();
        __syncthreads();
        if (pr.dims == 1) {
            if (pr.rec == REC_MINMOD)
                stage_tile<1, REC_MINMOD, RS, R, L1, 1, 1, BATCH_NT, true>(q, b, e.x, 0, 0, smem_raw);
            else if (pr.rec == REC_PPM)
                stage_tile<1, REC_PPM, RS, R, L1, 1, 1, BATCH_NT, true>(q, b, e.x, 0, 0, smem_raw);
            else
                stage_tile<1, REC_WENOZ, RS, R, L1, 1, 1, BATCH_NT, true>(q, b, e.x, 0, 0, smem_raw);
        } else {
            if (pr.rec == REC_MINMOD)
                stage_tile<2, REC_MINMOD, RS, R, TX2, TY2, 1, BATCH_NT, true>(q, b, e.x, e.y, 0, smem_raw);
            else if (pr.rec == REC_PPM)
                stage_tile<2, REC_PPM, RS, R, TX2, TY2, 1, BATCH_NT, true>(q, b, e.x, e.y, 0, smem_raw);
            else
                stage_tile<2, REC_WENOZ, RS, R, TX2, TY2, 1, BATCH_NT, true>(q, b, e.x, e.y, 0, smem_raw);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(a.done + e.p, 1ULL);
        }
    }
}

// tile shapes of the kernel variants the autotuner chooses among
template <typename R> struct BatchVariants;
template <> struct BatchVariants<float> {
    static constexpr int N = 4;
    static constexpr int TX2[N] = {32, 32, 64, 16}, TY2[N] = {8, 16, 4, 16}, L1[N] = {256, 512, 128, 256};
};
template <> struct BatchVariants<double> {
    static constexpr int N = 2;
    static constexpr int TX2[N] = {32, 16}, TY2[N] = {8, 8}, L1[N] = {256, 128};
};

template <typename R, int TX2, int TY2, int L1> constexpr size_t batch_smem() {
    return TileGeom<2, TX2, TY2, 1>::template smem_bytes<R>() > TileGeom<1, L1, 1, 1>::template smem_bytes<R>()
               ? TileGeom<2, TX2, TY2, 1>::template smem_bytes<R>()
               : TileGeom<1, L1, 1, 1>::template smem_bytes<R>();
}

// launch = false: set the kernel attributes and compute the grid only (before
// a stream capture)
template <typename R, int RS, int TX2, int TY2, int L1>
cudaError_t batch_launch_t(const BatchLaunch<R>& a, int ctas_per_sm, cudaStream_t s, int* grid_out, bool launch) {
    auto kern = k_batch<R, RS, TX2, TY2, L1>;
    constexpr size_t smem = batch_smem<R, TX2, TY2, L1>();
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
    int nsm = 0, maxb = 0;
    cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxb, kern, BATCH_NT, smem);
    if (e != cudaSuccess) return e;
    if (maxb < 1) return cudaErrorInvalidConfiguration;
    const int per = ctas_per_sm > 0 ? std::min(ctas_per_sm, maxb) : maxb;
    long long grid = (long long)per * nsm;
    if (grid > a.total) grid = a.total > 0 ? a.total : 1;
    *grid_out = (int)grid;
    if (!launch) return cudaSuccess;
    kern<<<(int)grid, BATCH_NT, smem, s>>>(a);
    return cudaGetLastError();
}

template <typename R, int RS>
cudaError_t batch_launch_rs(const BatchLaunch<R>& a, int variant, int ctas_per_sm, cudaStream_t s, int* grid,
                            bool launch) {
    using V = BatchVariants<R>;
    switch (variant) {
#define VB_BV(I)                                                                                        \
    case I:                                                                                             \
        if constexpr (I < V::N)                                                                         \
            return batch_launch_t<R, RS, V::TX2[I < V::N ? I : 0], V::TY2[I < V::N ? I : 0],            \
                                  V::L1[I < V::N ? I : 0]>(a, ctas_per_sm, s, grid, launch);             \
        break;
        VB_BV(0)
        VB_BV(1)
        VB_BV(2)
        VB_BV(3)
#undef VB_BV
        default:
            break;
    }
    return cudaErrorInvalidValue;
}

template <typename R>
cudaError_t batch_launch_impl(const BatchLaunch<R>& a, int riemann, int variant, int ctas_per_sm, cudaStream_t s,
                              int* grid, bool launch) {
    if (riemann == RS_HLLC) return batch_launch_rs<R, RS_HLLC>(a, variant, ctas_per_sm, s, grid, launch);
    return batch_launch_rs<R, RS_HLL>(a, variant, ctas_per_sm, s, grid, launch);
}

#define VB_INSTANTIATE_BATCH(R)                                                                          \
    template <>                                                                                         \
    cudaError_t batch_launch<R>(const BatchLaunch<R>& a, int riemann, int variant, int ctas_per_sm,      \
                                cudaStream_t s, int* grid, bool launch) {                               \
        return batch_launch_impl<R>(a, riemann, variant, ctas_per_sm, s, grid, launch);                 \
    }                                                                                                   \
    template <> int batch_num_variants<R>() { return BatchVariants<R>::N; }                              \
    template <> void batch_variant_shape<R>(int v, int* tx2, int* ty2, int* l1) {                         \
        *tx2 = BatchVariants<R>::TX2[v];                                                                \
        *ty2 = BatchVariants<R>::TY2[v];                                                                \
        *l1 = BatchVariants<R>::L1[v];                                                                  \
    }

}  // namespace vb
