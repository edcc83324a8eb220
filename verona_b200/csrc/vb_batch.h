// Batched problems: the launch description shared by the batch kernel
// (vb_batch.cuh) and its host API (vb_batch.cu).
#pragma once
#include "vb_ns.h"
#include <cuda_runtime.h>

#include "vb_internal.h"

namespace VB_NS {

constexpr int BATCH_NT = 256;  // threads per CTA of the batch kernel
constexpr unsigned BATCH_MAX_POLLS = 1u << 24;  // default wait bound, x ~128 ns: a few seconds

struct BatchProb {
    int dims, rec;
    int n0, n1;             // padded extents (n1 = 1 in 1D)
    int ntx, nty;           // tiles per axis (current variant)
    long long ntiles;
    long long offP, offU;   // element offset of variable 0 in the P / U pools
    long long vs;           // variable stride
    double dtdx[2][2];      // [full dt, half dt (RK2 stage 1)][axis]
    double dt;              // time step (the time of a step for a decaying FIXED face)
    int bc_kind[4];         // per face x-lo, x-hi, y-lo, y-hi: 0 outflow, 1 fixed, 2 nozzle (VB_BC_*)
    int bc_pad;
    double bc_par[4][8];    // FIXED {var (< 0: no decay), t_on, t_off, factor}; NOZZLE {radius, c1, c2,
                            // rho, u, u1[, u2]} (vb_set_boundary's parameters)
};

struct BatchTile {
    int p, x, y, pad;
};

template <typename R> struct BatchLaunch {
    const BatchProb* prob;
    const BatchTile* tiles;  // one stage's tiles, largest problems first
    long long T;             // tiles per stage
    long long total;         // nsteps * nstages * T
    int nstages, rk, cur0;   // cur0: P buffer holding the state at the first step
    unsigned max_polls;      // bound of a tile's wait for the previous stage (vb_batch_set_wait_limit)
    R* P0;
    R* P1;
    double* U0;
    double* U1;
    const double* time;        // per problem: its time at the start of the launch
    unsigned long long* done;  // per problem
    unsigned long long* next;  // ticket counter
    unsigned long long* counters;
    double gamma, floor_, tol;
    int n_iter, stats;
};

// one persistent launch of the batch kernel (instantiated for R = float in
// vb_batch_f32.cu and R = double in vb_batch_f64.cu); *grid receives the CTA
// count. launch = false only sets the kernel attributes and computes the grid.
template <typename R>
cudaError_t batch_launch(const BatchLaunch<R>& a, int riemann, int variant, int ctas_per_sm, cudaStream_t s,
                         int* grid, bool launch);
// advance every problem's device time by nsteps steps (t += dt, one step at a
// time, the same additions the host makes); the graph's last node
cudaError_t batch_advance_time(const BatchProb* prob, double* time, int nprob, int nsteps, cudaStream_t s);
// number of tile-shape variants and the shape of one: 2D tile TX2 x TY2, 1D pencil L1
template <typename R> int batch_num_variants();
template <typename R> void batch_variant_shape(int v, int* tx2, int* ty2, int* l1);

}  // namespace vb
