// Internal interfaces between the kernel translation units and the C ABI.
#pragma once
#include "vb_ns.h"
#include <cuda_runtime.h>
#include <stdint.h>

namespace VB_NS {

constexpr int NG = 3;  // ghost cells per side, as the reference's ParVector2D/3D

// Device counters written by the kernels (all uint64).
enum Counter {
    CNT_C2P_FAIL = 0,      // con2prim found no root (cell set to NaN, as the reference does)
    CNT_C2P_FALLBACK = 1,  // a later stage of the cascade / the bracketed phase was needed
    CNT_C2P_ITERS = 2,     // Newton iterations (statistics mode only)
    CNT_C2P_CELLS = 3,     // cells solved (statistics mode only)
    CNT_TIMEOUT = 4,       // a bounded wait in a persistent kernel gave up
    CNT_BAD_INDEX = 5,     // a work item outside its bounds was skipped
    CNT_C2P_FP64 = 6,      // cells solved by the FP64 Newton of the gated learned refinement (statistics mode)
    CNT_N = 8
};

// Con2prim strategy inside a stage.
enum { C2P_REFERENCE = 0, C2P_GUESS_W = 1 };

struct StageParams {
    int n[3];            // padded extents (unused axes = 1)
    long long sy, sz;    // strides of j and k in cells
    long long vs;        // stride between variables in elements
    double dtdx[3];      // dt_stage / dx_d
    double rk_a, rk_b;   // Uo = rk_a U0 + rk_b (Us - sum dtdx dF); rk_a == 0 -> Uo = Us - ...
    double gamma, floor_, tol;
    int n_iter;
    int c2p_mode;        // C2P_*
    int stats;           // 1: accumulate iteration statistics
    double w_rtol;       // C2P_GUESS_W: relative tolerance of the W Newton
    int w_max_newton;    // C2P_GUESS_W: Newton steps before the bracketed fallback
    const float* w_guess;  // C2P_GUESS_W: per-cell W guesses (nullptr: derive from Pin)
    int c2p_fp32;        // C2P_GUESS_W from learned guesses: precision-gated refinement (c2p_w_gated)
    unsigned int* defer_idx;  // gated fused learned con2prim: interior indices of the cells left to the FP64
                              //    W Newton (capacity: every interior cell), their count in *defer_n and
    unsigned int* defer_n;    //    their FP32 W guesses in defer_w0 (per padded cell); solved by
    float* defer_w0;          //    launch_c2p_deferred after the fused kernel
    unsigned long long* counters;
    int force_box;       // 1: use the box-tile kernel even where the z-marching one fits
    int split;           // 1: z-marching stencil kernel writes U only; k_c2p solves con2prim
    int skip_c2p;        // 1: the stencil kernel writes U only and launches no con2prim
    int pairs;           // 1: FP32-bulk 3D stages use the z-pair kernel where it exists
    int div_in_pout;     // 1: the stencil kernel left the FP32 divergence in Pout; the
                         //    con2prim kernel forms Uo = rk_a U0 + rk_b (Us - div) itself
    int want_div;        // 1: the caller's con2prim kernel (skip_c2p) accepts div_in_pout
    int c2p_rescue;      // 1: 1D / 2D cells whose reference Newton diverges are solved by the
                         //    bracketed W Newton (batched problems); 0: kept and counted as failures
    const void* tmap_in; // host CUtensorMap of Pin (encode_stage_tmap) for the TMA forms: the 3D
                         //    z-pair kernel's planes, k_stage's 2D tiles; nullptr: staged by loads
};

template <typename R> struct StageBufs {
    const R* Pin;
    R* Pout;
    const double* U0;
    const double* Us;
    double* Uo;
};

struct Grid {
    int dims, nv;
    int n[3];   // padded extents
    long long sy, sz, vs;  // SoA strides of j, k and the variable (sy >= n[0]: rows may be pitched)
};

// ---- launchers, explicitly instantiated for R = double (vb_stage_f64.cu) and
// R = float (vb_stage_f32.cu) --------------------------------------------------
template <typename R>
cudaError_t launch_stage(int dims, int rec, int rs, const StageParams& p, const StageBufs<R>& b,
                         cudaStream_t s, int* kernels);
// AoS (Julia column-major, variable fastest) FP64 -> internal SoA R; also U0 = PtoU(P) in FP64
template <typename R>
cudaError_t launch_load_prims(const Grid& g, const double* P_aos, R* P, double* U0, double gamma,
                              cudaStream_t s);
template <typename R>
cudaError_t launch_store_prims(const Grid& g, const R* P, double* P_aos, cudaStream_t s);
// interior cells of P -> the reference's interior layout (nvar, Nx, Ny[, Nz]), FP64,
// column-major, variable fastest; adds the count of NaN values to *nan_count
template <typename R>
cudaError_t launch_pack_interior(const Grid& g, const R* P, double* out, unsigned long long* nan_count,
                                 cudaStream_t s);
// initial condition generated on the device (vb_init_prims): P on every cell, U0 = PtoU(P)
struct InitIC {
    int kind;  // 0 ambient, 1 star + jet engine
    unsigned long long seed;
    double noise, rho, u;
    double dx[3], box[3];
    double r_max, r_eng, rho0, temp, outer, gamma0, engine_rho, engine_temp;
};
template <typename R>
cudaError_t launch_init_prims(const Grid& g, const InitIC& ic, R* P, double* U0, double gamma, cudaStream_t s);
// ghost cells of Pout = limit(ghost cells of Pin)
template <typename R>
cudaError_t launch_ghost_limit(const Grid& g, const R* Pin, R* Pout, double floor_, cudaStream_t s);
// boundary fill of one face (kind: 0 outflow, 2 nozzle); decay of a FIXED face
template <typename R>
cudaError_t launch_bc_face(const Grid& g, R* P, int face, int kind, const double* par, cudaStream_t s);
template <typename R>
cudaError_t launch_bc_decay(const Grid& g, R* P, int face, int var, double factor, cudaStream_t s);
// per-block maxima of the CFL signal speed into partial[], then one block reduces them to out
template <typename R>
cudaError_t launch_max_speed(const Grid& g, const R* P, double gamma, double* partial, int max_partial,
                             double* out, cudaStream_t s);

// 1D reference solver (src/1dim/algos.jl:58-315), FP64, one persistent CTA.
struct Ref1DState {
    int N;
    double *P, *Ph, *U, *Uh, *PL, *PR, *F;  // [3][N] each
};
cudaError_t launch_ref1d_init(const Ref1DState& st, const double* P_aos, double gamma, cudaStream_t s);
cudaError_t launch_ref1d_steps(const Ref1DState& st, double gamma, int rec, int n_iter, double tol,
                               double dt, double dx, int nsteps, cudaStream_t s);
cudaError_t launch_ref1d_store(const Ref1DState& st, double* P_aos, cudaStream_t s);

int max_speed_blocks(const Grid& g);

// FP32-bulk z-pair variant of the 3D stage (vb_stage_zp.cuh, instantiated in
// vb_stage_f32.cu): WENOZ reconstruction with HLL or HLLC
inline bool zp_available(int rec, int rs) { return rec >= 0 && rec <= 2 && (rs == 0 || rs == 1); }
cudaError_t launch_stage_zp(int rec, int rs, const StageParams& p, const StageBufs<float>& b, cudaStream_t s);
// tensor map of one SoA state array for the TMA forms of the stage kernels
// (3D FP32: the z-pair kernel's plane boxes; 2D: k_stage's tile boxes; out: a
// 64-byte aligned CUtensorMap); false where no TMA form exists or the layout
// does not allow one
template <typename R> bool encode_stage_tmap(void* out, const R* P, const Grid& g);
// 1 when launch_stage with these arguments leaves the FP32 divergence in Pout
// for the caller's con2prim kernel (z-pair kernel with skip_c2p and want_div)
template <typename R> int stage_div_in_pout(int dims, int rec, int rs, const StageParams& p);
// 1 when launch_stage with these arguments launches the stencil kernel and then
// the split con2prim kernel k_c2p (3D z-marching stage, split con2prim); the
// same work is then launch_stage with skip_c2p = 1 and want_div = 0 followed
// by launch_c2p (the profiling path records an event between the two)
template <typename R> int stage_split_c2p(int dims, const StageParams& p);

// split con2prim of a 3D stage on its own (vb_stage_zm.cuh)
template <typename R> cudaError_t launch_c2p(const StageParams& p, const StageBufs<R>& b, cudaStream_t s);

// learned guess of a split stage (vb_mlp.cu): W guess per interior cell of U
// (padded SoA, the grid of p) into w_guess (one float per padded cell)
cudaError_t launch_mlp_guess(const void* mlp_blob, const StageParams& p, const double* U, float* w_guess,
                             unsigned int* err, cudaStream_t s);
// the same guess and the W Newton from it in one kernel (vb_mlp.cu): U of the
// stage in, the floored P of every interior cell out
template <typename R>
cudaError_t launch_c2p_learned(const void* mlp_blob, const StageParams& p, const StageBufs<R>& b, unsigned int* err,
                               cudaStream_t s);
// the cells the gated fused kernel left (p.defer_idx, *p.defer_n, p.defer_w0):
// the FP64 W Newton from their guesses, floors, P (vb_mlp.cu)
template <typename R> cudaError_t launch_c2p_deferred(const StageParams& p, const StageBufs<R>& b, cudaStream_t s);

// point kernels (FP64, vb_stage_f64.cu)
cudaError_t launch_point_recon(int method, const double* q, double* out, int n, cudaStream_t s);
cudaError_t launch_point_flux(int dims, int axis, int rs, double g, const double* PL, const double* PR, double* F,
                              int n, cudaStream_t s);
cudaError_t launch_point_con2prim(int dims, double g, int n_iter, double tol, const double* U, double* P, int* ret,
                                  int n, cudaStream_t s);
cudaError_t launch_point_c2p_w(double g, const double* U, const double* W0, double rtol, int max_newton,
                               int max_bracket, double* P, int* iters, int* fallback, int n, cudaStream_t s);
cudaError_t launch_point_c2p_gated(double g, const double* U, const float* W0, double rtol, int max_newton,
                                   int max_bracket, double* P, int* iters, int* fp64, int n, cudaStream_t s);

}  // namespace vb

// FP64 stage kernels built with FMA contraction (vb_stage_f64c.cu, namespace
// vb_f64c): launch_stage<double> and launch_c2p<double> of that unit. p and b
// point to the caller's StageParams and StageBufs<double> (the same header, so
// the same layout; vb_f64c_stage_params_size() lets the caller check it).
cudaError_t vb_f64c_launch_stage(int dims, int rec, int rs, const void* p, const void* b, cudaStream_t s,
                                 int* kernels);
cudaError_t vb_f64c_launch_c2p(const void* p, const void* b, cudaStream_t s);
size_t vb_f64c_stage_params_size();
