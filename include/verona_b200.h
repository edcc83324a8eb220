/*
 * verona_b200.h -- C ABI of the B200 SRHD step library (libverona_b200.so).
 *
 * Drop-in for the per-timestep update of Wesenheit/Verona's HARM_HLL solvers:
 *   Verona3D.HARM_HLL   src/3dim/algos.jl:203-362
 *   Verona2D.HARM_HLL   src/2dim/algos.jl:192-324
 *   Verona1D.HARM_HLL   src/1dim/algos.jl:58-315
 * The Julia host keeps grid/state construction, boundary choice, the time
 * loop and HDF5 output; it hands the library the device pointer of P.arr and
 * calls vb_step between dumps. Plain pointers, sizes and an opaque handle
 * only: no C++ or framework types cross this boundary.
 *
 * Conventions
 *  - Every function returns VB_OK (0) or a negative VB_ERR_* code; the text
 *    of the last error of a handle is returned by vb_last_error(h) (or the
 *    last global error for h == NULL). No exceptions cross the ABI and no
 *    device code traps: con2prim failures are counted (vb_get_counters), as
 *    the reference marks them with NaN (src/3dim/structs.jl:612-619).
 *  - Primitive arrays at the boundary are the reference's own layout: FP64,
 *    column-major (nvar, Nx+6, Ny+6[, Nz+6]) with the variable index fastest
 *    and 3 ghost cells per side (src/3dim/structs.jl:28-64); nvar = 2 + dims,
 *    P = (rho, u, u^x[, u^y[, u^z]]). The 1D reference layout (nghost = 0)
 *    is (3, N) with no ghosts (src/1dim/structs.jl:22-34).
 *  - `stream` is a cudaStream_t (CUDA.jl: stream().handle); NULL is the
 *    legacy default stream. Work is enqueued on it; only functions that
 *    return host values or read host buffers synchronise it.
 *  - A handle belongs to one host thread and one device (the device current
 *    at vb_create).
 */
#ifndef VERONA_B200_H
#define VERONA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VB_ABI_VERSION 1

enum vb_status_code {
    VB_OK = 0,
    VB_ERR_ARG = -1,         /* invalid argument */
    VB_ERR_CUDA = -2,        /* CUDA runtime error (message in vb_last_error) */
    VB_ERR_STATE = -3,       /* call not valid in the handle's current state */
    VB_ERR_UNSUPPORTED = -4, /* option combination not provided */
    VB_ERR_NOMEM = -5,       /* device allocation failed */
    VB_ERR_TIMEOUT = -6      /* a bounded device-side wait gave up */
};

/* reconstruction, src/fluxlimiter.jl:183-200 (`reconstruction(::Val{M})`) */
enum { VB_RECON_MINMOD = 0, VB_RECON_PPM = 1, VB_RECON_WENOZ = 2 };
/* Riemann solver: the reference is HLL (src/3dim/algos.jl:149-174); HLLC is an extension */
enum { VB_RIEMANN_HLL = 0, VB_RIEMANN_HLLC = 1 };
/* time integrator: 2 = the reference's midpoint RK2 (src/3dim/algos.jl:279-327); 3 = SSP-RK3 */
enum { VB_RK2 = 2, VB_RK3 = 3 };
/* precision: FP64 everywhere (reference), or FP32 reconstruction/flux/divergence with
 * FP64 conserved variables, RK accumulation and con2prim */
enum { VB_PREC_FP64 = 0, VB_PREC_FP32_BULK = 1 };
/* con2prim initial guess: the cell's previous primitive state with the
 * reference's con2prim cascade (reference); the learned BF16 MLP guess
 * refined by the W Newton (3D only); or the previous state's W refined by that
 * same W Newton (2D and 3D: in 3D the learned path without the network, the
 * baseline of what the network gains; in 2D the state is padded to three
 * momenta with u^z = 0) */
enum { VB_GUESS_PREVIOUS = 0, VB_GUESS_LEARNED = 1, VB_GUESS_PREVIOUS_W = 2 };
/* boundary kinds of vb_set_boundary */
enum {
    VB_BC_OUTFLOW = 0, /* zero-gradient copy of the first interior cell (TurnOff's y/z/x-high copies) */
    VB_BC_FIXED = 1,   /* ghosts keep what was loaded; optional decay {var, t_on, t_off, factor} */
    VB_BC_NOZZLE = 2   /* {radius, c1, c2, rho, u, u1, u2, u3}: fixed inflow inside, outflow outside */
};
enum { VB_FACE_XLO = 0, VB_FACE_XHI = 1, VB_FACE_YLO = 2, VB_FACE_YHI = 3, VB_FACE_ZLO = 4, VB_FACE_ZHI = 5 };
/* indices of vb_get_counters */
enum {
    VB_CNT_C2P_FAIL = 0,     /* cells where con2prim found no root (set to NaN) */
    VB_CNT_C2P_FALLBACK = 1, /* cells that needed a fallback stage */
    VB_CNT_C2P_ITERS = 2,    /* Newton iterations (options.stats = 1) */
    VB_CNT_C2P_CELLS = 3,    /* cells solved (options.stats = 1) */
    VB_CNT_TIMEOUT = 4,      /* bounded device waits that gave up */
    VB_CNT_BAD_INDEX = 5,    /* out-of-range work items that were skipped */
    VB_CNT_C2P_FP64 = 6,     /* cells solved by the FP64 Newton (options.stats = 1; learned guess) */
    VB_CNT_N = 8
};

typedef struct vb_options {
    uint32_t version;     /* VB_ABI_VERSION */
    int32_t recon;        /* VB_RECON_*; the 2D/3D reference is WENOZ */
    int32_t riemann;      /* VB_RIEMANN_* */
    int32_t rk;           /* VB_RK2 | VB_RK3 */
    int32_t precision;    /* VB_PREC_* */
    int32_t guess;        /* VB_GUESS_* */
    int32_t n_iter;       /* Newton iteration cap: HARM_HLL kwargs[1] (src/3dim/algos.jl:290) */
    int32_t stats;        /* 1: count Newton iterations (slower) */
    double tol;           /* Newton tolerance: HARM_HLL kwargs[2] */
    double floor_;        /* density / internal-energy floor: HARM_HLL `floor` */
    double w_rtol;        /* learned guess: relative W tolerance of the refinement (1e-12) */
    int32_t w_max_newton; /* learned guess: Newton steps before the bracketed fallback (8) */
    int32_t c2p_fp32;     /* W-Newton guesses + FP32 bulk: 1 = precision-gated con2prim: an FP32
                           * Newton on the pressure where the guess has Lorentz factor below
                           * sqrt 2 and kinetic energy below 10 x the pressure, the FP64 W Newton
                           * elsewhere (for the learned guess, in a second kernel over the cells
                           * the gate leaves; default); 0 = the FP64 W Newton on every cell (the
                           * faster form once more than about 2 % of the cells are relativistic
                           * or cold and moving, since the second pass gathers them one by one,
                           * and with VB_GUESS_PREVIOUS_W, whose one-cell-per-thread kernel runs
                           * the FP64 fallback inline: 4.7 against 4.1 ms per 512^3 stage) */
    int32_t reserved_i[6];
    double reserved_d[4];
} vb_options;

typedef struct vb_solver* vb_handle;

/* Fill *o with the reference's defaults (WENOZ, HLL, RK2, FP64, previous-state
 * guess, n_iter 50, tol 1e-10, floor 1e-7) and the extensions' (w_rtol 1e-12,
 * w_max_newton 8, c2p_fp32 1). */
int vb_default_options(vb_options* o);

/* Create a solver for an nx x ny x nz interior grid (ny = nz = 1 in 1D,
 * nz = 1 in 2D). nghost = 3 selects the 2D/3D reference semantics and their
 * ghost-cell layout (src/{2,3}dim/algos.jl; also generic 1D); nghost = 0 with
 * dims = 1 selects the 1D reference solver on N = nx cells
 * (src/1dim/algos.jl:58-315). Replaces HARM_HLL's allocations
 * (src/3dim/algos.jl:221-257). */
int vb_create(vb_handle* h, int dims, int nx, int ny, int nz, int nghost, const vb_options* o);
int vb_destroy(vb_handle h);
const char* vb_last_error(vb_handle h);

/* Polytrope{T}(gamma), src/eos.jl:7-9 */
int vb_set_eos(vb_handle h, double gamma);
/* dx, dy, dz of HARM_HLL */
int vb_set_grid(vb_handle h, double dx, double dy, double dz);
/* Built-in replacement of the host `fun_bound` callback
 * (examples/Jet3D/HARM_jet_breakout.jl:131-158): applied on the device at the
 * start of every step, decay first, then faces y-lo, y-hi, z-lo, z-hi, x-lo,
 * x-hi. Default: OUTFLOW on every face. */
int vb_set_boundary(vb_handle h, int face, int kind, const double* params, int nparams);

/* Load P (device, reference layout) and compute U = PtoU(P) on all cells
 * (kernel_PtoU, src/3dim/structs.jl:66-81; called at src/3dim/algos.jl:259). */
int vb_load_prims(vb_handle h, const double* P_aos_dev, void* stream);
/* Write the current P into a device array of the reference layout. */
int vb_store_prims(vb_handle h, double* P_aos_dev, void* stream);
/* Host-buffer variants (pinned or pageable); they return after the copy. */
int vb_load_prims_host(vb_handle h, const double* P_aos_host, void* stream);
int vb_store_prims_host(vb_handle h, double* P_aos_host, void* stream);
/* Current conserved state U in the reference layout (device pointer). */
int vb_store_cons(vb_handle h, double* U_aos_dev, void* stream);

/* Initial conditions generated on the device, replacing the examples' host
 * loops over every cell (examples/Jet3D/HARM_jet_breakout.jl:72-118,
 * examples/Jet2D/HARM_jet_breakout.jl:37-72) followed by the upload. Every
 * cell, ghosts included, gets P; then U = PtoU(P) as vb_load_prims does.
 * The density noise is a standard normal per cell from (seed, padded linear
 * cell index): splitmix64 words and Box-Muller, reproducible for any launch
 * shape (the examples draw from per-thread MersenneTwister streams, whose
 * values depend on the thread schedule). */
enum {
    VB_IC_AMBIENT = 0, /* rho (1 + noise N(0,1)), u, zero velocity on every cell; any dims */
    VB_IC_STAR_JET = 1 /* the examples' stellar envelope with a jet engine; 2D and 3D */
};
typedef struct vb_ic_params {
    uint32_t version; /* VB_ABI_VERSION */
    int32_t kind;     /* VB_IC_* */
    uint64_t seed;
    double noise;     /* relative density noise (the examples: 3e-2) */
    double rho, u;    /* AMBIENT: density and internal energy density */
    /* STAR_JET: cell (i, j, k) (1-based over the padded grid) sits at X = i dx,
     * Y = j dy - box_Y, Z = k dz - box_Z with dx = box_X / (Nx + 6),
     * dy = 2 box_Y / (Ny + 6), dz = 2 box_Z / (Nz + 6); R = |(X, Y[, Z])|.
     * rho = rho0 (r_max / max(R, r_eng))^2 (1 + noise N) for R < r_max, else
     * outer; u = temp rho. For R < r_eng: rho *= engine_rho, u = engine_temp rho,
     * u^x = gamma0 / (1 - 1/gamma0^2) / cosh(s / r_eng)^8 with s = sqrt(X^2 + Y^2)
     * in 3D and s = Y in 2D (the examples' expressions). */
    double box[3];
    double r_max, r_eng, rho0, temp, outer, gamma0, engine_rho, engine_temp;
    double reserved_d[4];
} vb_ic_params;
/* Asynchronous dump of the interior primitives, the data of the reference's
 * SaveHDF5Gather / SaveHDF5Parallel (src/3dim/saving.jl:1-146:
 * Array(P.arr[:, 4:end-3, 4:end-3, 4:end-3]) and its NaN check); the caller
 * writes the HDF5 file ("data", plus "T" / "grid") as the reference does.
 * vb_dump_begin: at this point of `stream` the interior P is packed into
 * host_out's layout, (nvar, Nx, Ny[, Nz]) FP64 column-major, in a device
 * buffer of the handle (allocated on the first dump), and copied to host_out
 * on a copy stream of the handle while later work on `stream` (vb_step)
 * proceeds; host_out must stay valid until vb_dump_wait and should be pinned
 * (a pageable buffer makes the copy synchronous). The NaN values of the
 * snapshot are counted on the device. vb_dump_wait blocks until the copy has
 * landed and returns that count. One dump in flight per handle: a second
 * vb_dump_begin orders itself after the previous copy. */
int vb_dump_begin(vb_handle h, double* host_out, void* stream);
int vb_dump_wait(vb_handle h, uint64_t* nan_count);

/* Fill *ic with the example values for dims (2 or 3; AMBIENT: rho 1, u 3e-3). */
int vb_default_ic(int dims, int kind, vb_ic_params* ic);
int vb_init_prims(vb_handle h, const vb_ic_params* ic, void* stream);

/* Run nsteps iterations of the HARM_HLL time-loop body (src/3dim/algos.jl:274-329):
 * boundary fill, the RK stages, t += dt. */
int vb_step(vb_handle h, double dt, int nsteps, void* stream);
int vb_get_time(vb_handle h, double* t);
int vb_set_time(vb_handle h, double t);

/* Largest characteristic speed |lambda| over interior cells and axes (HARM
 * signal speeds of src/3dim/algos.jl:130-157 on cell-centred states); the
 * CFL dt of an adaptive driver is cfl / sum_d(c / dx_d). Synchronises. */
int vb_max_signal_speed(vb_handle h, double* c, void* stream);

/* Copy the device counters (VB_CNT_*) into out[0..n). Synchronises. */
int vb_get_counters(vb_handle h, uint64_t* out, int n, void* stream);
int vb_reset_counters(vb_handle h, void* stream);

/* Kernel variants (no counterpart in the reference; see verona_b200/autotune.py).
 * split_con2prim: 1 = the 3D stencil kernel writes U and a separate
 * barrier-free kernel solves con2prim; 0 = one fused kernel; -1 = library
 * default. force_box: 1 = use the box-tile stencil kernel for 3D even where
 * the z-marching kernel fits. Results are identical for every variant.
 * learned_fused (guess = VB_GUESS_LEARNED only): 1 = the network's guess and
 * the W Newton from it run in one kernel; 0 = a guess kernel writes one W per
 * cell and the con2prim kernel reads it; -1 = library default (1). Both start
 * the Newton from the same FP32-rounded guess.
 * fp32_pairs (precision = VB_PREC_FP32_BULK, 3D, every reconstruction with HLL or HLLC): 1 =
 * the z-pair stencil kernel (two cells per thread on packed FP32 pairs);
 * 0 = one cell per thread; -1 = library default (1). The two agree to FP32
 * rounding, not bitwise.
 * tma_tiles: 1 = the stencil kernels stage the state in shared memory as TMA
 * tiles (cp.async.bulk.tensor): in 3D (FP32 bulk, z-pair kernel) every plane
 * with its x/y halo, a ring of 6 planes per CTA; in 2D (both precisions) the
 * CTA's tile with its halo on both axes; 0 = staged by per-thread loads (3D:
 * the thread's own column, 4-byte asynchronous copies for the halo);
 * -1 = library default (1). Results are identical.
 * fp64_contract (precision = VB_PREC_FP64): 1 = the stencil and con2prim
 * kernels of the plain FP64 path built with FMA contraction (a * b + c
 * rounded once), fewer FP64 instructions per cell; not bit-identical to the
 * reference's rounding, held to the parity bar of 1e-10 per conserved field
 * instead; 0 = the reference's rounding, bit-identical to its arithmetic
 * (default). */
typedef struct vb_tuning {
    int32_t split_con2prim;
    int32_t force_box;
    int32_t learned_fused;
    int32_t fp32_pairs;
    int32_t tma_tiles;
    int32_t fp64_contract;
    int32_t reserved[2];
} vb_tuning;
int vb_set_tuning(vb_handle h, const vb_tuning* t);
int vb_get_tuning(vb_handle h, vb_tuning* t);
/* *active = 1 if vb_step stages the stencil tiles by TMA on this handle: the
 * tuning allows it (tma_tiles != 0) and both state buffers have a tensor map
 * (3D FP32 bulk, 2D); the z-pair kernel must also be the 3D kernel in use. */
int vb_tma_tiles_active(vb_handle h, int* active);

/* Device bytes held by the handle. */
int vb_memory_bytes(vb_handle h, uint64_t* bytes);

/* Profiling (no counterpart in the reference, which only prints wall-clock
 * rates, src/3dim/algos.jl:335-353). While enabled, every stage-kernel launch
 * is bracketed by CUDA events on the caller's stream and every kernel launch
 * of the library is counted. vb_profile_read synchronises on the last event,
 * returns the summed stage-kernel time (ms) and the launch counts since the
 * previous read, and resets them. */
int vb_profile_enable(vb_handle h, int enable);
int vb_profile_read(vb_handle h, double* stage_ms, int64_t* stage_launches, int64_t* all_launches);
/* The same, with the part of the stage time spent in the stencil kernel:
 * the stencil alone where con2prim runs in a kernel of its own (the learned
 * guess; the split 3D z-marching stages), else the fused stage kernel. */
int vb_profile_read2(vb_handle h, double* stage_ms, double* stencil_ms, int64_t* stage_launches,
                     int64_t* all_launches);

/* ---- point kernels: the FP64 device physics on n independent states ----------
 * Device pointers, struct-of-arrays: component k of point i at [k * n + i].
 * They mirror the reference's scalar functions one to one and serve as the
 * finest-grained parity seam. */
/* reconstruction(::Val{M}, q_im2..q_ip2) -> (qr_i, ql_ip1), src/fluxlimiter.jl:183-200;
 * q: 5 x n, out: 2 x n */
int vb_point_recon(int method, const double* q, double* out, int n, void* stream);
/* face flux of floored left/right primitive states along `axis` (HLL:
 * src/3dim/algos.jl:117-174; HLLC: extension); PL, PR, F: (2+dims) x n */
int vb_point_flux(int dims, int axis, int riemann, double gamma, const double* PL, const double* PR, double* F,
                  int n, void* stream);
/* con2prim per dimension (1D src/1dim/structs.jl:78-105, 2D src/2dim/structs.jl:249-330,
 * 3D src/3dim/structs.jl:218-628); P holds the guess on entry; ret (may be NULL)
 * receives the iteration count (1D/2D) or converged stage (3D), negative on failure */
int vb_point_con2prim(int dims, double gamma, int n_iter, double tol, const double* U, double* P, int* ret, int n,
                      void* stream);

/* ---- learned con2prim guess (extension; the reference warm-starts Newton from
 * the previous primitive state, src/3dim/structs.jl:277-287) ----------------------
 * A 4 -> 64 -> 64 -> 64 -> 1 ReLU MLP in BF16 on the tensor cores (tcgen05, FP32
 * accumulation in TMEM). With E = tau + D = -U2: features f = (log D, |S|/E,
 * log(E/D), Gamma) normalised by norm = {mean[4], 1/std[4]}; output y, the
 * pressure guess as a fraction of E: p0 = E max(y, 0), Newton start
 * W0 = E + p0. Parameters are one FP32 vector of vb_mlp_param_count() values:
 * W1[4][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4 (W[in][out]).
 * All array arguments are device pointers. */
typedef struct vb_mlp* vb_mlp_handle;
int vb_mlp_create(vb_mlp_handle* m);
int vb_mlp_destroy(vb_mlp_handle m);
const char* vb_mlp_last_error(vb_mlp_handle m);
int vb_mlp_param_count(void);
/* host arrays: params[vb_mlp_param_count()], norm[8] */
int vb_mlp_set_params(vb_mlp_handle m, const float* params, const float* norm, void* stream);
int vb_mlp_get_params(vb_mlp_handle m, float* params, float* norm, void* stream);
/* features (n x 4) and, if P != NULL, targets x = p/E (n) and loss weights
 * 1/(1+x)^2 (n; may be NULL) of n conserved states U (5 x n, FP64
 * struct-of-arrays; P likewise): the weighted squared error of y is the
 * squared relative error of the Newton start W0. */
int vb_mlp_features(vb_mlp_handle m, const double* U, const double* P, int n, double gamma, float* feat,
                    float* target, float* weight, void* stream);
/* tensor-core inference: out[n] = y(feat) */
int vb_mlp_forward(vb_mlp_handle m, const float* feat, int n, float* out, void* stream);
/* one optimisation step on n samples (weighted mean squared error on y,
 * weight may be NULL): forward and backward on the tensor cores, then Adam
 * with learning rate lr (lr = 0: gradients only); *loss (may be NULL)
 * receives the batch loss. Synchronises when loss != NULL. */
int vb_mlp_train_step(vb_mlp_handle m, const float* feat, const float* target, const float* weight, int n, float lr,
                      float* loss, void* stream);
/* host copy of the gradient of the last step (same layout as the parameters) */
int vb_mlp_get_grad(vb_mlp_handle m, float* grad, void* stream);
/* use the network as the con2prim guess of a 3D solver (options.guess =
 * VB_GUESS_LEARNED); the network must outlive the solver's use of it */
int vb_attach_mlp(vb_handle h, vb_mlp_handle m);

/* ---- allocation-free CFL reduction ----------------------------------------------
 * No counterpart in the reference. The same maximum signal speed as
 * vb_max_signal_speed, computed from a caller-owned device array in the
 * reference layout (FP64 AoS, 3 ghosts per side) of an nx x ny x nz interior
 * grid, written to the caller-owned device double *c_dev. For callers that
 * cannot have the library allocate device memory (a host whose memory pool
 * already owns the GPU, or code that must not trigger the implicit device
 * synchronisation of cudaMalloc/cudaFree): it calls no allocator; its only
 * scratch is a fixed 64 KiB array inside the library (8192 partial maxima),
 * held on every GPU that loads the library until the process exits. The
 * interior may have at most 8192 x 256 x 128 = 268,435,456 cells; larger
 * grids are rejected with VB_ERR_ARG. The first call on a device looks up the
 * scratch address and the SM count on that device, and again the first call
 * in a new CUDA context of it (after cudaDeviceReset); make those calls before
 * any stream capture. Calls share the scratch, so two calls whose kernels
 * overlap on the GPU race.
 * Errors: vb_noalloc_last_error(). */
int vb_max_signal_speed_noalloc(int dims, int nx, int ny, int nz, double gamma, const double* P_aos_dev,
                                double* c_dev, void* stream);
const char* vb_noalloc_last_error(void);

/* The learned path's refinement on n 3D states: Newton on W from the guesses
 * W0 (n) to |dW| <= rtol W, at most max_newton steps, then a bracketed Newton of
 * at most max_bracket steps; P (5 x n) receives the primitives, iters (may be
 * NULL) the total iterations (negative on failure), fallback (may be NULL) 1
 * where the bracketed phase ran. No counterpart in the reference. */
int vb_point_c2p_w(double gamma, const double* U, const double* W0, double rtol, int max_newton, int max_bracket,
                   double* P, int* iters, int* fallback, int n, void* stream);
/* The same refinement with the precision gate of the FP32-bulk learned path
 * (options.c2p_fp32): from the FP32 guesses W0 (n), an FP32 Newton on the
 * pressure where the guess has Lorentz factor below sqrt 2 and kinetic energy
 * below 10 x the guessed pressure (converged to |dp| <= 4e-7 p), else the FP64
 * W Newton of vb_point_c2p_w; fp64 (may be NULL) receives 1 where the FP64
 * Newton ran. No counterpart in the reference. */
int vb_point_c2p_gated(double gamma, const double* U, const float* W0, double rtol, int max_newton, int max_bracket,
                       double* P, int* iters, int* fp64, int n, void* stream);

/* ---- grid kernels one at a time (the reference's kernels as separate calls) ------
 * Caller-owned device arrays in the reference layout: FP64 AoS (2 + dims,
 * nx+6 [, ny+6 [, nz+6]]), variable fastest. For a caller that replaces single
 * kernels of HARM_HLL; the fused time loop is vb_step. FP64, bit-identical to
 * the reference's arithmetic. Errors: vb_grid_last_error().
 *   fluxes:   function_Fluxes of one axis (src/3dim/algos.jl:14-176,
 *             src/2dim/algos.jl:11-168): face i+1/2 into F[:, i] for every index
 *             in [2, n+2] (0-based, padded) on all active axes; face states are
 *             reconstructed with `recon`, floored at floor_, then the Riemann flux
 *   update:   function_Update (src/3dim/algos.jl:178-200): interior cells,
 *             Uout = U - dt/dx (Fx_i - Fx_{i-1}) - dt/dy (...) - dt/dz (...)
 *   con2prim: function_UtoP (src/3dim/structs.jl:218-628, src/2dim/structs.jl:249-330,
 *             src/1dim/structs.jl:78-105) on interior cells, P in: guess, out:
 *             primitives (NaN where no root); failures_dev (may be NULL) counts the
 *             cells where every stage gave up (a 3D stage that converges to a
 *             non-finite state also leaves NaN, as in the reference)
 *   prim2con: kernel_PtoU (src/3dim/structs.jl:66-81) on all cells
 *   limit:    function_Limit (src/3dim/algos.jl:5-12) on all cells */
int vb_grid_fluxes(int dims, int nx, int ny, int nz, const double* P_aos, double gamma, double floor_, int axis,
                   int recon, int riemann, double* F_aos, void* stream);
int vb_grid_update(int dims, int nx, int ny, int nz, const double* U_aos, const double* Fx, const double* Fy,
                   const double* Fz, double dt, double dx, double dy, double dz, double* Uout_aos, void* stream);
int vb_grid_con2prim(int dims, int nx, int ny, int nz, const double* U_aos, double gamma, int n_iter, double tol,
                     double* P_aos, uint64_t* failures_dev, void* stream);
int vb_grid_prim2con(int dims, int nx, int ny, int nz, const double* P_aos, double gamma, double* U_aos,
                     void* stream);
int vb_grid_limit(int dims, int nx, int ny, int nz, double* P_aos, double floor_, void* stream);
const char* vb_grid_last_error(void);

/* ---- batch of independent problems (extension; the reference advances one
 * grid per HARM_HLL call, src/1dim/algos.jl:58-68, src/2dim/algos.jl:192-208) --
 * Many 1D and 2D problems of uneven size advance together. Each has its own
 * interior size, reconstruction, cell widths and time step; all share gamma
 * and the options' riemann, rk, precision (FP64 or FP32 bulk), n_iter, tol
 * and floor_ (guess must be VB_GUESS_PREVIOUS); every face is outflow unless
 * vb_batch_set_boundary gives it another kind.
 * Each problem evolves exactly as a single-grid handle of the same dims and
 * options with 3 ghost cells would. vb_batch_step runs nsteps steps of every
 * problem as ONE persistent kernel launch, replayed from a CUDA graph: tiles
 * (TX2 x TY2 cells in 2D, pencils of L1 cells in 1D) of every RK stage of
 * every problem are taken in order by the CTAs of one grid, and a tile waits
 * (bounded) for the previous stage of its own problem only. Tile variants and
 * CTAs per SM are set by vb_batch_set_tuning (chosen by the Python autotuner,
 * verona_b200/autotune.py). Arrays are device pointers; the current device is
 * the handle's. */
typedef struct {
    int dims;      /* 1 or 2 */
    int nx, ny;    /* interior cells (ny = 1 when dims = 1) */
    int recon;     /* VB_RECON_* */
    double dx, dy; /* cell widths (dy unused when dims = 1) */
    double dt;     /* time step */
} vb_batch_problem;
typedef struct vb_batch* vb_batch_handle;
int vb_batch_create(vb_batch_handle* b, int nprob, const vb_batch_problem* probs, double gamma,
                    const vb_options* o);
int vb_batch_destroy(vb_batch_handle b);
const char* vb_batch_last_error(vb_batch_handle b); /* NULL handle: the last failed create */
/* Boundary of face `face` (VB_FACE_XLO .. VB_FACE_YHI; x faces only in 1D) of
 * problem i, with the kinds and parameters of vb_set_boundary: OUTFLOW (the
 * default on every face), FIXED (the loaded ghosts, with an optional decay
 * {var, t_on, t_off, factor} by the problem's own time) or NOZZLE {radius, c1,
 * c2, rho, u, u1[, u2]} -- so jets run in a batch, as Verona2D.HARM_HLL with
 * the examples' boundary callback (examples/Jet2D/HARM_jet_breakout.jl:84-99)
 * would run them one at a time. Synchronises the device. */
int vb_batch_set_boundary(vb_batch_handle b, int i, int face, int kind, const double* params, int nparams);
/* problem i's primitives, FP64 AoS (2 + dims, nx + 6 [, ny + 6]) as vb_load_prims */
int vb_batch_load_prims(vb_batch_handle b, int i, const double* P_aos, void* stream);
int vb_batch_store_prims(vb_batch_handle b, int i, double* P_aos, void* stream);
int vb_batch_step(vb_batch_handle b, int nsteps, void* stream);
int vb_batch_get_time(vb_batch_handle b, int i, double* t);
int vb_batch_get_counters(vb_batch_handle b, uint64_t* out /* VB_CNT_N */, void* stream); /* synchronises */
/* Synchronises `stream` and reports the outcome of the steps before it:
 * VB_ERR_TIMEOUT if a tile's bounded wait for the previous stage of its
 * problem gave up (VB_CNT_TIMEOUT > 0; the batch state is then undefined:
 * vb_batch_rollback or reload it), VB_ERR_STATE if work items were skipped as
 * out of range, else VB_OK. The counters accumulate until
 * vb_batch_reset_counters. No counterpart in the reference (its kernels have
 * no waits). */
int vb_batch_check(vb_batch_handle b, void* stream);
/* Bound of a tile's wait for the previous stage of its problem, in polls of
 * about 128 ns; 0 restores the default (2^24, a few seconds). Every wait ends
 * by construction (the tiles waited for are held by running CTAs); a smaller
 * bound only makes a stalled launch end sooner. */
int vb_batch_set_wait_limit(vb_batch_handle b, uint32_t max_polls);
int vb_batch_reset_counters(vb_batch_handle b, void* stream);
/* tile variants of a precision (0 for an invalid precision) and their shapes */
int vb_batch_num_variants(int precision);
int vb_batch_variant_shape(int precision, int variant, int* tile_x2, int* tile_y2, int* pencil1);
/* ctas_per_sm 0: as many as fit; the grid of the last launch is returned by get */
int vb_batch_set_tuning(vb_batch_handle b, int variant, int ctas_per_sm);
int vb_batch_get_tuning(vb_batch_handle b, int* variant, int* ctas_per_sm, int* grid);
int vb_batch_info(vb_batch_handle b, int64_t* interior_cells, int64_t* tiles_per_stage, int64_t* device_bytes);
/* copy of the state (P, U^n, times) and its restoration, e.g. around tuning runs */
int vb_batch_checkpoint(vb_batch_handle b, void* stream);
int vb_batch_rollback(vb_batch_handle b, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* VERONA_B200_H */
