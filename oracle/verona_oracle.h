/*
 * verona_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of Wesenheit/Verona's SRHD update (Julia), used as the
 * parity oracle for the CUDA path and as the timed CPU baseline. Nothing in the
 * product library links or calls this code; only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference arm do, and only to check or time against.
 *
 * Parity status: the reference (pure Julia + CUDA.jl) cannot run in this
 * environment, and it ships no tests or golden vectors, so the restatement
 * against the reference itself is "parity unpinned". It is pinned instead by
 * published known answers (Marti & Mueller 1994 problem 1 via an exact Riemann
 * solver), self-convergence, and conservation / symmetry / round-trip
 * properties (see tests/test_oracle_*.py).
 *
 * Layout: the reference's own column-major AoS layout, arr[var, i, j, k] with
 * the variable index fastest and 3 ghost cells per side (src/3dim/structs.jl:35).
 * All indices in this API are 0-based; comments cite the 1-based Julia lines.
 */
#ifndef VERONA_ORACLE_H
#define VERONA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_MINMOD = 0, OR_PPM = 1, OR_WENOZ = 2 };
enum { OR_HLL = 0, OR_HLLC = 1 };
enum { OR_BC_OUTFLOW = 0, OR_BC_FIXED = 1, OR_BC_NOZZLE = 2 };

/* point physics, exposed for unit tests ------------------------------------ */
void or_recon(int method, const double q[5], double out[2]);        /* (qr_i, ql_ip1) */
double or_sound_speed(double rho, double u, double gamma);
/* one face flux along axis d for ND states (nv = 2 + dims vars). PL/PR are
 * primitive states after the face floor; F receives the flux. */
void or_face_flux(int dims, int axis, int riemann, double gamma,
                  const double* PL, const double* PR, double* F);
void or_prim2con(int dims, double gamma, const double* P, double* U);
/* con2prim on one cell; returns the cascade stage that converged (3D) or the
 * Newton iteration count, negative on failure. P is the guess on entry. */
int or_con2prim(int dims, double gamma, int n_iter, double tol, const double* U, double* P);
/* row swaps of the 2D con2prim's pivoted LU (LU_dec_pivot!) made on the calling
 * thread since the previous call; the count is reset */
long long or_lu4_swaps_take(void);

/* 1D reference solver (src/1dim/algos.jl:58-315): N cells, no ghosts ---- */
typedef struct or1d or1d_t;
or1d_t* or1d_create(int N, const double* rho, const double* u, const double* ux,
                    double gamma, int rec, int n_iter, double tol);
void or1d_step(or1d_t* s, double dt, double dx, int nsteps);
void or1d_get(const or1d_t* s, double* rho, double* u, double* ux);
void or1d_get_cons(const or1d_t* s, double* U1, double* U2, double* U3);
void or1d_destroy(or1d_t* s);

/* ND solver, dims 1..3 with 3 ghost cells (src/2dim/algos.jl:192-324,
 * src/3dim/algos.jl:203-362 and extensions) --------------------------------- */
typedef struct ornd ornd_t;
/* n = interior sizes; P_aos = padded AoS primitives (nv, n0+6, n1+6, n2+6) */
ornd_t* ornd_create(int dims, const int n[3], const double* P_aos, double gamma,
                    double floor_, int n_iter, double tol, int recon, int riemann, int rk);
void ornd_set_grid(ornd_t* s, double dx, double dy, double dz);
/* face = 2*axis + side; kind OR_BC_*; params: FIXED {var, t_on, t_off, factor};
 * NOZZLE {radius, c1, c2, rho, u, u1, u2, u3} (radius/centers in cells) */
void ornd_set_boundary(ornd_t* s, int face, int kind, const double* params, int np);
void ornd_step(ornd_t* s, double dt, int nsteps);
void ornd_get_prims(const ornd_t* s, double* P_aos);
void ornd_get_cons(const ornd_t* s, double* U_aos);
double ornd_time(const ornd_t* s);
int64_t ornd_c2p_failures(const ornd_t* s);
void ornd_destroy(ornd_t* s);

/* single-kernel entry points on caller-owned AoS arrays, mirroring the
 * reference kernels one to one (for kernel-level parity tests) ----------- */
void ornd_k_fluxes(int dims, const int npad[3], const double* P, double gamma, double floor_,
                   double* F, int axis, int recon, int riemann);
void ornd_k_update(int dims, const int npad[3], const double* U, double* Ub, double dt,
                   const double dxs[3], const double* Fx, const double* Fy, const double* Fz);
void ornd_k_utop(int dims, const int npad[3], const double* U, double* P, double gamma,
                 int n_iter, double tol);
void ornd_k_ptou(int dims, const int npad[3], const double* P, double* U, double gamma);
void ornd_k_limit(int dims, const int npad[3], double* P, double floor_);

int or_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
