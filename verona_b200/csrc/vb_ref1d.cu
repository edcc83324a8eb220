// The reference's 1D solver, Verona1D.HARM_HLL (src/1dim/algos.jl:58-315),
// FP64, as one persistent CTA that runs every step of a call: each phase of
// the Julia loop becomes a block-wide pass over the N cells separated by
// __syncthreads(), so a whole shock-tube run is a single launch.
//
// The reference keeps state between stages that this kernel keeps too: the
// face arrays PL/PR start as copies of P and are only refreshed on the ranges
// the Julia loops write (src/1dim/algos.jl:91-117), so the edge faces keep
// their t = 0 values; cells 1, N-1, N (1-based) of U are never updated.
// Compiled with -fmad=false: bit-identical to the oracle restatement.
#include "vb_con2prim.cuh"
#include "vb_internal.h"

namespace vb {

constexpr int R1_THREADS = 1024;

__device__ __forceinline__ void ref1d_cons(double g, double p1, double p2, double p3, double* U) {
    double gamma = sqrt(sq(p3) + 1.0);
    double pressure = (g - 1.0) * p2;
    U[0] = p1 * gamma;
    U[1] = -(p2 + pressure + p1) * sq(gamma) + pressure;
    U[2] = (p2 + pressure + p1) * gamma * p3;
}

__device__ __forceinline__ void ref1d_flux(double g, double p1, double p2, double p3, double* F) {
    double gamma = sqrt(sq(p3) + 1.0);
    double pressure = (g - 1.0) * p2;
    F[0] = p1 * p3;
    F[1] = -(p2 + pressure + p1) * gamma * p3;
    F[2] = pressure + (p2 + pressure + p1) * sq(p3);
}

// reconstruction into PR/PL, HLL fluxes F, update Uout = Ubase - coef dF
__device__ void ref1d_stage(const Ref1DState& st, const double* P, const double* Ub, double* Uo, double coef,
                            double g, int rec) {
    const int N = st.N;
    const int tid = threadIdx.x;
    // src/1dim/algos.jl:91-117
    if (rec == REC_MINMOD) {
        for (int i = 1 + tid; i <= N - 2; i += blockDim.x)
            for (int v = 0; v < 3; ++v) {
                const double* q = P + v * N;
                minmod(q[i - 1], q[i], q[i + 1], st.PR[v * N + i - 1], st.PL[v * N + i]);
            }
    } else {
        for (int i = 2 + tid; i <= N - 3; i += blockDim.x)
            for (int v = 0; v < 3; ++v) {
                const double* q = P + v * N;
                if (rec == REC_PPM)
                    ppm(q[i - 2], q[i - 1], q[i], q[i + 1], q[i + 2], st.PR[v * N + i - 1], st.PL[v * N + i]);
                else
                    wenoz(q[i - 2], q[i - 1], q[i], q[i + 1], q[i + 2], st.PR[v * N + i - 1], st.PL[v * N + i]);
            }
    }
    __syncthreads();
    // PtoU/PtoF of both face arrays and the HLL loop over all faces (:233-282)
    for (int i = tid; i < N; i += blockDim.x) {
        double pl1 = st.PL[i], pl2 = st.PL[N + i], pl3 = st.PL[2 * N + i];
        double pr1 = st.PR[i], pr2 = st.PR[N + i], pr3 = st.PR[2 * N + i];
        double UL[3], UR[3], FL[3], FR[3];
        ref1d_cons(g, pr1, pr2, pr3, UR);
        ref1d_flux(g, pr1, pr2, pr3, FR);
        ref1d_cons(g, pl1, pl2, pl3, UL);
        ref1d_flux(g, pl1, pl2, pl3, FL);
        double vL = pl3 / sqrt(sq(pl3) + 1.0);
        double vR = pr3 / sqrt(sq(pr3) + 1.0);
        double CL = sound_speed(pl1, pl2, g);
        double CR = sound_speed(pr1, pr2, g);
        double sL = sq(CL) / ((sq(pl3) + 1.0) * (1.0 - sq(CL)));
        double sR = sq(CR) / ((sq(pr3) + 1.0) * (1.0 - sq(CR)));
        double Cmax = jmax((vL + sqrt(sL * (1.0 - sq(vL) + sL))) / (1.0 + sL),
                           (vR + sqrt(sR * (1.0 - sq(vR) + sR))) / (1.0 + sR));
        double Cmin = -jmin((vL - sqrt(sL * (1.0 - sq(vL) + sL))) / (1.0 + sL),
                            (vR - sqrt(sR * (1.0 - sq(vR) + sR))) / (1.0 + sR));
        for (int v = 0; v < 3; ++v) {
            double f;
            if (Cmax < 0)
                f = FR[v];
            else if (Cmin < 0)
                f = FL[v];
            else
                f = (FR[v] * Cmin + FL[v] * Cmax - Cmax * Cmin * (UR[v] - UL[v])) / (Cmax + Cmin);
            st.F[v * N + i] = f;
        }
    }
    __syncthreads();
    // i = 2:(N-2) (:284-288, :409-413)
    for (int i = 1 + tid; i <= N - 3; i += blockDim.x)
        for (int v = 0; v < 3; ++v) Uo[v * N + i] = Ub[v * N + i] - coef * (st.F[v * N + i] - st.F[v * N + i - 1]);
    __syncthreads();
}

__device__ void ref1d_utop(const Ref1DState& st, const double* U, double* P, double g, int n_iter, double tol) {
    const int N = st.N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double u[3] = {U[i], U[N + i], U[2 * N + i]};
        double p[3] = {P[i], P[N + i], P[2 * N + i]};
        c2p_1d(g, n_iter, tol, u, p);
        P[i] = p[0];
        P[N + i] = p[1];
        P[2 * N + i] = p[2];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(R1_THREADS) k_ref1d_steps(Ref1DState st, double g, int rec, int n_iter,
                                                            double tol, double dt, double dx, int nsteps) {
    const int N = st.N;
    const double c1 = 0.5 * dt / dx, c2 = dt / dx;
    for (int n = 0; n < nsteps; ++n) {
        ref1d_stage(st, st.P, st.U, st.Uh, c1, g, rec);
        for (int i = threadIdx.x; i < 3 * N; i += blockDim.x) st.Ph[i] = st.P[i];  // Phalf = deepcopy(P)
        __syncthreads();
        ref1d_utop(st, st.Uh, st.Ph, g, n_iter, tol);
        ref1d_stage(st, st.Ph, st.U, st.U, c2, g, rec);
        ref1d_utop(st, st.U, st.P, g, n_iter, tol);
    }
}

__global__ void k_ref1d_init(Ref1DState st, const double* __restrict__ Pa, double g) {
    const int N = st.N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        double p[3] = {Pa[3 * i], Pa[3 * i + 1], Pa[3 * i + 2]};
        double U[3];
        ref1d_cons(g, p[0], p[1], p[2], U);  // PtoU, src/1dim/structs.jl:58-66
        for (int v = 0; v < 3; ++v) {
            st.P[v * N + i] = p[v];
            st.Ph[v * N + i] = p[v];
            st.PL[v * N + i] = p[v];
            st.PR[v * N + i] = p[v];
            st.U[v * N + i] = U[v];
            st.Uh[v * N + i] = U[v];
            st.F[v * N + i] = 0.0;
        }
    }
}

__global__ void k_ref1d_store(Ref1DState st, double* __restrict__ Pa) {
    const int N = st.N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        for (int v = 0; v < 3; ++v) Pa[3 * i + v] = st.P[v * N + i];
}

cudaError_t launch_ref1d_init(const Ref1DState& st, const double* Pa, double g, cudaStream_t s) {
    k_ref1d_init<<<(st.N + 255) / 256, 256, 0, s>>>(st, Pa, g);
    return cudaGetLastError();
}

cudaError_t launch_ref1d_steps(const Ref1DState& st, double g, int rec, int n_iter, double tol, double dt,
                               double dx, int nsteps, cudaStream_t s) {
    if (nsteps <= 0) return cudaSuccess;
    k_ref1d_steps<<<1, R1_THREADS, 0, s>>>(st, g, rec, n_iter, tol, dt, dx, nsteps);
    return cudaGetLastError();
}

cudaError_t launch_ref1d_store(const Ref1DState& st, double* Pa, cudaStream_t s) {
    k_ref1d_store<<<(st.N + 255) / 256, 256, 0, s>>>(st, Pa);
    return cudaGetLastError();
}

}  // namespace vb
