// Grid-level entry points that mirror the reference's kernels one at a time,
// on caller-owned device arrays in the reference layout (FP64 AoS, variable
// fastest, padded extents n+6 on the active axes). They are the fine-grained
// seam for a caller that replaces single kernels of HARM_HLL; the time loop
// itself is the fused vb_step. FP64, built with -fmad=false: bit-identical to
// the oracle's k_fluxes / k_update / k_utop / k_ptou / k_limit.
//   vb_grid_fluxes     function_Fluxes of one axis, src/3dim/algos.jl:14-176
//                      (2D: src/2dim/algos.jl:11-168)
//   vb_grid_update     function_Update, src/3dim/algos.jl:178-200
//   vb_grid_con2prim   function_UtoP, src/3dim/structs.jl:218-628
//                      (2D: src/2dim/structs.jl:249-330; 1D: src/1dim/structs.jl:78-105)
//   vb_grid_prim2con   kernel_PtoU, src/3dim/structs.jl:66-81
//   vb_grid_limit      function_Limit, src/3dim/algos.jl:5-12
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/verona_b200.h"
#include "vb_con2prim.cuh"
#include "vb_internal.h"

namespace vb {

struct GridAoS {
    int dims, nv;
    int np[3];  // padded extents (1 on inactive axes)
    long long st[3];
    long long ncell;
};

static inline bool grid_aos(int dims, int nx, int ny, int nz, GridAoS& g) {
    if (dims < 1 || dims > 3 || nx < 1 || (dims > 1 && ny < 1) || (dims > 2 && nz < 1)) return false;
    g.dims = dims;
    g.nv = 2 + dims;
    const int n[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a) g.np[a] = a < dims ? n[a] + 2 * NG : 1;
    g.st[0] = 1;
    g.st[1] = g.np[0];
    g.st[2] = (long long)g.np[0] * g.np[1];
    g.ncell = (long long)g.np[0] * g.np[1] * g.np[2];
    return true;
}

__device__ __forceinline__ void cell_ijk(const GridAoS& g, long long c, int& i, int& j, int& k) {
    i = (int)(c % g.np[0]);
    j = (int)((c / g.np[0]) % g.np[1]);
    k = (int)(c / g.st[2]);
}

// true if (i, j, k) lies in [lo, np - hi) on every active axis
__device__ __forceinline__ bool in_range(const GridAoS& g, int i, int j, int k, int lo, int hi) {
    const int x[3] = {i, j, k};
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        if (a < g.dims) ok = ok && x[a] >= lo && x[a] < g.np[a] - hi;
    return ok;
}

template <int DIM, int REC, int RS>
__global__ void k_grid_fluxes(GridAoS g, const double* __restrict__ P, double gamma, double fl, int d,
                              double* __restrict__ F) {
    constexpr int NV = 2 + DIM;
    const long long sd = d == 0 ? g.st[0] : (d == 1 ? g.st[1] : g.st[2]);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(g, c, i, j, k);
        // faces i + 1/2 for every index in [2, n - 4] on all active axes
        if (!in_range(g, i, j, k, 2, 3)) continue;
        double PL[NV], PR[NV], Fo[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double* q = P + v;
            double qr, ql;
            recon<REC>(q[NV * (c - 2 * sd)], q[NV * (c - sd)], q[NV * c], q[NV * (c + sd)], q[NV * (c + 2 * sd)], qr,
                       ql);
            PL[v] = ql;
            recon<REC>(q[NV * (c - sd)], q[NV * c], q[NV * (c + sd)], q[NV * (c + 2 * sd)], q[NV * (c + 3 * sd)], qr,
                       ql);
            PR[v] = qr;
        }
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            PL[v] = jmax(fl, PL[v]);
            PR[v] = jmax(fl, PR[v]);
        }
        face_flux<DIM, RS>(d, gamma, PL, PR, Fo);
#pragma unroll
        for (int v = 0; v < NV; ++v) F[NV * c + v] = Fo[v];
    }
}

template <int DIM>
__global__ void k_grid_update(GridAoS g, const double* __restrict__ U, const double* __restrict__ Fx,
                              const double* __restrict__ Fy, const double* __restrict__ Fz, double dt, double dx,
                              double dy, double dz, double* __restrict__ Uo) {
    constexpr int NV = 2 + DIM;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(g, c, i, j, k);
        if (!in_range(g, i, j, k, 3, 3)) continue;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double r = U[NV * c + v];
            r = r - dt / dx * (Fx[NV * c + v] - Fx[NV * (c - g.st[0]) + v]);
            if (DIM > 1) r = r - dt / dy * (Fy[NV * c + v] - Fy[NV * (c - g.st[1]) + v]);
            if (DIM > 2) r = r - dt / dz * (Fz[NV * c + v] - Fz[NV * (c - g.st[2]) + v]);
            Uo[NV * c + v] = r;
        }
    }
}

template <int DIM>
__global__ void k_grid_con2prim(GridAoS g, const double* __restrict__ U, double gamma, int n_iter, double tol,
                                double* __restrict__ P, unsigned long long* failures) {
    constexpr int NV = 2 + DIM;
    unsigned long long nf = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(g, c, i, j, k);
        if (!in_range(g, i, j, k, 3, 3)) continue;
        double u[NV], p[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            u[v] = U[NV * c + v];
            p[v] = P[NV * c + v];
        }
        int r;
        if (DIM == 1)
            r = c2p_1d(gamma, n_iter, tol, u, p);
        else if (DIM == 2)
            r = c2p_2d(gamma, n_iter, tol, u, p);
        else
            r = c2p_3d(gamma, n_iter, tol, u, p);
        nf += (r < 0);
#pragma unroll
        for (int v = 0; v < NV; ++v) P[NV * c + v] = p[v];
    }
    if (failures && nf) atomicAdd(failures, nf);
}

template <int DIM>
__global__ void k_grid_prim2con(GridAoS g, const double* __restrict__ P, double gamma, double* __restrict__ U) {
    constexpr int NV = 2 + DIM;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        double p[NV], u[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) p[v] = P[NV * c + v];
        prim2con<DIM>(gamma, p, u);
#pragma unroll
        for (int v = 0; v < NV; ++v) U[NV * c + v] = u[v];
    }
}

__global__ void k_grid_limit(GridAoS g, double* __restrict__ P, double fl) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        P[g.nv * c + 0] = jmax(P[g.nv * c + 0], fl);
        P[g.nv * c + 1] = jmax(P[g.nv * c + 1], fl);
    }
}

static int blocks_for(long long n) {
    long long b = (n + 255) / 256;
    return (int)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

}  // namespace vb

using namespace vb;

static thread_local std::string g_grid_err;

static int gfail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_grid_err = buf;
    return code;
}

static int gdone(const char* what) {
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VB_OK : gfail(VB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

template <int DIM>
static void launch_fluxes(const GridAoS& g, int rec, int rs, const double* P, double gamma, double fl, int axis,
                          double* F, cudaStream_t s) {
    const int nb = blocks_for(g.ncell);
#define VB_GF(RC, RSC)                                                                        \
    if (rec == RC && rs == RSC) {                                                             \
        k_grid_fluxes<DIM, RC, RSC><<<nb, 256, 0, s>>>(g, P, gamma, fl, axis, F);             \
        return;                                                                               \
    }
    VB_GF(REC_MINMOD, RS_HLL)
    VB_GF(REC_MINMOD, RS_HLLC)
    VB_GF(REC_PPM, RS_HLL)
    VB_GF(REC_PPM, RS_HLLC)
    VB_GF(REC_WENOZ, RS_HLL)
    VB_GF(REC_WENOZ, RS_HLLC)
#undef VB_GF
}

extern "C" {

const char* vb_grid_last_error(void) { return g_grid_err.c_str(); }

int vb_grid_fluxes(int dims, int nx, int ny, int nz, const double* P_aos, double gamma, double floor_, int axis,
                   int recon, int riemann, double* F_aos, void* stream) {
    GridAoS g;
    if (!grid_aos(dims, nx, ny, nz, g)) return gfail(VB_ERR_ARG, "vb_grid_fluxes: dims %d size %d %d %d", dims, nx, ny, nz);
    if (!P_aos || !F_aos) return gfail(VB_ERR_ARG, "vb_grid_fluxes: null array");
    if (axis < 0 || axis >= dims) return gfail(VB_ERR_ARG, "vb_grid_fluxes: axis %d of a %dD grid", axis, dims);
    if (recon < VB_RECON_MINMOD || recon > VB_RECON_WENOZ || (riemann != VB_RIEMANN_HLL && riemann != VB_RIEMANN_HLLC))
        return gfail(VB_ERR_ARG, "vb_grid_fluxes: recon %d riemann %d", recon, riemann);
    cudaStream_t s = (cudaStream_t)stream;
    if (dims == 1) launch_fluxes<1>(g, recon, riemann, P_aos, gamma, floor_, axis, F_aos, s);
    else if (dims == 2) launch_fluxes<2>(g, recon, riemann, P_aos, gamma, floor_, axis, F_aos, s);
    else launch_fluxes<3>(g, recon, riemann, P_aos, gamma, floor_, axis, F_aos, s);
    return gdone("vb_grid_fluxes");
}

int vb_grid_update(int dims, int nx, int ny, int nz, const double* U_aos, const double* Fx, const double* Fy,
                   const double* Fz, double dt, double dx, double dy, double dz, double* Uout_aos, void* stream) {
    GridAoS g;
    if (!grid_aos(dims, nx, ny, nz, g)) return gfail(VB_ERR_ARG, "vb_grid_update: dims %d size %d %d %d", dims, nx, ny, nz);
    if (!U_aos || !Uout_aos || !Fx || (dims > 1 && !Fy) || (dims > 2 && !Fz))
        return gfail(VB_ERR_ARG, "vb_grid_update: null array");
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = blocks_for(g.ncell);
    if (dims == 1) k_grid_update<1><<<nb, 256, 0, s>>>(g, U_aos, Fx, Fy, Fz, dt, dx, dy, dz, Uout_aos);
    else if (dims == 2) k_grid_update<2><<<nb, 256, 0, s>>>(g, U_aos, Fx, Fy, Fz, dt, dx, dy, dz, Uout_aos);
    else k_grid_update<3><<<nb, 256, 0, s>>>(g, U_aos, Fx, Fy, Fz, dt, dx, dy, dz, Uout_aos);
    return gdone("vb_grid_update");
}

int vb_grid_con2prim(int dims, int nx, int ny, int nz, const double* U_aos, double gamma, int n_iter, double tol,
                     double* P_aos, uint64_t* failures_dev, void* stream) {
    GridAoS g;
    if (!grid_aos(dims, nx, ny, nz, g)) return gfail(VB_ERR_ARG, "vb_grid_con2prim: dims %d size %d %d %d", dims, nx, ny, nz);
    if (!U_aos || !P_aos || n_iter < 1) return gfail(VB_ERR_ARG, "vb_grid_con2prim: null array or n_iter %d", n_iter);
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = blocks_for(g.ncell);
    unsigned long long* f = reinterpret_cast<unsigned long long*>(failures_dev);
    if (dims == 1) k_grid_con2prim<1><<<nb, 256, 0, s>>>(g, U_aos, gamma, n_iter, tol, P_aos, f);
    else if (dims == 2) k_grid_con2prim<2><<<nb, 256, 0, s>>>(g, U_aos, gamma, n_iter, tol, P_aos, f);
    else k_grid_con2prim<3><<<nb, 256, 0, s>>>(g, U_aos, gamma, n_iter, tol, P_aos, f);
    return gdone("vb_grid_con2prim");
}

int vb_grid_prim2con(int dims, int nx, int ny, int nz, const double* P_aos, double gamma, double* U_aos,
                     void* stream) {
    GridAoS g;
    if (!grid_aos(dims, nx, ny, nz, g)) return gfail(VB_ERR_ARG, "vb_grid_prim2con: dims %d size %d %d %d", dims, nx, ny, nz);
    if (!P_aos || !U_aos) return gfail(VB_ERR_ARG, "vb_grid_prim2con: null array");
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = blocks_for(g.ncell);
    if (dims == 1) k_grid_prim2con<1><<<nb, 256, 0, s>>>(g, P_aos, gamma, U_aos);
    else if (dims == 2) k_grid_prim2con<2><<<nb, 256, 0, s>>>(g, P_aos, gamma, U_aos);
    else k_grid_prim2con<3><<<nb, 256, 0, s>>>(g, P_aos, gamma, U_aos);
    return gdone("vb_grid_prim2con");
}

int vb_grid_limit(int dims, int nx, int ny, int nz, double* P_aos, double floor_, void* stream) {
    GridAoS g;
    if (!grid_aos(dims, nx, ny, nz, g)) return gfail(VB_ERR_ARG, "vb_grid_limit: dims %d size %d %d %d", dims, nx, ny, nz);
    if (!P_aos) return gfail(VB_ERR_ARG, "vb_grid_limit: null array");
    k_grid_limit<<<blocks_for(g.ncell), 256, 0, (cudaStream_t)stream>>>(g, P_aos, floor_);
    return gdone("vb_grid_limit");
}

}  // extern "C"
