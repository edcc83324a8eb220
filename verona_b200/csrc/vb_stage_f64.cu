// Plain FP64 instantiation of the stage and per-step kernels. Built with
// -fmad=false so every operation rounds as the reference's Julia code does.
#include "vb_stage.cuh"
#include "vb_stage_zm.cuh"

namespace vb {
VB_INSTANTIATE_LAUNCHERS(double)
// tensor map of an FP64 state array: the box tile of k_stage in 2D
template <> bool encode_stage_tmap<double>(void* out, const double* P, const Grid& g) {
    return g.dims == 2 && encode_tile2_tmap<double, TileCfg<2>::TX, TileCfg<2>::TY>(out, P, g);
}
template cudaError_t launch_c2p<double>(const StageParams&, const StageBufs<double>&, cudaStream_t);

// ---- point kernels: the device physics on arrays of independent states
// (struct-of-arrays, component k of point i at [k * n + i]) -----------------
__global__ void k_point_recon(int method, const double* __restrict__ q, double* __restrict__ out, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double a[5];
        for (int k = 0; k < 5; ++k) a[k] = q[k * n + i];
        double qr = 0, ql = 0;
        if (method == REC_MINMOD) recon<REC_MINMOD>(a[0], a[1], a[2], a[3], a[4], qr, ql);
        else if (method == REC_PPM) recon<REC_PPM>(a[0], a[1], a[2], a[3], a[4], qr, ql);
        else recon<REC_WENOZ>(a[0], a[1], a[2], a[3], a[4], qr, ql);
        out[i] = qr;
        out[n + i] = ql;
    }
}

template <int DIM>
__global__ void k_point_flux(int axis, int rs, double g, const double* __restrict__ PL,
                             const double* __restrict__ PR, double* __restrict__ F, int n) {
    constexpr int NV = 2 + DIM;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double l[NV], r[NV], f[NV];
        for (int v = 0; v < NV; ++v) {
            l[v] = PL[v * n + i];
            r[v] = PR[v * n + i];
        }
        if (rs == RS_HLLC) face_flux<DIM, RS_HLLC>(axis, g, l, r, f);
        else face_flux<DIM, RS_HLL>(axis, g, l, r, f);
        for (int v = 0; v < NV; ++v) F[v * n + i] = f[v];
    }
}

template <int DIM>
__global__ void k_point_con2prim(double g, int n_iter, double tol, const double* __restrict__ U,
                                 double* __restrict__ P, int* __restrict__ ret, int n) {
    constexpr int NV = 2 + DIM;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double u[NV], p[NV];
        for (int v = 0; v < NV; ++v) {
            u[v] = U[v * n + i];
            p[v] = P[v * n + i];
        }
        int r = DIM == 1 ? c2p_1d(g, n_iter, tol, u, p) : DIM == 2 ? c2p_2d(g, n_iter, tol, u, p) : c2p_3d(g, n_iter, tol, u, p);
        for (int v = 0; v < NV; ++v) P[v * n + i] = p[v];
        if (ret) ret[i] = r;
    }
}

cudaError_t launch_point_recon(int method, const double* q, double* out, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_point_recon<<<grid_for(n, 256), 256, 0, s>>>(method, q, out, n);
    return cudaGetLastError();
}

cudaError_t launch_point_flux(int dims, int axis, int rs, double g, const double* PL, const double* PR, double* F,
                              int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    int nb = grid_for(n, 128);
    if (dims == 1) k_point_flux<1><<<nb, 128, 0, s>>>(axis, rs, g, PL, PR, F, n);
    else if (dims == 2) k_point_flux<2><<<nb, 128, 0, s>>>(axis, rs, g, PL, PR, F, n);
    else k_point_flux<3><<<nb, 128, 0, s>>>(axis, rs, g, PL, PR, F, n);
    return cudaGetLastError();
}

cudaError_t launch_point_con2prim(int dims, double g, int n_iter, double tol, const double* U, double* P, int* ret,
                                  int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    int nb = grid_for(n, 128);
    if (dims == 1) k_point_con2prim<1><<<nb, 128, 0, s>>>(g, n_iter, tol, U, P, ret, n);
    else if (dims == 2) k_point_con2prim<2><<<nb, 128, 0, s>>>(g, n_iter, tol, U, P, ret, n);
    else k_point_con2prim<3><<<nb, 128, 0, s>>>(g, n_iter, tol, U, P, ret, n);
    return cudaGetLastError();
}

// Newton on W from given guesses (the learned path's refinement), FP64
__global__ void k_point_c2p_w(double g, const double* __restrict__ U, const double* __restrict__ W0, double rtol,
                              int max_newton, int max_bracket, double* __restrict__ P, int* __restrict__ iters,
                              int* __restrict__ fallback, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double u[5], p[5];
        for (int v = 0; v < 5; ++v) u[v] = U[v * n + i];
        int fb = 0;
        int r = c2p_w(g, u, W0[i], rtol, max_newton, max_bracket, p, &fb);
        for (int v = 0; v < 5; ++v) P[v * n + i] = p[v];
        if (iters) iters[i] = r;
        if (fallback) fallback[i] = fb;
    }
}

cudaError_t launch_point_c2p_w(double g, const double* U, const double* W0, double rtol, int max_newton,
                               int max_bracket, double* P, int* iters, int* fallback, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_point_c2p_w<<<grid_for(n, 128), 128, 0, s>>>(g, U, W0, rtol, max_newton, max_bracket, P, iters, fallback, n);
    return cudaGetLastError();
}

// the learned guess's precision-gated refinement (c2p_w_gated) from FP32 guesses
__global__ void k_point_c2p_gated(double g, const double* __restrict__ U, const float* __restrict__ W0, double rtol,
                                  int max_newton, int max_bracket, double* __restrict__ P, int* __restrict__ iters,
                                  int* __restrict__ fp64, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double u[5], p[5];
        for (int v = 0; v < 5; ++v) u[v] = U[v * n + i];
        int fb = 0, f64 = 1;
        int r = c2p_w_gated(g, u, W0[i], rtol, max_newton, max_bracket, true, p, &fb, &f64);
        for (int v = 0; v < 5; ++v) P[v * n + i] = p[v];
        if (iters) iters[i] = r;
        if (fp64) fp64[i] = f64;
    }
}

cudaError_t launch_point_c2p_gated(double g, const double* U, const float* W0, double rtol, int max_newton,
                                   int max_bracket, double* P, int* iters, int* fp64, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_point_c2p_gated<<<grid_for(n, 128), 128, 0, s>>>(g, U, W0, rtol, max_newton, max_bracket, P, iters, fp64, n);
    return cudaGetLastError();
}

int max_speed_blocks(const Grid& g) {
    (void)g;
    return 148 * 4;
}
}  // namespace vb
