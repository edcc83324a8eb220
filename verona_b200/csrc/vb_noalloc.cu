// vb_max_signal_speed_noalloc: the CFL signal-speed reduction of
// vb_max_signal_speed, for callers that must not allocate device memory.
//
// Who needs it: a host whose device-memory pool already owns nearly all of
// the GPU (CUDA.jl's pool, or a framework's caching allocator) cannot let a
// library call cudaMalloc behind its back -- the call may fail, or fragment
// the pool -- and cudaMalloc/cudaFree may also synchronise the device in the
// middle of the caller's stream work. This entry point therefore takes the
// primitive array and the output location from the caller and keeps its
// only scratch (one partial maximum per thread block) in a fixed array
// compiled into the library.
//
// The scratch is a file-scope `static __device__` array: every GPU that
// loads the library holds its 64 KiB until the process exits. Host code must
// not pass the array's name to a kernel (on the host it is only a stand-in,
// not a device address); its device address is looked up with
// cudaGetSymbolAddress on the first call made while a device is current, and
// cached together with that device's SM count and the CUDA context it was
// looked up in. A call made in another context of the same device (after
// cudaDeviceReset, or after the host reset the device) looks both up again,
// so an address of a destroyed context is never used. Make the first call on
// a device, and the first after a reset, before any stream capture. All calls
// share the one array and it keeps the last call's contents: each call writes
// every partial it later reads, so nothing needs clearing, but two calls
// whose kernels overlap on the GPU (different streams, no ordering between
// them) race on it.
#include <cuda.h>
#include <cudaTypedefs.h>  // PFN_cuCtxGetCurrent
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/verona_b200.h"
#include "vb_stage.cuh"

namespace vb {

constexpr int NA_THREADS = MS_THREADS;           // 256 threads per block
constexpr int NA_CELLS_PER_THREAD = 128;         // cells one thread covers at most
constexpr int NA_MAX_BLOCKS = 8192;              // partials in the static scratch
constexpr long long NA_MAX_CELLS = (long long)NA_MAX_BLOCKS * NA_THREADS * NA_CELLS_PER_THREAD;
constexpr int NA_MAX_DEVICES = 64;

// The only scratch of this entry point: 8192 doubles = 64 KiB per device.
static __device__ __align__(256) double vb_noalloc_partial[NA_MAX_BLOCKS];

// Same per-cell physics and warp/block max as k_max_speed, reading the
// caller's array in the reference's AoS layout (variable fastest).
template <int DIM>
__global__ void __launch_bounds__(NA_THREADS) k_max_speed_aos(int n0, int n1, int n2, const double* __restrict__ Pa,
                                                              double gamma, double* __restrict__ partial) {
    constexpr int NV = 2 + DIM;
    const int N0 = n0 - 2 * NG;
    const int N1 = DIM > 1 ? n1 - 2 * NG : 1;
    const int N2 = DIM > 2 ? n2 - 2 * NG : 1;
    const long long tot = (long long)N0 * N1 * N2;
    double m = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        int i = (int)(e % N0) + NG;
        int j = DIM > 1 ? (int)((e / N0) % N1) + NG : 0;
        int k = DIM > 2 ? (int)(e / ((long long)N0 * N1)) + NG : 0;
        long long c = i + (long long)n0 * (j + (long long)n1 * k);
        double q[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) q[v] = Pa[c * NV + v];
        m = fmax(m, max_signal_speed<DIM>(gamma, q));
    }
    m = block_max(m);
    if (threadIdx.x == 0) partial[blockIdx.x] = m;
}

__global__ void __launch_bounds__(NA_THREADS) k_max_reduce_to(const double* __restrict__ partial, int n,
                                                              double* __restrict__ out) {
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, partial[i]);
    m = block_max(m);
    if (threadIdx.x == 0) *out = m;
}

// device address of vb_noalloc_partial and the SM count, looked up once per
// device and context
struct NaDevice {
    CUcontext ctx;
    double* partial;
    int sms;
};
static NaDevice g_na_dev[NA_MAX_DEVICES] = {};
static std::mutex g_na_mu;

// cuCtxGetCurrent through the runtime's entry-point query (no driver library
// is linked); nullptr where the driver does not provide it
static PFN_cuCtxGetCurrent_v4000 ctx_getter() {
    static PFN_cuCtxGetCurrent_v4000 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f);
    }();
    return fn;
}

static cudaError_t scratch_for_current_device(double** out, int* sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return cudaErrorInvalidDevice;
    PFN_cuCtxGetCurrent_v4000 get = ctx_getter();
    if (!get) return cudaErrorNotSupported;
    // the context current on this thread; null before the runtime has made the
    // device's primary context current (cudaGetSymbolAddress does that)
    CUcontext ctx = nullptr;
    if (get(&ctx) != CUDA_SUCCESS) return cudaErrorNotSupported;
    std::lock_guard<std::mutex> lock(g_na_mu);
    NaDevice& d = g_na_dev[dev];
    if (!d.partial || !ctx || d.ctx != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, vb_noalloc_partial);
        if (e != cudaSuccess) return e;
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        if (get(&ctx) != CUDA_SUCCESS || !ctx) return cudaErrorNotSupported;
        d.ctx = ctx;
        d.partial = static_cast<double*>(p);
        d.sms = n > 0 ? n : 1;
    }
    *out = d.partial;
    *sms = d.sms;
    return cudaSuccess;
}

}  // namespace vb

using namespace vb;

static thread_local char g_na_err[256];

extern "C" const char* vb_noalloc_last_error(void) { return g_na_err; }

static int na_fail(int code, const char* msg, cudaError_t e = cudaSuccess) {
    if (e != cudaSuccess)
        snprintf(g_na_err, sizeof g_na_err, "vb_max_signal_speed_noalloc: %s: %s", msg, cudaGetErrorString(e));
    else
        snprintf(g_na_err, sizeof g_na_err, "vb_max_signal_speed_noalloc: %s", msg);
    return code;
}

extern "C" int vb_max_signal_speed_noalloc(int dims, int nx, int ny, int nz, double gamma, const double* P_aos_dev,
                                           double* c_dev, void* stream) {
    g_na_err[0] = 0;
    if (dims < 1 || dims > 3) return na_fail(VB_ERR_ARG, "dims must be 1, 2 or 3");
    if (!P_aos_dev || !c_dev) return na_fail(VB_ERR_ARG, "null array");
    int nn[3] = {nx, dims > 1 ? ny : 1, dims > 2 ? nz : 1};
    for (int a = 0; a < dims; ++a)
        if (nn[a] < 1) return na_fail(VB_ERR_ARG, "interior size below 1");
    const long long cells = (long long)nn[0] * nn[1] * nn[2];
    if (cells > NA_MAX_CELLS) {
        snprintf(g_na_err, sizeof g_na_err,
                 "vb_max_signal_speed_noalloc: %lld interior cells exceed the maximum of %lld "
                 "(8192 partials x 256 threads x 128 cells); use vb_max_signal_speed",
                 cells, NA_MAX_CELLS);
        return VB_ERR_ARG;
    }
    double* partial = nullptr;
    int sms = 1;
    cudaError_t e = scratch_for_current_device(&partial, &sms);
    if (e != cudaSuccess) return na_fail(VB_ERR_CUDA, "cudaGetSymbolAddress", e);
    // enough blocks that no thread covers more than NA_CELLS_PER_THREAD cells,
    // and at least enough to fill the GPU (4 per SM) unless the grid is tiny;
    // at most NA_MAX_BLOCKS because cells <= NA_MAX_CELLS
    const long long per_block = (long long)NA_THREADS * NA_CELLS_PER_THREAD;
    const long long need = (cells + per_block - 1) / per_block;
    const long long fill = std::min((cells + NA_THREADS - 1) / NA_THREADS, 4LL * sms);
    const int nb = (int)std::min<long long>(std::max(need, fill), NA_MAX_BLOCKS);
    cudaStream_t s = (cudaStream_t)stream;
    const int n0 = nn[0] + 2 * NG, n1 = dims > 1 ? nn[1] + 2 * NG : 1, n2 = dims > 2 ? nn[2] + 2 * NG : 1;
    if (dims == 1) k_max_speed_aos<1><<<nb, NA_THREADS, 0, s>>>(n0, n1, n2, P_aos_dev, gamma, partial);
    else if (dims == 2) k_max_speed_aos<2><<<nb, NA_THREADS, 0, s>>>(n0, n1, n2, P_aos_dev, gamma, partial);
    else k_max_speed_aos<3><<<nb, NA_THREADS, 0, s>>>(n0, n1, n2, P_aos_dev, gamma, partial);
    e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(VB_ERR_CUDA, "partial-max launch", e);
    k_max_reduce_to<<<1, NA_THREADS, 0, s>>>(partial, nb, c_dev);
    e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(VB_ERR_CUDA, "final-max launch", e);
    return VB_OK;
}
