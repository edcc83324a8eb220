// C ABI of libverona_b200.so (include/verona_b200.h): handle lifecycle, state
// buffers and the time-loop body that replaces the inner loop of the
// reference's HARM_HLL (src/3dim/algos.jl:274-329, src/2dim/algos.jl:256-310,
// src/1dim/algos.jl:89-313).
//
// Device state of a 2D/3D handle (interior N, padded N+6 per axis):
//   P[2]   primitive ping-pong buffers, SoA (one contiguous array per
//          variable, x fastest), FP64 or FP32 (FP32-bulk precision)
//   U0, U1 conserved variables, SoA FP64 (U^n and the stage state)
//   cnt    VB_CNT_* counters; partial/out: CFL reduction scratch
//   stage  FP64 AoS staging buffer for host-pointer loads/stores (lazy)
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/verona_b200.h"
#include "vb_internal.h"

using namespace vb;

extern "C" const void* vb_mlp_blob_ptr(vb_mlp_handle m);  // vb_mlp.cu

struct vb_solver {
    int device = 0;
    int dims = 0, nv = 0, nghost = 3;
    int n[3] = {1, 1, 1};   // interior
    int np[3] = {1, 1, 1};  // padded
    long long ncell = 0, vs = 0;  // padded cells; elements between variable arrays
    long long sy = 0, sz = 0;       // strides of j and k in the SoA arrays (rows pitched)
    vb_options opt{};
    double gamma = 5.0 / 3.0;
    double dx[3] = {1.0, 1.0, 1.0};
    double t = 0.0;
    int bc_kind[6] = {0, 0, 0, 0, 0, 0};
    double bc_par[6][16] = {};
    bool loaded = false;
    // ND state
    void* P[2] = {nullptr, nullptr};
    int cur = 0;
    double* U0 = nullptr;
    double* U1 = nullptr;
    // 1D reference state
    Ref1DState r1{};
    // shared
    unsigned long long* cnt = nullptr;
    double* partial = nullptr;
    double* red_out = nullptr;
    int max_partial = 0;
    double* staging = nullptr;
    size_t bytes = 0;
    std::string err;
    // kernel variants
    vb_tuning tun{-1, 0, -1, -1, -1, 0, {0, 0}};
    // TMA tensor maps of P[0], P[1] (the TMA forms of the stage kernels: 3D FP32, 2D)
    alignas(64) unsigned char tmap[2][128] = {};
    bool tmap_ok[2] = {false, false};
    // learned con2prim guess
    const void* mlp_blob = nullptr;
    unsigned int* tc_err = nullptr;
    float* w_guess = nullptr;  // one W guess per padded cell
    unsigned int* defer_idx = nullptr;  // gated learned con2prim: cells left to FP64 (one slot per interior cell)
    unsigned int* defer_n = nullptr;    // their count
    // asynchronous dumps (vb_dump_begin / vb_dump_wait)
    double* dump_buf = nullptr;            // interior snapshot, reference interior layout
    unsigned long long* dump_nan = nullptr;  // device NaN count of the snapshot
    unsigned long long* dump_nan_host = nullptr;  // pinned
    cudaStream_t dump_stream = nullptr;
    cudaEvent_t dump_packed = nullptr, dump_copied = nullptr;
    bool dump_pending = false;
    // profiling
    bool prof = false;
    std::vector<cudaEvent_t> ev;
    size_t ev_used = 0;
    long long launches = 0, stage_launches = 0;
};

static thread_local std::string g_err;

static int fail(vb_handle h, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (h)
        h->err = buf;
    else
        g_err = buf;
    return code;
}

#define VB_CUDA(h, expr)                                                                             \
    do {                                                                                             \
        cudaError_t e_ = (expr);                                                                     \
        if (e_ != cudaSuccess) return fail(h, VB_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

static Grid grid_of(const vb_solver* h) {
    Grid g;
    g.dims = h->dims;
    g.nv = h->nv;
    for (int a = 0; a < 3; ++a) g.n[a] = h->np[a];
    g.sy = h->sy;
    g.sz = h->sz;
    g.vs = h->vs;
    return g;
}

static bool fp32(const vb_solver* h) { return h->opt.precision == VB_PREC_FP32_BULK; }

static int dev_alloc(vb_handle h, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(h, VB_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    h->bytes += bytes;
    return VB_OK;
}

extern "C" {

int vb_default_options(vb_options* o) {
    if (!o) return fail(nullptr, VB_ERR_ARG, "vb_default_options: null");
    memset(o, 0, sizeof *o);
    o->version = VB_ABI_VERSION;
    o->recon = VB_RECON_WENOZ;
    o->riemann = VB_RIEMANN_HLL;
    o->rk = VB_RK2;
    o->precision = VB_PREC_FP64;
    o->guess = VB_GUESS_PREVIOUS;
    o->n_iter = 50;
    o->stats = 0;
    o->tol = 1e-10;
    o->floor_ = 1e-7;
    o->w_rtol = 1e-12;
    o->w_max_newton = 8;
    o->c2p_fp32 = 1;
    return VB_OK;
}

const char* vb_last_error(vb_handle h) { return h ? h->err.c_str() : g_err.c_str(); }

int vb_destroy(vb_handle h) {
    if (!h) return VB_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    cudaFree(h->P[0]);
    cudaFree(h->P[1]);
    cudaFree(h->U0);
    cudaFree(h->U1);
    cudaFree(h->r1.P);
    cudaFree(h->cnt);
    cudaFree(h->partial);
    cudaFree(h->staging);
    cudaFree(h->tc_err);
    cudaFree(h->w_guess);
    cudaFree(h->defer_idx);
    cudaFree(h->defer_n);
    if (h->dump_stream) cudaStreamSynchronize(h->dump_stream);
    cudaFree(h->dump_buf);
    cudaFree(h->dump_nan);
    cudaFreeHost(h->dump_nan_host);
    if (h->dump_packed) cudaEventDestroy(h->dump_packed);
    if (h->dump_copied) cudaEventDestroy(h->dump_copied);
    if (h->dump_stream) cudaStreamDestroy(h->dump_stream);
    for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
    cudaSetDevice(prev);
    delete h;
    return VB_OK;
}

int vb_create(vb_handle* out, int dims, int nx, int ny, int nz, int nghost, const vb_options* o) {
    if (!out) return fail(nullptr, VB_ERR_ARG, "vb_create: null handle pointer");
    *out = nullptr;
    if (dims < 1 || dims > 3) return fail(nullptr, VB_ERR_ARG, "vb_create: dims must be 1, 2 or 3 (got %d)", dims);
    int nn[3] = {nx, dims > 1 ? ny : 1, dims > 2 ? nz : 1};
    for (int a = 0; a < dims; ++a)
        if (nn[a] < 1) return fail(nullptr, VB_ERR_ARG, "vb_create: interior size %d along axis %d", nn[a], a);
    if (!(nghost == 3 || (nghost == 0 && dims == 1)))
        return fail(nullptr, VB_ERR_ARG, "vb_create: nghost must be 3, or 0 with dims == 1 (got %d)", nghost);
    vb_options opt;
    vb_default_options(&opt);
    if (o) {
        if (o->version != VB_ABI_VERSION)
            return fail(nullptr, VB_ERR_ARG, "vb_create: options version %u, library %d", o->version, VB_ABI_VERSION);
        opt = *o;
    }
    if (opt.recon < 0 || opt.recon > 2) return fail(nullptr, VB_ERR_ARG, "vb_create: recon %d", opt.recon);
    if (opt.riemann < 0 || opt.riemann > 1) return fail(nullptr, VB_ERR_ARG, "vb_create: riemann %d", opt.riemann);
    if (opt.rk != 2 && opt.rk != 3) return fail(nullptr, VB_ERR_ARG, "vb_create: rk must be 2 or 3 (got %d)", opt.rk);
    if (opt.precision < 0 || opt.precision > 1)
        return fail(nullptr, VB_ERR_ARG, "vb_create: precision %d", opt.precision);
    if (opt.n_iter < 1 || opt.n_iter > 100000) return fail(nullptr, VB_ERR_ARG, "vb_create: n_iter %d", opt.n_iter);
    if (opt.guess < VB_GUESS_PREVIOUS || opt.guess > VB_GUESS_PREVIOUS_W)
        return fail(nullptr, VB_ERR_ARG, "vb_create: guess %d", opt.guess);
    if (opt.guess == VB_GUESS_LEARNED && dims != 3)
        return fail(nullptr, VB_ERR_UNSUPPORTED, "vb_create: the learned con2prim guess is provided for 3D grids");
    if (opt.guess == VB_GUESS_PREVIOUS_W && dims == 1)
        return fail(nullptr, VB_ERR_UNSUPPORTED, "vb_create: the previous-W con2prim guess is provided for 2D and 3D grids");
    if (nghost == 0 && (opt.riemann != VB_RIEMANN_HLL || opt.rk != 2 || opt.precision != VB_PREC_FP64))
        return fail(nullptr, VB_ERR_UNSUPPORTED,
                    "vb_create: the 1D reference layout (nghost=0) runs the reference scheme only (HLL, RK2, FP64)");

    vb_handle h = new vb_solver();
    cudaGetDevice(&h->device);
    h->dims = dims;
    h->nv = 2 + dims;
    h->nghost = nghost;
    h->opt = opt;
    for (int a = 0; a < 3; ++a) {
        h->n[a] = nn[a];
        h->np[a] = a < dims ? nn[a] + 2 * nghost : 1;
    }
    h->ncell = (long long)h->np[0] * h->np[1] * h->np[2];
    // 2D / 3D rows are pitched to a multiple of 4 cells, so that every row and
    // plane stride is a multiple of 16 bytes (the tensor-map stride rule of TMA)
    h->sy = dims >= 2 ? (h->np[0] + 3) / 4 * 4 : h->np[0];
    h->sz = h->sy * h->np[1];
    h->vs = (h->sz * h->np[2] + 31) / 32 * 32;  // each variable array starts on a 256-byte boundary
    int rc;
    if (nghost == 0) {
        const int N = nx;
        double* base = nullptr;
        if ((rc = dev_alloc(h, (void**)&base, sizeof(double) * 7 * 3 * (size_t)N))) {
            g_err = h->err;
            delete h;
            return rc;
        }
        h->r1.N = N;
        h->r1.P = base;
        h->r1.Ph = base + 3 * N;
        h->r1.U = base + 6 * N;
        h->r1.Uh = base + 9 * N;
        h->r1.PL = base + 12 * N;
        h->r1.PR = base + 15 * N;
        h->r1.F = base + 18 * N;
    } else {
        size_t pb = (fp32(h) ? sizeof(float) : sizeof(double)) * h->nv * (size_t)h->vs;
        size_t ub = sizeof(double) * h->nv * (size_t)h->vs;
        if ((rc = dev_alloc(h, &h->P[0], pb)) || (rc = dev_alloc(h, &h->P[1], pb)) ||
            (rc = dev_alloc(h, (void**)&h->U0, ub)) || (rc = dev_alloc(h, (void**)&h->U1, ub))) {
            g_err = h->err;
            vb_destroy(h);
            return rc;
        }
    }
    if (nghost != 0 && dims >= 2)
        for (int i = 0; i < 2; ++i)
            h->tmap_ok[i] = fp32(h) ? encode_stage_tmap<float>(h->tmap[i], (const float*)h->P[i], grid_of(h))
                                    : encode_stage_tmap<double>(h->tmap[i], (const double*)h->P[i], grid_of(h));
    h->max_partial = max_speed_blocks(grid_of(h));
    if ((rc = dev_alloc(h, (void**)&h->cnt, sizeof(unsigned long long) * CNT_N)) ||
        (rc = dev_alloc(h, (void**)&h->partial, sizeof(double) * (h->max_partial + 1)))) {
        g_err = h->err;
        vb_destroy(h);
        return rc;
    }
    h->red_out = h->partial + h->max_partial;
    cudaError_t e = cudaMemset(h->cnt, 0, sizeof(unsigned long long) * CNT_N);
    if (e != cudaSuccess) {
        g_err = cudaGetErrorString(e);
        vb_destroy(h);
        return VB_ERR_CUDA;
    }
    *out = h;
    return VB_OK;
}

int vb_set_eos(vb_handle h, double gamma) {
    if (!h) return fail(nullptr, VB_ERR_ARG, "null handle");
    if (!(gamma > 1.0 && gamma < 3.0)) return fail(h, VB_ERR_ARG, "vb_set_eos: gamma %g outside (1, 3)", gamma);
    if (h->loaded) return fail(h, VB_ERR_STATE, "vb_set_eos: call before vb_load_prims (U is derived from it)");
    h->gamma = gamma;
    return VB_OK;
}

int vb_set_grid(vb_handle h, double dx, double dy, double dz) {
    if (!h) return fail(nullptr, VB_ERR_ARG, "null handle");
    double d[3] = {dx, dy, dz};
    for (int a = 0; a < h->dims; ++a)
        if (!(d[a] > 0.0)) return fail(h, VB_ERR_ARG, "vb_set_grid: spacing %g along axis %d", d[a], a);
    for (int a = 0; a < 3; ++a) h->dx[a] = d[a];
    return VB_OK;
}

int vb_set_boundary(vb_handle h, int face, int kind, const double* par, int np) {
    if (!h) return fail(nullptr, VB_ERR_ARG, "null handle");
    if (h->nghost == 0) return fail(h, VB_ERR_STATE, "vb_set_boundary: the 1D reference layout has fixed end cells");
    if (face < 0 || face >= 2 * h->dims) return fail(h, VB_ERR_ARG, "vb_set_boundary: face %d for dims %d", face, h->dims);
    if (kind < 0 || kind > 2) return fail(h, VB_ERR_ARG, "vb_set_boundary: kind %d", kind);
    if (np < 0 || np > 16 || (np > 0 && !par)) return fail(h, VB_ERR_ARG, "vb_set_boundary: %d params", np);
    if (kind == VB_BC_FIXED && np > 0 && np < 4)
        return fail(h, VB_ERR_ARG, "vb_set_boundary: FIXED decay needs {var, t_on, t_off, factor}");
    if (kind == VB_BC_FIXED && np >= 4 && (par[0] < 0 || par[0] >= h->nv))
        return fail(h, VB_ERR_ARG, "vb_set_boundary: decay variable %g", par[0]);
    if (kind == VB_BC_NOZZLE && np < 5 + h->dims)
        return fail(h, VB_ERR_ARG, "vb_set_boundary: NOZZLE needs {radius, c1, c2, rho, u, u1..u%d}", h->dims);
    h->bc_kind[face] = kind;
    memset(h->bc_par[face], 0, sizeof h->bc_par[face]);
    for (int i = 0; i < np; ++i) h->bc_par[face][i] = par[i];
    if (kind == VB_BC_FIXED && np == 0) h->bc_par[face][0] = -1.0;  // no decay
    return VB_OK;
}

int vb_load_prims(vb_handle h, const double* Pa, void* stream) {
    if (!h || !Pa) return fail(h, VB_ERR_ARG, "vb_load_prims: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (h->nghost == 0) {
        VB_CUDA(h, launch_ref1d_init(h->r1, Pa, h->gamma, s));
    } else {
        Grid g = grid_of(h);
        if (fp32(h))
            VB_CUDA(h, launch_load_prims<float>(g, Pa, (float*)h->P[h->cur], h->U0, h->gamma, s));
        else
            VB_CUDA(h, launch_load_prims<double>(g, Pa, (double*)h->P[h->cur], h->U0, h->gamma, s));
    }
    h->loaded = true;
    return VB_OK;
}

int vb_store_prims(vb_handle h, double* Pa, void* stream) {
    if (!h || !Pa) return fail(h, VB_ERR_ARG, "vb_store_prims: null argument");
    if (!h->loaded) return fail(h, VB_ERR_STATE, "vb_store_prims: no state loaded");
    cudaStream_t s = (cudaStream_t)stream;
    if (h->nghost == 0) {
        VB_CUDA(h, launch_ref1d_store(h->r1, Pa, s));
    } else {
        Grid g = grid_of(h);
        if (fp32(h))
            VB_CUDA(h, launch_store_prims<float>(g, (const float*)h->P[h->cur], Pa, s));
        else
            VB_CUDA(h, launch_store_prims<double>(g, (const double*)h->P[h->cur], Pa, s));
    }
    return VB_OK;
}

static size_t aos_bytes(const vb_solver* h) {
    return sizeof(double) * h->nv * (size_t)(h->nghost == 0 ? h->n[0] : h->ncell);
}

static int ensure_staging(vb_handle h) {
    if (h->staging) return VB_OK;
    return dev_alloc(h, (void**)&h->staging, aos_bytes(h));
}

int vb_load_prims_host(vb_handle h, const double* Pa, void* stream) {
    if (!h || !Pa) return fail(h, VB_ERR_ARG, "vb_load_prims_host: null argument");
    int rc = ensure_staging(h);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    VB_CUDA(h, cudaMemcpyAsync(h->staging, Pa, aos_bytes(h), cudaMemcpyHostToDevice, s));
    rc = vb_load_prims(h, h->staging, stream);
    if (rc) return rc;
    VB_CUDA(h, cudaStreamSynchronize(s));
    return VB_OK;
}

int vb_store_prims_host(vb_handle h, double* Pa, void* stream) {
    if (!h || !Pa) return fail(h, VB_ERR_ARG, "vb_store_prims_host: null argument");
    int rc = ensure_staging(h);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    rc = vb_store_prims(h, h->staging, stream);
    if (rc) return rc;
    VB_CUDA(h, cudaMemcpyAsync(Pa, h->staging, aos_bytes(h), cudaMemcpyDeviceToHost, s));
    VB_CUDA(h, cudaStreamSynchronize(s));
    return VB_OK;
}

int vb_store_cons(vb_handle h, double* Ua, void* stream) {
    if (!h || !Ua) return fail(h, VB_ERR_ARG, "vb_store_cons: null argument");
    if (!h->loaded) return fail(h, VB_ERR_STATE, "vb_store_cons: no state loaded");
    cudaStream_t s = (cudaStream_t)stream;
    if (h->nghost == 0) {
        Ref1DState t = h->r1;
        t.P = h->r1.U;  // the store kernel transposes r1.P; point it at U
        VB_CUDA(h, launch_ref1d_store(t, Ua, s));
    } else {
        VB_CUDA(h, launch_store_prims<double>(grid_of(h), h->U0, Ua, s));
    }
    return VB_OK;
}

static size_t interior_bytes(const vb_solver* h) {
    return sizeof(double) * h->nv * (size_t)h->n[0] * h->n[1] * h->n[2];
}

int vb_dump_begin(vb_handle h, double* host_out, void* stream) {
    if (!h || !host_out) return fail(h, VB_ERR_ARG, "vb_dump_begin: null argument");
    if (h->nghost == 0) return fail(h, VB_ERR_UNSUPPORTED, "vb_dump_begin: the 1D reference layout stores with vb_store_prims_host");
    if (!h->loaded) return fail(h, VB_ERR_STATE, "vb_dump_begin: no state loaded");
    if (!h->dump_buf) {
        int rc = dev_alloc(h, (void**)&h->dump_buf, interior_bytes(h));
        if (rc) return rc;
        rc = dev_alloc(h, (void**)&h->dump_nan, sizeof(unsigned long long));
        if (rc) return rc;
        VB_CUDA(h, cudaMallocHost((void**)&h->dump_nan_host, sizeof(unsigned long long)));
        VB_CUDA(h, cudaStreamCreateWithFlags(&h->dump_stream, cudaStreamNonBlocking));
        VB_CUDA(h, cudaEventCreateWithFlags(&h->dump_packed, cudaEventDisableTiming));
        VB_CUDA(h, cudaEventCreateWithFlags(&h->dump_copied, cudaEventDisableTiming));
    }
    cudaStream_t s = (cudaStream_t)stream;
    // the previous dump's copy must have read the snapshot buffer before it is overwritten
    if (h->dump_pending) VB_CUDA(h, cudaStreamWaitEvent(s, h->dump_copied, 0));
    VB_CUDA(h, cudaMemsetAsync(h->dump_nan, 0, sizeof(unsigned long long), s));
    Grid g = grid_of(h);
    if (fp32(h))
        VB_CUDA(h, launch_pack_interior<float>(g, (const float*)h->P[h->cur], h->dump_buf, h->dump_nan, s));
    else
        VB_CUDA(h, launch_pack_interior<double>(g, (const double*)h->P[h->cur], h->dump_buf, h->dump_nan, s));
    VB_CUDA(h, cudaEventRecord(h->dump_packed, s));
    VB_CUDA(h, cudaStreamWaitEvent(h->dump_stream, h->dump_packed, 0));
    VB_CUDA(h, cudaMemcpyAsync(host_out, h->dump_buf, interior_bytes(h), cudaMemcpyDeviceToHost, h->dump_stream));
    VB_CUDA(h, cudaMemcpyAsync(h->dump_nan_host, h->dump_nan, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                               h->dump_stream));
    VB_CUDA(h, cudaEventRecord(h->dump_copied, h->dump_stream));
    h->dump_pending = true;
    return VB_OK;
}

int vb_dump_wait(vb_handle h, uint64_t* nan_count) {
    if (!h) return fail(nullptr, VB_ERR_ARG, "vb_dump_wait: null handle");
    if (!h->dump_pending) return fail(h, VB_ERR_STATE, "vb_dump_wait: no dump in flight");
    VB_CUDA(h, cudaEventSynchronize(h->dump_copied));
    h->dump_pending = false;
    if (nan_count) *nan_count = *h->dump_nan_host;
    return VB_OK;
}

int vb_default_ic(int dims, int kind, vb_ic_params* ic) {
    if (!ic || dims < 1 || dims > 3 || kind < VB_IC_AMBIENT || kind > VB_IC_STAR_JET)
        return fail(nullptr, VB_ERR_ARG, "vb_default_ic: bad argument");
    *ic = vb_ic_params{};
    ic->version = VB_ABI_VERSION;
    ic->kind = kind;
    ic->seed = 42;  // the examples' seed
    ic->noise = 3e-2;
    ic->rho = 1.0;
    ic->u = 3e-3;
    if (dims == 3) {  // examples/Jet3D/HARM_jet_breakout.jl:46-61
        ic->box[0] = 480.0;
        ic->box[1] = 120.0;
        ic->box[2] = 120.0;
        ic->r_eng = 5.0;
        ic->engine_rho = 1e-2;
    } else {  // examples/Jet2D/HARM_jet_breakout.jl:26-36
        ic->box[0] = 800.0;
        ic->box[1] = 200.0;
        ic->box[2] = 0.0;
        ic->r_eng = 2.0;
        ic->engine_rho = 1e-3;
    }
    ic->r_max = 100.0;
    ic->rho0 = 2.5e-2;
    ic->temp = 1e-5;
    ic->outer = 1e-4;
    ic->gamma0 = 10.0;
    ic->engine_temp = 1e-5;
    return VB_OK;
}

int vb_init_prims(vb_handle h, const vb_ic_params* ic, void* stream) {
    if (!h || !ic) return fail(h, VB_ERR_ARG, "vb_init_prims: null argument");
    if (ic->version != VB_ABI_VERSION) return fail(h, VB_ERR_ARG, "vb_init_prims: version %u", ic->version);
    if (h->nghost == 0) return fail(h, VB_ERR_UNSUPPORTED, "vb_init_prims: the 1D reference layout loads host arrays");
    if (ic->kind != VB_IC_AMBIENT && ic->kind != VB_IC_STAR_JET)
        return fail(h, VB_ERR_ARG, "vb_init_prims: kind %d", ic->kind);
    if (ic->kind == VB_IC_STAR_JET && h->dims < 2)
        return fail(h, VB_ERR_UNSUPPORTED, "vb_init_prims: the star + jet condition is 2D or 3D");
    if (ic->kind == VB_IC_STAR_JET && (!(ic->r_eng > 0.0) || !(ic->r_max > 0.0) || !(ic->gamma0 > 1.0)))
        return fail(h, VB_ERR_ARG, "vb_init_prims: r_eng, r_max > 0 and gamma0 > 1 required");
    InitIC c{};
    c.kind = ic->kind;
    c.seed = ic->seed;
    c.noise = ic->noise;
    c.rho = ic->rho;
    c.u = ic->u;
    for (int a = 0; a < 3; ++a) {
        c.box[a] = ic->box[a];
        c.dx[a] = (a == 0 ? 1.0 : 2.0) * ic->box[a] / (double)h->np[a];
    }
    c.r_max = ic->r_max;
    c.r_eng = ic->r_eng;
    c.rho0 = ic->rho0;
    c.temp = ic->temp;
    c.outer = ic->outer;
    c.gamma0 = ic->gamma0;
    c.engine_rho = ic->engine_rho;
    c.engine_temp = ic->engine_temp;
    cudaStream_t s = (cudaStream_t)stream;
    Grid g = grid_of(h);
    if (fp32(h))
        VB_CUDA(h, launch_init_prims<float>(g, c, (float*)h->P[h->cur], h->U0, h->gamma, s));
    else
        VB_CUDA(h, launch_init_prims<double>(g, c, (double*)h->P[h->cur], h->U0, h->gamma, s));
    h->loaded = true;
    return VB_OK;
}

}  // extern "C"

// three events per stage: start, after the stencil launcher, after the stage's con2prim
static int prof_events(vb_handle h, cudaEvent_t* a, cudaEvent_t* m, cudaEvent_t* b) {
    while (h->ev.size() < h->ev_used + 3) {
        cudaEvent_t e;
        VB_CUDA(h, cudaEventCreate(&e));
        h->ev.push_back(e);
    }
    *a = h->ev[h->ev_used];
    *m = h->ev[h->ev_used + 1];
    *b = h->ev[h->ev_used + 2];
    h->ev_used += 3;
    return VB_OK;
}

// boundary fill at the start of a step (decay, then y-lo, y-hi, z-lo, z-hi, x-lo, x-hi)
template <typename R> static int bc_fill(vb_handle h, R* P, cudaStream_t s) {
    Grid g = grid_of(h);
    for (int face = 0; face < 2 * h->dims; ++face) {
        if (h->bc_kind[face] != VB_BC_FIXED) continue;
        const double* par = h->bc_par[face];
        if (par[0] < 0) continue;
        if (!(h->t > par[1] && h->t < par[2])) continue;
        VB_CUDA(h, launch_bc_decay<R>(g, P, face, (int)par[0], par[3], s));
        h->launches += 1;
    }
    static const int order[6] = {2, 3, 4, 5, 0, 1};
    for (int oi = 0; oi < 6; ++oi) {
        int face = order[oi];
        if (face / 2 >= h->dims || h->bc_kind[face] == VB_BC_FIXED) continue;
        VB_CUDA(h, launch_bc_face<R>(g, P, face, h->bc_kind[face], h->bc_par[face], s));
        h->launches += 1;
    }
    return VB_OK;
}

// split con2prim by default in 3D, where the stencil kernel then runs without
// holding its registers through the divergent Newton (measured faster there)
static int default_split(const vb_solver* h) { return h->dims == 3 ? 1 : 0; }

template <typename R> static int step_nd(vb_handle h, double dt, cudaStream_t s) {
    Grid g = grid_of(h);
    R* P[2] = {(R*)h->P[0], (R*)h->P[1]};
    int c = h->cur;
    int rc = bc_fill<R>(h, P[c], s);
    if (rc) return rc;
    StageParams p{};
    for (int a = 0; a < 3; ++a) p.n[a] = h->np[a];
    p.sy = g.sy;
    p.sz = g.sz;
    p.vs = h->vs;
    p.gamma = h->gamma;
    p.floor_ = h->opt.floor_;
    p.tol = h->opt.tol;
    p.n_iter = h->opt.n_iter;
    p.stats = h->opt.stats;
    const bool w_newton = h->opt.guess == VB_GUESS_LEARNED || h->opt.guess == VB_GUESS_PREVIOUS_W;
    p.c2p_mode = w_newton ? C2P_GUESS_W : C2P_REFERENCE;
    p.w_rtol = h->opt.w_rtol;
    p.w_max_newton = h->opt.w_max_newton;
    p.w_guess = nullptr;
    p.c2p_fp32 = fp32(h) && w_newton && h->opt.c2p_fp32 == 1;
    p.counters = h->cnt;
    p.force_box = h->tun.force_box;
    p.split = h->tun.split_con2prim < 0 ? default_split(h) : h->tun.split_con2prim;
    // 2D with the previous-W guess: that con2prim runs only in the split kernel
    if (h->dims == 2 && h->opt.guess == VB_GUESS_PREVIOUS_W) p.split = 1;
    p.skip_c2p = 0;
    p.pairs = h->tun.fp32_pairs != 0;
    if (h->opt.guess == VB_GUESS_LEARNED) {
        if (!h->mlp_blob) return fail(h, VB_ERR_STATE, "vb_step: guess = LEARNED needs vb_attach_mlp");
        p.skip_c2p = 1;
        // the fused learned con2prim forms U from the divergence; the separate
        // guess kernel of the two-kernel form reads a formed U
        p.want_div = h->tun.learned_fused != 0;
    }
    const bool tma = h->tun.tma_tiles != 0;
    // the FMA-contracted FP64 kernels (vb_stage_f64c.cu) for the plain FP64 path
    const bool contract = std::is_same<R, double>::value && h->tun.fp64_contract == 1;
    if (contract && vb_f64c_stage_params_size() != sizeof(StageParams))
        return fail(h, VB_ERR_STATE, "vb_step: FMA-contracted FP64 unit built from another StageParams");
    auto stage = [&](const R* Pin, R* Pout, const double* Us, double* Uo, double dts, double a, double b) -> int {
        for (int d = 0; d < 3; ++d) p.dtdx[d] = d < h->dims ? dts / h->dx[d] : 0.0;
        p.tmap_in = nullptr;
        for (int i = 0; i < 2; ++i)
            if (tma && h->tmap_ok[i] && (const void*)Pin == h->P[i]) p.tmap_in = h->tmap[i];
        p.rk_a = a;
        p.rk_b = b;
        StageBufs<R> bufs{Pin, Pout, h->U0, Us, Uo};
        cudaEvent_t e0 = nullptr, em = nullptr, e1 = nullptr;
        if (h->prof) {
            int rc2 = prof_events(h, &e0, &em, &e1);
            if (rc2) return rc2;
            VB_CUDA(h, cudaEventRecord(e0, s));
        }
        int nk = 0;
        if (h->prof && stage_split_c2p<R>(h->dims, p)) {
            // the same two kernels as launch_stage would launch, with the
            // profiling event between them: the stencil alone, then k_c2p
            StageParams q = p;
            q.skip_c2p = 1;
            q.want_div = 0;
            if (contract)
                VB_CUDA(h, vb_f64c_launch_stage(h->dims, h->opt.recon, h->opt.riemann, &q, &bufs, s, &nk));
            else
                VB_CUDA(h, launch_stage<R>(h->dims, h->opt.recon, h->opt.riemann, q, bufs, s, &nk));
            VB_CUDA(h, cudaEventRecord(em, s));
            if (contract)
                VB_CUDA(h, vb_f64c_launch_c2p(&p, &bufs, s));
            else
                VB_CUDA(h, launch_c2p<R>(p, bufs, s));
            nk = 2;
        } else {
            if (contract)
                VB_CUDA(h, vb_f64c_launch_stage(h->dims, h->opt.recon, h->opt.riemann, &p, &bufs, s, &nk));
            else
                VB_CUDA(h, launch_stage<R>(h->dims, h->opt.recon, h->opt.riemann, p, bufs, s, &nk));
            if (h->prof) VB_CUDA(h, cudaEventRecord(em, s));
        }
        if (p.skip_c2p) {
            // learned guess: the network's W per cell, then the W Newton from it
            StageParams q = p;
            q.skip_c2p = 0;
            q.c2p_mode = C2P_GUESS_W;
            q.div_in_pout = stage_div_in_pout<R>(h->dims, h->opt.recon, h->opt.riemann, p);
            if (h->tun.learned_fused != 0) {
                if (q.c2p_fp32 && h->defer_idx) {
                    // precision-gated: FP32 in the fused kernel, the rest by the FP64 pass
                    q.defer_idx = h->defer_idx;
                    q.defer_n = h->defer_n;
                    q.defer_w0 = h->w_guess;
                    VB_CUDA(h, cudaMemsetAsync(h->defer_n, 0, sizeof(unsigned int), s));
                    VB_CUDA(h, launch_c2p_learned<R>(h->mlp_blob, q, bufs, h->tc_err, s));
                    VB_CUDA(h, launch_c2p_deferred<R>(q, bufs, s));
                    h->launches += 2;
                } else {
                    VB_CUDA(h, launch_c2p_learned<R>(h->mlp_blob, q, bufs, h->tc_err, s));
                    h->launches += 1;
                }
            } else {
                VB_CUDA(h, launch_mlp_guess(h->mlp_blob, p, Uo, h->w_guess, h->tc_err, s));
                q.w_guess = h->w_guess;
                VB_CUDA(h, launch_c2p<R>(q, bufs, s));
                h->launches += 2;
            }
        }
        if (h->prof) VB_CUDA(h, cudaEventRecord(e1, s));
        VB_CUDA(h, launch_ghost_limit<R>(g, Pin, Pout, h->opt.floor_, s));
        h->launches += nk + 1;
        h->stage_launches += 1;
        return VB_OK;
    };
    if (h->opt.rk == 3) {
        // SSP-RK3 (Shu & Osher): U1 = U - dt L(P); U2 = 3/4 U + 1/4 (U1 - dt L(P1));
        // U = 1/3 U + 2/3 (U2 - dt L(P2))
        if ((rc = stage(P[c], P[1 - c], h->U0, h->U1, dt, 0.0, 1.0))) return rc;
        if ((rc = stage(P[1 - c], P[c], h->U1, h->U1, dt, 0.75, 0.25))) return rc;
        if ((rc = stage(P[c], P[1 - c], h->U1, h->U0, dt, 1.0 / 3.0, 2.0 / 3.0))) return rc;
        h->cur = 1 - c;
    } else {
        // midpoint RK2 of the reference: Uhalf = U - dt/2 L(P); U = U - dt L(Phalf)
        if ((rc = stage(P[c], P[1 - c], h->U0, h->U1, dt / 2, 0.0, 1.0))) return rc;
        if ((rc = stage(P[1 - c], P[c], h->U0, h->U0, dt, 0.0, 1.0))) return rc;
    }
    return VB_OK;
}

extern "C" {

int vb_step(vb_handle h, double dt, int nsteps, void* stream) {
    if (!h) return fail(nullptr, VB_ERR_ARG, "null handle");
    if (!h->loaded) return fail(h, VB_ERR_STATE, "vb_step: call vb_load_prims first");
    if (!(dt > 0.0) || nsteps < 0) return fail(h, VB_ERR_ARG, "vb_step: dt %g, nsteps %d", dt, nsteps);
    cudaStream_t s = (cudaStream_t)stream;
    if (h->nghost == 0) {
        VB_CUDA(h, launch_ref1d_steps(h->r1, h->gamma, h->opt.recon, h->opt.n_iter, h->opt.tol, dt, h->dx[0],
                                      nsteps, s));
        h->launches += 1;
        for (int n = 0; n < nsteps; ++n) h->t += dt;
        return VB_OK;
    }
    for (int n = 0; n < nsteps; ++n) {
        int rc = fp32(h) ? step_nd<float>(h, dt, s) : step_nd<double>(h, dt, s);
        if (rc) return rc;
        h->t += dt;
    }
    return VB_OK;
}

int vb_get_time(vb_handle h, double* t) {
    if (!h || !t) return fail(h, VB_ERR_ARG, "vb_get_time: null argument");
    *t = h->t;
    return VB_OK;
}

int vb_set_time(vb_handle h, double t) {
    if (!h) return fail(nullptr, VB_ERR_ARG, "null handle");
    h->t = t;
    return VB_OK;
}

int vb_max_signal_speed(vb_handle h, double* c, void* stream) {
    if (!h || !c) return fail(h, VB_ERR_ARG, "vb_max_signal_speed: null argument");
    if (!h->loaded) return fail(h, VB_ERR_STATE, "vb_max_signal_speed: no state loaded");
    if (h->nghost == 0) return fail(h, VB_ERR_UNSUPPORTED, "vb_max_signal_speed: not provided for the 1D reference layout");
    cudaStream_t s = (cudaStream_t)stream;
    Grid g = grid_of(h);
    if (fp32(h))
        VB_CUDA(h, launch_max_speed<float>(g, (const float*)h->P[h->cur], h->gamma, h->partial, h->max_partial,
                                           h->red_out, s));
    else
        VB_CUDA(h, launch_max_speed<double>(g, (const double*)h->P[h->cur], h->gamma, h->partial,
                                            h->max_partial, h->red_out, s));
    VB_CUDA(h, cudaMemcpyAsync(c, h->red_out, sizeof(double), cudaMemcpyDeviceToHost, s));
    VB_CUDA(h, cudaStreamSynchronize(s));
    return VB_OK;
}

int vb_get_counters(vb_handle h, uint64_t* out, int n, void* stream) {
    if (!h || !out || n < 0) return fail(h, VB_ERR_ARG, "vb_get_counters: bad argument");
    unsigned long long tmp[CNT_N];
    unsigned int tce = 0;
    cudaStream_t s = (cudaStream_t)stream;
    VB_CUDA(h, cudaMemcpyAsync(tmp, h->cnt, sizeof tmp, cudaMemcpyDeviceToHost, s));
    if (h->tc_err) VB_CUDA(h, cudaMemcpyAsync(&tce, h->tc_err, sizeof tce, cudaMemcpyDeviceToHost, s));
    VB_CUDA(h, cudaStreamSynchronize(s));
    tmp[CNT_TIMEOUT] += tce ? 1 : 0;
    for (int i = 0; i < n; ++i) out[i] = i < CNT_N ? tmp[i] : 0;
    return VB_OK;
}

int vb_reset_counters(vb_handle h, void* stream) {
    if (!h) return fail(nullptr, VB_ERR_ARG, "null handle");
    VB_CUDA(h, cudaMemsetAsync(h->cnt, 0, sizeof(unsigned long long) * CNT_N, (cudaStream_t)stream));
    return VB_OK;
}

int vb_profile_enable(vb_handle h, int enable) {
    if (!h) return fail(nullptr, VB_ERR_ARG, "null handle");
    h->prof = enable != 0;
    h->ev_used = 0;
    h->launches = h->stage_launches = 0;
    return VB_OK;
}

int vb_profile_read2(vb_handle h, double* stage_ms, double* stencil_ms, int64_t* stage_launches,
                     int64_t* all_launches) {
    if (!h || !stage_ms || !stencil_ms || !stage_launches || !all_launches)
        return fail(h, VB_ERR_ARG, "vb_profile_read: null argument");
    double tot = 0.0, sten = 0.0;
    if (h->ev_used) VB_CUDA(h, cudaEventSynchronize(h->ev[h->ev_used - 1]));
    for (size_t i = 0; i + 2 < h->ev_used; i += 3) {
        float ms = 0.f, ms1 = 0.f;
        VB_CUDA(h, cudaEventElapsedTime(&ms, h->ev[i], h->ev[i + 2]));
        VB_CUDA(h, cudaEventElapsedTime(&ms1, h->ev[i], h->ev[i + 1]));
        tot += ms;
        sten += ms1;
    }
    *stage_ms = tot;
    *stencil_ms = sten;
    *stage_launches = h->stage_launches;
    *all_launches = h->launches;
    h->ev_used = 0;
    h->launches = h->stage_launches = 0;
    return VB_OK;
}

int vb_profile_read(vb_handle h, double* stage_ms, int64_t* stage_launches, int64_t* all_launches) {
    double sten = 0.0;
    return vb_profile_read2(h, stage_ms, &sten, stage_launches, all_launches);
}

int vb_attach_mlp(vb_handle h, vb_mlp_handle m) {
    if (!h || !m) return fail(h, VB_ERR_ARG, "vb_attach_mlp: null argument");
    if (h->dims != 3 || h->nghost != 3) return fail(h, VB_ERR_UNSUPPORTED, "vb_attach_mlp: 3D grids only");
    if (!h->w_guess) {
        int rc = dev_alloc(h, (void**)&h->w_guess, sizeof(float) * (size_t)h->vs);
        if (rc) return rc;
    }
    if (!h->defer_idx) {
        const size_t cells = (size_t)h->n[0] * h->n[1] * h->n[2];
        int rc = dev_alloc(h, (void**)&h->defer_idx, sizeof(unsigned int) * cells);
        if (!rc) rc = dev_alloc(h, (void**)&h->defer_n, sizeof(unsigned int));
        if (rc) return rc;
    }
    if (!h->tc_err) {
        int rc = dev_alloc(h, (void**)&h->tc_err, sizeof(unsigned int));
        if (rc) return rc;
        VB_CUDA(h, cudaMemset(h->tc_err, 0, sizeof(unsigned int)));
    }
    h->mlp_blob = vb_mlp_blob_ptr(m);
    return VB_OK;
}

int vb_set_tuning(vb_handle h, const vb_tuning* t) {
    if (!h || !t) return fail(h, VB_ERR_ARG, "vb_set_tuning: null argument");
    if (t->split_con2prim < -1 || t->split_con2prim > 1 || t->force_box < 0 || t->force_box > 1 ||
        t->learned_fused < -1 || t->learned_fused > 1 || t->fp32_pairs < -1 || t->fp32_pairs > 1 ||
        t->tma_tiles < -1 || t->tma_tiles > 1 || t->fp64_contract < 0 || t->fp64_contract > 1)
        return fail(h, VB_ERR_ARG,
                    "vb_set_tuning: split_con2prim in {-1,0,1}, force_box and fp64_contract in {0,1}, learned_fused, "
                    "fp32_pairs and tma_tiles in {-1,0,1}");
    h->tun = *t;
    return VB_OK;
}

int vb_get_tuning(vb_handle h, vb_tuning* t) {
    if (!h || !t) return fail(h, VB_ERR_ARG, "vb_get_tuning: null argument");
    *t = h->tun;
    return VB_OK;
}

int vb_tma_tiles_active(vb_handle h, int* active) {
    if (!h || !active) return fail(h, VB_ERR_ARG, "vb_tma_tiles_active: null argument");
    *active = h->tun.tma_tiles != 0 && h->tmap_ok[0] && h->tmap_ok[1] ? 1 : 0;
    return VB_OK;
}

int vb_memory_bytes(vb_handle h, uint64_t* bytes) {
    if (!h || !bytes) return fail(h, VB_ERR_ARG, "vb_memory_bytes: null argument");
    *bytes = h->bytes;
    return VB_OK;
}

int vb_point_recon(int method, const double* q, double* out, int n, void* stream) {
    if (!q || !out || n < 0 || method < 0 || method > 2) return fail(nullptr, VB_ERR_ARG, "vb_point_recon: bad argument");
    VB_CUDA(nullptr, launch_point_recon(method, q, out, n, (cudaStream_t)stream));
    return VB_OK;
}

int vb_point_flux(int dims, int axis, int riemann, double gamma, const double* PL, const double* PR, double* F, int n,
                  void* stream) {
    if (dims < 1 || dims > 3 || axis < 0 || axis >= dims || riemann < 0 || riemann > 1 || !PL || !PR || !F || n < 0)
        return fail(nullptr, VB_ERR_ARG, "vb_point_flux: bad argument");
    VB_CUDA(nullptr, launch_point_flux(dims, axis, riemann, gamma, PL, PR, F, n, (cudaStream_t)stream));
    return VB_OK;
}

int vb_point_con2prim(int dims, double gamma, int n_iter, double tol, const double* U, double* P, int* ret, int n,
                      void* stream) {
    if (dims < 1 || dims > 3 || n_iter < 1 || !U || !P || n < 0)
        return fail(nullptr, VB_ERR_ARG, "vb_point_con2prim: bad argument");
    VB_CUDA(nullptr, launch_point_con2prim(dims, gamma, n_iter, tol, U, P, ret, n, (cudaStream_t)stream));
    return VB_OK;
}

int vb_point_c2p_w(double gamma, const double* U, const double* W0, double rtol, int max_newton, int max_bracket,
                   double* P, int* iters, int* fallback, int n, void* stream) {
    if (!U || !W0 || !P || n < 0 || max_newton < 0 || max_bracket < 0 || !(rtol > 0))
        return fail(nullptr, VB_ERR_ARG, "vb_point_c2p_w: bad argument");
    VB_CUDA(nullptr, launch_point_c2p_w(gamma, U, W0, rtol, max_newton, max_bracket, P, iters, fallback, n,
                                        (cudaStream_t)stream));
    return VB_OK;
}

int vb_point_c2p_gated(double gamma, const double* U, const float* W0, double rtol, int max_newton, int max_bracket,
                       double* P, int* iters, int* fp64, int n, void* stream) {
    if (!U || !W0 || !P || n < 0 || max_newton < 0 || max_bracket < 0 || !(rtol > 0))
        return fail(nullptr, VB_ERR_ARG, "vb_point_c2p_gated: bad argument");
    VB_CUDA(nullptr, launch_point_c2p_gated(gamma, U, W0, rtol, max_newton, max_bracket, P, iters, fp64, n,
                                            (cudaStream_t)stream));
    return VB_OK;
}

}  // extern "C"
