// C ABI of the batch of independent problems (vb_batch_*, include/verona_b200.h).
// No counterpart in the reference, which advances one grid per HARM_HLL call;
// each problem of a batch follows that call's time loop for its dimension
// (src/1dim, src/2dim algos.jl) with the options of the single-grid solver.
//
// Device state: one pool per buffer kind holding every problem back to back
// (problem i at element offset off[i], SoA with stride vs[i] per variable):
//   P[2]  primitive ping-pong pools (FP32 in FP32-bulk precision, else FP64)
//   U[2]  conserved pools, FP64 (U^n and the stage state)
//   done  per-problem completion counters, next: the ticket counter
// vb_batch_step replays a CUDA graph of {reset counters, one persistent
// launch of k_batch over nsteps steps}; graphs are cached per (nsteps, buffer
// parity) and rebuilt when the tile variant changes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <utility>
#include <vector>

#include "../../include/verona_b200.h"
#include "vb_batch.h"

using namespace vb;

struct vb_batch {
    int device = 0;
    vb_options opt{};
    double gamma = 5.0 / 3.0;
    std::vector<vb_batch_problem> probs;
    std::vector<BatchProb> hp;
    std::vector<long long> off;
    std::vector<double> t;
    long long pool = 0;  // elements per pool
    long long cells = 0;
    BatchProb* dprob = nullptr;
    BatchTile* dtiles = nullptr;
    long long T = 0;
    void* P[2] = {nullptr, nullptr};
    double* U[2] = {nullptr, nullptr};
    void* ckP = nullptr;  // checkpoint of P[cur], U[0]
    double* ckU = nullptr;
    int ck_cur = 0;
    std::vector<double> ck_t;
    bool has_ck = false;
    double* dtime = nullptr;    // per problem: its time, on the device (the decay windows of FIXED faces)
    double* ck_time = nullptr;  // checkpoint of dtime
    unsigned long long* done = nullptr;
    unsigned long long* next = nullptr;
    unsigned long long* cnt = nullptr;
    int cur = 0;
    int variant = 0, ctas_per_sm = 0, last_grid = 0;
    unsigned max_polls = 0;  // 0: BATCH_MAX_POLLS
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
    cudaStream_t cap = nullptr;
    size_t bytes = 0;
    std::string err;
    bool fp32() const { return opt.precision == VB_PREC_FP32_BULK; }
    size_t psize() const { return fp32() ? sizeof(float) : sizeof(double); }
};

static thread_local std::string g_berr;

static int bfail(vb_batch_handle b, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (b)
        b->err = buf;
    else
        g_berr = buf;
    return code;
}

#define BCUDA(b, expr)                                                                                   \
    do {                                                                                                 \
        cudaError_t e_ = (expr);                                                                         \
        if (e_ != cudaSuccess) return bfail(b, VB_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));     \
    } while (0)

static int balloc(vb_batch_handle b, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return bfail(b, VB_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    b->bytes += bytes;
    return VB_OK;
}

static void drop_graphs(vb_batch_handle b) {
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
}

static int variants_of(int precision) {
    return precision == VB_PREC_FP32_BULK ? batch_num_variants<float>() : batch_num_variants<double>();
}
static void shape_of(int precision, int v, int* tx2, int* ty2, int* l1) {
    if (precision == VB_PREC_FP32_BULK)
        batch_variant_shape<float>(v, tx2, ty2, l1);
    else
        batch_variant_shape<double>(v, tx2, ty2, l1);
}

// tile counts of the current variant and the stage's ticket order (largest
// problems first, tiles of a problem in row order)
static int build_tiles(vb_batch_handle b) {
    int tx2, ty2, l1;
    shape_of(b->opt.precision, b->variant, &tx2, &ty2, &l1);
    const int np = (int)b->probs.size();
    for (int i = 0; i < np; ++i) {
        const vb_batch_problem& q = b->probs[i];
        BatchProb& h = b->hp[i];
        h.ntx = q.dims == 1 ? (q.nx + l1 - 1) / l1 : (q.nx + tx2 - 1) / tx2;
        h.nty = q.dims == 1 ? 1 : (q.ny + ty2 - 1) / ty2;
        h.ntiles = (long long)h.ntx * h.nty;
    }
    std::vector<int> order(np);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        long long cx = (long long)b->probs[x].nx * b->probs[x].ny, cy = (long long)b->probs[y].nx * b->probs[y].ny;
        return cx > cy;
    });
    std::vector<BatchTile> tiles;
    for (int i : order)
        for (int y = 0; y < b->hp[i].nty; ++y)
            for (int x = 0; x < b->hp[i].ntx; ++x) tiles.push_back(BatchTile{i, x, y, 0});
    b->T = (long long)tiles.size();
    if (b->dtiles) cudaFree(b->dtiles);
    b->dtiles = nullptr;
    int rc = balloc(b, (void**)&b->dtiles, sizeof(BatchTile) * tiles.size());
    if (rc) return rc;
    BCUDA(b, cudaMemcpy(b->dtiles, tiles.data(), sizeof(BatchTile) * tiles.size(), cudaMemcpyHostToDevice));
    BCUDA(b, cudaMemcpy(b->dprob, b->hp.data(), sizeof(BatchProb) * np, cudaMemcpyHostToDevice));
    drop_graphs(b);
    return VB_OK;
}

static Grid grid_of(vb_batch_handle b, int i) {
    const BatchProb& h = b->hp[i];
    Grid g;
    g.dims = h.dims;
    g.nv = 2 + h.dims;
    g.n[0] = h.n0;
    g.n[1] = h.n1;
    g.n[2] = 1;
    g.sy = h.n0;
    g.sz = (long long)h.n0 * h.n1;
    g.vs = h.vs;
    return g;
}

template <typename R> static BatchLaunch<R> launch_desc(vb_batch_handle b, int nsteps, int cur0) {
    BatchLaunch<R> a{};
    a.prob = b->dprob;
    a.tiles = b->dtiles;
    a.T = b->T;
    a.nstages = b->opt.rk == VB_RK3 ? 3 : 2;
    a.total = (long long)nsteps * a.nstages * b->T;
    a.rk = b->opt.rk == VB_RK3 ? 3 : 2;
    a.cur0 = cur0;
    a.P0 = (R*)b->P[0];
    a.P1 = (R*)b->P[1];
    a.U0 = b->U[0];
    a.U1 = b->U[1];
    a.time = b->dtime;
    a.done = b->done;
    a.next = b->next;
    a.counters = b->cnt;
    a.gamma = b->gamma;
    a.floor_ = b->opt.floor_;
    a.tol = b->opt.tol;
    a.n_iter = b->opt.n_iter;
    a.stats = b->opt.stats;
    a.max_polls = b->max_polls ? b->max_polls : BATCH_MAX_POLLS;
    return a;
}

template <typename R> static cudaError_t launch_any(vb_batch_handle b, int nsteps, int cur0, cudaStream_t s, bool go) {
    BatchLaunch<R> a = launch_desc<R>(b, nsteps, cur0);
    return batch_launch<R>(a, b->opt.riemann, b->variant, b->ctas_per_sm, s, &b->last_grid, go);
}

static int graph_for(vb_batch_handle b, int nsteps, int cur0, cudaGraphExec_t* out) {
    auto key = std::make_pair(nsteps, cur0);
    auto it = b->graphs.find(key);
    if (it != b->graphs.end()) {
        *out = it->second;
        return VB_OK;
    }
    // attributes and grid outside the capture
    BCUDA(b, b->fp32() ? launch_any<float>(b, nsteps, cur0, b->cap, false)
                       : launch_any<double>(b, nsteps, cur0, b->cap, false));
    BCUDA(b, cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaMemsetAsync(b->done, 0, sizeof(unsigned long long) * b->probs.size(), b->cap);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->next, 0, sizeof(unsigned long long), b->cap);
    if (e == cudaSuccess)
        e = b->fp32() ? launch_any<float>(b, nsteps, cur0, b->cap, true)
                      : launch_any<double>(b, nsteps, cur0, b->cap, true);
    if (e == cudaSuccess) e = batch_advance_time(b->dprob, b->dtime, (int)b->probs.size(), nsteps, b->cap);
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(b->cap, &graph);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return bfail(b, VB_ERR_CUDA, "vb_batch_step: graph capture: %s",
                     cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return bfail(b, VB_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    b->graphs[key] = exec;
    *out = exec;
    return VB_OK;
}

extern "C" {

const char* vb_batch_last_error(vb_batch_handle b) { return b ? b->err.c_str() : g_berr.c_str(); }

int vb_batch_destroy(vb_batch_handle b) {
    if (!b) return VB_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    drop_graphs(b);
    if (b->cap) cudaStreamDestroy(b->cap);
    cudaFree(b->P[0]);
    cudaFree(b->P[1]);
    cudaFree(b->U[0]);
    cudaFree(b->U[1]);
    cudaFree(b->ckP);
    cudaFree(b->ckU);
    cudaFree(b->dprob);
    cudaFree(b->dtiles);
    cudaFree(b->dtime);
    cudaFree(b->ck_time);
    cudaFree(b->done);
    cudaFree(b->next);
    cudaFree(b->cnt);
    cudaSetDevice(prev);
    delete b;
    return VB_OK;
}

int vb_batch_create(vb_batch_handle* out, int nprob, const vb_batch_problem* probs, double gamma,
                    const vb_options* o) {
    if (!out || !probs || nprob < 1) return bfail(nullptr, VB_ERR_ARG, "vb_batch_create: no problems");
    *out = nullptr;
    vb_options opt;
    vb_default_options(&opt);
    if (o) {
        if (o->version != VB_ABI_VERSION)
            return bfail(nullptr, VB_ERR_ARG, "vb_batch_create: options version %d, expected %d", o->version,
                         VB_ABI_VERSION);
        opt = *o;
    }
    if (!(gamma > 1.0)) return bfail(nullptr, VB_ERR_ARG, "vb_batch_create: gamma %g must exceed 1", gamma);
    if (opt.riemann != VB_RIEMANN_HLL && opt.riemann != VB_RIEMANN_HLLC)
        return bfail(nullptr, VB_ERR_ARG, "vb_batch_create: riemann %d", opt.riemann);
    if (opt.rk != VB_RK2 && opt.rk != VB_RK3) return bfail(nullptr, VB_ERR_ARG, "vb_batch_create: rk %d", opt.rk);
    if (opt.precision != VB_PREC_FP64 && opt.precision != VB_PREC_FP32_BULK)
        return bfail(nullptr, VB_ERR_ARG, "vb_batch_create: precision %d", opt.precision);
    if (opt.guess != VB_GUESS_PREVIOUS)
        return bfail(nullptr, VB_ERR_UNSUPPORTED, "vb_batch_create: batches use the previous-state guess");
    for (int i = 0; i < nprob; ++i) {
        const vb_batch_problem& q = probs[i];
        if (q.dims != 1 && q.dims != 2) return bfail(nullptr, VB_ERR_ARG, "problem %d: dims %d (1 or 2)", i, q.dims);
        if (q.nx < 1 || (q.dims == 2 && q.ny < 1) || (q.dims == 1 && q.ny != 1))
            return bfail(nullptr, VB_ERR_ARG, "problem %d: size %d x %d", i, q.nx, q.ny);
        if (q.recon < VB_RECON_MINMOD || q.recon > VB_RECON_WENOZ)
            return bfail(nullptr, VB_ERR_ARG, "problem %d: recon %d", i, q.recon);
        if (!(q.dx > 0.0) || (q.dims == 2 && !(q.dy > 0.0)) || !(q.dt > 0.0))
            return bfail(nullptr, VB_ERR_ARG, "problem %d: dx %g dy %g dt %g", i, q.dx, q.dy, q.dt);
    }
    vb_batch_handle b = new vb_batch();
    cudaGetDevice(&b->device);
    b->opt = opt;
    b->gamma = gamma;
    b->probs.assign(probs, probs + nprob);
    b->hp.resize(nprob);
    b->off.resize(nprob);
    b->t.assign(nprob, 0.0);
    long long off = 0;
    for (int i = 0; i < nprob; ++i) {
        const vb_batch_problem& q = probs[i];
        BatchProb& h = b->hp[i];
        memset(&h, 0, sizeof h);
        h.dims = q.dims;
        h.rec = q.recon;
        h.n0 = q.nx + 2 * NG;
        h.n1 = q.dims == 2 ? q.ny + 2 * NG : 1;
        h.vs = ((long long)h.n0 * h.n1 + 31) / 32 * 32;
        h.offP = h.offU = off;
        b->off[i] = off;
        off += (long long)(2 + q.dims) * h.vs;
        // dt / dx and (dt / 2) / dx, as the single-grid stage computes them
        const double dth = q.dt / 2;
        h.dtdx[0][0] = q.dt / q.dx;
        h.dtdx[1][0] = dth / q.dx;
        h.dtdx[0][1] = q.dims == 2 ? q.dt / q.dy : 0.0;
        h.dtdx[1][1] = q.dims == 2 ? dth / q.dy : 0.0;
        h.dt = q.dt;  // every face outflow (bc_kind 0) until vb_batch_set_boundary
        b->cells += (long long)q.nx * q.ny;
    }
    b->pool = off;
    int rc = 0;
    const size_t pb = b->psize() * (size_t)off, ub = sizeof(double) * (size_t)off;
    if ((rc = balloc(b, &b->P[0], pb)) || (rc = balloc(b, &b->P[1], pb)) || (rc = balloc(b, (void**)&b->U[0], ub)) ||
        (rc = balloc(b, (void**)&b->U[1], ub)) || (rc = balloc(b, (void**)&b->dprob, sizeof(BatchProb) * nprob)) ||
        (rc = balloc(b, (void**)&b->done, sizeof(unsigned long long) * nprob)) ||
        (rc = balloc(b, (void**)&b->dtime, sizeof(double) * nprob)) ||
        (rc = balloc(b, (void**)&b->next, sizeof(unsigned long long))) ||
        (rc = balloc(b, (void**)&b->cnt, sizeof(unsigned long long) * CNT_N))) {
        g_berr = b->err;
        vb_batch_destroy(b);
        return rc;
    }
    cudaError_t e = cudaMemset(b->P[0], 0, pb);
    if (e == cudaSuccess) e = cudaMemset(b->P[1], 0, pb);
    if (e == cudaSuccess) e = cudaMemset(b->U[0], 0, ub);
    if (e == cudaSuccess) e = cudaMemset(b->U[1], 0, ub);
    if (e == cudaSuccess) e = cudaMemset(b->cnt, 0, sizeof(unsigned long long) * CNT_N);
    if (e == cudaSuccess) e = cudaMemset(b->dtime, 0, sizeof(double) * nprob);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        g_berr = std::string("vb_batch_create: ") + cudaGetErrorString(e);
        vb_batch_destroy(b);
        return VB_ERR_CUDA;
    }
    if ((rc = build_tiles(b))) {
        g_berr = b->err;
        vb_batch_destroy(b);
        return rc;
    }
    *out = b;
    return VB_OK;
}

int vb_batch_load_prims(vb_batch_handle b, int i, const double* P_aos, void* stream) {
    if (!b || !P_aos) return bfail(b, VB_ERR_ARG, "vb_batch_load_prims: null argument");
    if (i < 0 || i >= (int)b->probs.size()) return bfail(b, VB_ERR_ARG, "vb_batch_load_prims: problem %d", i);
    cudaStream_t s = (cudaStream_t)stream;
    Grid g = grid_of(b, i);
    if (b->fp32())
        BCUDA(b, launch_load_prims<float>(g, P_aos, (float*)b->P[b->cur] + b->off[i], b->U[0] + b->off[i], b->gamma, s));
    else
        BCUDA(b, launch_load_prims<double>(g, P_aos, (double*)b->P[b->cur] + b->off[i], b->U[0] + b->off[i], b->gamma,
                                           s));
    b->t[i] = 0.0;
    BCUDA(b, cudaMemsetAsync(b->dtime + i, 0, sizeof(double), s));
    return VB_OK;
}

int vb_batch_store_prims(vb_batch_handle b, int i, double* P_aos, void* stream) {
    if (!b || !P_aos) return bfail(b, VB_ERR_ARG, "vb_batch_store_prims: null argument");
    if (i < 0 || i >= (int)b->probs.size()) return bfail(b, VB_ERR_ARG, "vb_batch_store_prims: problem %d", i);
    cudaStream_t s = (cudaStream_t)stream;
    Grid g = grid_of(b, i);
    if (b->fp32())
        BCUDA(b, launch_store_prims<float>(g, (const float*)b->P[b->cur] + b->off[i], P_aos, s));
    else
        BCUDA(b, launch_store_prims<double>(g, (const double*)b->P[b->cur] + b->off[i], P_aos, s));
    return VB_OK;
}

int vb_batch_step(vb_batch_handle b, int nsteps, void* stream) {
    if (!b) return bfail(nullptr, VB_ERR_ARG, "null batch");
    if (nsteps < 0) return bfail(b, VB_ERR_ARG, "vb_batch_step: nsteps %d", nsteps);
    if (nsteps == 0) return VB_OK;
    cudaGraphExec_t g = nullptr;
    int rc = graph_for(b, nsteps, b->cur, &g);
    if (rc) return rc;
    BCUDA(b, cudaGraphLaunch(g, (cudaStream_t)stream));
    if (b->opt.rk == VB_RK3 && (nsteps & 1)) b->cur ^= 1;
    // t += dt once per step, as the single-grid solver and the device time advance it
    for (size_t i = 0; i < b->probs.size(); ++i)
        for (int k = 0; k < nsteps; ++k) b->t[i] += b->probs[i].dt;
    return VB_OK;
}

int vb_batch_get_time(vb_batch_handle b, int i, double* t) {
    if (!b || !t || i < 0 || i >= (int)b->probs.size()) return bfail(b, VB_ERR_ARG, "vb_batch_get_time: argument");
    *t = b->t[i];
    return VB_OK;
}

int vb_batch_set_boundary(vb_batch_handle b, int i, int face, int kind, const double* par, int np) {
    if (!b) return bfail(nullptr, VB_ERR_ARG, "null batch");
    if (i < 0 || i >= (int)b->probs.size()) return bfail(b, VB_ERR_ARG, "vb_batch_set_boundary: problem %d", i);
    const int dims = b->probs[i].dims, nv = 2 + dims;
    if (face < 0 || face >= 2 * dims)
        return bfail(b, VB_ERR_ARG, "vb_batch_set_boundary: face %d for dims %d", face, dims);
    if (kind < 0 || kind > 2) return bfail(b, VB_ERR_ARG, "vb_batch_set_boundary: kind %d", kind);
    if (np < 0 || np > 8 || (np > 0 && !par)) return bfail(b, VB_ERR_ARG, "vb_batch_set_boundary: %d params", np);
    if (kind == VB_BC_FIXED && np > 0 && np < 4)
        return bfail(b, VB_ERR_ARG, "vb_batch_set_boundary: FIXED decay needs {var, t_on, t_off, factor}");
    if (kind == VB_BC_FIXED && np >= 4 && (par[0] < 0 || par[0] >= nv))
        return bfail(b, VB_ERR_ARG, "vb_batch_set_boundary: decay variable %g", par[0]);
    if (kind == VB_BC_NOZZLE && np < 5 + dims)
        return bfail(b, VB_ERR_ARG, "vb_batch_set_boundary: NOZZLE needs {radius, c1, c2, rho, u, u1..u%d}", dims);
    BatchProb& h = b->hp[i];
    h.bc_kind[face] = kind;
    for (int k = 0; k < 8; ++k) h.bc_par[face][k] = k < np ? par[k] : 0.0;
    if (kind == VB_BC_FIXED && np == 0) h.bc_par[face][0] = -1.0;  // no decay
    // the descriptor is read by launches already queued: replace it in order
    BCUDA(b, cudaDeviceSynchronize());
    BCUDA(b, cudaMemcpy(b->dprob + i, &h, sizeof(BatchProb), cudaMemcpyHostToDevice));
    return VB_OK;
}

int vb_batch_set_wait_limit(vb_batch_handle b, uint32_t max_polls) {
    if (!b) return bfail(nullptr, VB_ERR_ARG, "null batch");
    if (max_polls == b->max_polls) return VB_OK;
    b->max_polls = max_polls;
    drop_graphs(b);  // the limit is a kernel argument baked into the cached graphs
    return VB_OK;
}

int vb_batch_check(vb_batch_handle b, void* stream) {
    if (!b) return bfail(nullptr, VB_ERR_ARG, "null batch");
    unsigned long long h[CNT_N];
    BCUDA(b, cudaMemcpyAsync(h, b->cnt, sizeof h, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    BCUDA(b, cudaStreamSynchronize((cudaStream_t)stream));
    if (h[CNT_TIMEOUT])
        return bfail(b, VB_ERR_TIMEOUT,
                     "vb_batch_check: %llu bounded waits of the batch kernel gave up; the state of the batch is "
                     "undefined (vb_batch_rollback or reload it)",
                     h[CNT_TIMEOUT]);
    if (h[CNT_BAD_INDEX])
        return bfail(b, VB_ERR_STATE, "vb_batch_check: %llu work items out of range were skipped", h[CNT_BAD_INDEX]);
    return VB_OK;
}

int vb_batch_get_counters(vb_batch_handle b, uint64_t* out, void* stream) {
    if (!b || !out) return bfail(b, VB_ERR_ARG, "vb_batch_get_counters: null argument");
    unsigned long long h[CNT_N];
    BCUDA(b, cudaMemcpyAsync(h, b->cnt, sizeof h, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    BCUDA(b, cudaStreamSynchronize((cudaStream_t)stream));
    for (int i = 0; i < VB_CNT_N; ++i) out[i] = h[i];
    return VB_OK;
}

int vb_batch_reset_counters(vb_batch_handle b, void* stream) {
    if (!b) return bfail(nullptr, VB_ERR_ARG, "null batch");
    BCUDA(b, cudaMemsetAsync(b->cnt, 0, sizeof(unsigned long long) * CNT_N, (cudaStream_t)stream));
    return VB_OK;
}

int vb_batch_num_variants(int precision) {
    if (precision != VB_PREC_FP64 && precision != VB_PREC_FP32_BULK) return 0;
    return variants_of(precision);
}

int vb_batch_variant_shape(int precision, int variant, int* tile_x2, int* tile_y2, int* pencil1) {
    if (!tile_x2 || !tile_y2 || !pencil1 || variant < 0 || variant >= vb_batch_num_variants(precision))
        return bfail(nullptr, VB_ERR_ARG, "vb_batch_variant_shape: precision %d variant %d", precision, variant);
    shape_of(precision, variant, tile_x2, tile_y2, pencil1);
    return VB_OK;
}

int vb_batch_set_tuning(vb_batch_handle b, int variant, int ctas_per_sm) {
    if (!b) return bfail(nullptr, VB_ERR_ARG, "null batch");
    if (variant < 0 || variant >= variants_of(b->opt.precision) || ctas_per_sm < 0 || ctas_per_sm > 32)
        return bfail(b, VB_ERR_ARG, "vb_batch_set_tuning: variant %d, CTAs per SM %d", variant, ctas_per_sm);
    if (variant == b->variant && ctas_per_sm == b->ctas_per_sm) return VB_OK;
    b->variant = variant;
    b->ctas_per_sm = ctas_per_sm;
    return build_tiles(b);
}

int vb_batch_get_tuning(vb_batch_handle b, int* variant, int* ctas_per_sm, int* grid) {
    if (!b || !variant || !ctas_per_sm || !grid) return bfail(b, VB_ERR_ARG, "vb_batch_get_tuning: null argument");
    *variant = b->variant;
    *ctas_per_sm = b->ctas_per_sm;
    *grid = b->last_grid;
    return VB_OK;
}

int vb_batch_info(vb_batch_handle b, int64_t* interior_cells, int64_t* tiles_per_stage, int64_t* bytes) {
    if (!b || !interior_cells || !tiles_per_stage || !bytes) return bfail(b, VB_ERR_ARG, "vb_batch_info: null argument");
    *interior_cells = b->cells;
    *tiles_per_stage = b->T;
    *bytes = (int64_t)b->bytes;
    return VB_OK;
}

int vb_batch_checkpoint(vb_batch_handle b, void* stream) {
    if (!b) return bfail(nullptr, VB_ERR_ARG, "null batch");
    const size_t pb = b->psize() * (size_t)b->pool, ub = sizeof(double) * (size_t)b->pool;
    const size_t tb = sizeof(double) * b->probs.size();
    if (!b->ckP) {
        int rc = balloc(b, &b->ckP, pb);
        if (!rc) rc = balloc(b, (void**)&b->ckU, ub);
        if (!rc) rc = balloc(b, (void**)&b->ck_time, tb);
        if (rc) return rc;
    }
    cudaStream_t s = (cudaStream_t)stream;
    BCUDA(b, cudaMemcpyAsync(b->ckP, b->P[b->cur], pb, cudaMemcpyDeviceToDevice, s));
    BCUDA(b, cudaMemcpyAsync(b->ckU, b->U[0], ub, cudaMemcpyDeviceToDevice, s));
    BCUDA(b, cudaMemcpyAsync(b->ck_time, b->dtime, tb, cudaMemcpyDeviceToDevice, s));
    b->ck_cur = b->cur;
    b->ck_t = b->t;
    b->has_ck = true;
    return VB_OK;
}

int vb_batch_rollback(vb_batch_handle b, void* stream) {
    if (!b) return bfail(nullptr, VB_ERR_ARG, "null batch");
    if (!b->has_ck) return bfail(b, VB_ERR_STATE, "vb_batch_rollback: no checkpoint");
    const size_t pb = b->psize() * (size_t)b->pool, ub = sizeof(double) * (size_t)b->pool;
    cudaStream_t s = (cudaStream_t)stream;
    b->cur = b->ck_cur;
    BCUDA(b, cudaMemcpyAsync(b->P[b->cur], b->ckP, pb, cudaMemcpyDeviceToDevice, s));
    BCUDA(b, cudaMemcpyAsync(b->U[0], b->ckU, ub, cudaMemcpyDeviceToDevice, s));
    BCUDA(b, cudaMemcpyAsync(b->dtime, b->ck_time, sizeof(double) * b->probs.size(), cudaMemcpyDeviceToDevice, s));
    b->t = b->ck_t;
    return VB_OK;
}

}  // extern "C"
