// Learned con2prim initial guess: a 4 -> 64 -> 64 -> 64 -> 1 ReLU MLP in
// BF16 on the sm_100a tensor cores (tcgen05, FP32 accumulation in TMEM).
//
// Inputs per cell (the conserved state only), with E = tau + D = -U2 the
// total energy: f = (log D, |S|/E, log(E/D), Gamma_eos), normalised by the
// training-set mean and standard deviation. The network predicts
// x = p / E (in [0, Gamma - 1) for physical states); the pressure guess is
// p0 = E max(y, 0) and the Newton start W0 = E + p0 = E (1 + max(y, 0))
// (U2 = T^t_t = p - W). Training minimises ((y - x) / (1 + x))^2, the squared
// relative error of W0. (log p itself is ill-conditioned in U for cold
// relativistic flows, where p sits below the precision of E.) Newton on W
// then refines the guess to the requested relative tolerance, with a
// bracketed fallback (vb_con2prim.cuh, c2p_w).
//
// Kernels
//   k_mlp_pack      FP32 master parameters -> BF16 operand blobs in the
//                   tensor-core layout (forward W^T and backward W copies)
//   k_mlp_features  conserved states -> normalised features and targets
//   k_mlp_forward   features -> y, 128 cells per tile (inference only)
//   k_mlp_guess     split-stage guess: U -> features -> MLP -> W0 per cell;
//                   the stage's con2prim kernel then runs the W Newton from it
//
// Inference folds every bias into its MMA: the activation operand carries two
// constant columns of ones and the weight operand the bias split into a BF16
// high part and a BF16 remainder (bias error ~2^-17 relative), so an epilogue
// is one TMEM load, ReLU + BF16 packing in one cvt per pair, and the shared
// stores of the next operand.
//   k_mlp_train     forward + backward of 128-sample tiles; every GEMM
//                   (three forward layers, two backward input-gradients and
//                   all weight/bias gradients) runs as tcgen05.mma; weight
//                   gradients accumulate in TMEM across a CTA's tiles
//   k_mlp_adam      Adam update of the FP32 master parameters
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/verona_b200.h"
#include "vb_con2prim.cuh"
#include "vb_index.cuh"
#include "vb_internal.h"
#include "vb_tc.cuh"

namespace vb {

constexpr int MLP_IN = 4, MLP_H = 64, MLP_KIN = 16;  // layer-1 K padded to one MMA
constexpr int MLP_KH = MLP_H + 16;                   // inference K of layers 2, 3: 64 + bias columns
constexpr int TILE = 128;                            // cells per tile = MMA M
constexpr uint32_t MAX_POLLS = 1u << 26;             // bounded mbarrier waits
// FP32 master parameter vector: W1[4][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + MLP_IN * MLP_H, OFF_W2 = OFF_B1 + MLP_H, OFF_B2 = OFF_W2 + MLP_H * MLP_H,
              OFF_W3 = OFF_B2 + MLP_H, OFF_B3 = OFF_W3 + MLP_H * MLP_H, OFF_W4 = OFF_B3 + MLP_H, OFF_B4 = OFF_W4 + MLP_H,
              N_PARAMS = OFF_B4 + 1;

// device blob: BF16 operands in the K-major core-matrix layout, then FP32 vectors
struct MlpBlob {
    __nv_bfloat16 w1t[MLP_H * MLP_KIN];  // B of layer 1: rows = out (64), K = in (16, padded)
    __nv_bfloat16 w2t[MLP_H * MLP_H];    // B of layer 2: rows = out, K = in
    __nv_bfloat16 w3t[MLP_H * MLP_H];    // B of layer 3
    __nv_bfloat16 w2n[MLP_H * MLP_H];    // B of dh1 = dz2 W2^T: rows = in, K = out
    __nv_bfloat16 w3n[MLP_H * MLP_H];    // B of dh2 = dz3 W3^T
    __nv_bfloat16 w1i[MLP_H * MLP_KIN];  // inference B of layer 1: W1^T, b1 high, b1 remainder in K 4, 5
    __nv_bfloat16 w2i[MLP_H * MLP_KH];   // inference B of layer 2: W2^T, b2 high, b2 remainder in K 64, 65
    __nv_bfloat16 w3i[MLP_H * MLP_KH];   // inference B of layer 3
    float b1[MLP_H], b2[MLP_H], b3[MLP_H], w4[MLP_H];
    float b4;
    float mu[MLP_IN], isd[MLP_IN];
};

// bounded mbarrier wait whose outcome every thread of the CTA agrees on (a
// barrier is reached by all threads either way)
__device__ __forceinline__ bool cta_wait(uint64_t* mbar, uint32_t parity, unsigned int* err) {
    const bool ok = tc::mbar_wait(mbar, parity, err, MAX_POLLS);
    return !__syncthreads_or(!ok);
}

__device__ __forceinline__ float relu(float z) { return fmaxf(z, 0.0f); }
__device__ __forceinline__ float drelu(float z) { return z > 0.0f ? 1.0f : 0.0f; }

// ---- features -------------------------------------------------------------------
__device__ __forceinline__ void cell_features(const double* U, double gamma, const float* mu, const float* isd,
                                              float* f, double* logD) {
    const double D = U[0];
    const double S = sqrt(U[2] * U[2] + U[3] * U[3] + U[4] * U[4]);
    const double E = -U[1];
    const double ld = log(fmax(D, 1e-300));
    *logD = ld;
    float raw[4] = {(float)ld, (float)(S / E), (float)log(fmax(E / D, 1e-300)), (float)gamma};
#pragma unroll
    for (int i = 0; i < 4; ++i) f[i] = (raw[i] - mu[i]) * isd[i];
}

__global__ void k_mlp_pack(const float* __restrict__ prm, const float* __restrict__ norm, MlpBlob* __restrict__ blob) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    char* base = reinterpret_cast<char*>(blob);
    for (int e = t; e < MLP_H * MLP_KIN; e += stride) {  // w1t[o][i]
        int o = e / MLP_KIN, i = e % MLP_KIN;
        float w = i < MLP_IN ? prm[OFF_W1 + i * MLP_H + o] : 0.0f;
        *reinterpret_cast<__nv_bfloat16*>(base + offsetof(MlpBlob, w1t) + tc::kmajor_off(MLP_H, o, i)) =
            __float2bfloat16(w);
    }
    for (int e = t; e < MLP_H * MLP_H; e += stride) {
        int a = e / MLP_H, c = e % MLP_H;  // W[in=a][out=c]
        float w2 = prm[OFF_W2 + a * MLP_H + c], w3 = prm[OFF_W3 + a * MLP_H + c];
        *reinterpret_cast<__nv_bfloat16*>(base + offsetof(MlpBlob, w2t) + tc::kmajor_off(MLP_H, c, a)) =
            __float2bfloat16(w2);
        *reinterpret_cast<__nv_bfloat16*>(base + offsetof(MlpBlob, w3t) + tc::kmajor_off(MLP_H, c, a)) =
            __float2bfloat16(w3);
        *reinterpret_cast<__nv_bfloat16*>(base + offsetof(MlpBlob, w2n) + tc::kmajor_off(MLP_H, a, c)) =
            __float2bfloat16(w2);
        *reinterpret_cast<__nv_bfloat16*>(base + offsetof(MlpBlob, w3n) + tc::kmajor_off(MLP_H, a, c)) =
            __float2bfloat16(w3);
    }
    // inference operands with the biases as two extra K columns (high + remainder)
    auto put = [&](size_t off, int R, int row, int k, float v) {
        *reinterpret_cast<__nv_bfloat16*>(base + off + tc::kmajor_off(R, row, k)) = __float2bfloat16(v);
    };
    auto hi = [](float b) { return __bfloat162float(__float2bfloat16(b)); };
    for (int e = t; e < MLP_H * MLP_KIN; e += stride) {
        int o = e / MLP_KIN, i = e % MLP_KIN;
        float b = prm[OFF_B1 + o];
        float w = i < MLP_IN ? prm[OFF_W1 + i * MLP_H + o] : (i == MLP_IN ? hi(b) : (i == MLP_IN + 1 ? b - hi(b) : 0.0f));
        put(offsetof(MlpBlob, w1i), MLP_H, o, i, w);
    }
    for (int e = t; e < MLP_H * MLP_KH; e += stride) {
        int o = e / MLP_KH, a = e % MLP_KH;  // row = out o, K = in a
        float b2 = prm[OFF_B2 + o], b3 = prm[OFF_B3 + o];
        float w2 = a < MLP_H ? prm[OFF_W2 + a * MLP_H + o] : (a == MLP_H ? hi(b2) : (a == MLP_H + 1 ? b2 - hi(b2) : 0.0f));
        float w3 = a < MLP_H ? prm[OFF_W3 + a * MLP_H + o] : (a == MLP_H ? hi(b3) : (a == MLP_H + 1 ? b3 - hi(b3) : 0.0f));
        put(offsetof(MlpBlob, w2i), MLP_H, o, a, w2);
        put(offsetof(MlpBlob, w3i), MLP_H, o, a, w3);
    }
    for (int e = t; e < MLP_H; e += stride) {
        blob->b1[e] = prm[OFF_B1 + e];
        blob->b2[e] = prm[OFF_B2 + e];
        blob->b3[e] = prm[OFF_B3 + e];
        blob->w4[e] = prm[OFF_W4 + e];
    }
    if (t == 0) {
        blob->b4 = prm[OFF_B4];
        for (int i = 0; i < MLP_IN; ++i) {
            blob->mu[i] = norm[i];
            blob->isd[i] = norm[MLP_IN + i];
        }
    }
}

// features, targets x = p / E and loss weights 1 / (1 + x)^2 (so the
// weighted squared error is that of W0 relative to W) of n states
// (U, P: 5 x n SoA FP64)
__global__ void k_mlp_features(const double* __restrict__ U, const double* __restrict__ P, int n, double gamma,
                               const float* __restrict__ norm, float* __restrict__ feat, float* __restrict__ target,
                               float* __restrict__ weight) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double u[5];
        for (int v = 0; v < 5; ++v) u[v] = U[v * (long long)n + i];
        float f[4];
        double ld;
        cell_features(u, gamma, norm, norm + MLP_IN, f, &ld);
        for (int k = 0; k < 4; ++k) feat[i * 4 + k] = f[k];
        if (P && target) {
            const double p = (gamma - 1.0) * P[1 * (long long)n + i];
            const double x = p / (-u[1]);
            target[i] = (float)x;
            if (weight) weight[i] = (float)(1.0 / ((1.0 + x) * (1.0 + x)));
        }
    }
}

// ---- shared memory of the inference path -------------------------------------------------
// The layer-1 operand a1 [cells x 16] (4 features, 1, 1, zeros) occupies the
// first two K chunks of h: the layer-1 MMA has completed before h1 is written.
struct InferSmem {
    __nv_bfloat16 h[TILE * MLP_KH];  // a1, then h1, then h2 [cells x 80]: 64 activations, 1, 1, zeros
    __nv_bfloat16 w1i[MLP_H * MLP_KIN];
    __nv_bfloat16 w2i[MLP_H * MLP_KH];
    __nv_bfloat16 w3i[MLP_H * MLP_KH];
    float w4[MLP_H];
    float b4, mu[MLP_IN], isd[MLP_IN];
    uint64_t mbar;
    uint32_t tmem_base;
};

__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
    __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&p);
}
// max(lo, 0), max(hi, 0) rounded to BF16 and packed (lo in the low half)
__device__ __forceinline__ uint32_t relu_bf16x2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// Weights into shared memory, and the constant columns of the activation
// operand h (K 64, 65 = 1 multiply the bias columns of w2i / w3i; 66..79 = 0).
__device__ void load_weights_infer(InferSmem& s, const MlpBlob* __restrict__ blob) {
    const int t = threadIdx.x, nt = blockDim.x;
    auto cp = [&](void* dst, const void* src, size_t bytes) {
        const uint4* x = reinterpret_cast<const uint4*>(src);
        uint4* y = reinterpret_cast<uint4*>(dst);
        for (int i = t; i < (int)(bytes / 16); i += nt) y[i] = x[i];
    };
    cp(s.w1i, blob->w1i, sizeof(s.w1i));
    cp(s.w2i, blob->w2i, sizeof(s.w2i));
    cp(s.w3i, blob->w3i, sizeof(s.w3i));
    for (int i = t; i < MLP_H; i += nt) s.w4[i] = blob->w4[i];
    if (t == 0) {
        s.b4 = blob->b4;
        for (int i = 0; i < MLP_IN; ++i) {
            s.mu[i] = blob->mu[i];
            s.isd[i] = blob->isd[i];
        }
    }
    char* hb = reinterpret_cast<char*>(s.h);
    for (int r = t; r < TILE; r += nt) {
        *reinterpret_cast<uint4*>(hb + tc::kmajor_off(TILE, r, MLP_H)) = make_uint4(bf16x2(1.0f, 1.0f), 0u, 0u, 0u);
        *reinterpret_cast<uint4*>(hb + tc::kmajor_off(TILE, r, MLP_H + 8)) = make_uint4(0u, 0u, 0u, 0u);
    }
}

// store one row (this thread's cell) of a K-major [TILE x 64] BF16 operand
__device__ __forceinline__ void store_row64(__nv_bfloat16* buf, int row, const float* v) {
    char* b = reinterpret_cast<char*>(buf);
#pragma unroll
    for (int c = 0; c < 8; ++c) {  // 8 K chunks of 8 values = 16 bytes each
        __nv_bfloat162 p0 = __floats2bfloat162_rn(v[8 * c + 0], v[8 * c + 1]);
        __nv_bfloat162 p1 = __floats2bfloat162_rn(v[8 * c + 2], v[8 * c + 3]);
        __nv_bfloat162 p2 = __floats2bfloat162_rn(v[8 * c + 4], v[8 * c + 5]);
        __nv_bfloat162 p3 = __floats2bfloat162_rn(v[8 * c + 6], v[8 * c + 7]);
        uint4 q;
        q.x = *reinterpret_cast<uint32_t*>(&p0);
        q.y = *reinterpret_cast<uint32_t*>(&p1);
        q.z = *reinterpret_cast<uint32_t*>(&p2);
        q.w = *reinterpret_cast<uint32_t*>(&p3);
        *reinterpret_cast<uint4*>(b + tc::kmajor_off(TILE, row, 8 * c)) = q;
    }
}

__device__ __forceinline__ void store_row16(__nv_bfloat16* buf, int row, const float* f4) {
    char* b = reinterpret_cast<char*>(buf);
    __nv_bfloat162 p0 = __floats2bfloat162_rn(f4[0], f4[1]);
    __nv_bfloat162 p1 = __floats2bfloat162_rn(f4[2], f4[3]);
    uint4 q;
    q.x = *reinterpret_cast<uint32_t*>(&p0);
    q.y = *reinterpret_cast<uint32_t*>(&p1);
    q.z = 0u;
    q.w = 0u;
    *reinterpret_cast<uint4*>(b + tc::kmajor_off(TILE, row, 0)) = q;
    *reinterpret_cast<uint4*>(b + tc::kmajor_off(TILE, row, 8)) = make_uint4(0u, 0u, 0u, 0u);
}

// ReLU of 32 FP32 accumulators (columns 32 * half ..), as BF16, into row `row`
// of the K-major [TILE x 80] activation operand
__device__ __forceinline__ void store_row32_relu(__nv_bfloat16* buf, int row, const float* v, int half) {
    char* b = reinterpret_cast<char*>(buf);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        uint4 q;
        q.x = relu_bf16x2(v[8 * c + 0], v[8 * c + 1]);
        q.y = relu_bf16x2(v[8 * c + 2], v[8 * c + 3]);
        q.z = relu_bf16x2(v[8 * c + 4], v[8 * c + 5]);
        q.w = relu_bf16x2(v[8 * c + 6], v[8 * c + 7]);
        *reinterpret_cast<uint4*>(b + tc::kmajor_off(TILE, row, 32 * half + 8 * c)) = q;
    }
}

// ReLU of 64 FP32 accumulators, as BF16, into row `row` (K 0..63) of the
// K-major [TILE x 80] activation operand
__device__ __forceinline__ void store_row64_relu(__nv_bfloat16* buf, int row, const float* v) {
    char* b = reinterpret_cast<char*>(buf);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        uint4 q;
        q.x = relu_bf16x2(v[8 * c + 0], v[8 * c + 1]);
        q.y = relu_bf16x2(v[8 * c + 2], v[8 * c + 3]);
        q.z = relu_bf16x2(v[8 * c + 4], v[8 * c + 5]);
        q.w = relu_bf16x2(v[8 * c + 6], v[8 * c + 7]);
        *reinterpret_cast<uint4*>(b + tc::kmajor_off(TILE, row, 8 * c)) = q;
    }
}

// One MLP forward for the CTA's 128 cells (thread t = cell / row t). f: this
// thread's 4 normalised features; returns y, the predicted p / E. The caller
// holds TMEM (64 columns at s.tmem_base) and the mbarrier; `phase` counts
// completed commits. Returns false if a bounded wait ran out.
__device__ bool mlp_forward_tile(InferSmem& s, const float* f, float& y, uint32_t& phase, unsigned int* err) {
    const int t = threadIdx.x, warp = t >> 5;
    const uint32_t tmem = s.tmem_base;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    constexpr uint32_t ID64 = tc::idesc_bf16_f32(TILE, MLP_H);
    {
        char* b = reinterpret_cast<char*>(s.h);
        *reinterpret_cast<uint4*>(b + tc::kmajor_off(TILE, t, 0)) =
            make_uint4(bf16x2(f[0], f[1]), bf16x2(f[2], f[3]), bf16x2(1.0f, 1.0f), 0u);
        *reinterpret_cast<uint4*>(b + tc::kmajor_off(TILE, t, 8)) = make_uint4(0u, 0u, 0u, 0u);
    }
    tc::fence_proxy_async();
    __syncthreads();
    float z[32];
    // layer 1 (K = 16: one MMA; bias in K 4, 5)
    if (t == 0) {
        tc::fence_after_sync();
        tc::mma_bf16(tmem, tc::operand_desc(s.h, TILE, 0), tc::operand_desc(s.w1i, MLP_H, 0), ID64, 0);
        tc::mma_commit(&s.mbar);
    }
    if (!cta_wait(&s.mbar, phase & 1, err)) return false;
    ++phase;
    tc::fence_after_sync();
#pragma unroll
    for (int half = 0; half < 2; ++half) {  // 32 TMEM columns at a time
        tc::tmem_ld32(trow + 32 * half, z);
        store_row32_relu(s.h, t, z, half);
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    // layers 2 and 3 (K = 80: five MMAs each; bias in K 64, 65)
#pragma unroll 1
    for (int layer = 0; layer < 2; ++layer) {
        const __nv_bfloat16* w = layer == 0 ? s.w2i : s.w3i;
        if (t == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int k = 0; k < MLP_KH / 16; ++k)
                tc::mma_bf16(tmem, tc::operand_desc(s.h, TILE, k), tc::operand_desc(w, MLP_H, k), ID64, k > 0);
            tc::mma_commit(&s.mbar);
        }
        if (!cta_wait(&s.mbar, phase & 1, err)) return false;
        ++phase;
        tc::fence_after_sync();
        if (layer == 0) {  // the layer-2 MMA has completed: h1 can be overwritten by h2
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                tc::tmem_ld32(trow + 32 * half, z);
                store_row32_relu(s.h, t, z, half);
            }
            tc::fence_proxy_async();
            tc::fence_before_sync();
            __syncthreads();
        }
    }
    float acc = s.b4;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        tc::tmem_ld32(trow + 32 * half, z);
#pragma unroll
        for (int i = 0; i < 32; ++i) acc = fmaf(s.w4[32 * half + i], relu(z[i]), acc);
    }
    y = acc;
    tc::fence_before_sync();
    __syncthreads();  // all TMEM loads of this tile done before the next tile's MMA
    return true;
}

// shared prologue / epilogue of the inference kernels: weights, TMEM, mbarrier.
// The allocation permit is given up right after the allocation: a CTA that
// still holds it keeps the next CTA of the kernel off the SM.
__device__ __forceinline__ void infer_begin(InferSmem& s, const MlpBlob* __restrict__ blob) {
    load_weights_infer(s, blob);
    if (threadIdx.x < 32) {
        tc::tmem_alloc(&s.tmem_base, 64);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) tc::mbar_init(&s.mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
}
__device__ __forceinline__ void infer_end(InferSmem& s) {
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_dealloc(s.tmem_base, 64);
}

__global__ void __launch_bounds__(TILE) k_mlp_forward(const MlpBlob* __restrict__ blob, const float* __restrict__ feat,
                                                      int n, float* __restrict__ out, unsigned int* err) {
    extern __shared__ __align__(128) unsigned char smraw[];
    InferSmem& s = *reinterpret_cast<InferSmem*>(smraw);
    const int t = threadIdx.x;
    infer_begin(s, blob);
    uint32_t phase = 0;
    const int ntiles = (n + TILE - 1) / TILE;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int i = tile * TILE + t;
        float f[4] = {0.f, 0.f, 0.f, 0.f};
        if (i < n)
            for (int k = 0; k < 4; ++k) f[k] = feat[i * 4 + k];
        float y = 0.f;
        if (!mlp_forward_tile(s, f, y, phase, err)) break;
        if (i < n) out[i] = y;
    }
    infer_end(s);
}

// ---- learned W guesses of a split stage ------------------------------------------------
struct GuessArgs {
    int n[3];
    long long sy, sz, vs;
    float gamma;
    const double* U;  // conserved state of the stage, padded SoA
    float* w_guess;   // one per padded cell (interior cells written)
    unsigned int* err;
};

// the features of cell_features in FP32 arithmetic (they feed a BF16 network)
__device__ __forceinline__ void guess_features(const double* U, float gamma, const float* mu, const float* isd,
                                               float* f) {
    const float D = (float)U[0], E = (float)(-U[1]);
    const float S = sqrtf((float)(U[2] * U[2] + U[3] * U[3] + U[4] * U[4]));
    const float raw[4] = {__logf(fmaxf(D, 1e-30f)), __fdividef(S, E), __logf(fmaxf(__fdividef(E, D), 1e-30f)), gamma};
#pragma unroll
    for (int i = 0; i < 4; ++i) f[i] = (raw[i] - mu[i]) * isd[i];
}

// interior cell e of the grid -> padded linear index; false past the end
__device__ __forceinline__ bool guess_cell(const CellMap& cm, long long e, long long tot, long long& c) {
    if (e >= tot) return false;
    c = cm.padded((uint32_t)e);
    return true;
}

// One thread per cell of a 128-cell tile; the next tile's state is loaded
// before the current tile's network runs.
__global__ void __launch_bounds__(TILE) k_mlp_guess(const MlpBlob* __restrict__ blob, GuessArgs a) {
    extern __shared__ __align__(128) unsigned char smraw[];
    InferSmem& s = *reinterpret_cast<InferSmem*>(smraw);
    const int t = threadIdx.x;
    infer_begin(s, blob);
    const int N0 = a.n[0] - 2 * NG, N1 = a.n[1] - 2 * NG, N2 = a.n[2] - 2 * NG;
    const long long tot = (long long)N0 * N1 * N2;  // < 2^32 (launch_mlp_guess)
    const long long ntiles = (tot + TILE - 1) / TILE;
    CellMap cm;
    cm.init(N0, N1, a.sy, a.sz, NG);
    uint32_t phase = 0;
    long long tile = blockIdx.x;
    long long c = 0;
    bool ok = tile < ntiles && guess_cell(cm, tile * TILE + t, tot, c);
    double u[5] = {1.0, -2.0, 0.0, 0.0, 0.0};
    if (ok)
#pragma unroll
        for (int v = 0; v < 5; ++v) u[v] = a.U[v * a.vs + c];
    for (; tile < ntiles; tile += gridDim.x) {
        const long long nt = tile + gridDim.x;
        long long cn = 0;
        const bool okn = nt < ntiles && guess_cell(cm, nt * TILE + t, tot, cn);
        double un[5] = {1.0, -2.0, 0.0, 0.0, 0.0};
        if (okn)
#pragma unroll
            for (int v = 0; v < 5; ++v) un[v] = a.U[v * a.vs + cn];
        float f[4];
        guess_features(u, a.gamma, s.mu, s.isd, f);
        float y = 0.f;
        if (!mlp_forward_tile(s, f, y, phase, a.err)) break;
        if (ok) a.w_guess[c] = (float)(-u[1] * (1.0 + (double)fmaxf(y, 0.0f)));
        ok = okn;
        c = cn;
#pragma unroll
        for (int v = 0; v < 5; ++v) u[v] = un[v];
    }
    infer_end(s);
}

// ---- training ---------------------------------------------------------------------
// TMEM columns of the training kernel
constexpr uint32_t TC_G1 = 0, TC_G2 = 64, TC_G3 = 128, TC_G4 = 192, TC_Z1 = 256, TC_Z2 = 320, TC_Z3 = 384,
                   TC_DH = 448, TC_NCOL = 512;

struct TrainSmem {
    __nv_bfloat16 a1[TILE * MLP_KIN];     // x, K-major [cells x 16]
    __nv_bfloat16 h[TILE * MLP_H];        // h1 then h2, K-major [cells x 64]
    __nv_bfloat16 dz[TILE * MLP_H];       // dz3 then dz2, K-major [cells x 64]
    __nv_bfloat16 at[TILE * TILE];        // transposed activations [128 rows (features, ones) x 128 cells]
    __nv_bfloat16 dzt[MLP_H * TILE];      // dz^T [64 x 128 cells]
    __nv_bfloat16 dyt[16 * TILE];         // dy^T [16 x 128 cells], row 0 used
    __nv_bfloat16 w1t[MLP_H * MLP_KIN];
    __nv_bfloat16 w2t[MLP_H * MLP_H];
    __nv_bfloat16 w3t[MLP_H * MLP_H];
    __nv_bfloat16 w2n[MLP_H * MLP_H];
    __nv_bfloat16 w3n[MLP_H * MLP_H];
    float b1[MLP_H], b2[MLP_H], b3[MLP_H], w4[MLP_H];
    float b4;
    float loss[TILE / 32];
    uint64_t mbar;
    uint32_t tmem_base;
};

__device__ __forceinline__ void st_bf16(__nv_bfloat16* buf, int R, int row, int k, float v) {
    *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(buf) + tc::kmajor_off(R, row, k)) = __float2bfloat16(v);
}

// issue-and-wait helper: thread 0 runs `issue`, all threads wait on the commit
template <typename F>
__device__ __forceinline__ bool run_mma(TrainSmem& s, uint32_t& phase, unsigned int* err, F issue) {
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc::fence_after_sync();
        issue();
        tc::mma_commit(&s.mbar);
    }
    if (!cta_wait(&s.mbar, phase & 1, err)) return false;
    ++phase;
    tc::fence_after_sync();
    return true;
}

__global__ void __launch_bounds__(TILE, 1) k_mlp_train(const MlpBlob* __restrict__ blob, const float* __restrict__ feat,
                                                       const float* __restrict__ target, const float* __restrict__ weight,
                                                       int n, float inv_batch, float* __restrict__ grad,
                                                       float* __restrict__ loss_out, unsigned int* err) {
    extern __shared__ __align__(128) unsigned char smraw[];
    TrainSmem& s = *reinterpret_cast<TrainSmem*>(smraw);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    // weights
    {
        auto cp = [&](void* dst, const void* src, size_t bytes) {
            const uint4* a = reinterpret_cast<const uint4*>(src);
            uint4* b = reinterpret_cast<uint4*>(dst);
            for (int i = t; i < (int)(bytes / 16); i += TILE) b[i] = a[i];
        };
        cp(s.w1t, blob->w1t, sizeof(s.w1t));
        cp(s.w2t, blob->w2t, sizeof(s.w2t));
        cp(s.w3t, blob->w3t, sizeof(s.w3t));
        cp(s.w2n, blob->w2n, sizeof(s.w2n));
        cp(s.w3n, blob->w3n, sizeof(s.w3n));
        for (int i = t; i < MLP_H; i += TILE) {
            s.b1[i] = blob->b1[i];
            s.b2[i] = blob->b2[i];
            s.b3[i] = blob->b3[i];
            s.w4[i] = blob->w4[i];
        }
        if (t == 0) s.b4 = blob->b4;
        // transposed-activation and dy^T buffers start at zero (unused rows stay zero)
        uint4 z = make_uint4(0u, 0u, 0u, 0u);
        for (int i = t; i < (int)(sizeof(s.at) / 16); i += TILE) reinterpret_cast<uint4*>(s.at)[i] = z;
        for (int i = t; i < (int)(sizeof(s.dyt) / 16); i += TILE) reinterpret_cast<uint4*>(s.dyt)[i] = z;
    }
    if (t < 32) {
        tc::tmem_alloc(&s.tmem_base, TC_NCOL);
        tc::tmem_relinquish();  // a CTA holding the permit keeps the next CTA off the SM
    }
    if (t == 0) tc::mbar_init(&s.mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = s.tmem_base;
    const uint32_t lanebase = (uint32_t)(warp * 32) << 16;
    constexpr uint32_t ID64 = tc::idesc_bf16_f32(TILE, MLP_H);
    constexpr uint32_t ID16 = tc::idesc_bf16_f32(TILE, 16);
    uint32_t phase = 0;
    uint32_t gacc = 0;  // weight-gradient accumulation flag (0 on the CTA's first tile)
    float loss = 0.0f;
    const int ntiles = (n + TILE - 1) / TILE;
    bool good = true;
    for (int tile = blockIdx.x; tile < ntiles && good; tile += gridDim.x) {
        const int i = tile * TILE + t;
        const bool ok = i < n;
        float x[4] = {0.f, 0.f, 0.f, 0.f}, tgt = 0.f, wgt = 0.f;
        if (ok) {
            for (int k = 0; k < 4; ++k) x[k] = feat[i * 4 + k];
            tgt = target[i];
            wgt = weight ? weight[i] : 1.0f;
        }
        float z[64], g[64];
        // ---- forward ----
        store_row16(s.a1, t, x);
        good = run_mma(s, phase, err, [&] {
            tc::mma_bf16(tm + TC_Z1, tc::operand_desc(s.a1, TILE, 0), tc::operand_desc(s.w1t, MLP_H, 0), ID64, 0);
        });
        if (!good) break;
        tc::tmem_ld64(tm + lanebase + TC_Z1, z);
#pragma unroll
        for (int k = 0; k < 64; ++k) g[k] = relu(z[k] + s.b1[k]);
        store_row64(s.h, t, g);
        good = run_mma(s, phase, err, [&] {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                tc::mma_bf16(tm + TC_Z2, tc::operand_desc(s.h, TILE, k), tc::operand_desc(s.w2t, MLP_H, k), ID64, k > 0);
        });
        if (!good) break;
        tc::tmem_ld64(tm + lanebase + TC_Z2, z);
#pragma unroll
        for (int k = 0; k < 64; ++k) g[k] = relu(z[k] + s.b2[k]);
        store_row64(s.h, t, g);
        good = run_mma(s, phase, err, [&] {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                tc::mma_bf16(tm + TC_Z3, tc::operand_desc(s.h, TILE, k), tc::operand_desc(s.w3t, MLP_H, k), ID64, k > 0);
        });
        if (!good) break;
        tc::tmem_ld64(tm + lanebase + TC_Z3, z);
        float y = s.b4;
#pragma unroll
        for (int k = 0; k < 64; ++k) {
            g[k] = relu(z[k] + s.b3[k]);
            y = fmaf(s.w4[k], g[k], y);
        }
        const float r = ok ? (y - tgt) : 0.0f;
        loss += wgt * r * r;
        const float dy = 2.0f * wgt * r * inv_batch;
        // ---- layer 4 gradients: [h3^T; 1] x dy^T ----
#pragma unroll
        for (int k = 0; k < 64; ++k) st_bf16(s.at, TILE, k, t, ok ? g[k] : 0.0f);
        st_bf16(s.at, TILE, 64, t, ok ? 1.0f : 0.0f);
        st_bf16(s.dyt, 16, 0, t, dy);
        // dz3 = dy w4 * relu'(z3)
#pragma unroll
        for (int k = 0; k < 64; ++k) g[k] = dy * s.w4[k] * drelu(z[k] + s.b3[k]);
        store_row64(s.dz, t, g);
#pragma unroll
        for (int k = 0; k < 64; ++k) st_bf16(s.dzt, MLP_H, k, t, g[k]);
        good = run_mma(s, phase, err, [&] {
#pragma unroll
            for (int k = 0; k < 8; ++k)
                tc::mma_bf16(tm + TC_G4, tc::operand_desc(s.at, TILE, k), tc::operand_desc(s.dyt, 16, k), ID16,
                             gacc | (uint32_t)(k > 0));
        });
        if (!good) break;
        // ---- layer 3: dW3 = [h2^T; 1] dz3, dh2 = dz3 W3^T ----
        tc::tmem_ld64(tm + lanebase + TC_Z2, z);
#pragma unroll
        for (int k = 0; k < 64; ++k) st_bf16(s.at, TILE, k, t, ok ? relu(z[k] + s.b2[k]) : 0.0f);
        good = run_mma(s, phase, err, [&] {
#pragma unroll
            for (int k = 0; k < 8; ++k)
                tc::mma_bf16(tm + TC_G3, tc::operand_desc(s.at, TILE, k), tc::operand_desc(s.dzt, MLP_H, k), ID64,
                             gacc | (uint32_t)(k > 0));
#pragma unroll
            for (int k = 0; k < 4; ++k)
                tc::mma_bf16(tm + TC_DH, tc::operand_desc(s.dz, TILE, k), tc::operand_desc(s.w3n, MLP_H, k), ID64, k > 0);
        });
        if (!good) break;
        tc::tmem_ld64(tm + lanebase + TC_DH, g);
#pragma unroll
        for (int k = 0; k < 64; ++k) g[k] = g[k] * drelu(z[k] + s.b2[k]);  // dz2 (z holds z2)
        store_row64(s.dz, t, g);
#pragma unroll
        for (int k = 0; k < 64; ++k) st_bf16(s.dzt, MLP_H, k, t, g[k]);
        // ---- layer 2: dW2 = [h1^T; 1] dz2, dh1 = dz2 W2^T ----
        tc::tmem_ld64(tm + lanebase + TC_Z1, z);
#pragma unroll
        for (int k = 0; k < 64; ++k) st_bf16(s.at, TILE, k, t, ok ? relu(z[k] + s.b1[k]) : 0.0f);
        good = run_mma(s, phase, err, [&] {
#pragma unroll
            for (int k = 0; k < 8; ++k)
                tc::mma_bf16(tm + TC_G2, tc::operand_desc(s.at, TILE, k), tc::operand_desc(s.dzt, MLP_H, k), ID64,
                             gacc | (uint32_t)(k > 0));
#pragma unroll
            for (int k = 0; k < 4; ++k)
                tc::mma_bf16(tm + TC_DH, tc::operand_desc(s.dz, TILE, k), tc::operand_desc(s.w2n, MLP_H, k), ID64, k > 0);
        });
        if (!good) break;
        tc::tmem_ld64(tm + lanebase + TC_DH, g);
#pragma unroll
        for (int k = 0; k < 64; ++k) g[k] = g[k] * drelu(z[k] + s.b1[k]);  // dz1 (z holds z1)
#pragma unroll
        for (int k = 0; k < 64; ++k) st_bf16(s.dzt, MLP_H, k, t, g[k]);
        // ---- layer 1: dW1 = [x^T; 1] dz1 (rows 5..64 of the transposed buffer cleared) ----
#pragma unroll
        for (int k = 0; k < 65; ++k) {
            float v = k < 4 ? x[k] : (k == 4 ? 1.0f : 0.0f);
            st_bf16(s.at, TILE, k, t, ok ? v : 0.0f);
        }
        good = run_mma(s, phase, err, [&] {
#pragma unroll
            for (int k = 0; k < 8; ++k)
                tc::mma_bf16(tm + TC_G1, tc::operand_desc(s.at, TILE, k), tc::operand_desc(s.dzt, MLP_H, k), ID64,
                             gacc | (uint32_t)(k > 0));
        });
        if (!good) break;
        gacc = 1;
    }
    // loss
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0) atomicAdd(loss_out, loss);
    // weight gradients: rows 0..64 of G1..G3 (warps 0..2), G4 column 0
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (good && gacc) {
        const int row = t;  // TMEM lane = row
        float v[64];
        if (warp < 3) {
            tc::tmem_ld64(tm + lanebase + TC_G1, v);
            if (row < 4)
                for (int o = 0; o < 64; ++o) atomicAdd(grad + OFF_W1 + row * MLP_H + o, v[o]);
            if (row == 4)
                for (int o = 0; o < 64; ++o) atomicAdd(grad + OFF_B1 + o, v[o]);
            tc::tmem_ld64(tm + lanebase + TC_G2, v);
            if (row < 64)
                for (int o = 0; o < 64; ++o) atomicAdd(grad + OFF_W2 + row * MLP_H + o, v[o]);
            if (row == 64)
                for (int o = 0; o < 64; ++o) atomicAdd(grad + OFF_B2 + o, v[o]);
            tc::tmem_ld64(tm + lanebase + TC_G3, v);
            if (row < 64)
                for (int o = 0; o < 64; ++o) atomicAdd(grad + OFF_W3 + row * MLP_H + o, v[o]);
            if (row == 64)
                for (int o = 0; o < 64; ++o) atomicAdd(grad + OFF_B3 + o, v[o]);
            tc::tmem_ld64(tm + lanebase + TC_G4, v);  // columns 192..255: column 0 = layer-4 gradient
            if (row < 64) atomicAdd(grad + OFF_W4 + row, v[0]);
            if (row == 64) atomicAdd(grad + OFF_B4, v[0]);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (t < 32) tc::tmem_dealloc(tm, TC_NCOL);
}

__global__ void k_mlp_adam(float* __restrict__ prm, const float* __restrict__ grad, float* __restrict__ m,
                           float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float gi = grad[i];
        float mi = b1 * m[i] + (1.0f - b1) * gi;
        float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        prm[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

}  // namespace vb

using namespace vb;

struct vb_mlp {
    int device = 0;
    float* prm = nullptr;   // FP32 master parameters
    float* grad = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    float* norm = nullptr;  // mu[4], isd[4]
    float* loss = nullptr;
    unsigned int* err = nullptr;
    MlpBlob* blob = nullptr;
    int adam_t = 0;
    std::string msg;
};

static thread_local std::string g_mlp_err;

static int mfail(vb_mlp_handle m, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (m)
        m->msg = buf;
    else
        g_mlp_err = buf;
    return code;
}

#define MCUDA(m, expr)                                                                                  \
    do {                                                                                                \
        cudaError_t e_ = (expr);                                                                        \
        if (e_ != cudaSuccess) return mfail(m, VB_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));    \
    } while (0)

static int mlp_check_err(vb_mlp_handle m, cudaStream_t s) {
    unsigned int e = 0;
    MCUDA(m, cudaMemcpyAsync(&e, m->err, sizeof e, cudaMemcpyDeviceToHost, s));
    MCUDA(m, cudaStreamSynchronize(s));
    if (e) {
        cudaMemsetAsync(m->err, 0, sizeof(unsigned int), s);
        return mfail(m, VB_ERR_TIMEOUT, "a bounded tensor-core wait ran out (error flag %u)", e);
    }
    return VB_OK;
}

static int pack(vb_mlp_handle m, cudaStream_t s) {
    k_mlp_pack<<<16, 256, 0, s>>>(m->prm, m->norm, m->blob);
    MCUDA(m, cudaGetLastError());
    return VB_OK;
}

namespace vb {
// used by vb_api.cu for the learned-guess stage
cudaError_t launch_mlp_guess(const void* mlp_blob, const StageParams& p, const double* U, float* w_guess,
                             unsigned int* err, cudaStream_t s) {
    GuessArgs a{};
    for (int i = 0; i < 3; ++i) a.n[i] = p.n[i];
    a.sy = p.sy;
    a.sz = p.sz;
    a.vs = p.vs;
    a.gamma = (float)p.gamma;
    a.U = U;
    a.w_guess = w_guess;
    a.err = err;
    static unsigned long long attr = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(attr >> (dev & 63) & 1ULL)) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_guess, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sizeof(InferSmem));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k_mlp_guess, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        attr |= 1ULL << (dev & 63);
    }
    const long long cells = (long long)(p.n[0] - 2 * NG) * (p.n[1] - 2 * NG) * (p.n[2] - 2 * NG);
    if ((unsigned long long)cells > MAX_CELLS_U32) return cudaErrorInvalidValue;
    const long long tiles = (cells + TILE - 1) / TILE;
    const int nb = (int)std::min<long long>(tiles, 148LL * 4);
    k_mlp_guess<<<nb, TILE, sizeof(InferSmem), s>>>((const MlpBlob*)mlp_blob, a);
    return cudaGetLastError();
}

// ---- fused learned con2prim of a split stage ------------------------------------------
// k_mlp_guess followed by k_c2p in one persistent kernel: per 128-cell tile,
// U is read once, the network's W0 stays in the thread that runs the W Newton
// from it (no W guess array in HBM), and the Newton's FP64 work of the other
// CTAs on the SM overlaps each CTA's MMA round trips. W0 is rounded to FP32
// exactly as the two-kernel form stores it, so both forms start the Newton
// from the same guess. With p.div_in_pout the stencil kernel left the FP32
// divergence in Pout, and this kernel forms U = rk_a U0 + rk_b (Us - div)
// (written to Uo) before the features; the next tile's inputs are loaded
// before the current tile's Newton, whose latency covers them.
// GATED (the precision-gated refinement, options.c2p_fp32): every cell the
// FP32 gate admits is finished here by the FP32 pressure Newton; the others
// are appended, with their guess, to a list (one atomic per warp) that
// k_c2p_deferred solves with the FP64 W Newton after this kernel, so this
// kernel carries no FP64 Newton and keeps its registers for the network.
template <typename R, bool GATED>
__global__ void __launch_bounds__(TILE, 5) k_c2p_learned(const MlpBlob* __restrict__ blob, StageParams p,
                                                         StageBufs<R> b, unsigned int* err) {
    extern __shared__ __align__(128) unsigned char smraw[];
    InferSmem& s = *reinterpret_cast<InferSmem*>(smraw);
    const int t = threadIdx.x;
    infer_begin(s, blob);
    const int N0 = p.n[0] - 2 * NG, N1 = p.n[1] - 2 * NG, N2 = p.n[2] - 2 * NG;
    const long long tot = (long long)N0 * N1 * N2;
    const long long ntiles = (tot + TILE - 1) / TILE;
    const long long vs = p.vs;
    CellMap cm;  // tot < 2^32 (launch_c2p_learned)
    cm.init(N0, N1, p.sy, p.sz, NG);
    auto cell = [&](long long e, long long& c) -> bool {
        if (e >= tot) return false;
        c = cm.padded((uint32_t)e);
        return true;
    };
    const bool div = p.div_in_pout != 0, rk = p.rk_a != 0.0;
    // raw inputs of one cell: U of the stage, or (Us, U0, div)
    struct Raw {
        double us[5], u0[5];
        float d[5];
    };
    auto load = [&](long long cc, Raw& r) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            r.us[v] = div ? b.Us[v * vs + cc] : b.Uo[v * vs + cc];
            r.u0[v] = div && rk ? b.U0[v * vs + cc] : 0.0;
            r.d[v] = div ? (float)b.Pout[v * vs + cc] : 0.0f;
        }
    };
    auto form = [&](const Raw& r, long long cc, double* uo) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            if (div) {
                double x = r.us[v] - (double)r.d[v];
                if (rk) x = p.rk_a * r.u0[v] + p.rk_b * x;
                uo[v] = x;
                b.Uo[v * vs + cc] = x;
            } else {
                uo[v] = r.us[v];
            }
        }
    };
    unsigned long long n_fail = 0, n_fb = 0, n_it = 0, n_cells = 0;
    uint32_t phase = 0;
    long long tile = blockIdx.x;
    long long c = 0;
    bool ok = tile < ntiles && cell(tile * TILE + t, c);
    double u[5] = {1.0, -2.0, 0.0, 0.0, 0.0};
    if (ok) {
        Raw r;
        load(c, r);
        form(r, c, u);
    }
    for (; tile < ntiles; tile += gridDim.x) {
        const long long nt = tile + gridDim.x;
        long long cn = 0;
        const bool okn = nt < ntiles && cell(nt * TILE + t, cn);
        float f[4];
        guess_features(u, (float)p.gamma, s.mu, s.isd, f);
        float y = 0.f;
        if (!mlp_forward_tile(s, f, y, phase, err)) break;
        Raw rn;
        if (okn) load(cn, rn);
        // the guess rounded to FP32 exactly as the two-kernel form stores it
        const float W0 = (float)(-u[1] * (1.0 + (double)fmaxf(y, 0.0f)));
        if constexpr (GATED) {
            // FP32 pressure Newton where the gate admits the cell; the rest to the list
            double P[5];
            int r = 0;
            const bool done = ok && c2p_try_fp32(p.gamma, u, W0, P, &r);
            if (done) {
                n_it += r;
                n_cells += 1;
                P[0] = jmax(P[0], p.floor_);
                P[1] = jmax(P[1], p.floor_);
#pragma unroll
                for (int v = 0; v < 5; ++v) b.Pout[v * vs + c] = (R)P[v];
            }
            const bool defer = ok && !done;
            const unsigned m = __ballot_sync(0xffffffffu, defer);
            if (m) {
                const int lane = t & 31, leader = __ffs(m) - 1;
                unsigned base = 0;
                if (lane == leader) base = atomicAdd(p.defer_n, (unsigned)__popc(m));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (defer) {
                    p.defer_idx[base + __popc(m & ((1u << lane) - 1u))] = (unsigned)(tile * TILE + t);
                    p.defer_w0[c] = W0;
                }
            }
        } else if (ok) {
            // the FP64 W Newton on every cell
            double P[5];
            int fb;
            const int r = c2p_w(p.gamma, u, (double)W0, p.w_rtol, p.w_max_newton, 4 * p.n_iter, P, &fb);
            n_fail += (r < 0);
            n_fb += fb;
            n_it += (r < 0 ? -r : r);
            n_cells += 1;
            P[0] = jmax(P[0], p.floor_);
            P[1] = jmax(P[1], p.floor_);
#pragma unroll
            for (int v = 0; v < 5; ++v) b.Pout[v * vs + c] = (R)P[v];
        }
        if (okn) form(rn, cn, u);
        ok = okn;
        c = cn;
    }
    infer_end(s);
    unsigned long long* cnt = p.counters;
    if (!cnt) return;
    if (n_fail) atomicAdd(cnt + CNT_C2P_FAIL, n_fail);
    if (p.stats) {
        for (int o = 16; o > 0; o >>= 1) {
            n_fb += __shfl_xor_sync(0xffffffffu, n_fb, o);
            n_it += __shfl_xor_sync(0xffffffffu, n_it, o);
            n_cells += __shfl_xor_sync(0xffffffffu, n_cells, o);
        }
        if ((t & 31) == 0) {
            if (n_fb) atomicAdd(cnt + CNT_C2P_FALLBACK, n_fb);
            if (n_it) atomicAdd(cnt + CNT_C2P_ITERS, n_it);
            if (n_cells) atomicAdd(cnt + CNT_C2P_CELLS, n_cells);
            // ungated: every cell ran the FP64 Newton (gated: k_c2p_deferred counts them)
            if (!GATED && n_cells) atomicAdd(cnt + CNT_C2P_FP64, n_cells);
        }
    } else if (n_fb) {
        atomicAdd(cnt + CNT_C2P_FALLBACK, n_fb);
    }
}

template <typename R, bool GATED>
cudaError_t launch_c2p_learned_t(const void* mlp_blob, const StageParams& p, const StageBufs<R>& b, unsigned int* err,
                                 cudaStream_t s) {
    static unsigned long long attr = 0;
    static int resident[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    const int d = dev & 63;
    if (!(attr >> d & 1ULL)) {
        cudaError_t e = cudaFuncSetAttribute(k_c2p_learned<R, GATED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sizeof(InferSmem));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k_c2p_learned<R, GATED>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        // 5 CTAs per SM: the launch bound (96 registers x 128 threads), 5 x 43 KB of
        // shared memory and 5 x 64 TMEM columns all fit (the occupancy query
        // reported 1 per SM here, which left the SM idle during each MMA round trip;
        // measured on the 512^3 jet: 5 per SM 1.4 % faster than 4 at 124 registers)
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        resident[d] = 5 * std::max(1, sms);
        attr |= 1ULL << d;
    }
    const long long cells = (long long)(p.n[0] - 2 * NG) * (p.n[1] - 2 * NG) * (p.n[2] - 2 * NG);
    if ((unsigned long long)cells > MAX_CELLS_U32) return cudaErrorInvalidValue;
    const long long tiles = (cells + TILE - 1) / TILE;
    const int nb = (int)std::min<long long>(tiles, resident[d]);
    if (nb <= 0) return cudaSuccess;
    k_c2p_learned<R, GATED><<<nb, TILE, sizeof(InferSmem), s>>>((const MlpBlob*)mlp_blob, p, b, err);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_c2p_learned(const void* mlp_blob, const StageParams& p, const StageBufs<R>& b, unsigned int* err,
                               cudaStream_t s) {
    if (p.c2p_fp32 && p.defer_idx && p.defer_n && p.defer_w0)
        return launch_c2p_learned_t<R, true>(mlp_blob, p, b, err, s);
    return launch_c2p_learned_t<R, false>(mlp_blob, p, b, err, s);
}
template cudaError_t launch_c2p_learned<float>(const void*, const StageParams&, const StageBufs<float>&,
                                               unsigned int*, cudaStream_t);
template cudaError_t launch_c2p_learned<double>(const void*, const StageParams&, const StageBufs<double>&,
                                                unsigned int*, cudaStream_t);

// The cells the gated fused kernel left to FP64: the W Newton from their FP32
// guesses (as the ungated kernel runs it), the floors, P. The count is read on
// the device, bounded by the list's capacity (every interior cell).
template <typename R>
__global__ void __launch_bounds__(256) k_c2p_deferred(StageParams p, StageBufs<R> b) {
    const int N0 = p.n[0] - 2 * NG, N1 = p.n[1] - 2 * NG, N2 = p.n[2] - 2 * NG;
    const unsigned long long cap = (unsigned long long)N0 * N1 * N2;
    const unsigned long long n = std::min<unsigned long long>(*p.defer_n, cap);
    CellMap cm;  // interior cells < 2^32 (launch_c2p_deferred)
    cm.init(N0, N1, p.sy, p.sz, NG);
    const long long vs = p.vs;
    unsigned long long n_fail = 0, n_fb = 0, n_it = 0, n_cells = 0;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned e = p.defer_idx[i];
        if ((unsigned long long)e >= cap) {
            if (p.counters) atomicAdd(p.counters + CNT_BAD_INDEX, 1ULL);
            continue;
        }
        const long long c = cm.padded(e);
        double U[5], P[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) U[v] = b.Uo[v * vs + c];
        int fb;
        const int r = c2p_w(p.gamma, U, (double)p.defer_w0[c], p.w_rtol, p.w_max_newton, 4 * p.n_iter, P, &fb);
        n_fail += (r < 0);
        n_fb += fb;
        n_it += (r < 0 ? -r : r);
        n_cells += 1;
        P[0] = jmax(P[0], p.floor_);
        P[1] = jmax(P[1], p.floor_);
#pragma unroll
        for (int v = 0; v < 5; ++v) b.Pout[v * vs + c] = (R)P[v];
    }
    unsigned long long* cnt = p.counters;
    if (!cnt) return;
    if (n_fail) atomicAdd(cnt + CNT_C2P_FAIL, n_fail);
    if (p.stats) {
        for (int o = 16; o > 0; o >>= 1) {
            n_fb += __shfl_xor_sync(0xffffffffu, n_fb, o);
            n_it += __shfl_xor_sync(0xffffffffu, n_it, o);
            n_cells += __shfl_xor_sync(0xffffffffu, n_cells, o);
        }
        if ((threadIdx.x & 31) == 0) {
            if (n_fb) atomicAdd(cnt + CNT_C2P_FALLBACK, n_fb);
            if (n_it) atomicAdd(cnt + CNT_C2P_ITERS, n_it);
            if (n_cells) {
                atomicAdd(cnt + CNT_C2P_CELLS, n_cells);
                atomicAdd(cnt + CNT_C2P_FP64, n_cells);
            }
        }
    } else if (n_fb) {
        atomicAdd(cnt + CNT_C2P_FALLBACK, n_fb);
    }
}

template <typename R> cudaError_t launch_c2p_deferred(const StageParams& p, const StageBufs<R>& b, cudaStream_t s) {
    const long long cells = (long long)(p.n[0] - 2 * NG) * (p.n[1] - 2 * NG) * (p.n[2] - 2 * NG);
    if ((unsigned long long)cells > MAX_CELLS_U32 || !p.defer_idx || !p.defer_n || !p.defer_w0)
        return cudaErrorInvalidValue;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int nb = (int)std::max<long long>(1, std::min<long long>((cells + 255) / 256, 8LL * std::max(1, sms)));
    k_c2p_deferred<R><<<nb, 256, 0, s>>>(p, b);
    return cudaGetLastError();
}
template cudaError_t launch_c2p_deferred<float>(const StageParams&, const StageBufs<float>&, cudaStream_t);
template cudaError_t launch_c2p_deferred<double>(const StageParams&, const StageBufs<double>&, cudaStream_t);
}  // namespace vb

extern "C" {

const char* vb_mlp_last_error(vb_mlp_handle m) { return m ? m->msg.c_str() : g_mlp_err.c_str(); }

int vb_mlp_create(vb_mlp_handle* out) {
    if (!out) return mfail(nullptr, VB_ERR_ARG, "vb_mlp_create: null");
    vb_mlp_handle m = new vb_mlp();
    cudaGetDevice(&m->device);
    cudaError_t e = cudaSuccess;
    e = cudaMalloc((void**)&m->prm, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->grad, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->m, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->v, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->norm, sizeof(float) * 2 * MLP_IN);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->err, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->blob, sizeof(MlpBlob));
    if (e == cudaSuccess) e = cudaMemset(m->err, 0, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(m->m, 0, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMemset(m->v, 0, sizeof(float) * N_PARAMS);
    if (e != cudaSuccess) {
        vb_mlp_destroy(m);
        return mfail(nullptr, VB_ERR_NOMEM, "vb_mlp_create: %s", cudaGetErrorString(e));
    }
    *out = m;
    return VB_OK;
}

int vb_mlp_destroy(vb_mlp_handle m) {
    if (!m) return VB_OK;
    cudaFree(m->prm);
    cudaFree(m->grad);
    cudaFree(m->m);
    cudaFree(m->v);
    cudaFree(m->norm);
    cudaFree(m->loss);
    cudaFree(m->err);
    cudaFree(m->blob);
    delete m;
    return VB_OK;
}

int vb_mlp_param_count(void) { return N_PARAMS; }

int vb_mlp_set_params(vb_mlp_handle m, const float* params, const float* norm, void* stream) {
    if (!m || !params || !norm) return mfail(m, VB_ERR_ARG, "vb_mlp_set_params: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    MCUDA(m, cudaMemcpyAsync(m->prm, params, sizeof(float) * N_PARAMS, cudaMemcpyHostToDevice, s));
    MCUDA(m, cudaMemcpyAsync(m->norm, norm, sizeof(float) * 2 * MLP_IN, cudaMemcpyHostToDevice, s));
    MCUDA(m, cudaMemsetAsync(m->m, 0, sizeof(float) * N_PARAMS, s));
    MCUDA(m, cudaMemsetAsync(m->v, 0, sizeof(float) * N_PARAMS, s));
    m->adam_t = 0;
    int rc = pack(m, s);
    if (rc) return rc;
    MCUDA(m, cudaStreamSynchronize(s));
    return VB_OK;
}

int vb_mlp_get_params(vb_mlp_handle m, float* params, float* norm, void* stream) {
    if (!m || !params) return mfail(m, VB_ERR_ARG, "vb_mlp_get_params: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    MCUDA(m, cudaMemcpyAsync(params, m->prm, sizeof(float) * N_PARAMS, cudaMemcpyDeviceToHost, s));
    if (norm) MCUDA(m, cudaMemcpyAsync(norm, m->norm, sizeof(float) * 2 * MLP_IN, cudaMemcpyDeviceToHost, s));
    MCUDA(m, cudaStreamSynchronize(s));
    return VB_OK;
}

int vb_mlp_features(vb_mlp_handle m, const double* U, const double* P, int n, double gamma, float* feat,
                    float* target, float* weight, void* stream) {
    if (!m || !U || !feat || n < 0) return mfail(m, VB_ERR_ARG, "vb_mlp_features: bad argument");
    if (n == 0) return VB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    k_mlp_features<<<std::min((n + 255) / 256, 148 * 16), 256, 0, s>>>(U, P, n, gamma, m->norm, feat, target,
                                                                        weight);
    MCUDA(m, cudaGetLastError());
    return VB_OK;
}

int vb_mlp_forward(vb_mlp_handle m, const float* feat, int n, float* out, void* stream) {
    if (!m || !feat || !out || n < 0) return mfail(m, VB_ERR_ARG, "vb_mlp_forward: bad argument");
    if (n == 0) return VB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    MCUDA(m, cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(InferSmem)));
    MCUDA(m, cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    int tiles = (n + TILE - 1) / TILE;
    k_mlp_forward<<<std::min(tiles, 148 * 4), TILE, sizeof(InferSmem), s>>>(m->blob, feat, n, out, m->err);
    MCUDA(m, cudaGetLastError());
    return mlp_check_err(m, s);
}

int vb_mlp_train_step(vb_mlp_handle m, const float* feat, const float* target, const float* weight, int n, float lr,
                      float* loss, void* stream) {
    if (!m || !feat || !target || n <= 0 || !(lr >= 0.0f)) return mfail(m, VB_ERR_ARG, "vb_mlp_train_step: bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    MCUDA(m, cudaMemsetAsync(m->grad, 0, sizeof(float) * N_PARAMS, s));
    MCUDA(m, cudaMemsetAsync(m->loss, 0, sizeof(float), s));
    MCUDA(m, cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem)));
    int tiles = (n + TILE - 1) / TILE;
    k_mlp_train<<<std::min(tiles, 148), TILE, sizeof(TrainSmem), s>>>(m->blob, feat, target, weight, n,
                                                                       1.0f / (float)n, m->grad, m->loss, m->err);
    MCUDA(m, cudaGetLastError());
    if (lr > 0.0f) {
        m->adam_t += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        float c1 = 1.0f - powf(b1, (float)m->adam_t), c2 = 1.0f - powf(b2, (float)m->adam_t);
        k_mlp_adam<<<(N_PARAMS + 255) / 256, 256, 0, s>>>(m->prm, m->grad, m->m, m->v, N_PARAMS, lr, b1, b2, 1e-8f, c1,
                                                           c2);
        MCUDA(m, cudaGetLastError());
        int rc = pack(m, s);
        if (rc) return rc;
    }
    if (loss) {
        float l = 0.f;
        MCUDA(m, cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
        int rc = mlp_check_err(m, s);
        if (rc) return rc;
        *loss = l / (float)n;
    }
    return VB_OK;
}

int vb_mlp_get_grad(vb_mlp_handle m, float* grad, void* stream) {
    if (!m || !grad) return mfail(m, VB_ERR_ARG, "vb_mlp_get_grad: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    MCUDA(m, cudaMemcpyAsync(grad, m->grad, sizeof(float) * N_PARAMS, cudaMemcpyDeviceToHost, s));
    MCUDA(m, cudaStreamSynchronize(s));
    return VB_OK;
}

const void* vb_mlp_blob_ptr(vb_mlp_handle m) { return m ? (const void*)m->blob : nullptr; }
unsigned int* vb_mlp_err_ptr(vb_mlp_handle m) { return m ? m->err : nullptr; }
int vb_mlp_check(vb_mlp_handle m, void* stream) { return m ? mlp_check_err(m, (cudaStream_t)stream) : VB_ERR_ARG; }

}  // extern "C"
