// Interior-cell enumeration of the per-cell kernels (con2prim, learned guess):
// cell e, x fastest, of an N0 x N1 x N2 interior box -> padded linear index.
//
// The two divisions per cell use multiply-high against invariant divisors
// (T. Granlund, P. Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, round-up method valid for every 32-bit
// dividend): a runtime 64-bit division is a long emulated sequence on the
// GPU and dominated the instruction count of these kernels. Callers keep the
// interior cell count below 2^32.
#pragma once
#include "vb_ns.h"
#include <stdint.h>

namespace VB_NS {

__host__ __device__ __forceinline__ uint32_t umulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

struct DivU32 {
    uint32_t m, s1, s2;
    __host__ __device__ __forceinline__ void init(uint32_t d) {  // d >= 1
        uint32_t l = 0;                                           // ceil(log2 d)
        while (l < 32 && (1ull << l) < d) ++l;
        m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
        s1 = l < 1 ? l : 1;
        s2 = l > 0 ? l - 1 : 0;
    }
    __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const {
        const uint32_t t = umulhi32(m, n);
        return (t + ((n - t) >> s1)) >> s2;
    }
};

constexpr unsigned long long MAX_CELLS_U32 = 0xFFFFFFFFull;

struct CellMap {
    DivU32 dx, dy;
    uint32_t n0, n1;
    long long sy, sz;
    int ng;
    __host__ __device__ __forceinline__ void init(int N0, int N1, long long sy_, long long sz_, int ng_) {
        n0 = (uint32_t)N0;
        n1 = (uint32_t)N1;
        dx.init(n0);
        dy.init(n1);
        sy = sy_;
        sz = sz_;
        ng = ng_;
    }
    // interior cell e < N0 * N1 * N2 -> padded linear index
    __host__ __device__ __forceinline__ long long padded(uint32_t e) const {
        const uint32_t q = dx.div(e);
        const uint32_t i = e - q * n0;
        const uint32_t k = dy.div(q);
        const uint32_t j = q - k * n1;
        return (long long)(i + ng) + sy * (long long)(j + ng) + sz * (long long)(k + ng);
    }
};

}  // namespace vb
