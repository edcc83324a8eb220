// Host side of the TMA tensor maps of the state arrays. The driver's encoder
// (cuTensorMapEncodeTiled) is reached through the runtime's entry-point query,
// so the library links no driver library.
#pragma once
#include "vb_ns.h"
#include <cuda.h>
#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled
#include <cuda_runtime.h>
#include <stdint.h>

namespace VB_NS {

inline PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            fn = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    return encode;
}

// Tiled tensor map (no interleave, no swizzle, zero fill outside the tensor)
// of a state array of `rank` dimensions, innermost first; stride[d] is the
// byte stride of dimension d + 1. out: a 64-byte aligned CUtensorMap. False
// where the encoder is missing or a TMA rule is not met (16-byte aligned base
// and strides, 16-byte multiple inner box extent, box extents <= 256).
inline bool encode_tmap(void* out, const void* base, int elem_bytes, int rank, const cuuint64_t* dim,
                        const cuuint64_t* stride, const cuuint32_t* box) {
    if (!out || !base || ((uintptr_t)out & 63) || ((uintptr_t)base & 15) || rank < 1 || rank > 5) return false;
    if ((box[0] * (cuuint32_t)elem_bytes) % 16) return false;
    for (int d = 0; d < rank; ++d)
        if (box[d] == 0 || box[d] > 256 || dim[d] == 0) return false;
    for (int d = 0; d + 1 < rank; ++d)
        if (stride[d] % 16) return false;
    PFN_cuTensorMapEncodeTiled_v12000 encode = tmap_encoder();
    if (!encode) return false;
    const cuuint32_t estride[5] = {1, 1, 1, 1, 1};
    return encode(static_cast<CUtensorMap*>(out),
                  elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                  (cuuint32_t)rank, const_cast<void*>(base), dim, stride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace vb
