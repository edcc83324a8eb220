// FP32-bulk instantiation: primitive arrays, reconstruction, Riemann fluxes
// and flux differences in FP32; conserved variables, the RK accumulation and
// con2prim in FP64. Built with FMA contraction enabled.
#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled

#include "vb_stage.cuh"
#include "vb_stage_zm.cuh"
#include "vb_stage_zp.cuh"

namespace vb {
cudaError_t launch_stage_zp(int rs, const StageParams& p, const StageBufs<float>& b, cudaStream_t s) {
    return dispatch_stage_zp(rs, p, b, s);
}

// Tensor map of a 3D FP32 state array for the TMA form of the z-pair kernel:
// dims (x, y, z, variable) with byte strides (4 sy, 4 sz, 4 vs), every one a
// multiple of 16 (rows are pitched to 4 cells); the box is one plane of every
// variable with its x/y halo. The driver's encoder is reached through the
// runtime's entry-point query, so the library links no driver library.
bool encode_plane_tmap(void* out, const float* P, const Grid& g) {
    using TG = ZpTmaGeom<ZpCfg::TX, ZpCfg::TY>;
    if (g.dims != 3 || g.nv != 5 || !P || ((uintptr_t)out & 63) || ((uintptr_t)P & 15)) return false;
    if ((g.sy * 4) % 16 || (g.sz * 4) % 16 || (g.vs * 4) % 16) return false;
    static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            fn = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if (!encode) return false;
    const cuuint64_t dim[4] = {(cuuint64_t)g.n[0], (cuuint64_t)g.n[1], (cuuint64_t)g.n[2], 5};
    const cuuint64_t stride[3] = {(cuuint64_t)g.sy * 4, (cuuint64_t)g.sz * 4, (cuuint64_t)g.vs * 4};
    const cuuint32_t box[4] = {TG::BXW, TG::EY, 1, 5};
    const cuuint32_t estride[4] = {1, 1, 1, 1};
    return encode(static_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(P), dim,
                  stride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
VB_INSTANTIATE_LAUNCHERS(float)
template cudaError_t launch_c2p<float>(const StageParams&, const StageBufs<float>&, cudaStream_t);
}  // namespace vb
