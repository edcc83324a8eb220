// FP32-bulk instantiation: primitive arrays, reconstruction, Riemann fluxes
// and flux differences in FP32; conserved variables, the RK accumulation and
// con2prim in FP64. Built with FMA contraction enabled.
#include "vb_stage.cuh"
#include "vb_stage_zm.cuh"
#include "vb_stage_zp.cuh"

namespace vb {
cudaError_t launch_stage_zp(int rec, int rs, const StageParams& p, const StageBufs<float>& b, cudaStream_t s) {
    return dispatch_stage_zp(rec, rs, p, b, s);
}

// Tensor maps of an FP32 state array. 3D, for the TMA form of the z-pair
// kernel: dims (x, y, z, variable) with byte strides (4 sy, 4 sz, 4 vs), every
// one a multiple of 16 (rows are pitched to 4 cells); the box is one plane of
// every variable with its x/y halo. 2D: the box tile of k_stage.
template <> bool encode_stage_tmap<float>(void* out, const float* P, const Grid& g) {
    if (g.dims == 2) return encode_tile2_tmap<float, TileCfg<2>::TX, TileCfg<2>::TY>(out, P, g);
    using TG = ZpTmaGeom<ZpCfg::TX, ZpCfg::TY>;
    if (g.dims != 3 || g.nv != 5) return false;
    const cuuint64_t dim[4] = {(cuuint64_t)g.n[0], (cuuint64_t)g.n[1], (cuuint64_t)g.n[2], 5};
    const cuuint64_t stride[3] = {(cuuint64_t)g.sy * 4, (cuuint64_t)g.sz * 4, (cuuint64_t)g.vs * 4};
    const cuuint32_t box[4] = {TG::BXW, TG::EY, 1, 5};
    return encode_tmap(out, P, 4, 4, dim, stride, box);
}
VB_INSTANTIATE_LAUNCHERS(float)
template cudaError_t launch_c2p<float>(const StageParams&, const StageBufs<float>&, cudaStream_t);
}  // namespace vb
