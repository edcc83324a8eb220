// FP32-bulk instantiation: primitive arrays, reconstruction, Riemann fluxes
// and flux differences in FP32; conserved variables, the RK accumulation and
// con2prim in FP64. Built with FMA contraction enabled.
#include "vb_stage.cuh"
#include "vb_stage_zm.cuh"
#include "vb_stage_zp.cuh"

namespace vb {
cudaError_t launch_stage_zp(int rs, const StageParams& p, const StageBufs<float>& b, cudaStream_t s) {
    return dispatch_stage_zp(rs, p, b, s);
}
VB_INSTANTIATE_LAUNCHERS(float)
template cudaError_t launch_c2p<float>(const StageParams&, const StageBufs<float>&, cudaStream_t);
}  // namespace vb
