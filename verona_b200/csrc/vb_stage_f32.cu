// FP32-bulk instantiation: primitive arrays, reconstruction, Riemann fluxes
// and flux differences in FP32; conserved variables, the RK accumulation and
// con2prim in FP64. Built with FMA contraction enabled.
#include "vb_stage.cuh"
#include "vb_stage_zm.cuh"

namespace vb {
VB_INSTANTIATE_LAUNCHERS(float)
template cudaError_t launch_c2p<float>(const StageParams&, const StageBufs<float>&, cudaStream_t);
}  // namespace vb
