// Plain FP64 instantiation of the stage and per-step kernels. Built with
// -fmad=false so every operation rounds as the reference's Julia code does.
#include "vb_stage.cuh"

namespace vb {
VB_INSTANTIATE_LAUNCHERS(double)

int max_speed_blocks(const Grid& g) {
    (void)g;
    return 148 * 4;
}
}  // namespace vb
