// FP32-bulk batch kernel (FP64 U and con2prim). Built with FMA contraction and
// approximate FP32 divide / square root, as vb_stage_f32.cu.
#include "vb_batch.cuh"

namespace vb {
VB_INSTANTIATE_BATCH(float)
}  // namespace vb
