// Plain FP64 batch kernel. Built with -fmad=false, as vb_stage_f64.cu, so each
// problem rounds as the single-grid FP64 solver.
#include "vb_batch.cuh"

namespace vb {
VB_INSTANTIATE_BATCH(double)
}  // namespace vb
