// FP64 stage kernels with FMA contraction: the same 3D z-marching stencil,
// split con2prim and box-tile kernels as vb_stage_f64.cu, built with
// -fmad=true, so that a * b + c rounds once. The reference's Julia code never
// contracts, so this form is not bit-identical to it; it is a plain FP64 path
// held to the parity bar of 1e-10 per conserved field instead (selected by
// vb_tuning.fp64_contract). The kernels live in namespace vb_f64c (VB_NS), so
// their names do not collide with the uncontracted instantiation; the two
// bridge functions below take the caller's StageParams / StageBufs<double>,
// which come from the same header text and so have the same layout.
#define VB_NS vb_f64c
#include "vb_stage.cuh"
#include "vb_stage_zm.cuh"

namespace vb_f64c {
template cudaError_t launch_stage<double>(int, int, int, const StageParams&, const StageBufs<double>&, cudaStream_t,
                                          int*);
template cudaError_t launch_c2p<double>(const StageParams&, const StageBufs<double>&, cudaStream_t);
}  // namespace vb_f64c

cudaError_t vb_f64c_launch_stage(int dims, int rec, int rs, const void* p, const void* b, cudaStream_t s,
                                 int* kernels) {
    return vb_f64c::launch_stage<double>(dims, rec, rs, *static_cast<const vb_f64c::StageParams*>(p),
                                         *static_cast<const vb_f64c::StageBufs<double>*>(b), s, kernels);
}

cudaError_t vb_f64c_launch_c2p(const void* p, const void* b, cudaStream_t s) {
    return vb_f64c::launch_c2p<double>(*static_cast<const vb_f64c::StageParams*>(p),
                                       *static_cast<const vb_f64c::StageBufs<double>*>(b), s);
}

size_t vb_f64c_stage_params_size() { return sizeof(vb_f64c::StageParams); }
