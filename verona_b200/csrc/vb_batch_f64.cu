// Plain FP64 batch kernel. Built with -fmad=false, as vb_stage_f64.cu, so each
// problem rounds as the single-grid FP64 solver.
#include "vb_batch.cuh"

namespace vb {
VB_INSTANTIATE_BATCH(double)

// one thread per problem: t += dt, nsteps times, in the order the host adds them
__global__ void k_batch_time(const BatchProb* __restrict__ prob, double* __restrict__ time, int nprob, int nsteps) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nprob; p += gridDim.x * blockDim.x) {
        double t = time[p];
        const double dt = prob[p].dt;
        for (int k = 0; k < nsteps; ++k) t += dt;
        time[p] = t;
    }
}

cudaError_t batch_advance_time(const BatchProb* prob, double* time, int nprob, int nsteps, cudaStream_t s) {
    k_batch_time<<<(nprob + 127) / 128, 128, 0, s>>>(prob, time, nprob, nsteps);
    return cudaGetLastError();
}
}  // namespace vb
