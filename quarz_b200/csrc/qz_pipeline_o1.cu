// qz_pipeline_o1.cu -- the pipelined kernel for Adams-Bashforth order 1 (qz_pipeline_kernels.cuh).
#include "qz_pipeline_kernels.cuh"

namespace qzb {

template <>
cudaError_t pipeline_launch_ord<1>(const PipeArgs& P, int grid, size_t smem, cudaStream_t s) {
    return launch_o<1>(P, grid, smem, s);
}

template <>
int pipeline_occupancy_ord<1>(const PipeArgs& P, size_t smem) {
    return occupancy_o<1>(P, smem);
}

}  // namespace qzb
