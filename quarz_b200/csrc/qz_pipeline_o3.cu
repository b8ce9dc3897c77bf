// qz_pipeline_o3.cu -- the pipelined kernel for Adams-Bashforth order 3 (qz_pipeline_kernels.cuh).
#include "qz_pipeline_kernels.cuh"

namespace qzb {

template <>
cudaError_t pipeline_launch_ord<3>(const PipeArgs& P, int grid, size_t smem, cudaStream_t s) {
    return launch_o<3>(P, grid, smem, s);
}

template <>
int pipeline_occupancy_ord<3>(const PipeArgs& P, size_t smem) {
    return occupancy_o<3>(P, smem);
}

}  // namespace qzb
