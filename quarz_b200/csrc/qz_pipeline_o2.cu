// qz_pipeline_o2.cu -- the pipelined kernel for Adams-Bashforth order 2 (qz_pipeline_kernels.cuh).
#include "qz_pipeline_kernels.cuh"

namespace qzb {

template <>
cudaError_t pipeline_launch_ord<2>(const PipeArgs& P, int grid, size_t smem, cudaStream_t s) {
    return launch_o<2>(P, grid, smem, s);
}

template <>
int pipeline_occupancy_ord<2>(const PipeArgs& P, size_t smem) {
    return occupancy_o<2>(P, smem);
}

}  // namespace qzb
