// qz_pipeline_o4.cu -- the pipelined kernel for Adams-Bashforth order 4 (qz_pipeline_kernels.cuh).
#include "qz_pipeline_kernels.cuh"

namespace qzb {

template <>
cudaError_t pipeline_launch_ord<4>(const PipeArgs& P, int grid, size_t smem, cudaStream_t s) {
    return launch_o<4>(P, grid, smem, s);
}

template <>
int pipeline_occupancy_ord<4>(const PipeArgs& P, size_t smem) {
    return occupancy_o<4>(P, smem);
}

}  // namespace qzb
