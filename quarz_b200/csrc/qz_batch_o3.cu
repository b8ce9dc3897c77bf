// qz_batch_o3.cu -- the batch kernel for Adams-Bashforth order 3 (qz_batch_kernels.cuh).
#include "qz_batch_kernels.cuh"

namespace qzb {

template <>
cudaError_t batch_launch_ord<3>(const BatchArgs& B, int grid, size_t smem, cudaStream_t s) {
    if (B.with_m1)
        return B.with_ext ? launch_t<3, true, true>(B, grid, smem, s) : launch_t<3, true, false>(B, grid, smem, s);
    return B.with_ext ? launch_t<3, false, true>(B, grid, smem, s) : launch_t<3, false, false>(B, grid, smem, s);
}

template <>
int batch_occupancy_ord<3>(bool with_m1, bool with_ext, size_t smem) {
    if (with_m1) return with_ext ? occupancy_t<3, true, true>(smem) : occupancy_t<3, true, false>(smem);
    return with_ext ? occupancy_t<3, false, true>(smem) : occupancy_t<3, false, false>(smem);
}

}  // namespace qzb
