// qz_batch_o4.cu -- the batch kernel for Adams-Bashforth order 4 (qz_batch_kernels.cuh).
#include "qz_batch_kernels.cuh"

namespace qzb {

template <>
cudaError_t batch_launch_ord<4>(const BatchArgs& B, int grid, size_t smem, cudaStream_t s) {
    if (B.with_m1)
        return B.with_ext ? launch_t<4, true, true>(B, grid, smem, s) : launch_t<4, true, false>(B, grid, smem, s);
    return B.with_ext ? launch_t<4, false, true>(B, grid, smem, s) : launch_t<4, false, false>(B, grid, smem, s);
}

template <>
int batch_occupancy_ord<4>(bool with_m1, bool with_ext, size_t smem) {
    if (with_m1) return with_ext ? occupancy_t<4, true, true>(smem) : occupancy_t<4, true, false>(smem);
    return with_ext ? occupancy_t<4, false, true>(smem) : occupancy_t<4, false, false>(smem);
}

}  // namespace qzb
