// qz_batch_m1w.cu -- the batch kernel for modes = 1 instances with 513..1024 radial nodes: the kernel of
// qz_batch_kernels.cuh compiled for CTAs of 1024 threads in namespace qzb_w (as qz_sweep_m1w.cu does for
// the stand-alone sweep), holding only the m = 1 sweep. qz_batch_run launches it after the 512-thread
// batch kernel, with its own queue of the wide instances; launch_batch_m1w takes the argument block as
// bytes (qzb::BatchArgs and qzb_w::BatchArgs are the same definition).
#define QZ_SWEEP_THREADS 1024
#define qzb qzb_w
#include "qz_batch_kernels.cuh"

namespace qzb_w {
namespace {

template <int ORD, bool EXT>
cudaError_t launch_w(const BatchArgs& B, int grid, size_t smem, cudaStream_t s, int* per_sm) {
    if (per_sm) {
        *per_sm = occupancy_t<ORD, true, EXT>(smem);
        return cudaSuccess;
    }
    return launch_t<ORD, true, EXT>(B, grid, smem, s);
}

template <int ORD>
cudaError_t launch_o(const BatchArgs& B, int grid, size_t smem, cudaStream_t s, int* per_sm) {
    return B.with_ext ? launch_w<ORD, true>(B, grid, smem, s, per_sm) : launch_w<ORD, false>(B, grid, smem, s, per_sm);
}

}  // namespace

// per_sm != nullptr: only the number of resident CTAs per SM for this configuration
cudaError_t launch_batch_wide(const BatchArgs& B, int grid, size_t smem, cudaStream_t s, int* per_sm) {
    switch (B.ord) {
        case 1: return launch_o<1>(B, grid, smem, s, per_sm);
        case 2: return launch_o<2>(B, grid, smem, s, per_sm);
        case 3: return launch_o<3>(B, grid, smem, s, per_sm);
        case 4: return launch_o<4>(B, grid, smem, s, per_sm);
        case 5: return launch_o<5>(B, grid, smem, s, per_sm);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace qzb_w

#undef qzb

namespace qzb {

size_t batch_m1w_static_bytes() {
    return sizeof(qzb_w::BatchInst) + sizeof(double) * 17 * (qzb_w::kSweepThreads / 32) + 256;
}

cudaError_t launch_batch_m1w(const void* args, size_t args_size, int grid, size_t smem, cudaStream_t s,
                             int* per_sm) {
    if (!args || args_size != sizeof(qzb_w::BatchArgs)) return cudaErrorInvalidValue;
    return qzb_w::launch_batch_wide(*static_cast<const qzb_w::BatchArgs*>(args), grid, smem, s, per_sm);
}

}  // namespace qzb
