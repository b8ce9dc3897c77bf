// qz_batch.cu -- many independent runs (a parameter scan) in one persistent launch.
//
// Each CTA takes the next instance from a queue (largest first) and runs all of it as
// Simulation::run does (src/Simulation.cpp:1370-1448): the step-0 beam deposit, then per step the
// sweep (qz_sweep_body.cuh), the moment sums of every beam (Beam::sums, src/Beam.cpp:1133-1155) and,
// before the last sweep, the push of every beam with the next deposit (src/Beam.cpp:725-785,
// :900-1131). Instances differ in grid, box, plasma and beams; their sweep arguments are copied into
// shared memory, the field and beam-source buffers are the CTA's slot, and the beams are pushed by
// the CTA itself with the grid arrays the sweep left in shared memory. Instances with modes = 1 run
// the m = 1 sweep (qz_sweep_m1_body.cuh) with their own source scratch.
#include "qz_batch_kernels.cuh"

namespace qzb {

namespace {

template <int ORD>
int occ(bool m1, bool ext, size_t smem) { return batch_occupancy_ord<ORD>(m1, ext, smem); }

}  // namespace

int batch_max_grid(int ord, bool with_m1, bool with_ext, size_t smem, int* sms) {
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    *sms = nsm;
    int per = 0;
    switch (ord) {
        case 1: per = occ<1>(with_m1, with_ext, smem); break;
        case 2: per = occ<2>(with_m1, with_ext, smem); break;
        case 3: per = occ<3>(with_m1, with_ext, smem); break;
        case 4: per = occ<4>(with_m1, with_ext, smem); break;
        case 5: per = occ<5>(with_m1, with_ext, smem); break;
        default: return 0;
    }
    return per * nsm;
}

cudaError_t launch_batch(const BatchArgs& B, int grid, size_t smem, cudaStream_t s) {
    switch (B.ord) {
        case 1: return batch_launch_ord<1>(B, grid, smem, s);
        case 2: return batch_launch_ord<2>(B, grid, smem, s);
        case 3: return batch_launch_ord<3>(B, grid, smem, s);
        case 4: return batch_launch_ord<4>(B, grid, smem, s);
        case 5: return batch_launch_ord<5>(B, grid, smem, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace qzb
