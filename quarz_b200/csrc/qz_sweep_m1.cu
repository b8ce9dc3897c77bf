// qz_sweep_m1.cu -- stand-alone launch of the modes = 1 sweep (qz_sweep_m1_body.cuh): one CTA runs
// the whole xi sweep of one time step.
#include "qz_sweep_m1_body.cuh"

namespace qzb {

size_t sweep_m1_smem_bytes(int M) {
    return sizeof(double) * ((size_t)24 * M + 2 * 16 * (kSweepThreads / 32)) + 16;
}

namespace {
// EXT: the variant for decks with the smoothing filter or static (analytic) beam sources
template <int ORD, bool EXT>
__global__ void __launch_bounds__(kSweepThreads, 1) sweep_m1_kernel(const SweepArgs A) {
    extern __shared__ double smem_raw[];
    NoGate g;
    sweep_m1_body<ORD, NoGate, EXT>(A, smem_raw, g);
}

template <int ORD, bool EXT>
cudaError_t launch_e(const SweepArgs& A, size_t smem, cudaStream_t stream) {
    cudaError_t e = cudaFuncSetAttribute(sweep_m1_kernel<ORD, EXT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    sweep_m1_kernel<ORD, EXT><<<1, kSweepThreads, smem, stream>>>(A);
    return cudaGetLastError();
}

template <int ORD>
cudaError_t launch_t(const SweepArgs& A, size_t smem, cudaStream_t stream) {
    return (A.filter || A.bstat) ? launch_e<ORD, true>(A, smem, stream) : launch_e<ORD, false>(A, smem, stream);
}
}  // namespace

cudaError_t launch_sweep_m1(const SweepArgs& A, cudaStream_t stream) {
    if (A.M > kSweepThreads && A.M <= 2 * kSweepThreads) return launch_sweep_m1w(&A, sizeof(A), stream);
    if (A.M > kSweepThreads || A.M < 3) return cudaErrorInvalidValue;
    const size_t smem = sweep_m1_smem_bytes(A.M);
    switch (A.ord) {
        case 1: return launch_t<1>(A, smem, stream);
        case 2: return launch_t<2>(A, smem, stream);
        case 3: return launch_t<3>(A, smem, stream);
        case 4: return launch_t<4>(A, smem, stream);
        case 5: return launch_t<5>(A, smem, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace qzb
