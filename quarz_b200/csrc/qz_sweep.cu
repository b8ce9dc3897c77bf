// qz_sweep.cu -- stand-alone sweep launch: one CTA runs the whole xi sweep of one time step
// (the sweep itself is in qz_sweep_body.cuh).
#include "qz_sweep_body.cuh"

namespace qzb {

// EXT: the variant for decks with the smoothing filter or static (analytic) beam sources
template <int ORD, bool REG, int kMaxR, bool EXT>
__global__ void __launch_bounds__(kSweepThreads, 1) sweep_m0_kernel(const SweepArgs A) {
    extern __shared__ double smem_raw[];
    NoGate g;
    sweep_body<ORD, REG, kMaxR, NoGate, EXT>(A, smem_raw, g);
}

size_t sweep_m0_smem_bytes(int M, bool dbuf, bool const_smem, bool filter, int pcache) {
    size_t d = (size_t)(3 + 2 + 6 + (dbuf ? 18 : 9)) * M + 2 * 8 * (kSweepThreads / 32);
    if (const_smem) d += 13 * (size_t)M;
    if (filter) d += 4 * (size_t)M + 2 * 14 * (kSweepThreads / 32);
    // + lost, flag, 14 exponent maxima and counters, the cells-crossed word (128 B with the particle copy
    // behind them: 6 doubles and a cell index per particle)
    if (pcache > 0) return sizeof(double) * d + 128 + (size_t)pcache * (6 * sizeof(double) + sizeof(int));
    return sizeof(double) * d + 16 + 4 * 16;
}

namespace {
template <int ORD, bool REG, int RM, bool EXT>
cudaError_t launch_t(const SweepArgs& A, size_t smem, cudaStream_t stream) {
    cudaError_t e = cudaFuncSetAttribute(sweep_m0_kernel<ORD, REG, RM, EXT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    sweep_m0_kernel<ORD, REG, RM, EXT><<<1, kSweepThreads, smem, stream>>>(A);
    return cudaGetLastError();
}

template <int ORD, bool EXT>
cudaError_t launch_e(const SweepArgs& A, size_t smem, cudaStream_t stream) {
    const bool reg = A.np <= kSweepThreads;
    if (A.rows_per_thread == 1)
        return reg ? launch_t<ORD, true, 1, EXT>(A, smem, stream) : launch_t<ORD, false, 1, EXT>(A, smem, stream);
    return reg ? launch_t<ORD, true, 4, EXT>(A, smem, stream) : launch_t<ORD, false, 4, EXT>(A, smem, stream);
}

template <int ORD>
cudaError_t launch_o(const SweepArgs& A, size_t smem, cudaStream_t stream) {
    return (A.filter || A.bstat) ? launch_e<ORD, true>(A, smem, stream) : launch_e<ORD, false>(A, smem, stream);
}
}  // namespace

cudaError_t launch_sweep_m0(const SweepArgs& A, cudaStream_t stream) {
    if (A.rows_per_thread < 1 || A.rows_per_thread > 4) return cudaErrorInvalidValue;
    const size_t smem = sweep_m0_smem_bytes(A.M, A.dbuf, A.const_smem, A.filter != 0, A.pcache);
    switch (A.ord) {
        case 1: return launch_o<1>(A, smem, stream);
        case 2: return launch_o<2>(A, smem, stream);
        case 3: return launch_o<3>(A, smem, stream);
        case 4: return launch_o<4>(A, smem, stream);
        case 5: return launch_o<5>(A, smem, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace qzb
