// qz_sweep_m1w.cu -- the modes = 1 sweep for 513..1024 radial nodes (Simulation::step_fields with
// modes = 1, src/Simulation.cpp:636-795): the body of qz_sweep_m1_body.cuh compiled for CTAs of 1024
// threads, one radial node per thread, so that its block scans still run over the whole radial line.
//
// The sweep headers are compiled here with kSweepThreads = 1024 inside namespace qzb_w (the macro below
// renames the namespace), so none of their inline functions, built for 512 threads in the other units,
// is shared with this one. The library calls the kernels through launch_sweep_m1w, which takes the
// argument block as bytes (qzb::SweepArgs and qzb_w::SweepArgs are the same definition).
//
// At 1024 threads a thread has 64 registers (the 512-thread body uses 128), so the body keeps more of
// its state in local memory; shared memory holds 24 arrays of M doubles (192 KB at M = 1024).
#define QZ_SWEEP_THREADS 1024
#define qzb qzb_w
#include "qz_sweep_m1_body.cuh"

namespace qzb_w {

size_t sweep_m1_smem_bytes(int M) {
    return sizeof(double) * ((size_t)24 * M + 2 * 16 * (kSweepThreads / 32)) + 16;
}

namespace {
template <int ORD, bool EXT>
__global__ void __launch_bounds__(kSweepThreads, 1) sweep_m1w_kernel(const SweepArgs A) {
    extern __shared__ double smem_raw[];
    NoGate g;
    sweep_m1_body<ORD, NoGate, EXT>(A, smem_raw, g);
}

template <int ORD, bool EXT>
cudaError_t launch_e(const SweepArgs& A, size_t smem, cudaStream_t stream) {
    cudaError_t e = cudaFuncSetAttribute(sweep_m1w_kernel<ORD, EXT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    sweep_m1w_kernel<ORD, EXT><<<1, kSweepThreads, smem, stream>>>(A);
    return cudaGetLastError();
}

template <int ORD>
cudaError_t launch_t(const SweepArgs& A, size_t smem, cudaStream_t stream) {
    return (A.filter || A.bstat) ? launch_e<ORD, true>(A, smem, stream) : launch_e<ORD, false>(A, smem, stream);
}
}  // namespace

cudaError_t launch_sweep_m1(const SweepArgs& A, cudaStream_t stream) {
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

}  // namespace qzb_w

#undef qzb

namespace qzb {

size_t sweep_m1w_smem_bytes(int M) { return qzb_w::sweep_m1_smem_bytes(M); }

cudaError_t launch_sweep_m1w(const void* args, size_t args_size, cudaStream_t stream) {
    if (!args || args_size != sizeof(qzb_w::SweepArgs)) return cudaErrorInvalidValue;
    return qzb_w::launch_sweep_m1(*static_cast<const qzb_w::SweepArgs*>(args), stream);
}

}  // namespace qzb
