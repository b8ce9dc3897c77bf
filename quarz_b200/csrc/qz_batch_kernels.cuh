#pragma once
// qz_batch_kernels.cuh -- many independent runs (a parameter scan) in one persistent launch.
//
// Each CTA takes the next instance from a queue (largest first) and runs all of it as
// Simulation::run does (src/Simulation.cpp:1370-1448): the step-0 beam deposit, then per step the
// sweep (qz_sweep_body.cuh), the moment sums of every beam (Beam::sums, src/Beam.cpp:1133-1155) and,
// before the last sweep, the push of every beam with the next deposit (src/Beam.cpp:725-785,
// :900-1131). Instances differ in grid, box, plasma and beams; their sweep arguments are copied into
// shared memory, the field and beam-source buffers are the CTA's slot, and the beams are pushed by
// the CTA itself with the grid arrays the sweep left in shared memory. Instances with modes = 1 run
// the m = 1 sweep (qz_sweep_m1_body.cuh) with their own source scratch.
#include "qz_beam_body.cuh"
#include "qz_sweep_body.cuh"
#include "qz_sweep_m1_body.cuh"

namespace qzb {

namespace {

using beam_detail::deposit_one;
using beam_detail::PState7;
using beam_detail::push_one;
using beam_detail::sums_add;

constexpr int kT = kSweepThreads;

__device__ __forceinline__ unsigned long long batch_timer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// beam work of one instance by the whole CTA: moments (step n) of every beam, then, when push,
// the push with the fields of step n and the deposit into bsrc (zeroed first)
__device__ void beam_phase(const BatchInst& I, const SweepArgs& A, const BatchArgs& B, int n, bool push, bool startup,
                           double* red) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (push) {
        const size_t nb = (size_t)A.K * A.M * (I.modes ? B_NC1 : B_NC0);
        for (size_t t = tid; t < nb; t += kT) const_cast<double*>(A.bsrc)[t] = 0.0;
        __syncthreads();
    }
    // the sweep leaves the grid in shared memory (qz_sweep_body.cuh carve: r, 1/V, 1/h first)
    extern __shared__ double smem_raw[];
    const double* r = smem_raw;
    const double* iV = smem_raw + A.M;
    const double* ih = smem_raw + 2 * A.M;
    for (int q = 0; q < I.nbeams; ++q) {
        BeamArgs Bb = I.beam[q];
        Bb.r = r;
        Bb.inv_V = iV;
        Bb.inv_h = ih;
        const double qm = Bb.q / Bb.m;
        const double h = 0.5 * qm * B.dt;
        const double hs = startup ? 0.5 * qm * (-0.5 * B.dt) : 0.0;
        double acc[17];
#pragma unroll
        for (int c = 0; c < 17; ++c) acc[c] = 0.0;
        for (long i = tid; i < Bb.n; i += kT) {
            PState7 p;
            p.w = Bb.w[i];
            if (p.w == 0.0) continue;
            p.x = Bb.x[i]; p.y = Bb.y[i]; p.px = Bb.px[i]; p.py = Bb.py[i]; p.pz = Bb.pz[i]; p.xi = Bb.xi[i];
            sums_add(acc, p, I.gref[q], I.xiref[q]);
            if (!push) continue;
            if (I.rigid[q]) {
                deposit_one(Bb, const_cast<double*>(A.bsrc), p.x, p.y, p.px, p.py, p.pz, p.xi, p.w);
                continue;
            }
            const bool alive = push_one<false>(Bb, A.fld, p, h, hs, B.dt);
            Bb.x[i] = p.x; Bb.y[i] = p.y; Bb.px[i] = p.px; Bb.py[i] = p.py; Bb.pz[i] = p.pz; Bb.xi[i] = p.xi;
            if (!alive) {
                Bb.w[i] = 0.0;
                continue;
            }
            deposit_one(Bb, const_cast<double*>(A.bsrc), p.x, p.y, p.px, p.py, p.pz, p.xi, p.w);
        }
        // deterministic block reduction of the 17 sums
#pragma unroll
        for (int c = 0; c < 17; ++c) {
            double x = acc[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) red[c * (kT / 32) + warp] = x;
        }
        __syncthreads();
        if (tid < 17) {
            double v = 0.0;
            for (int w = 0; w < kT / 32; ++w) v += red[tid * (kT / 32) + w];
            I.mom[((size_t)n * I.nbeams + q) * 17 + tid] = v;
        }
        __syncthreads();
    }
}

// the step-0 deposit of every beam into the (zeroed) slot
__device__ void beam_deposit0(const BatchInst& I, const SweepArgs& A) {
    const int tid = threadIdx.x;
    const size_t nb = (size_t)A.K * A.M * (I.modes ? B_NC1 : B_NC0);
    for (size_t t = tid; t < nb; t += kT) const_cast<double*>(A.bsrc)[t] = 0.0;
    __syncthreads();
    for (int q = 0; q < I.nbeams; ++q) {
        const BeamArgs& Bb = I.beam[q];
        for (long i = tid; i < Bb.n; i += kT) {
            const double w = Bb.w[i];
            if (w == 0.0) continue;
            deposit_one(Bb, const_cast<double*>(A.bsrc), Bb.x[i], Bb.y[i], Bb.px[i], Bb.py[i], Bb.pz[i], Bb.xi[i], w);
        }
    }
    __syncthreads();
}

// WITH_M1: the batch holds modes = 1 instances (the m = 0 only variant keeps the m = 1 body out of the
// kernel and its register allocation)
// EXT: the variant whose sweeps handle the smoothing filter (some instance has plasma.smooth_length)
template <int ORD, bool WITH_M1, bool EXT>
__global__ void __launch_bounds__(kSweepThreads, 1) batch_kernel(const __grid_constant__ BatchArgs B) {
    extern __shared__ double smem_raw[];
    __shared__ BatchInst I;
    __shared__ int s_inst;
    __shared__ double red[17 * (kT / 32)];
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_inst = atomicAdd(B.next, 1);
        __syncthreads();
        const int qi = s_inst;
        if (qi >= B.ninst) break;
        if (tid == 0) {
            I = B.inst[B.order[qi]];
            I.sw.bsrc = B.bsrc + blockIdx.x * B.bsrc_slot;
            I.sw.fld = B.fld + blockIdx.x * B.fld_slot;
            I.sw.diag = B.diag + blockIdx.x * B.diag_slot;
            I.sw.timing = nullptr;
        }
        __syncthreads();
        const SweepArgs& A = I.sw;
        const bool reg = A.np <= kSweepThreads;
        (void)reg;
        unsigned long long t_start = 0, t_mark = 0, t_sweep = 0, t_beam = 0;
        if (B.trace && tid == 0) t_start = t_mark = batch_timer();
        beam_deposit0(I, A);
        for (int n = 0; n <= B.nsteps; ++n) {
            if (B.trace && tid == 0) { const unsigned long long t = batch_timer(); t_beam += t - t_mark; t_mark = t; }
            NoGate g;
            if (WITH_M1 && I.modes) {
                if constexpr (WITH_M1) sweep_m1_body<ORD, NoGate, EXT>(A, smem_raw, g);
            } else if constexpr (kSweepThreads == 512) {     // (the 1024-thread build runs m = 1 only)
                if (A.rows_per_thread == 1) {
                    if (reg) sweep_body<ORD, true, 1, NoGate, EXT>(A, smem_raw, g);
                    else sweep_body<ORD, false, 1, NoGate, EXT>(A, smem_raw, g);
                } else {
                    sweep_body<ORD, false, 4, NoGate, EXT>(A, smem_raw, g);
                }
            }
            __syncthreads();
            if (B.trace && tid == 0) { const unsigned long long t = batch_timer(); t_sweep += t - t_mark; t_mark = t; }
            beam_phase(I, A, B, n, n < B.nsteps, n == 0, red);
        }
        __syncthreads();
        if (B.trace && tid == 0) {
            const unsigned long long t = batch_timer();
            unsigned long long* o = B.trace + (size_t)B.order[qi] * kBatchTrace;
            o[0] = blockIdx.x; o[1] = t_start; o[2] = t; o[3] = t_sweep; o[4] = t_beam + (t - t_mark);
        }
    }
}

template <int ORD, bool WITH_M1, bool EXT>
cudaError_t launch_t(const BatchArgs& B, int grid, size_t smem, cudaStream_t s) {
    cudaError_t e =
        cudaFuncSetAttribute(batch_kernel<ORD, WITH_M1, EXT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    batch_kernel<ORD, WITH_M1, EXT><<<grid, kSweepThreads, smem, s>>>(B);
    return cudaGetLastError();
}

template <int ORD, bool WITH_M1, bool EXT>
int occupancy_t(size_t smem) {
    if (cudaFuncSetAttribute(batch_kernel<ORD, WITH_M1, EXT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batch_kernel<ORD, WITH_M1, EXT>, kSweepThreads, smem) !=
        cudaSuccess)
        return 0;
    return nb;
}

}  // namespace

// the batch kernel of one Adams-Bashforth order (with / without modes = 1 instances, with / without the
// smoothing filter), defined by qz_batch_o<ORD>.cu: one translation unit per order, built in parallel
template <int ORD>
cudaError_t batch_launch_ord(const BatchArgs& B, int grid, size_t smem, cudaStream_t s);
template <int ORD>
int batch_occupancy_ord(bool with_m1, bool with_ext, size_t smem);

}  // namespace qzb
