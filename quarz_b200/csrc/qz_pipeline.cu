// qz_pipeline.cu -- consecutive time steps of Simulation::run (src/Simulation.cpp:1370-1448) in one
// cooperative launch, so that the sequential xi sweeps of consecutive steps run concurrently on
// different SMs instead of one after another on one SM.
//
// Roles. CTAs [0, nsweep) run whole sweeps (qz_sweep_body.cuh), step n on CTA n % nsweep. In the other
// CTAs every warp is a worker: it claims (step, bucket) tasks that are ready and, per bucket, adds the
// moment sums of Beam::sums for that step, pushes the particles with that step's fields (Beam::push)
// and deposits them into the next step's beam sources (Beam::deposit), all in one pass.
//
// Ordering (every wait spins on an acquire load, bounded by %globaltimer; on time-out it records the
// place in *err and returns, and every other wait gives up as soon as *err is set):
//  - sweep n reads beam-source rows <= r only when every bucket whose initial lowest cell is <= r has
//    finished its push of step n-1 (particles only move to larger xi cells, so no other particle can
//    deposit into those rows);
//  - the push of (n, b) gathers rows <= cmax_b + 1 of step n's fields: it waits for sweep n to have
//    stored them, and for bucket b's push of step n-1 (the same particles);
//  - rings: sweep n writes field slot n % ring once the push of step n - ring is done; the sweep zeroes
//    each beam-source row when it no longer needs it, so that slot is clean for step n + ring, whose
//    depositors wait for sweep n to finish.
// A task is claimed only once it is ready, oldest step first, so workers never hold a task they
// wait on; sweeps wait only for pushes of older steps, so with all CTAs resident (cooperative launch)
// the waits cannot form a cycle. Data written by other SMs during the launch (fields, beam sources, particles, bucket bounds)
// is read with ld.global.cg, so that no stale L1 line is used.
#include "qz_pipeline_kernels.cuh"

#include <cub/device/device_radix_sort.cuh>

namespace qzb {

namespace {

// ---------------------------------------------------------------- ordering the beam by (xi cell, r cell)
// sort key of a particle: (xi cell + 1) * M + radial cell, removed particles last ((K + 2) * M): the
// xi cell orders the push tasks along the sweep, the radial cell puts particles that deposit into the
// same nodes next to each other (the deposit sums runs of equal cells across a warp)
__global__ void cell_keys_kernel(const BeamArgs B, unsigned* __restrict__ keys, int* __restrict__ vals,
                                 int* __restrict__ nlive) {
    int cnt = 0;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < B.n; i += stride) {
        const bool live = B.w[i] != 0.0;
        const double X = B.x[i], Y = B.y[i];
        const int jr = locate(B.r, B.N, B.R, sqrt(X * X + Y * Y));
        keys[i] = live ? (unsigned)(xi_cell(B, B.xi[i]) + 1) * (unsigned)B.M + (unsigned)jr
                       : (unsigned)(B.K + 2) * (unsigned)B.M;
        vals[i] = (int)i;
        cnt += live ? 1 : 0;
    }
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(nlive, cnt);
}

// dst = src permuted by idx (7 columns of n), orig_out = orig_in permuted the same way
__global__ void gather7_kernel(const double* __restrict__ src, double* __restrict__ dst, const int* __restrict__ idx,
                               const int* __restrict__ orig_in, int* __restrict__ orig_out, long n) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const long j = idx[p];
#pragma unroll
        for (int c = 0; c < 7; ++c) dst[c * n + p] = src[c * n + j];
        orig_out[p] = orig_in[j];
    }
}

// first sorted live particle of each group of xi cells: start[g] = first i with key >= g * width
// (width = span * M: keys sorted by (xi cell + 1) * M + radial cell), start[ngroups] = nlive
__global__ void group_starts_kernel(const unsigned* __restrict__ keys, long nlive, int width, int ngroups,
                                    int* __restrict__ start) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g > ngroups) return;
    if (g == ngroups) {
        start[g] = (int)nlive;
        return;
    }
    const unsigned key = (unsigned)g * (unsigned)width;
    long lo = 0, hi = nlive;                          // lower bound of key in keys[0, nlive)
    while (lo < hi) {
        const long mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1; else hi = mid;
    }
    start[g] = (int)lo;
}

__global__ void iota_kernel(int* __restrict__ p, long n) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = (int)i;
}

// dst[orig[p]] = src[p] for the 7 columns: back to the caller's particle order
__global__ void scatter7_kernel(const double* __restrict__ src, double* __restrict__ dst, const int* __restrict__ orig,
                                long n) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const long j = orig[p];
#pragma unroll
        for (int c = 0; c < 7; ++c) dst[c * n + j] = src[c * n + p];
    }
}

int grid_of(long n, int threads) {
    long b = (n + threads - 1) / threads;
    if (b > 148L * 8) b = 148L * 8;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

size_t cell_sort_temp_bytes(long n) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned*)nullptr, (unsigned*)nullptr, (const int*)nullptr,
                                    (int*)nullptr, (int)n, 0, 32);
    return bytes;
}

cudaError_t cell_sort(const BeamArgs& B, double* cols, double* stage, int* orig, int* orig_stage,
                      const CellSortBuf& buf, cudaStream_t s) {
    if (B.n <= 0) return cudaSuccess;
    const int n = (int)B.n;
    cudaError_t e = cudaMemsetAsync(buf.nlive, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    cell_keys_kernel<<<grid_of(n, 256), 256, 0, s>>>(B, buf.keys[0], buf.vals[0], buf.nlive);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int bits = 1;
    while (bits < 32 && (1ull << bits) <= (unsigned long long)(B.K + 2) * (unsigned long long)B.M) ++bits;
    size_t bytes = buf.tmp_bytes;
    e = cub::DeviceRadixSort::SortPairs(buf.tmp, bytes, buf.keys[0], buf.keys[1], buf.vals[0], buf.vals[1], n, 0, bits,
                                        s);
    if (e != cudaSuccess) return e;
    gather7_kernel<<<grid_of(n, 256), 256, 0, s>>>(cols, stage, buf.vals[1], orig, orig_stage, (long)n);
    return cudaGetLastError();
}

cudaError_t fill_iota(int* p, long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    iota_kernel<<<grid_of(n, 256), 256, 0, s>>>(p, n);
    return cudaGetLastError();
}

cudaError_t unpermute7(const double* src, double* dst, const int* orig, long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    scatter7_kernel<<<grid_of(n, 256), 256, 0, s>>>(src, dst, orig, n);
    return cudaGetLastError();
}

cudaError_t group_starts(const CellSortBuf& buf, long nlive, int width, int ngroups, int* start, cudaStream_t s) {
    group_starts_kernel<<<(ngroups + 1 + 127) / 128, 128, 0, s>>>(buf.keys[1], nlive, width, ngroups, start);
    return cudaGetLastError();
}

size_t pipeline_smem_bytes(int modes, int M, bool dbuf, bool const_smem, bool filter, int pcache) {
    const size_t sweep = modes == 1 ? sweep_m1_smem_bytes(M) : sweep_m0_smem_bytes(M, dbuf, const_smem, filter, pcache);
    const size_t worker = sizeof(double) * (4 * (size_t)M + (size_t)(kSweepThreads / 32) * 17 * 32) + 64;
    return sweep > worker ? sweep : worker;
}

int pipeline_max_grid(const PipeArgs& P, int* sms) {
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    *sms = nsm;
    const size_t smem = pipeline_smem_bytes(P.modes, P.sw.M, P.sw.dbuf, P.sw.const_smem, P.sw.filter != 0, P.sw.pcache);
    int per = 0;
    switch (P.sw.ord) {
        case 1: per = pipeline_occupancy_ord<1>(P, smem); break;
        case 2: per = pipeline_occupancy_ord<2>(P, smem); break;
        case 3: per = pipeline_occupancy_ord<3>(P, smem); break;
        case 4: per = pipeline_occupancy_ord<4>(P, smem); break;
        case 5: per = pipeline_occupancy_ord<5>(P, smem); break;
        default: return 0;
    }
    return per * nsm;
}

cudaError_t launch_pipeline(const PipeArgs& P, int grid, cudaStream_t stream) {
    if (P.sw.rows_per_thread < 1 || P.sw.rows_per_thread > 4) return cudaErrorInvalidValue;
    if (P.nsweep < 1 || grid <= P.nsweep || P.ring < 2 || P.nbeams > kMaxBeams) return cudaErrorInvalidValue;
    const size_t smem = pipeline_smem_bytes(P.modes, P.sw.M, P.sw.dbuf, P.sw.const_smem, P.sw.filter != 0, P.sw.pcache);
    switch (P.sw.ord) {
        case 1: return pipeline_launch_ord<1>(P, grid, smem, stream);
        case 2: return pipeline_launch_ord<2>(P, grid, smem, stream);
        case 3: return pipeline_launch_ord<3>(P, grid, smem, stream);
        case 4: return pipeline_launch_ord<4>(P, grid, smem, stream);
        case 5: return pipeline_launch_ord<5>(P, grid, smem, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_moments_reduce(const PipeArgs& P, double* mom, cudaStream_t s) {
    if (!P.pmom || P.nbeams < 1) return cudaSuccess;
    moments_reduce_kernel<<<(P.nsteps + 1) * P.nbeams, 32, 0, s>>>(P, mom);
    return cudaGetLastError();
}

}  // namespace qzb
