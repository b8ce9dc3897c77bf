// qz_beam.cu -- beam deposit, field gather + Vay push, and moment sums (sm_100a, FP64).
//
// Beam::deposit (src/Beam.cpp:725-785), Beam::advance with the Vay pusher (src/Beam.cpp:948-1131,
// src/Pushers.hpp:63-68) and Beam::sums (src/Beam.cpp:1133-1155). The particle arrays are SoA in
// HBM; one thread owns one particle per grid-stride step, so every load and store of the 7
// particle columns is coalesced. The field store is read through L2 (a bilinear gather of the
// (xi, r) cell, 4 x 6 doubles for m = 0); deposits are FP64 reductions into L2. The push can be
// fused with the deposit of the next time step (the particle is deposited right after it moved).
#include "qz_beam_body.cuh"

#include <atomic>
#include <mutex>

#include <cuda.h>

namespace qzb {

namespace {

using namespace beam_detail;
constexpr int kBeamThreads = 256;

__global__ void __launch_bounds__(kBeamThreads) beam_deposit_kernel(const BeamArgs B, double* __restrict__ bsrc) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < B.n; i += stride) {
        const double wi = B.w[i];
        if (wi == 0.0) continue;
        deposit_one(B, bsrc, B.x[i], B.y[i], B.px[i], B.py[i], B.pz[i], B.xi[i], wi);
    }
}

// the largest |w| of a beam (non-negative doubles order like their bit patterns, so an integer
// maximum of the bits is the maximum)
__global__ void __launch_bounds__(kBeamThreads) beam_wmax_kernel(const BeamArgs B, double* __restrict__ wmax) {
    const long stride = (long)gridDim.x * blockDim.x;
    double m = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < B.n; i += stride) m = fmax(m, fabs(B.w[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0)
        atomicMax(reinterpret_cast<unsigned long long*>(wmax), (unsigned long long)__double_as_longlong(m));
}

// e^{-z} I0(z), e^{-z} I1(z) by the polynomial approximations of Abramowitz & Stegun 9.8.1-9.8.4
// (relative error below 2e-7; the reference's choice, src/Beam.cpp:215-234)
__device__ __forceinline__ void bessel_i01_scaled(double z, double& i0, double& i1) {
    if (z < 3.75) {
        const double t = (z / 3.75) * (z / 3.75);
        const double I0 = 1.0 + t * (3.5156229 + t * (3.0899424 + t * (1.2067492 + t * (0.2659732
                          + t * (0.0360768 + t * 0.0045813)))));
        const double I1 = z * (0.5 + t * (0.87890594 + t * (0.51498869 + t * (0.15084934 + t * (0.02658733
                          + t * (0.00301532 + t * 0.00032411))))));
        const double e = exp(-z);
        i0 = I0 * e;
        i1 = I1 * e;
    } else {
        const double u = 3.75 / z, sq = 1.0 / sqrt(z);
        i0 = sq * (0.39894228 + u * (0.01328592 + u * (0.00225319 + u * (-0.00157565 + u * (0.00916281
             + u * (-0.02057706 + u * (0.02635537 + u * (-0.01647633 + u * 0.00392377))))))));
        i1 = sq * (0.39894228 + u * (-0.03988024 + u * (-0.00362018 + u * (0.00163801 + u * (-0.01031555
             + u * (0.02282967 + u * (-0.02895312 + u * (0.01787654 - u * 0.00420059))))))));
    }
}

// one thread per (slice, node): the displaced Gaussian's azimuthal modes 0 and 1 through the scaled Bessel
// functions of z = r d / sigma_r^2, added to rho, rho - J_z = (1 - v_z) rho and J_z = v_z rho
__global__ void __launch_bounds__(kBeamThreads) deposit_analytic_kernel(const AnalyticArgs P,
                                                                        double* __restrict__ bsrc) {
    const long n = (long)P.K * P.M;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        const int k = (int)(t / P.M), j = (int)(t - (long)k * P.M);
        const double xi = P.xi_min + k * P.dxi;
        if (xi < P.cut) continue;
        double fxi;
        if (P.flat) fxi = (fabs(xi - P.xi0) <= 0.5 * P.len) ? 1.0 : 0.0;
        else fxi = exp(-0.5 * (xi - P.xi0) * (xi - P.xi0) / (P.sxi * P.sxi));
        if (fxi == 0.0) continue;
        const double cx = P.x0 + P.xs * (xi - P.xi0), cy = P.y0 + P.ys * (xi - P.xi0);
        const double d = sqrt(cx * cx + cy * cy);
        const double r = P.r[j];
        double i0, i1;
        bessel_i01_scaled(r * d / P.s2, i0, i1);
        const double env = P.q * P.n0 * fxi * exp(-0.5 * (r - d) * (r - d) / P.s2);
        const double rho0 = env * i0;
        double* o = bsrc + (size_t)t * P.bnc;
        o[B_RHO0] += rho0;
        o[B_RT0] += rho0 * P.omvz;
        o[B_JZ0] += rho0 * P.vz;
        if (P.m1 && d > 0.0) {
            const double f1r = env * i1 * (cx / d), f1i = -env * i1 * (cy / d);
            o[B_RHO1R] += f1r; o[B_RHO1I] += f1i;
            o[B_RT1R] += f1r * P.omvz; o[B_RT1I] += f1i * P.omvz;
            o[B_JZ1R] += f1r * P.vz; o[B_JZ1I] += f1i * P.vz;
        }
    }
}

// Beam::slice_sums (src/Beam.cpp:1195-1217). Lanes of a warp that fall into the same bin in lane order
// (the library keeps beams in xi order after a pipelined run) are summed by a segmented shuffle scan first;
// the last lane of each run adds its 9 sums to L2 with FP64 atomics.
__global__ void __launch_bounds__(kBeamThreads) slice_sums_kernel(const BeamArgs B, double lo, double db, int nbins,
                                                                  double* __restrict__ out) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long stride = (long)gridDim.x * blockDim.x;
    const long nround = (B.n + 31) / 32 * 32;             // every lane of a warp runs the same iterations
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nround; i += stride) {
        double v[9];
        int key = -1 - lane;
        if (i < B.n && B.w[i] != 0.0) {
            const double w = B.w[i];
            const int b = (int)floor(((0.0 - B.xi[i]) - lo) / db);
            if (b >= 0 && b < nbins) {
                key = b;
                const double X = B.x[i], Y = B.y[i], PX = B.px[i], PY = B.py[i], PZ = B.pz[i];
                const double g = sqrt(1.0 + PX * PX + PY * PY + PZ * PZ);
                v[0] = w; v[1] = w * X; v[2] = w * Y; v[3] = w * (X * X); v[4] = w * (Y * Y); v[5] = w * g;
                v[6] = w * PX; v[7] = w * (PX * PX); v[8] = w * (X * PX);
            }
        }
        if (key < 0)
#pragma unroll
            for (int c = 0; c < 9; ++c) v[c] = 0.0;
        const int kprev = __shfl_up_sync(FULL, key, 1);
        const bool head = lane == 0 || kprev != key;
        const int seg = __popc(__ballot_sync(FULL, head) & (FULL >> (31 - lane)));
#pragma unroll
        for (int st = 1; st < 32; st <<= 1) {
            const int sp = __shfl_up_sync(FULL, seg, st);
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                const double vp = __shfl_up_sync(FULL, v[c], st);
                if (lane >= st && sp == seg) v[c] += vp;
            }
        }
        const int knext = __shfl_down_sync(FULL, key, 1);
        if (key >= 0 && (lane == 31 || knext != key))
#pragma unroll
            for (int c = 0; c < 9; ++c) atomicAdd(out + 9 * (size_t)key + c, v[c]);
    }
}

template <bool kDeposit>
__global__ void __launch_bounds__(kBeamThreads) beam_push_kernel(const BeamArgs B, const double* __restrict__ fld,
                                                                 double dt_kick, double dt, int move,
                                                                 double* __restrict__ bsrc_next) {
    const double qm = B.q / B.m;
    const double xmin = B.xi_min, xmax = B.xi_min + (B.K - 1) * B.dxi;
    const double R = B.R;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < B.n; i += stride) {
        const double wi = B.w[i];
        if (wi == 0.0) continue;
        const double X = B.x[i], Y = B.y[i], XI = B.xi[i];
        double c, sn;
        V3 E, Bf;
        gather<false>(B, fld, X, Y, XI, c, sn, E, Bf);
        V3 u = {B.px[i], B.py[i], B.pz[i]};
        const double h = 0.5 * qm * dt_kick;
        if (!move) {                 // leapfrog start-up: explicit kick (src/Beam.cpp:1038-1044)
            const double g0 = sqrt(1.0 + dot3(u, u));
            const double ig = 1.0 / g0;
            const V3 v = {ig * u.x, ig * u.y, ig * u.z};
            const V3 vxb = cross3(v, Bf);
            const double h2 = 2.0 * h;
            u = {u.x + h2 * (E.x + vxb.x), u.y + h2 * (E.y + vxb.y), u.z + h2 * (E.z + vxb.z)};
            B.px[i] = u.x; B.py[i] = u.y; B.pz[i] = u.z;
            continue;
        }
        u = B.pusher ? push_u(B.pusher, u, E, Bf, h) : vay(u, E, Bf, h);
        const double p2 = u.x * u.x + u.y * u.y;
        const double gam = sqrt(1.0 + p2 + u.z * u.z);
        const double omvz = (1.0 + p2) / (gam * (gam + u.z));
        const double xn = X + u.x / gam * dt, yn = Y + u.y / gam * dt;
        const double xin = XI + omvz * dt;
        B.x[i] = xn; B.y[i] = yn;
        B.px[i] = u.x; B.py[i] = u.y; B.pz[i] = u.z;
        B.xi[i] = xin;
        double wn = wi;
        if (xn * xn + yn * yn >= R * R || xin < xmin || xin > xmax) { wn = 0.0; B.w[i] = 0.0; }
        if (kDeposit && wn != 0.0) deposit_one(B, bsrc_next, xn, yn, u.x, u.y, u.z, xin, wn);
    }
}

// moment sums: fixed grid, fixed per-thread order, fixed tree -> deterministic
constexpr int kSumThreads = 256;

__global__ void __launch_bounds__(kSumThreads) beam_sums_partial(const BeamArgs B, double gref, double xiref,
                                                                 double* __restrict__ partial) {
    double acc[17];
#pragma unroll
    for (int c = 0; c < 17; ++c) acc[c] = 0.0;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < B.n; i += stride) {
        const double w = B.w[i];
        if (w == 0.0) continue;
        const double PX = B.px[i], PY = B.py[i], PZ = B.pz[i], X = B.x[i], Y = B.y[i];
        const double g = sqrt(1.0 + PX * PX + PY * PY + PZ * PZ);
        const double G = g - gref, XI = B.xi[i] - xiref;
        const double v[15] = {G, G * G, XI, XI * XI, X * X + Y * Y, X, Y, X * X, Y * Y,
                              PX, PY, PX * PX, PY * PY, X * PX, Y * PY};
        acc[16] += 1.0;
        acc[0] += w;
#pragma unroll
        for (int c = 0; c < 15; ++c) acc[c + 1] += w * v[c];
    }
    __shared__ double red[17][kSumThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 17; ++c) {
        double v = acc[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[c][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 17) {
        double v = 0.0;
        for (int w = 0; w < kSumThreads / 32; ++w) v += red[threadIdx.x][w];
        partial[(size_t)blockIdx.x * 17 + threadIdx.x] = v;
    }
}

__global__ void beam_sums_final(const double* __restrict__ partial, int nblocks, double* __restrict__ out17) {
    const int c = threadIdx.x;
    if (c >= 17) return;
    double v = 0.0;
    for (int b = 0; b < nblocks; ++b) v += partial[(size_t)b * 17 + c];
    out17[c] = v;
}

int grid_for(long n) {
    long b = (n + kBeamThreads - 1) / kBeamThreads;
    const long cap = 148L * 8;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

}  // namespace

int beam_sums_blocks(long n) {
    long b = (n + kSumThreads - 1) / kSumThreads;
    if (b > 148L * 4) b = 148L * 4;
    if (b < 1) b = 1;
    return (int)b;
}

cudaError_t launch_beam_deposit(const BeamArgs& B, double* bsrc, cudaStream_t s) {
    if (B.n <= 0) return cudaSuccess;
    beam_deposit_kernel<<<grid_for(B.n), kBeamThreads, 0, s>>>(B, bsrc);
    return cudaGetLastError();
}

cudaError_t launch_beam_wmax(const BeamArgs& B, double* wmax, cudaStream_t s) {
    if (B.n <= 0) return cudaSuccess;
    beam_wmax_kernel<<<grid_for(B.n), kBeamThreads, 0, s>>>(B, wmax);
    return cudaGetLastError();
}

cudaError_t launch_slice_sums(const BeamArgs& B, double lo, double db, int nbins, double* out, cudaStream_t s) {
    if (B.n <= 0) return cudaSuccess;
    slice_sums_kernel<<<grid_for(B.n), kBeamThreads, 0, s>>>(B, lo, db, nbins, out);
    return cudaGetLastError();
}

cudaError_t launch_deposit_analytic(const AnalyticArgs& P, double* bsrc, cudaStream_t s) {
    const long n = (long)P.K * P.M;
    if (n <= 0) return cudaSuccess;
    deposit_analytic_kernel<<<grid_for(n), kBeamThreads, 0, s>>>(P, bsrc);
    return cudaGetLastError();
}

cudaError_t launch_beam_push(const BeamArgs& B, const double* fld, double dt_kick, double dt_drift, int move,
                             cudaStream_t s) {
    if (B.n <= 0) return cudaSuccess;
    beam_push_kernel<false><<<grid_for(B.n), kBeamThreads, 0, s>>>(B, fld, dt_kick, dt_drift, move, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_beam_push_deposit(const BeamArgs& B, const double* fld, double dt_kick, double dt_drift,
                                     double* bsrc_next, cudaStream_t s) {
    if (B.n <= 0) return cudaSuccess;
    beam_push_kernel<true><<<grid_for(B.n), kBeamThreads, 0, s>>>(B, fld, dt_kick, dt_drift, 1, bsrc_next);
    return cudaGetLastError();
}

cudaError_t launch_beam_sums(const BeamArgs& B, double gref, double xiref, double* partial, int nblocks,
                             double* out17, cudaStream_t s) {
    beam_sums_partial<<<nblocks, kSumThreads, 0, s>>>(B, gref, xiref, partial);
    beam_sums_final<<<1, 32, 0, s>>>(partial, nblocks, out17);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- context identity
// The unique id of the CUDA context current on this thread (cuCtxGetId), or 0 when there is none
// or the driver cannot tell. Device memory and the addresses of a module's static arrays belong to
// one context: a cudaDeviceReset ends it, and the next runtime call creates a new one with a new
// id. Addresses cached per device are therefore cached together with this id. The driver entry
// points are fetched through the runtime, so the library does not link libcuda.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    if (get_current(&c) != CUDA_SUCCESS || c == nullptr) return 0;
    unsigned long long id = 0;
    if (get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// ---------------------------------------------------------------- moment sums without allocation
// Partial-sum scratch of beam_sums_static in static device memory: one 17-double row per block of
// beam_sums_partial, sized for the block cap of beam_sums_blocks (148 x 4 blocks, 80,512 bytes per
// device). Every row the final reduction reads is written by the same call first, so nothing in it
// has to start at zero; two calls in flight at once on one device (other streams, other host
// threads) share it and race.
static __device__ __align__(256) double g_sums_static[17 * kSumsStaticBlocks];

constexpr int kMaxDevices = 64;

namespace {
struct StaticAddr {
    std::atomic<unsigned long long> ctx{0};     // context the address was looked up in
    std::atomic<double*> ptr{nullptr};
};
StaticAddr g_static[kMaxDevices];
std::mutex g_static_mu;
}  // namespace

cudaError_t beam_sums_static(const BeamArgs& B, double gref, double xiref, double* out17, cudaStream_t s,
                             int* nblocks_needed) {
    const int nb = beam_sums_blocks(B.n);
    *nblocks_needed = nb;
    // beam_sums_blocks caps the grid at the array's row count and the partial kernel strides over
    // the particles, so this holds for every n; it guards that invariant
    if (nb > kSumsStaticBlocks) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    StaticAddr& a = g_static[dev];
    // fast path: the address was looked up in the context that is current now
    unsigned long long ctx = current_context_id();
    double* partial = nullptr;
    if (ctx != 0 && a.ctx.load(std::memory_order_acquire) == ctx) {
        partial = a.ptr.load(std::memory_order_relaxed);
    } else {
        // set-up, once per device and context, with that device current: the address of this
        // device's copy of the static scratch (no allocation; the module's static memory exists
        // once the module is loaded). A cudaDeviceReset ends the context, and with it the
        // address; the next call looks it up again in the new context.
        std::lock_guard<std::mutex> lock(g_static_mu);
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sums_static);
        if (e != cudaSuccess) return e;
        partial = static_cast<double*>(p);
        ctx = current_context_id();           // the lookup made the device's primary context current
        if (ctx != 0) {
            a.ptr.store(partial, std::memory_order_relaxed);
            a.ctx.store(ctx, std::memory_order_release);
        }
    }
    return launch_beam_sums(B, gref, xiref, partial, nb, out17, s);
}

}  // namespace qzb
