// qz_beam.cu -- beam deposit, field gather + Vay push, and moment sums (sm_100a, FP64).
//
// Beam::deposit (src/Beam.cpp:725-785), Beam::advance with the Vay pusher (src/Beam.cpp:948-1131,
// src/Pushers.hpp:171-176) and Beam::sums (src/Beam.cpp:1133-1155). The particle arrays are SoA in
// HBM; one thread owns one particle per grid-stride step, so every load and store of the 7
// particle columns is coalesced. The field store is read through L2 (a bilinear gather of the
// (xi, r) cell, 4 x 6 doubles for m = 0); deposits are FP64 reductions into L2. The push can be
// fused with the deposit of the next time step (the particle is deposited right after it moved).
#include "qz_device.cuh"
#include "qz_internal.h"

#include <mutex>

namespace qzb {

namespace {

constexpr int kBeamThreads = 256;

__device__ __forceinline__ void deposit_one(const BeamArgs& B, double* __restrict__ bsrc, double X, double Y,
                                            double PX, double PY, double PZ, double XI, double wi) {
    const double R = B.R;
    const double r = sqrt(X * X + Y * Y);
    if (r > R) return;
    const double c = r > 0.0 ? X / r : 1.0, s = r > 0.0 ? Y / r : 0.0;
    const double sx = (XI - B.xi_min) * B.idxi;
    const int k = B.ngp ? (int)floor(sx + 0.5) : (int)floor(sx);
    const int nloc = B.K;
    if (k < -1 || k >= nloc) return;
    const double tk = B.ngp ? 0.0 : sx - k;
    const double p2 = PX * PX + PY * PY;
    const double gam = sqrt(1.0 + p2 + PZ * PZ);
    const double omvz = (1.0 + p2) / (gam * (gam + PZ));
    const double vz = PZ / gam, vx = PX / gam, vy = PY / gam;
    const double vr = c * vx + s * vy, vt = c * vy - s * vx;
    int j;
    double t;
    weights(B.r, B.inv_h, B.N, R, r, j, t);
    const double Wr[2] = {1.0 - t, t};
    const double Wk[2] = {1.0 - tk, tk};
    const double q = B.q;
    const int nc = B.modes ? B_NC1 : B_NC0;
    const int na = B.ngp ? 1 : 2;
    for (int a = 0; a < na; ++a) {
        const int kk = k + a;
        if (kk < 0 || kk >= nloc) continue;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int jj = j + b;
            double* o = bsrc + ((size_t)kk * B.M + jj) * nc;
            const double d = wi * q * Wk[a] * Wr[b] * B.inv_V[jj] * B.idxi;
            atomicAdd(o + B_RT0, d * omvz);
            atomicAdd(o + B_JZ0, d * vz);
            atomicAdd(o + B_JP1R, d * vr);
            atomicAdd(o + B_JP1I, d * vt);
            atomicAdd(o + B_RHO0, d);
            if (B.modes) {
                atomicAdd(o + B_RT1R, d * omvz * c);
                atomicAdd(o + B_RT1I, -d * omvz * s);
                atomicAdd(o + B_JZ1R, d * vz * c);
                atomicAdd(o + B_JZ1I, -d * vz * s);
                atomicAdd(o + B_RHO1R, d * c);
                atomicAdd(o + B_RHO1I, -d * s);
                atomicAdd(o + B_JP0R, d * vx);
                atomicAdd(o + B_JP0I, d * vy);
                const double c2 = c * c - s * s, s2 = 2.0 * c * s;
                atomicAdd(o + B_JP2R, d * (vx * c2 + vy * s2));
                atomicAdd(o + B_JP2I, d * (vy * c2 - vx * s2));
            }
        }
    }
}

__global__ void __launch_bounds__(kBeamThreads) beam_deposit_kernel(const BeamArgs B, double* __restrict__ bsrc) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < B.n; i += stride) {
        const double wi = B.w[i];
        if (wi == 0.0) continue;
        deposit_one(B, bsrc, B.x[i], B.y[i], B.px[i], B.py[i], B.pz[i], B.xi[i], wi);
    }
}

// bilinear (xi, r) gather and mode sums at the particle (src/Beam.cpp:972-1008)
__device__ __forceinline__ void gather(const BeamArgs& B, const double* __restrict__ fld, double X, double Y,
                                       double XI, double& c, double& sn, V3& E, V3& Bf) {
    const double r = sqrt(X * X + Y * Y);
    c = r > 0.0 ? X / r : 1.0;
    sn = r > 0.0 ? Y / r : 0.0;
    double s = (XI - B.xi_min) * B.idxi;
    const int nloc = B.K;
    int k;
    double tk;
    if (B.ngp) {
        k = (int)floor(s + 0.5);
        k = k < 0 ? 0 : (k > nloc - 1 ? nloc - 1 : k);
        tk = 0.0;
    } else {
        k = (int)floor(s);
        if (k < 0) { k = 0; s = 0.0; }
        if (k > nloc - 2) { k = nloc - 2; s = nloc - 1; }
        tk = s - k;
    }
    const int k1 = B.ngp ? k : k + 1;
    int j;
    double t;
    weights(B.r, B.inv_h, B.N, B.R, r, j, t);
    const int nc = B.modes ? F_NC1 : F_NC0;
    const double* f00 = fld + ((size_t)k * B.M + j) * nc;
    const double* f01 = f00 + nc;
    const double* f10 = fld + ((size_t)k1 * B.M + j) * nc;
    const double* f11 = f10 + nc;
    auto bil = [&](int comp) {
        return (1.0 - tk) * ((1.0 - t) * f00[comp] + t * f01[comp]) + tk * ((1.0 - t) * f10[comp] + t * f11[comp]);
    };
    if (B.modes) {
        // eval_vector / eval_scalar with m = 1 (src/SliceData.hpp:70-83)
        const double c2 = c * c - sn * sn, s2 = 2.0 * c * sn;
        {
            const double r0 = bil(F_EP0R), i0 = bil(F_EP0I), r1 = bil(F_EP1R), i1 = bil(F_EP1I);
            const double r2 = bil(F_EP2R), i2 = bil(F_EP2I);
            E.x = r1 * c - i1 * sn;
            E.y = r1 * sn + i1 * c;
            E.x += r0 + r2 * c2 - i2 * s2;
            E.y += i0 + r2 * s2 + i2 * c2;
        }
        {
            const double r0 = bil(F_BP0R), i0 = bil(F_BP0I), r1 = bil(F_BP1R), i1 = bil(F_BP1I);
            const double r2 = bil(F_BP2R), i2 = bil(F_BP2I);
            Bf.x = r1 * c - i1 * sn;
            Bf.y = r1 * sn + i1 * c;
            Bf.x += r0 + r2 * c2 - i2 * s2;
            Bf.y += i0 + r2 * s2 + i2 * c2;
        }
        E.z = bil(F_EZ0) + 2.0 * (bil(F_EZ1R) * c - bil(F_EZ1I) * sn);
        Bf.z = bil(F_BZ0) + 2.0 * (bil(F_BZ1R) * c - bil(F_BZ1I) * sn);
    } else {
        const double er = bil(F_EP1R), ei = bil(F_EP1I), br = bil(F_BP1R), bi = bil(F_BP1I);
        E.x = er * c - ei * sn;
        E.y = er * sn + ei * c;
        Bf.x = br * c - bi * sn;
        Bf.y = br * sn + bi * c;
        E.z = bil(F_EZ0);
        Bf.z = bil(F_BZ0);
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
        gather(B, fld, X, Y, XI, c, sn, E, Bf);
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
        u = vay(u, E, Bf, h);
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

// ---------------------------------------------------------------- moment sums without allocation
// Partial-sum scratch of beam_sums_static in static device memory: one 17-double row per block of
// beam_sums_partial, sized for the block cap of beam_sums_blocks (148 x 4 blocks, 80,512 bytes per
// device). Every row the final reduction reads is written by the same call first, so nothing in it
// has to start at zero; two calls in flight at once on one device (other streams, other host
// threads) share it and race.
static __device__ __align__(256) double g_sums_static[17 * kSumsStaticBlocks];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
double* g_static_ptr[kMaxDevices] = {};
}  // namespace

cudaError_t beam_sums_static(const BeamArgs& B, double gref, double xiref, double* out17, cudaStream_t s,
                             int* nblocks_needed) {
    const int nb = beam_sums_blocks(B.n);
    *nblocks_needed = nb;
    if (nb > kSumsStaticBlocks) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    double* partial = nullptr;
    {
        // set-up, once per device, with that device current: the address of this device's copy
        // of the static scratch (no allocation; the module's static memory already exists)
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (!g_static_ptr[dev]) {
            void* ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_sums_static);
            if (e != cudaSuccess) return e;
            g_static_ptr[dev] = static_cast<double*>(ptr);
        }
        partial = g_static_ptr[dev];
    }
    return launch_beam_sums(B, gref, xiref, partial, nb, out17, s);
}

}  // namespace qzb
