// qz_device.cuh -- device helpers shared by the sweep and beam kernels (sm_100a, FP64).
//
// Layout conventions are the reference's (QUARZ v2.0.0):
//   field store  fld(k, j, c)   LayoutRight, c fastest   src/FieldStore.hpp:9-13, src/Simulation.cpp:179
//   beam sources bsrc(k, j, c)  LayoutRight               src/FieldStore.hpp:16-20, src/Simulation.cpp:180
//   diagnostics  diag(k, j, c)  LayoutRight               src/Simulation.hpp:44
// k: slice (head first, internal xi = xi_min + k dxi), j: radial node, c: component.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace qzb {

// field components (src/FieldStore.hpp:9-13)
enum FieldComp : int {
    F_EP1R = 0, F_EP1I, F_BP1R, F_BP1I, F_EZ0, F_BZ0,
    F_EP0R, F_EP0I, F_EP2R, F_EP2I, F_BP0R, F_BP0I, F_BP2R, F_BP2I,
    F_EZ1R, F_EZ1I, F_BZ1R, F_BZ1I,
    F_NC0 = 6, F_NC1 = 18
};
// beam source components (src/FieldStore.hpp:16-20)
enum BeamComp : int {
    B_RT0 = 0, B_JZ0, B_JP1R, B_JP1I, B_RHO0,
    B_RT1R, B_RT1I, B_JZ1R, B_JZ1I, B_JP0R, B_JP0I, B_JP2R, B_JP2I, B_RHO1R, B_RHO1I,
    B_NC0 = 5, B_NC1 = 15
};
// diagnostics (src/Simulation.hpp:44)
enum DiagComp : int { D_PSI0 = 0, D_NE0, D_NI0, D_PSI1R, D_PSI1I, D_NE1R, D_NE1I, D_NI1R, D_NI1I, D_NC0 = 3, D_NC1 = 9 };

// Cell of x on the node array r[0..N] (r_j <= x < r_{j+1}), x clamped to [0, R];
// src/RadialGrid.hpp:73-82 (binary search, same result for every x).
__device__ __forceinline__ int locate(const double* __restrict__ r, int N, double R, double x) {
    if (x <= 0.0) return 0;
    if (x >= R) return N - 1;
    int lo = 0, hi = N;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (r[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

// the cell locate() returns, found by walking up to 4 cells from a guess (particles move little per
// step), the binary search when the walk fails or there is no guess (guess < 0)
__device__ __forceinline__ int locate_near(const double* __restrict__ r, int N, double R, double x, int guess) {
    if (guess < 0 || !(x > 0.0) || !(x < R)) return locate(r, N, R, x);
    int j = guess > N - 1 ? N - 1 : guess;
#pragma unroll 1
    for (int step = 0; step < 4; ++step) {
        if (r[j] > x) { if (j == 0) break; --j; continue; }
        if (r[j + 1] <= x) { if (j == N - 1) break; ++j; continue; }
        return j;
    }
    return locate(r, N, R, x);
}

// cell and clamped fractional position (src/RadialGrid.hpp:84-88)
__device__ __forceinline__ void weights(const double* __restrict__ r, const double* __restrict__ inv_h, int N,
                                        double R, double x, int& j, double& t) {
    j = locate(r, N, R, x);
    double tt = (x - r[j]) * inv_h[j];
    t = tt < 0.0 ? 0.0 : (tt > 1.0 ? 1.0 : tt);
}

// per-particle geometry (src/PlasmaSpecies.cpp:52-70)
struct PGeo {
    double r, c, s;
    int j;
    double W0, W1, ih, Wor0, Wor1;
};

__device__ __forceinline__ PGeo geometry(const double* __restrict__ r, const double* __restrict__ inv_h, int N,
                                         double R, double x, double y) {
    PGeo p;
    p.r = sqrt(x * x + y * y);
    if (p.r > 0.0) { p.c = x / p.r; p.s = y / p.r; } else { p.c = 1.0; p.s = 0.0; }
    double t;
    weights(r, inv_h, N, R, p.r, p.j, t);
    p.ih = inv_h[p.j];
    p.W0 = 1.0 - t;
    p.W1 = t;
    const double ir = p.r > 0.0 ? 1.0 / p.r : 0.0;
    p.Wor0 = (p.j == 0) ? 0.0 : p.W0 * ir;
    p.Wor1 = (p.j == 0) ? p.ih : p.W1 * ir;
    return p;
}

// the same geometry when the cell j of the particle is already known (no search)
__device__ __forceinline__ PGeo geometry_in(const double* __restrict__ r, const double* __restrict__ inv_h, double x,
                                            double y, int j) {
    PGeo p;
    p.r = sqrt(x * x + y * y);
    if (p.r > 0.0) { p.c = x / p.r; p.s = y / p.r; } else { p.c = 1.0; p.s = 0.0; }
    p.j = j;
    double tt = (p.r - r[j]) * inv_h[j];
    const double t = tt < 0.0 ? 0.0 : (tt > 1.0 ? 1.0 : tt);
    p.ih = inv_h[j];
    p.W0 = 1.0 - t;
    p.W1 = t;
    const double ir = p.r > 0.0 ? 1.0 / p.r : 0.0;
    p.Wor0 = (j == 0) ? 0.0 : p.W0 * ir;
    p.Wor1 = (j == 0) ? p.ih : p.W1 * ir;
    return p;
}

__device__ __forceinline__ double lin(const double* __restrict__ f, const PGeo& p) {
    return p.W0 * f[p.j] + p.W1 * f[p.j + 1];
}

// ---------------------------------------------------------------- Vay pusher (src/Pushers.hpp:144-176)
struct V3 { double x, y, z; };
__device__ __forceinline__ double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross3(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double gamma2_root(double x, double c) {
    const double s = sqrt(x * x + c);
    return x >= 0.0 ? x + s : (s > -x ? c / (s - x) : 1.0);
}
__device__ __forceinline__ V3 solve_implicit(V3 a, V3 b) {
    const double b2 = dot3(b, b), ab = dot3(a, b);
    const double g2 = gamma2_root(0.5 * (1.0 + dot3(a, a) - b2), b2 + ab * ab);
    const double g = sqrt(g2);
    const V3 axb = cross3(a, b);
    const double inv = 1.0 / (g2 + b2);
    return {inv * (g2 * a.x + g * axb.x + ab * b.x), inv * (g2 * a.y + g * axb.y + ab * b.y),
            inv * (g2 * a.z + g * axb.z + ab * b.z)};
}
__device__ __forceinline__ V3 vay(V3 u, V3 E, V3 B, double eps) {
    const double g0 = sqrt(1.0 + dot3(u, u));
    const double e2 = 2.0 * eps, eg = eps / g0;
    const V3 uxb = cross3(u, B);
    const V3 up = {u.x + e2 * E.x + eg * uxb.x, u.y + e2 * E.y + eg * uxb.y, u.z + e2 * E.z + eg * uxb.z};
    return solve_implicit(up, {eps * B.x, eps * B.y, eps * B.z});
}

}  // namespace qzb
