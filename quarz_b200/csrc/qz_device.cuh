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

// Exact beam deposits (m = 0 runs): a contribution v to node j becomes t = v scale_j (scale_j = 2^-qe_j
// from a bound on every contribution to that node, so |t| < 2^(2S)), split into t = hi 2^S + lo with
// hi = floor(t / 2^S) and lo = t - hi 2^S rounded to an integer, and hi and lo are added to two
// independent accumulators with FP64 reductions. Every limb is an integer of magnitude at most 2^S and
// a value receives fewer than 2^(53-S) of them (S is chosen on the host from the particle count), so
// every partial sum is an integer below 2^53: each FP64 add is exact and the sums do not depend on the
// order of the adds, so the deposit is reproducible bit for bit. (FP64 reductions are the faster atomic
// path here: with one reduction per value, a push task of the pipelined pinched-witness run took 251 us
// with 64-bit integer reductions and 175 us with FP64 ones.)
// The value is (2^S sum_hi + sum_lo) 2^qe_j.
__device__ __forceinline__ void beam_fx_add(double* hi_p, long lo_off, double v, double scale, double inv2s,
                                            double two_s) {
    if (v == 0.0) return;
    const double t = v * scale;
    const double hi = floor(t * inv2s);
    const double lo = rint(fma(-hi, two_s, t));           // fma exact: t - hi 2^S in [0, 2^S)
    atomicAdd(hi_p, hi);
    atomicAdd(hi_p + lo_off, lo);
}
__device__ __forceinline__ double beam_fx_value(double hi_sum, double lo_sum, double quantum, double two_s) {
    return fma(hi_sum, two_s, lo_sum) * quantum;
}

// Cell of x on the node array r[0..N] (r_j <= x < r_{j+1}), x clamped to [0, R];
// src/RadialGrid.hpp:35-44 (binary search, same result for every x).
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

// cell and clamped fractional position (src/RadialGrid.hpp:35-50)
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

// ---------------------------------------------------------------- Vay pusher (src/Pushers.hpp:36-68)
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
__device__ __forceinline__ V3 vay(V3 u, V3 E, V3 B, double eps);

// The other beam pushers of src/Pushers.hpp:64-95 (<beam>.pusher). Boris (1970): half electric kick,
// rotation by t = eps B / gamma(u-), half kick.
__device__ __forceinline__ V3 boris(V3 u, V3 E, V3 B, double eps) {
    const V3 um = {u.x + eps * E.x, u.y + eps * E.y, u.z + eps * E.z};
    const double g = sqrt(1.0 + dot3(um, um));
    const double f = eps / g;
    const V3 t = {f * B.x, f * B.y, f * B.z};
    const double sf = 2.0 / (1.0 + dot3(t, t));
    const V3 s = {sf * t.x, sf * t.y, sf * t.z};
    const V3 c1 = cross3(um, t);
    const V3 w = {um.x + c1.x, um.y + c1.y, um.z + c1.z};
    const V3 c2 = cross3(w, s);
    return {um.x + c2.x + eps * E.x, um.y + c2.y + eps * E.y, um.z + c2.z + eps * E.z};
}

// Higuera & Cary (2017): the rotation with the gamma of the time-centred momentum
__device__ __forceinline__ V3 higuera_cary(V3 u, V3 E, V3 B, double eps) {
    const V3 um = {u.x + eps * E.x, u.y + eps * E.y, u.z + eps * E.z};
    const V3 tau = {eps * B.x, eps * B.y, eps * B.z};
    const double us = dot3(um, tau), tt = dot3(tau, tau);
    const double sig = 1.0 + dot3(um, um) - tt;
    const double gp = sqrt(0.5 * (sig + sqrt(sig * sig + 4.0 * (tt + us * us))));
    const double ig = 1.0 / gp;
    const V3 t = {ig * tau.x, ig * tau.y, ig * tau.z};
    const double s = 1.0 / (1.0 + dot3(t, t));
    const double ut = dot3(um, t);
    const V3 c = cross3(um, t);
    const V3 upl = {s * (um.x + ut * t.x + c.x), s * (um.y + ut * t.y + c.y), s * (um.z + ut * t.z + c.z)};
    const V3 c2 = cross3(upl, t);
    return {upl.x + eps * E.x + c2.x, upl.y + eps * E.y + c2.y, upl.z + eps * E.z + c2.z};
}

// the implicit midpoint push: ubar = (u + eps E) + (ubar / gamma(ubar)) x eps B solved exactly, u+ = 2 ubar - u
__device__ __forceinline__ V3 imp(V3 u, V3 E, V3 B, double eps) {
    const V3 ub = solve_implicit({u.x + eps * E.x, u.y + eps * E.y, u.z + eps * E.z}, {eps * B.x, eps * B.y, eps * B.z});
    return {2.0 * ub.x - u.x, 2.0 * ub.y - u.y, 2.0 * ub.z - u.z};
}

// <beam>.pusher (src/Beam.cpp:72-78): 0 vay, 1 boris, 2 hc, 3 imp
__device__ __forceinline__ V3 push_u(int kind, V3 u, V3 E, V3 B, double eps) {
    switch (kind) {
        case 1: return boris(u, E, B, eps);
        case 2: return higuera_cary(u, E, B, eps);
        case 3: return imp(u, E, B, eps);
        default: return vay(u, E, B, eps);
    }
}

__device__ __forceinline__ V3 vay(V3 u, V3 E, V3 B, double eps) {
    const double g0 = sqrt(1.0 + dot3(u, u));
    const double e2 = 2.0 * eps, eg = eps / g0;
    const V3 uxb = cross3(u, B);
    const V3 up = {u.x + e2 * E.x + eg * uxb.x, u.y + e2 * E.y + eg * uxb.y, u.z + e2 * E.z + eg * uxb.z};
    return solve_implicit(up, {eps * B.x, eps * B.y, eps * B.z});
}

}  // namespace qzb
