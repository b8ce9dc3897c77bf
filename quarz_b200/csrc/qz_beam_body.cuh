// qz_beam_body.cuh -- device functions of the beam path (deposit, gather + Vay push, moment sums),
// shared by the stand-alone beam kernels (qz_beam.cu) and the time-step pipeline (qz_pipeline.cu).
//
// Beam::deposit (src/Beam.cpp:725-785), Beam::advance with the Vay pusher (src/Beam.cpp:948-1131,
// src/Pushers.hpp:63-68), Beam::sums (src/Beam.cpp:1133-1155).
#pragma once
#include "qz_device.cuh"
#include "qz_internal.h"

namespace qzb {
namespace beam_detail {

// kL2: the data was written by other SMs during the same launch, so it is read from L2 (ld.global.cg)
template <bool kL2>
__device__ __forceinline__ double fload(const double* p) { return kL2 ? __ldcg(p) : *p; }

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
            if (B.fx_scale) {                       // exact (m = 0 runs of qz_sim)
                const double sc = B.fx_scale[jj];
                beam_fx_add(o + B_RT0, B.fx_lo, d * omvz, sc, B.fx_inv2s, B.fx_2s);
                beam_fx_add(o + B_JZ0, B.fx_lo, d * vz, sc, B.fx_inv2s, B.fx_2s);
                beam_fx_add(o + B_JP1R, B.fx_lo, d * vr, sc, B.fx_inv2s, B.fx_2s);
                beam_fx_add(o + B_JP1I, B.fx_lo, d * vt, sc, B.fx_inv2s, B.fx_2s);
                beam_fx_add(o + B_RHO0, B.fx_lo, d, sc, B.fx_inv2s, B.fx_2s);
                continue;
            }
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

// The part of the m = 0 deposit that the m = 0 sweep reads, returned instead of applied: rho - J_z,
// J_z and J_theta (B_RT0, B_JZ0, B_JP1I; the sweep never reads the beam's J_r and rho, and a field file
// deposits its beam density again) of one particle, v[(2 a + b) * 3 + c] for row k + a, node j + b,
// rows out of the box carrying zero. Returns false when the particle deposits nothing (outside the wall
// or box). jguess: a nearby radial cell (the gather's, before the push moved the particle), or < 0
constexpr int kDep0 = 3;                             // components of deposit_vals0
__device__ __forceinline__ bool deposit_vals0(const BeamArgs& B, double X, double Y, double PX, double PY, double PZ,
                                              double XI, double wi, int jguess, int& k, int& j,
                                              double (&v)[4 * kDep0]) {
    const double R = B.R;
    const double r = sqrt(X * X + Y * Y);
    if (r > R) return false;
    const double c = r > 0.0 ? X / r : 1.0, s = r > 0.0 ? Y / r : 0.0;
    const double sx = (XI - B.xi_min) * B.idxi;
    k = B.ngp ? (int)floor(sx + 0.5) : (int)floor(sx);
    const int nloc = B.K;
    if (k < -1 || k >= nloc) return false;
    const double tk = B.ngp ? 0.0 : sx - k;
    const double p2 = PX * PX + PY * PY;
    const double gam = sqrt(1.0 + p2 + PZ * PZ);
    const double omvz = (1.0 + p2) / (gam * (gam + PZ));
    const double vz = PZ / gam, vx = PX / gam, vy = PY / gam;
    const double vt = c * vy - s * vx;
    // the cell of r (src/RadialGrid.hpp:35-50): a short walk from the guess, the search otherwise
    j = locate_near(B.r, B.N, R, r, jguess);
    double t = (r - B.r[j]) * B.inv_h[j];
    t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
    const double Wr[2] = {1.0 - t, t};
    const double Wk[2] = {1.0 - tk, tk};
    const double q = B.q;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const int kk = k + a;
        const bool row = (a == 0 || !B.ngp) && kk >= 0 && kk < nloc;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const double d = row ? wi * q * Wk[a] * Wr[b] * B.inv_V[j + b] * B.idxi : 0.0;
            double* o = v + (2 * a + b) * kDep0;
            o[0] = d * omvz;
            o[1] = d * vz;
            o[2] = d * vt;
        }
    }
    return true;
}

// adds the contributions of deposit_vals0 into bsrc (FP64 reductions into L2, or exact)
__device__ __forceinline__ void deposit_add0(const BeamArgs& B, double* __restrict__ bsrc, int k, int j,
                                             const double (&v)[4 * kDep0]) {
    constexpr int comp[kDep0] = {B_RT0, B_JZ0, B_JP1I};
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const int kk = k + a;
        if (kk < 0 || kk >= B.K || (a == 1 && B.ngp)) continue;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            double* o = bsrc + ((size_t)kk * B.M + j + b) * B_NC0;
            if (B.fx_scale) {
                const double sc = B.fx_scale[j + b];
#pragma unroll
                for (int c = 0; c < kDep0; ++c)
                    beam_fx_add(o + comp[c], B.fx_lo, v[(2 * a + b) * kDep0 + c], sc, B.fx_inv2s, B.fx_2s);
            } else {
#pragma unroll
                for (int c = 0; c < kDep0; ++c) atomicAdd(o + comp[c], v[(2 * a + b) * kDep0 + c]);
            }
        }
    }
}

// The part of the m = 1 deposit that the m = 1 sweep reads (rho - J_z, J_z and J_perp in modes 0 and 1,
// J_perp also in mode 2; not the beam densities), per corner: deposit_setup1 takes the particle's cell,
// weights and velocities once (deposit_one's m = 1 branch, src/Beam.cpp:725-785), deposit_corner1 the 12
// values of corner (row k + a, node j + b), deposit_add1 adds them with FP64 reductions.
constexpr int kDep1 = 12;
struct Dep1 {
    int k, j;
    double d0, tk, t, c, s, omvz, vz, vx, vy, vr, vt;
};
__device__ __forceinline__ bool deposit_setup1(const BeamArgs& B, double X, double Y, double PX, double PY, double PZ,
                                               double XI, double wi, int jguess, Dep1& D) {
    const double R = B.R;
    const double r = sqrt(X * X + Y * Y);
    if (r > R) return false;
    D.c = r > 0.0 ? X / r : 1.0;
    D.s = r > 0.0 ? Y / r : 0.0;
    const double sx = (XI - B.xi_min) * B.idxi;
    D.k = B.ngp ? (int)floor(sx + 0.5) : (int)floor(sx);
    if (D.k < -1 || D.k >= B.K) return false;
    D.tk = B.ngp ? 0.0 : sx - D.k;
    const double p2 = PX * PX + PY * PY;
    const double gam = sqrt(1.0 + p2 + PZ * PZ);
    D.omvz = (1.0 + p2) / (gam * (gam + PZ));
    D.vz = PZ / gam; D.vx = PX / gam; D.vy = PY / gam;
    D.vr = D.c * D.vx + D.s * D.vy;
    D.vt = D.c * D.vy - D.s * D.vx;
    D.j = locate_near(B.r, B.N, R, r, jguess);
    const double t = (r - B.r[D.j]) * B.inv_h[D.j];
    D.t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
    D.d0 = wi * B.q;
    return true;
}
// corner (a, b): v in the order B_RT0, B_RT1R, B_RT1I, B_JZ0, B_JZ1R, B_JZ1I, B_JP0R, B_JP0I, B_JP1R,
// B_JP1I, B_JP2R, B_JP2I; zero for a row outside the box or the second row of the ngp shape
__device__ __forceinline__ void deposit_corner1(const BeamArgs& B, const Dep1& D, int a, int b,
                                                double (&v)[kDep1]) {
    const int kk = D.k + a;
    const bool row = (a == 0 || !B.ngp) && kk >= 0 && kk < B.K;
    const double Wk = a ? D.tk : 1.0 - D.tk, Wr = b ? D.t : 1.0 - D.t;
    const double d = row ? D.d0 * Wk * Wr * B.inv_V[D.j + b] * B.idxi : 0.0;
    const double c2 = D.c * D.c - D.s * D.s, s2 = 2.0 * D.c * D.s;
    v[0] = d * D.omvz; v[1] = d * D.omvz * D.c; v[2] = -d * D.omvz * D.s;
    v[3] = d * D.vz; v[4] = d * D.vz * D.c; v[5] = -d * D.vz * D.s;
    v[6] = d * D.vx; v[7] = d * D.vy;
    v[8] = d * D.vr; v[9] = d * D.vt;
    v[10] = d * (D.vx * c2 + D.vy * s2); v[11] = d * (D.vy * c2 - D.vx * s2);
}
__device__ __forceinline__ void deposit_add1(const BeamArgs& B, double* __restrict__ bsrc, int kk, int jj,
                                             const double (&v)[kDep1]) {
    if (kk < 0 || kk >= B.K) return;
    constexpr int comp[kDep1] = {B_RT0, B_RT1R, B_RT1I, B_JZ0, B_JZ1R, B_JZ1I, B_JP0R, B_JP0I, B_JP1R, B_JP1I,
                                 B_JP2R, B_JP2I};
    double* o = bsrc + ((size_t)kk * B.M + jj) * B_NC1;
#pragma unroll
    for (int c = 0; c < kDep1; ++c) atomicAdd(o + comp[c], v[c]);
}

// bilinear (xi, r) gather and mode sums at the particle (src/Beam.cpp:972-1008)
template <bool kL2>
__device__ __forceinline__ void gather(const BeamArgs& B, const double* __restrict__ fld, double X, double Y,
                                       double XI, double& c, double& sn, V3& E, V3& Bf, int* jcell = nullptr) {
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
    if (jcell) *jcell = j;
    const int nc = B.modes ? F_NC1 : F_NC0;
    const double* f00 = fld + ((size_t)k * B.M + j) * nc;
    const double* f01 = f00 + nc;
    const double* f10 = fld + ((size_t)k1 * B.M + j) * nc;
    const double* f11 = f10 + nc;
    auto bil = [&](int comp) {
        return (1.0 - tk) * ((1.0 - t) * fload<kL2>(f00 + comp) + t * fload<kL2>(f01 + comp)) +
               tk * ((1.0 - t) * fload<kL2>(f10 + comp) + t * fload<kL2>(f11 + comp));
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


// One particle of Beam::advance (src/Beam.cpp:948-1131): gather at the old position, optional explicit
// start-up kick with the same fields (h_start != 0, src/Beam.cpp:1038-1044), Vay with h = q/m dt_kick/2,
// drift, removal at the wall or outside the box. Returns false when the particle was removed.
struct PState7 {
    double x, y, px, py, pz, xi, w;
};

template <bool kL2>
__device__ __forceinline__ bool push_one(const BeamArgs& B, const double* __restrict__ fld, PState7& p, double h,
                                         double h_start, double dt, int* jcell = nullptr) {
    double c, sn;
    V3 E, Bf;
    gather<kL2>(B, fld, p.x, p.y, p.xi, c, sn, E, Bf, jcell);
    V3 u = {p.px, p.py, p.pz};
    if (h_start != 0.0) {
        const double g0 = sqrt(1.0 + dot3(u, u));
        const double ig = 1.0 / g0;
        const V3 v = {ig * u.x, ig * u.y, ig * u.z};
        const V3 vxb = cross3(v, Bf);
        const double h2 = 2.0 * h_start;
        u = {u.x + h2 * (E.x + vxb.x), u.y + h2 * (E.y + vxb.y), u.z + h2 * (E.z + vxb.z)};
    }
    u = vay(u, E, Bf, h);
    const double p2 = u.x * u.x + u.y * u.y;
    const double gam = sqrt(1.0 + p2 + u.z * u.z);
    const double omvz = (1.0 + p2) / (gam * (gam + u.z));
    const double xn = p.x + u.x / gam * dt, yn = p.y + u.y / gam * dt;
    const double xin = p.xi + omvz * dt;
    const double xmin = B.xi_min, xmax = B.xi_min + (B.K - 1) * B.dxi;
    p.x = xn; p.y = yn; p.px = u.x; p.py = u.y; p.pz = u.z; p.xi = xin;
    if (xn * xn + yn * yn >= B.R * B.R || xin < xmin || xin > xmax) {
        p.w = 0.0;
        return false;
    }
    return true;
}

// the weighted moments of Beam::sums (src/Beam.cpp:1133-1155) of one particle, added to acc[17]
__device__ __forceinline__ void sums_add(double* acc, const PState7& p, double gref, double xiref) {
    const double g = sqrt(1.0 + p.px * p.px + p.py * p.py + p.pz * p.pz);
    const double G = g - gref, XI = p.xi - xiref;
    const double v[15] = {G, G * G, XI, XI * XI, p.x * p.x + p.y * p.y, p.x, p.y, p.x * p.x, p.y * p.y,
                          p.px, p.py, p.px * p.px, p.py * p.py, p.x * p.px, p.y * p.py};
    acc[16] += 1.0;
    acc[0] += p.w;
#pragma unroll
    for (int c = 0; c < 15; ++c) acc[c + 1] += p.w * v[c];
}

// sums_add into one lane's accumulators in shared memory (a[c * 32], c = 0..16): the same operations
__device__ __forceinline__ void sums_add_lane(double* a, const PState7& p, double gref, double xiref) {
    const double g = sqrt(1.0 + p.px * p.px + p.py * p.py + p.pz * p.pz);
    const double G = g - gref, XI = p.xi - xiref;
    const double v[15] = {G, G * G, XI, XI * XI, p.x * p.x + p.y * p.y, p.x, p.y, p.x * p.x, p.y * p.y,
                          p.px, p.py, p.px * p.px, p.py * p.py, p.x * p.px, p.y * p.py};
    a[16 * 32] += 1.0;
    a[0] += p.w;
#pragma unroll
    for (int c = 0; c < 15; ++c) a[(c + 1) * 32] += p.w * v[c];
}

// the xi cell of a particle for bucketing: floor((xi - xi_min)/dxi) clamped to [-1, K-1]
__device__ __forceinline__ int xi_cell(const BeamArgs& B, double xi) {
    const double s = (xi - B.xi_min) * B.idxi;
    if (!(s >= -1.0)) return -1;
    if (s >= (double)(B.K - 1)) return B.K - 1;
    return (int)floor(s);
}

}  // namespace beam_detail
}  // namespace qzb
