// qz_adjoint.cu -- the adjoint (reverse mode) of an m = 0 run on the device: the gradient of any
// linear function of the last step's beam moment sums with respect to every initial beam particle.
// The reference has no gradients; this differentiates this library's own forward exactly:
//
//   beam moment sums   Beam::sums (src/Beam.cpp:1133-1155)                      sums_back_kernel
//   beam push          Beam::push / advance (src/Beam.cpp:900-905, :948-1131)    push_back_kernel
//   the sweep          Simulation::step_fields (src/Simulation.cpp:636-795)      sweep_back_kernel
//   beam deposit       Beam::deposit (src/Beam.cpp:725-785)                      deposit_back_kernel
//
// The reverse sweep runs the slices from the tail to the head in one CTA, one radial row and one
// plasma particle per thread, with the plasma state of every slice recorded by the forward sweep of
// the same step (SweepArgs::traj). Its transposed tridiagonal solves reuse the forward's factorised
// scans: each operator L (L0, L1D - chi, L1F - chi) becomes symmetric when its interior rows are
// scaled by a diagonal F (L0 = D^-1 S with D = V / 2pi; F = r dV for the fv_rows operators), so
// L^-T lam = F L^-1 (F^-1 lam) on the non-Dirichlet rows, and the Dirichlet rows carry no adjoint.
// Particle removal, cell changes and clamps are piecewise constant: their derivative is zero.
#include "qz_beam_body.cuh"
#include "qz_sweep_body.cuh"

namespace qzb {
namespace adj {

using beam_detail::PState7;

__device__ __forceinline__ V3 add3(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 mul3(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }

// ------------------------------------------------------------------ Vay in reverse
// solve_implicit(a, b) -> r: la, lb += (dr/da)^T lr, (dr/db)^T lr
__device__ void solve_implicit_back(V3 a, V3 b, V3 lr, V3& la, V3& lb) {
    const double b2 = dot3(b, b), ab = dot3(a, b);
    const double X = 0.5 * (1.0 + dot3(a, a) - b2), Cc = b2 + ab * ab;
    const double g2 = gamma2_root(X, Cc);
    const double g = sqrt(g2);
    const V3 axb = cross3(a, b);
    const double inv = 1.0 / (g2 + b2);
    const V3 qv = {g2 * a.x + g * axb.x + ab * b.x, g2 * a.y + g * axb.y + ab * b.y, g2 * a.z + g * axb.z + ab * b.z};
    const V3 lq = mul3(inv, lr);
    const double l_inv = dot3(lr, qv);
    double l_g2 = -l_inv * inv * inv, l_b2 = -l_inv * inv * inv;
    l_g2 += dot3(lq, a);
    la = add3(la, mul3(g2, lq));
    const double l_g = dot3(lq, axb);
    const V3 laxb = mul3(g, lq);
    double l_ab = dot3(lq, b);
    lb = add3(lb, mul3(ab, lq));
    la = add3(la, cross3(b, laxb));
    lb = add3(lb, cross3(laxb, a));
    l_g2 += l_g / (2.0 * g);
    const double sq = sqrt(X * X + Cc);                 // g2 = X + sqrt(X^2 + C) on both branches
    const double l_X = l_g2 * (1.0 + X / sq), l_C = l_g2 / (2.0 * sq);
    la = add3(la, mul3(l_X, a));
    l_b2 += l_C - 0.5 * l_X;
    l_ab += 2.0 * ab * l_C;
    la = add3(la, mul3(l_ab, b));
    lb = add3(lb, mul3(l_ab, a));
    lb = add3(lb, mul3(2.0 * l_b2, b));
}

// vay(u, E, B, eps) in reverse
__device__ void vay_back(V3 u, V3 E, V3 B, double eps, V3 lout, V3& lu, V3& lE, V3& lB) {
    const double g0 = sqrt(1.0 + dot3(u, u));
    const V3 uxB = cross3(u, B);
    const V3 up = add3(add3(u, mul3(2.0 * eps, E)), mul3(eps / g0, uxB));
    V3 lup = {0, 0, 0}, lb = {0, 0, 0};
    solve_implicit_back(up, mul3(eps, B), lout, lup, lb);
    lB = add3(lB, mul3(eps, lb));
    lu = add3(lu, lup);
    lE = add3(lE, mul3(2.0 * eps, lup));
    const V3 lc = mul3(eps / g0, lup);
    lu = add3(lu, cross3(B, lc));
    lB = add3(lB, cross3(lc, u));
    const double l_ig0 = eps * dot3(lup, uxB);
    lu = add3(lu, mul3(-l_ig0 / (g0 * g0 * g0), u));
}

// omvz = (1 + px^2 + py^2) / (gam (gam + pz)) in reverse: lp += l d(omvz)/dp
__device__ __forceinline__ void omvz_back(double px, double py, double pz, double l, double (&lp)[3]) {
    const double A = 1.0 + px * px + py * py;
    const double G = sqrt(A + pz * pz);
    const double den = G * (G + pz);
    const double lA = l / den;
    const double lG = -l * A * (2.0 * G + pz) / (den * den);
    const double lpz = -l * A * G / (den * den);
    lp[0] += lA * 2.0 * px + lG * px / G;
    lp[1] += lA * 2.0 * py + lG * py / G;
    lp[2] += lpz + lG * pz / G;
}

// (lr, lc, ls) at (x, y) -> (lx, ly), with c = x / r, s = y / r
__device__ __forceinline__ void polar_back(double r, double c, double s, double lr, double lc, double ls, double& lx,
                                           double& ly) {
    if (!(r > 0.0)) return;
    lx += lr * c + lc * s * s / r - ls * c * s / r;
    ly += lr * s - lc * c * s / r + ls * c * c / r;
}

// ------------------------------------------------------------------ beam kernels
// lam: 7 columns of n (x y px py pz xi w), the adjoint of the beam's current state

// Beam::sums in reverse: lam += d(lamS . sums)/d(particle)
__global__ void sums_back_kernel(BeamArgs B, double gref, double xiref, const double* __restrict__ lamS,
                                 double* __restrict__ lam) {
    const long n = B.n;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double w = B.w[i];
        if (w == 0.0) continue;
        const double PX = B.px[i], PY = B.py[i], PZ = B.pz[i], X = B.x[i], Y = B.y[i];
        const double g = sqrt(1.0 + PX * PX + PY * PY + PZ * PZ);
        const double G = g - gref, XI = B.xi[i] - xiref;
        const double v[15] = {G, G * G, XI, XI * XI, X * X + Y * Y, X, Y, X * X, Y * Y, PX, PY, PX * PX, PY * PY,
                              X * PX, Y * PY};
        double lw = lamS[0];
#pragma unroll
        for (int c = 0; c < 15; ++c) lw += lamS[c + 1] * v[c];
        const double* lv = lamS + 1;
        const double lG = w * (lv[0] + 2.0 * G * lv[1]);
        lam[i] += w * (2.0 * X * lv[4] + lv[5] + 2.0 * X * lv[7] + PX * lv[13]);
        lam[n + i] += w * (2.0 * Y * lv[4] + lv[6] + 2.0 * Y * lv[8] + PY * lv[14]);
        lam[2 * n + i] += lG * PX / g + w * (lv[9] + 2.0 * PX * lv[11] + X * lv[13]);
        lam[3 * n + i] += lG * PY / g + w * (lv[10] + 2.0 * PY * lv[12] + Y * lv[14]);
        lam[4 * n + i] += lG * PZ / g;
        lam[5 * n + i] += w * (lv[2] + 2.0 * XI * lv[3]);
        lam[6 * n + i] += lw;
    }
}

// One push of particle i (start-up half kick when startup, gather, Vay, drift) in reverse. On entry
// l7 is the adjoint after the push, on exit before it; the field adjoint is added to lfld (K, M, 6).
// kAgg: instead of adding to lfld, return the 24 contributions (6 components x corners (k, j), (k, j+1),
// (k+1, j), (k+1, j+1)) in g with key = k M + j (-1 when none), for a warp-aggregated update
template <bool kAgg>
__device__ void push_back_one(const BeamArgs& B, const double* __restrict__ fld, long i, double (&l7)[7],
                              double* __restrict__ lfld, double dt_kick, double dt, int startup, double (&g)[24],
                              int& key) {
    key = -1;
    const int M = B.M, nloc = B.K;
    const double qm = B.q / B.m;
    const double xmin = B.xi_min, xmax = B.xi_min + (B.K - 1) * B.dxi;
    if (B.w[i] == 0.0) {
#pragma unroll
        for (int c = 0; c < 6; ++c) l7[c] = 0.0;
        return;
    }
    const double X = B.x[i], Y = B.y[i], XI = B.xi[i];
    const double r = sqrt(X * X + Y * Y);
    const double c = r > 0.0 ? X / r : 1.0, sn = r > 0.0 ? Y / r : 0.0;
    double sl = (XI - xmin) * B.idxi;
    int k;
    bool kclamp = false;
    double tk;
    if (B.ngp) {            // the nearest slice, piecewise constant in xi: no xi derivative
        k = min(max((int)floor(sl + 0.5), 0), nloc - 1);
        tk = 0.0;
        kclamp = true;
    } else {
        k = (int)floor(sl);
        if (k < 0) { k = 0; sl = 0; kclamp = true; }
        if (k > nloc - 2) { k = nloc - 2; sl = nloc - 1; kclamp = true; }
        tk = sl - k;
    }
    const int k1 = B.ngp ? k : k + 1;
    int j;
    double t;
    weights(B.r, B.inv_h, B.N, B.R, r, j, t);
    const double* f00 = fld + ((size_t)k * M + j) * F_NC0;
    const double* f01 = f00 + F_NC0;
    const double* f10 = fld + ((size_t)k1 * M + j) * F_NC0;
    const double* f11 = f10 + F_NC0;
    auto bil = [&](int cm) {
        return (1.0 - tk) * ((1.0 - t) * f00[cm] + t * f01[cm]) + tk * ((1.0 - t) * f10[cm] + t * f11[cm]);
    };
    const double er = bil(F_EP1R), ei = bil(F_EP1I), br = bil(F_BP1R), bi = bil(F_BP1I);
    const V3 E = {er * c - ei * sn, er * sn + ei * c, bil(F_EZ0)};
    const V3 Bf = {br * c - bi * sn, br * sn + bi * c, bil(F_BZ0)};
    const V3 u0 = {B.px[i], B.py[i], B.pz[i]};
    V3 u1 = u0;
    const double hs = 0.5 * qm * (-0.5 * dt_kick);
    double g00 = 1.0;
    if (startup) {
        g00 = sqrt(1.0 + dot3(u0, u0));
        const double ig = 1.0 / g00;
        const V3 v = {ig * u0.x, ig * u0.y, ig * u0.z};
        const V3 vxb = cross3(v, Bf);
        const double h2 = 2.0 * hs;
        u1 = {u0.x + h2 * (E.x + vxb.x), u0.y + h2 * (E.y + vxb.y), u0.z + h2 * (E.z + vxb.z)};
    }
    const double h = 0.5 * qm * dt_kick;
    const V3 u2 = vay(u1, E, Bf, h);
    const double p2 = u2.x * u2.x + u2.y * u2.y;
    const double gam = sqrt(1.0 + p2 + u2.z * u2.z);
    const double omvz = (1.0 + p2) / (gam * (gam + u2.z));
    const double xn = X + u2.x / gam * dt, yn = Y + u2.y / gam * dt;
    const double xin = XI + omvz * dt;
    if (xn * xn + yn * yn >= B.R * B.R || xin < xmin || xin > xmax) {     // removed by this push
#pragma unroll
        for (int cc = 0; cc < 7; ++cc) l7[cc] = 0.0;
        return;
    }
    // drift
    double lX = l7[0], lY = l7[1], lxi = l7[5];
    V3 lu2 = {l7[2], l7[3], l7[4]};
    const double lgam = -(l7[0] * u2.x + l7[1] * u2.y) * dt / (gam * gam);
    lu2.x += l7[0] * dt / gam;
    lu2.y += l7[1] * dt / gam;
    double lp[3] = {0.0, 0.0, 0.0};
    omvz_back(u2.x, u2.y, u2.z, l7[5] * dt, lp);
    lu2 = {lu2.x + lp[0] + lgam * u2.x / gam, lu2.y + lp[1] + lgam * u2.y / gam, lu2.z + lp[2] + lgam * u2.z / gam};
    V3 lu1 = {0, 0, 0}, lE = {0, 0, 0}, lB = {0, 0, 0};
    vay_back(u1, E, Bf, h, lu2, lu1, lE, lB);
    V3 lu0 = lu1;
    if (startup) {
        const V3 lw = mul3(2.0 * hs, lu1);                  // w = E + (u0 x B) / g00
        lE = add3(lE, lw);
        const V3 lcr = mul3(1.0 / g00, lw);
        lu0 = add3(lu0, cross3(Bf, lcr));
        lB = add3(lB, cross3(lcr, u0));
        const double l_ig = dot3(lw, cross3(u0, Bf));
        lu0 = add3(lu0, mul3(-l_ig / (g00 * g00 * g00), u0));
    }
    const double l_er = lE.x * c + lE.y * sn, l_ei = -lE.x * sn + lE.y * c;
    const double l_br = lB.x * c + lB.y * sn, l_bi = -lB.x * sn + lB.y * c;
    const double l_c = lE.x * er + lE.y * ei + lB.x * br + lB.y * bi;
    const double l_s = -lE.x * ei + lE.y * er - lB.x * bi + lB.y * br;
    const double lcomp[6] = {l_er, l_ei, l_br, l_bi, lE.z, lB.z};
    const int comp[6] = {F_EP1R, F_EP1I, F_BP1R, F_BP1I, F_EZ0, F_BZ0};
    double l_tk = 0.0, l_t = 0.0;
    if (kAgg) key = k * M + j;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int cm = comp[q];
        const double l = lcomp[q];
        if (kAgg) {
            g[q * 4 + 0] = l * (1.0 - tk) * (1.0 - t);
            g[q * 4 + 1] = l * (1.0 - tk) * t;
            g[q * 4 + 2] = l * tk * (1.0 - t);
            g[q * 4 + 3] = l * tk * t;
        } else {
            double* g00p = lfld + ((size_t)k * M + j) * F_NC0;
            double* g10p = lfld + ((size_t)k1 * M + j) * F_NC0;
            atomicAdd(g00p + cm, l * (1.0 - tk) * (1.0 - t));
            atomicAdd(g00p + F_NC0 + cm, l * (1.0 - tk) * t);
            if (!B.ngp) {
                atomicAdd(g10p + cm, l * tk * (1.0 - t));
                atomicAdd(g10p + F_NC0 + cm, l * tk * t);
            }
        }
        l_tk += l * (((1.0 - t) * f10[cm] + t * f11[cm]) - ((1.0 - t) * f00[cm] + t * f01[cm]));
        l_t += l * ((1.0 - tk) * (f01[cm] - f00[cm]) + tk * (f11[cm] - f10[cm]));
    }
    if (!kclamp) lxi += l_tk * B.idxi;
    const double tt = (r - B.r[j]) * B.inv_h[j];
    const double l_r = (tt > 0.0 && tt < 1.0) ? l_t * B.inv_h[j] : 0.0;
    polar_back(r, c, sn, l_r, l_c, l_s, lX, lY);
    l7[0] = lX; l7[1] = lY; l7[2] = lu0.x; l7[3] = lu0.y; l7[4] = lu0.z; l7[5] = lxi;
    // l7[6] (w) is carried unchanged: the push does not change the weight
}

__global__ void push_back_kernel(BeamArgs B, const double* __restrict__ fld, double* __restrict__ lam,
                                 double* __restrict__ lfld, double dt_kick, double dt, int startup) {
    const long n = B.n;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double l7[7];
#pragma unroll
        for (int c = 0; c < 7; ++c) l7[c] = lam[c * n + i];
        double g[24];                                // (unused: this kernel adds to lfld directly)
        int key;
        push_back_one<false>(B, fld, i, l7, lfld, dt_kick, dt, startup, g, key);
#pragma unroll
        for (int c = 0; c < 7; ++c) lam[c * n + i] = l7[c];
    }
}

// Beam::deposit of particle i in reverse (m = 0, linear or ngp xi shape): l7 += d(lbsrc . bsrc)/d(particle);
// kL2: lbsrc was written by other SMs during the same launch
template <bool kL2>
__device__ void deposit_back_one(const BeamArgs& B, const double* __restrict__ lbsrc, long i, double (&l7)[7]) {
    const int M = B.M, nloc = B.K;
    const double wi = B.w[i];
    if (wi == 0.0) return;
    const double X = B.x[i], Y = B.y[i];
    const double r = sqrt(X * X + Y * Y);
    if (r > B.R) return;
    const double c = r > 0.0 ? X / r : 1.0, sn = r > 0.0 ? Y / r : 0.0;
    const double sx = (B.xi[i] - B.xi_min) * B.idxi;
    const int k = B.ngp ? (int)floor(sx + 0.5) : (int)floor(sx);
    if (k < -1 || k >= nloc) return;
    const double tk = B.ngp ? 0.0 : sx - k;
    const int na = B.ngp ? 1 : 2;
    const double PX = B.px[i], PY = B.py[i], PZ = B.pz[i];
    const double p2 = PX * PX + PY * PY;
    const double gam = sqrt(1.0 + p2 + PZ * PZ);
    const double omvz = (1.0 + p2) / (gam * (gam + PZ));
    const double vz = PZ / gam, vx = PX / gam, vy = PY / gam;
    const double vr = c * vx + sn * vy, vt = c * vy - sn * vx;
    int j;
    double t;
    weights(B.r, B.inv_h, B.N, B.R, r, j, t);
    const double Wr[2] = {1.0 - t, t};
    const double Wk[2] = {1.0 - tk, tk};
    double l_omvz = 0, l_vz = 0, l_vr = 0, l_vt = 0, l_w = 0, lWk[2] = {0, 0}, lWr[2] = {0, 0};
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const int kk = k + a;
        if (a >= na || kk < 0 || kk >= nloc) continue;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int jj = j + b;
            const double* L = lbsrc + ((size_t)kk * M + jj) * B_NC0;
            const double base = B.q * B.inv_V[jj] * B.idxi;
            const double d = wi * Wk[a] * Wr[b] * base;
            const double L0 = beam_detail::fload<kL2>(L + B_RT0), L1 = beam_detail::fload<kL2>(L + B_JZ0);
            const double L2 = beam_detail::fload<kL2>(L + B_JP1R), L3 = beam_detail::fload<kL2>(L + B_JP1I);
            const double ld = L0 * omvz + L1 * vz + L2 * vr + L3 * vt;
            l_omvz += L0 * d;
            l_vz += L1 * d;
            l_vr += L2 * d;
            l_vt += L3 * d;
            l_w += ld * Wk[a] * Wr[b] * base;
            lWk[a] += ld * wi * Wr[b] * base;
            lWr[b] += ld * wi * Wk[a] * base;
        }
    }
    l7[6] += l_w;
    if (!B.ngp) l7[5] += (lWk[1] - lWk[0]) * B.idxi;
    const double tt = (r - B.r[j]) * B.inv_h[j];
    const double l_r = (tt > 0.0 && tt < 1.0) ? (lWr[1] - lWr[0]) * B.inv_h[j] : 0.0;
    const double l_vx = l_vr * c - l_vt * sn, l_vy = l_vr * sn + l_vt * c;
    const double l_c = l_vr * vx + l_vt * vy, l_s = l_vr * vy - l_vt * vx;
    polar_back(r, c, sn, l_r, l_c, l_s, l7[0], l7[1]);
    double lp[3] = {l_vx / gam, l_vy / gam, l_vz / gam};
    const double l_g = -(l_vx * PX + l_vy * PY + l_vz * PZ) / (gam * gam);
    lp[0] += l_g * PX / gam;
    lp[1] += l_g * PY / gam;
    lp[2] += l_g * PZ / gam;
    omvz_back(PX, PY, PZ, l_omvz, lp);
    l7[2] += lp[0];
    l7[3] += lp[1];
    l7[4] += lp[2];
}

__global__ void deposit_back_kernel(BeamArgs B, const double* __restrict__ lbsrc, double* __restrict__ lam) {
    const long n = B.n;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        if (B.w[i] == 0.0) continue;
        double l7[7];
#pragma unroll
        for (int c = 0; c < 7; ++c) l7[c] = lam[c * n + i];
        deposit_back_one<false>(B, lbsrc, i, l7);
#pragma unroll
        for (int c = 0; c < 7; ++c) lam[c * n + i] = l7[c];
    }
}

// ------------------------------------------------------------------ the reverse sweep
// shared-memory arrays of one slice (M each)
struct AdjSm {
    double *r, *iv, *ih, *F1;                       // grid; F1 = r dV (symmetriser of L1D / L1F)
    double *wpr, *ez, *bz, *bpr, *bpi, *chi;        // forward values of the slice
    double *l_wpr, *l_ez, *l_bz, *l_bpr, *l_bpi;    // adjoints of the fields
    double *l_rhot, *l_drho, *l_jz, *l_chi, *l_jpi, *l_Sr, *l_Si;   // adjoints of the sources
    double *t0, *t1;                                // scratch
    double* tot;                                    // scan scratch (2 x 8 x kW)
    double* lam;                                    // particle adjoints ((5 + 5 ord) x kSweepThreads)
    int* flag;                                      // gate result broadcast
};
constexpr int kAdjArrays = 22;
constexpr int kMaxOrd = 5;                          // the particle adjoints' room: AB order up to 5

__device__ __forceinline__ AdjSm carve_adj(double* p, int M) {
    AdjSm S;
    double** a[kAdjArrays] = {&S.r, &S.iv, &S.ih, &S.F1, &S.wpr, &S.ez, &S.bz, &S.bpr, &S.bpi, &S.chi, &S.l_wpr,
                              &S.l_ez, &S.l_bz, &S.l_bpr, &S.l_bpi, &S.l_rhot, &S.l_drho, &S.l_jz, &S.l_chi, &S.l_jpi,
                              &S.l_Sr, &S.l_Si};
    for (int i = 0; i < kAdjArrays; ++i) { *a[i] = p; p += M; }
    S.t0 = p; p += M;
    S.t1 = p; p += M;
    S.tot = p; p += 2 * 8 * kW;
    S.lam = p; p += (size_t)(5 + 5 * kMaxOrd) * kSweepThreads;
    S.flag = reinterpret_cast<int*>(p);
    return S;
}

// geometry adjoints of one particle: r, c, s, W0, W1, Wor0, Wor1
struct GeoAdj { double r, c, s, W0, W1, Wor0, Wor1; };

__device__ __forceinline__ void geo_back(const AdjSm& S, const PGeo& g, GeoAdj& a, double& lx, double& ly) {
    if (g.j > 0 && g.r > 0.0) {
        a.W0 += a.Wor0 / g.r;
        a.W1 += a.Wor1 / g.r;
        a.r -= (a.Wor0 * g.W0 + a.Wor1 * g.W1) / (g.r * g.r);
    }
    const double tt = (g.r - S.r[g.j]) * g.ih;
    if (tt > 0.0 && tt < 1.0) a.r += (a.W1 - a.W0) * g.ih;
    polar_back(g.r, g.c, g.s, a.r, a.c, a.s, lx, ly);
}

// lin(f) at the particle in reverse: the adjoints of the nodes j, j+1 (appended to val, which the caller
// scatters) and of the weights
__device__ __forceinline__ void lin_back(const PGeo& g, const double* f, double l, GeoAdj& a, double (&val)[10],
                                         int& na) {
    val[na++] = l * g.W0;
    val[na++] = l * g.W1;
    a.W0 += l * f[g.j];
    a.W1 += l * f[g.j + 1];
}

// plasma particle state and its adjoint
template <int ORD>
struct PAdj {
    double x, y, px, py, dl;
    double h[ORD][5];
};

// PlasmaSpecies::push (src/PlasmaSpecies.cpp:561-668) of one particle in reverse, with the forward's
// history rotation (h[0] newest). L: adjoint after the push (in), before (out). Returns false when the
// push removed the particle (no adjoint flows through it).
// The field adjoints at the particle's nodes j, j+1 are returned in sc (W+, E_z, B_z, B_r, B_theta; node j
// then j+1 each) with jc = j, for a warp-aggregated update by the caller.
template <int ORD>
__device__ bool push_back(const AdjSm& S, const SweepArgs& A, const PState<ORD>& P, bool first, PAdj<ORD>& L,
                          double (&sc)[10], int& jc) {
    const double qm = P.qm;
    const PGeo g = geometry(S.r, S.ih, A.N, A.R, P.x, P.y);
    const double R1 = lin(S.wpr, g), Ez = lin(S.ez, g), Bz = lin(S.bz, g);
    const double BR = lin(S.bpr, g), BI = lin(S.bpi, g);
    const double Wx = R1 * g.c, Wy = R1 * g.s;
    const double Bx = BR * g.c - BI * g.s, By = BR * g.s + BI * g.c;
    const double PX = P.px, PY = P.py, D = P.dl;
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D;
    double fv[5];
    fv[0] = PX * invd;
    fv[1] = PY * invd;
    fv[2] = qm * (gam * Wx * invd + By + PY * Bz * invd);
    fv[3] = qm * (gam * Wy * invd - Bx - PX * Bz * invd);
    fv[4] = qm * ((PX * Wx + PY * Wy) * invd - Ez);
    double hc[ORD][5];                                 // history after the write, before a reflection
#pragma unroll
    for (int m = 0; m < ORD; ++m)
#pragma unroll
        for (int v = 0; v < 5; ++v) hc[m][v] = (first || m == 0) ? fv[v] : P.h[m - 1][v];
    double sum[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int m = 0; m < ORD; ++m)
#pragma unroll
        for (int v = 0; v < 5; ++v) sum[v] += A.ab[m] * hc[m][v];
    const double dxi = A.dxi;
    const double xn = P.x + dxi * sum[0], yn = P.y + dxi * sum[1];
    const double pxn = PX + dxi * sum[2], pyn = PY + dxi * sum[3];
    const double dn = D + dxi * sum[4];
    const double gn = (1.0 + pxn * pxn + pyn * pyn + dn * dn) / (2.0 * dn);
    if (!(dn > A.delta_min) || gn > A.max_qsa * dn) return false;
    const double rn = sqrt(xn * xn + yn * yn);
    double lpre[4] = {L.x, L.y, L.px, L.py};
    double lhc[ORD][5];
#pragma unroll
    for (int m = 0; m < ORD; ++m)
#pragma unroll
        for (int v = 0; v < 5; ++v) lhc[m][v] = L.h[m][v];
    if (rn > A.R) {                                    // the wall reflection in reverse
        const double rr = 2.0 * A.R - rn;
        if (rr < 0.0) return false;
        const double nx = xn / rn, ny = yn / rn;
        double lnx = L.x * rr, lny = L.y * rr, lrn = -(L.x * nx + L.y * ny);
        auto refl = [&](double v0, double v1, double l0, double l1, double& o0, double& o1) {
            const double ln_ = l0 * nx + l1 * ny, vn_ = v0 * nx + v1 * ny;
            o0 = l0 - 2.0 * ln_ * nx;
            o1 = l1 - 2.0 * ln_ * ny;
            lnx += -2.0 * (ln_ * v0 + vn_ * l0);
            lny += -2.0 * (ln_ * v1 + vn_ * l1);
        };
        refl(pxn, pyn, L.px, L.py, lpre[2], lpre[3]);
#pragma unroll
        for (int m = 0; m < ORD; ++m) {
            refl(hc[m][0], hc[m][1], L.h[m][0], L.h[m][1], lhc[m][0], lhc[m][1]);
            refl(hc[m][2], hc[m][3], L.h[m][2], L.h[m][3], lhc[m][2], lhc[m][3]);
        }
        const double ldot = lnx * nx + lny * ny;
        lpre[0] = (lnx - nx * ldot) / rn + lrn * nx;
        lpre[1] = (lny - ny * ldot) / rn + lrn * ny;
    }
    const double lsum[5] = {dxi * lpre[0], dxi * lpre[1], dxi * lpre[2], dxi * lpre[3], dxi * L.dl};
#pragma unroll
    for (int m = 0; m < ORD; ++m)
#pragma unroll
        for (int v = 0; v < 5; ++v) lhc[m][v] += A.ab[m] * lsum[v];
    double lfv[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        lfv[v] = lhc[0][v];
        if (first)
#pragma unroll
            for (int m = 1; m < ORD; ++m) lfv[v] += lhc[m][v];
    }
    // the history before the push: h_old[m] became h[m + 1] (the oldest is dropped)
#pragma unroll
    for (int m = 0; m < ORD; ++m)
#pragma unroll
        for (int v = 0; v < 5; ++v) L.h[m][v] = (!first && m + 1 < ORD) ? lhc[m + 1][v] : 0.0;
    double l_X = lpre[0], l_Y = lpre[1], l_PX = lpre[2], l_PY = lpre[3], l_D = L.dl;
    double l_gam = 0, l_invd = 0, l_Wx = 0, l_Wy = 0, l_Ez = 0, l_Bz = 0, l_Bx = 0, l_By = 0;
    l_PX += lfv[0] * invd; l_invd += lfv[0] * PX;
    l_PY += lfv[1] * invd; l_invd += lfv[1] * PY;
    l_gam += lfv[2] * qm * Wx * invd;
    l_Wx += lfv[2] * qm * gam * invd;
    l_invd += lfv[2] * qm * (gam * Wx + PY * Bz);
    l_By += lfv[2] * qm;
    l_PY += lfv[2] * qm * Bz * invd;
    l_Bz += lfv[2] * qm * PY * invd;
    l_gam += lfv[3] * qm * Wy * invd;
    l_Wy += lfv[3] * qm * gam * invd;
    l_invd += lfv[3] * qm * (gam * Wy - PX * Bz);
    l_Bx -= lfv[3] * qm;
    l_PX -= lfv[3] * qm * Bz * invd;
    l_Bz -= lfv[3] * qm * PX * invd;
    l_PX += lfv[4] * qm * Wx * invd;
    l_PY += lfv[4] * qm * Wy * invd;
    l_Wx += lfv[4] * qm * PX * invd;
    l_Wy += lfv[4] * qm * PY * invd;
    l_invd += lfv[4] * qm * (PX * Wx + PY * Wy);
    l_Ez -= lfv[4] * qm;
    l_PX += l_gam * PX * invd;
    l_PY += l_gam * PY * invd;
    l_D += l_gam * (0.5 - (1.0 + PX * PX + PY * PY) * 0.5 * invd * invd);
    l_D -= l_invd * invd * invd;
    GeoAdj ga = {0, 0, 0, 0, 0, 0, 0};
    ga.c = l_Wx * R1 + l_Bx * BR + l_By * BI;
    ga.s = l_Wy * R1 - l_Bx * BI + l_By * BR;
    double val[10];
    int na = 0;
    lin_back(g, S.wpr, l_Wx * g.c + l_Wy * g.s, ga, val, na);
    lin_back(g, S.ez, l_Ez, ga, val, na);
    lin_back(g, S.bz, l_Bz, ga, val, na);
    lin_back(g, S.bpr, l_Bx * g.c + l_By * g.s, ga, val, na);
    lin_back(g, S.bpi, -l_Bx * g.s + l_By * g.c, ga, val, na);
#pragma unroll
    for (int c = 0; c < 10; ++c) sc[c] = val[c];
    jc = g.j;
    geo_back(S, g, ga, l_X, l_Y);
    L.x = l_X; L.y = l_Y; L.px = l_PX; L.py = l_PY; L.dl = l_D;
    return true;
}

// PlasmaSpecies::deposit_S (src/PlasmaSpecies.cpp:508-559, m = 0) of one particle in reverse:
// L += state adjoint; the field adjoints (W+, E_z, B_z at nodes j, j+1) are returned in sc, jc = j
template <int ORD>
__device__ void S_back(const AdjSm& S, const SweepArgs& A, const PState<ORD>& P, double (&L)[5], double (&sc)[6],
                       int& jc) {
    const double q0 = P.q, qm = P.qm;
    const PGeo g = geometry(S.r, S.ih, A.N, A.R, P.x, P.y);
    const double R1 = lin(S.wpr, g), Ez = lin(S.ez, g), Bz = lin(S.bz, g);
    const double Wx = R1 * g.c, Wy = R1 * g.s;
    const double PX = P.px, PY = P.py, D = P.dl;
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D, invd2 = invd * invd;
    const double ux = PX * invd, uy = PY * invd;
    const double ur = g.c * ux + g.s * uy, uth = g.c * uy - g.s * ux;
    const double dD = qm * ((PX * Wx + PY * Wy) * invd - Ez);
    const double nx_ = qm * (gam * Wx + PY * Bz) - PX * dD, ny_ = qm * (gam * Wy - PX * Bz) - PY * dD;
    const double ax = nx_ * invd2, ay = ny_ * invd2;
    const double wq = P.w * q0;
    GeoAdj ga = {0, 0, 0, 0, 0, 0, 0};
    double l_ax = 0, l_ay = 0, l_ux = 0, l_uy = 0, l_ur = 0, l_uth = 0;
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        const int jj = g.j + cc;
        const double W = cc ? g.W1 : g.W0, Wor = cc ? g.Wor1 : g.Wor0, dW = cc ? g.ih : -g.ih;
        const double iv = S.iv[jj] * wq;
        const double f2 = uth * Wor;
        const double Ar = ax * W + ux * ur * dW + f2 * uy;
        const double Ai = ay * W + uy * ur * dW - f2 * ux;
        const double LSr = S.l_Sr[jj], LSi = S.l_Si[jj];
        const double lAr = iv * (LSr * g.c - LSi * g.s);
        const double lAi = iv * (LSr * g.s + LSi * g.c);
        ga.c += iv * (LSr * Ar + LSi * Ai);
        ga.s += iv * (LSr * Ai - LSi * Ar);
        l_ax += lAr * W;
        l_ay += lAi * W;
        if (cc) ga.W1 += lAr * ax + lAi * ay; else ga.W0 += lAr * ax + lAi * ay;
        l_ux += lAr * ur * dW - lAi * f2;
        l_uy += lAr * f2 + lAi * ur * dW;
        l_ur += (lAr * ux + lAi * uy) * dW;
        const double l_f2 = lAr * uy - lAi * ux;
        l_uth += l_f2 * Wor;
        if (cc) ga.Wor1 += l_f2 * uth; else ga.Wor0 += l_f2 * uth;
    }
    double l_PX = 0, l_PY = 0, l_D = 0, l_gam = 0, l_invd = 0, l_Wx = 0, l_Wy = 0, l_Ez = 0, l_Bz = 0, l_dD = 0;
    l_invd += (l_ax * nx_ + l_ay * ny_) * 2.0 * invd;
    {
        const double lnx = l_ax * invd2, lny = l_ay * invd2;
        l_gam += qm * (lnx * Wx + lny * Wy);
        l_Wx += lnx * qm * gam;
        l_Wy += lny * qm * gam;
        l_PY += lnx * qm * Bz;
        l_PX -= lny * qm * Bz;
        l_Bz += qm * (lnx * PY - lny * PX);
        l_PX -= lnx * dD;
        l_PY -= lny * dD;
        l_dD -= lnx * PX + lny * PY;
    }
    l_PX += l_dD * qm * Wx * invd;
    l_PY += l_dD * qm * Wy * invd;
    l_Wx += l_dD * qm * PX * invd;
    l_Wy += l_dD * qm * PY * invd;
    l_invd += l_dD * qm * (PX * Wx + PY * Wy);
    l_Ez -= l_dD * qm;
    ga.c += l_ur * ux + l_uth * uy;
    ga.s += l_ur * uy - l_uth * ux;
    l_ux += l_ur * g.c - l_uth * g.s;
    l_uy += l_ur * g.s + l_uth * g.c;
    l_PX += l_ux * invd; l_invd += l_ux * PX;
    l_PY += l_uy * invd; l_invd += l_uy * PY;
    l_PX += l_gam * PX * invd;
    l_PY += l_gam * PY * invd;
    l_D += l_gam * (0.5 - (1.0 + PX * PX + PY * PY) * 0.5 * invd2);
    l_D -= l_invd * invd2;
    ga.c += l_Wx * R1;
    ga.s += l_Wy * R1;
    double val[10];
    int na = 0;
    lin_back(g, S.wpr, l_Wx * g.c + l_Wy * g.s, ga, val, na);
    lin_back(g, S.ez, l_Ez, ga, val, na);
    lin_back(g, S.bz, l_Bz, ga, val, na);
#pragma unroll
    for (int c = 0; c < 6; ++c) sc[c] = val[c];
    jc = g.j;
    double lx = 0.0, ly = 0.0;
    geo_back(S, g, ga, lx, ly);
    L[0] += lx; L[1] += ly; L[2] += l_PX; L[3] += l_PY; L[4] += l_D;
}

// PlasmaSpecies::deposit (src/PlasmaSpecies.cpp:409-478, m = 0) of one particle in reverse, from the
// source adjoints (rho and the densities feed nothing downstream; J_r is not used at m = 0)
template <int ORD>
__device__ void deposit_back(const AdjSm& S, const SweepArgs& A, const PState<ORD>& P, double (&L)[5]) {
    const double q0 = P.q, qm = P.qm;
    const PGeo g = geometry(S.r, S.ih, A.N, A.R, P.x, P.y);
    const double PX = P.px, PY = P.py, D = P.dl;
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D;
    const double pz = gam - D;
    const double ux = PX * invd, uy = PY * invd;
    const double uth = g.c * uy - g.s * ux;
    const double wq = P.w * q0;
    GeoAdj ga = {0, 0, 0, 0, 0, 0, 0};
    double l_pzd = 0, l_invd = 0, l_ur = 0, l_uth = 0;
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        const int jj = g.j + cc;
        const double W = cc ? g.W1 : g.W0, dW = cc ? g.ih : -g.ih;
        const double iv = S.iv[jj];
        const double a = wq * W * iv;
        const double la = S.l_rhot[jj] + S.l_jz[jj] * pz * invd + S.l_chi[jj] * qm * invd + S.l_jpi[jj] * uth;
        l_pzd += S.l_jz[jj] * a;
        l_invd += S.l_chi[jj] * a * qm;
        l_ur += S.l_drho[jj] * wq * dW * iv;
        l_uth += S.l_jpi[jj] * a;
        if (cc) ga.W1 += la * wq * iv; else ga.W0 += la * wq * iv;
    }
    double l_PX = l_pzd * PX * invd * invd, l_PY = l_pzd * PY * invd * invd;
    double l_D = -l_pzd * (1.0 + PX * PX + PY * PY) * invd * invd * invd;
    ga.c += l_ur * ux + l_uth * uy;
    ga.s += l_ur * uy - l_uth * ux;
    const double l_ux = l_ur * g.c - l_uth * g.s, l_uy = l_ur * g.s + l_uth * g.c;
    l_PX += l_ux * invd; l_invd += l_ux * PX;
    l_PY += l_uy * invd; l_invd += l_uy * PY;
    l_D -= l_invd * invd * invd;
    double lx = 0.0, ly = 0.0;
    geo_back(S, g, ga, lx, ly);
    L[0] += lx; L[1] += ly; L[2] += l_PX; L[3] += l_PY; L[4] += l_D;
}

// lam_f[j] of f -> grad f (src/FieldSolver.cpp:193-211) transposed, gathered at node j from l (shared)
__device__ __forceinline__ double grad_T_at(const SweepArgs& A, const double* gm, const double* g0, const double* gp,
                                            const double* l, int j) {
    const int N = A.N;
    double v = 0.0;
    if (j + 1 >= 1 && j + 1 <= N - 1) v += gm[j + 1] * l[j + 1];
    if (j >= 1 && j <= N - 1) v += g0[j] * l[j];
    if (j - 1 >= 1 && j - 1 <= N - 1) v += gp[j - 1] * l[j - 1];
    if (j == N) v += g0[N] * l[N];
    if (j == N - 1) v += gm[N] * l[N];
    if (j == N - 2) v += gp[N] * l[N];
    return v;
}

// the gate of a stand-alone reverse sweep: nothing to wait for
struct AdjNoGate {
    static constexpr bool kActive = false;
    __device__ bool before_slice(int) { return true; }    // warp 0: the field adjoint of row k is final
    __device__ void slice_done(int) {}                     // thread 0, after the barrier ending slice k
};

// One sweep in reverse by the calling CTA (all kSweepThreads threads): slices K-1 .. 0. The gate
// orders it against the beam adjoint tasks when several steps run concurrently. Returns false when a
// gate wait gave up.
// The smoothing filter of the forward (plasma.smooth_length) on NS shared arrays of one operator, one row per
// thread (row i). transpose = false: f <- F^-1 f (the forward filter, for chi). transpose = true:
// lam <- F^-T lam. F0 = D^-1 S with D = V / 2 pi and S symmetric, so F0^-T lam = V F0^-1 (lam / V). F1 is Q^-1 S
// on its interior rows (Q = r dV, the symmetriser of L1D) with identity rows 0 and N, row N - 1 coupled to
// x_N: F1^-T lam = Q F1^-1 (lam / Q) on the interior, lam_0 on row 0 and lam_N - c_{N-1} mu_{N-1} on row N.
// The Thomas factors fc (3 x M per operator) are the forward's. Ends with a barrier.
template <int NS>
__device__ __noinline__ void filter_rows_adj(double* const (&arr)[NS], int op, bool transpose, const double* fc,
                                             int M, int N, double Vi, double iVi, double F1i, double iF1i,
                                             double* tot, double* tot2) {
    const int i = threadIdx.x;
    const bool row = i < M, inner = i >= 1 && i < N;
    const double* F = fc + (size_t)op * 3 * M;
    double rr = 0.0, af = 1.0, ab = 1.0;
    if (row) { rr = F[i]; af = F[M + i]; ab = F[2 * M + i]; }
    double scale_in = 1.0, scale_out = 1.0;
    if (transpose) {
        scale_in = op == 0 ? iVi : (inner ? iF1i : 0.0);
        scale_out = op == 0 ? Vi : F1i;
    }
    double lam[NS], d[NS];
#pragma unroll
    for (int e = 0; e < NS; ++e) {
        lam[e] = row ? arr[e][i] : 0.0;
        d[e] = rr * (lam[e] * scale_in);
    }
    double y[NS];
    scan_fwd<NS>(af, d, y, tot);
#pragma unroll
    for (int e = 0; e < NS; ++e) y[e] = row ? fma(af, y[e], d[e]) : 0.0;
    double x[NS];
    scan_bwd<NS>(row ? ab : 1.0, y, x, tot2);
    if (row)
#pragma unroll
        for (int e = 0; e < NS; ++e) {
            const double v = fma(ab, x[e], y[e]);
            if (!transpose || op == 0) arr[e][i] = v * scale_out;
            else if (inner) arr[e][i] = v * scale_out;
            else if (i == 0) arr[e][i] = lam[e];
        }
    __syncthreads();
    if (transpose && op == 1 && i == N) {
        const double cN1 = -fc[(size_t)3 * M + 2 * M + N - 1] / fc[(size_t)3 * M + N - 1];   // c_{N-1} of F1
#pragma unroll
        for (int e = 0; e < NS; ++e) arr[e][N] = lam[e] - cN1 * arr[e][N - 1];
    }
    __syncthreads();
}

// Slice checkpointing (SweepArgs::traj_every = C > 1): the forward kept the plasma state of the slices
// k = 0, C, 2C, ... only. Before the reverse sweep reaches the last slice of segment [k0, k1] it pushes
// its particle again from the checkpoint k0 through slices k0 .. k1 - 1, with the fields the forward
// gathered there (the field store and the W+ record: the same inputs, the same push_particle), and
// keeps the states P_k0 .. P_k1 in seg (slot k - k0): the forward's trajectory bit for bit, at
// K / C + C states per sweep instead of K. The field arrays of S serve as scratch (the reverse loads
// them again for every slice); only the calling thread's particle is written and read.
template <int ORD>
__device__ void recompute_segment(const SweepArgs& A, const AdjSm& S, const double* __restrict__ ck,
                                  const double* __restrict__ fld, const double* __restrict__ wrec,
                                  double* __restrict__ seg, int k0, int k1, bool has_p, double qsp, double qmsp) {
    const int M = A.M, N = A.N, npad = A.npad, tid = threadIdx.x;
    const size_t nv = 6 + 5 * (size_t)ORD;
    PState<ORD> P;
    P.q = qsp; P.qm = qmsp;
    P.w = 0.0;
    auto put = [&](int slot) {
        double* T = seg + (size_t)slot * nv * npad + tid;
        T[0] = P.x; T[npad] = P.y; T[2 * (size_t)npad] = P.px; T[3 * (size_t)npad] = P.py;
        T[4 * (size_t)npad] = P.dl; T[5 * (size_t)npad] = P.w;
#pragma unroll
        for (int m = 0; m < ORD; ++m)
#pragma unroll
            for (int v = 0; v < 5; ++v) T[(6 + (size_t)m * 5 + v) * npad] = P.h[m][v];
    };
    if (has_p) {
        const double* T = ck + tid;
        P.x = T[0]; P.y = T[npad]; P.px = T[2 * (size_t)npad]; P.py = T[3 * (size_t)npad];
        P.dl = T[4 * (size_t)npad]; P.w = T[5 * (size_t)npad];
#pragma unroll
        for (int m = 0; m < ORD; ++m)
#pragma unroll
            for (int v = 0; v < 5; ++v) P.h[m][v] = T[(6 + (size_t)m * 5 + v) * npad];
        put(0);
    }
    sweep_detail::Smem F{};
    F.wr1 = S.wpr; F.ez = S.ez; F.bz = S.bz; F.bpr = S.bpr; F.bpi = S.bpi;
    double ab[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) ab[m] = A.ab[m];
    for (int k = k0; k < k1; ++k) {
        __syncthreads();                             // the arrays' previous contents are no longer read
        if (tid < M) {
            const double* Fk = fld + ((size_t)k * M + tid) * F_NC0;
            S.wpr[tid] = wrec ? wrec[(size_t)k * M + tid] : Fk[F_EP1R] - Fk[F_BP1I];
            S.bpr[tid] = Fk[F_BP1R];
            S.bpi[tid] = Fk[F_BP1I];
            S.ez[tid] = Fk[F_EZ0];
            S.bz[tid] = Fk[F_BZ0];
        }
        __syncthreads();
        if (has_p) {
            if (P.w != 0.0)
                (void)sweep_detail::push_particle<ORD>(P, geometry(S.r, S.ih, N, A.R, P.x, P.y), F, A, k == 0, ab,
                                                       A.dxi);
            put(k + 1 - k0);
        }
    }
    __syncthreads();
}

template <int ORD, class Gate, bool FILT = false>
__device__ bool sweep_back_body(const SweepArgs& A, const double* __restrict__ traj, const double* __restrict__ fld,
                                const double* lfld, double* __restrict__ lbsrc, double* smem_raw, Gate& gate,
                                const double* __restrict__ wrec = nullptr, double* __restrict__ seg = nullptr) {
    const int M = A.M, N = A.N, K = A.K, tid = threadIdx.x;
    const int np = A.np, npad = A.npad;
    const AdjSm S = carve_adj(smem_raw, M);
    const double* q = A.consts;                     // stencils, 1/r, L0 Thomas, L1D and L1F rows (13 x M)
    const double *gm = q, *g0 = q + M, *gp = q + 2 * M, *ir = q + 3 * M;
    const double *l0r = q + 4 * M, *l0f = q + 5 * M, *l0b = q + 6 * M;
    const double *l1a = q + 7 * M, *l1b = q + 8 * M, *l1c = q + 9 * M;
    const double *lfa = q + 10 * M, *lfb = q + 11 * M, *lfc = q + 12 * M;
    const int i = tid, lane = tid & 31;              // this thread's row
    const bool row = i < M;
    if (row) {
        S.r[i] = A.r[i];
        S.iv[i] = A.inv_V[i];
        S.ih[i] = i < N ? A.inv_h[i] : 0.0;
    }
    __syncthreads();
    // this thread's row constants: the symmetrisers F = r_j dV_j of L1D / L1F (dV_N = h_{N-1} / 2) and
    // V_j of L0, with their reciprocals (no divide inside the slice loop)
    double F1i = 1.0, iF1i = 1.0, Vi = 1.0, iVi = 1.0;
    if (row) {
        const double hm = i > 0 ? A.r[i] - A.r[i - 1] : 0.0, hp = i < N ? A.r[i + 1] - A.r[i] : 0.0;
        F1i = A.r[i] * 0.5 * (hm + hp);
        iF1i = F1i > 0.0 ? 1.0 / F1i : 0.0;
        iVi = A.inv_V[i];
        Vi = 1.0 / iVi;
        S.F1[i] = F1i;
    }
    const size_t nv = 6 + 5 * (size_t)ORD;
    const double fcoef = A.flux_coef;
    // the adjoint of this thread's particle, carried from slice k + 1 to slice k: shared memory, so
    // that no particle value stays in registers across the block scans
    constexpr int NL = 5 + 5 * ORD;
    double* Lsm = S.lam;                             // (NL, kSweepThreads)
#pragma unroll
    for (int v = 0; v < NL; ++v) Lsm[v * kSweepThreads + tid] = 0.0;
    const bool has_p = tid < np;
    double qsp = -1.0, qmsp = -1.0;
    if (has_p) species_params(A, tid, qsp, qmsp);
    int par = 0;
    unsigned long long* tim = A.timing;              // optional: clock cycles per phase, slots 9..15
    long long t_prev = (tim && tid == 0) ? clock64() : 0;
#define ADJ_MARK(ph)                                                          \
    do {                                                                      \
        if (tim && tid == 0) {                                                \
            const long long tn = clock64();                                   \
            tim[9 + (ph)] += (unsigned long long)(tn - t_prev);               \
            t_prev = tn;                                                      \
        }                                                                     \
    } while (0)
    // where the state of slice k is read: the whole trajectory (cur = traj, kbase = 0), or the
    // recomputed segment of slice k (cur = seg, kbase = its first slice)
    if (A.traj_every > 1 && !seg) return false;      // a checkpointed trajectory needs the segment buffer
    const int every = A.traj_every > 1 ? A.traj_every : 1;
    const double* cur = traj;
    int kbase = 0;
    // this thread's particle P_k from the trajectory (the history only when asked)
    auto load_p = [&](int k, PState<ORD>& P, bool hist) {
        P.q = qsp; P.qm = qmsp;
        P.w = 0.0;
        P.x = P.y = P.px = P.py = 0.0;
        P.dl = 1.0;
        if (!has_p) return;
        const double* T = cur + (size_t)(k - kbase) * nv * npad + tid;
        P.x = T[0]; P.y = T[npad]; P.px = T[2 * (size_t)npad]; P.py = T[3 * (size_t)npad];
        P.dl = T[4 * (size_t)npad]; P.w = T[5 * (size_t)npad];
        if (hist)
#pragma unroll
            for (int m = 0; m < ORD; ++m)
#pragma unroll
                for (int v = 0; v < 5; ++v) P.h[m][v] = T[(6 + (size_t)m * 5 + v) * npad];
    };
    for (int k = K - 1; k >= 0; --k) {
        if (every > 1 && (k == K - 1 || (k + 1) % every == 0)) {
            // the segment ending at slice k, pushed again from its checkpoint (needs no gate: the
            // forward's records are complete)
            const int g = k / every;
            recompute_segment<ORD>(A, S, traj + (size_t)g * nv * npad, fld, wrec, seg, g * every, k, has_p, qsp, qmsp);
            cur = seg;
            kbase = g * every;
        }
        if (Gate::kActive) {                         // the field adjoint of row k is complete
            if (tid < 32) {
                const bool ok = gate.before_slice(k);
                if (tid == 0) *S.flag = ok ? 1 : 0;
            }
            __syncthreads();
            if (!*S.flag) return false;
        }
        // ---- this slice's fields and field adjoints (store in reverse)
        bool alive = false;
        if (has_p) alive = cur[(size_t)(k - kbase) * nv * npad + 5 * (size_t)npad + tid] != 0.0;
        ADJ_MARK(0);
        if (row) {
            const double* F = fld + ((size_t)k * M + i) * F_NC0;
            const double* LF = lfld + ((size_t)k * M + i) * F_NC0;
            S.wpr[i] = wrec ? wrec[(size_t)k * M + i] : F[F_EP1R] - F[F_BP1I];
            S.bpr[i] = F[F_BP1R];
            S.bpi[i] = F[F_BP1I];
            S.ez[i] = F[F_EZ0];
            S.bz[i] = F[F_BZ0];
            S.chi[i] = 0.0;
            double lf[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) lf[c] = beam_detail::fload<Gate::kActive>(LF + c);
            S.l_wpr[i] = lf[F_EP1R];
            S.l_bpi[i] = lf[F_EP1R] + lf[F_BP1I];
            S.l_bpr[i] = lf[F_BP1R] - lf[F_EP1I];
            S.l_ez[i] = lf[F_EZ0];
            S.l_bz[i] = lf[F_BZ0];
            S.l_rhot[i] = S.l_drho[i] = S.l_jz[i] = S.l_chi[i] = S.l_jpi[i] = S.l_Sr[i] = S.l_Si[i] = 0.0;
        }
        __syncthreads();
        // ---- chi of the slice (the plasma deposit of P_k) and the push of slice k in reverse; the
        // shared-memory updates are summed over runs of lanes on the same node first (blowout piles
        // many particles into a few sheath and axis cells)
        {
            PState<ORD> P;
            load_p(k, P, k + 1 < K);
            double cv[2] = {0.0, 0.0};
            int key = -1 - lane;
            if (alive) {
                const PGeo g = geometry(S.r, S.ih, N, A.R, P.x, P.y);
                cv[0] = P.w * P.q * g.W0 * S.iv[g.j] * P.qm / P.dl;
                cv[1] = P.w * P.q * g.W1 * S.iv[g.j + 1] * P.qm / P.dl;
                key = g.j;
            }
            if (warp_runs_sum<2>(key, cv) && key >= 0) {
                double* adr[2] = {S.chi + key, S.chi + key + 1};
                add_multi<2>(adr, cv);
            }
            PAdj<ORD> Lp;
            bool kept = false;
            double sc[10];
            int jc = -1;
            if (alive && k + 1 < K) {
                Lp.x = Lsm[0 * kSweepThreads + tid]; Lp.y = Lsm[1 * kSweepThreads + tid];
                Lp.px = Lsm[2 * kSweepThreads + tid]; Lp.py = Lsm[3 * kSweepThreads + tid];
                Lp.dl = Lsm[4 * kSweepThreads + tid];
#pragma unroll
                for (int m = 0; m < ORD; ++m)
#pragma unroll
                    for (int v = 0; v < 5; ++v) Lp.h[m][v] = Lsm[(5 + m * 5 + v) * kSweepThreads + tid];
                kept = push_back<ORD>(S, A, P, k == 0, Lp, sc, jc);
            }
            if (!kept) {
#pragma unroll
                for (int c = 0; c < 10; ++c) sc[c] = 0.0;
            }
            key = kept ? jc : -1 - lane;
            if (warp_runs_sum<10>(key, sc) && key >= 0) {
                double* adr[10] = {S.l_wpr + key, S.l_wpr + key + 1, S.l_ez + key, S.l_ez + key + 1, S.l_bz + key,
                                   S.l_bz + key + 1, S.l_bpr + key, S.l_bpr + key + 1, S.l_bpi + key, S.l_bpi + key + 1};
                add_multi<10>(adr, sc);
            }
            // the adjoint of P_k so far: the push's, or nothing
            Lsm[0 * kSweepThreads + tid] = kept ? Lp.x : 0.0;
            Lsm[1 * kSweepThreads + tid] = kept ? Lp.y : 0.0;
            Lsm[2 * kSweepThreads + tid] = kept ? Lp.px : 0.0;
            Lsm[3 * kSweepThreads + tid] = kept ? Lp.py : 0.0;
            Lsm[4 * kSweepThreads + tid] = kept ? Lp.dl : 0.0;
#pragma unroll
            for (int m = 0; m < ORD; ++m)
#pragma unroll
                for (int v = 0; v < 5; ++v) Lsm[(5 + m * 5 + v) * kSweepThreads + tid] = kept ? Lp.h[m][v] : 0.0;
        }
        __syncthreads();
        if constexpr (FILT) {                         // B+ saw the smoothed chi (src/Simulation.cpp:823-835)
            double* const fa[1] = {S.chi};
            filter_rows_adj<1>(fa, 0, false, A.fconsts, M, N, Vi, iVi, F1i, iF1i, S.tot + (par++ & 1) * 8 * kW,
                               S.tot + (par++ & 1) * 8 * kW);
        }
        ADJ_MARK(1);
        // ---- B+ (src/Simulation.cpp:535-591) in reverse: mu = F (L - chi)^-1 (F^-1 lam) per system
        {
            double m[2][4], ra[2], rbv[2], rc[2], rd[2];
#pragma unroll
            for (int sy = 0; sy < 2; ++sy) {
                m[sy][0] = 1.0; m[sy][1] = 0.0; m[sy][2] = 0.0; m[sy][3] = 1.0;
                ra[sy] = 0.0; rbv[sy] = 1.0; rc[sy] = 0.0; rd[sy] = 0.0;
            }
            if (row) {
                // sys 0: L1D - chi (rows 0, N Dirichlet); sys 1: L1F - chi (row 0 Dirichlet)
                ra[0] = l1a[i]; rbv[0] = l1b[i]; rc[0] = i > 0 ? l1c[i - 1] : 0.0;
                if (i >= 1 && i < N) { rbv[0] -= S.chi[i]; rd[0] = S.l_bpr[i] * iF1i; }
                ra[1] = lfa[i]; rbv[1] = lfb[i]; rc[1] = i > 0 ? lfc[i - 1] : 0.0;
                if (i >= 1) { rbv[1] -= S.chi[i]; rd[1] = S.l_bpi[i] * iF1i; }
#pragma unroll
                for (int sy = 0; sy < 2; ++sy) {
                    m[sy][0] = rbv[sy]; m[sy][1] = -ra[sy] * rc[sy]; m[sy][2] = 1.0; m[sy][3] = 0.0;
                    renorm(m[sy][0], m[sy][1], m[sy][2], m[sy][3]);
                }
            }
            double pp[2], qq[2];
            scan_pivots<2>(m, pp, qq, S.tot + (par++ & 1) * 8 * kW);
            double rinv[2], fA[2], fB[2];
#pragma unroll
            for (int sy = 0; sy < 2; ++sy) {
                rinv[sy] = 0.0; fA[sy] = 1.0; fB[sy] = 0.0;
                if (!row) continue;
                const double pn = rbv[sy] * pp[sy] - ra[sy] * rc[sy] * qq[sy];
                rinv[sy] = pp[sy] / pn;
                fA[sy] = -rinv[sy] * ra[sy];
                fB[sy] = rinv[sy] * rd[sy];
            }
            double yy[2];
            scan_fwd_n<2>(fA, fB, yy, S.tot + (par++ & 1) * 8 * kW);
            double y[2], bA[2], bB[2];
#pragma unroll
            for (int sy = 0; sy < 2; ++sy) {
                y[sy] = row ? fma(fA[sy], yy[sy], fB[sy]) : 0.0;
                const double c = row ? (sy ? lfc[i] : l1c[i]) : 0.0;
                bA[sy] = row ? -(c * rinv[sy]) : 1.0;
                bB[sy] = y[sy];
            }
            double xx[2];
            scan_bwd_n<2>(bA, bB, xx, S.tot + (par++ & 1) * 8 * kW);
            if (row) {
                const double mu0 = (i >= 1 && i < N) ? fma(bA[0], xx[0], y[0]) * F1i : 0.0;
                const double mu1 = (i >= 1) ? fma(bA[1], xx[1], y[1]) * F1i : 0.0;
                S.l_chi[i] = mu0 * S.bpr[i] + mu1 * S.bpi[i];
                S.l_Si[i] = -mu0;
                S.l_Sr[i] = mu1;                     // lam of the B_theta right-hand side (J_z' + S_r)
                S.t0[i] = mu1;
            }
        }
        __syncthreads();
        ADJ_MARK(2);
        if (row) S.l_jz[i] = grad_T_at(A, gm, g0, gp, S.t0, i) - (i == N ? fcoef * S.t0[N] : 0.0);
        if constexpr (FILT) {                         // the S+ filter (src/Simulation.cpp:810-812) in reverse
            double* const fa[2] = {S.l_Sr, S.l_Si};
            filter_rows_adj<2>(fa, 1, true, A.fconsts, M, N, Vi, iVi, F1i, iF1i, S.tot + (par++ & 1) * 8 * kW,
                               S.tot + (par++ & 1) * 8 * kW);
        }
        // ---- the S deposit in reverse (adds to lam of W+, E_z, B_z)
        {
            double sc[6] = {0, 0, 0, 0, 0, 0};
            int key = -1 - lane;
            if (alive) {
                PState<ORD> P;
                load_p(k, P, false);
                double l5[5] = {0, 0, 0, 0, 0};
                int jc = 0;
                S_back<ORD>(S, A, P, l5, sc, jc);
                key = jc;
#pragma unroll
                for (int v = 0; v < 5; ++v) Lsm[v * kSweepThreads + tid] += l5[v];
            }
            if (warp_runs_sum<6>(key, sc) && key >= 0) {
                double* adr[6] = {S.l_wpr + key, S.l_wpr + key + 1, S.l_ez + key, S.l_ez + key + 1, S.l_bz + key,
                                  S.l_bz + key + 1};
                add_multi<6>(adr, sc);
            }
        }
        __syncthreads();
        ADJ_MARK(3);
        // ---- psi (W+ = -psi'), E_z, B_z: three L0 systems, mu = V L0^-1 (lam / V) on rows < N
        if (row) S.t1[i] = -S.l_wpr[i];
        __syncthreads();
        {
            double d[3] = {0.0, 0.0, 0.0};
            double af = 1.0, rr = 0.0, ab = 1.0;
            if (row) {
                af = l0f[i]; rr = l0r[i]; ab = l0b[i];
                if (i < N) {
                    d[0] = S.l_bz[i] * iVi;
                    d[1] = grad_T_at(A, gm, g0, gp, S.t1, i) * iVi;   // lam of psi
                    d[2] = S.l_ez[i] * iVi;
                }
            }
            double cB[3];
#pragma unroll
            for (int e = 0; e < 3; ++e) cB[e] = rr * d[e];
            double yb[3];
            scan_fwd<3>(af, cB, yb, S.tot + (par++ & 1) * 8 * kW);
            double y[3];
#pragma unroll
            for (int e = 0; e < 3; ++e) y[e] = row ? fma(af, yb[e], cB[e]) : 0.0;
            double xa[3];
            scan_bwd<3>(row ? ab : 1.0, y, xa, S.tot + (par++ & 1) * 8 * kW);
            if (row) {
                double mu[3] = {0.0, 0.0, 0.0};
                if (i < N) {
#pragma unroll
                    for (int e = 0; e < 3; ++e) mu[e] = fma(ab, xa[e], y[e]) * Vi;
                }
                S.t0[i] = -mu[0];                    // lam of the B_z right-hand side -(J_th' + J_th / r)
                S.l_rhot[i] = -mu[1];
                S.l_drho[i] = -mu[2];
            }
        }
        __syncthreads();
        ADJ_MARK(4);
        if (row) {
            // J_theta: (grad_odd + over_r)^T of t0, the adjoint of (grad_odd + over_r) J_theta
            double v = grad_T_at(A, gm, g0, gp, S.t0, i);
            if (i == 1) v += ir[0] * S.t0[0] * 2.0;  // grad_odd row 0 (f1 / r1) and over_r row 0 (f1 ir0)
            if (i >= 1) v += ir[i] * S.t0[i];
            S.l_jpi[i] = v;
            // the beam source adjoints of rows k and k +- 1 (combine_sources, src/Simulation.cpp:408-457)
            double* Lk = lbsrc + ((size_t)k * M + i) * B_NC0;
            Lk[B_RT0] += S.l_rhot[i];
            Lk[B_JZ0] += S.l_jz[i];
            Lk[B_JP1I] += v;
            const double ld = S.l_drho[i] * A.idxi;
            const size_t st = (size_t)M * B_NC0;
            if (A.ngp) {     // the backward difference (the row ahead of the box head is zero)
                Lk[B_RT0] += ld;
                if (k > 0) Lk[B_RT0 - (ptrdiff_t)st] -= ld;
            } else if (K > 1) {
                if (k == 0) { Lk[st + B_RT0] += ld; Lk[B_RT0] -= ld; }
                else if (k == K - 1) { Lk[B_RT0] += ld; Lk[B_RT0 - (ptrdiff_t)st] -= ld; }
                else { Lk[st + B_RT0] += 0.5 * ld; Lk[B_RT0 - (ptrdiff_t)st] -= 0.5 * ld; }
            }
        }
        __syncthreads();
        if constexpr (FILT) {   // the filter of the plasma deposit in reverse (the beams came after it)
            double* const f0[4] = {S.l_rhot, S.l_drho, S.l_jz, S.l_chi};
            filter_rows_adj<4>(f0, 0, true, A.fconsts, M, N, Vi, iVi, F1i, iF1i, S.tot + (par++ & 1) * 8 * kW,
                               S.tot + (par++ & 1) * 8 * kW);
            double* const f1[1] = {S.l_jpi};
            filter_rows_adj<1>(f1, 1, true, A.fconsts, M, N, Vi, iVi, F1i, iF1i, S.tot + (par++ & 1) * 8 * kW,
                               S.tot + (par++ & 1) * 8 * kW);
        }
        ADJ_MARK(5);
        // ---- the plasma deposit of P_k in reverse
        if (alive) {
            PState<ORD> P;
            load_p(k, P, false);
            double l5[5] = {0, 0, 0, 0, 0};
            deposit_back<ORD>(S, A, P, l5);
#pragma unroll
            for (int v = 0; v < 5; ++v) Lsm[v * kSweepThreads + tid] += l5[v];
        }
        __syncthreads();
        ADJ_MARK(6);
        if (Gate::kActive && tid == 0) gate.slice_done(k);   // beam-source adjoint rows > k are final
    }
#undef ADJ_MARK
    return true;
}

template <int ORD, bool FILT>
__global__ void __launch_bounds__(kSweepThreads, 1) sweep_back_kernel(const __grid_constant__ SweepArgs A,
                                                                       const double* __restrict__ traj,
                                                                       const double* __restrict__ fld,
                                                                       const double* __restrict__ lfld,
                                                                       double* __restrict__ lbsrc) {
    extern __shared__ double smem_raw[];
    AdjNoGate g;
    sweep_back_body<ORD, AdjNoGate, FILT>(A, traj, fld, lfld, lbsrc, smem_raw, g);
}

// ------------------------------------------------------------------ the reverse pass as a pipeline
// Every wait spins on an acquire load, bounded by %globaltimer: on time-out it records the place in
// *err and returns, and every other wait gives up as soon as *err is set.
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
enum AdjWaitSite { AW_ROWS = 1, AW_TASK = 2 };

// wait until *p <= v
__device__ bool wait_le(const AdjPipeArgs& P, const int* p, int v, int site) {
    if (ld_acquire(p) <= v) return true;
    const unsigned long long t0 = gtimer();
    for (;;) {
        __nanosleep(64);
        if (ld_acquire(p) <= v) return true;
        if (ld_acquire(P.err) != 0) return false;
        if (gtimer() - t0 > P.timeout_ns) {
            atomicCAS(P.err, 0, (site << 8) | 1);
            return false;
        }
    }
}

struct AdjGateState {
    int n;          // step of this reverse sweep
    int cursor;     // buckets [cursor, nbk) are known to have finished their task of step n
};

struct AdjPipeGate {
    static constexpr bool kActive = true;
    const AdjPipeArgs* P;
    AdjGateState* g;    // shared
    // warp 0: every bucket that can add to the field adjoint of row k has finished its push of step n
    // in reverse. Those are the buckets from the first whose running maximum of (highest cell + 1)
    // reaches k; they finish from the tail, so the lanes walk 32 buckets at a time downwards.
    __device__ bool before_slice(int k) {
        const int lane = threadIdx.x & 31;
        const int n = g->n, nbk = P->nbk;
        const int* pm = P->pmax + (size_t)n * nbk;
        int lo = 0, hi = nbk;                                 // first b with pm[b] >= k
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(pm + mid) >= k) hi = mid; else lo = mid + 1;
        }
        const int need = lo;
        int c = g->cursor;
        while (c > need) {
            const int b = c - 1 - lane;
            const bool done = b < need || ld_acquire(P->bdone + b) <= n;
            const unsigned m = __ballot_sync(0xffffffffu, done);
            const int run = (m == 0xffffffffu) ? 32 : __ffs(~m) - 1;
            c = max(c - run, need);
            if (run == 32 || c <= need) continue;
            bool ok = true;
            if (lane == 0) ok = wait_le(*P, P->bdone + (c - 1), n, AW_ROWS);
            if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) return false;
        }
        __syncwarp();
        if (lane == 0) g->cursor = c;
        __syncwarp();
        return ld_acquire(P->err) == 0;
    }
    // thread 0 after the barrier ending slice k: the beam-source adjoint rows > k are final
    __device__ void slice_done(int k) {
        __threadfence();
        st_release(P->prog + g->n, k);
    }
};

template <int ORD, bool FILT>
__device__ void adj_sweep_role(const AdjPipeArgs& P, double* smem) {
    __shared__ AdjGateState gs;
    const int T = P.nsteps;
    for (int l = blockIdx.x; l < T; l += P.nsweep) {
        const int n = T - 1 - l;
        if (threadIdx.x == 0) {
            gs.n = n;
            gs.cursor = P.nbk;
        }
        __syncthreads();
        AdjPipeGate g{&P, &gs};
        if (!sweep_back_body<ORD, AdjPipeGate, FILT>(
                P.sw, P.traj + (size_t)n * P.traj_slot, P.fld + (size_t)n * P.fld_slot,
                P.lfld + (size_t)n * P.lfld_slot, P.lbsrc + (size_t)n * P.lbsrc_slot, smem, g,
                P.wrec ? P.wrec + (size_t)n * (P.fld_slot / F_NC0) : nullptr,
                P.seg ? P.seg + (size_t)blockIdx.x * P.seg_slot : nullptr))
            return;
        __syncthreads();
    }
}

// task (layer l, bucket b), step n = nsteps - 1 - l: bucket b finished step n + 1, and the beam-source
// adjoint of step n + 1 is final on the bucket's rows there
__device__ __forceinline__ bool adj_task_ready(const AdjPipeArgs& P, int l, int b) {
    const int T = P.nsteps, n = T - 1 - l;
    if (n + 1 <= T - 1) {
        if (ld_acquire(P.bdone + b) > n + 1) return false;
        const int cm = __ldg(P.cmin + (size_t)(n + 1) * P.nbk + b);
        if (cm != 0x7fffffff && ld_acquire(P.prog + n + 1) > max(max(cm, 0) - 1, 0)) return false;
    }
    return true;
}

// warp-collective: claim a ready task, lowest layer first (tail buckets first within a layer)
__device__ __forceinline__ bool adj_claim(const AdjPipeArgs& P, int& l, int& b) {
    const int lane = threadIdx.x & 31;
    const int last = P.nsteps;                                 // layers 0 .. nsteps
    const unsigned long long t0 = gtimer();
    unsigned sleep_ns = 64;
    for (;;) {
        if (ld_acquire(P.err) != 0) return false;
        const int lo = __shfl_sync(0xffffffffu, lane == 0 ? ld_acquire(P.lo) : 0, 0);
        if (lo > last) return false;
        for (int base = lo; base <= last; base += 32) {
            const int m = base + lane;
            int idx = P.nbk;
            bool ready = false;
            if (m <= last) {
                idx = ld_acquire(P.next + m);
                if (idx < P.nbk) ready = adj_task_ready(P, m, P.nbk - 1 - idx);
            }
            const unsigned full = __ballot_sync(0xffffffffu, idx >= P.nbk);
            if (base == lo && (full & 1u)) {
                const int c = (~full == 0u) ? 32 : __ffs(~full) - 1;
                if (lane == 0) atomicMax(P.lo, base + c);
            }
            unsigned rm = __ballot_sync(0xffffffffu, ready);
            const int rot = (int)((blockIdx.x * (kSweepThreads / 32) + (threadIdx.x >> 5)) & 31);
            while (rm) {
                const unsigned hi = rm >> rot, low = rm & ((1u << rot) - 1u);
                const int src = hi ? rot + __ffs(hi) - 1 : __ffs(low) - 1;
                int got = 0;
                if (lane == src) got = atomicCAS(P.next + m, idx, idx + 1) == idx ? 1 : 0;
                if (__shfl_sync(0xffffffffu, got, src)) {
                    l = base + src;
                    b = P.nbk - 1 - __shfl_sync(0xffffffffu, idx, src);
                    return true;
                }
                rm &= ~(1u << src);
            }
        }
        __nanosleep(sleep_ns);
        sleep_ns = min(2 * sleep_ns, 8192u);
        if (gtimer() - t0 > P.timeout_ns) {
            if (lane == 0) atomicCAS(P.err, 0, (AW_TASK << 8) | 1);
            return false;
        }
    }
}

__device__ __forceinline__ void beam_at(BeamArgs& B, const AdjPipeArgs& P, int bb, int step) {
    const double* d = P.snap + (size_t)step * P.snap_step + P.snap_off[bb];
    const long n = B.n;
    B.x = const_cast<double*>(d); B.y = B.x + n; B.px = B.x + 2 * n; B.py = B.x + 3 * n; B.pz = B.x + 4 * n;
    B.xi = B.x + 5 * n; B.w = B.x + 6 * n;
}

__device__ void adj_worker_role(const AdjPipeArgs& P, double* smem) {
    const int tid = threadIdx.x, lane = tid & 31;
    const int M = P.sw.M, N = P.sw.N;
    double* r = smem;
    double* ih = r + M;
    double* iV = ih + M;
    for (int j = tid; j < M; j += kSweepThreads) {
        r[j] = P.sw.r[j];
        iV[j] = P.sw.inv_V[j];
        if (j < N) ih[j] = P.sw.inv_h[j];
    }
    __syncthreads();
    const int T = P.nsteps;
    int l, b;
    while (adj_claim(P, l, b)) {
        const int n = T - 1 - l;
        const int bb = __ldg(P.bk_beam + b);
        const long i0 = __ldg(P.bk_start + b), i1 = __ldg(P.bk_end + b);
        BeamArgs B1 = P.beam[bb], B0 = P.beam[bb];
        B1.r = B0.r = r;
        B1.inv_h = B0.inv_h = ih;
        B1.inv_V = B0.inv_V = iV;
        if (n + 1 <= T - 1) beam_at(B1, P, bb, n + 1);
        if (n >= 0) beam_at(B0, P, bb, n);
        const long nn = B0.n;
        double* lam = P.lam + P.lam_off[bb];
        const double* lb1 = P.lbsrc + (size_t)(n + 1) * P.lbsrc_slot;
        const double* fld = P.fld + (size_t)(n >= 0 ? n : 0) * P.fld_slot;
        double* lfld = P.lfld + (size_t)(n >= 0 ? n : 0) * P.lfld_slot;
        const int startup = (n == 0 && P.startup[bb]) ? 1 : 0;
        const bool rigid = P.rigid[bb] != 0;
        // lanes in step over the bucket (runs of equal cells sum their field adjoints across the warp)
        for (long base = i0; base < i1; base += 32) {
            const long i = base + lane;
            double g[24];
            int key = -1;
            if (i < i1) {
                double l7[7];
#pragma unroll
                for (int c = 0; c < 7; ++c) l7[c] = __ldcg(lam + c * nn + i);
                if (n + 1 <= T - 1) deposit_back_one<true>(B1, lb1, i, l7);
                if (n >= 0 && !rigid) push_back_one<true>(B0, fld, i, l7, lfld, P.dt, P.dt, startup, g, key);
#pragma unroll
                for (int c = 0; c < 7; ++c) __stcg(lam + c * nn + i, l7[c]);
            }
            if (n >= 0 && !rigid) {
                if (key < 0) {
                    key = -1 - lane;
#pragma unroll
                    for (int c = 0; c < 24; ++c) g[c] = 0.0;
                }
                if (warp_runs_sum<24>(key, g) && key >= 0) {
                    double* g0 = lfld + (size_t)key * F_NC0;             // (k, j); (k+1, j) is M rows on
                    double* g1 = g0 + (size_t)M * F_NC0;
                    const int comp[6] = {F_EP1R, F_EP1I, F_BP1R, F_BP1I, F_EZ0, F_BZ0};
#pragma unroll
                    for (int q = 0; q < 6; ++q) {
                        atomicAdd(g0 + comp[q], g[q * 4 + 0]);
                        atomicAdd(g0 + F_NC0 + comp[q], g[q * 4 + 1]);
                        if (!B0.ngp) {        // ngp: one row (k may be the last slice)
                            atomicAdd(g1 + comp[q], g[q * 4 + 2]);
                            atomicAdd(g1 + F_NC0 + comp[q], g[q * 4 + 3]);
                        }
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0) {
            __threadfence();
            st_release(P.bdone + b, n);
        }
        __syncwarp();
    }
}

template <int ORD, bool FILT>
__global__ void __launch_bounds__(kSweepThreads, 1) adjoint_pipeline_kernel(const __grid_constant__ AdjPipeArgs P) {
    extern __shared__ double smem_raw[];
    if ((int)blockIdx.x < P.nsweep)
        adj_sweep_role<ORD, FILT>(P, smem_raw);
    else
        adj_worker_role(P, smem_raw);
}

// lowest / highest live xi cell of bucket b at step n, from the snapshots (one warp per (n, b))
__global__ void bucket_cells_kernel(const __grid_constant__ AdjPipeArgs P, int* __restrict__ cmin,
                                    int* __restrict__ cmax) {
    const int lane = threadIdx.x & 31;
    const long w = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long total = (long)(P.nsteps + 1) * P.nbk;
    if (w >= total) return;
    const int n = (int)(w / P.nbk), b = (int)(w % P.nbk);
    const int bb = P.bk_beam[b];
    BeamArgs B = P.beam[bb];
    beam_at(B, P, bb, n);
    int lo = 0x7fffffff, hi = -2;
    for (long i = P.bk_start[b] + lane; i < P.bk_end[b]; i += 32) {
        if (B.w[i] == 0.0) continue;
        const int c = beam_detail::xi_cell(B, B.xi[i]);
        lo = min(lo, c);
        hi = max(hi, c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) {
        cmin[w] = lo;
        cmax[w] = hi;
    }
}

// per step: pmax[b] = max over b' <= b of (cmax + 1) (a serial scan per step: nbk is a few thousand)
__global__ void bucket_pmax_kernel(const __grid_constant__ AdjPipeArgs P, const int* __restrict__ cmax,
                                   int* __restrict__ pmax) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.nsteps) return;
    int m = -1;
    for (int b = 0; b < P.nbk; ++b) {
        m = max(m, cmax[(size_t)n * P.nbk + b] + 1);
        pmax[(size_t)n * P.nbk + b] = m;
    }
}

template <int ORD>
cudaError_t launch_adj_pipe_t(const AdjPipeArgs& P, int grid, size_t smem, cudaStream_t st) {
    auto fn = P.sw.filter ? adjoint_pipeline_kernel<ORD, true> : adjoint_pipeline_kernel<ORD, false>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    void* args[] = {(void*)&P};
    return cudaLaunchCooperativeKernel((const void*)fn, dim3(grid), dim3(kSweepThreads), args, smem, st);
}

template <int ORD>
int adj_pipe_occupancy_t(size_t smem, bool filt) {
    auto fn = filt ? adjoint_pipeline_kernel<ORD, true> : adjoint_pipeline_kernel<ORD, false>;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kSweepThreads, smem) != cudaSuccess) return 0;
    return nb;
}

template <int ORD>
cudaError_t launch_sweep_back_t(const SweepArgs& A, const double* traj, const double* fld, const double* lfld,
                                double* lbsrc, cudaStream_t st) {
    const size_t smem = adjoint_sweep_smem_bytes(A.M);
    auto fn = A.filter ? sweep_back_kernel<ORD, true> : sweep_back_kernel<ORD, false>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    fn<<<1, kSweepThreads, smem, st>>>(A, traj, fld, lfld, lbsrc);
    return cudaGetLastError();
}

}  // namespace adj

size_t adjoint_sweep_smem_bytes(int M) {
    return sizeof(double) * ((size_t)(adj::kAdjArrays + 2) * M + 2 * 8 * (kSweepThreads / 32) +
                             (size_t)(5 + 5 * adj::kMaxOrd) * kSweepThreads) + 16;
}

cudaError_t launch_sweep_back(const SweepArgs& A, const double* traj, const double* fld, const double* lfld,
                              double* lbsrc, cudaStream_t st) {
    if (A.M > kSweepThreads || A.np > kSweepThreads) return cudaErrorInvalidValue;
    switch (A.ord) {
        case 1: return adj::launch_sweep_back_t<1>(A, traj, fld, lfld, lbsrc, st);
        case 2: return adj::launch_sweep_back_t<2>(A, traj, fld, lfld, lbsrc, st);
        case 3: return adj::launch_sweep_back_t<3>(A, traj, fld, lfld, lbsrc, st);
        case 4: return adj::launch_sweep_back_t<4>(A, traj, fld, lfld, lbsrc, st);
        case 5: return adj::launch_sweep_back_t<5>(A, traj, fld, lfld, lbsrc, st);
        default: return cudaErrorInvalidValue;
    }
}

size_t adjoint_pipeline_smem_bytes(int M) {
    const size_t worker = sizeof(double) * 3 * (size_t)M + 64;
    const size_t sweep = adjoint_sweep_smem_bytes(M);
    return sweep > worker ? sweep : worker;
}

int adjoint_pipeline_max_grid(const AdjPipeArgs& P, int* sms) {
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    *sms = nsm;
    const size_t smem = adjoint_pipeline_smem_bytes(P.sw.M);
    int per = 0;
    switch (P.sw.ord) {
        case 1: per = adj::adj_pipe_occupancy_t<1>(smem, P.sw.filter != 0); break;
        case 2: per = adj::adj_pipe_occupancy_t<2>(smem, P.sw.filter != 0); break;
        case 3: per = adj::adj_pipe_occupancy_t<3>(smem, P.sw.filter != 0); break;
        case 4: per = adj::adj_pipe_occupancy_t<4>(smem, P.sw.filter != 0); break;
        case 5: per = adj::adj_pipe_occupancy_t<5>(smem, P.sw.filter != 0); break;
        default: return 0;
    }
    return per * nsm;
}

cudaError_t launch_adjoint_pipeline(const AdjPipeArgs& P, int grid, cudaStream_t st) {
    if (P.sw.M > kSweepThreads || P.sw.np > kSweepThreads || P.nsweep < 1 || grid <= P.nsweep ||
        P.nbeams > kMaxBeams || P.nsteps < 1)
        return cudaErrorInvalidValue;
    const size_t smem = adjoint_pipeline_smem_bytes(P.sw.M);
    switch (P.sw.ord) {
        case 1: return adj::launch_adj_pipe_t<1>(P, grid, smem, st);
        case 2: return adj::launch_adj_pipe_t<2>(P, grid, smem, st);
        case 3: return adj::launch_adj_pipe_t<3>(P, grid, smem, st);
        case 4: return adj::launch_adj_pipe_t<4>(P, grid, smem, st);
        case 5: return adj::launch_adj_pipe_t<5>(P, grid, smem, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_bucket_cells(const AdjPipeArgs& P, int* cmin, int* cmax, int* pmax, cudaStream_t st) {
    if (P.nbk <= 0) return cudaSuccess;
    const long warps = (long)(P.nsteps + 1) * P.nbk;
    adj::bucket_cells_kernel<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(P, cmin, cmax);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    adj::bucket_pmax_kernel<<<(P.nsteps + 63) / 64, 64, 0, st>>>(P, cmax, pmax);
    return cudaGetLastError();
}

static int beam_grid(long n) {
    long g = (n + 255) / 256;
    return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

cudaError_t launch_sums_back(const BeamArgs& B, double gref, double xiref, const double* lamS, double* lam,
                             cudaStream_t st) {
    if (B.n == 0) return cudaSuccess;
    adj::sums_back_kernel<<<beam_grid(B.n), 256, 0, st>>>(B, gref, xiref, lamS, lam);
    return cudaGetLastError();
}

cudaError_t launch_push_back(const BeamArgs& B, const double* fld, double* lam, double* lfld, double dt_kick, double dt,
                             int startup, cudaStream_t st) {
    if (B.n == 0) return cudaSuccess;
    adj::push_back_kernel<<<beam_grid(B.n), 256, 0, st>>>(B, fld, lam, lfld, dt_kick, dt, startup);
    return cudaGetLastError();
}

cudaError_t launch_deposit_back(const BeamArgs& B, const double* lbsrc, double* lam, cudaStream_t st) {
    if (B.n == 0) return cudaSuccess;
    adj::deposit_back_kernel<<<beam_grid(B.n), 256, 0, st>>>(B, lbsrc, lam);
    return cudaGetLastError();
}

}  // namespace qzb
