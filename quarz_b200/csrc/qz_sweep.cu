// qz_sweep.cu -- the quasi-static xi sweep of one time step as ONE persistent CTA (sm_100a, FP64).
//
// Replaces the per-slice kernel chain of Simulation::step_fields (src/Simulation.cpp:636-795):
//   zero_sources -> PlasmaSpecies::deposit -> combine_sources -> solve_slice_fields
//   (psi, E_z, W+, B_z, deposit_S, B+) -> store_slice -> PlasmaSpecies::push
// for azimuthal mode m = 0.
//
// Layout. All radial arrays of a slice (sources, fields, grid, stencils, operator rows) live in
// shared memory. With at most kThreads plasma particles, thread p owns particle p and keeps its
// state -- position, momentum, Delta, weight and the Adams-Bashforth history -- in registers for
// the whole sweep; larger plasmas keep the state in a global scratch buffer instead.
//
// Slice schedule (4 block barriers per slice when the sources are double-buffered):
//   P2  warps 0-2: psi (+W+), E_z, B_z solves          | warps 3-15: sources of slice k+1 = beam + background
//   P3  all: S+ deposit
//   P4  warps 0-1: B_r, B_theta solves
//   P5  all: store slice k; push k -> k+1 and deposit into the sources of slice k+1
// Every tridiagonal system is solved by ONE warp (partition method: each lane eliminates a chunk of
// C rows; the chunk couplings form a 32-unknown system solved by warp-shuffle cyclic reduction).
#include "qz_device.cuh"
#include "qz_internal.h"

namespace qzb {

namespace {

constexpr int kThreads = kSweepThreads;

// ---------------------------------------------------------------- warp-level tridiagonal solve
// Rows come from `rows(ii, i, a, b, c, d)` for row i = lane*C + ii of the lane's chunk (rows i >= M
// are identity rows). q: 3*32*C doubles of scratch, transposed [ii][lane]. x: result, by row.
template <class Rows>
__device__ __forceinline__ void warp_solve(const Rows& rows, const int C, const int M, double* __restrict__ q,
                                           double* __restrict__ x) {
    const int l = threadIdx.x & 31;
    double* qa = q;
    double* qc = q + 32 * C;
    double* qd = q + 64 * C;
    const int s = l * C;
    double a0, b0, c0, d0;
    rows(0, s, a0, b0, c0, d0);
    double a, b, c, d;
    rows(1, s + 1, a, b, c, d);
    double rr = 1.0 / b;
    double pa = a * rr, pc = c * rr, pd = d * rr;
    qa[32 + l] = pa; qc[32 + l] = pc; qd[32 + l] = pd;
    for (int ii = 2; ii < C; ++ii) {
        rows(ii, s + ii, a, b, c, d);
        rr = 1.0 / (b - a * pc);
        pd = rr * (d - a * pd);
        pa = -rr * a * pa;
        pc = rr * c;
        qa[ii * 32 + l] = pa; qc[ii * 32 + l] = pc; qd[ii * 32 + l] = pd;
    }
    const double Ba = pa, Bc = pc, Bd = pd;     // chunk-end row: x_e + Ba x_s + Bc x_{next s} = Bd
    if (C >= 4) {
        double na = qa[(C - 2) * 32 + l], nc = qc[(C - 2) * 32 + l], nd = qd[(C - 2) * 32 + l];
        for (int ii = C - 3; ii >= 1; --ii) {
            const double cn = qc[ii * 32 + l];
            nd = qd[ii * 32 + l] - cn * nd;
            na = qa[ii * 32 + l] - cn * na;
            nc = -cn * nc;
            qa[ii * 32 + l] = na; qc[ii * 32 + l] = nc; qd[ii * 32 + l] = nd;
        }
    }
    double r1a, r1c, r1d;                        // row s+1 in terms of x_s and x_e
    if (C >= 3) { r1a = qa[32 + l]; r1c = qc[32 + l]; r1d = qd[32 + l]; }
    else { r1a = Ba; r1c = Bc; r1d = Bd; }
    // chunk-start row: aA x_{prev e} + bA x_s + cA x_e = dA
    const double aA = (l == 0) ? 0.0 : a0;
    const double bA = b0 - c0 * r1a, cA = -c0 * r1c, dA = d0 - c0 * r1d;
    // eliminate x_s of this lane and of the next lane from the chunk-end row: a system in x_e only
    const unsigned FULL = 0xffffffffu;
    const double aAn = __shfl_down_sync(FULL, aA, 1), bAn = __shfl_down_sync(FULL, bA, 1);
    const double cAn = __shfl_down_sync(FULL, cA, 1), dAn = __shfl_down_sync(FULL, dA, 1);
    const double u = Ba / bA;
    const double v = (l < 31) ? Bc / bAn : 0.0;
    double ea = -u * aA;
    double eb = 1.0 - u * cA - (l < 31 ? v * aAn : 0.0);
    double ec = (l < 31) ? -v * cAn : 0.0;
    double ed = Bd - u * dA - (l < 31 ? v * dAn : 0.0);
#pragma unroll
    for (int st = 1; st < 32; st *= 2) {
        const double al = __shfl_up_sync(FULL, ea, st), bl = __shfl_up_sync(FULL, eb, st);
        const double cl = __shfl_up_sync(FULL, ec, st), dl = __shfl_up_sync(FULL, ed, st);
        const double ah = __shfl_down_sync(FULL, ea, st), bh = __shfl_down_sync(FULL, eb, st);
        const double ch = __shfl_down_sync(FULL, ec, st), dh = __shfl_down_sync(FULL, ed, st);
        const bool lo = l - st >= 0, hi = l + st < 32;
        const double alpha = lo ? -ea / bl : 0.0;
        const double gamma = hi ? -ec / bh : 0.0;
        const double na = lo ? alpha * al : 0.0;
        const double nc = hi ? gamma * ch : 0.0;
        const double nb = eb + (lo ? alpha * cl : 0.0) + (hi ? gamma * ah : 0.0);
        const double nd = ed + (lo ? alpha * dl : 0.0) + (hi ? gamma * dh : 0.0);
        ea = na; eb = nb; ec = nc; ed = nd;
    }
    const double xe = ed / eb;
    const double xep = __shfl_up_sync(FULL, xe, 1);
    const double xs = (dA - (l > 0 ? aA * xep : 0.0) - cA * xe) / bA;
    if (s < M) x[s] = xs;
    if (s + C - 1 < M) x[s + C - 1] = xe;
    for (int ii = 1; ii < C - 1; ++ii) {
        const int i = s + ii;
        if (i < M) x[i] = qd[ii * 32 + l] - qa[ii * 32 + l] * xs - qc[ii * 32 + l] * xe;
    }
}

// ---------------------------------------------------------------- shared-memory layout
struct Src {                                              // plasma + beam sources of one slice
    double *rhot, *drho, *jz, *chi, *ne, *ni, *jpi1, *S1r, *S1i;
};

struct Smem {
    double *r, *iv, *ih;                                  // grid
    double *gm, *g0, *gp, *ir;                            // gradient stencils, 1/r
    double* src0;                                         // sources: 9 arrays, twice when A.dbuf
    double *bgt, *bgr;                                    // neutralising background
    double *psi, *ez, *bz, *wr1, *bpr, *bpi;              // fields of the slice
    const double* opT;                                    // operator rows (shared or global)
    double* q;                                            // solver scratch (shared or global)
    int* lost;
};

__device__ __forceinline__ Smem carve(double* base, const SweepArgs& A) {
    const int M = A.M, C = A.C;
    Smem S;
    double* p = base;
    S.r = p; p += M; S.iv = p; p += M; S.ih = p; p += M;
    S.gm = p; p += M; S.g0 = p; p += M; S.gp = p; p += M; S.ir = p; p += M;
    S.src0 = p;
    p += (A.dbuf ? 18 : 9) * (size_t)M;
    S.bgt = p; p += M; S.bgr = p; p += M;
    S.psi = p; p += M; S.ez = p; p += M; S.bz = p; p += M; S.wr1 = p; p += M; S.bpr = p; p += M; S.bpi = p; p += M;
    if (A.opT_smem) { S.opT = p; p += 9 * 32 * C; } else { S.opT = A.opT; }
    if (A.q_smem) { S.q = p; p += 9 * 32 * C; } else { S.q = A.q_global; }
    S.lost = reinterpret_cast<int*>(p);
    return S;
}

// beam source values of slice k at node j needed by the m = 0 sweep (src/Simulation.cpp:420-441):
// rho - J_z, its xi-derivative (central / one-sided, or backward for ngp), J_z, J_theta
struct BeamRow { double rt, drt, jz, jt; };

__device__ __forceinline__ BeamRow beam_row(const SweepArgs& A, int k, int j) {
    const size_t st = (size_t)A.M * B_NC0;
    const double* bk = A.bsrc + (size_t)k * st + (size_t)j * B_NC0;
    BeamRow r;
    r.rt = bk[B_RT0];
    r.jz = bk[B_JZ0];
    r.jt = bk[B_JP1I];
    const int K = A.K;
    if (A.ngp) {
        const double prev = (k > 0) ? bk[B_RT0 - (ptrdiff_t)st] : 0.0;
        r.drt = (r.rt - prev) * A.idxi;
    } else if (K == 1) {
        r.drt = 0.0;
    } else if (k == 0) {
        r.drt = (bk[st + B_RT0] - r.rt) * A.idxi;
    } else if (k == K - 1) {
        r.drt = (r.rt - bk[B_RT0 - (ptrdiff_t)st]) * A.idxi;
    } else {
        r.drt = 0.5 * (bk[st + B_RT0] - bk[B_RT0 - (ptrdiff_t)st]) * A.idxi;
    }
    return r;
}

// the 9 source arrays of buffer b
__device__ __forceinline__ Src src_of(const Smem& S, int M, int b) {
    double* p = S.src0 + (size_t)b * 9 * M;
    Src s;
    s.rhot = p; s.drho = p + M; s.jz = p + 2 * M; s.chi = p + 3 * M; s.ne = p + 4 * M;
    s.ni = p + 5 * M; s.jpi1 = p + 6 * M; s.S1r = p + 7 * M; s.S1i = p + 8 * M;
    return s;
}

// initial source values of a slice: background + beam; the plasma deposit is added on top
__device__ __forceinline__ void init_sources(const Src& s, const Smem& S, int j, const BeamRow& br) {
    s.rhot[j] = S.bgt[j] + br.rt;
    s.drho[j] = br.drt;
    s.jz[j] = br.jz;
    s.jpi1[j] = br.jt;
    s.chi[j] = 0.0;
    s.ne[j] = 0.0;
    s.ni[j] = S.bgr[j] > 0.0 ? S.bgr[j] : 0.0;
    s.S1r[j] = 0.0;
    s.S1i[j] = 0.0;
}

// 3-point non-uniform gradient at node i (src/FieldSolver.cpp:263-281); odd: axis value f1/r1
__device__ __forceinline__ double grad_at(const Smem& S, int N, const double* f, int i, bool odd) {
    if (i == 0) return odd ? f[1] * S.ir[0] : 0.0;
    if (i == N) return S.g0[N] * f[N] + S.gm[N] * f[N - 1] + S.gp[N] * f[N - 2];
    return S.gm[i] * f[i - 1] + S.g0[i] * f[i] + S.gp[i] * f[i + 1];
}

// ---------------------------------------------------------------- one plasma particle
// history h[m] holds the force m pushes ago (h[0] newest): the reference's ring buffer
// (src/PlasmaSpecies.cpp:621-632) with the slot rotation done by moving values.
template <int ORD>
struct PState {
    double x, y, px, py, dl, w;
    double h[ORD][5];
    double q, qm;
};

template <int ORD>
__device__ __forceinline__ void pload(PState<ORD>& P, const double* __restrict__ ps, int npad, int p) {
    P.x = ps[p]; P.y = ps[npad + p]; P.px = ps[2 * (size_t)npad + p]; P.py = ps[3 * (size_t)npad + p];
    P.dl = ps[4 * (size_t)npad + p]; P.w = ps[5 * (size_t)npad + p];
#pragma unroll
    for (int m = 0; m < ORD; ++m)
#pragma unroll
        for (int v = 0; v < 5; ++v) P.h[m][v] = ps[(6 + (size_t)m * 5 + v) * npad + p];
}

template <int ORD>
__device__ __forceinline__ void pstore(const PState<ORD>& P, double* __restrict__ ps, int npad, int p) {
    ps[p] = P.x; ps[npad + p] = P.y; ps[2 * (size_t)npad + p] = P.px; ps[3 * (size_t)npad + p] = P.py;
    ps[4 * (size_t)npad + p] = P.dl; ps[5 * (size_t)npad + p] = P.w;
#pragma unroll
    for (int m = 0; m < ORD; ++m)
#pragma unroll
        for (int v = 0; v < 5; ++v) ps[(6 + (size_t)m * 5 + v) * npad + p] = P.h[m][v];
}

__device__ __forceinline__ void species_params(const SweepArgs& A, int p, double& q, double& qm) {
    int s = 0;
    while (s + 1 < A.nsp && p >= A.sp_off[s + 1]) ++s;
    q = A.sp_q[s];
    qm = A.sp_qm[s];
}

// src/PlasmaSpecies.cpp:409-478, m = 0 (plasma rho and J_r feed nothing on this path: not deposited)
template <int ORD>
__device__ __forceinline__ void deposit_particle(const PState<ORD>& P, const PGeo& g, const Src& s, const Smem& S) {
    const double PX = P.px, PY = P.py, D = P.dl, w = P.w;
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D;
    const double pz = gam - D;
    const double ux = PX * invd, uy = PY * invd;
    const double ur = g.c * ux + g.s * uy, uth = g.c * uy - g.s * ux;
    const double wq = w * P.q;
    double* dens = (P.q < 0.0) ? s.ne : s.ni;
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        const int jj = g.j + cc;
        const double iv = S.iv[jj];
        const double Wc = cc ? g.W1 : g.W0;
        const double dWc = cc ? g.ih : -g.ih;
        const double a = wq * Wc * iv;
        const double dr = wq * ur * dWc * iv;
        const double vjz = a * pz * invd, vchi = a * P.qm * invd;
        const double vn = w * Wc * iv * gam * invd;
        atomicAdd(&s.rhot[jj], a);
        atomicAdd(&s.drho[jj], dr);
        atomicAdd(&s.jz[jj], vjz);
        atomicAdd(&s.chi[jj], vchi);
        atomicAdd(&dens[jj], vn);
        atomicAdd(&s.jpi1[jj], a * uth);
    }
}

// src/PlasmaSpecies.cpp:508-559, m = 0
template <int ORD>
__device__ __forceinline__ void depositS_particle(const PState<ORD>& P, const PGeo& g, const Src& s, const Smem& S) {
    const double qm = P.qm;
    const double PX = P.px, PY = P.py, D = P.dl;
    const double r1 = lin(S.wr1, g);
    const double Wx = r1 * g.c - 0.0 * g.s, Wy = r1 * g.s + 0.0 * g.c;
    const double Ez = lin(S.ez, g), Bz = lin(S.bz, g);
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D;
    const double ux = PX * invd, uy = PY * invd;
    const double ur = g.c * ux + g.s * uy, uth = g.c * uy - g.s * ux;
    const double dD = qm * ((PX * Wx + PY * Wy) * invd - Ez);
    const double ax = (qm * (gam * Wx + PY * Bz) * invd) * invd - PX * dD * invd * invd;
    const double ay = (qm * (gam * Wy - PX * Bz) * invd) * invd - PY * dD * invd * invd;
    const double wq = P.w * P.q;
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        const int jj = g.j + cc;
        const double iv = S.iv[jj] * wq;
        const double Wc = cc ? g.W1 : g.W0;
        const double dWc = cc ? g.ih : -g.ih;
        const double Worc = cc ? g.Wor1 : g.Wor0;
        double Ar = ax * Wc + ux * ur * dWc;
        double Ai = ay * Wc + uy * ur * dWc;
        const double f2 = uth * Worc;
        Ar += f2 * uy;
        Ai -= f2 * ux;
        atomicAdd(&s.S1r[jj], iv * (Ar * g.c + Ai * g.s));
        atomicAdd(&s.S1i[jj], iv * (Ai * g.c - Ar * g.s));
    }
}

// src/PlasmaSpecies.cpp:561-668 with uniform steps (the classical AB coefficients); returns false
// when the particle is removed (trapped or beyond the wall)
template <int ORD>
__device__ __forceinline__ bool push_particle(PState<ORD>& P, const PGeo& g, const Smem& S, const SweepArgs& A,
                                              bool first) {
    const double qm = P.qm;
    const double X = P.x, Y = P.y, PX = P.px, PY = P.py, D = P.dl;
    const double r1 = lin(S.wr1, g);
    const double Wx = r1 * g.c - 0.0 * g.s, Wy = r1 * g.s + 0.0 * g.c;
    const double Ez = lin(S.ez, g), Bz = lin(S.bz, g);
    const double br = lin(S.bpr, g), bi = lin(S.bpi, g);
    const double Bx = br * g.c - bi * g.s, By = br * g.s + bi * g.c;
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D;
    double fv[5];
    fv[0] = PX * invd;
    fv[1] = PY * invd;
    fv[2] = qm * (gam * Wx * invd + By + PY * Bz * invd);
    fv[3] = qm * (gam * Wy * invd - Bx - PX * Bz * invd);
    fv[4] = qm * ((PX * Wx + PY * Wy) * invd - Ez);
    if (first) {
#pragma unroll
        for (int m = 0; m < ORD; ++m)
#pragma unroll
            for (int v = 0; v < 5; ++v) P.h[m][v] = fv[v];
    } else {
#pragma unroll
        for (int m = ORD - 1; m > 0; --m)
#pragma unroll
            for (int v = 0; v < 5; ++v) P.h[m][v] = P.h[m - 1][v];
#pragma unroll
        for (int v = 0; v < 5; ++v) P.h[0][v] = fv[v];
    }
    double sum[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int m = 0; m < ORD; ++m) {
        const double cm = A.ab[m];
#pragma unroll
        for (int v = 0; v < 5; ++v) sum[v] += cm * P.h[m][v];
    }
    const double dxi = A.dxi;
    double xn = X + dxi * sum[0], yn = Y + dxi * sum[1];
    double pxn = PX + dxi * sum[2], pyn = PY + dxi * sum[3];
    const double dn = D + dxi * sum[4];
    const double gn = (1.0 + pxn * pxn + pyn * pyn + dn * dn) / (2.0 * dn);
    if (!(dn > A.delta_min) || gn > A.max_qsa * dn) {
        P.w = 0.0;
        return false;
    }
    const double R = A.R;
    const double rn = sqrt(xn * xn + yn * yn);
    if (rn > R) {                    // specular reflection at the wall, incl. the history
        const double nx = xn / rn, ny = yn / rn;
        const double rr = 2.0 * R - rn;
        if (rr < 0.0) { P.w = 0.0; return false; }
        xn = nx * rr; yn = ny * rr;
        const double pn = pxn * nx + pyn * ny;
        pxn -= 2.0 * pn * nx; pyn -= 2.0 * pn * ny;
#pragma unroll
        for (int m = 0; m < ORD; ++m) {
            const double a = P.h[m][0] * nx + P.h[m][1] * ny;
            P.h[m][0] -= 2.0 * a * nx; P.h[m][1] -= 2.0 * a * ny;
            const double b = P.h[m][2] * nx + P.h[m][3] * ny;
            P.h[m][2] -= 2.0 * b * nx; P.h[m][3] -= 2.0 * b * ny;
        }
    }
    P.x = xn; P.y = yn; P.px = pxn; P.py = pyn; P.dl = dn;
    return true;
}

}  // namespace

template <int ORD, bool REG>
__global__ void __launch_bounds__(kThreads, 1) sweep_m0_kernel(const SweepArgs A) {
    extern __shared__ double smem_raw[];
    const int M = A.M, N = A.N, K = A.K, C = A.C;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Smem S = carve(smem_raw, A);
    const int np = A.np, npad = A.npad;
    const double R = A.R;
    unsigned long long* tim = A.timing;
    long long t_prev = 0;
    if (tim && tid == 0) t_prev = clock64();
#define PHASE_MARK(ph)                                                        \
    do {                                                                      \
        if (tim && tid == 0) {                                                \
            const long long tn = clock64();                                   \
            tim[ph] += (unsigned long long)(tn - t_prev);                     \
            t_prev = tn;                                                      \
        }                                                                     \
    } while (0)

    // ---------------- prologue: grid, operators, fresh plasma, background (src/Simulation.cpp:653-708)
    for (int j = tid; j < M; j += kThreads) {
        S.r[j] = A.r[j];
        S.iv[j] = A.inv_V[j];
        S.ih[j] = (j < N) ? A.inv_h[j] : 0.0;
        S.gm[j] = A.gm[j]; S.g0[j] = A.g0[j]; S.gp[j] = A.gp[j]; S.ir[j] = A.ir[j];
        S.bgt[j] = 0.0;
        S.bgr[j] = 0.0;
        S.bpr[j] = 0.0;
        S.bpi[j] = 0.0;
        src_of(S, M, 0).ne[j] = 0.0;
    }
    if (A.opT_smem)
        for (int t = tid; t < 9 * 32 * C; t += kThreads) const_cast<double*>(S.opT)[t] = A.opT[t];
    if (tid == 0) *S.lost = 0;
    PState<ORD> P;
    int J = 0;                                             // cell of the thread's particle
    if (REG) {
        if (tid < np) {
            P.x = A.p_init[tid]; P.y = A.p_init[npad + tid]; P.px = A.p_init[2 * npad + tid];
            P.py = A.p_init[3 * npad + tid]; P.dl = A.p_init[4 * npad + tid]; P.w = A.p_init[5 * npad + tid];
#pragma unroll
            for (int m = 0; m < ORD; ++m)
#pragma unroll
                for (int v = 0; v < 5; ++v) P.h[m][v] = 0.0;
            species_params(A, tid, P.q, P.qm);
        } else {
            P.w = 0.0;
        }
    } else {
        for (int p = tid; p < np; p += kThreads) {
#pragma unroll
            for (int v = 0; v < 6; ++v) A.ps[(size_t)v * npad + p] = A.p_init[(size_t)v * npad + p];
            for (int v = 0; v < 5 * ORD; ++v) A.ps[(size_t)(6 + v) * npad + p] = 0.0;
        }
    }
    __syncthreads();
    // immobile species deposit into the background; mobile ones are subtracted (neutralisation,
    // src/Simulation.cpp:672-684); src[0].ne is the scratch of the mobile deposit
    for (int p = tid; p < A.nbg; p += kThreads) {
        const double x = A.bg_p[p], y = A.bg_p[A.nbg + p], wq = A.bg_p[2 * A.nbg + p];
        if (wq == 0.0) continue;
        const PGeo g = geometry(S.r, S.ih, N, R, x, y);
        const double a0 = wq * g.W0 * S.iv[g.j], a1 = wq * g.W1 * S.iv[g.j + 1];
        atomicAdd(&S.bgt[g.j], a0); atomicAdd(&S.bgr[g.j], a0);
        atomicAdd(&S.bgt[g.j + 1], a1); atomicAdd(&S.bgr[g.j + 1], a1);
    }
    if (A.neutralize) {
        for (int p = tid; p < np; p += kThreads) {
            const double w = A.p_init[5 * (size_t)npad + p];
            if (w == 0.0) continue;
            double q, qm;
            species_params(A, p, q, qm);
            const PGeo g = geometry(S.r, S.ih, N, R, A.p_init[p], A.p_init[npad + p]);
            const double a0 = w * q * g.W0 * S.iv[g.j], a1 = w * q * g.W1 * S.iv[g.j + 1];
            atomicAdd(&src_of(S, M, 0).ne[g.j], a0);
            atomicAdd(&src_of(S, M, 0).ne[g.j + 1], a1);
        }
    }
    __syncthreads();
    for (int j = tid; j < M; j += kThreads) {
        if (A.neutralize) { S.bgt[j] -= src_of(S, M, 0).ne[j]; S.bgr[j] -= src_of(S, M, 0).ne[j]; }
        init_sources(src_of(S, M, 0), S, j, beam_row(A, 0, j));
    }
    __syncthreads();
    // deposit of slice 0
    if (REG) {
        if (tid < np && P.w != 0.0) {
            const PGeo G = geometry(S.r, S.ih, N, R, P.x, P.y);
            J = G.j;
            deposit_particle(P, G, src_of(S, M, 0), S);
        }
    } else {
        for (int p = tid; p < np; p += kThreads) {
            PState<ORD> Q;
            pload(Q, A.ps, npad, p);
            if (Q.w == 0.0) continue;
            species_params(A, p, Q.q, Q.qm);
            deposit_particle(Q, geometry(S.r, S.ih, N, R, Q.x, Q.y), src_of(S, M, 0), S);
        }
    }
    __syncthreads();
    PHASE_MARK(0);

    // warps 3.. initialise the sources of the next slice while warps 0-2 solve (A.dbuf)
    constexpr int kInitBase = 96;
    constexpr int kInitThreads = kThreads - kInitBase;

    for (int k = 0; k < K; ++k) {
        const Src s = src_of(S, M, A.dbuf ? (k & 1) : 0);
        const Src sn = src_of(S, M, A.dbuf ? ((k + 1) & 1) : 0);
        // ---------------- P2: psi, E_z, B_z (src/Simulation.cpp:797-807, :477-532)
        if (warp < 3) {
            double* q = S.q + warp * 3 * 32 * C;
            const double* aT = S.opT;                            // L0
            const double* bT = aT + 32 * C;
            const double* cT = bT + 32 * C;
            if (warp == 0) {
                auto rows = [&](int ii, int i, double& a, double& b, double& c, double& d) {
                    const int t = ii * 32 + lane;
                    a = aT[t]; b = bT[t]; c = cT[t];
                    d = (i < N) ? -1.0 * s.rhot[i] : 0.0;    // L0: Dirichlet row N; padding rows identity
                };
                warp_solve(rows, C, M, q, S.psi);
                __syncwarp();
                for (int ii = 0; ii < C; ++ii) {               // W+ mode 1: w1 = -psi' (src/Simulation.cpp:477-498)
                    const int i = lane * C + ii;
                    if (i < M) S.wr1[i] = -grad_at(S, N, S.psi, i, false);
                }
            } else if (warp == 1) {
                auto rows = [&](int ii, int i, double& a, double& b, double& c, double& d) {
                    const int t = ii * 32 + lane;
                    a = aT[t]; b = bT[t]; c = cT[t];
                    d = (i < N) ? -1.0 * s.drho[i] : 0.0;
                };
                warp_solve(rows, C, M, q, S.ez);
            } else {
                auto rows = [&](int ii, int i, double& a, double& b, double& c, double& d) {
                    const int t = ii * 32 + lane;
                    a = aT[t]; b = bT[t]; c = cT[t];
                    if (i < N) {                                // L B_z = -(J_theta' + J_theta/r)
                        const double t1 = grad_at(S, N, s.jpi1, i, true);
                        const double t2 = (i == 0 ? s.jpi1[1] : s.jpi1[i]) * S.ir[i];
                        d = 1.0 * (-(t1 + t2));
                    } else {
                        d = 0.0;
                    }
                };
                warp_solve(rows, C, M, q, S.bz);
            }
        } else if (A.dbuf && k + 1 < K) {
            for (int j = tid - kInitBase; j < M; j += kInitThreads) init_sources(sn, S, j, beam_row(A, k + 1, j));
        }
        __syncthreads();
        PHASE_MARK(1);

        // ---------------- P3: S+ (src/PlasmaSpecies.cpp:508-559)
        if (REG) {
            if (tid < np && P.w != 0.0) depositS_particle(P, geometry_in(S.r, S.ih, P.x, P.y, J), s, S);
        } else {
            for (int p = tid; p < np; p += kThreads) {
                PState<ORD> Q;
                pload(Q, A.ps, npad, p);
                if (Q.w == 0.0) continue;
                species_params(A, p, Q.q, Q.qm);
                depositS_particle(Q, geometry(S.r, S.ih, N, R, Q.x, Q.y), s, S);
            }
        }
        __syncthreads();
        PHASE_MARK(2);

        // ---------------- P4: B+ (src/Simulation.cpp:535-591, m = 0: one pass); sources of k+1
        if (warp == 0) {
            const double* aT = S.opT + 1 * 3 * 32 * C;              // (L1D - chi) B_r0 = -S_i
            const double* bT = aT + 32 * C;
            const double* cT = bT + 32 * C;
            auto rows = [&](int ii, int i, double& a, double& b, double& c, double& d) {
                const int t = ii * 32 + lane;
                a = aT[t]; b = bT[t]; c = cT[t];
                if (i >= 1 && i < N) {
                    b = b - s.chi[i];
                    d = 1.0 * (-s.S1i[i]);
                } else {
                    d = 0.0;
                }
            };
            warp_solve(rows, C, M, S.q, S.bpr);
        } else if (warp == 1) {
            const double* aT = S.opT + 2 * 3 * 32 * C;              // (L1F - chi) B_theta0 = J_z' + S_r
            const double* bT = aT + 32 * C;
            const double* cT = bT + 32 * C;
            const double fc = A.flux_coef;
            auto rows = [&](int ii, int i, double& a, double& b, double& c, double& d) {
                const int t = ii * 32 + lane;
                a = aT[t]; b = bT[t]; c = cT[t];
                if (i >= 1 && i <= N) {
                    b = b - s.chi[i];
                    d = 1.0 * (grad_at(S, N, s.jz, i, false) + s.S1r[i]);
                    if (i == N) d -= fc * s.jz[N];             // flux wall g = J_z(R)
                } else {
                    d = 0.0;
                }
            };
            warp_solve(rows, C, M, S.q + 3 * 32 * C, S.bpi);
        }
        __syncthreads();
        PHASE_MARK(3);

        // ---------------- P5: store slice k; push k -> k+1 and deposit into slice k+1
        {
            const size_t fb = (size_t)k * M;
            for (int j = tid; j < M; j += kThreads) {
                double* F = A.fld + (fb + j) * F_NC0;
                F[F_EP1R] = S.wr1[j] + S.bpi[j];
                F[F_EP1I] = 0.0 - S.bpr[j];
                F[F_BP1R] = S.bpr[j];
                F[F_BP1I] = S.bpi[j];
                F[F_EZ0] = S.ez[j];
                F[F_BZ0] = S.bz[j];
                double* D = A.diag + (fb + j) * D_NC0;
                D[D_PSI0] = S.psi[j];
                D[D_NE0] = s.ne[j];
                D[D_NI0] = s.ni[j];
            }
        }
        if (k + 1 < K) {
            if (!A.dbuf) {
                __syncthreads();                                    // store read the sources
                for (int j = tid; j < M; j += kThreads) init_sources(sn, S, j, beam_row(A, k + 1, j));
                __syncthreads();
            }
            const bool first = (k == 0);
            if (REG) {
                if (tid < np && P.w != 0.0) {
                    if (push_particle(P, geometry_in(S.r, S.ih, P.x, P.y, J), S, A, first)) {
                        const PGeo G = geometry(S.r, S.ih, N, R, P.x, P.y);
                        J = G.j;
                        deposit_particle(P, G, sn, S);
                    } else {
                        atomicAdd(S.lost, 1);
                    }
                }
            } else {
                for (int p = tid; p < np; p += kThreads) {
                    PState<ORD> Q;
                    pload(Q, A.ps, npad, p);
                    if (Q.w == 0.0) continue;
                    species_params(A, p, Q.q, Q.qm);
                    const PGeo g = geometry(S.r, S.ih, N, R, Q.x, Q.y);
                    if (push_particle(Q, g, S, A, first)) {
                        deposit_particle(Q, geometry(S.r, S.ih, N, R, Q.x, Q.y), sn, S);
                    } else {
                        atomicAdd(S.lost, 1);
                    }
                    pstore(Q, A.ps, npad, p);
                }
            }
        }
        __syncthreads();
        PHASE_MARK(4);
    }
    if (REG && tid < np) pstore(P, A.ps, npad, tid);
    if (tid == 0 && A.counters) atomicAdd(&A.counters[0], (unsigned long long)*S.lost);
#undef PHASE_MARK
}

size_t sweep_m0_smem_bytes(int M, int C, bool dbuf, bool opT_smem, bool q_smem) {
    size_t d = (size_t)(dbuf ? 33 : 24) * M;
    if (opT_smem) d += 9 * 32 * (size_t)C;
    if (q_smem) d += 9 * 32 * (size_t)C;
    return sizeof(double) * d + 16;
}

namespace {
template <int ORD, bool REG>
cudaError_t launch_t(const SweepArgs& A, size_t smem, cudaStream_t stream) {
    cudaError_t e = cudaFuncSetAttribute(sweep_m0_kernel<ORD, REG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    sweep_m0_kernel<ORD, REG><<<1, kThreads, smem, stream>>>(A);
    return cudaGetLastError();
}

template <int ORD>
cudaError_t launch_o(const SweepArgs& A, size_t smem, cudaStream_t stream) {
    return A.np <= kThreads ? launch_t<ORD, true>(A, smem, stream) : launch_t<ORD, false>(A, smem, stream);
}
}  // namespace

cudaError_t launch_sweep_m0(const SweepArgs& A, cudaStream_t stream) {
    const size_t smem = sweep_m0_smem_bytes(A.M, A.C, A.dbuf, A.opT_smem, A.q_smem);
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
