// qz_sweep_m1_body.cuh -- the quasi-static xi sweep of one time step with azimuthal modes m = 0, 1
// (Simulation::step_fields, src/Simulation.cpp:636-795, with modes = 1) by ONE CTA (sm_100a, FP64).
//
// Per slice (src/Simulation.cpp:728-783):
//   sources   plasma deposit of rho - J_z, its xi-derivative, J_z, chi, density, J+ in modes 0 / 1
//             (src/PlasmaSpecies.cpp:409-478) + beam sources + neutralising background
//   P2        psi and E_z (L0 for mode 0, L1D for mode 1; src/Simulation.cpp:797-819) and B_z
//             (src/Simulation.cpp:501-532): 9 systems with fixed Thomas factors, one forward and one
//             backward grouped scan; W+ from psi (src/Simulation.cpp:477-498)
//   P3        S+ in modes 0, 1, 2 (src/PlasmaSpecies.cpp:508-559)
//   P4        B+ (src/Simulation.cpp:535-591): one pivot scan for the four chi_0-dependent operators
//             L1D, L1F (flux wall), L0, L2D, then `picard` iterations, each a grouped forward and
//             backward scan over the 6 right-hand sides coupled through chi_1
//   P5        store the slice (18 field and 9 diagnostic components), push the plasma by AB and
//             deposit it into the next slice (src/PlasmaSpecies.cpp:561-668)
//
// Shared memory holds the grid and the fields of the slice that particles gather (24 arrays of M
// doubles: 98 KB at M = 512), which leaves L1 room for the register spills of this large body. The
// sources (30 arrays) live in a per-CTA global scratch that stays in L2: particles deposit into them
// with native FP64 reductions (warp-aggregated first), where shared-memory FP64 adds would be
// compare-and-swap loops; they are read back through L2 (ld.global.cg), never through L1. The
// operator constants come through the read-only path; the plasma state (ntheta particles per ring,
// with its AB history) lives in another per-CTA global scratch.
#pragma once
#include "qz_sweep_body.cuh"

namespace qzb {

namespace m1_detail {

using namespace sweep_detail;

struct Msc { double *a0, *ar, *ai; };                  // scalar in modes: f0 + 2 Re(f1 e^{i theta})
struct Mvec { double *r0, *i0, *r1, *i1, *r2, *i2; };  // vector V+ = sum_k v_k e^{i k theta}, k = 0, 1, 2

struct Src1 {                                          // the sources of one slice (global scratch)
    Msc rhot, drho, jz, chi, ne, ni;
    Mvec jp, S;
};

struct Smem1 {
    double *r, *iv, *ih;
    Msc psi, ez, bz;
    Mvec wp, bp;
    double* tot;                                       // scan scratch: 2 x 16 x kW
    int* lost;
    int* flag;
};

__device__ __forceinline__ Msc take3(double*& p, int M) {
    Msc m;
    m.a0 = p; m.ar = p + M; m.ai = p + 2 * M;
    p += 3 * (size_t)M;
    return m;
}
__device__ __forceinline__ Mvec take6(double*& p, int M) {
    Mvec v;
    v.r0 = p; v.i0 = p + M; v.r1 = p + 2 * M; v.i1 = p + 3 * M; v.r2 = p + 4 * M; v.i2 = p + 5 * M;
    p += 6 * (size_t)M;
    return v;
}

// sources of buffer b of the global scratch (2 x 30 x M doubles: double-buffered, so that the push
// of slice k deposits straight into slice k+1)
__device__ __forceinline__ Src1 src1_of(double* scratch, int M, int b) {
    Src1 S;
    double* g = scratch + (size_t)b * 30 * M;
    S.rhot = take3(g, M); S.drho = take3(g, M); S.jz = take3(g, M); S.chi = take3(g, M);
    S.ne = take3(g, M); S.ni = take3(g, M);
    S.jp = take6(g, M); S.S = take6(g, M);
    return S;
}

// shared memory: grid, fields, scan scratch
__device__ __forceinline__ Smem1 carve1(double* base, int M) {
    Smem1 S;
    double* p = base;
    S.r = p; p += M; S.iv = p; p += M; S.ih = p; p += M;
    S.psi = take3(p, M); S.ez = take3(p, M); S.bz = take3(p, M);
    S.wp = take6(p, M); S.bp = take6(p, M);
    S.tot = p; p += 2 * 16 * kW;
    S.lost = reinterpret_cast<int*>(p);
    S.flag = S.lost + 1;
    return S;
}

// operator constants (global, read-only): stencils, 1/r, L0 Thomas factors, L1D and L1F rows (consts,
// 13 x M), L1D Thomas factors, L0 rows, L2D rows (consts1, 9 x M)
struct Consts1 {
    const double *gm, *g0, *gp, *ir;
    const double *l0r, *l0f, *l0b;
    const double *l1a, *l1b, *l1c, *lfa, *lfb, *lfc;
    const double *d1r, *d1f, *d1b;
    const double *o0a, *o0b, *o0c, *o2a, *o2b, *o2c;
};

__device__ __forceinline__ Consts1 consts1(const SweepArgs& A) {
    const int M = A.M;
    const double* q = A.consts;
    const double* u = A.consts1;
    Consts1 C;
    C.gm = q; C.g0 = q + M; C.gp = q + 2 * M; C.ir = q + 3 * M;
    C.l0r = q + 4 * M; C.l0f = q + 5 * M; C.l0b = q + 6 * M;
    C.l1a = q + 7 * M; C.l1b = q + 8 * M; C.l1c = q + 9 * M;
    C.lfa = q + 10 * M; C.lfb = q + 11 * M; C.lfc = q + 12 * M;
    C.d1r = u; C.d1f = u + M; C.d1b = u + 2 * M;
    C.o0a = u + 3 * M; C.o0b = u + 4 * M; C.o0c = u + 5 * M;
    C.o2a = u + 6 * M; C.o2b = u + 7 * M; C.o2c = u + 8 * M;
    return C;
}

__device__ __forceinline__ double ldc(const double* p) { return __ldg(p); }

// 3-point non-uniform gradients (src/FieldSolver.cpp:193-219)
__device__ __forceinline__ double grad1(const Consts1& C, int N, const double* f, int i, bool odd) {
    if (i == 0) return odd ? f[1] * ldc(C.ir) : 0.0;
    if (i == N) return ldc(C.g0 + N) * f[N] + ldc(C.gm + N) * f[N - 1] + ldc(C.gp + N) * f[N - 2];
    return ldc(C.gm + i) * f[i - 1] + ldc(C.g0 + i) * f[i] + ldc(C.gp + i) * f[i + 1];
}
__device__ __forceinline__ double over_r1(const Consts1& C, const double* f, int i) {
    return (i == 0 ? f[1] : f[i]) * ldc(C.ir + i);
}
// the same on a source array in the global scratch, read through L2 (deposited by reductions)
__device__ __forceinline__ double lg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ double grad1g(const Consts1& C, int N, const double* f, int i, bool odd) {
    if (i == 0) return odd ? lg(f + 1) * ldc(C.ir) : 0.0;
    if (i == N) return ldc(C.g0 + N) * lg(f + N) + ldc(C.gm + N) * lg(f + N - 1) + ldc(C.gp + N) * lg(f + N - 2);
    return ldc(C.gm + i) * lg(f + i - 1) + ldc(C.g0 + i) * lg(f + i) + ldc(C.gp + i) * lg(f + i + 1);
}
__device__ __forceinline__ double over_r1g(const Consts1& C, const double* f, int i) {
    return (i == 0 ? lg(f + 1) : lg(f + i)) * ldc(C.ir + i);
}

// ---------------------------------------------------------------- grouped scans
// Forward exclusive scan of NB affine maps y -> a[g[b]] y + b[b] sharing NA slopes (g maps each
// right-hand side to its system), thread order = row order, y_{-1} = 0.
template <int NA, int NB>
__device__ __forceinline__ void scan_fwd_g(const double (&a)[NA], const double (&b)[NB], const int (&g)[NB],
                                           double (&yb)[NB], double* tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double A[NA], B[NB];
#pragma unroll
    for (int s = 0; s < NA; ++s) A[s] = a[s];
#pragma unroll
    for (int r = 0; r < NB; ++r) B[r] = b[r];
#pragma unroll
    for (int st = 1; st < 32; st <<= 1) {
        double Ap[NA], Bp[NB];
#pragma unroll
        for (int s = 0; s < NA; ++s) Ap[s] = __shfl_up_sync(FULL, A[s], st);
#pragma unroll
        for (int r = 0; r < NB; ++r) Bp[r] = __shfl_up_sync(FULL, B[r], st);
        if (lane >= st) {
#pragma unroll
            for (int r = 0; r < NB; ++r) B[r] = fma(A[g[r]], Bp[r], B[r]);
#pragma unroll
            for (int s = 0; s < NA; ++s) A[s] *= Ap[s];
        }
    }
    if (lane == 31) {
#pragma unroll
        for (int s = 0; s < NA; ++s) tot[kW * s + warp] = A[s];
#pragma unroll
        for (int r = 0; r < NB; ++r) tot[kW * (NA + r) + warp] = B[r];
    }
    double eA[NA], eB[NB];
#pragma unroll
    for (int s = 0; s < NA; ++s) { eA[s] = __shfl_up_sync(FULL, A[s], 1); if (lane == 0) eA[s] = 1.0; }
#pragma unroll
    for (int r = 0; r < NB; ++r) { eB[r] = __shfl_up_sync(FULL, B[r], 1); if (lane == 0) eB[r] = 0.0; }
    __syncthreads();
    double ta[NA], tb[NB];
#pragma unroll
    for (int s = 0; s < NA; ++s) ta[s] = lane < kW ? tot[kW * s + lane] : 1.0;
#pragma unroll
    for (int r = 0; r < NB; ++r) tb[r] = lane < kW ? tot[kW * (NA + r) + lane] : 0.0;
#pragma unroll
    for (int st = 1; st < kW; st <<= 1) {
        double ap[NA], bp[NB];
#pragma unroll
        for (int s = 0; s < NA; ++s) ap[s] = __shfl_up_sync(FULL, ta[s], st);
#pragma unroll
        for (int r = 0; r < NB; ++r) bp[r] = __shfl_up_sync(FULL, tb[r], st);
        if (lane >= st) {
#pragma unroll
            for (int r = 0; r < NB; ++r) tb[r] = fma(ta[g[r]], bp[r], tb[r]);
#pragma unroll
            for (int s = 0; s < NA; ++s) ta[s] *= ap[s];
        }
    }
#pragma unroll
    for (int r = 0; r < NB; ++r) {
        const double cw = __shfl_sync(FULL, tb[r], (warp + 31) & 31);
        yb[r] = fma(eA[g[r]], warp > 0 ? cw : 0.0, eB[r]);
    }
}

// Backward exclusive scan of x -> a[g[b]] x + b[b], x_{end} = 0.
template <int NA, int NB>
__device__ __forceinline__ void scan_bwd_g(const double (&a)[NA], const double (&b)[NB], const int (&g)[NB],
                                           double (&xa)[NB], double* tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double A[NA], B[NB];
#pragma unroll
    for (int s = 0; s < NA; ++s) A[s] = a[s];
#pragma unroll
    for (int r = 0; r < NB; ++r) B[r] = b[r];
#pragma unroll
    for (int st = 1; st < 32; st <<= 1) {
        double An[NA], Bn[NB];
#pragma unroll
        for (int s = 0; s < NA; ++s) An[s] = __shfl_down_sync(FULL, A[s], st);
#pragma unroll
        for (int r = 0; r < NB; ++r) Bn[r] = __shfl_down_sync(FULL, B[r], st);
        if (lane + st < 32) {
#pragma unroll
            for (int r = 0; r < NB; ++r) B[r] = fma(A[g[r]], Bn[r], B[r]);
#pragma unroll
            for (int s = 0; s < NA; ++s) A[s] *= An[s];
        }
    }
    if (lane == 0) {
#pragma unroll
        for (int s = 0; s < NA; ++s) tot[kW * s + warp] = A[s];
#pragma unroll
        for (int r = 0; r < NB; ++r) tot[kW * (NA + r) + warp] = B[r];
    }
    double eA[NA], eB[NB];
#pragma unroll
    for (int s = 0; s < NA; ++s) { eA[s] = __shfl_down_sync(FULL, A[s], 1); if (lane == 31) eA[s] = 1.0; }
#pragma unroll
    for (int r = 0; r < NB; ++r) { eB[r] = __shfl_down_sync(FULL, B[r], 1); if (lane == 31) eB[r] = 0.0; }
    __syncthreads();
    double ta[NA], tb[NB];
#pragma unroll
    for (int s = 0; s < NA; ++s) ta[s] = lane < kW ? tot[kW * s + lane] : 1.0;
#pragma unroll
    for (int r = 0; r < NB; ++r) tb[r] = lane < kW ? tot[kW * (NA + r) + lane] : 0.0;
#pragma unroll
    for (int st = 1; st < kW; st <<= 1) {
        double an[NA], bn[NB];
#pragma unroll
        for (int s = 0; s < NA; ++s) an[s] = __shfl_down_sync(FULL, ta[s], st);
#pragma unroll
        for (int r = 0; r < NB; ++r) bn[r] = __shfl_down_sync(FULL, tb[r], st);
        if (lane + st < kW) {
#pragma unroll
            for (int r = 0; r < NB; ++r) tb[r] = fma(ta[g[r]], bn[r], tb[r]);
#pragma unroll
            for (int s = 0; s < NA; ++s) ta[s] *= an[s];
        }
    }
#pragma unroll
    for (int r = 0; r < NB; ++r) {
        const double cw = __shfl_sync(FULL, tb[r], (warp + 1) & 31);
        xa[r] = fma(eA[g[r]], warp < kW - 1 ? cw : 0.0, eB[r]);
    }
}

// ---------------------------------------------------------------- sources of a slice
// beam sources of slice k at node j (src/Simulation.cpp:408-457): rho - J_z in modes 0 / 1 and its
// xi-derivative, J_z, J+ (rho itself feeds nothing on this path)
struct BeamRow1 { double rt[3], drt[3], jz[3], jp[6]; };

template <bool kL2, bool kStat = false>
__device__ __forceinline__ BeamRow1 beam_row1(const SweepArgs& A, const double* bsrc, int k, int j) {
    const size_t st = (size_t)A.M * B_NC1;
    const double* bk = bsrc + (size_t)k * st + (size_t)j * B_NC1;
    BeamRow1 r;
    const int rc[3] = {B_RT0, B_RT1R, B_RT1I};
    const int K = A.K;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const int c = rc[e];
        r.rt[e] = ldbs<kL2, kStat>(A, bsrc, bk + c);
        if (A.ngp) {
            const double prev = (k > 0) ? ldbs<kL2, kStat>(A, bsrc, bk + c - (ptrdiff_t)st) : 0.0;
            r.drt[e] = (r.rt[e] - prev) * A.idxi;
        } else if (K == 1) {
            r.drt[e] = 0.0;
        } else if (k == 0) {
            r.drt[e] = (ldbs<kL2, kStat>(A, bsrc, bk + st + c) - r.rt[e]) * A.idxi;
        } else if (k == K - 1) {
            r.drt[e] = (r.rt[e] - ldbs<kL2, kStat>(A, bsrc, bk + c - (ptrdiff_t)st)) * A.idxi;
        } else {
            r.drt[e] = 0.5 * (ldbs<kL2, kStat>(A, bsrc, bk + st + c) - ldbs<kL2, kStat>(A, bsrc, bk + c - (ptrdiff_t)st)) * A.idxi;
        }
    }
    r.jz[0] = ldbs<kL2, kStat>(A, bsrc, bk + B_JZ0); r.jz[1] = ldbs<kL2, kStat>(A, bsrc, bk + B_JZ1R);
    r.jz[2] = ldbs<kL2, kStat>(A, bsrc, bk + B_JZ1I);
    r.jp[0] = ldbs<kL2, kStat>(A, bsrc, bk + B_JP0R); r.jp[1] = ldbs<kL2, kStat>(A, bsrc, bk + B_JP0I);
    r.jp[2] = ldbs<kL2, kStat>(A, bsrc, bk + B_JP1R); r.jp[3] = ldbs<kL2, kStat>(A, bsrc, bk + B_JP1I);
    r.jp[4] = ldbs<kL2, kStat>(A, bsrc, bk + B_JP2R); r.jp[5] = ldbs<kL2, kStat>(A, bsrc, bk + B_JP2I);
    return r;
}

// initial sources of slice k at node j: background + beam; the plasma deposit is added on top.
// bg: (3, M) background rho - J_z = rho of the immobile species minus the neutralised mobile ones
__device__ __forceinline__ void init_sources1(const Src1& T, const double* bg, int M, int j, const BeamRow1& b) {
    const double g0 = __ldcg(bg + j), gr = __ldcg(bg + M + j), gi = __ldcg(bg + 2 * M + j);
    T.rhot.a0[j] = g0 + b.rt[0]; T.rhot.ar[j] = gr + b.rt[1]; T.rhot.ai[j] = gi + b.rt[2];
    T.drho.a0[j] = b.drt[0]; T.drho.ar[j] = b.drt[1]; T.drho.ai[j] = b.drt[2];
    T.jz.a0[j] = b.jz[0]; T.jz.ar[j] = b.jz[1]; T.jz.ai[j] = b.jz[2];
    T.jp.r0[j] = b.jp[0]; T.jp.i0[j] = b.jp[1]; T.jp.r1[j] = b.jp[2];
    T.jp.i1[j] = b.jp[3]; T.jp.r2[j] = b.jp[4]; T.jp.i2[j] = b.jp[5];
    T.chi.a0[j] = 0.0; T.chi.ar[j] = 0.0; T.chi.ai[j] = 0.0;
    T.ne.a0[j] = 0.0; T.ne.ar[j] = 0.0; T.ne.ai[j] = 0.0;
    T.ni.a0[j] = g0 > 0.0 ? g0 : 0.0; T.ni.ar[j] = 0.0; T.ni.ai[j] = 0.0;
    T.S.r0[j] = 0.0; T.S.i0[j] = 0.0; T.S.r1[j] = 0.0; T.S.i1[j] = 0.0; T.S.r2[j] = 0.0; T.S.i2[j] = 0.0;
}

// with the filter: the plasma deposit of a slice starts from zero (beam and background come after the filter)
__device__ __forceinline__ void init_sources1_zero(const Src1& T, int M, int j) {
    const Msc sc[6] = {T.rhot, T.drho, T.jz, T.chi, T.ne, T.ni};
#pragma unroll
    for (int c = 0; c < 6; ++c) { sc[c].a0[j] = 0.0; sc[c].ar[j] = 0.0; sc[c].ai[j] = 0.0; }
    T.jp.r0[j] = 0.0; T.jp.i0[j] = 0.0; T.jp.r1[j] = 0.0; T.jp.i1[j] = 0.0; T.jp.r2[j] = 0.0; T.jp.i2[j] = 0.0;
    T.S.r0[j] = 0.0; T.S.i0[j] = 0.0; T.S.r1[j] = 0.0; T.S.i1[j] = 0.0; T.S.r2[j] = 0.0; T.S.i2[j] = 0.0;
}

// ---------------------------------------------------------------- smoothing filter (modes = 1)
// FieldSolver::filter (src/FieldSolver.cpp:148-161) of NB source arrays of the global scratch, each with
// F0, F1 or F2 (op), on one row per thread in place: Thomas with the host-factored pivots fc (3 x M per
// operator), its substitutions as grouped block scans (tot, tot2: the two scratch halves). Every thread reads
// and writes only its own row. Only the kernel variants for filtered decks (EXT) contain it.
template <int NB>
__device__ __forceinline__ void filter_rows1(const FilterSet<NB> fs, const double* __restrict__ fc, int M, double* tot,
                                          double* tot2) {
    const int i = threadIdx.x;
    const bool row = i < M;
    double a[3], d[NB], y[NB];
#pragma unroll
    for (int s = 0; s < 3; ++s) a[s] = row ? __ldg(fc + (size_t)s * 3 * M + M + i) : 1.0;
#pragma unroll
    for (int e = 0; e < NB; ++e) d[e] = row ? __ldg(fc + (size_t)fs.op[e] * 3 * M + i) * __ldcg(fs.f[e] + i) : 0.0;
    scan_fwd_g<3, NB>(a, d, fs.op, y, tot);
#pragma unroll
    for (int e = 0; e < NB; ++e) y[e] = fma(a[fs.op[e]], y[e], d[e]);
#pragma unroll
    for (int s = 0; s < 3; ++s) a[s] = row ? __ldg(fc + (size_t)s * 3 * M + 2 * M + i) : 1.0;
    double x[NB];
    scan_bwd_g<3, NB>(a, y, fs.op, x, tot2);
    if (row)
#pragma unroll
        for (int e = 0; e < NB; ++e) fs.f[e][i] = fma(a[fs.op[e]], x[e], y[e]);
}

// Simulation::filter_plasma_sources (src/Simulation.cpp:823-835, modes = 1) on the plasma deposit of the
// slice in buffer T, then combine_sources (src/Simulation.cpp:430-452): the background and the beam row
// of slice k added, as the reference adds them after the filter. Ends with a barrier.
template <bool kL2>
__device__ __forceinline__ void filter_sources1(const SweepArgs& A, const Src1& T, const double* bg,
                                                const double* bsrc, int k, double* tot, int& scan_par) {
    const int M = A.M, i = threadIdx.x;
    const Msc sc[6] = {T.rhot, T.drho, T.jz, T.chi, T.ne, T.ni};
    FilterSet<12> fa, fb;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        fa.f[3 * c] = sc[c].a0; fa.f[3 * c + 1] = sc[c].ar; fa.f[3 * c + 2] = sc[c].ai;
        fa.op[3 * c] = 0; fa.op[3 * c + 1] = 1; fa.op[3 * c + 2] = 1;
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        fb.f[3 * c] = sc[4 + c].a0; fb.f[3 * c + 1] = sc[4 + c].ar; fb.f[3 * c + 2] = sc[4 + c].ai;
        fb.op[3 * c] = 0; fb.op[3 * c + 1] = 1; fb.op[3 * c + 2] = 1;
    }
    fb.f[6] = T.jp.r0; fb.f[7] = T.jp.i0; fb.f[8] = T.jp.r1; fb.f[9] = T.jp.i1; fb.f[10] = T.jp.r2; fb.f[11] = T.jp.i2;
    fb.op[6] = fb.op[7] = 0; fb.op[8] = fb.op[9] = 1; fb.op[10] = fb.op[11] = 2;
    double* t0 = tot + (scan_par++ & 1) * 16 * kW;
    double* t1 = tot + (scan_par++ & 1) * 16 * kW;
    filter_rows1<12>(fa, A.fconsts, M, t0, t1);
    filter_rows1<12>(fb, A.fconsts, M, t0, t1);
    if (i < M) {
        const BeamRow1 b = beam_row1<kL2, true>(A, bsrc, k, i);
        const double g0 = __ldcg(bg + i), gr = __ldcg(bg + M + i), gi = __ldcg(bg + 2 * M + i);
        T.rhot.a0[i] = lg(T.rhot.a0 + i) + (g0 + b.rt[0]);
        T.rhot.ar[i] = lg(T.rhot.ar + i) + (gr + b.rt[1]);
        T.rhot.ai[i] = lg(T.rhot.ai + i) + (gi + b.rt[2]);
        T.drho.a0[i] = lg(T.drho.a0 + i) + b.drt[0];
        T.drho.ar[i] = lg(T.drho.ar + i) + b.drt[1];
        T.drho.ai[i] = lg(T.drho.ai + i) + b.drt[2];
        T.jz.a0[i] = lg(T.jz.a0 + i) + b.jz[0];
        T.jz.ar[i] = lg(T.jz.ar + i) + b.jz[1];
        T.jz.ai[i] = lg(T.jz.ai + i) + b.jz[2];
        double* jp[6] = {T.jp.r0, T.jp.i0, T.jp.r1, T.jp.i1, T.jp.r2, T.jp.i2};
#pragma unroll
        for (int c = 0; c < 6; ++c) jp[c][i] = lg(jp[c] + i) + b.jp[c];
        if (g0 > 0.0) T.ni.a0[i] = lg(T.ni.a0 + i) + g0;
    }
    __syncthreads();
}

// ---------------------------------------------------------------- particles
// the field of the slice at a particle (src/PlasmaSpecies.cpp:75-89, src/SliceData.hpp:70-83)
struct PF1 { double Wx, Wy, Bx, By, Bz, Ez; };

__device__ __forceinline__ void eval_vec(const Mvec& v, const PGeo& g, double& vx, double& vy) {
    const double r0 = lin(v.r0, g), i0 = lin(v.i0, g), r1 = lin(v.r1, g), i1 = lin(v.i1, g);
    const double r2 = lin(v.r2, g), i2 = lin(v.i2, g);
    const double c = g.c, s = g.s;
    vx = r1 * c - i1 * s;
    vy = r1 * s + i1 * c;
    const double c2 = c * c - s * s, s2 = 2.0 * c * s;
    vx += r0 + r2 * c2 - i2 * s2;
    vy += i0 + r2 * s2 + i2 * c2;
}
__device__ __forceinline__ double eval_sc(const Msc& f, const PGeo& g) {
    return lin(f.a0, g) + 2.0 * (lin(f.ar, g) * g.c - lin(f.ai, g) * g.s);
}

__device__ __forceinline__ PF1 gather1(const Smem1& S, const PGeo& g, bool needB) {
    PF1 F;
    eval_vec(S.wp, g, F.Wx, F.Wy);
    F.Ez = eval_sc(S.ez, g);
    F.Bz = eval_sc(S.bz, g);
    F.Bx = F.By = 0.0;
    if (needB) eval_vec(S.bp, g, F.Bx, F.By);
    return F;
}

// The plasma deposit of one particle (src/PlasmaSpecies.cpp:409-478, m = 1), 21 values per node in
// three chunks of 7 so that each warp-aggregated add holds 14 values:
//   chunk 0: rhot a0 ar ai, drho a0 ar ai, jz a0
//   chunk 1: jz ar ai, chi a0 ar ai, dens a0 ar
//   chunk 2: dens ai, jp r1 i1 r0 i0 r2 i2
struct Dep1 {
    double a[2], dr[2], th[2], vjz[2], vchi[2], vn[2];
    double c, s, ux, uy, ur, uth, c2, s2;
};

template <int ORD>
__device__ __forceinline__ Dep1 dep1_basics(const PState<ORD>& P, const PGeo& g, const Smem1& S) {
    Dep1 d;
    const double PX = P.px, PY = P.py, D = P.dl, w = P.w;
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D;
    const double pz = gam - D;
    d.ux = PX * invd; d.uy = PY * invd;
    d.c = g.c; d.s = g.s;
    d.ur = g.c * d.ux + g.s * d.uy;
    d.uth = g.c * d.uy - g.s * d.ux;
    d.c2 = g.c * g.c - g.s * g.s;
    d.s2 = 2.0 * g.c * g.s;
    const double wq = w * P.q;
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        const double iv = S.iv[g.j + cc];
        const double Wc = cc ? g.W1 : g.W0;
        const double dWc = cc ? g.ih : -g.ih;
        const double Worc = cc ? g.Wor1 : g.Wor0;
        d.a[cc] = wq * Wc * iv;
        d.dr[cc] = wq * d.ur * dWc * iv;
        d.th[cc] = wq * d.uth * Worc * iv;
        d.vjz[cc] = d.a[cc] * pz * invd;
        d.vchi[cc] = d.a[cc] * P.qm * invd;
        d.vn[cc] = w * Wc * iv * gam * invd;
    }
    return d;
}

template <int CH>
__device__ __forceinline__ void dep1_chunk(const Dep1& d, double (&v)[14]) {
    const double c = d.c, s = d.s;
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        double* o = v + 7 * cc;
        const double a = d.a[cc], dr = d.dr[cc], th = d.th[cc];
        if (CH == 0) {
            o[0] = a; o[1] = a * c; o[2] = -a * s;
            o[3] = dr; o[4] = dr * c - th * s; o[5] = -dr * s - th * c;
            o[6] = d.vjz[cc];
        } else if (CH == 1) {
            o[0] = d.vjz[cc] * c; o[1] = -d.vjz[cc] * s;
            o[2] = d.vchi[cc]; o[3] = d.vchi[cc] * c; o[4] = -d.vchi[cc] * s;
            o[5] = d.vn[cc]; o[6] = d.vn[cc] * c;
        } else {
            o[0] = -d.vn[cc] * s;
            o[1] = a * d.ur; o[2] = a * d.uth; o[3] = a * d.ux; o[4] = a * d.uy;
            o[5] = a * (d.ux * d.c2 + d.uy * d.s2); o[6] = a * (d.uy * d.c2 - d.ux * d.s2);
        }
    }
}

template <int CH>
__device__ __forceinline__ void dep1_addr(const Src1& T, int jj, bool neg, double** o) {
    const Msc& dens = neg ? T.ne : T.ni;
    if (CH == 0) {
        o[0] = T.rhot.a0 + jj; o[1] = T.rhot.ar + jj; o[2] = T.rhot.ai + jj;
        o[3] = T.drho.a0 + jj; o[4] = T.drho.ar + jj; o[5] = T.drho.ai + jj;
        o[6] = T.jz.a0 + jj;
    } else if (CH == 1) {
        o[0] = T.jz.ar + jj; o[1] = T.jz.ai + jj;
        o[2] = T.chi.a0 + jj; o[3] = T.chi.ar + jj; o[4] = T.chi.ai + jj;
        o[5] = dens.a0 + jj; o[6] = dens.ar + jj;
    } else {
        o[0] = dens.ai + jj;
        o[1] = T.jp.r1 + jj; o[2] = T.jp.i1 + jj; o[3] = T.jp.r0 + jj; o[4] = T.jp.i0 + jj;
        o[5] = T.jp.r2 + jj; o[6] = T.jp.i2 + jj;
    }
}

// warp-wide: every lane calls it (active = the lane has a particle)
__device__ __forceinline__ void deposit1_warp(bool active, int j, bool neg, const Dep1& d, const Src1& T) {
    const int lane = threadIdx.x & 31;
    const int key = active ? 2 * j + (neg ? 0 : 1) : -1 - lane;
    {
        double v[14];
        if (active) dep1_chunk<0>(d, v); else for (int i = 0; i < 14; ++i) v[i] = 0.0;
        if (warp_runs_sum<14>(key, v) && active) {
            double* adr[14];
            dep1_addr<0>(T, j, neg, adr);
            dep1_addr<0>(T, j + 1, neg, adr + 7);
#pragma unroll
            for (int q = 0; q < 14; ++q) atomicAdd(adr[q], v[q]);
        }
    }
    {
        double v[14];
        if (active) dep1_chunk<1>(d, v); else for (int i = 0; i < 14; ++i) v[i] = 0.0;
        if (warp_runs_sum<14>(key, v) && active) {
            double* adr[14];
            dep1_addr<1>(T, j, neg, adr);
            dep1_addr<1>(T, j + 1, neg, adr + 7);
#pragma unroll
            for (int q = 0; q < 14; ++q) atomicAdd(adr[q], v[q]);
        }
    }
    {
        double v[14];
        if (active) dep1_chunk<2>(d, v); else for (int i = 0; i < 14; ++i) v[i] = 0.0;
        if (warp_runs_sum<14>(key, v) && active) {
            double* adr[14];
            dep1_addr<2>(T, j, neg, adr);
            dep1_addr<2>(T, j + 1, neg, adr + 7);
#pragma unroll
            for (int q = 0; q < 14; ++q) atomicAdd(adr[q], v[q]);
        }
    }
}

// S+ of one particle in modes k = 1, 0, 2 (src/PlasmaSpecies.cpp:508-559): v[6 cc + 2 m + (0|1)] for
// node j + cc, mode order (1, 0, 2), real / imaginary part
template <int ORD>
__device__ __forceinline__ void depositS1_values(const PState<ORD>& P, const PGeo& g, const Smem1& S,
                                                 double (&v)[12]) {
    const double qm = P.qm;
    const double PX = P.px, PY = P.py, D = P.dl;
    const PF1 F = gather1(S, g, false);
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D;
    const double ux = PX * invd, uy = PY * invd;
    const double ur = g.c * ux + g.s * uy, uth = g.c * uy - g.s * ux;
    const double dD = qm * ((PX * F.Wx + PY * F.Wy) * invd - F.Ez);
    const double ax = (qm * (gam * F.Wx + PY * F.Bz) * invd) * invd - PX * dD * invd * invd;
    const double ay = (qm * (gam * F.Wy - PX * F.Bz) * invd) * invd - PY * dD * invd * invd;
    const double wq = P.w * P.q;
    const double c2 = g.c * g.c - g.s * g.s, s2 = 2.0 * g.c * g.s;
    const double ckk[3] = {g.c, 1.0, c2}, skk[3] = {g.s, 0.0, s2};
    const int kk[3] = {1, 0, 2};
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        const double iv = S.iv[g.j + cc] * wq;
        const double Wc = cc ? g.W1 : g.W0;
        const double dWc = cc ? g.ih : -g.ih;
        const double Worc = cc ? g.Wor1 : g.Wor0;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            double Ar = ax * Wc + ux * ur * dWc;
            double Ai = ay * Wc + uy * ur * dWc;
            if (kk[m] != 0) {
                const double f2 = kk[m] * uth * Worc;
                Ar += f2 * uy;
                Ai -= f2 * ux;
            }
            v[6 * cc + 2 * m] = iv * (Ar * ckk[m] + Ai * skk[m]);
            v[6 * cc + 2 * m + 1] = iv * (Ai * ckk[m] - Ar * skk[m]);
        }
    }
}

__device__ __forceinline__ void depositS1_warp(bool active, int j, double (&v)[12], const Src1& T) {
    const int lane = threadIdx.x & 31;
    if (!active)
#pragma unroll
        for (int i = 0; i < 12; ++i) v[i] = 0.0;
    const int key = active ? j : -1 - lane;
    if (warp_runs_sum<12>(key, v) && active) {
        double* adr[12];
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int jj = j + cc;
            adr[6 * cc + 0] = T.S.r1 + jj; adr[6 * cc + 1] = T.S.i1 + jj;
            adr[6 * cc + 2] = T.S.r0 + jj; adr[6 * cc + 3] = T.S.i0 + jj;
            adr[6 * cc + 4] = T.S.r2 + jj; adr[6 * cc + 5] = T.S.i2 + jj;
        }
#pragma unroll
        for (int q = 0; q < 12; ++q) atomicAdd(adr[q], v[q]);
    }
}

// src/PlasmaSpecies.cpp:561-668 with uniform steps, the fields already gathered
template <int ORD>
__device__ __forceinline__ bool push1(PState<ORD>& P, const PF1& F, const SweepArgs& A, bool first) {
    const double qm = P.qm;
    const double X = P.x, Y = P.y, PX = P.px, PY = P.py, D = P.dl;
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D;
    double fv[5];
    fv[0] = PX * invd;
    fv[1] = PY * invd;
    fv[2] = qm * (gam * F.Wx * invd + F.By + PY * F.Bz * invd);
    fv[3] = qm * (gam * F.Wy * invd - F.Bx - PX * F.Bz * invd);
    fv[4] = qm * ((PX * F.Wx + PY * F.Wy) * invd - F.Ez);
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
    if (rn > R) {
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

// deposit of all particles of the scratch into the current source arrays (warp by warp)
template <int ORD, class Gate>
__device__ __forceinline__ void deposit_all1(const SweepArgs& A, const Smem1& S, const Src1& T, Gate& gate) {
    const int tid = threadIdx.x, lane = tid & 31;
    const int np = A.np, npad = A.npad, N = A.N;
    for (int base = tid - lane; base < np; base += kThreads) {
        const int p = base + lane;
        bool act = false;
        int j = 0;
        bool neg = true;
        Dep1 d;
        if (p < np) {
            PState<ORD> Q;
            pload(Q, gate.ps(A), npad, p);
            species_params(A, p, Q.q, Q.qm);
            if (Q.w != 0.0) {
                const PGeo g = geometry(S.r, S.ih, N, A.R, Q.x, Q.y);
                j = g.j;
                neg = Q.q < 0.0;
                d = dep1_basics(Q, g, S);
                act = true;
            }
        }
        deposit1_warp(act, j, neg, d, T);
    }
}

// row i of the B+ systems (src/FieldSolver.cpp:172-191 with chi = chi_0):
//   sys 0: L1D - chi (Dirichlet 0, N)   sys 1: L1F - chi (Dirichlet 0, flux row N)
//   sys 2: L0 - chi (regular axis, Dirichlet N)   sys 3: L2D - chi (Dirichlet 0, N)
// a, b, c of the row and c_{i-1}; dir = the row is a Dirichlet row (its right-hand side is 0)
__device__ __forceinline__ void row_bp(const Consts1& C, const Src1& T, int N, int sys, int i, double& a, double& b,
                                       double& c, double& cm, bool& dir) {
    const double chi = lg(T.chi.a0 + i);
    if (sys == 0) {
        a = ldc(C.l1a + i); b = ldc(C.l1b + i); c = ldc(C.l1c + i); cm = i > 0 ? ldc(C.l1c + i - 1) : 0.0;
        dir = (i == 0 || i == N);
    } else if (sys == 1) {
        a = ldc(C.lfa + i); b = ldc(C.lfb + i); c = ldc(C.lfc + i); cm = i > 0 ? ldc(C.lfc + i - 1) : 0.0;
        dir = (i == 0);
    } else if (sys == 2) {
        a = ldc(C.o0a + i); b = ldc(C.o0b + i); c = ldc(C.o0c + i); cm = i > 0 ? ldc(C.o0c + i - 1) : 0.0;
        dir = (i == N);
    } else {
        a = ldc(C.o2a + i); b = ldc(C.o2b + i); c = ldc(C.o2c + i); cm = i > 0 ? ldc(C.o2c + i - 1) : 0.0;
        dir = (i == 0 || i == N);
    }
    if (!dir) b = b - chi;
}

}  // namespace m1_detail

using namespace m1_detail;

size_t sweep_m1_smem_bytes(int M);

// One m = 1 sweep by the calling CTA (kThreads threads, one radial row per thread: M <= kThreads).
// EXT: the variant that also handles the smoothing filter (A.filter) and static beam sources (A.bstat)
template <int ORD, class Gate, bool EXT = false>
__device__ __forceinline__ bool sweep_m1_body(const SweepArgs& A, double* smem_raw, Gate& gate) {
    const int M = A.M, N = A.N, K = A.K;
    const int tid = threadIdx.x;
    const int i = tid;                                           // this thread's row
    const bool row = i < M;
    const Smem1 S = carve1(smem_raw, M);
    double* const scr = gate.srcs(A);                            // 2 x 30 x M sources, global
    const Consts1 C = consts1(A);
    const int np = A.np, npad = A.npad, lane = tid & 31;
    const double R = A.R;
    double* bg = gate.bgs(A);                                    // (3, M) background, global scratch
    unsigned long long* tim = A.timing;                          // optional: clock cycles per phase
    long long t_prev = (tim && tid == 0) ? clock64() : 0;
#define M1_MARK(ph)                                                           \
    do {                                                                      \
        if (tim && tid == 0) {                                                \
            const long long tn = clock64();                                   \
            tim[ph] += (unsigned long long)(tn - t_prev);                     \
            t_prev = tn;                                                      \
        }                                                                     \
    } while (0)

    // ---------------- prologue: grid, fresh plasma, background (src/Simulation.cpp:653-708)
    if (row) {
        S.r[i] = A.r[i];
        S.iv[i] = A.inv_V[i];
        S.ih[i] = (i < N) ? A.inv_h[i] : 0.0;
        S.bp.r0[i] = S.bp.i0[i] = S.bp.r1[i] = S.bp.i1[i] = S.bp.r2[i] = S.bp.i2[i] = 0.0;
        const Src1 T = src1_of(scr, M, 0);
        T.rhot.a0[i] = T.rhot.ar[i] = T.rhot.ai[i] = 0.0;             // scratch: immobile rho
        T.drho.a0[i] = T.drho.ar[i] = T.drho.ai[i] = 0.0;             // scratch: mobile rho
    }
    if (tid == 0) *S.lost = 0;
    for (int p = tid; p < np; p += kThreads) {
#pragma unroll
        for (int v = 0; v < 6; ++v) gate.ps(A)[(size_t)v * npad + p] = A.p_init[(size_t)v * npad + p];
        for (int v = 0; v < 5 * ORD; ++v) gate.ps(A)[(size_t)(6 + v) * npad + p] = 0.0;
    }
    __syncthreads();
    // src/PlasmaSpecies.cpp:480-506 for the immobile species and, when neutralising, the fresh mobile ones
    for (int p = tid; p < A.nbg; p += kThreads) {
        const double x = A.bg_p[p], y = A.bg_p[A.nbg + p], wq = A.bg_p[2 * A.nbg + p];
        if (wq == 0.0) continue;
        const PGeo g = geometry(S.r, S.ih, N, R, x, y);
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int jj = g.j + cc;
            const double a = wq * (cc ? g.W1 : g.W0) * S.iv[jj];
            const Src1 T = src1_of(scr, M, 0);
            atomicAdd(T.rhot.a0 + jj, a);
            atomicAdd(T.rhot.ar + jj, a * g.c);
            atomicAdd(T.rhot.ai + jj, -a * g.s);
        }
    }
    if (A.neutralize)
        for (int p = tid; p < np; p += kThreads) {
            const double w = A.p_init[5 * (size_t)npad + p];
            if (w == 0.0) continue;
            double q, qm;
            species_params(A, p, q, qm);
            const PGeo g = geometry(S.r, S.ih, N, R, A.p_init[p], A.p_init[npad + p]);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int jj = g.j + cc;
                const double a = w * q * (cc ? g.W1 : g.W0) * S.iv[jj];
                const Src1 T = src1_of(scr, M, 0);
                atomicAdd(T.drho.a0 + jj, a);
                atomicAdd(T.drho.ar + jj, a * g.c);
                atomicAdd(T.drho.ai + jj, -a * g.s);
            }
        }
    __syncthreads();
    if (row) {
        const Src1 T = src1_of(scr, M, 0);
        bg[i] = lg(T.rhot.a0 + i) - lg(T.drho.a0 + i);
        bg[M + i] = lg(T.rhot.ar + i) - lg(T.drho.ar + i);
        bg[2 * M + i] = lg(T.rhot.ai + i) - lg(T.drho.ai + i);
    }
    if (Gate::kActive && tid < 32) {                     // warp 0 checks the beam-source rows
        const bool ok = gate.before_rows(K - 1 < 2 ? K - 1 : 2);
        if (tid == 0) *S.flag = ok ? 1 : 0;
    }
    __syncthreads();
    if (Gate::kActive && !*S.flag) return false;
    const bool filt = EXT && A.filter;
    int scan_par = 0;
    if (filt) {                     // the background is smoothed like the plasma (src/Simulation.cpp:685-690)
        FilterSet<3> fg;
        fg.f[0] = bg; fg.f[1] = bg + M; fg.f[2] = bg + 2 * M;
        fg.op[0] = 0; fg.op[1] = fg.op[2] = 1;
        double* t0 = S.tot + (scan_par++ & 1) * 16 * kW;
        double* t1 = S.tot + (scan_par++ & 1) * 16 * kW;
        filter_rows1<3>(fg, A.fconsts, M, t0, t1);
        if (row) init_sources1_zero(src1_of(scr, M, 0), M, i);
    } else if (row) {
        init_sources1(src1_of(scr, M, 0), bg, M, i, beam_row1<Gate::kActive, EXT>(A, gate.bsrc(A), 0, i));
    }
    __syncthreads();
    deposit_all1<ORD>(A, S, src1_of(scr, M, 0), gate);
    __syncthreads();
    M1_MARK(0);

    const double fc = A.flux_coef;
    const int niter = A.picard > 0 ? A.picard : 1;
    for (int k = 0; k < K; ++k) {
        const int cb = k & 1;                                    // this slice's source buffer
        // the next slice's sources: background + beam (the push of this slice deposits on top); the
        // buffer's previous content (slice k-1) was last read before the end of slice k-1
        if (filt) {
            if (k + 1 < K && row) init_sources1_zero(src1_of(scr, M, cb ^ 1), M, i);
            filter_sources1<Gate::kActive>(A, src1_of(scr, M, cb), bg, gate.bsrc(A), k, S.tot, scan_par);
        } else if (k + 1 < K && row) {
            init_sources1(src1_of(scr, M, cb ^ 1), bg, M, i, beam_row1<Gate::kActive, EXT>(A, gate.bsrc(A), k + 1, i));
        }
        // ---------------- P2: psi, E_z, B_z (9 systems with fixed Thomas factors)
        //   L0: psi0 = -rhot0, ez0 = -drho0, bz0 = -(J_theta1' + J_theta1 / r)
        //   L1D: psi1 r/i, ez1 r/i, bz1 r/i
        {
            const Src1 T = src1_of(scr, M, cb);
            double d[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) d[e] = 0.0;
            double f0 = 1.0, r0 = 0.0, b0 = 1.0, f1 = 1.0, r1 = 0.0, b1 = 1.0;
            if (row) {
                f0 = ldc(C.l0f + i); r0 = ldc(C.l0r + i); b0 = ldc(C.l0b + i);
                f1 = ldc(C.d1f + i); r1 = ldc(C.d1r + i); b1 = ldc(C.d1b + i);
                if (i < N) {
                    d[0] = -1.0 * lg(T.rhot.a0 + i);
                    d[1] = -1.0 * lg(T.drho.a0 + i);
                    const double t1 = grad1g(C, N, T.jp.i1, i, true), t2 = over_r1g(C, T.jp.i1, i);
                    d[2] = 1.0 * (-(t1 + t2));
                }
                if (i >= 1 && i < N) {
                    d[3] = -1.0 * lg(T.rhot.ar + i);
                    d[4] = -1.0 * lg(T.rhot.ai + i);
                    d[5] = -1.0 * lg(T.drho.ar + i);
                    d[6] = -1.0 * lg(T.drho.ai + i);
                    const double D1r = grad1g(C, N, T.jp.r2, i, true) + 2.0 * over_r1g(C, T.jp.r2, i);
                    const double D1i = grad1g(C, N, T.jp.i2, i, true) + 2.0 * over_r1g(C, T.jp.i2, i);
                    const double Dmr = grad1g(C, N, T.jp.r0, i, false), Dmi = grad1g(C, N, T.jp.i0, i, false);
                    d[7] = 1.0 * (-0.5 * (D1i + Dmi));
                    d[8] = 1.0 * (0.5 * (D1r - Dmr));
                }
            }
            const int grp[9] = {0, 0, 0, 1, 1, 1, 1, 1, 1};
            const double fa[2] = {f0, f1};
            double fb[9], yb[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) fb[e] = (e < 3 ? r0 : r1) * d[e];
            scan_fwd_g<2, 9>(fa, fb, grp, yb, S.tot + (scan_par++ & 1) * 16 * kW);
            double y[9];                                            // no row: identity (y = 0)
#pragma unroll
            for (int e = 0; e < 9; ++e) y[e] = row ? fma(e < 3 ? f0 : f1, yb[e], fb[e]) : 0.0;
            const double ba[2] = {b0, b1};
            double xa[9];
            scan_bwd_g<2, 9>(ba, y, grp, xa, S.tot + (scan_par++ & 1) * 16 * kW);
            if (row) {
                double x[9];
#pragma unroll
                for (int e = 0; e < 9; ++e) x[e] = fma(e < 3 ? b0 : b1, xa[e], y[e]);
                S.psi.a0[i] = x[0]; S.ez.a0[i] = x[1]; S.bz.a0[i] = x[2];
                S.psi.ar[i] = x[3]; S.psi.ai[i] = x[4];
                S.ez.ar[i] = x[5]; S.ez.ai[i] = x[6];
                S.bz.ar[i] = x[7]; S.bz.ai[i] = x[8];
            }
        }
        __syncthreads();
        // W+ = -(d/dx + i d/dy) psi (src/Simulation.cpp:477-498)
        if (row) {
            const double t1 = grad1(C, N, S.psi.a0, i, false);
            const double t2 = grad1(C, N, S.psi.ar, i, true), t3 = over_r1(C, S.psi.ar, i);
            const double t4 = grad1(C, N, S.psi.ai, i, true), t5 = over_r1(C, S.psi.ai, i);
            S.wp.r1[i] = -t1;
            S.wp.i1[i] = 0.0;
            S.wp.r2[i] = -(t2 - t3);
            S.wp.i2[i] = -(t4 - t5);
            S.wp.r0[i] = -(t2 + t3);
            S.wp.i0[i] = (t4 + t5);
        }
        __syncthreads();
        M1_MARK(1);

        // ---------------- P3: S+ (src/PlasmaSpecies.cpp:508-559)
        for (int base = tid - lane; base < np; base += kThreads) {
            const int p = base + lane;
            bool act = false;
            int j = 0;
            double v[12];
            if (p < np) {
                PState<ORD> Q;
                pload(Q, gate.ps(A), npad, p);
                species_params(A, p, Q.q, Q.qm);
                if (Q.w != 0.0) {
                    const PGeo g = geometry(S.r, S.ih, N, R, Q.x, Q.y);
                    j = g.j;
                    depositS1_values(Q, g, S, v);
                    act = true;
                }
            }
            depositS1_warp(act, j, v, src1_of(scr, M, cb));
        }
        __syncthreads();
        M1_MARK(2);

        // ---------------- P4: B+ (src/Simulation.cpp:535-591)
        if (filt) {                 // S+ smoothed (src/Simulation.cpp:810-816): each thread's own row, the only
            const Src1 T = src1_of(scr, M, cb);                  // one its B+ right-hand sides read
            FilterSet<6> fsS;
            fsS.f[0] = T.S.r0; fsS.f[1] = T.S.i0; fsS.f[2] = T.S.r1; fsS.f[3] = T.S.i1; fsS.f[4] = T.S.r2;
            fsS.f[5] = T.S.i2;
            fsS.op[0] = fsS.op[1] = 0; fsS.op[2] = fsS.op[3] = 1; fsS.op[4] = fsS.op[5] = 2;
            double* t0 = S.tot + (scan_par++ & 1) * 16 * kW;
            double* t1 = S.tot + (scan_par++ & 1) * 16 * kW;
            filter_rows1<6>(fsS, A.fconsts, M, t0, t1);
        }
        {
            const Src1 T = src1_of(scr, M, cb);
            // fixed part of the right-hand sides: (d/dx + i d/dy) J_z + S
            double gr[6] = {0, 0, 0, 0, 0, 0};                   // g r1 i1 r0 i0 r2 i2
            double ra[4], rbv[4], rc[4], rcm[4];
            bool dir[4];
            double m[4][4];
#pragma unroll
            for (int sy = 0; sy < 4; ++sy) {
                m[sy][0] = 1.0; m[sy][1] = 0.0; m[sy][2] = 0.0; m[sy][3] = 1.0;
                ra[sy] = 0.0; rbv[sy] = 1.0; rc[sy] = 0.0; rcm[sy] = 0.0; dir[sy] = true;
            }
            if (row) {
                const double t1 = grad1g(C, N, T.jz.a0, i, false);
                const double t2 = grad1g(C, N, T.jz.ar, i, true), t3 = over_r1g(C, T.jz.ar, i);
                const double t4 = grad1g(C, N, T.jz.ai, i, true), t5 = over_r1g(C, T.jz.ai, i);
                gr[0] = t1 + lg(T.S.r1 + i);
                gr[1] = lg(T.S.i1 + i);
                gr[2] = (t2 + t3) + lg(T.S.r0 + i);
                gr[3] = -(t4 + t5) + lg(T.S.i0 + i);
                gr[4] = (t2 - t3) + lg(T.S.r2 + i);
                gr[5] = (t4 - t5) + lg(T.S.i2 + i);
#pragma unroll
                for (int sy = 0; sy < 4; ++sy) {
                    row_bp(C, T, N, sy, i, ra[sy], rbv[sy], rc[sy], rcm[sy], dir[sy]);
                    // T_i = [[b_i, -a_i c_{i-1}], [1, 0]], renormalised as scan_pivots needs
                    m[sy][0] = rbv[sy]; m[sy][1] = -ra[sy] * rcm[sy]; m[sy][2] = 1.0; m[sy][3] = 0.0;
                    renorm(m[sy][0], m[sy][1], m[sy][2], m[sy][3]);
                }
            }
            double pp[4], qq[4];
            scan_pivots<4>(m, pp, qq, S.tot + (scan_par++ & 1) * 16 * kW);
            double rinv[4], fa[4], ba[4];
#pragma unroll
            for (int sy = 0; sy < 4; ++sy) {
                rinv[sy] = 1.0; fa[sy] = 1.0; ba[sy] = 1.0;
                if (!row) continue;
                const double pn = rbv[sy] * pp[sy] - ra[sy] * rcm[sy] * qq[sy];
                rinv[sy] = pp[sy] / pn;                          // 1/u_i = p_{i-1} / p_i
                fa[sy] = -rinv[sy] * ra[sy];
                ba[sy] = -(rc[sy] * rinv[sy]);
            }
            const int grp[6] = {0, 1, 2, 2, 3, 3};             // r1 (L1D), i1 (L1F), r0 i0 (L0), r2 i2 (L2D)
            const double chr = row ? lg(T.chi.ar + i) : 0.0, chi_i = row ? lg(T.chi.ai + i) : 0.0;
            const double jzN = lg(T.jz.a0 + N);
            for (int it = 0; it < niter; ++it) {
                double d[6] = {0, 0, 0, 0, 0, 0};
                if (row) {
                    const double cr = chr, ci = chi_i;
                    const double b0r = S.bp.r0[i], b0i = S.bp.i0[i], b1r = S.bp.r1[i], b1i = S.bp.i1[i];
                    const double b2r = S.bp.r2[i], b2i = S.bp.i2[i];
                    double r1v = -gr[1], i1v = gr[0];
                    double r0v = -gr[3], i0v = gr[2], r2v = -gr[5], i2v = gr[4];
                    r0v += cr * b1r + ci * b1i;  i0v += cr * b1i - ci * b1r;
                    r1v += cr * b0r - ci * b0i + cr * b2r + ci * b2i;
                    i1v += cr * b0i + ci * b0r + cr * b2i - ci * b2r;
                    r2v += cr * b1r - ci * b1i;  i2v += cr * b1i + ci * b1r;
                    d[0] = dir[0] ? 0.0 : 1.0 * r1v;
                    d[1] = dir[1] ? 0.0 : 1.0 * i1v;
                    if (i == N && !dir[1]) d[1] -= fc * jzN;
                    d[2] = dir[2] ? 0.0 : 1.0 * r0v;
                    d[3] = dir[2] ? 0.0 : 1.0 * i0v;
                    d[4] = dir[3] ? 0.0 : 1.0 * r2v;
                    d[5] = dir[3] ? 0.0 : 1.0 * i2v;
                }
                double fb[6], yb[6];
#pragma unroll
                for (int e = 0; e < 6; ++e) fb[e] = rinv[grp[e]] * d[e];
                scan_fwd_g<4, 6>(fa, fb, grp, yb, S.tot + (scan_par++ & 1) * 16 * kW);
                double y[6];
#pragma unroll
                for (int e = 0; e < 6; ++e) y[e] = row ? fma(fa[grp[e]], yb[e], fb[e]) : 0.0;
                double xa[6];
                scan_bwd_g<4, 6>(ba, y, grp, xa, S.tot + (scan_par++ & 1) * 16 * kW);
                double x[6];
#pragma unroll
                for (int e = 0; e < 6; ++e) x[e] = fma(ba[grp[e]], xa[e], y[e]);
                // one step of iterative refinement with the same factors: the pivots come from a prefix
                // product, slightly less accurate than Thomas' recurrence on these ill-conditioned rows
                // (L1D on a 100x-stretched grid); r = d - A x with the exact rows, then x += A^-1 r
                if (row) {                                              // (each thread reads only its own bp row above)
                    S.bp.r1[i] = x[0]; S.bp.i1[i] = x[1];
                    S.bp.r0[i] = x[2]; S.bp.i0[i] = x[3];
                    S.bp.r2[i] = x[4]; S.bp.i2[i] = x[5];
                }
                __syncthreads();
                double rr[6] = {0, 0, 0, 0, 0, 0};
                if (row) {
                    double* const xs[6] = {S.bp.r1, S.bp.i1, S.bp.r0, S.bp.i0, S.bp.r2, S.bp.i2};
#pragma unroll
                    for (int e = 0; e < 6; ++e) {
                        const int sy = grp[e];
                        const double xm = i > 0 ? xs[e][i - 1] : 0.0, xp = i < N ? xs[e][i + 1] : 0.0;
                        rr[e] = d[e] - (ra[sy] * xm + rbv[sy] * x[e] + rc[sy] * xp);
                    }
                }
#pragma unroll
                for (int e = 0; e < 6; ++e) fb[e] = rinv[grp[e]] * rr[e];
                scan_fwd_g<4, 6>(fa, fb, grp, yb, S.tot + (scan_par++ & 1) * 16 * kW);
#pragma unroll
                for (int e = 0; e < 6; ++e) y[e] = row ? fma(fa[grp[e]], yb[e], fb[e]) : 0.0;
                scan_bwd_g<4, 6>(ba, y, grp, xa, S.tot + (scan_par++ & 1) * 16 * kW);
                if (row) {
#pragma unroll
                    for (int e = 0; e < 6; ++e) x[e] += fma(ba[grp[e]], xa[e], y[e]);
                    S.bp.r1[i] = x[0]; S.bp.i1[i] = x[1];
                    S.bp.r0[i] = x[2]; S.bp.i0[i] = x[3];
                    S.bp.r2[i] = x[4]; S.bp.i2[i] = x[5];
                }
            }
        }
        __syncthreads();
        M1_MARK(3);

        // ---------------- P5: store slice k (src/Simulation.cpp:594-633)
        if (row) {
            const Src1 T = src1_of(scr, M, cb);
            const size_t fb = (size_t)k * M;
            double* F = gate.fld(A) + (fb + i) * F_NC1;
            F[F_EP1R] = S.wp.r1[i] + S.bp.i1[i];
            F[F_EP1I] = S.wp.i1[i] - S.bp.r1[i];
            F[F_BP1R] = S.bp.r1[i];
            F[F_BP1I] = S.bp.i1[i];
            F[F_EZ0] = S.ez.a0[i];
            F[F_BZ0] = S.bz.a0[i];
            F[F_EP0R] = S.wp.r0[i] + S.bp.i0[i];
            F[F_EP0I] = S.wp.i0[i] - S.bp.r0[i];
            F[F_EP2R] = S.wp.r2[i] + S.bp.i2[i];
            F[F_EP2I] = S.wp.i2[i] - S.bp.r2[i];
            F[F_BP0R] = S.bp.r0[i];
            F[F_BP0I] = S.bp.i0[i];
            F[F_BP2R] = S.bp.r2[i];
            F[F_BP2I] = S.bp.i2[i];
            F[F_EZ1R] = S.ez.ar[i];
            F[F_EZ1I] = S.ez.ai[i];
            F[F_BZ1R] = S.bz.ar[i];
            F[F_BZ1I] = S.bz.ai[i];
            double* D = gate.diag(A) + (fb + i) * D_NC1;
            D[D_PSI0] = S.psi.a0[i];
            D[D_NE0] = lg(T.ne.a0 + i);
            D[D_NI0] = lg(T.ni.a0 + i);
            D[D_PSI1R] = S.psi.ar[i];
            D[D_PSI1I] = S.psi.ai[i];
            D[D_NE1R] = lg(T.ne.ar + i);
            D[D_NE1I] = lg(T.ne.ai + i);
            D[D_NI1R] = lg(T.ni.ar + i);
            D[D_NI1I] = lg(T.ni.ai + i);
        }
        if (k + 1 < K) {
            // push every particle with the fields of slice k and deposit it into slice k+1 (the other
            // source buffer, initialised at the start of this slice)
            const bool first = (k == 0);
            const Src1 Tn = src1_of(scr, M, cb ^ 1);
            for (int base = tid - lane; base < np; base += kThreads) {
                const int p = base + lane;
                bool act = false;
                int j = 0;
                bool neg = true;
                Dep1 d;
                if (p < np) {
                    PState<ORD> Q;
                    pload(Q, gate.ps(A), npad, p);
                    species_params(A, p, Q.q, Q.qm);
                    if (Q.w != 0.0) {
                        const PGeo g = geometry(S.r, S.ih, N, R, Q.x, Q.y);
                        const PF1 F = gather1(S, g, true);
                        if (push1(Q, F, A, first)) {
                            const PGeo g2 = geometry(S.r, S.ih, N, R, Q.x, Q.y);
                            j = g2.j;
                            neg = Q.q < 0.0;
                            d = dep1_basics(Q, g2, S);
                            act = true;
                        } else {
                            atomicAdd(S.lost, 1);
                        }
                        pstore(Q, gate.ps(A), npad, p);
                    }
                }
                deposit1_warp(act, j, neg, d, Tn);
            }
            __syncthreads();
            M1_MARK(4);
        }
        if (Gate::kActive) gate.slice_done_all(k);
        __syncthreads();
        if (Gate::kActive) {
            if (tid < 32) {                                   // warp 0: publish slice k, check the next rows
                bool ok = true;
                if (tid == 0) ok = gate.slice_done(k);
                ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
                if (ok && k + 1 < K) ok = gate.before_rows(k + 3 < K ? k + 3 : K - 1);
                if (tid == 0) *S.flag = ok ? 1 : 0;
            }
            __syncthreads();
            if (!*S.flag) return false;
        }
    }
    if (tid == 0 && A.counters) atomicAdd(&A.counters[0], (unsigned long long)*S.lost);
    return true;
#undef M1_MARK
}

}  // namespace qzb
