// qz_sweep_body.cuh -- the quasi-static xi sweep of one time step by ONE CTA (sm_100a, FP64).
//
// Replaces the per-slice kernel chain of Simulation::step_fields (src/Simulation.cpp:636-795):
//   zero_sources -> PlasmaSpecies::deposit -> combine_sources -> solve_slice_fields
//   (psi, E_z, W+, B_z, deposit_S, B+) -> store_slice -> PlasmaSpecies::push
// for azimuthal mode m = 0.
//
// Layout. The radial arrays of a slice (sources, fields, grid, stencils, operator rows) live in shared
// memory (the constant ones fall back to global memory for very large grids). With at most 512
// plasma particles, thread p owns particle p and keeps its state -- position, momentum, Delta,
// weight and the Adams-Bashforth history -- in registers for the whole sweep; larger plasmas keep
// the state in a global scratch buffer.
//
// Tridiagonal solves. Every system is solved by all 512 threads at once: thread t owns rows
// [t*R, t*R + R), and the three Thomas recurrences -- pivots u_i = b_i - a_i c_{i-1} / u_{i-1},
// forward y_i = (d_i - a_i y_{i-1}) / u_i, backward x_i = y_i - (c_i / u_i) x_{i+1} -- are evaluated
// as block-wide scans: pivots as normalised prefix products of 2x2 matrices, the substitutions as
// scans of affine maps. Each scan costs five warp-shuffle levels and one block barrier. The psi,
// E_z and B_z systems share the constant operator L0, whose pivots are computed once on the host.
//
// Slice schedule (4 phase barriers + 5 scan barriers per slice):
//   P2  psi, E_z, B_z (two scans, three right-hand sides); sources of slice k+1 = beam + background
//   P3  S+ deposit by the particles
//   P4  B_r, B_theta (pivot scan + forward and backward scans of the two systems)
//   P5  store slice k; push k -> k+1 and deposit into the sources of slice k+1
#pragma once
#include "qz_device.cuh"
#include "qz_internal.h"

namespace qzb {

namespace sweep_detail {

constexpr int kThreads = kSweepThreads;
constexpr int kW = kThreads / 32;
constexpr unsigned FULL = 0xffffffffu;

// Gate of a stand-alone sweep: no other CTA to wait for or to inform.
struct NoGate {
    static constexpr bool kActive = false;
    __device__ bool before_rows(int) { return true; }       // warp 0: beam-source rows <= row are final
    __device__ void slice_done_all(int) {}                   // every thread, after its stores of slice k
    __device__ bool slice_done(int) { return true; }         // thread 0, after the barrier: publish slice k
    // this sweep's buffers
    __device__ const double* bsrc(const SweepArgs& A) const { return A.bsrc; }
    __device__ double* fld(const SweepArgs& A) const { return A.fld; }
    __device__ double* diag(const SweepArgs& A) const { return A.diag; }
    __device__ double* ps(const SweepArgs& A) const { return A.ps; }
    __device__ double* srcs(const SweepArgs& A) const { return A.srcs; }
    __device__ double* bgs(const SweepArgs& A) const { return A.bgs; }
    __device__ double* traj(const SweepArgs& A) const { return A.traj; }
    __device__ double* wrec(const SweepArgs& A) const { return A.wrec; }
};

// ---------------------------------------------------------------- block scans
// Shared scratch for the warp totals of one scan: 8 x kW doubles; two of them alternate.

// exact power-of-two rescaling of a 2x2 matrix (its largest entry into [1, 2))
__device__ __forceinline__ void renorm(double& m00, double& m01, double& m10, double& m11) {
    const double mx = fmax(fmax(fabs(m00), fabs(m01)), fmax(fabs(m10), fabs(m11)));
    if (!(mx > 0.0) || !(mx < 1e300)) return;
    const int e = ((__double2hiint(mx) >> 20) & 0x7ff) - 1023;
    const double s = __hiloint2double((1023 - e) << 20, 0);
    m00 *= s; m01 *= s; m10 *= s; m11 *= s;
}

// Exclusive forward scan of the affine maps y -> a y + b (thread order = row order), applied to
// y_{-1} = 0: yb[r] is y just before this thread's rows.
template <int NR>
__device__ __forceinline__ void scan_fwd(double a, const double (&b)[NR], double (&yb)[NR], double* tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double A = a, B[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) B[r] = b[r];
#pragma unroll
    for (int st = 1; st < 32; st <<= 1) {
        const double Ap = __shfl_up_sync(FULL, A, st);
        double Bp[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) Bp[r] = __shfl_up_sync(FULL, B[r], st);
        if (lane >= st) {
#pragma unroll
            for (int r = 0; r < NR; ++r) B[r] = fma(A, Bp[r], B[r]);
            A *= Ap;
        }
    }
    if (lane == 31) {
        tot[warp] = A;
#pragma unroll
        for (int r = 0; r < NR; ++r) tot[kW * (1 + r) + warp] = B[r];
    }
    double eA = __shfl_up_sync(FULL, A, 1), eB[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) eB[r] = __shfl_up_sync(FULL, B[r], 1);
    if (lane == 0) {
        eA = 1.0;
#pragma unroll
        for (int r = 0; r < NR; ++r) eB[r] = 0.0;
    }
    __syncthreads();
    double ta = lane < kW ? tot[lane] : 1.0, tb[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) tb[r] = lane < kW ? tot[kW * (1 + r) + lane] : 0.0;
#pragma unroll
    for (int st = 1; st < kW; st <<= 1) {
        const double ap = __shfl_up_sync(FULL, ta, st);
        double bp[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) bp[r] = __shfl_up_sync(FULL, tb[r], st);
        if (lane >= st) {
#pragma unroll
            for (int r = 0; r < NR; ++r) tb[r] = fma(ta, bp[r], tb[r]);
            ta *= ap;
        }
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const double cw = __shfl_sync(FULL, tb[r], (warp + 31) & 31);
        yb[r] = fma(eA, warp > 0 ? cw : 0.0, eB[r]);
    }
}

// Exclusive backward scan of x -> a x + b applied to x_{end} = 0: xa[r] is x just after this
// thread's rows.
template <int NR>
__device__ __forceinline__ void scan_bwd(double a, const double (&b)[NR], double (&xa)[NR], double* tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double A = a, B[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) B[r] = b[r];
#pragma unroll
    for (int st = 1; st < 32; st <<= 1) {
        const double An = __shfl_down_sync(FULL, A, st);
        double Bn[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) Bn[r] = __shfl_down_sync(FULL, B[r], st);
        if (lane + st < 32) {
#pragma unroll
            for (int r = 0; r < NR; ++r) B[r] = fma(A, Bn[r], B[r]);
            A *= An;
        }
    }
    if (lane == 0) {
        tot[warp] = A;
#pragma unroll
        for (int r = 0; r < NR; ++r) tot[kW * (1 + r) + warp] = B[r];
    }
    double eA = __shfl_down_sync(FULL, A, 1), eB[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) eB[r] = __shfl_down_sync(FULL, B[r], 1);
    if (lane == 31) {
        eA = 1.0;
#pragma unroll
        for (int r = 0; r < NR; ++r) eB[r] = 0.0;
    }
    __syncthreads();
    double ta = lane < kW ? tot[lane] : 1.0, tb[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) tb[r] = lane < kW ? tot[kW * (1 + r) + lane] : 0.0;
#pragma unroll
    for (int st = 1; st < kW; st <<= 1) {
        const double an = __shfl_down_sync(FULL, ta, st);
        double bn[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) bn[r] = __shfl_down_sync(FULL, tb[r], st);
        if (lane + st < kW) {
#pragma unroll
            for (int r = 0; r < NR; ++r) tb[r] = fma(ta, bn[r], tb[r]);
            ta *= an;
        }
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const double cw = __shfl_sync(FULL, tb[r], (warp + 1) & 31);
        xa[r] = fma(eA, warp < kW - 1 ? cw : 0.0, eB[r]);
    }
}

// The same two scans for NS independent systems, each with its own map y -> a[s] y + b[s].
template <int NS>
__device__ __forceinline__ void scan_fwd_n(const double (&a)[NS], const double (&b)[NS], double (&yb)[NS],
                                           double* tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double A[NS], B[NS];
#pragma unroll
    for (int r = 0; r < NS; ++r) { A[r] = a[r]; B[r] = b[r]; }
#pragma unroll
    for (int st = 1; st < 32; st <<= 1) {
        double Ap[NS], Bp[NS];
#pragma unroll
        for (int r = 0; r < NS; ++r) { Ap[r] = __shfl_up_sync(FULL, A[r], st); Bp[r] = __shfl_up_sync(FULL, B[r], st); }
        if (lane >= st)
#pragma unroll
            for (int r = 0; r < NS; ++r) { B[r] = fma(A[r], Bp[r], B[r]); A[r] *= Ap[r]; }
    }
    if (lane == 31)
#pragma unroll
        for (int r = 0; r < NS; ++r) { tot[kW * (2 * r) + warp] = A[r]; tot[kW * (2 * r + 1) + warp] = B[r]; }
    double eA[NS], eB[NS];
#pragma unroll
    for (int r = 0; r < NS; ++r) {
        eA[r] = __shfl_up_sync(FULL, A[r], 1);
        eB[r] = __shfl_up_sync(FULL, B[r], 1);
        if (lane == 0) { eA[r] = 1.0; eB[r] = 0.0; }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NS; ++r) {
        double ta = lane < kW ? tot[kW * (2 * r) + lane] : 1.0, tb = lane < kW ? tot[kW * (2 * r + 1) + lane] : 0.0;
#pragma unroll
        for (int st = 1; st < kW; st <<= 1) {
            const double ap = __shfl_up_sync(FULL, ta, st), bp = __shfl_up_sync(FULL, tb, st);
            if (lane >= st) { tb = fma(ta, bp, tb); ta *= ap; }
        }
        const double cw = __shfl_sync(FULL, tb, (warp + 31) & 31);
        yb[r] = fma(eA[r], warp > 0 ? cw : 0.0, eB[r]);
    }
}

template <int NS>
__device__ __forceinline__ void scan_bwd_n(const double (&a)[NS], const double (&b)[NS], double (&xa)[NS],
                                           double* tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double A[NS], B[NS];
#pragma unroll
    for (int r = 0; r < NS; ++r) { A[r] = a[r]; B[r] = b[r]; }
#pragma unroll
    for (int st = 1; st < 32; st <<= 1) {
        double An[NS], Bn[NS];
#pragma unroll
        for (int r = 0; r < NS; ++r) { An[r] = __shfl_down_sync(FULL, A[r], st); Bn[r] = __shfl_down_sync(FULL, B[r], st); }
        if (lane + st < 32)
#pragma unroll
            for (int r = 0; r < NS; ++r) { B[r] = fma(A[r], Bn[r], B[r]); A[r] *= An[r]; }
    }
    if (lane == 0)
#pragma unroll
        for (int r = 0; r < NS; ++r) { tot[kW * (2 * r) + warp] = A[r]; tot[kW * (2 * r + 1) + warp] = B[r]; }
    double eA[NS], eB[NS];
#pragma unroll
    for (int r = 0; r < NS; ++r) {
        eA[r] = __shfl_down_sync(FULL, A[r], 1);
        eB[r] = __shfl_down_sync(FULL, B[r], 1);
        if (lane == 31) { eA[r] = 1.0; eB[r] = 0.0; }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NS; ++r) {
        double ta = lane < kW ? tot[kW * (2 * r) + lane] : 1.0, tb = lane < kW ? tot[kW * (2 * r + 1) + lane] : 0.0;
#pragma unroll
        for (int st = 1; st < kW; st <<= 1) {
            const double an = __shfl_down_sync(FULL, ta, st), bn = __shfl_down_sync(FULL, tb, st);
            if (lane + st < kW) { tb = fma(ta, bn, tb); ta *= an; }
        }
        const double cw = __shfl_sync(FULL, tb, (warp + 1) & 31);
        xa[r] = fma(eA[r], warp < kW - 1 ? cw : 0.0, eB[r]);
    }
}

// Exclusive scan of 2x2 matrix products (later rows on the left) for NS systems: on return
// (p[s], q[s]) = first column of the product of all matrices before this thread's rows.
template <int NS>
__device__ __forceinline__ void scan_pivots(double (&m)[NS][4], double (&p)[NS], double (&q)[NS], double* tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // The thread's matrices must come renormalised (largest entry in [1, 2)); a product of at most 32 such
    // matrices stays below 2^63 and the products of the 16 renormalised warp totals below 2^31, so the
    // scan renormalises once per lane after the warp stage instead of at every level. Renormalising
    // scales by powers of two, which is exact, and the pivots use only ratios of p and q: the results
    // are the same bits either way.
#pragma unroll
    for (int st = 1; st < 32; st <<= 1) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const double p00 = __shfl_up_sync(FULL, m[s][0], st), p01 = __shfl_up_sync(FULL, m[s][1], st);
            const double p10 = __shfl_up_sync(FULL, m[s][2], st), p11 = __shfl_up_sync(FULL, m[s][3], st);
            if (lane >= st) {
                const double n00 = m[s][0] * p00 + m[s][1] * p10, n01 = m[s][0] * p01 + m[s][1] * p11;
                const double n10 = m[s][2] * p00 + m[s][3] * p10, n11 = m[s][2] * p01 + m[s][3] * p11;
                m[s][0] = n00; m[s][1] = n01; m[s][2] = n10; m[s][3] = n11;
            }
        }
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) renorm(m[s][0], m[s][1], m[s][2], m[s][3]);
    if (lane == 31)
#pragma unroll
        for (int s = 0; s < NS; ++s)
#pragma unroll
            for (int e = 0; e < 4; ++e) tot[kW * (4 * s + e) + warp] = m[s][e];
    double ex[NS][4];
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int e = 0; e < 4; ++e) ex[s][e] = __shfl_up_sync(FULL, m[s][e], 1);
    if (lane == 0)
#pragma unroll
        for (int s = 0; s < NS; ++s) { ex[s][0] = 1.0; ex[s][1] = 0.0; ex[s][2] = 0.0; ex[s][3] = 1.0; }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        double t00 = lane < kW ? tot[kW * (4 * s) + lane] : 1.0, t01 = lane < kW ? tot[kW * (4 * s + 1) + lane] : 0.0;
        double t10 = lane < kW ? tot[kW * (4 * s + 2) + lane] : 0.0, t11 = lane < kW ? tot[kW * (4 * s + 3) + lane] : 1.0;
#pragma unroll
        for (int st = 1; st < kW; st <<= 1) {
            const double p00 = __shfl_up_sync(FULL, t00, st), p01 = __shfl_up_sync(FULL, t01, st);
            const double p10 = __shfl_up_sync(FULL, t10, st), p11 = __shfl_up_sync(FULL, t11, st);
            if (lane >= st) {
                const double n00 = t00 * p00 + t01 * p10, n01 = t00 * p01 + t01 * p11;
                const double n10 = t10 * p00 + t11 * p10, n11 = t10 * p01 + t11 * p11;
                t00 = n00; t01 = n01; t10 = n10; t11 = n11;
            }
        }
        const int src = (warp + 31) & 31;
        double c00 = __shfl_sync(FULL, t00, src), c10 = __shfl_sync(FULL, t10, src);
        if (warp == 0) { c00 = 1.0; c10 = 0.0; }
        // column 0 of (within-warp exclusive product) x (carry of the earlier warps)
        p[s] = ex[s][0] * c00 + ex[s][1] * c10;
        q[s] = ex[s][2] * c00 + ex[s][3] * c10;
    }
}

// ---------------------------------------------------------------- batched shared-memory adds
// All NA updates of one thread are issued together (independent compare-and-swap rounds) instead
// of one serialised atomic loop per address. Lock-free: every round at least one contender of
// each address succeeds, so the loop ends after at most one round per contender.
template <int NA>
__device__ __forceinline__ void add_multi(double* const (&p)[NA], const double (&v)[NA]) {
    unsigned long long old[NA];
#pragma unroll
    for (int i = 0; i < NA; ++i) old[i] = __double_as_longlong(*reinterpret_cast<volatile double*>(p[i]));
    unsigned pend = (1u << NA) - 1u;
    for (int round = 0; pend && round < 4 * kThreads; ++round) {
#pragma unroll
        for (int i = 0; i < NA; ++i)
            if (pend & (1u << i)) {
                const unsigned long long nv = __double_as_longlong(__longlong_as_double(old[i]) + v[i]);
                const unsigned long long got = atomicCAS(reinterpret_cast<unsigned long long*>(p[i]), old[i], nv);
                if (got == old[i]) pend &= ~(1u << i); else old[i] = got;
            }
    }
}

// Warp aggregation of deposits: lanes holding contributions to the same cell form runs of equal
// keys in lane order (plasma particles stay close to their radial loading order); a segmented
// warp-shuffle scan sums each run, and only the last lane of a run updates shared memory. Runs
// split by reordering only cost extra updates, never correctness. Blowout piles tens of particles
// into a few sheath or axis cells, where per-particle updates of the same word would serialise.
template <int NV>
__device__ __forceinline__ bool warp_runs_sum(int key, double (&v)[NV]) {
    const int lane = threadIdx.x & 31;
    const int kprev = __shfl_up_sync(FULL, key, 1);
    const bool head = (lane == 0) || (kprev != key);
    const unsigned heads = __ballot_sync(FULL, head);
    if (heads == FULL) return true;                   // no shared cell in this warp
    const unsigned le = heads & (0xffffffffu >> (31 - lane));     // run heads at or below this lane
    const int seg = __popc(le);
    // the scan levels the longest run of the warp needs: a level of stride st adds only within runs
    // longer than st, so stopping after them leaves every sum as the full scan gives it, bit for bit
    const int maxoff = (int)__reduce_max_sync(FULL, (unsigned)(lane - (31 - __clz(le))));
#pragma unroll 1
    for (int st = 1; st <= maxoff; st <<= 1) {
        const int sp = __shfl_up_sync(FULL, seg, st);
        double vp[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) vp[i] = __shfl_up_sync(FULL, v[i], st);
        if (lane >= st && sp == seg)
#pragma unroll
            for (int i = 0; i < NV; ++i) v[i] += vp[i];
    }
    const int knext = __shfl_down_sync(FULL, key, 1);
    return (lane == 31) || (knext != key);
}

// ---------------------------------------------------------------- exact, order-independent deposits
// The contributions of a deposit to a node array are summed as 64-bit integers in units of a power-
// of-two quantum q, so the sum is the same whatever order the warps add in: every deposit, and with
// it the whole sweep, is reproducible bit for bit. q is chosen per deposit and per array from the
// largest contribution (its binary exponent: a block-wide maximum taken before the adds) and from
// the most contributions one node can receive (2^bits; every partial sum stays below 2^63 quanta).
// Relative to the largest contribution of the deposit the quantum is 2^(bits - 62): about one unit
// in the last place of FP64 for the 511 plasma particles of a slice. A non-finite contribution makes
// its array's values of that deposit NaN.
__device__ __forceinline__ int fx_bexp(double v) {         // biased exponent: 0 for 0, 2047 for Inf / NaN
    return (int)((__double_as_longlong(v) >> 52) & 0x7ff);
}
__device__ __forceinline__ int fx_qexp(int e, int bits) { return e - 1085 + bits; }   // (e - 1022) + bits - 63
// 1 / quantum (0 when every contribution is zero) and the quantum of a block maximum e
__device__ __forceinline__ double fx_scale(int e, int bits) { return e == 0 ? 0.0 : scalbn(1.0, -fx_qexp(e, bits)); }
__device__ __forceinline__ double fx_quantum(int e, int bits) { return scalbn(1.0, fx_qexp(e, bits)); }
__device__ __forceinline__ void fx_add(double* p, double v, double scale) {
    if (v != 0.0) atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double2ll_rn(v * scale));
}
// the value of an accumulator (its 64 bits as stored in the double slot p); e == 2047: a non-finite
// contribution was seen
__device__ __forceinline__ double fx_value(const double* p, int e, double quantum) {
    if (e == 2047) return __longlong_as_double(0x7ff8000000000000LL);
    return (double)__double_as_longlong(*p) * quantum;
}
// warp-wide: E[c] = max(E[c], the largest e[c] of the warp's lanes) (shared-memory block maxima)
template <int NC>
__device__ __forceinline__ void fx_max(const int (&e)[NC], int* E) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const unsigned m = __reduce_max_sync(FULL, (unsigned)e[c]);
        if ((threadIdx.x & 31) == 0 && m) atomicMax(E + c, (int)m);
    }
}
// headroom bits for n contributions per node: 2^bits > 2 n
__device__ __forceinline__ int fx_bits(int n) { return 34 - __clz(n > 1 ? n : 1); }

// ---------------------------------------------------------------- shared-memory layout
struct Src {                                              // plasma + beam sources of one slice
    double *rhot, *drho, *jz, *chi, *ne, *ni, *jpi1, *S1r, *S1i;
};

struct Smem {
    double *r, *iv, *ih;                                  // grid
    const double *gm, *g0, *gp, *ir;                      // gradient stencils, 1/r
    const double *l0r, *l0f, *l0b;                        // L0 Thomas: 1/u, -a/u, -c/u
    const double *l1a, *l1b, *l1c, *lfa, *lfb, *lfc;      // L1D and L1F rows
    double* src0;                                         // sources: 9 arrays, twice when A.dbuf
    double *bgt, *bgr;                                    // neutralising background
    double *psi, *ez, *bz, *wr1, *bpr, *bpi;              // fields of the slice (wr1 = -psi')
    double* tot;                                          // scan scratch, 2 x 8 x kW
    double* stage;                                        // A.filter: beam + background part of the next slice (4 x M)
    double* ftot;                                         // A.filter: scan scratch of the filter, 2 x 14 x kW
    int* lost;
    int* flag;                                            // gate result broadcast
    // block maxima of the deposits' exponents: [0, 7) the plasma deposit (rho - J_z, d/dxi, J_z, chi,
    // n_e, n_i, J_theta), [7, 9) the S deposit, [9, 11) the background and neutralising deposits; then
    // counters: [11] extra sub-slices, [12] particles removed as trapped, [13] non-finite deposits
    int* fx;
    unsigned long long* cmax;                             // most cells crossed (sub-slicing), as double bits
    // A.pcache > 0 (plasma in global memory, np = A.pcache): a copy of every particle's x y px py Delta w
    // (pc, 6 x np) and its radial cell (pj), written through with the global state whenever a particle
    // moves; the passes that only read the particles take them from here, without a cell search
    double* pc;
    int* pj;
};

__device__ __forceinline__ Smem carve(double* base, const SweepArgs& A) {
    const int M = A.M;
    Smem S;
    double* p = base;
    S.r = p; p += M; S.iv = p; p += M; S.ih = p; p += M;
    const double* q = A.const_smem ? p : A.consts;
    S.gm = q; S.g0 = q + M; S.gp = q + 2 * M; S.ir = q + 3 * M;
    S.l0r = q + 4 * M; S.l0f = q + 5 * M; S.l0b = q + 6 * M;
    S.l1a = q + 7 * M; S.l1b = q + 8 * M; S.l1c = q + 9 * M;
    S.lfa = q + 10 * M; S.lfb = q + 11 * M; S.lfc = q + 12 * M;
    if (A.const_smem) p += 13 * (size_t)M;
    S.src0 = p;
    p += (A.dbuf ? 18 : 9) * (size_t)M;
    S.bgt = p; p += M; S.bgr = p; p += M;
    S.psi = p; p += M; S.ez = p; p += M; S.bz = p; p += M; S.wr1 = p; p += M; S.bpr = p; p += M; S.bpi = p; p += M;
    S.tot = p; p += 2 * 8 * kW;
    S.stage = S.ftot = nullptr;
    if (A.filter) { S.stage = p; p += 4 * (size_t)M; S.ftot = p; p += 2 * 14 * kW; }
    S.lost = reinterpret_cast<int*>(p);
    S.flag = S.lost + 1;
    S.fx = S.lost + 2;
    S.cmax = reinterpret_cast<unsigned long long*>(S.lost + 16);
    S.pc = A.pcache ? reinterpret_cast<double*>(reinterpret_cast<char*>(S.lost) + 128) : nullptr;
    S.pj = A.pcache ? reinterpret_cast<int*>(S.pc + 6 * (size_t)A.pcache) : nullptr;
    return S;
}

__device__ __forceinline__ Src src_of(const Smem& S, int M, int b) {
    double* p = S.src0 + (size_t)b * 9 * M;
    Src s;
    s.rhot = p; s.drho = p + M; s.jz = p + 2 * M; s.chi = p + 3 * M; s.ne = p + 4 * M;
    s.ni = p + 5 * M; s.jpi1 = p + 6 * M; s.S1r = p + 7 * M; s.S1i = p + 8 * M;
    return s;
}

// beam source values of slice k at node j needed by the m = 0 sweep (src/Simulation.cpp:420-441):
// rho - J_z, its xi-derivative (central / one-sided, or backward for ngp), J_z, J_theta
struct BeamRow { double rt, drt, jz, jt; };

template <bool kL2>                       // kL2: the rows were written by other SMs, read them from L2
__device__ __forceinline__ double ldb(const double* p) { return kL2 ? __ldcg(p) : *p; }

// one beam-source value at p (inside bsrc): the pushed beams' deposit plus, in kernels built for it
// (kStat), the static (analytic) sources when present
template <bool kL2, bool kStat>
__device__ __forceinline__ double ldbs(const SweepArgs& A, const double* bsrc, const double* p) {
    const double v = ldb<kL2>(p);
    if constexpr (kStat) return A.bstat ? v + __ldg(A.bstat + (p - bsrc)) : v;
    return v;
}

// component c of node j of the guard row (the slice ahead of a later slab's first one): doubles, or two
// limbs (the high row, then the low row M B_NC0 values further) when bsrc has the exact format
__device__ __forceinline__ double guard_at(const SweepArgs& A, int j, int c) {
    if (!A.bguard) return 0.0;
    const double* g = A.bguard + (size_t)j * B_NC0 + c;
    return A.bq ? beam_fx_value(g[0], g[(size_t)A.M * B_NC0], A.bq[j], A.bfx_2s) : g[0];
}

template <bool kL2, bool kStat = false>
__device__ __forceinline__ BeamRow beam_row(const SweepArgs& A, const double* bsrc, int k, int j) {
    const size_t st = (size_t)A.M * B_NC0;
    const double* bk = bsrc + (size_t)k * st + (size_t)j * B_NC0;
    // one value of node j: a double, or the exact two-limb accumulator (A.bq) turned into its value
    const double qj = A.bq ? A.bq[j] : 0.0;
    auto ld = [&](const double* p) -> double {
        if (A.bq) {
            const double v = beam_fx_value(ldb<kL2>(p), ldb<kL2>(p + A.bfx_lo), qj, A.bfx_2s);
            if constexpr (kStat) return A.bstat ? v + __ldg(A.bstat + (p - bsrc)) : v;
            return v;
        }
        return ldbs<kL2, kStat>(A, bsrc, p);
    };
    BeamRow r;
    r.rt = ld(bk + B_RT0);
    r.jz = ld(bk + B_JZ0);
    r.jt = ld(bk + B_JP1I);
    const int K = A.K;
    // the slice ahead of slice 0: none at the box head, the guard row in a later slab of a staged run
    const double guard = guard_at(A, j, B_RT0);
    if (A.ngp) {
        const double prev = (k > 0) ? ld(bk + B_RT0 - (ptrdiff_t)st) : guard;
        r.drt = (r.rt - prev) * A.idxi;
    } else if (K == 1) {
        r.drt = 0.0;
    } else if (k == 0) {
        r.drt = A.bguard ? 0.5 * (ld(bk + st + B_RT0) - guard) * A.idxi : (ld(bk + st + B_RT0) - r.rt) * A.idxi;
    } else if (k == K - 1) {
        r.drt = (r.rt - ld(bk + B_RT0 - (ptrdiff_t)st)) * A.idxi;
    } else {
        r.drt = 0.5 * (ld(bk + st + B_RT0) - ld(bk + B_RT0 - (ptrdiff_t)st)) * A.idxi;
    }
    return r;
}

// initial source values of a slice: background + beam; the plasma deposit is added on top. With the
// smoothing filter (kernels built with kExt only) the plasma deposit starts from zero and the beam +
// background part is staged, to be added after the filter (filter_sources).
template <bool kExt>
__device__ __forceinline__ void init_sources(const Src& s, const Smem& S, int j, const BeamRow& br, int M) {
    if (kExt && S.stage) {
        S.stage[j] = S.bgt[j] + br.rt;
        S.stage[M + j] = br.drt;
        S.stage[2 * M + j] = br.jz;
        S.stage[3 * M + j] = br.jt;
        s.rhot[j] = 0.0;
        s.drho[j] = 0.0;
        s.jz[j] = 0.0;
        s.jpi1[j] = 0.0;
        s.ni[j] = 0.0;
    } else {
        s.rhot[j] = S.bgt[j] + br.rt;
        s.drho[j] = br.drt;
        s.jz[j] = br.jz;
        s.jpi1[j] = br.jt;
        s.ni[j] = S.bgr[j] > 0.0 ? S.bgr[j] : 0.0;
    }
    s.chi[j] = 0.0;
    s.ne[j] = 0.0;
    s.S1r[j] = 0.0;
    s.S1i[j] = 0.0;
}

// the values a slice's 7 deposit arrays start from at node j (init_sources' values, for deposits
// whose accumulators cannot hold them); with the smoothing filter the beam + background part goes to
// the stage and the arrays start from zero
template <bool kExt>
__device__ __forceinline__ void init_base(const Smem& S, int j, const BeamRow& br, int M, double (&base)[7]) {
    if (kExt && S.stage) {
        S.stage[j] = S.bgt[j] + br.rt;
        S.stage[M + j] = br.drt;
        S.stage[2 * M + j] = br.jz;
        S.stage[3 * M + j] = br.jt;
#pragma unroll
        for (int c = 0; c < 7; ++c) base[c] = 0.0;
    } else {
        base[0] = S.bgt[j] + br.rt;
        base[1] = br.drt;
        base[2] = br.jz;
        base[3] = 0.0;
        base[4] = 0.0;
        base[5] = S.bgr[j] > 0.0 ? S.bgr[j] : 0.0;
        base[6] = br.jt;
    }
}

// The radial smoothing filter f <- F_n^{-1} f (FieldSolver::filter, src/FieldSolver.cpp:148-161) of NS
// shared-memory arrays in place, each with F0 (op 0) or F1 (op 1): Thomas with the host-factored pivots
// A.fconsts, its two substitutions as block scans over the thread's rows [row0, row0 + Rw). Every thread
// reads and writes only its own rows; the caller puts a barrier before (the arrays are complete) and, when
// other threads read them next, after. Only the kernel variants for filtered decks (EXT) contain it.
template <int NS>
struct FilterSet { double* f[NS]; int op[NS]; };

template <int NS, int kMaxR>
__device__ __forceinline__ void filter_rows(const FilterSet<NS> fs, const double* __restrict__ fc, int M, int Rw,
                                         double* tot) {
    const int row0 = threadIdx.x * Rw;
    double a[NS], b[NS], d[kMaxR][NS];
#pragma unroll
    for (int e = 0; e < NS; ++e) { a[e] = 1.0; b[e] = 0.0; }
#pragma unroll
    for (int u = 0; u < kMaxR; ++u) {
        const int i = row0 + u;
#pragma unroll
        for (int e = 0; e < NS; ++e) {
            d[u][e] = 0.0;
            if (u >= Rw || i >= M) continue;
            const double* F = fc + (size_t)fs.op[e] * 3 * M;
            d[u][e] = fs.f[e][i];
            const double rr = F[i], af = F[M + i];
            b[e] = fma(af, b[e], rr * d[u][e]);
            a[e] *= af;
        }
    }
    double y[NS];
    scan_fwd_n<NS>(a, b, y, tot);
#pragma unroll
    for (int u = 0; u < kMaxR; ++u) {
        const int i = row0 + u;
#pragma unroll
        for (int e = 0; e < NS; ++e) {
            if (u >= Rw || i >= M) continue;
            const double* F = fc + (size_t)fs.op[e] * 3 * M;
            y[e] = fma(F[M + i], y[e], F[i] * d[u][e]);
            d[u][e] = y[e];
        }
    }
#pragma unroll
    for (int e = 0; e < NS; ++e) { a[e] = 1.0; b[e] = 0.0; }
#pragma unroll
    for (int u = kMaxR - 1; u >= 0; --u) {
        const int i = row0 + u;
        if (u >= Rw || i >= M) continue;
#pragma unroll
        for (int e = 0; e < NS; ++e) {
            const double ab = fc[(size_t)fs.op[e] * 3 * M + 2 * M + i];
            b[e] = fma(ab, b[e], d[u][e]);
            a[e] *= ab;
        }
    }
    double x[NS];
    scan_bwd_n<NS>(a, b, x, tot + 2 * NS * kW);
#pragma unroll
    for (int u = kMaxR - 1; u >= 0; --u) {
        const int i = row0 + u;
        if (u >= Rw || i >= M) continue;
#pragma unroll
        for (int e = 0; e < NS; ++e) {
            x[e] = fma(fc[(size_t)fs.op[e] * 3 * M + 2 * M + i], x[e], d[u][e]);
            fs.f[e][i] = x[e];
        }
    }
}

// Simulation::filter_plasma_sources (src/Simulation.cpp:823-835, m = 0) on the plasma deposit of a slice,
// then the staged beam + background part added as combine_sources does (src/Simulation.cpp:430-437):
// rho - J_z, its xi-derivative, J_z, chi, n_e, n_i with F0 and J_theta with F1. Ends with a barrier.
template <int kMaxR>
__device__ __forceinline__ void filter_sources(const Src& s, const Smem& S, const SweepArgs& A, int Rw) {
    FilterSet<7> fs;
    double* arr[7] = {s.rhot, s.drho, s.jz, s.chi, s.ne, s.ni, s.jpi1};
#pragma unroll
    for (int e = 0; e < 7; ++e) { fs.f[e] = arr[e]; fs.op[e] = e == 6 ? 1 : 0; }
    filter_rows<7, kMaxR>(fs, A.fconsts, A.M, Rw, S.ftot);
    const int M = A.M, row0 = threadIdx.x * Rw;
#pragma unroll
    for (int u = 0; u < kMaxR; ++u) {
        const int i = row0 + u;
        if (u >= Rw || i >= M) continue;
        s.rhot[i] += S.stage[i];
        s.drho[i] += S.stage[M + i];
        s.jz[i] += S.stage[2 * M + i];
        s.jpi1[i] += S.stage[3 * M + i];
        if (S.bgr[i] > 0.0) s.ni[i] += S.bgr[i];
    }
    __syncthreads();
}

// 3-point non-uniform gradient at node i (src/FieldSolver.cpp:193-211); odd: axis value f1/r1
__device__ __forceinline__ double grad_at(const Smem& S, int N, const double* f, int i, bool odd) {
    if (i == 0) return odd ? f[1] * S.ir[0] : 0.0;
    if (i == N) return S.g0[N] * f[N] + S.gm[N] * f[N - 1] + S.gp[N] * f[N - 2];
    return S.gm[i] * f[i - 1] + S.g0[i] * f[i] + S.gp[i] * f[i + 1];
}

// cell of x starting from a guess (the previous cell): walks for small moves, bisects otherwise;
// the same cell as locate() (src/RadialGrid.hpp:35-44) for every x
__device__ __forceinline__ int locate_from(const double* __restrict__ r, int N, double R, double x, int j) {
    if (x <= 0.0) return 0;
    if (x >= R) return N - 1;
    j = j < 0 ? 0 : (j > N - 1 ? N - 1 : j);
#pragma unroll 1
    for (int step = 0; step < 3; ++step) {
        if (r[j] > x) { if (j == 0) break; --j; continue; }
        if (r[j + 1] <= x) { if (j == N - 1) break; ++j; continue; }
        return j;
    }
    if (r[j] <= x && x < r[j + 1]) return j;
    return locate(r, N, R, x);
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

// x y px py Delta w of particle p: from the shared copy (A.pcache) or from the global state
template <int ORD>
__device__ __forceinline__ void pbase(PState<ORD>& P, const Smem& S, const SweepArgs& A, const double* __restrict__ ps,
                                      int npad, int p) {
    if (A.pcache) {
        const size_t n = (size_t)A.pcache;
        P.x = S.pc[p]; P.y = S.pc[n + p]; P.px = S.pc[2 * n + p]; P.py = S.pc[3 * n + p];
        P.dl = S.pc[4 * n + p]; P.w = S.pc[5 * n + p];
    } else {
        P.x = ps[p]; P.y = ps[npad + p]; P.px = ps[2 * (size_t)npad + p]; P.py = ps[3 * (size_t)npad + p];
        P.dl = ps[4 * (size_t)npad + p]; P.w = ps[5 * (size_t)npad + p];
    }
}
template <int ORD>
__device__ __forceinline__ void pbase_put(const PState<ORD>& P, const Smem& S, const SweepArgs& A, int p) {
    if (!A.pcache) return;
    const size_t n = (size_t)A.pcache;
    S.pc[p] = P.x; S.pc[n + p] = P.y; S.pc[2 * n + p] = P.px; S.pc[3 * n + p] = P.py;
    S.pc[4 * n + p] = P.dl; S.pc[5 * n + p] = P.w;
}
// AB history of particle p from the global state
template <int ORD>
__device__ __forceinline__ void phist(PState<ORD>& P, const double* __restrict__ ps, int npad, int p) {
#pragma unroll
    for (int m = 0; m < ORD; ++m)
#pragma unroll
        for (int v = 0; v < 5; ++v) P.h[m][v] = ps[(6 + (size_t)m * 5 + v) * npad + p];
}

// the geometry of particle p at (x, y): from its kept cell (A.pcache; the cell locate() would find) or by
// the search
__device__ __forceinline__ PGeo pgeo(const Smem& S, const SweepArgs& A, int N, double R, int p, double x, double y) {
    return A.pcache ? geometry_in(S.r, S.ih, x, y, S.pj[p]) : geometry(S.r, S.ih, N, R, x, y);
}

__device__ __forceinline__ void species_params(const SweepArgs& A, int p, double& q, double& qm) {
    int s = 0;
    while (s + 1 < A.nsp && p >= A.sp_off[s + 1]) ++s;
    q = A.sp_q[s];
    qm = A.sp_qm[s];
}

// W+ mode 1 at the particle: lin(w1), w1 = -psi' (src/Simulation.cpp:477-498)
__device__ __forceinline__ double w1_at(const Smem& S, int N, const PGeo& g) { return lin(S.wr1, g); }

// src/PlasmaSpecies.cpp:409-478, m = 0 (plasma rho and J_r feed nothing on this path: not deposited).
// Contributions of one particle to nodes j (v[0..5]) and j+1 (v[6..11]): rho - J_z, d/dxi, J_z, chi,
// density, J_theta.
template <int ORD>
__device__ __forceinline__ void deposit_values(const PState<ORD>& P, const PGeo& g, const Smem& S, double (&v)[12]) {
    const double PX = P.px, PY = P.py, D = P.dl, w = P.w;
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D;
    const double pz = gam - D;
    const double ux = PX * invd, uy = PY * invd;
    const double ur = g.c * ux + g.s * uy, uth = g.c * uy - g.s * ux;
    const double wq = w * P.q;
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
        v[6 * cc + 0] = a;
        v[6 * cc + 1] = dr;
        v[6 * cc + 2] = vjz;
        v[6 * cc + 3] = vchi;
        v[6 * cc + 4] = vn;
        v[6 * cc + 5] = a * uth;
    }
}

// The plasma deposit of a slice, exact (see fx_add): phase A sums each warp's runs of equal
// (cell, species sign) and takes the block maxima of the run sums' exponents; after a barrier phase B
// adds the quantised run sums into the accumulator arrays; after another barrier deposit_finish turns
// the accumulators into values. The 7 arrays in this order: rho - J_z, d/dxi, J_z, chi, n_e, n_i,
// J_theta (n_e takes the negative species, n_i the positive ones).
__device__ __forceinline__ double* dep_arr(const Src& s, int c) {
    switch (c) {
        case 0: return s.rhot;
        case 1: return s.drho;
        case 2: return s.jz;
        case 3: return s.chi;
        case 4: return s.ne;
        case 5: return s.ni;
        default: return s.jpi1;
    }
}

// warp-wide phase A: every lane calls it (active = the lane has a particle); key = 2 j + (positive
// species). Returns whether the lane holds a run sum to add; kExp: also take the exponent maxima
// into E (a deposit that recomputes its values for phase B calls it again without)
template <bool kExp>
__device__ __forceinline__ bool deposit_runs(bool active, int j, bool neg, double (&v)[12], int* E) {
    const int lane = threadIdx.x & 31;
    if (!active)
#pragma unroll
        for (int i = 0; i < 12; ++i) v[i] = 0.0;
    const int key = active ? 2 * j + (neg ? 0 : 1) : -1 - lane;
    const bool tail = warp_runs_sum<12>(key, v) && active;
    if constexpr (kExp) {
        int e[7] = {0, 0, 0, 0, 0, 0, 0};
        if (tail) {
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                const int ec = max(fx_bexp(v[c]), fx_bexp(v[6 + c]));
                if (c < 4) e[c] = ec;
                else if (c == 4) e[neg ? 4 : 5] = ec;
                else e[6] = ec;
            }
        }
        fx_max<7>(e, E);
    }
    return tail;
}

// phase B: the run sum of a tail lane into the accumulators of nodes j and j + 1
__device__ __forceinline__ void deposit_add(bool tail, int j, bool neg, const double (&v)[12], const Src& acc,
                                            const int* E, int bits) {
    if (!tail) return;
    const double s0 = fx_scale(E[0], bits), s1 = fx_scale(E[1], bits), s2 = fx_scale(E[2], bits);
    const double s3 = fx_scale(E[3], bits), s4 = fx_scale(E[neg ? 4 : 5], bits), s6 = fx_scale(E[6], bits);
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        const int jj = j + cc;
        fx_add(acc.rhot + jj, v[6 * cc + 0], s0);
        fx_add(acc.drho + jj, v[6 * cc + 1], s1);
        fx_add(acc.jz + jj, v[6 * cc + 2], s2);
        fx_add(acc.chi + jj, v[6 * cc + 3], s3);
        fx_add((neg ? acc.ne : acc.ni) + jj, v[6 * cc + 4], s4);
        fx_add(acc.jpi1 + jj, v[6 * cc + 5], s6);
    }
}

// the values of node j: dst = base + accumulated deposit (acc and dst may be the same arrays)
__device__ __forceinline__ void deposit_finish(const Src& dst, const Src& acc, int j, const double (&base)[7],
                                               const int* E, int bits) {
#pragma unroll
    for (int c = 0; c < 7; ++c)
        dep_arr(dst, c)[j] = base[c] + fx_value(dep_arr(acc, c) + j, E[c], fx_quantum(E[c], bits));
}

// src/PlasmaSpecies.cpp:508-559, m = 0: S+ contributions to nodes j (v[0..1]) and j+1 (v[2..3])
template <int ORD>
__device__ __forceinline__ void depositS_values(const PState<ORD>& P, const PGeo& g, const Smem& S, int N,
                                                double (&v)[4]) {
    const double qm = P.qm;
    const double PX = P.px, PY = P.py, D = P.dl;
    const double r1 = w1_at(S, N, g);
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
        v[2 * cc] = iv * (Ar * g.c + Ai * g.s);
        v[2 * cc + 1] = iv * (Ai * g.c - Ar * g.s);
    }
}

// the S deposit of a slice, exact like the plasma deposit: phase A (run sums, exponent maxima into
// E[0..1] for S_r, S_i), phase B after a barrier (adds into the slice's S arrays, which start at 0),
// then each thread turns its own rows into values (depositS_finish) before the B+ solve reads them
template <bool kExp>
__device__ __forceinline__ bool depositS_runs(bool active, int j, double (&v)[4], int* E) {
    const int lane = threadIdx.x & 31;
    if (!active)
#pragma unroll
        for (int i = 0; i < 4; ++i) v[i] = 0.0;
    const int key = active ? j : -1 - lane;
    const bool tail = warp_runs_sum<4>(key, v) && active;
    if constexpr (kExp) {
        int e[2] = {0, 0};
        if (tail) {
            e[0] = max(fx_bexp(v[0]), fx_bexp(v[2]));
            e[1] = max(fx_bexp(v[1]), fx_bexp(v[3]));
        }
        fx_max<2>(e, E);
    }
    return tail;
}

__device__ __forceinline__ void depositS_add(bool tail, int j, const double (&v)[4], const Src& s, const int* E,
                                             int bits) {
    if (!tail) return;
    const double sr = fx_scale(E[0], bits), si = fx_scale(E[1], bits);
    fx_add(s.S1r + j, v[0], sr);
    fx_add(s.S1i + j, v[1], si);
    fx_add(s.S1r + j + 1, v[2], sr);
    fx_add(s.S1i + j + 1, v[3], si);
}

__device__ __forceinline__ void depositS_finish(const Src& s, int i, const int* E, int bits) {
    s.S1r[i] = fx_value(s.S1r + i, E[0], fx_quantum(E[0], bits));
    s.S1i[i] = fx_value(s.S1i + i, E[1], fx_quantum(E[1], bits));
}

// src/PlasmaSpecies.cpp:561-668 with uniform steps (the classical AB coefficients); returns 1 when the
// particle moved, 0 when it was removed beyond the wall, -1 when removed as trapped (Delta <= delta_min
// or gamma > max_qsa Delta: no longer quasi-static, src/PlasmaSpecies.cpp:636-650)
template <int ORD>
__device__ __forceinline__ int push_particle(PState<ORD>& P, const PGeo& g, const Smem& S, const SweepArgs& A,
                                              bool first, const double (&ab)[5], double h) {
    const double qm = P.qm;
    const double X = P.x, Y = P.y, PX = P.px, PY = P.py, D = P.dl;
    const double r1 = w1_at(S, A.N, g);
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
        const double cm = ab[m];
#pragma unroll
        for (int v = 0; v < 5; ++v) sum[v] += cm * P.h[m][v];
    }
    const double dxi = h;
    double xn = X + dxi * sum[0], yn = Y + dxi * sum[1];
    double pxn = PX + dxi * sum[2], pyn = PY + dxi * sum[3];
    const double dn = D + dxi * sum[4];
    const double gn = (1.0 + pxn * pxn + pyn * pyn + dn * dn) / (2.0 * dn);
    if (!(dn > A.delta_min) || gn > A.max_qsa * dn) {
        P.w = 0.0;
        return -1;
    }
    const double R = A.R;
    const double rn = sqrt(xn * xn + yn * yn);
    if (rn > R) {                    // specular reflection at the wall, incl. the history
        const double nx = xn / rn, ny = yn / rn;
        const double rr = 2.0 * R - rn;
        if (rr < 0.0) { P.w = 0.0; return 0; }
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
    return 1;
}

// Adams-Bashforth coefficients for history points t[0..ord) (t[0] the newest push) and the step h: the
// integrals over [t0, t0 + h] of the Lagrange basis, by 3-point Gauss-Legendre (exact for the degree <= 4
// needed), src/PlasmaSpecies.cpp:30-48
template <int ORD>
__device__ __forceinline__ void ab_variable(const double (&t)[ORD], double h, double (&c)[5]) {
    const double gx[3] = {-0.7745966692414834, 0.0, 0.7745966692414834};
    const double gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
#pragma unroll
    for (int m = 0; m < 5; ++m) c[m] = 0.0;
#pragma unroll
    for (int m = 0; m < ORD; ++m) {
        double sm = 0.0;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double tt = t[0] + 0.5 * h * (1.0 + gx[q]);
            double l = 1.0;
#pragma unroll
            for (int n = 0; n < ORD; ++n)
                if (n != m) l *= (tt - t[n]) / (t[m] - t[n]);
            sm += 0.5 * gw[q] * l;
        }
        c[m] = sm;
    }
}

// the radial cells a particle would cross in a step of dxi: its straight path's length over the cell
// size at the path's closest approach to the axis (src/PlasmaSpecies.cpp:814-830)
__device__ __forceinline__ double cells_crossed(const Smem& S, int N, double R, double X, double Y, double PX,
                                                double PY, double D, double dxi) {
    const double X1 = X + dxi * PX / D, Y1 = Y + dxi * PY / D;
    const double dx = X1 - X, dy = Y1 - Y, l2 = dx * dx + dy * dy;
    double t = l2 > 0.0 ? -(X * dx + Y * dy) / l2 : 0.0;
    t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
    const double xm = X + t * dx, ym = Y + t * dy;
    return sqrt(l2) * S.ih[locate(S.r, N, R, sqrt(xm * xm + ym * ym))];
}

// the beam sources of a sub-slice at xi_k + ds: slice k's, extrapolated linearly with their xi-derivative
// (src/Simulation.cpp:431-432); the derivative of rho - J_z itself is slice k's
template <bool kL2, bool kStat>
__device__ __forceinline__ BeamRow beam_row_at(const SweepArgs& A, const double* bsrc, int k, int j, double ds) {
    BeamRow r = beam_row<kL2, kStat>(A, bsrc, k, j);
    if (ds == 0.0) return r;
    // the xi-derivatives of J_z and J_theta by the same difference as that of rho - J_z
    const int K = A.K;
    auto row = [&](int kk) { return beam_row<kL2, kStat>(A, bsrc, kk, j); };
    double djz = 0.0, djt = 0.0;
    if (A.ngp) {
        const BeamRow p = k > 0 ? row(k - 1) : BeamRow{0.0, 0.0, guard_at(A, j, B_JZ0), guard_at(A, j, B_JP1I)};
        djz = (r.jz - p.jz) * A.idxi;
        djt = (r.jt - p.jt) * A.idxi;
    } else if (K > 1) {
        const BeamRow a = k == 0 ? r : row(k - 1), b = k == K - 1 ? r : row(k + 1);
        const double f = (k == 0 || k == K - 1) ? 1.0 : 0.5;
        djz = f * (b.jz - a.jz) * A.idxi;
        djt = f * (b.jt - a.jt) * A.idxi;
    }
    r.rt += ds * r.drt;
    r.jz += ds * djz;
    r.jt += ds * djt;
    return r;
}

// right-hand sides of the psi, E_z, B_z systems at row i (src/Simulation.cpp:798-799, :517-527)
__device__ __forceinline__ void rhs_l0(const Smem& S, const Src& s, int N, int i, double& d0, double& d1,
                                       double& d2) {
    d0 = d1 = d2 = 0.0;
    if (i < N) {
        d0 = -1.0 * s.rhot[i];
        d1 = -1.0 * s.drho[i];
        const double t1 = grad_at(S, N, s.jpi1, i, true);
        const double t2 = (i == 0 ? s.jpi1[1] : s.jpi1[i]) * S.ir[i];
        d2 = 1.0 * (-(t1 + t2));
    }
}

// row i of (L1D - chi) (sys 0) and (L1F - chi) (sys 1) with its right-hand side
// (src/FieldSolver.cpp:172-191, src/Simulation.cpp:535-591)
__device__ __forceinline__ void row_b(const Smem& S, const Src& s, int N, double fc, int sys, int i, double& a,
                                      double& b, double& cm, double& d) {
    if (sys == 0) {
        a = S.l1a[i]; b = S.l1b[i]; cm = i > 0 ? S.l1c[i - 1] : 0.0;
        if (i >= 1 && i < N) { b = b - s.chi[i]; d = 1.0 * (-s.S1i[i]); } else { d = 0.0; }
    } else {
        a = S.lfa[i]; b = S.lfb[i]; cm = i > 0 ? S.lfc[i - 1] : 0.0;
        if (i >= 1) {
            b = b - s.chi[i];
            d = 1.0 * (grad_at(S, N, s.jz, i, false) + s.S1r[i]);
            if (i == N) d -= fc * s.jz[N];
        } else {
            d = 0.0;
        }
    }
}

}  // namespace sweep_detail

using namespace sweep_detail;

// One sweep by the calling CTA (all kThreads threads). The gate G orders it against other CTAs when
// several time steps run concurrently (NoGate: a stand-alone sweep). Returns false if a gate wait
// gave up (the CTA then stops at the next slice boundary). EXT: the kernel also handles the smoothing
// filter (A.filter) and static beam sources (A.bstat); without it both are ignored, and the kernel of
// plain decks carries none of their code.
template <int ORD, bool REG, int kMaxR, class Gate, bool EXT = false>
__device__ __forceinline__ bool sweep_body(const SweepArgs& A, double* smem_raw, Gate& gate) {
    const int M = A.M, N = A.N, K = A.K, Rw = kMaxR == 1 ? 1 : A.rows_per_thread;   // rows per thread
    const int tid = threadIdx.x;
    const Smem S = carve(smem_raw, A);
    const int np = A.np, npad = A.npad;
    const double R = A.R;
    const int row0 = tid * Rw;                                  // this thread's rows [row0, row0 + Rw)
    unsigned long long* tim = A.timing;
    long long t_prev = 0, t_sub = 0;
    if (tim && tid == 0) t_prev = clock64();
#define PHASE_MARK(ph)                                                        \
    do {                                                                      \
        if (tim && tid == 0) {                                                \
            const long long tn = clock64();                                   \
            atomicAdd(tim + (ph), (unsigned long long)(tn - t_prev));         \
            t_prev = tn;                                                      \
        }                                                                     \
    } while (0)
#define SUB_MARK(slot)                                                        \
    do {                                                                      \
        if (tim && tid == 0) {                                                \
            const long long tn = clock64();                                   \
            atomicAdd(tim + (slot), (unsigned long long)(tn - t_sub));        \
            t_sub = tn;                                                       \
        }                                                                     \
    } while (0)

    // ---------------- prologue: grid, operators, fresh plasma, background (src/Simulation.cpp:653-708)
    for (int j = tid; j < M; j += kThreads) {
        S.r[j] = A.r[j];
        S.iv[j] = A.inv_V[j];
        S.ih[j] = (j < N) ? A.inv_h[j] : 0.0;
        S.bgt[j] = 0.0;
        S.bgr[j] = 0.0;
        S.bpr[j] = 0.0;
        S.bpi[j] = 0.0;
        src_of(S, M, 0).ne[j] = 0.0;
    }
    if (A.const_smem)
        for (int t = tid; t < 13 * M; t += kThreads) const_cast<double*>(S.gm)[t] = A.consts[t];
    if (tid == 0) *S.lost = 0;
    if (tid < 14) S.fx[tid] = 0;
    const int bits_p = fx_bits(np), bits_bg = fx_bits(A.nbg);
    PState<ORD> P;
    int J = 0;                                             // cell of the thread's particle
    if (REG) {
        if (tid < np) {
            if (A.pin) {                                  // a later slab: the plasma handed on, with its history
                pload(P, A.pin, npad, tid);
            } else {
                P.x = A.p_init[tid]; P.y = A.p_init[npad + tid]; P.px = A.p_init[2 * npad + tid];
                P.py = A.p_init[3 * npad + tid]; P.dl = A.p_init[4 * npad + tid]; P.w = A.p_init[5 * npad + tid];
#pragma unroll
                for (int m = 0; m < ORD; ++m)
#pragma unroll
                    for (int v = 0; v < 5; ++v) P.h[m][v] = 0.0;
            }
            species_params(A, tid, P.q, P.qm);
        } else {
            P.x = P.y = P.px = P.py = 0.0;
            P.dl = 1.0;
            P.w = 0.0;
            P.q = P.qm = -1.0;
#pragma unroll
            for (int m = 0; m < ORD; ++m)
#pragma unroll
                for (int v = 0; v < 5; ++v) P.h[m][v] = 0.0;
        }
    } else {
        for (int p = tid; p < np; p += kThreads) {
            if (A.pin) {
                for (int v = 0; v < 6 + 5 * ORD; ++v) gate.ps(A)[(size_t)v * npad + p] = A.pin[(size_t)v * npad + p];
            } else {
#pragma unroll
                for (int v = 0; v < 6; ++v) gate.ps(A)[(size_t)v * npad + p] = A.p_init[(size_t)v * npad + p];
                for (int v = 0; v < 5 * ORD; ++v) gate.ps(A)[(size_t)(6 + v) * npad + p] = 0.0;
            }
            if (A.pcache) {
                const double* src = A.pin ? A.pin : A.p_init;
#pragma unroll
                for (int v = 0; v < 6; ++v) S.pc[(size_t)v * A.pcache + p] = src[(size_t)v * npad + p];
            }
        }
    }
    __syncthreads();
    // immobile species deposit into the background; mobile ones are subtracted (neutralisation,
    // src/Simulation.cpp:672-684); src[0].ne is the scratch of the mobile deposit. Both exact: a pass
    // for the exponent maxima, a barrier, a pass of quantised adds, a barrier, then the values.
    double* const ne0 = src_of(S, M, 0).ne;
    for (int pass = 0; pass < 2; ++pass) {
        int ebg = 0, ene = 0;
        for (int p = tid; p < A.nbg; p += kThreads) {
            const double x = A.bg_p[p], y = A.bg_p[A.nbg + p], wq = A.bg_p[2 * A.nbg + p];
            if (wq == 0.0) continue;
            const PGeo g = geometry(S.r, S.ih, N, R, x, y);
            const double a0 = wq * g.W0 * S.iv[g.j], a1 = wq * g.W1 * S.iv[g.j + 1];
            if (pass == 0) {
                ebg = max(ebg, max(fx_bexp(a0), fx_bexp(a1)));
            } else {
                const double sc = fx_scale(S.fx[9], bits_bg);
                fx_add(S.bgt + g.j, a0, sc);
                fx_add(S.bgr + g.j, a0, sc);
                fx_add(S.bgt + g.j + 1, a1, sc);
                fx_add(S.bgr + g.j + 1, a1, sc);
            }
        }
        if (A.neutralize)
            for (int p = tid; p < np; p += kThreads) {
                const double w = A.p_init[5 * (size_t)npad + p];
                if (w == 0.0) continue;
                double q, qm;
                species_params(A, p, q, qm);
                const PGeo g = geometry(S.r, S.ih, N, R, A.p_init[p], A.p_init[npad + p]);
                const double a0 = w * q * g.W0 * S.iv[g.j], a1 = w * q * g.W1 * S.iv[g.j + 1];
                if (pass == 0) {
                    ene = max(ene, max(fx_bexp(a0), fx_bexp(a1)));
                } else {
                    const double sc = fx_scale(S.fx[10], bits_p);
                    fx_add(ne0 + g.j, a0, sc);
                    fx_add(ne0 + g.j + 1, a1, sc);
                }
            }
        if (pass == 0) {
            const int e2[2] = {ebg, ene};
            fx_max<2>(e2, S.fx + 9);
        }
        __syncthreads();
    }
    for (int j = tid; j < M; j += kThreads) {
        const double qb = fx_quantum(S.fx[9], bits_bg), qn = fx_quantum(S.fx[10], bits_p);
        S.bgt[j] = fx_value(S.bgt + j, S.fx[9], qb);
        S.bgr[j] = fx_value(S.bgr + j, S.fx[9], qb);
        ne0[j] = fx_value(ne0 + j, S.fx[10], qn);
    }
    if (Gate::kActive && tid < 32) {                     // warp 0 checks the beam-source rows
        const bool ok = gate.before_rows(K - 1 < 2 ? K - 1 : 2);
        if (tid == 0) *S.flag = ok ? 1 : 0;
    }
    __syncthreads();
    if (Gate::kActive && !*S.flag) return false;
    if (EXT && A.filter) {              // the background is smoothed like the plasma (src/Simulation.cpp:685-690)
        if (A.neutralize)
            for (int j = tid; j < M; j += kThreads) {
                S.bgt[j] -= ne0[j];
                S.bgr[j] -= ne0[j];
            }
        __syncthreads();
        FilterSet<2> fb;
        fb.f[0] = S.bgt; fb.f[1] = S.bgr; fb.op[0] = fb.op[1] = 0;
        filter_rows<2, kMaxR>(fb, A.fconsts, M, Rw, S.ftot);
        __syncthreads();
    } else if (A.neutralize) {
        for (int j = tid; j < M; j += kThreads) {
            S.bgt[j] -= ne0[j];
            S.bgr[j] -= ne0[j];
        }
    }
    // slice 0's arrays accumulate its plasma deposit from zero; its start values (background + beam,
    // init_base) are added when the deposit is finished
    {
        const Src s0 = src_of(S, M, 0);
        for (int j = tid; j < M; j += kThreads) {
#pragma unroll
            for (int c = 0; c < 7; ++c) dep_arr(s0, c)[j] = 0.0;
            s0.S1r[j] = 0.0;
            s0.S1i[j] = 0.0;
        }
    }
    __syncthreads();
    // deposit of slice 0
    const int lane = tid & 31;
    {
        const Src s0 = src_of(S, M, 0);
        if (REG) {
            const bool act = tid < np && P.w != 0.0;
            double v[12];
            if (act) {
                const PGeo G = geometry(S.r, S.ih, N, R, P.x, P.y);
                J = G.j;
                deposit_values(P, G, S, v);
            }
            const bool tail = deposit_runs<true>(act, J, P.q < 0.0, v, S.fx);
            __syncthreads();
            deposit_add(tail, J, P.q < 0.0, v, s0, S.fx, bits_p);
        } else {
            for (int pass = 0; pass < 2; ++pass) {
                if (pass == 1) __syncthreads();
                for (int base = tid - lane; base < np; base += kThreads) {
                    const int p = base + lane;
                    PState<ORD> Q;
                    bool act = false;
                    int j = 0;
                    double v[12];
                    if (p < np) {
                        pbase(Q, S, A, gate.ps(A), npad, p);
                        species_params(A, p, Q.q, Q.qm);
                        act = Q.w != 0.0;
                        if (act) {
                            // the first pass searches the cell and keeps it for the later passes
                            const PGeo g = pass == 0 ? geometry(S.r, S.ih, N, R, Q.x, Q.y)
                                                     : pgeo(S, A, N, R, p, Q.x, Q.y);
                            if (pass == 0 && A.pcache) S.pj[p] = g.j;
                            j = g.j;
                            deposit_values(Q, g, S, v);
                        }
                    }
                    const bool neg = act && Q.q < 0.0;
                    if (pass == 0) {
                        deposit_runs<true>(act, j, neg, v, S.fx);
                    } else {
                        const bool tail = deposit_runs<false>(act, j, neg, v, S.fx);
                        deposit_add(tail, j, neg, v, s0, S.fx, bits_p);
                    }
                }
            }
        }
        __syncthreads();
        if (tid == 0)
            for (int c = 0; c < 7; ++c) S.fx[13] += (S.fx[c] == 2047) + (c < 2 && S.fx[9 + c] == 2047);
        for (int j = tid; j < M; j += kThreads) {
            double b0[7];
            init_base<EXT>(S, j, beam_row<Gate::kActive, EXT>(A, gate.bsrc(A), 0, j), M, b0);
            deposit_finish(s0, s0, j, b0, S.fx, bits_p);
        }
    }
    __syncthreads();
    PHASE_MARK(0);

    int scan_par = 0;                                            // alternates the scan scratch
    const double fc = A.flux_coef;
    // The xi positions of the last ORD pushes (tn[0] the newest; the same in every thread) give the
    // Adams-Bashforth coefficients of the next push: the classical ones for uniform steps, the
    // variable-step ones after adaptive sub-slicing (src/PlasmaSpecies.cpp:561-580). A slab whose plasma
    // was pushed before continues uniform steps of dxi.
    double xcur = 0.0, hlast = A.pin_pushed ? A.dxi : 0.0, tn[ORD], abc[5];
#pragma unroll
    for (int m = 0; m < ORD; ++m) tn[m] = -(m + 1) * A.dxi;
    auto coeffs = [&](double h, bool first) {
        if (first) {
#pragma unroll
            for (int m = 0; m < ORD; ++m) tn[m] = xcur - m * h;
        } else {
#pragma unroll
            for (int m = ORD - 1; m > 0; --m) tn[m] = tn[m - 1];
            tn[0] = xcur;
        }
        bool uniform = true;
#pragma unroll
        for (int m = 1; m < ORD; ++m) uniform = uniform && fabs((tn[m - 1] - tn[m]) - h) <= 1e-9 * h;
        if (uniform) {
#pragma unroll
            for (int m = 0; m < 5; ++m) abc[m] = A.ab[m];
        } else {
            ab_variable<ORD>(tn, h, abc);
        }
        xcur += h;
        hlast = h;
    };
    for (int k = 0; k < K; ++k) {
    // the passes of slice k: its own, then its sub-slices (adaptive sub-slicing, src/Simulation.cpp:755-781):
    // each pushes by dxi / nsub; a sub-slice re-deposits the plasma and re-solves the fields with the beam
    // sources extrapolated from slice k; only the slice itself is stored
    int nsub = 1;
    for (int ss = 0; ss < nsub; ++ss) {
        // the plasma state at the start of slice k (every slice, or the checkpoint slices)
        const int tevery = A.traj_every > 1 ? A.traj_every : 1;
        if (double* const trj = ss == 0 && k % tevery == 0 ? gate.traj(A) : nullptr) {
            double* T = trj + (size_t)(k / tevery) * (6 + 5 * (size_t)ORD) * npad;
            if (REG) {
                if (tid < np) {
                    T[tid] = P.x; T[npad + tid] = P.y; T[2 * (size_t)npad + tid] = P.px;
                    T[3 * (size_t)npad + tid] = P.py; T[4 * (size_t)npad + tid] = P.dl;
                    T[5 * (size_t)npad + tid] = P.w;
#pragma unroll
                    for (int m = 0; m < ORD; ++m)
#pragma unroll
                        for (int v = 0; v < 5; ++v) T[(6 + (size_t)m * 5 + v) * npad + tid] = P.h[m][v];
                }
            } else {
                for (int p = tid; p < np; p += kThreads)
                    for (int v = 0; v < 6 + 5 * ORD; ++v) T[(size_t)v * npad + p] = gate.ps(A)[(size_t)v * npad + p];
            }
        }
        const Src s = src_of(S, M, A.dbuf ? (k & 1) : 0);
        const Src sn = src_of(S, M, A.dbuf ? ((k + 1) & 1) : 0);
        if constexpr (EXT)
            if (A.filter) filter_sources<kMaxR>(s, S, A, Rw);
        if (tim && tid == 0) t_sub = clock64();
        // beam rows of slice k+1 for this thread's nodes (consumed below, latency overlaps the solves)
        BeamRow pre[kMaxR];
        if (A.dbuf && k + 1 < K && ss == 0)
#pragma unroll
            for (int u = 0; u < kMaxR; ++u)
                if (u < Rw && row0 + u < M) pre[u] = beam_row<Gate::kActive, EXT>(A, gate.bsrc(A), k + 1, row0 + u);

        // ---------------- P2: psi, E_z, B_z with L0 (src/Simulation.cpp:797-807, :501-532)
        {
            // forward: y_i = (-a_i/u_i) y_{i-1} + d_i/u_i
            double cA = 1.0, cB[3] = {0.0, 0.0, 0.0};
            double dv[kMaxR][3];
#pragma unroll
            for (int u = 0; u < kMaxR; ++u) {
                const int i = row0 + u;
                dv[u][0] = dv[u][1] = dv[u][2] = 0.0;
                if (u >= Rw || i >= M) continue;
                rhs_l0(S, s, N, i, dv[u][0], dv[u][1], dv[u][2]);
                const double rr = S.l0r[i], af = S.l0f[i];
#pragma unroll
                for (int e = 0; e < 3; ++e) cB[e] = fma(af, cB[e], rr * dv[u][e]);
                cA *= af;
            }
            SUB_MARK(5);
            double yb[3];
            scan_fwd<3>(cA, cB, yb, S.tot + (scan_par++ & 1) * 8 * kW);
            SUB_MARK(6);
            const double ypsi_prev = yb[0];                         // y of psi just before this thread's rows
            double y[kMaxR][3];
#pragma unroll
            for (int u = 0; u < kMaxR; ++u) {
                const int i = row0 + u;
                y[u][0] = y[u][1] = y[u][2] = 0.0;
                if (u >= Rw || i >= M) continue;
                const double rr = S.l0r[i], af = S.l0f[i];
#pragma unroll
                for (int e = 0; e < 3; ++e) { yb[e] = fma(af, yb[e], rr * dv[u][e]); y[u][e] = yb[e]; }
            }
            // backward: x_i = (-c_i/u_i) x_{i+1} + y_i
            double bA = 1.0, bB[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int u = kMaxR - 1; u >= 0; --u) {
                const int i = row0 + u;
                if (u >= Rw || i >= M) continue;
                const double ab = S.l0b[i];
#pragma unroll
                for (int e = 0; e < 3; ++e) bB[e] = fma(ab, bB[e], y[u][e]);
                bA *= ab;
            }
            double xa[3];
            scan_bwd<3>(bA, bB, xa, S.tot + (scan_par++ & 1) * 8 * kW);
            SUB_MARK(7);
            // psi on the window [row0 - 1, row0 + Rw]: the rows of this thread, x after them (the
            // backward carry) and x before them, x_{row0-1} = y_{row0-1} - (c/u)_{row0-1} x_{row0}
            // with y_{row0-1} the forward carry -- so W+ = -psi' needs no further exchange
            double pw[kMaxR + 2];
            pw[kMaxR + 1] = 0.0;
            {
                double xr = xa[0];
#pragma unroll
                for (int u = kMaxR; u >= 1; --u) pw[u] = 0.0;
                const int last = (row0 + Rw <= M ? Rw : M - row0);
                if (last >= 0) pw[last + 1 > kMaxR + 1 ? kMaxR + 1 : last + 1] = xr;
            }
#pragma unroll
            for (int u = kMaxR - 1; u >= 0; --u) {
                const int i = row0 + u;
                if (u >= Rw || i >= M) continue;
                const double ab = S.l0b[i];
#pragma unroll
                for (int e = 0; e < 3; ++e) xa[e] = fma(ab, xa[e], y[u][e]);
                S.psi[i] = xa[0];
                S.ez[i] = xa[1];
                S.bz[i] = xa[2];
                pw[u + 1] = xa[0];
            }
            pw[0] = (row0 >= 1 && row0 < M) ? fma(S.l0b[row0 - 1], pw[1], ypsi_prev) : 0.0;
#pragma unroll
            for (int u = 0; u < kMaxR; ++u) {
                const int i = row0 + u;
                if (u >= Rw || i >= M) continue;
                if (i == 0) {
                    S.wr1[0] = -0.0;
                } else if (i < N) {
                    S.wr1[i] = -(S.gm[i] * pw[u] + S.g0[i] * pw[u + 1] + S.gp[i] * pw[u + 2]);
                }
                if (i == N - 1) {                                  // the one-sided wall stencil needs psi_{N-2..N}
                    S.wr1[N] = -(S.g0[N] * pw[u + 2] + S.gm[N] * pw[u + 1] + S.gp[N] * pw[u]);
                }
            }
            if (A.dbuf && k + 1 < K && ss == 0)
#pragma unroll
                for (int u = 0; u < kMaxR; ++u)
                    if (u < Rw && row0 + u < M) init_sources<EXT>(sn, S, row0 + u, pre[u], M);
            SUB_MARK(8);
        }
        __syncthreads();
        PHASE_MARK(1);

        // ---------------- P3: S+ (src/PlasmaSpecies.cpp:508-559), exact
        if (tid < 7) S.fx[tid] = 0;           // the plasma deposit's maxima (read last before P2's barrier)
        if (tid == 7) *S.cmax = 0ull;         // the cells-crossed maximum (read last at the last P5)
        if (REG) {
            const bool act = tid < np && P.w != 0.0;
            double v[4];
            if (act) depositS_values(P, geometry_in(S.r, S.ih, P.x, P.y, J), S, N, v);
            const bool tail = depositS_runs<true>(act, J, v, S.fx + 7);
            __syncthreads();
            depositS_add(tail, J, v, s, S.fx + 7, bits_p);
        } else {
            for (int pass = 0; pass < 2; ++pass) {
                if (pass == 1) __syncthreads();
                for (int base = tid - lane; base < np; base += kThreads) {
                    const int p = base + lane;
                    bool act = false;
                    int j = 0;
                    double v[4];
                    if (p < np) {
                        PState<ORD> Q;
                        pbase(Q, S, A, gate.ps(A), npad, p);
                        species_params(A, p, Q.q, Q.qm);
                        act = Q.w != 0.0;
                        if (act) {
                            const PGeo g = pgeo(S, A, N, R, p, Q.x, Q.y);
                            j = g.j;
                            depositS_values(Q, g, S, N, v);
                        }
                    }
                    if (pass == 0) {
                        depositS_runs<true>(act, j, v, S.fx + 7);
                    } else {
                        const bool tail = depositS_runs<false>(act, j, v, S.fx + 7);
                        depositS_add(tail, j, v, s, S.fx + 7, bits_p);
                    }
                }
            }
        }
        __syncthreads();
        PHASE_MARK(2);
        // this thread's rows of S+ into values: the only rows its B+ rows (and the filter) read
        if (tid == 0) S.fx[13] += (S.fx[7] == 2047) + (S.fx[8] == 2047);
#pragma unroll
        for (int u = 0; u < kMaxR; ++u)
            if (u < Rw && row0 + u < M) depositS_finish(s, row0 + u, S.fx + 7, bits_p);

        // ---------------- P4: B+ (src/Simulation.cpp:535-591, m = 0: one pass)
        //   (L1D - chi) B_r0 = -S_i (rows 0, N Dirichlet); (L1F - chi) B_theta0 = J_z' + S_r, flux wall J_z(R)
        if (EXT && A.filter) {              // S+ smoothed with F1 (src/Simulation.cpp:810-812): the rows of
            FilterSet<2> fsS;               // this thread, which are the only ones its B+ rows read
            fsS.f[0] = s.S1r; fsS.f[1] = s.S1i; fsS.op[0] = fsS.op[1] = 1;
            filter_rows<2, kMaxR>(fsS, A.fconsts, M, Rw, S.ftot);
        }
        {
            // pivots: product of T_i = [[b_i, -a_i c_{i-1}], [1, 0]] over the thread's rows
            double m[2][4];
#pragma unroll
            for (int sy = 0; sy < 2; ++sy) { m[sy][0] = 1.0; m[sy][1] = 0.0; m[sy][2] = 0.0; m[sy][3] = 1.0; }
            double ra[kMaxR][2], rb[kMaxR][2], rc[kMaxR][2], rd[kMaxR][2];
#pragma unroll
            for (int u = 0; u < kMaxR; ++u) {
                const int i = row0 + u;
#pragma unroll
                for (int sy = 0; sy < 2; ++sy) {
                    ra[u][sy] = 0.0; rb[u][sy] = 1.0; rc[u][sy] = 0.0; rd[u][sy] = 0.0;
                    if (u >= Rw || i >= M) continue;
                    row_b(S, s, N, fc, sy, i, ra[u][sy], rb[u][sy], rc[u][sy], rd[u][sy]);
                    const double t01 = -ra[u][sy] * rc[u][sy];
                    const double n00 = rb[u][sy] * m[sy][0] + t01 * m[sy][2];
                    const double n01 = rb[u][sy] * m[sy][1] + t01 * m[sy][3];
                    m[sy][2] = m[sy][0]; m[sy][3] = m[sy][1];
                    m[sy][0] = n00; m[sy][1] = n01;
                    renorm(m[sy][0], m[sy][1], m[sy][2], m[sy][3]);
                }
            }
            double pp[2], qq[2];
            scan_pivots<2>(m, pp, qq, S.tot + (scan_par++ & 1) * 8 * kW);
            // this thread's pivots (rc holds c_{i-1}; rinv = 1/u_i = p_{i-1}/p_i), forward composites
            double rinv[kMaxR][2];
            double fA[2] = {1.0, 1.0}, fB[2] = {0.0, 0.0};
#pragma unroll
            for (int u = 0; u < kMaxR; ++u) {
                const int i = row0 + u;
#pragma unroll
                for (int sy = 0; sy < 2; ++sy) {
                    rinv[u][sy] = 0.0;
                    if (u >= Rw || i >= M) continue;
                    const double pn = rb[u][sy] * pp[sy] - ra[u][sy] * rc[u][sy] * qq[sy];
                    qq[sy] = pp[sy];
                    pp[sy] = pn;
                    const double rr = qq[sy] / pp[sy];
                    const double sc = fabs(pp[sy]);
                    if (sc > 1e100 || sc < 1e-100) { pp[sy] /= sc; qq[sy] /= sc; }
                    rinv[u][sy] = rr;
                    const double af = -rr * ra[u][sy];
                    fB[sy] = fma(af, fB[sy], rr * rd[u][sy]);
                    fA[sy] *= af;
                }
            }
            // forward substitution of both systems
            double yy[2];
            scan_fwd_n<2>(fA, fB, yy, S.tot + (scan_par++ & 1) * 8 * kW);
            double y[kMaxR][2];
#pragma unroll
            for (int u = 0; u < kMaxR; ++u) {
                const int i = row0 + u;
#pragma unroll
                for (int sy = 0; sy < 2; ++sy) {
                    y[u][sy] = 0.0;
                    if (u >= Rw || i >= M) continue;
                    yy[sy] = fma(-rinv[u][sy] * ra[u][sy], yy[sy], rinv[u][sy] * rd[u][sy]);
                    y[u][sy] = yy[sy];
                }
            }
            // backward substitution: x_i = -(c_i / u_i) x_{i+1} + y_i
            double bA[2] = {1.0, 1.0}, bB[2] = {0.0, 0.0};
#pragma unroll
            for (int u = kMaxR - 1; u >= 0; --u) {
                const int i = row0 + u;
                if (u >= Rw || i >= M) continue;
#pragma unroll
                for (int sy = 0; sy < 2; ++sy) {
                    const double c = sy ? S.lfc[i] : S.l1c[i];
                    const double ab = -(c * rinv[u][sy]);
                    bB[sy] = fma(ab, bB[sy], y[u][sy]);
                    bA[sy] *= ab;
                }
            }
            double xx[2];
            scan_bwd_n<2>(bA, bB, xx, S.tot + (scan_par++ & 1) * 8 * kW);
#pragma unroll
            for (int u = kMaxR - 1; u >= 0; --u) {
                const int i = row0 + u;
                if (u >= Rw || i >= M) continue;
#pragma unroll
                for (int sy = 0; sy < 2; ++sy) {
                    const double c = sy ? S.lfc[i] : S.l1c[i];
                    xx[sy] = fma(-(c * rinv[u][sy]), xx[sy], y[u][sy]);
                }
                S.bpr[i] = xx[0];
                S.bpi[i] = xx[1];
            }
        }
        __syncthreads();
        PHASE_MARK(3);

        // ---------------- P5: store slice k; push k -> k+1 (or to the next sub-slice) and deposit
        if (tid >= 7 && tid < 9) S.fx[tid] = 0;   // the S deposit's maxima (read last before P4's barrier)
        // adaptive sub-slicing, decided in the slice's own pass from the particles as they stand
        // (src/Simulation.cpp:837-847): nsub = ceil(max cells crossed / max_cells_per_step), at least
        // ceil(dxi / (2 h_last)) (the step at most doubles), at most substep_max
        if (ss == 0 && A.max_cells > 0.0 && k + 1 < K) {
            double c = 0.0;
            if (REG) {
                if (tid < np && P.w != 0.0) c = cells_crossed(S, N, R, P.x, P.y, P.px, P.py, P.dl, A.dxi);
            } else {
                for (int p = tid; p < np; p += kThreads) {
                    const double* ps = gate.ps(A);
                    if (ps[5 * (size_t)npad + p] == 0.0) continue;
                    c = fmax(c, cells_crossed(S, N, R, ps[p], ps[npad + p], ps[2 * (size_t)npad + p],
                                              ps[3 * (size_t)npad + p], ps[4 * (size_t)npad + p], A.dxi));
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) c = fmax(c, __shfl_xor_sync(FULL, c, o));
            if (lane == 0 && c > 0.0) atomicMax(S.cmax, (unsigned long long)__double_as_longlong(c));
            __syncthreads();
            const double cm = __longlong_as_double((long long)*S.cmax);
            int n = cm <= A.max_cells ? 1 : (int)ceil(cm / A.max_cells);
            if (hlast > 0.0) n = max(n, (int)ceil(A.dxi / (2.0 * hlast) - 1e-9));
            nsub = min(n, A.substep_max > 0 ? A.substep_max : 64);
            if (tid == 0 && nsub > 1) S.fx[11] += nsub - 1;
        }
        const double hstep = A.dxi / nsub;
        const bool to_next = ss == nsub - 1;       // this push's deposit builds slice k+1, else the next sub-slice
        // The accumulators of the deposit: buffer s (with double-buffered sources its slice is stored and the
        // next slice's start values already sit in sn; with one buffer s is sn). Its values go to sn for
        // the next slice, or stay in s for the next sub-slice. Zeroed (all 9 arrays) after the store.
        const Src acc = s;
        const Src dst = to_next ? sn : s;
        {
            const size_t fb = (size_t)k * M;
            for (int j = tid; j < M; j += kThreads) {
                if (ss == 0) {
                    double* F = gate.fld(A) + (fb + j) * F_NC0;
                    F[F_EP1R] = S.wr1[j] + S.bpi[j];
                    F[F_EP1I] = 0.0 - S.bpr[j];
                    F[F_BP1R] = S.bpr[j];
                    F[F_BP1I] = S.bpi[j];
                    F[F_EZ0] = S.ez[j];
                    F[F_BZ0] = S.bz[j];
                    double* D = gate.diag(A) + (fb + j) * D_NC0;
                    D[D_PSI0] = S.psi[j];
                    D[D_NE0] = s.ne[j];
                    D[D_NI0] = s.ni[j];
                    if (double* const W = gate.wrec(A)) W[fb + j] = S.wr1[j];
                }
                if (k + 1 < K) {
#pragma unroll
                    for (int c = 0; c < 7; ++c) dep_arr(acc, c)[j] = 0.0;
                    acc.S1r[j] = 0.0;
                    acc.S1i[j] = 0.0;
                }
            }
        }
        if (k + 1 < K) {
            // the beam part the deposit's values start from, for this thread's rows: slice k+1's (one
            // buffer), or slice k's extrapolated to the next sub-slice
            BeamRow nxt[kMaxR];
            if (!to_next || !A.dbuf)
#pragma unroll
                for (int u = 0; u < kMaxR; ++u)
                    if (u < Rw && row0 + u < M)
                        nxt[u] = to_next ? beam_row<Gate::kActive, EXT>(A, gate.bsrc(A), k + 1, row0 + u)
                                         : beam_row_at<Gate::kActive, EXT>(A, gate.bsrc(A), k, row0 + u,
                                                                            (ss + 1) * hstep);
            const bool first = (k == 0) && (ss == 0) && !A.pin_pushed;
            coeffs(hstep, first);
            if (REG) {
                bool act = tid < np && P.w != 0.0;
                double v[12];
                if (act) {
                    const int pr = push_particle(P, geometry_in(S.r, S.ih, P.x, P.y, J), S, A, first, abc, hstep);
                    if (pr > 0) {
                        const double rn = sqrt(P.x * P.x + P.y * P.y);
                        J = locate_from(S.r, N, R, rn, J);
                        deposit_values(P, geometry_in(S.r, S.ih, P.x, P.y, J), S, v);
                    } else {
                        act = false;
                        atomicAdd(S.lost, 1);
                        if (pr < 0) atomicAdd(S.fx + 12, 1);
                    }
                }
                const bool tail = deposit_runs<true>(act, J, P.q < 0.0, v, S.fx);
                __syncthreads();
                deposit_add(tail, J, P.q < 0.0, v, acc, S.fx, bits_p);
            } else {
                // pass 0 pushes and takes the exponent maxima; pass 1 recomputes the deposit values of
                // the pushed particles and adds them
                for (int pass = 0; pass < 2; ++pass) {
                    if (pass == 1) __syncthreads();
                    for (int base = tid - lane; base < np; base += kThreads) {
                        const int p = base + lane;
                        bool act = false;
                        int j = 0;
                        double v[12];
                        PState<ORD> Q;
                        if (p < np) {
                            pbase(Q, S, A, gate.ps(A), npad, p);
                            species_params(A, p, Q.q, Q.qm);
                            if (Q.w != 0.0) {
                                if (pass == 0) {
                                    phist(Q, gate.ps(A), npad, p);
                                    const PGeo g = pgeo(S, A, N, R, p, Q.x, Q.y);
                                    const int pr = push_particle(Q, g, S, A, first, abc, hstep);
                                    if (pr > 0) {
                                        PGeo g2;
                                        if (A.pcache) {        // the new cell by a short walk from the old one
                                            const int jn = locate_from(S.r, N, R, sqrt(Q.x * Q.x + Q.y * Q.y), g.j);
                                            g2 = geometry_in(S.r, S.ih, Q.x, Q.y, jn);
                                            S.pj[p] = jn;
                                        } else {
                                            g2 = geometry(S.r, S.ih, N, R, Q.x, Q.y);
                                        }
                                        j = g2.j;
                                        deposit_values(Q, g2, S, v);
                                        act = true;
                                    } else {
                                        atomicAdd(S.lost, 1);
                                        if (pr < 0) atomicAdd(S.fx + 12, 1);
                                    }
                                    pstore(Q, gate.ps(A), npad, p);
                                    pbase_put(Q, S, A, p);
                                } else {
                                    const PGeo g2 = pgeo(S, A, N, R, p, Q.x, Q.y);
                                    j = g2.j;
                                    deposit_values(Q, g2, S, v);
                                    act = true;
                                }
                            }
                        }
                        const bool neg = act && Q.q < 0.0;
                        if (pass == 0) {
                            deposit_runs<true>(act, j, neg, v, S.fx);
                        } else {
                            const bool tail = deposit_runs<false>(act, j, neg, v, S.fx);
                            deposit_add(tail, j, neg, v, acc, S.fx, bits_p);
                        }
                    }
                }
            }
            __syncthreads();
            if (tid == 0)
                for (int c = 0; c < 7; ++c) S.fx[13] += S.fx[c] == 2047;
#pragma unroll
            for (int u = 0; u < kMaxR; ++u) {
                const int i = row0 + u;
                if (u >= Rw || i >= M) continue;
                double b0[7];
                if (to_next && A.dbuf) {
#pragma unroll
                    for (int c = 0; c < 7; ++c) b0[c] = dep_arr(sn, c)[i];
                } else {
                    init_base<EXT>(S, i, nxt[u], M, b0);
                }
                deposit_finish(dst, acc, i, b0, S.fx, bits_p);
            }
        }
        if (Gate::kActive && to_next) gate.slice_done_all(k);          // every thread, before the barrier
        __syncthreads();
        PHASE_MARK(4);
        if (Gate::kActive && to_next) {
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
    }   // the passes of slice k
    }
    if (A.pout) {
        // a slab that hands its plasma on: push the last slice too (src/Simulation.cpp:755, the push of the
        // last local slice produces the state entering the next slab), no deposit
        const bool first = (K == 1) && !A.pin_pushed;
        coeffs(A.dxi, first);
        if (REG) {
            if (tid < np && P.w != 0.0) {
                const int pr = push_particle(P, geometry_in(S.r, S.ih, P.x, P.y, J), S, A, first, abc, A.dxi);
                if (pr <= 0) { atomicAdd(S.lost, 1); if (pr < 0) atomicAdd(S.fx + 12, 1); }
            }
            if (tid < np) pstore(P, A.pout, npad, tid);
        } else {
            for (int p = tid; p < np; p += kThreads) {
                PState<ORD> Q;
                pload(Q, gate.ps(A), npad, p);
                species_params(A, p, Q.q, Q.qm);
                if (Q.w != 0.0) {
                    const int pr = push_particle(Q, geometry(S.r, S.ih, N, R, Q.x, Q.y), S, A, first, abc, A.dxi);
                    if (pr <= 0) { atomicAdd(S.lost, 1); if (pr < 0) atomicAdd(S.fx + 12, 1); }
                }
                pstore(Q, gate.ps(A), npad, p);
                pstore(Q, A.pout, npad, p);
            }
        }
        __syncthreads();
    }
    if (REG && tid < np) pstore(P, gate.ps(A), npad, tid);
    if (tid == 0 && A.counters) {
        atomicAdd(&A.counters[0], (unsigned long long)*S.lost);
        if (S.fx[13]) atomicAdd(&A.counters[1], (unsigned long long)S.fx[13]);
        if (S.fx[12]) atomicAdd(&A.counters[2], (unsigned long long)S.fx[12]);
        if (S.fx[11]) atomicAdd(&A.counters[3], (unsigned long long)S.fx[11]);
    }
    return true;
#undef PHASE_MARK
#undef SUB_MARK
}



}  // namespace qzb
