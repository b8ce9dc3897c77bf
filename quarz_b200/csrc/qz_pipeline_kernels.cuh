#pragma once
// qz_pipeline_kernels.cuh -- consecutive time steps of Simulation::run (src/Simulation.cpp:1370-1448) in one
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
#include "qz_beam_body.cuh"
#include "qz_sweep_body.cuh"
#include "qz_sweep_m1_body.cuh"

#include <cub/device/device_radix_sort.cuh>

namespace qzb {

namespace {

using beam_detail::deposit_one;
using beam_detail::PState7;
using beam_detail::push_one;
using beam_detail::sums_add;
using beam_detail::xi_cell;

constexpr int kT = kSweepThreads;

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// where a wait gave up: *err = (site << 8) | 1
enum WaitSite { W_RING = 1, W_ROWS = 2, W_TASK = 3 };

// Wait until *p >= v. Bounded: gives up after P.timeout_ns, or as soon as another CTA reported an error.
__device__ bool wait_ge(const PipeArgs& P, const int* p, int v, int site) {
    if (ld_acquire(p) >= v) return true;
    const unsigned long long t0 = gtimer();
    for (;;) {
        __nanosleep(64);
        if (ld_acquire(p) >= v) return true;
        if (ld_acquire(P.err) != 0) return false;
        if (gtimer() - t0 > P.timeout_ns) {
            atomicCAS(P.err, 0, (site << 8) | 1);
            return false;
        }
    }
}

// Per-sweep state of the gate, in shared memory so that it holds no registers across the slice loop.
struct GateState {
    const double* bsrc;   // this step's ring slots
    double* fld;
    double* diag;
    double* ps;           // this CTA's plasma scratch
    int n;                // time step of this sweep
    int cursor;           // buckets [0, cursor) are known to have pushed step n-1
};

// The gate of a sweep inside the pipeline (the hooks sweep_body calls).
struct PipeGate {
    static constexpr bool kActive = true;
    const PipeArgs* P;    // the kernel's __grid_constant__ parameter block
    GateState* g;         // shared

    __device__ const double* bsrc(const SweepArgs&) const { return g->bsrc; }
    __device__ double* fld(const SweepArgs&) const { return g->fld; }
    __device__ double* diag(const SweepArgs&) const { return g->diag; }
    __device__ double* ps(const SweepArgs&) const { return g->ps; }
    __device__ double* bgs(const SweepArgs&) const { return P->m1s + blockIdx.x * P->m1s_slot; }
    __device__ double* srcs(const SweepArgs&) const { return P->m1s + blockIdx.x * P->m1s_slot + 3 * (size_t)P->sw.M; }
    __device__ double* traj(const SweepArgs&) const { return P->traj ? P->traj + (size_t)g->n * P->traj_slot : nullptr; }
    __device__ double* wrec(const SweepArgs& A) const {
        return P->wrec ? P->wrec + (size_t)g->n * A.K * A.M : nullptr;
    }

    // warp 0 (all 32 lanes): beam-source rows <= r are final. The lanes look at 32 buckets at once and
    // advance over the finished prefix; the first unfinished one is waited for (bounded).
    __device__ bool before_rows(int r) {
        const int lane = threadIdx.x & 31;
        const int need = P->cnt_le[r];
        int c = g->cursor;
        const int n = g->n;
        while (c < need) {
            const int b = c + lane;
            const bool done = b >= need || ld_acquire(P->bdone + b) >= n - 1;
            const unsigned m = __ballot_sync(0xffffffffu, done);
            const int run = (m == 0xffffffffu) ? 32 : __ffs(~m) - 1;   // finished buckets from c on
            c = min(c + run, need);                   // lanes past `need` count as finished: never beyond it
            if (run == 32 || c >= need) continue;
            // bucket c is not finished yet: lane 0 waits for it
            bool ok = true;
            if (lane == 0) {
                const unsigned long long t0 = P->trace ? gtimer() : 0ull;
                ok = wait_ge(*P, P->bdone + c, n - 1, W_ROWS);
                if (ok && P->trace) {                 // the longest wait of this sweep: for which bucket
                    unsigned long long* tr = P->trace + (size_t)kTraceStride * n;
                    const unsigned long long dtw = gtimer() - t0;
                    if (dtw > tr[18]) {
                        tr[18] = dtw;
                        tr[19] = (unsigned long long)c;
                        tr[20] = (unsigned long long)r;
                        tr[21] = (unsigned long long)(long long)__ldcg(P->bk_cmax + c);
                    }
                }
            }
            if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) return false;
        }
        __syncwarp();
        if (lane == 0) g->cursor = c;
        __syncwarp();
        return true;
    }
    // every thread, after its stores of slice k: row k-1 of the beam sources is no longer needed
    __device__ void slice_done_all(int k) {
        if (k >= 1) {
            const int nr = P->sw.M * P->bnc;
            double* row = const_cast<double*>(g->bsrc) + (size_t)(k - 1) * nr;
            for (int i = threadIdx.x; i < nr; i += kT) __stcg(row + i, 0.0);
            if (P->sw.bq)                            // the low limbs of the exact deposits
                for (int i = threadIdx.x; i < nr; i += kT) __stcg(row + P->sw.bfx_lo + i, 0.0);
        }
    }
    // thread 0, after the barrier that ends slice k: publish it (the fence covers the stores of the
    // whole CTA, which the barrier ordered before it)
    __device__ bool slice_done(int k) {
        __threadfence();
        st_release(P->prog + g->n, k + 1);
        if (P->trace) {                               // progress marks at every 16th of the box
            const int K = P->sw.K;
            const int j = (16 * (k + 1)) / K;
            if (j > (16 * k) / K)
                P->trace[(size_t)kTraceStride * g->n + 1 + j] = gtimer();
        }
        return ld_acquire(P->err) == 0;
    }
};

template <int MODES, int ORD, bool REG, int kMaxR, bool EXT>
__device__ __forceinline__ void sweep_role(const PipeArgs& P, double* smem) {
    __shared__ int s_ok;
    __shared__ GateState gs;
    const int tid = threadIdx.x;
    const int K = P.sw.K, M = P.sw.M;
    for (int n = blockIdx.x; n <= P.nsteps; n += P.nsweep) {
        const int slot = n % P.ring;
        if (tid == 0) {
            s_ok = (n < P.ring) ? 1 : (wait_ge(P, P.pdone + (n - P.ring), P.nbk, W_RING) ? 1 : 0);
            gs.bsrc = P.bsrc + slot * P.bsrc_slot;
            gs.fld = P.fld + slot * P.fld_slot;
            gs.diag = P.diag + slot * P.diag_slot;
            gs.ps = P.ps + blockIdx.x * P.ps_slot;
            gs.n = n;
            gs.cursor = 0;
        }
        __syncthreads();
        if (!s_ok) return;
        if (P.trace && tid == 0) P.trace[(size_t)kTraceStride * n] = gtimer();
        PipeGate g{&P, &gs};
        const bool ok = MODES == 1 ? sweep_m1_body<ORD, PipeGate, EXT>(P.sw, smem, g)
                                   : sweep_body<ORD, REG, kMaxR, PipeGate, EXT>(P.sw, smem, g);
        if (!ok) return;
        // the last row (the others were zeroed slice by slice)
        const int nr = M * P.bnc;
        double* row = P.bsrc + slot * P.bsrc_slot + (size_t)(K - 1) * nr;
        for (int i = tid; i < nr; i += kT) __stcg(row + i, 0.0);
        if (P.sw.bq)
            for (int i = tid; i < nr; i += kT) __stcg(row + P.sw.bfx_lo + i, 0.0);
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release(P.sdone + n, 1);
            if (P.trace) P.trace[(size_t)kTraceStride * n + 1] = gtimer();
        }
    }
}

// Is task (m, b) ready: bucket b pushed step m-1, and (for a push) step m's fields stored up to the
// bucket's cells and the next step's beam-source slot clean. Every condition only ever turns true.
__device__ __forceinline__ bool task_ready(const PipeArgs& P, int m, int b) {
    if (ld_acquire(P.bdone + b) < m - 1) return false;
    if (m >= P.nsteps) return true;                       // moments of the final state only
    const int cm = __ldcg(P.bk_cmax + b);
    if (ld_acquire(P.prog + m) < min(max(cm, 0) + 2, P.sw.K)) return false;
    if (m + 1 >= P.ring && ld_acquire(P.sdone + (m + 1 - P.ring)) < 1) return false;
    return true;
}

// Warp-collective: claim the oldest ready task. Lane i looks at step lo + i (+32, ...), the lowest
// ready step is claimed with a CAS on its next-bucket counter, so a claimed task never waits. Returns
// false when every task is claimed, or on an error / time-out (recorded in *err).
__device__ __forceinline__ bool claim_task(const PipeArgs& P, int last, int& n, int& b, unsigned long long* st) {
    const int lane = threadIdx.x & 31;
    const unsigned long long t0 = gtimer();
    unsigned sleep_ns = 64;       // back off while nothing is ready: idle warps must not flood L2
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
                if (idx < P.nbk) ready = task_ready(P, m, idx);
            }
            const unsigned full = __ballot_sync(0xffffffffu, idx >= P.nbk);
            if (base == lo && (full & 1u)) {              // steps lo, lo+1, ... fully claimed
                const int c = (~full == 0u) ? 32 : __ffs(~full) - 1;
                if (lane == 0) atomicMax(P.lo, base + c);
            }
            unsigned rm = __ballot_sync(0xffffffffu, ready);
            // warps start at different ready steps (oldest first only for warp 0 of each rotation), so
            // that they do not all race for one step's counter
            const int rot = (int)((blockIdx.x * (kT / 32) + (threadIdx.x >> 5)) & 31);
            while (rm) {
                const unsigned hi = rm >> rot, low = rm & ((1u << rot) - 1u);
                const int src = hi ? rot + __ffs(hi) - 1 : __ffs(low) - 1;
                int got = 0;
                if (lane == src) got = atomicCAS(P.next + m, idx, idx + 1) == idx ? 1 : 0;
                if (__shfl_sync(0xffffffffu, got, src)) {
                    ++st[0];
                    n = base + src;
                    b = __shfl_sync(0xffffffffu, idx, src);
                    return true;
                }
                rm &= ~(1u << src);
                ++st[2];
            }
        }
        ++st[1];
        __nanosleep(sleep_ns);
        sleep_ns = min(2 * sleep_ns, 8192u);
        if (gtimer() - t0 > P.timeout_ns) {
            if (lane == 0) atomicCAS(P.err, 0, (W_TASK << 8) | 1);
            return false;
        }
    }
}

// Worker CTAs: every warp is an independent worker that claims (step, bucket) tasks.
__device__ __forceinline__ void worker_role(const PipeArgs& P, double* smem) {
    const int tid = threadIdx.x, lane = tid & 31;
    const int M = P.sw.M, N = P.sw.N, K = P.sw.K;
    // grid arrays in shared memory: the binary search of every lookup stays on chip; so do the node
    // scales of the exact deposits (a global load of them before every quantisation stalled each warp
    // on L2 latency: ~10k cycles per 32-particle iteration)
    double* r = smem;
    double* ih = r + M;
    double* iV = ih + M;
    double* fxs = iV + M + (size_t)(kT / 32) * 17 * 32;        // behind the per-warp moment slots
    const double* fx_src = nullptr;
    for (int q = 0; q < P.nbeams && !fx_src; ++q) fx_src = P.beam[q].fx_scale;
    for (int j = tid; j < M; j += kT) {
        r[j] = P.sw.r[j];
        iV[j] = P.sw.inv_V[j];
        if (j < N) ih[j] = P.sw.inv_h[j];
        if (fx_src) fxs[j] = fx_src[j];
    }
    __syncthreads();
    const int last = P.pmom ? P.nsteps : P.nsteps - 1;     // the last step with tasks
    int n, b;
    // trace totals: tasks, scans that found nothing, lost claims, ns in tasks (registers); ns waiting for a
    // task and ns in the moments passes are added to the trace directly (no register held for them)
    unsigned long long st[4] = {0, 0, 0, 0};
    unsigned long long* const wtot = P.trace ? P.trace + (size_t)kTraceStride * (P.nsteps + 1) : nullptr;
    unsigned long long t_idle = P.trace ? gtimer() : 0ull;
    while (claim_task(P, last, n, b, st)) {
        const unsigned long long t_task = P.trace ? gtimer() : 0ull;
        if (P.trace && lane == 0) atomicAdd(wtot + 4, t_task - t_idle);
        const bool push = n < P.nsteps;
        const int bb = __ldg(P.bk_beam + b);
        const long i0 = __ldg(P.bk_start + b), i1 = __ldg(P.bk_end + b);
        BeamArgs Bb = P.beam[bb];
        Bb.r = r;
        Bb.inv_h = ih;
        Bb.inv_V = iV;
        if (Bb.fx_scale) Bb.fx_scale = fxs;                      // (every beam of a run has the same scales)
        const double* fld = P.fld + (size_t)(n % P.ring) * P.fld_slot;
        double* bnext = P.bsrc + (size_t)((n + 1) % P.ring) * P.bsrc_slot;
        // bring the task's inputs towards L2 while it starts: the particle columns, the field rows it
        // gathers and the beam-source rows it deposits into (a warp issues one prefetch per 128 B line)
        if (push) {
            const int c0 = max(__ldg(P.bk_cmin + b), 0);
            const int c1 = min(__ldcg(P.bk_cmax + b) + 2, K - 1);
            if (c1 >= c0) {
                const double* f0 = fld + (size_t)c0 * M * (P.modes ? F_NC1 : F_NC0);
                const long fl = (long)(c1 - c0 + 1) * M * (P.modes ? F_NC1 : F_NC0);
                for (long o = (long)lane * 16; o < fl; o += 32 * 16) prefetch_l2(f0 + o);
                const double* b0 = bnext + (size_t)c0 * M * P.bnc;
                const long bl = (long)(c1 - c0 + 1) * M * P.bnc;
                for (long o = (long)lane * 16; o < bl; o += 32 * 16) prefetch_l2(b0 + o);
                if (Bb.fx_scale)                            // the low limbs of the exact deposits
                    for (long o = (long)lane * 16; o < bl; o += 32 * 16) prefetch_l2(b0 + Bb.fx_lo + o);
            }
            const long pn = i1 - i0;
            for (long o = (long)lane * 16; o < pn; o += 32 * 16) {
                prefetch_l2(Bb.x + i0 + o); prefetch_l2(Bb.y + i0 + o); prefetch_l2(Bb.px + i0 + o);
                prefetch_l2(Bb.py + i0 + o); prefetch_l2(Bb.pz + i0 + o); prefetch_l2(Bb.xi + i0 + o);
                prefetch_l2(Bb.w + i0 + o);
            }
        }
        const double qm = Bb.q / Bb.m;
        const double h = 0.5 * qm * P.dt_kick;
        const double hs = (n == 0 && P.startup[bb]) ? 0.5 * qm * (-0.5 * P.dt_kick) : 0.0;
        const bool rigid = P.rigid[bb] != 0;
        const double gref = P.gref[bb], xiref = P.xiref[bb];
        // moments of step n (before the push), a pass of their own so that the 17 sums are not live
        // during the push; it also brings the bucket's particles into L1 for the push
        // m = 0 pushes add the moment sums inside the push loop, each lane into its own shared-memory
        // accumulators in the same particle order as this separate pass (the result is the same bits)
        const bool fuse = P.pmom && push && P.modes == 0;
        double* macc = iV + M + (size_t)(tid >> 5) * 17 * 32;        // this warp's [17][32]
        if (fuse)
#pragma unroll
            for (int c = 0; c < 17; ++c) macc[c * 32 + lane] = 0.0;
        if (P.pmom && !fuse) {
            double acc[17];
#pragma unroll
            for (int c = 0; c < 17; ++c) acc[c] = 0.0;
            for (long i = i0 + lane; i < i1; i += 32) {
                PState7 p;
                p.w = __ldcg(Bb.w + i);
                if (p.w == 0.0) continue;
                p.x = __ldcg(Bb.x + i); p.y = __ldcg(Bb.y + i);
                p.px = __ldcg(Bb.px + i); p.py = __ldcg(Bb.py + i); p.pz = __ldcg(Bb.pz + i);
                p.xi = __ldcg(Bb.xi + i);
                sums_add(acc, p, gref, xiref);
            }
            double mine = 0.0;
#pragma unroll
            for (int c = 0; c < 17; ++c) {
                double x = acc[c];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                if (lane == c) mine = x;
            }
            if (lane < 17) P.pmom[((size_t)n * P.nbk + b) * 17 + lane] = mine;
        }
        if (push && P.snap) {                        // the bucket before its push (for the adjoint)
            double* sn = P.snap + (size_t)n * P.snap_step + P.snap_off[bb];
            const double* cols[7] = {Bb.x, Bb.y, Bb.px, Bb.py, Bb.pz, Bb.xi, Bb.w};
#pragma unroll
            for (int c = 0; c < 7; ++c)
                for (long i = i0 + lane; i < i1; i += 32) __stcg(sn + (size_t)c * Bb.n + i, __ldcg(cols[c] + i));
        }
        if (P.trace && lane == 0) atomicAdd(wtot + 5, gtimer() - t_task);
        int cmax = -2;
        if (!push) {
            // moments only (the state after the last push)
        } else if (P.modes == 0) {
            // m = 0: particles are in (xi cell, r cell) order, so neighbouring lanes mostly deposit into
            // the same 2 x 2 cells: sum runs of equal cells across the warp, one reduction per run
            for (long base = i0; base < i1; base += 32) {
                const long i = base + lane;
                bool dep = false;
                int dk = 0, dj = 0;
                double v[4 * beam_detail::kDep0];
                if (i < i1) {
                    PState7 p;
                    p.w = __ldcg(Bb.w + i);
                    if (p.w != 0.0) {
                        p.x = __ldcg(Bb.x + i); p.y = __ldcg(Bb.y + i);
                        p.px = __ldcg(Bb.px + i); p.py = __ldcg(Bb.py + i); p.pz = __ldcg(Bb.pz + i);
                        p.xi = __ldcg(Bb.xi + i);
                        if (fuse) beam_detail::sums_add_lane(macc + lane, p, gref, xiref);
                        if (push) {
                            bool alive = true;
                            int jg = 0;
                            if (!rigid) {
                                alive = P.fld_l1 ? push_one<false>(Bb, fld, p, h, hs, P.dt_drift, &jg)
                                                 : push_one<true>(Bb, fld, p, h, hs, P.dt_drift, &jg);
                                __stcg(Bb.x + i, p.x); __stcg(Bb.y + i, p.y);
                                __stcg(Bb.px + i, p.px); __stcg(Bb.py + i, p.py); __stcg(Bb.pz + i, p.pz);
                                __stcg(Bb.xi + i, p.xi);
                                if (!alive) __stcg(Bb.w + i, 0.0);
                            } else {
                                jg = -1;
                            }
                            if (alive) {
                                dep = beam_detail::deposit_vals0(Bb, p.x, p.y, p.px, p.py, p.pz, p.xi, p.w, jg, dk,
                                                                 dj, v);
                                cmax = max(cmax, xi_cell(Bb, p.xi));
                            }
                        }
                    }
                }
                if (!dep)
#pragma unroll
                    for (int c = 0; c < 4 * beam_detail::kDep0; ++c) v[c] = 0.0;
                const int key = dep ? (dk + 1) * M + dj : -1 - lane;
                if (warp_runs_sum<4 * beam_detail::kDep0>(key, v) && dep) beam_detail::deposit_add0(Bb, bnext, dk, dj, v);
            }
        } else if (P.modes == 1) {
            // m = 1: the same runs of equal cells across the warp, summed per corner (12 components each)
            for (long base = i0; base < i1; base += 32) {
                const long i = base + lane;
                bool dep = false;
                beam_detail::Dep1 D;
                D.k = D.j = 0;
                if (i < i1) {
                    PState7 p;
                    p.w = __ldcg(Bb.w + i);
                    if (p.w != 0.0) {
                        p.x = __ldcg(Bb.x + i); p.y = __ldcg(Bb.y + i);
                        p.px = __ldcg(Bb.px + i); p.py = __ldcg(Bb.py + i); p.pz = __ldcg(Bb.pz + i);
                        p.xi = __ldcg(Bb.xi + i);
                        bool alive = true;
                        int jg = -1;
                        if (!rigid) {
                            alive = P.fld_l1 ? push_one<false>(Bb, fld, p, h, hs, P.dt_drift, &jg)
                                             : push_one<true>(Bb, fld, p, h, hs, P.dt_drift, &jg);
                            __stcg(Bb.x + i, p.x); __stcg(Bb.y + i, p.y);
                            __stcg(Bb.px + i, p.px); __stcg(Bb.py + i, p.py); __stcg(Bb.pz + i, p.pz);
                            __stcg(Bb.xi + i, p.xi);
                            if (!alive) __stcg(Bb.w + i, 0.0);
                        }
                        if (alive) {
                            dep = beam_detail::deposit_setup1(Bb, p.x, p.y, p.px, p.py, p.pz, p.xi, p.w, jg, D);
                            cmax = max(cmax, xi_cell(Bb, p.xi));
                        }
                    }
                }
                const int key = dep ? (D.k + 1) * M + D.j : -1 - lane;
#pragma unroll 1
                for (int cr = 0; cr < 4; ++cr) {
                    const int a = cr >> 1, b = cr & 1;
                    if (a == 1 && Bb.ngp) continue;                  // (uniform: the beam's shape)
                    double v[beam_detail::kDep1];
                    if (dep) beam_detail::deposit_corner1(Bb, D, a, b, v);
                    else
#pragma unroll
                        for (int c = 0; c < beam_detail::kDep1; ++c) v[c] = 0.0;
                    if (warp_runs_sum<beam_detail::kDep1>(key, v) && dep)
                        beam_detail::deposit_add1(Bb, bnext, D.k + a, D.j + b, v);
                }
            }
        } else
        for (long i = i0 + lane; i < i1; i += 32) {
            PState7 p;
            p.w = __ldcg(Bb.w + i);
            if (p.w == 0.0) continue;
            p.x = __ldcg(Bb.x + i); p.y = __ldcg(Bb.y + i);
            p.px = __ldcg(Bb.px + i); p.py = __ldcg(Bb.py + i); p.pz = __ldcg(Bb.pz + i);
            p.xi = __ldcg(Bb.xi + i);
            if (!push) continue;
            if (rigid) {
                deposit_one(Bb, bnext, p.x, p.y, p.px, p.py, p.pz, p.xi, p.w);
                cmax = max(cmax, xi_cell(Bb, p.xi));
                continue;
            }
            const bool alive = P.fld_l1 ? push_one<false>(Bb, fld, p, h, hs, P.dt_drift)
                                        : push_one<true>(Bb, fld, p, h, hs, P.dt_drift);
            __stcg(Bb.x + i, p.x); __stcg(Bb.y + i, p.y);
            __stcg(Bb.px + i, p.px); __stcg(Bb.py + i, p.py); __stcg(Bb.pz + i, p.pz);
            __stcg(Bb.xi + i, p.xi);
            if (!alive) {
                __stcg(Bb.w + i, 0.0);
                continue;
            }
            deposit_one(Bb, bnext, p.x, p.y, p.px, p.py, p.pz, p.xi, p.w);
            cmax = max(cmax, xi_cell(Bb, p.xi));
        }
        if (fuse) {
            double mine = 0.0;
#pragma unroll
            for (int c = 0; c < 17; ++c) {
                double x = macc[c * 32 + lane];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                if (lane == c) mine = x;
            }
            if (lane < 17) P.pmom[((size_t)n * P.nbk + b) * 17 + lane] = mine;
        }
        // bucket result: the highest live cell after the push
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
        __syncwarp();
        if (lane == 0) {
            // never below the previous bound: cells only grow, and a bucket may have no live particle
            if (push) __stcg(P.bk_cmax + b, max(cmax, __ldcg(P.bk_cmax + b)));
            __threadfence();
            if (push) st_release(P.bdone + b, n);
            atomicAdd(P.pdone + n, 1);
        }
        __syncwarp();
        if (P.trace) {
            t_idle = gtimer();
            st[3] += t_idle - t_task;
        }
    }
    if (P.trace && lane == 0) {
        unsigned long long* ws = P.trace + (size_t)kTraceStride * (P.nsteps + 1);
        for (int c = 0; c < 4; ++c) atomicAdd(ws + c, st[c]);
    }
}

// EXT: the variant whose sweeps handle the smoothing filter and static (analytic) beam sources
template <int MODES, int ORD, bool REG, int kMaxR, bool EXT = false>
__global__ void __launch_bounds__(kSweepThreads, 1) pipeline_kernel(const __grid_constant__ PipeArgs P) {
    extern __shared__ double smem_raw[];
    if ((int)blockIdx.x < P.nsweep)
        sweep_role<MODES, ORD, REG, kMaxR, EXT>(P, smem_raw);
    else
        worker_role(P, smem_raw);
}

// moments of step n, beam q: the bucket partials of that beam in bucket order (deterministic)
__global__ void moments_reduce_kernel(const __grid_constant__ PipeArgs P, double* __restrict__ mom) {
    const int n = blockIdx.x / P.nbeams, q = blockIdx.x % P.nbeams, c = threadIdx.x;
    if (c >= 17) return;
    double v = 0.0;
    for (int b = 0; b < P.nbk; ++b)
        if (P.bk_beam[b] == q) v += P.pmom[((size_t)n * P.nbk + b) * 17 + c];
    mom[((size_t)n * P.nbeams + q) * 17 + c] = v;
}

template <int MODES, int ORD, bool REG, int RM, bool EXT = false>
cudaError_t launch_t(const PipeArgs& P, int grid, size_t smem, cudaStream_t stream) {
    auto fn = pipeline_kernel<MODES, ORD, REG, RM, EXT>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    void* args[] = {(void*)&P};
    return cudaLaunchCooperativeKernel((const void*)fn, dim3(grid), dim3(kSweepThreads), args, smem, stream);
}

template <int MODES, int ORD, bool REG, int RM, bool EXT = false>
int occupancy_t(size_t smem) {
    auto fn = pipeline_kernel<MODES, ORD, REG, RM, EXT>;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kSweepThreads, smem) != cudaSuccess) return 0;
    return nb;
}

// modes = 1 runs one row per thread with the plasma in the scratch (REG and kMaxR unused: false, 1)
template <int ORD, bool EXT>
cudaError_t launch_e(const PipeArgs& P, int grid, size_t smem, cudaStream_t s) {
    const bool reg = P.sw.np <= kSweepThreads;
    if (P.sw.rows_per_thread == 1)
        return reg ? launch_t<0, ORD, true, 1, EXT>(P, grid, smem, s) : launch_t<0, ORD, false, 1, EXT>(P, grid, smem, s);
    return reg ? launch_t<0, ORD, true, 4, EXT>(P, grid, smem, s) : launch_t<0, ORD, false, 4, EXT>(P, grid, smem, s);
}

template <int ORD>
cudaError_t launch_o(const PipeArgs& P, int grid, size_t smem, cudaStream_t s) {
    const bool ext = P.sw.filter || P.sw.bstat;
    if (P.modes == 1)
        return ext ? launch_t<1, ORD, false, 1, true>(P, grid, smem, s) : launch_t<1, ORD, false, 1, false>(P, grid, smem, s);
    return ext ? launch_e<ORD, true>(P, grid, smem, s) : launch_e<ORD, false>(P, grid, smem, s);
}

template <int ORD, bool EXT>
int occupancy_e(const PipeArgs& P, size_t smem) {
    const bool reg = P.sw.np <= kSweepThreads;
    if (P.sw.rows_per_thread == 1)
        return reg ? occupancy_t<0, ORD, true, 1, EXT>(smem) : occupancy_t<0, ORD, false, 1, EXT>(smem);
    return reg ? occupancy_t<0, ORD, true, 4, EXT>(smem) : occupancy_t<0, ORD, false, 4, EXT>(smem);
}

template <int ORD>
int occupancy_o(const PipeArgs& P, size_t smem) {
    const bool ext = P.sw.filter || P.sw.bstat;
    if (P.modes == 1) return ext ? occupancy_t<1, ORD, false, 1, true>(smem) : occupancy_t<1, ORD, false, 1, false>(smem);
    return ext ? occupancy_e<ORD, true>(P, smem) : occupancy_e<ORD, false>(P, smem);
}

}  // namespace

// the pipelined kernel of one Adams-Bashforth order (its variants for modes, plasma layout and the
// smoothing filter), defined by qz_pipeline_o<ORD>.cu: one translation unit per order, built in parallel
template <int ORD>
cudaError_t pipeline_launch_ord(const PipeArgs& P, int grid, size_t smem, cudaStream_t s);
template <int ORD>
int pipeline_occupancy_ord(const PipeArgs& P, size_t smem);

}  // namespace qzb
