// qz_internal.h -- kernel argument blocks and launchers shared by the .cu files of libqz_b200.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace qzb {

// threads of a sweep CTA: 512, or 1024 in the translation units of the wide m = 1 sweep (modes = 1
// with 513..1024 radial nodes, one node per thread), which compile these headers in namespace qzb_w
#ifndef QZ_SWEEP_THREADS
#define QZ_SWEEP_THREADS 512
#endif
constexpr int kSweepThreads = QZ_SWEEP_THREADS;
constexpr int kMaxSpecies = 4;

// Everything the m = 0 sweep kernel reads or writes. Pointers are device pointers.
struct SweepArgs {
    int M, N, K;                    // nodes, cells, slices
    int rows_per_thread;            // tridiagonal rows owned by one thread: ceil(M / kSweepThreads)
    double R, dxi, idxi;
    const double* r;                // nodes [M]
    const double* inv_h;            // 1/h [N]
    const double* inv_V;            // 1/V [M]
    // per-node constants, 13 arrays of M: gradient stencils gm g0 gp, 1/r (src/FieldSolver.cpp:157-176);
    // L0 Thomas factors 1/u, -a/u, -c/u; rows a b c of L1D and of L1F (src/FieldSolver.cpp:117-156)
    const double* consts;
    double flux_coef;               // coefficient of g in the flux row of L1F
    // mobile plasma species: particles [sp_off[s], sp_off[s+1])
    int nsp;
    int sp_off[kMaxSpecies + 1];
    double sp_q[kMaxSpecies], sp_qm[kMaxSpecies];
    int np, npad;                   // particles, stride of the state arrays
    int ord;                        // Adams-Bashforth order
    double ab[5];                   // its coefficients (uniform steps)
    double delta_min, max_qsa;
    double max_cells;               // pusher.max_cells_per_step: adaptive sub-slicing (0: off), m = 0
    int substep_max;                // pusher.substep_max
    const double* p_init;           // fresh plasma at the head: (6, npad) x y px py Delta w
    int nbg;                        // immobile particles (background)
    const double* bg_p;             // (3, nbg): x, y, w*q
    int neutralize;
    double* ps;                     // working state (6 + 5*ord, npad), used when np > kSweepThreads
    const double* bsrc;             // beam sources (K, M, 5)
    int ngp;
    double* fld;                    // (K, M, 6)
    double* diag;                   // (K, M, 3)
    // [0] plasma particles removed, [1] deposits with a non-finite contribution (per slice and array),
    // [2] plasma particles removed as trapped (Delta <= delta_min or gamma > max_qsa Delta), [3] sub-slices
    // beyond the regular slices (adaptive sub-slicing)
    unsigned long long* counters;
    unsigned long long* timing;     // optional: clock cycles per phase [6]
    int dbuf;                       // double-buffered slice sources (push fused with the next deposit)
    int const_smem;                 // per-node constants copied into shared memory
    int pcache;                     // > 0 (= np, plasma in global memory): a shared-memory copy of the
                                    // particles' positions, momenta and cells (Smem::pc)
    // modes = 1 only
    int picard;                     // B+ iterations (src/Simulation.cpp:560)
    const double* consts1;          // 9 x M: L1D Thomas 1/u, -a/u, -c/u; L0 rows a b c; L2D rows a b c
    double* bgs;                    // (3, M) scratch: background rho - J_z in modes 0 / 1
    double* srcs;                   // (2 x 30, M) scratch: the sources of this slice and of the next
    // optional, m = 0 (the adjoint's recomputation): the plasma state at the start of every slice,
    // (K, 6 + 5 * ord, npad): x y px py Delta w, then the AB history h[m][v] (m pushes ago); with
    // traj_every = C > 1 only at the checkpoint slices k = 0, C, 2C, ... (slot k / C), the reverse
    // sweep pushing the plasma again from them. wrec (K, M): the W+ radial field the plasma push of
    // every slice gathered (the field store holds it only summed with B_theta)
    double* traj;
    int traj_every;
    double* wrec;
    // optional, m = 0: radial smoothing of the plasma sources (plasma.smooth_length,
    // src/Simulation.cpp:63-66, :685-690, :810-835)
    int filter;
    const double* fconsts;          // 9 x M: Thomas factors 1/u, -a/u, -c/u of F0, then of F1, then of F2
    // optional: beam sources that do not change between steps (analytic rigid beams), (K, M, B_NC),
    // added to bsrc wherever the sweep reads it
    const double* bstat;
    // optional, m = 0: bsrc in the exact two-limb format of the beam deposits (BeamArgs::fx_scale):
    // bq[j] the quantum of node j, bfx_2s = 2^S
    const double* bq;
    double bfx_2s;
    long bfx_lo;
    // optional, m = 0: one slab of a xi-pipelined run (qz_sweep_run_stage). pin: the plasma entering
    // the slab's first slice ((6 + 5 ord, npad) like ps; null: the fresh plasma of the box head) and
    // pin_pushed: whether it has been pushed before (its AB history is filled); bguard: the beam sources
    // of the slice just ahead of the slab (M x B_NC0 values, null: none); pout: where the plasma goes
    // after the push of the slab's last slice (null: that slice is not pushed)
    const double* pin;
    int pin_pushed;
    const double* bguard;
    double* pout;
};

size_t sweep_m0_smem_bytes(int M, bool dbuf, bool const_smem, bool filter = false, int pcache = 0);
cudaError_t launch_sweep_m0(const SweepArgs& A, cudaStream_t stream);
// the modes = 1 sweep: one CTA, one radial row per thread (M <= kSweepThreads), plasma in A.ps
size_t sweep_m1_smem_bytes(int M);
cudaError_t launch_sweep_m1(const SweepArgs& A, cudaStream_t stream);
// the modes = 1 sweep with 1024 threads (513..1024 nodes, qz_sweep_m1w.cu): args points to a SweepArgs of
// args_size bytes
size_t sweep_m1w_smem_bytes(int M);
cudaError_t launch_sweep_m1w(const void* args, size_t args_size, cudaStream_t stream);

// the adjoint of an m = 0 run (qz_adjoint.cu): one CTA runs the sweep of one step in reverse, from
// the field-store adjoint lfld (K, M, 6) to the beam-source adjoint lbsrc (K, M, 5, accumulated),
// with the plasma trajectory recorded by the forward sweep; M and np at most kSweepThreads
size_t adjoint_sweep_smem_bytes(int M);
cudaError_t launch_sweep_back(const SweepArgs& A, const double* traj, const double* fld, const double* lfld,
                              double* lbsrc, cudaStream_t stream);

// Beam particles (SoA, device) and the box they live in.
struct BeamArgs {
    double *x, *y, *px, *py, *pz, *xi, *w;
    long n;
    double q, m;
    // grid
    int M, N;
    double R;
    const double* r;
    const double* inv_h;
    const double* inv_V;
    // box
    double xi_min, dxi, idxi;
    int K, ngp, modes;
    int pusher;                     // 0 vay, 1 boris, 2 hc, 3 imp (stand-alone push kernels only)
    // exact deposits (m = 0 runs of qz_sim): when fx_scale is set, bsrc holds two integer-valued
    // limbs per value, the high limb where the double would be and the low limb fx_lo doubles further;
    // a contribution v to node j is t = v fx_scale[j] (a power of two), split at S bits (beam_fx_add)
    const double* fx_scale;
    double fx_inv2s, fx_2s;         // 2^-S, 2^S
    long fx_lo;
};

cudaError_t launch_beam_deposit(const BeamArgs& B, double* bsrc, cudaStream_t s);
// the largest |w| of the beam's particles into *wmax (device; start it at 0): the bound of the exact
// deposits' quantum
cudaError_t launch_beam_wmax(const BeamArgs& B, double* wmax, cudaStream_t s);
// Beam::deposit_analytic (src/Beam.cpp:236-279): a rigid beam's sources at every (slice, node)
struct AnalyticArgs {
    double q, n0, s2, xi0, sxi, len, cut, x0, y0, xs, ys, vz, omvz;
    int flat, m1;
    const double* r;            // nodes [M] (device)
    int M, K, bnc;
    double xi_min, dxi;
};
cudaError_t launch_deposit_analytic(const AnalyticArgs& P, double* bsrc, cudaStream_t s);
// Beam::slice_sums (src/Beam.cpp:1195-1217): 9 sums per bin of the user xi in [lo, lo + nbins db), added
// into out (9 x nbins, cleared by the caller)
cudaError_t launch_slice_sums(const BeamArgs& B, double lo, double db, int nbins, double* out, cudaStream_t s);
cudaError_t launch_beam_push(const BeamArgs& B, const double* fld, double dt_kick, double dt_drift, int move,
                             cudaStream_t s);
cudaError_t launch_beam_push_deposit(const BeamArgs& B, const double* fld, double dt_kick, double dt_drift,
                                     double* bsrc_next, cudaStream_t s);
cudaError_t launch_beam_sums(const BeamArgs& B, double gref, double xiref, double* partial, int nblocks,
                             double* out17, cudaStream_t s);
int beam_sums_blocks(long n);
// Block cap of beam_sums_blocks (148 x 4), the row count of the static scratch of beam_sums_static.
constexpr int kSumsStaticBlocks = 148 * 4;
// beam_sums with the partial sums in a static __device__ array instead of caller- or library-
// allocated memory; the first call on a device looks up that device's address of the array.
// *nblocks_needed: the rows the call needs (cudaErrorInvalidValue when above kSumsStaticBlocks).
cudaError_t beam_sums_static(const BeamArgs& B, double gref, double xiref, double* out17, cudaStream_t s,
                             int* nblocks_needed);
// Unique id of the CUDA context current on this thread (0 when none or unknown): device addresses
// cached per device are valid only while the context they were taken in lives.
unsigned long long current_context_id();

// ---------------------------------------------------------------- time-step pipeline
// Consecutive time steps of Simulation::run in one cooperative launch: CTAs [0, nsweep) each run whole
// sweeps (steps n = blockIdx.x, +nsweep, ...); the other CTAs push beam buckets (a bucket is a run of
// particles of one beam, sorted by xi cell). Step n+1's sweep at slice k only needs the beam sources
// of rows <= k+3, i.e. the push of step n of the buckets whose particles sit in those rows, which in
// turn needs step n's fields a few slices further: consecutive steps run concurrently, staggered by
// a few slices. Particles only move towards larger xi cells (1 - v_z > 0), so the lowest cell of a
// bucket when it was formed is a lower bound for all later steps.
constexpr int kMaxBeams = 4;

struct PipeArgs {
    SweepArgs sw;                   // bsrc / fld / diag / ps of sw are unused: rings below
    int nsteps;                     // sweeps 0..nsteps, pushes 0..nsteps-1
    int nsweep;                     // CTAs running sweeps
    int ring;                       // slots of the field / diagnostics / beam-source rings
    // the push workers gather the fields through L1: set when no field slot is reused within the run
    // (ring > nsteps) and every field row starts on a 128-byte line, so no cached line can hold a row
    // before the sweep published it (rows are only read once published, and kernels start with L1 clean)
    int fld_l1;
    int modes, bnc;                 // azimuthal modes (0 / 1), beam-source components per node
    size_t fld_slot, diag_slot, bsrc_slot, ps_slot;   // doubles per slot (ps: per sweep CTA)
    double *fld, *diag, *bsrc, *ps;
    double* m1s;                    // modes = 1: per sweep CTA, background (3 M) + source buffers (60 M)
    size_t m1s_slot;
    int nbeams;
    BeamArgs beam[kMaxBeams];
    int rigid[kMaxBeams], startup[kMaxBeams];
    double gref[kMaxBeams], xiref[kMaxBeams];
    double dt_kick, dt_drift;
    int nbk;                        // buckets, ordered by their initial lowest xi cell
    const int *bk_beam, *bk_start, *bk_end;
    int* bk_cmax;                   // highest xi cell of the bucket's live particles (before the next push)
    const int* bk_cmin;             // lowest xi cell of the bucket when it was formed (a lower bound after)
    const int* cnt_le;              // [K]: number of buckets whose initial lowest cell is <= row
    double* pmom;                   // (nsteps + 1, nbk, 17) partial moment sums, or null
    // synchronisation words (device; set before the launch)
    int* prog;                      // [nsteps + 1] slices stored by sweep n (0)
    int* sdone;                     // [nsteps + 1] sweep n finished, its beam-source slot is zero again (0)
    int* pdone;                     // [nsteps + 1] bucket tasks finished for step n (0)
    int* bdone;                     // [nbk] last step whose push finished (-1)
    int* next;                      // [nsteps + 1] next unclaimed bucket of step n (0)
    int* err;                       // != 0: a wait gave up, (site << 8) | 1 (0)
    int* lo;                        // steps below *lo have every task claimed (0)
    unsigned long long timeout_ns;  // limit of every wait
    // optional, for the adjoint (m = 0): the plasma trajectory of every sweep (slot per step, see
    // SweepArgs::traj) and the beams of every step before its push (snap + n * snap_step + snap_off[beam],
    // 7 columns of the beam's n, the run's particle order); with them the rings hold every step
    double* traj;
    size_t traj_slot;
    double* wrec;                   // W+ radial field per slice (SweepArgs::wrec), slot of K M per step
    double* snap;
    size_t snap_step;
    long snap_off[kMaxBeams];
    unsigned long long* trace;      // optional, kTraceStride per step: %globaltimer at the start and end of
                                    // sweep n, when it passed each 16th of the box, then its longest wait
                                    // for beam rows (ns, bucket, row, bucket's cmax); after the steps:
                                    // kWorkerTotals worker totals (see worker_role)
};
constexpr int kTraceStride = 22;
constexpr int kWorkerTotals = 6;    // trace totals of the push workers after the steps

size_t pipeline_smem_bytes(int modes, int M, bool dbuf, bool const_smem, bool filter = false, int pcache = 0);
// resident CTAs of the pipeline kernel on this device (0 if it cannot run); *sms: the SM count
int pipeline_max_grid(const PipeArgs& P, int* sms);
// cooperative launch of grid CTAs (fails unless all of them can be resident at once)
cudaError_t launch_pipeline(const PipeArgs& P, int grid, cudaStream_t stream);
// mom (nsteps + 1, nbeams, 17) from the bucket partials, in bucket order
cudaError_t launch_moments_reduce(const PipeArgs& P, double* mom, cudaStream_t s);

// Ordering a beam by (xi cell, radial cell) (stable radix sort; removed particles last) for the
// pipeline's buckets. Buffers of n entries: keys[2], vals[2]; tmp of cell_sort_temp_bytes(n).
struct CellSortBuf {
    unsigned* keys[2];
    int* vals[2];
    void* tmp;
    size_t tmp_bytes;
    int* nlive;                 // device: live particles of the last sort
};
size_t cell_sort_temp_bytes(long n);
// stage (7 x n) = cols sorted by cell, orig_stage = orig permuted the same way
cudaError_t cell_sort(const BeamArgs& B, double* cols, double* stage, int* orig, int* orig_stage,
                      const CellSortBuf& buf, cudaStream_t s);
cudaError_t fill_iota(int* p, long n, cudaStream_t s);
// dst (7 x n) = src in the caller's order: dst[c][orig[p]] = src[c][p]
cudaError_t unpermute7(const double* src, double* dst, const int* orig, long n, cudaStream_t s);
// start[g] = first live particle of the last sort in xi cells [g span - 1, g span + span - 2] (g < ngroups;
// width = span * M), start[ngroups] = nlive
cudaError_t group_starts(const CellSortBuf& buf, long nlive, int width, int ngroups, int* start, cudaStream_t s);

// ---------------------------------------------------------------- batched independent runs
// Many independent instances (each its own grid, box, plasma and beams) in one persistent launch: a
// CTA takes the next instance from a queue and runs all of it (Simulation::run: sweeps, moment sums,
// pushes) with its own slot of field / beam-source buffers. Instances are queued largest first.
constexpr int kBatchBeams = 2;

// The reverse pass of a pipelined run in one cooperative launch (qz_adjoint.cu): reverse sweeps on
// CTAs [0, nsweep) (step n on CTA (nsteps - 1 - n) % nsweep), warp workers elsewhere claiming layer
// tasks (n, b) for n = nsteps-1 .. -1: the beam-deposit adjoint of step n + 1 and the push adjoint of
// step n of bucket b. Inputs from the forward pipeline with recording: fields and trajectories of
// every step, the beams of every step (snap).
struct AdjPipeArgs {
    SweepArgs sw;
    int nsteps, nsweep;
    const double* fld;  size_t fld_slot;      // forward fields, slot n = step n
    const double* traj; size_t traj_slot;     // plasma trajectories, slot n (checkpoints when sw.traj_every > 1)
    const double* wrec;                       // W+ radial field per slice, slot n of fld_slot / 6 (or null)
    double* seg;        size_t seg_slot;      // sw.traj_every > 1: the recomputed states of one segment per
                                              // sweep CTA (traj_every x (6 + 5 ord) x npad each)
    double* lfld;       size_t lfld_slot;     // field-store adjoint of step n (zero before the launch)
    double* lbsrc;      size_t lbsrc_slot;    // beam-source adjoint of step n (zero before the launch)
    int nbeams;
    BeamArgs beam[kMaxBeams];                 // grid and box; the particle pointers are set per task
    int rigid[kMaxBeams], startup[kMaxBeams];
    const double* snap; size_t snap_step; long snap_off[kMaxBeams];
    double* lam; long lam_off[kMaxBeams];     // particle adjoint, 7 columns of n per beam (run order)
    double dt;
    int nbk;
    const int *bk_beam, *bk_start, *bk_end;
    const int* cmin;                          // [(nsteps + 1) * nbk] lowest live xi cell of bucket b at step n
    const int* pmax;                          // [nsteps * nbk] max over buckets <= b of (highest cell + 1)
    int* prog;                                // [nsteps] lowest slice finished by reverse sweep n (K)
    int* bdone;                               // [nbk] lowest step whose task finished (nsteps; -1 at the end)
    int* next;                                // [nsteps + 1] claimed tasks of layer l = nsteps - 1 - n (0)
    int* err;                                 // (site << 8) | 1 when a wait gave up (0)
    int* lo;                                  // layers below *lo have every task claimed (0)
    unsigned long long timeout_ns;
};
size_t adjoint_pipeline_smem_bytes(int M);
int adjoint_pipeline_max_grid(const AdjPipeArgs& P, int* sms);
cudaError_t launch_adjoint_pipeline(const AdjPipeArgs& P, int grid, cudaStream_t stream);
// per (step, bucket) the lowest and highest live xi cells of the snapshots (empty: INT_MAX / -2), and
// per step < nsteps the running maximum over buckets of (highest + 1)
cudaError_t launch_bucket_cells(const AdjPipeArgs& P, int* cmin, int* cmax, int* pmax, cudaStream_t stream);

// beam adjoints (qz_adjoint.cu); lam: 7 columns of n (x y px py pz xi w)
cudaError_t launch_sums_back(const BeamArgs& B, double gref, double xiref, const double* lamS, double* lam,
                             cudaStream_t stream);
cudaError_t launch_push_back(const BeamArgs& B, const double* fld, double* lam, double* lfld, double dt_kick,
                             double dt, int startup, cudaStream_t stream);
cudaError_t launch_deposit_back(const BeamArgs& B, const double* lbsrc, double* lam, cudaStream_t stream);

struct BatchInst {
    SweepArgs sw;                   // bsrc / fld / diag are the slot's, set by the kernel
    int modes;                      // 0, or 1 (the m = 1 sweep: M <= kSweepThreads)
    int nbeams;
    BeamArgs beam[kBatchBeams];     // grid pointers are set by the kernel (shared-memory copies)
    int rigid[kBatchBeams];
    double gref[kBatchBeams], xiref[kBatchBeams];
    double* mom;                    // (nsteps + 1, nbeams, 17)
};

struct BatchArgs {
    const BatchInst* inst;          // device array
    const int* order;               // queue order (largest first)
    int ninst;
    int nsteps;
    double dt;
    int ord;
    int with_m1;                    // some instances have modes = 1
    int with_ext;                   // some instances use the smoothing filter (the kernel variant with it)
    double *fld, *diag, *bsrc;      // per slot (= CTA)
    size_t fld_slot, diag_slot, bsrc_slot;
    int* next;                      // queue head (0)
    // optional, kBatchTrace words per instance (by instance index): the CTA that ran it, %globaltimer at
    // its start and end, ns in its sweeps, ns in its beam phases
    unsigned long long* trace;
};
constexpr int kBatchTrace = 5;

cudaError_t launch_batch(const BatchArgs& B, int grid, size_t smem, cudaStream_t stream);
int batch_max_grid(int ord, bool with_m1, bool with_ext, size_t smem, int* sms);
// the batch kernel for modes = 1 instances with 513..1024 nodes (1024 threads, qz_batch_m1w.cu): args points
// to a BatchArgs of args_size bytes; per_sm != nullptr asks only for the resident CTAs per SM
size_t batch_m1w_static_bytes();
cudaError_t launch_batch_m1w(const void* args, size_t args_size, int grid, size_t smem, cudaStream_t s, int* per_sm);

}  // namespace qzb
