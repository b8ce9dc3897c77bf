/* qz_b200.h -- C ABI of libqz_b200.so: the B200 hot path of QUARZ (quasi-static xi sweep,
 * beam deposit, field gather + Vay push, beam moments).
 *
 * Conventions
 *   - Every entry point returns qz_status: 0 = ok, > 0 = error (qz_last_error() has the text).
 *     No C++ exception crosses this boundary.
 *   - "dev" pointers are CUDA device pointers on the current device; "host" pointers are host
 *     memory. All arrays are FP64, LayoutRight (last index fastest), exactly the layouts of the
 *     reference's Kokkos Views:
 *        fld  (K, M, F_NC)  F_NC = 6 (m = 0) / 18 (m = 1)   src/FieldStore.hpp:9-13
 *        bsrc (K, M, B_NC)  B_NC = 5 / 15                   src/FieldStore.hpp:16-20
 *        diag (K, M, D_NC)  D_NC = 3 / 9                    src/Simulation.hpp:44
 *     k = slice (head first; internal xi = xi_min + k dxi, xi_internal = -xi_user), j = node.
 *   - `stream` is a cudaStream_t passed as void* (NULL: the legacy default stream).
 *   - Handles are not thread-safe: one handle per host thread / stream.
 */
#ifndef QZ_B200_H
#define QZ_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int qz_status;
enum {
    QZ_OK = 0,
    QZ_ERR_ARG = 1,          /* invalid argument (null pointer, size, option) */
    QZ_ERR_CUDA = 2,         /* a CUDA call failed */
    QZ_ERR_UNSUPPORTED = 3,  /* option not on this path (e.g. laser, ionization) */
    QZ_ERR_NOMEM = 4,        /* device or host allocation failed */
    QZ_ERR_SIZE = 5          /* problem too large for this kernel configuration */
};

/* text of the last error of the calling thread ("" if none) */
const char* qz_last_error(void);
/* library version string */
const char* qz_version(void);

/* ------------------------------------------------------------------ radial grid + operators
 * Replaces RadialGrid::RadialGrid(nodes) + RadialGrid::finalize (src/RadialGrid.cpp:104-148) and
 * FieldSolver::FieldSolver (src/FieldSolver.cpp:113-179): hat-function volumes, the tridiagonal
 * rows of L0 / L1D / L1F / L2D and the gradient stencils, uploaded to the device.
 * nodes: host, M values, 0 = r_0 < r_1 < ... < r_{M-1} = R. */
typedef struct qz_grid qz_grid;
qz_status qz_grid_create(const double* nodes_host, int M, qz_grid** out);
qz_status qz_grid_destroy(qz_grid* g);
/* host copies of V_j (M) and, for op = 0..3 (L0, L1D, L1F, L2D), the rows a, b, c (M each) */
qz_status qz_grid_volumes(const qz_grid* g, double* V_host);
qz_status qz_grid_operator(const qz_grid* g, int op, double* a_host, double* b_host, double* c_host,
                           double* flux_coef);

/* ------------------------------------------------------------------ the xi sweep
 * Replaces Simulation::step_fields' per-slice chain (src/Simulation.cpp:636-795) with the plasma of
 * PlasmaSpecies (load src/PlasmaSpecies.cpp:202-295, deposit :409-478, deposit_rho :480-506,
 * deposit_S :508-559, push :561-668) and the field solves of Simulation::solve_slice_fields
 * (src/Simulation.cpp:797-819). Single rank, constant dxi (no sub-slicing), no laser / ionization.
 * The radial smoothing of the plasma sources (plasma.smooth_length, src/Simulation.cpp:63-66, :685-690,
 * :810-835; FieldSolver::set_filter / filter, src/FieldSolver.cpp:111-161) is on this path for modes 0 and 1. */
typedef struct {
    double q, m;             /* <name>.charge, <name>.mass */
    int ppc, ntheta;         /* <name>.ppc, <name>.ntheta */
    int mobile;              /* <name>.mobile */
    double density;          /* <name>.density factor */
    double rmax;             /* plasma.rmax (use 1e300 for none) */
    double channel_depth, channel_radius;   /* plasma.radial = channel when channel_radius > 0 */
} qz_species;

typedef struct {
    int modes;               /* 0: m = 0 only; 1: m = 0 and 1 */
    int picard;              /* solver.picard */
    int ab_order;            /* pusher.ab_order, 1..5 */
    double delta_min;        /* pusher.delta_min */
    double max_qsa;          /* pusher.max_qsa_factor */
    double xi_min;           /* internal xi of slice 0 (= -xi.max) */
    double dxi;              /* xi.step */
    int K;                   /* slices */
    int ngp;                 /* beams.xi_shape = ngp */
    int neutralize;          /* plasma.neutralize */
    int nspecies;
    qz_species species[4];
    double smooth_length;    /* plasma.smooth_length (0: off) */
    double max_cells_per_step; /* pusher.max_cells_per_step: adaptive sub-slicing with variable-step AB
                                  (src/Simulation.cpp:755-781, :837-847; 0: off); modes = 0, without the
                                  smoothing filter, not in stages or the adjoint */
    int substep_max;         /* pusher.substep_max (0: the reference's default, 64) */
} qz_sweep_params;

typedef struct {
    unsigned long long lost;      /* plasma particles removed (trapped or beyond the wall; the reference's
                                     lost counter, src/PlasmaSpecies.cpp:639-655) */
    unsigned long long nonfinite; /* deposits (per slice and array) that met a NaN or Inf contribution: the
                                     array's values of that slice are NaN */
    unsigned long long trapped;   /* of lost: removed as trapped (Delta <= delta_min or gamma > max_qsa Delta) */
    unsigned long long giveup;    /* pipelined runs that ended because a bounded wait timed out */
    unsigned long long subslices; /* sub-slices beyond the regular slices (adaptive sub-slicing; the
                                     reference's "extra sub-slices", src/Simulation.cpp:782) */
} qz_counters;

typedef struct qz_sweep qz_sweep;
qz_status qz_sweep_create(const qz_grid* g, const qz_sweep_params* p, qz_sweep** out);
qz_status qz_sweep_destroy(qz_sweep* s);
/* One sweep. bsrc (dev, read), fld / diag (dev, written), counters (host, optional, accumulated). */
qz_status qz_sweep_run(qz_sweep* s, const double* bsrc_dev, double* fld_dev, double* diag_dev,
                       qz_counters* counters_host, void* stream);
/* plasma state after the last sweep: out_host (6, n) = x y px py Delta w; returns n in *n */
qz_status qz_sweep_plasma(qz_sweep* s, double* out_host, int cap, int* n);

/* The plasma a slab of a xi-pipelined run hands to the next one (the plasma part of the message of
   Simulation::make_message, src/Simulation.cpp:851-870, and PlasmaSpecies::pack_state,
   src/PlasmaSpecies.cpp:317-334): the sweep's np particles with stride npad as (6 + 5 order) device rows
   x y px py Delta w, then the Adams-Bashforth history h[m][v] (the force m pushes ago, v = d/dxi of x, y,
   px, py, Delta), and whether the particles have been pushed (their history is filled). */
typedef struct {
    double* state;
    int np, npad, order;
    int pushed;
} qz_plasma_state;
/* the shape of a sweep's plasma state (allocate (6 + 5 order) x npad doubles) */
qz_status qz_sweep_state_shape(qz_sweep* s, int* np, int* npad, int* order);
/* One sweep over a slab of the box, a stage of the reference's xi-pipelined multi-rank run
   (Simulation::step_fields with a message, src/Simulation.cpp:714-731, :755, and Simulation::run,
   :1380-1400). The sweep s was created with the slab's slices (K and xi_min of the slab). in: the
   plasma entering the slab's first slice (NULL: the fresh plasma of the box head); bguard (dev, M x
   B_NC of the slab's sweep, NULL: none): the beam sources of the slice just ahead of the slab (the
   upstream slab's last row, Simulation::set_guard, :459-465); out (NULL: none): receives the plasma
   after the push of the slab's last slice, the state entering the next slab. A slab that takes a guard
   or hands its plasma on needs the ngp xi shape; modes = 0, without the smoothing filter. Two or more
   slabs run one after the other give the fields and plasma of the whole sweep bit for bit. */
qz_status qz_sweep_run_stage(qz_sweep* s, const double* bsrc_dev, const double* bguard_dev, const qz_plasma_state* in,
                             double* fld_dev, double* diag_dev, qz_plasma_state* out, qz_counters* counters_host,
                             void* stream);
/* per-phase clock cycles of the last run, 16 counters: [0] prologue, [1] psi/E_z/B_z phase, [2] S+ deposit,
   [3] B+ phase, [4] store + push + deposit, [5..8] parts of phase 1; enable = 1 turns the counters on for
   later runs */
qz_status qz_sweep_timing(qz_sweep* s, int enable, unsigned long long* cycles16_host);

/* ------------------------------------------------------------------ beams
 * A beam is a view of 7 device columns (x y px py pz xi w), internal xi.
 * Replaces Beam::deposit (src/Beam.cpp:725-785), Beam::push / advance with the Vay pusher
 * (src/Beam.cpp:900-905, :948-1131) and Beam::sums (src/Beam.cpp:1133-1155). */
typedef struct {
    double *x, *y, *px, *py, *pz, *xi, *w;
    int64_t n;
    double q, m;
    int pusher;              /* <name>.pusher (src/Beam.cpp:72-78): 0 vay (default, also when left zero),
                                1 boris, 2 hc (Higuera-Cary), 3 imp (implicit midpoint); imp_rr is not here */
} qz_beam_view;

typedef struct {
    double xi_min, dxi;
    int K;
    int ngp;
    int modes;
} qz_box;

/* adds the beam's sources to bsrc (dev, (K, M, B_NC)); bsrc is NOT cleared */
qz_status qz_beam_deposit(const qz_grid* g, const qz_beam_view* b, const qz_box* box, double* bsrc_dev,
                          void* stream);
/* Exact beam sources outside qz_sim (a staged run): the node quanta of the two-limb format qz_sim's m = 0
   runs use (qz_sim_set_exact), for up to nparticles beam particles whose weights satisfy
   sum over beams of max |w q| <= wq. qz_beam_deposit_fx adds a beam into bsrc2 (dev, 2 x K x M x B_NC0:
   the high limbs, then the low limbs; zero it first) with them; qz_sweep_set_exact_sources(s, fx) makes
   s read its bsrc, and a stage's guard row (2 x M x B_NC0), in that format (NULL: plain doubles again).
   Sums of integer limbs do not depend on the order of the adds, so slabs that deposit their own particles
   give the beam sources of the whole box bit for bit: a staged run then equals the single-GPU run in its
   fields and particles, as the reference's pipelined MPI run does (README.md:1755-1758). modes = 0.
   No counterpart in the reference (its deposits are atomic FP64 adds). */
typedef struct qz_fx qz_fx;
qz_status qz_fx_create(const qz_grid* g, double dxi, double wq, int64_t nparticles, qz_fx** out);
qz_status qz_fx_destroy(qz_fx* fx);
qz_status qz_beam_deposit_fx(const qz_grid* g, const qz_beam_view* b, const qz_box* box, const qz_fx* fx,
                             double* bsrc2_dev, void* stream);
qz_status qz_sweep_set_exact_sources(qz_sweep* s, const qz_fx* fx);
/* advance by dt (move = 1) or the explicit start-up kick (move = 0) with the fields fld (dev) */
qz_status qz_beam_advance(const qz_grid* g, qz_beam_view* b, const qz_box* box, const double* fld_dev,
                          double dt_kick, double dt_drift, int move, void* stream);
/* Beam::push: start-up half kick when *started == 0 (then *started = 1), then a full step. */
qz_status qz_beam_push(const qz_grid* g, qz_beam_view* b, const qz_box* box, const double* fld_dev,
                       double dt_kick, double dt_drift, int* started, void* stream);
/* Beam::push followed by Beam::deposit of the moved particle into bsrc_next (dev, not cleared):
   the two passes of consecutive time steps in one pass over the particles */
qz_status qz_beam_push_deposit(const qz_grid* g, qz_beam_view* b, const qz_box* box, const double* fld_dev,
                               double dt_kick, double dt_drift, int* started, double* bsrc_next_dev,
                               void* stream);
/* A noise-free rigid beam deposited directly on the grid (<name>.analytic = 1, src/Beam.cpp:183-203):
   rho = q n0 f(xi) exp(-|x_perp - c(xi)|^2 / 2 sigma_r^2) moving at v_z(gamma), f gaussian (sigma_xi) or
   flat-top (length), centroid c = (x0, y0) + (x_slope, y_slope) (xi - xi0). Internal xi for xi0 and xi_cut
   (slices with xi < xi_cut get nothing; -1e300 for none) and internal slopes (d x_c / d xi_internal). */
typedef struct {
    double q, n0, sigma_r;
    double xi0, sigma_xi;
    int flattop;
    double length;
    double xi_cut;
    double x0, y0, x_slope, y_slope;
    double gamma;
} qz_analytic_beam;

/* Beam::deposit_analytic (src/Beam.cpp:236-279): adds the beam's sources to bsrc (dev, (K, M, B_NC), not
   cleared); offsets and slopes need box->modes = 1 */
qz_status qz_beam_deposit_analytic(const qz_grid* g, const qz_analytic_beam* b, const qz_box* box, double* bsrc_dev,
                                   void* stream);

/* Beam::slice_sums (src/Beam.cpp:1195-1217), the per-slice beam diagnostics of output.beam_slices: nbins
   equal bins of the USER xi (= -internal xi) over [lo, hi), 9 sums per bin into out_dev (9 x nbins, dev,
   overwritten): w, w x, w y, w x^2, w y^2, w gamma, w px, w px^2, w x px. The reference copies the beam to
   the host for this; here it stays on the device. FP64 atomics: the order of summation, and so the last
   bits, can differ from call to call. */
qz_status qz_beam_slice_sums(const qz_beam_view* b, double lo, double hi, int nbins, double* out_dev, void* stream);

/* Simulation::write_fields (src/Simulation.cpp:878-993): the field file fields_NNNNNN.bin, version 3, of one
   sweep, as the reference writes it without output groups: int32 {3, M, K, mode1}, float64 t, r[M], xi[K]
   (user xi, increasing: the head of the box is the last row), int32 ncomp, then ncomp x {char name[16],
   float64 data[K][M]}; names psi ez er eth br bth bz ne ni rhob, and with modes = 1 <name>_c / <name>_s of
   psi ez bz ne ni rhob er eth br bth. fld (K, M, F_NC), diag (K, M, D_NC), bsrc (K, M, B_NC; NULL writes a
   zero rhob) are device arrays when on_device != 0, else host arrays; nodes_host: the M radial nodes.
   Columns of parts this library does not build are not written: the densities of ionizable species
   (nz_<species>) and the laser envelope (a_re, a_im). */
qz_status qz_write_fields(const char* path, const double* nodes_host, int M, const qz_box* box, double t,
                          const double* fld, const double* diag, const double* bsrc, int on_device);

/* the 17 moment sums of Beam::sums into out17 (dev); deterministic order */
qz_status qz_beam_sums(const qz_beam_view* b, double gref, double xiref, double* out17_dev, void* stream);
/* qz_beam_sums without any device allocation, for callers that cannot allocate (a host whose
   device memory all belongs to its own pool allocator; a step loop that cannot take the device-wide
   synchronisation of cudaFree). No counterpart in the reference: it is an addition of this library.
   The partial sums live in a static device array of 17 x 592 doubles (80,512 bytes per device),
   enough for any n: the reduction uses at most 592 blocks. A request for more rows than that fails
   with QZ_ERR_SIZE. The first call on each device does the set-up (looks up the array's address with
   that device current) and should be made before any stream capture. Nothing has to be zeroed
   beforehand. Calls in flight at the same time on one device share the array and race: order
   them on one stream or serialise them on the host. Same result as qz_beam_sums. */
qz_status qz_beam_sums_noalloc(const qz_beam_view* b, double gref, double xiref, double* out17_dev, void* stream);

/* The reference's gaussian generator (Beam::init_gaussian, src/Beam.cpp:483-570) on the host, with
   the same std::mt19937_64 / std::normal_distribution stream. out_host: n x 7 (internal xi).
   sxi <= 0 selects the flattop profile of length -sxi. Returns the particle count in *n. */
qz_status qz_sample_gaussian(double n0, double sigma_r, double xi0_internal, double sigma_xi, double gamma0,
                             double espread, double emit_n, double cut, double x0, double y0, double xs_internal,
                             double ys_internal, double xp0, double yp0, int64_t nparticles, int nsym,
                             int mirror_y, uint64_t seed, double xi_cut_internal, double* out_host,
                             double* gref, double* xiref, int64_t* n);

/* ------------------------------------------------------------------ whole time steps
 * Simulation::run's loop (src/Simulation.cpp:1370-1448) for constant dt: per step one sweep and
 * (except after the last sweep) one push of every non-rigid beam, with the next step's beam
 * deposit fused into the push. Beams are given as HOST arrays (n x 7) and copied in; results
 * (fields, moments, final particles) are copied back. */
typedef struct qz_sim qz_sim;
qz_status qz_sim_create(const qz_grid* g, const qz_sweep_params* p, qz_sim** out);
qz_status qz_sim_destroy(qz_sim* s);
qz_status qz_sim_add_beam(qz_sim* s, const double* p7_host, int64_t n, double q, double m, int rigid,
                          double gref, double xiref);
/* an analytic rigid beam (qz_beam_deposit_analytic): deposited once into a static source array that every
   sweep of the sim adds to the pushed beams' sources. It has no particles, so it is not one of the sim's
   beams: nbeams, the moments and qz_sim_beam count only the particle beams. */
qz_status qz_sim_add_analytic_beam(qz_sim* s, const qz_analytic_beam* b);
/* the pusher of particle beam b (qz_beam_view.pusher). A run with a pusher other than Vay goes step by step
   (the time-step pipeline pushes with Vay); the adjoint refuses it. */
qz_status qz_sim_set_beam_pusher(qz_sim* s, int b, int pusher);
/* qz_beam_slice_sums of particle beam b of the sim as it stands (after the last run), into out_host
   (9 x nbins, host) */
qz_status qz_sim_beam_slice_sums(qz_sim* s, int b, double lo, double hi, int nbins, double* out_host);
/* qz_write_fields of the sim's last sweep at time t: its fields and diagnostics, and as rhob the beam
   sources re-deposited from the beams as they stand (not pushed after that sweep) plus the analytic
   ones. The re-deposit sums in another order than the deposit the sweep read, so rhob agrees with
   the sources of that sweep to rounding, not bit for bit. */
qz_status qz_sim_write_fields(qz_sim* s, double t, const char* path);
/* run nsteps (nsteps+1 sweeps); moments_host: (nsteps+1, nbeams, 17) or NULL.
   By default (modes 0 or 1, at most 4 beams) the whole run is ONE cooperative launch in which the sweeps of
   consecutive steps run concurrently on different SMs, each slice gated on the beam pushes of the
   previous step that can deposit into it, and the pushes are gated on the fields they gather: the
   same arithmetic as the step-by-step loop of Simulation::run (src/Simulation.cpp:1370-1448), with
   the beam deposits summed in a different order. The beams are kept in xi-cell order on the device
   (qz_sim_beam returns them in the caller's order). */
qz_status qz_sim_run(qz_sim* s, int nsteps, double dt, double* moments_host, void* stream);
/* Schedule of qz_sim_run: pipelined = 0 runs the steps one kernel after another (one sweep launch,
   then one push launch per beam, per step); sweep_ctas = CTAs running sweeps (0: one per step, up to
   the SMs left for at least max(8, 2 SMs/5) push CTAs); a push task (bucket) holds at most `bucket`
   particles (0: 512) of at most `span` neighbouring xi cells (0: 1) -- the next step's sweep trails
   the previous one by about span + 5 slices; timeout_s = limit of every wait inside the pipelined
   launch (0: keep, default 20 s), after which the launch ends and qz_sim_run returns QZ_ERR_CUDA.
   No counterpart in the reference (its own pipelining over time steps is across MPI ranks,
   src/Simulation.cpp:851-870). */
qz_status qz_sim_set_schedule(qz_sim* s, int pipelined, int sweep_ctas, int bucket, int span, double timeout_s);
/* exact = 1 (the default): the beam deposits of m = 0 runs (up to 2^25 beam particles) are exact integer
   sums (two integer-valued limbs per value, each sum below 2^53, added with FP64 reductions), so runs
   repeat bit for bit; exact = 0: FP64 reductions of the values, faster (one reduction per value and half
   the beam-source memory) but their summation order, and so the last bits, vary from run to run. No
   counterpart in the reference (its OpenMP and GPU deposits use atomic adds). */
qz_status qz_sim_set_exact(qz_sim* s, int exact);
/* The next run starts every beam's leapfrog again (the start-up half kick of Beam::push,
   src/Beam.cpp:903, src/Simulation.cpp:1434-1436): a new run from beams set with qz_sim_set_beam, which
   otherwise continue where the last run left them. */
qz_status qz_sim_restart(qz_sim* s);
/* the schedule of the last qz_sim_run: grid, sweep CTAs, push CTAs, ring slots, buckets, bucket size,
   pipelined (1/0), cell span of a bucket */
qz_status qz_sim_schedule(qz_sim* s, int* info8);
/* GPU time (ms, CUDA events on the run's stream) of the parts of the last pipelined run: [0] set-up
   (beam ordering, buckets, step-0 beam deposit), [1] the pipelined kernel, [2] moments and copies. */
qz_status qz_sim_times(qz_sim* s, double* ms3);
/* Replace beam b's particles (7 x n SoA in the caller's order, x y px py pz xi w) from device memory
   (on_device = 1) or host memory; the started flag of the leapfrog is kept. */
qz_status qz_sim_set_beam(qz_sim* s, int b, const double* cols7, int on_device, void* stream);
/* Timeline of the last pipelined run, 22 values per step n: GPU clock (ns, %globaltimer) at the start
   and the end of sweep n, when it had stored 1/16, 2/16, ... 16/16 of the slices, then its longest
   wait for beam-source rows (ns, bucket, row, the bucket's highest cell); after the steps 6 totals of
   the push workers (warps): tasks, scans that found no ready task, claims lost to another worker, ns
   spent in tasks, ns waiting for a ready task, ns in the moments passes. Up to cap values;
   *n = 22 (nsteps+1) + 6. enable = 1 records it in later runs. */
qz_status qz_sim_trace(qz_sim* s, int enable, unsigned long long* out, int cap, int* n);
/* qz_sim_run with the beams in HOST memory: copies every beam in (cols_host[b]: 7 x n SoA in the
   caller's order, x y px py pz xi w), runs nsteps, and copies the particles back into cols_host in
   the same order. Pinned host memory makes the copies asynchronous. */
qz_status qz_sim_run_host(qz_sim* s, int nsteps, double dt, double* const* cols_host, double* moments_host,
                          void* stream);
/* copy out the field store / diagnostics of the last sweep (host, K*M*F_NC / K*M*D_NC) */
qz_status qz_sim_fields(qz_sim* s, double* fld_host, double* diag_host);
/* copy out beam b's particles (host, n x 7) */
qz_status qz_sim_beam(qz_sim* s, int b, double* p7_host);
qz_status qz_sim_counters(qz_sim* s, qz_counters* out);
/* One time step with HOST beam buffers, the per-step call of an adapter whose beams live in host
   memory (Simulation::step_fields + Beam::push on host Views, src/Simulation.cpp:1396-1442): copies
   every beam in (cols_host[b]: 7 x n SoA, x y px py pz xi w), deposits all beams, sweeps, computes
   the moments (moments_host: nbeams x 17, or NULL), pushes the non-rigid beams when push != 0, and
   copies the particles back into cols_host. Pinned host memory makes the copies asynchronous. */
qz_status qz_sim_step_host(qz_sim* s, double* const* cols_host, double dt_kick, double dt_drift, int push,
                           double* moments_host, void* stream);

/* The adjoint of a run (no reference counterpart; modes = 0, linear or ngp xi shape, one mobile plasma
 * species with at most 512 particles per slice, M <= 512). Runs nsteps like qz_sim_run (step by step,
 * keeping the beams of every step on the device; the beams must not have been pushed yet), then the
 * reverse pass: the beam pushes, sweeps and beam deposits of every step in reverse order.
 *   lamS_host  (nbeams, 17): the adjoint of the last step's moment sums (Beam::sums order), i.e. J is
 *              sum(lamS * sums) or the linearisation of a function of the sums
 *   lam_host   per beam a 7 x n SoA host array (x y px py pz xi w, the caller's particle order):
 *              receives dJ / d(initial particle)
 *   mom_host   optional ((nsteps+1), nbeams, 17): the forward's moment sums
 *   ms2        optional: the forward's and the reverse pass's device time (ms)
 * The sim ends at the last step, as after qz_sim_run. */
qz_status qz_sim_adjoint(qz_sim* s, int nsteps, double dt, const double* lamS_host, double* const* lam_host,
                         double* mom_host, double* ms2, void* stream);
/* The same with the seed computed from the forward's moment sums: after the forward, fn(moments
   ((nsteps+1), nbeams, 17, host), nsteps, nbeams, lamS (nbeams x 17, to fill), user) is called once on
   the calling thread -- for an objective such as the witness energy spread, whose linearisation
   depends on the last step's sums, without a second forward run. */
typedef void (*qz_adjoint_seed_fn)(const double* moments, int nsteps, int nbeams, double* lamS, void* user);
qz_status qz_sim_adjoint_fn(qz_sim* s, int nsteps, double dt, qz_adjoint_seed_fn fn, void* user,
                            double* const* lam_host, double* mom_host, double* ms2, void* stream);
/* Slice checkpointing of the pipelined adjoint: the forward keeps the plasma state of every C-th slice
   of each step (and the W+ radial field of every slice), and the reverse sweep pushes the plasma again
   from those checkpoints one segment of C slices at a time, reproducing the forward's states bit for
   bit. every = 0 (the default): C = ceil(sqrt(K)); every = 1: the state of every slice is kept (no
   recomputation; memory K / C times larger); every > 1: that C (at most K). The step-by-step adjoint
   keeps one step's states at a time and ignores it. No counterpart in the reference. */
qz_status qz_sim_set_adjoint_checkpoint(qz_sim* s, int every);
/* Clock cycles per phase of the run's sweeps (qz_sweep_timing of the sim's sweep): 16 counters,
   accumulated by thread 0 of every sweep while enabled (all sweeps of a pipelined run together);
   0..8 the forward sweep's phases, 9..15 those of the step-by-step adjoint's reverse sweep.
   cycles16 may be NULL. */
qz_status qz_sim_timing(qz_sim* s, int enable, unsigned long long* cycles16);

/* ------------------------------------------------------------------ batched independent runs
 * A parameter scan: many independent small runs (each its own grid, box, plasma and up to 2 beams,
 * modes 0 or 1 (M <= 1024 for modes 1), one AB order for all) in ONE persistent launch, a CTA per
 * instance taken from a queue (largest first); m = 1 instances with more than 512 nodes run after it in a
 * second launch of 1024-thread CTAs. No counterpart in the reference, which runs one deck per process; each instance
 * is Simulation::run (src/Simulation.cpp:1370-1448) for constant dt. */
typedef struct qz_batch qz_batch;
qz_status qz_batch_create(qz_batch** out);
qz_status qz_batch_destroy(qz_batch* b);
/* adds an instance: its grid nodes, sweep parameters and beams (host rows of 7: x y px py pz xi w,
   internal xi); *index = its position */
qz_status qz_batch_add(qz_batch* b, const double* nodes, int M, const qz_sweep_params* p, int nbeams,
                       const double* const* p7_host, const int64_t* n, const double* q, const double* m,
                       const int* rigid, const double* gref, const double* xiref, int* index);
/* runs every instance nsteps (nsteps+1 sweeps); moments_host: for each instance in order of addition,
   (nsteps+1, nbeams, 17) moment sums, concatenated; the beams stay on the device (advanced) */
qz_status qz_batch_run(qz_batch* b, int nsteps, double dt, double* moments_host, void* stream);
/* instances, CTAs of the last run, its kernel time (ms), 0 */
qz_status qz_batch_info(qz_batch* b, double* out4);
/* The tuning of instance `index` (from qz_batch_add): its shared-memory layout for modes = 0, a bit set
   (1: double-buffered slice sources, 2: per-node constants in shared memory, 4: the copy of plasma kept in
   global memory, np > 512), or -1 to keep the current one; and its cost, the key of the largest-first
   queue, or <= 0 to keep it. qz_batch_add picks the fastest layout that fits and the estimate
   K (M + 4 np) + 2 N_beam; the autotuner (quarz_b200.tune) measures both instead. Fails with QZ_ERR_SIZE
   for a layout that does not fit the device's shared memory. qz_batch_tuning reads them back.
   No counterpart in the reference. */
qz_status qz_batch_set_tuning(qz_batch* b, int index, int layout, double cost);
qz_status qz_batch_tuning(qz_batch* b, int index, int* layout, double* cost);
/* Per-instance timeline of the next runs (enable = 1; 0 stops recording): qz_batch_trace then gives, for
   each instance of the last run in qz_batch_add order, 5 values: the CTA that ran it, its start and end
   (ms from the first start), ms in its sweeps, ms in its beam phases (moments, pushes, deposits). out
   holds n >= the instance count rows. The autotuner (quarz_b200.tune) fits its cost model to these
   times. No counterpart in the reference (it runs a scan as separate processes). */
qz_status qz_batch_set_trace(qz_batch* b, int enable);
qz_status qz_batch_trace(qz_batch* b, double* out, int n);

#ifdef __cplusplus
}
#endif
#endif
