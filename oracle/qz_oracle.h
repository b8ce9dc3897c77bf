/* qz_oracle.h -- CPU restatement of the QUARZ hot path, used ONLY as a test checker.
 *
 * TEST INFRASTRUCTURE. Nothing in the product (quarz_b200/) links, loads or calls this
 * library. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / --impl
 * reference leg may use it, and only to check or to time the reference algorithm on the
 * host cores.
 *
 * What it restates (QUARZ v2.0.0, file:line within the reference project):
 *   radial grid          src/RadialGrid.cpp:14-86 (generators), :106-148 (volumes)
 *   field operators      src/FieldSolver.cpp:90-103 (fv_rows), :113-179 (L0/L1D/L1F/L2D, stencils)
 *   solve / gradients    src/FieldSolver.cpp:172-219
 *   tridiagonal          src/Tridiag.cpp:28-162 (Thomas, PCR, partition)
 *   plasma species      src/PlasmaSpecies.cpp:14-48 (AB), :57-89 (geometry/gather), :202-295 (load),
 *                        :409-478 (deposit), :480-506 (deposit_rho), :508-559 (deposit_S), :561-668 (push)
 *   sweep                src/Simulation.cpp:394-457 (zero/combine), :477-633 (W+, Bz, B+, store),
 *                        :636-795 (step_fields), :797-819 (solve_slice_fields), :1370-1448 (run)
 *   beam                 src/Beam.cpp:483-570 (gaussian sampler), :725-785 (deposit), :900-905 (push),
 *                        :948-1131 (advance, Vay only), :1133-1192 (sums / from_sums)
 *   pushers              src/Pushers.hpp:36-68 (gamma2_root, solve_implicit, vay)
 *   adjoint (m = 0)      qz_oracle_adj.c: the reverse of all of the above for one run (no
 *                        reference counterpart; pinned by central differences of this forward)
 *   mode sums            src/SliceData.hpp:70-83
 *
 * Parity is pinned against the reference's own unit tests (tests/test_solvers.cpp,
 * tests/test_pushers.cpp, tests/test_ab.cpp) and its stored validation numbers
 * (validation/reference_full.txt, reference_quick.txt); see tests/test_oracle_*.py.
 *
 * Arithmetic: FP64 throughout, single-threaded, particles in index order (the reference's
 * serial summation order); build with -ffp-contract=off so every expression rounds as written.
 */
#ifndef QZ_ORACLE_H
#define QZ_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- random numbers used by the reference's beam generator (inputs only) ---- */
typedef struct { uint64_t mt[312]; int idx; int have_saved; double saved; } qzo_rng;
void     qzo_rng_seed(qzo_rng* g, uint64_t seed);
uint64_t qzo_rng_u64(qzo_rng* g);
double   qzo_rng_canonical(qzo_rng* g);      /* uniform [0,1) with 53 bits */
double   qzo_rng_normal(qzo_rng* g);         /* N(0,1), polar method with one cached variate */

/* ---- grid generators ---- */
int qzo_make_uniform(double R, double dr, double* out, int cap);
int qzo_make_regions(double R, const double* ends, const double* hs, int nreg, double max_ratio,
                     double* out, int cap);

/* ---- stand-alone pieces for unit tests ---- */
enum { QZO_THOMAS = 0, QZO_PCR = 1, QZO_PARTITION = 2 };
int qzo_tridiag(int method, int M, const double* a, const double* b, const double* c, const double* d,
                double* x);
/* (L_op - chi) f = scale*rhs on the grid given by nodes; op: 0 L0, 1 L1D, 2 L1F, 3 L2D.
   chi/wall may be NULL. */
int qzo_field_solve(const double* nodes, int M, int op, int method, const double* rhs, const double* chi,
                    const double* wall, double scale, double* f);
/* operator rows (a,b,c of length M each) and gradient stencils (gm,g0,gp,ir of length M) */
int qzo_operator_rows(const double* nodes, int M, int op, double* a, double* b, double* c, double* flux_coef);
int qzo_stencils(const double* nodes, int M, double* gm, double* g0, double* gp, double* ir);
int qzo_grid_volumes(const double* nodes, int M, double* V);
void qzo_vay(const double u[3], const double E[3], const double B[3], double eps, double out[3]);
/* the beam pushers of src/Pushers.hpp on n momenta (3 per row) with eps per row: kind 0 vay, 1 boris,
   2 higuera-cary, 3 imp */
int qzo_push(int kind, long n, const double* u, const double* E, const double* B, const double* eps, double* out);
int qzo_ab_coeffs(int order, double* c);
int qzo_ab_variable(int order, const double* t, double h, double* c);

/* ---- whole-deck simulation ---- */
typedef struct {
    int modes;            /* 0 or 1 */
    int picard;           /* B+ Picard iterations (1 for m = 0) */
    int ab_order;         /* 1..5 */
    double delta_min, max_qsa;
    double xi_min, dxi;   /* internal xi of slice 0, slice spacing */
    int K;                /* slices */
    int ngp;              /* beams.xi_shape = ngp */
    int tridiag;          /* QZO_THOMAS / PCR / PARTITION */
    int neutralize;
    double smooth_length; /* plasma.smooth_length: radial smoothing of the plasma sources (0: off) */
    double max_cells;     /* pusher.max_cells_per_step: adaptive sub-slicing (0: off) */
    int substep_max;      /* pusher.substep_max */
} qzo_params;

typedef struct {
    double q, m;
    int ppc, ntheta;
    int mobile;
    double density;       /* <name>.density factor */
    double rmax;          /* plasma.rmax (1e300: none) */
    double channel_depth, channel_radius;   /* radial = channel when channel_radius > 0 */
} qzo_species_params;

typedef struct qzo_sim qzo_sim;

qzo_sim* qzo_sim_create(const qzo_params* p, const double* nodes, int M);
void     qzo_sim_destroy(qzo_sim* s);
int      qzo_sim_add_species(qzo_sim* s, const qzo_species_params* sp);
/* particles: n x 7 (x y px py pz xi w), internal xi; gref/xiref as computed by the generator */
int      qzo_sim_add_beam(qzo_sim* s, const double* p7, long n, double q, double m, int rigid,
                          double gref, double xiref);
/* sample the reference's gaussian beam; writes the 7-column particles (internal xi) to out
   (capacity n*7) and gref/xiref; returns the number of particles */
long     qzo_sample_gaussian(double n0, double sr, double xi0_int, double sxi, double gamma0, double espread,
                             double emit, double cut, double cx0, double cy0, double cxs, double cys,
                             double xp0, double yp0, long np, int nrot, int mirror, uint64_t seed, double xcut,
                             double* out, double* gref, double* xiref);
/* a noise-free rigid beam deposited on the grid (<name>.analytic = 1, src/Beam.cpp:183-203):
   charge q, density n0, radius sigma_r, centre xi0 (internal), sigma_xi (gaussian) or length (flattop = 1),
   head cut xi_cut (internal; -1e300 for none), centroid (x0, y0) + (xs, ys) (xi - xi0), gamma. No particles:
   its moment sums are zero and it is never pushed. */
int      qzo_sim_add_analytic_beam(qzo_sim* s, double q, double n0, double sigma_r, double xi0, double sigma_xi,
                                   int flattop, double length, double xi_cut, double x0, double y0, double xs,
                                   double ys, double gamma);
/* the pusher of beam b (<name>.pusher, src/Beam.cpp:72-78): 0 vay (default), 1 boris, 2 hc, 3 imp */
int      qzo_sim_set_beam_pusher(qzo_sim* s, int b, int kind);
/* the radial smoothing filter f <- (1 - div a^2 grad)^{-1} f of angular number n = 0, 1, 2 with a^2 = a2 in
   every cell (FieldSolver::set_filter / filter, src/FieldSolver.cpp:111-161), in place on f (M) */
int      qzo_filter(const double* nodes, int M, double a2, int n, double* f);
/* e^{-z} I0(z), e^{-z} I1(z) by the polynomial approximations of Abramowitz & Stegun 9.8.1-9.8.4 */
void     qzo_bessel_i01_scaled(double z, double* i0, double* i1);
/* one quasi-static sweep (beam deposit + plasma load + sweep), as Simulation::step_fields */
/* sub-slices beyond the regular slices so far (adaptive sub-slicing) */
long     qzo_sim_subslices(const qzo_sim* s);
int      qzo_sim_step_fields(qzo_sim* s, double t);
/* beam push of every non-rigid beam */
int      qzo_sim_push_beams(qzo_sim* s, double dt_kick, double dt_drift);
/* 17 moment sums of beam b (Beam::sums) */
int      qzo_sim_beam_sums(const qzo_sim* s, int b, double out[17]);
int      qzo_sim_beam_get(const qzo_sim* s, int b, double* p7);   /* n x 7 copy out */
/* Beam::slice_sums (src/Beam.cpp:1195-1217) of n x 7 particle rows: 9 sums per bin of the user xi in [lo, hi) */
int      qzo_slice_sums(const double* p7, long n, double lo, double hi, int nbins, double* out);
long     qzo_sim_beam_count(const qzo_sim* s, int b);
/* field store (K, M, F_NC), beam sources (K, M, B_NC), diagnostics (K, M, D_NC): read-only views */
const double* qzo_sim_fld(const qzo_sim* s);
const double* qzo_sim_bsrc(const qzo_sim* s);
const double* qzo_sim_diag(const qzo_sim* s);
long     qzo_sim_lost(const qzo_sim* s);
/* plasma state of species sp after the last sweep (x y px py dl w, n values each) */
int      qzo_sim_plasma_get(const qzo_sim* s, int sp, double* out6, int cap);
/* run the reference time loop: nsteps+1 sweeps and nsteps pushes with constant dt;
   moments (17 per beam per step, step-major) go to mom if non-NULL */
int      qzo_sim_run(qzo_sim* s, int nsteps, double dt, double* mom);
/* beam deposit only (into the sim's bsrc, which is zeroed first) */
int      qzo_sim_deposit_beams(qzo_sim* s);
/* the adjoint of a run (qz_oracle_adj.c; m = 0, linear xi shape, one mobile species): runs nsteps
   like qzo_sim_run from the current (not yet pushed) beams, then in reverse returns in lam_out, for
   every beam in order, its (n, 7) rows d(J)/d(x y px py pz xi w of each initial particle) with
   J = sum(lamS * last step's moment sums), lamS (nb, 17). mom as in qzo_sim_run. 0, or -2 when the
   deck is outside the adjoint's scope. */
int      qzo_sim_adjoint(qzo_sim* s, int nsteps, double dt, const double* lamS, double* lam_out, double* mom);

#ifdef __cplusplus
}
#endif
#endif
