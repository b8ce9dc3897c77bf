// qz_internal.h -- kernel argument blocks and launchers shared by the .cu files of libqz_b200.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace qzb {

constexpr int kSweepThreads = 512;
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
    const double* p_init;           // fresh plasma at the head: (6, npad) x y px py Delta w
    int nbg;                        // immobile particles (background)
    const double* bg_p;             // (3, nbg): x, y, w*q
    int neutralize;
    double* ps;                     // working state (6 + 5*ord, npad), used when np > kSweepThreads
    const double* bsrc;             // beam sources (K, M, 5)
    int ngp;
    double* fld;                    // (K, M, 6)
    double* diag;                   // (K, M, 3)
    unsigned long long* counters;   // [0] plasma particles removed
    unsigned long long* timing;     // optional: clock cycles per phase [6]
    int dbuf;                       // double-buffered slice sources (push fused with the next deposit)
    int const_smem;                 // per-node constants copied into shared memory
};

size_t sweep_m0_smem_bytes(int M, bool dbuf, bool const_smem);
cudaError_t launch_sweep_m0(const SweepArgs& A, cudaStream_t stream);

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
};

cudaError_t launch_beam_deposit(const BeamArgs& B, double* bsrc, cudaStream_t s);
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

}  // namespace qzb
