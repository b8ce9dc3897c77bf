// qz_abi.cu -- the extern "C" boundary of libqz_b200.so (declared in include/qz_b200.h) and the
// host-side set-up it needs: grid volumes and operator rows (computed on the host in FP64 exactly
// as the reference does, then uploaded), the fresh plasma of the box head, the gaussian beam
// generator, and the time-step runner.
#include "qz_b200.h"
#include "qz_internal.h"
#include "qz_device.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <new>
#include <random>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

qz_status fail(qz_status code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define QZ_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(QZ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

constexpr double PI = 3.14159265358979323846;

template <class T>
qz_status dev_upload(T** dst, const std::vector<T>& src) {
    *dst = nullptr;
    if (src.empty()) return QZ_OK;
    QZ_CUDA(cudaMalloc((void**)dst, sizeof(T) * src.size()));
    QZ_CUDA(cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice));
    return QZ_OK;
}

}  // namespace

// ===================================================================== grid
struct qz_grid {
    int M = 0, N = 0;
    double R = 0;
    std::vector<double> r, h, rmid, V, inv_h, inv_V;
    std::vector<double> opa[4], opb[4], opc[4];
    double flux_coef = 0;
    std::vector<double> gm, g0, gp, ir;
    std::vector<double> consts;  // per-node constants of the sweep (13 x M)
    std::vector<double> consts1; // and of the modes = 1 sweep (9 x M)
    // device
    double *d_r = nullptr, *d_inv_h = nullptr, *d_inv_V = nullptr, *d_consts = nullptr, *d_consts1 = nullptr;
    ~qz_grid() {
        for (double* p : {d_r, d_inv_h, d_inv_V, d_consts, d_consts1})
            if (p) cudaFree(p);
    }
};

namespace {

// rows of the finite-volume operator L_n, n >= 1 (src/FieldSolver.cpp:90-103)
void fv_rows(const qz_grid& g, int n, std::vector<double>& a, std::vector<double>& b, std::vector<double>& c) {
    const int N = g.N, M = N + 1;
    a.assign(M, 0.0); b.assign(M, 0.0); c.assign(M, 0.0);
    b[0] = 1.0;
    b[N] = 1.0;
    auto kp = [&](int j) { return 1.0 / (g.h[j] * std::pow(g.rmid[j], 2 * n - 1)); };
    for (int j = 1; j < N; ++j) {
        const double dV = 0.5 * (g.h[j] + g.h[j - 1]);
        const double pre = std::pow(g.r[j], n - 1) / dV;
        c[j] = pre * std::pow(g.r[j + 1], n) * kp(j);
        a[j] = pre * std::pow(g.r[j - 1], n) * kp(j - 1);
        b[j] = -pre * std::pow(g.r[j], n) * (kp(j) + kp(j - 1));
    }
}


}  // namespace

extern "C" const char* qz_last_error(void) { return g_err.c_str(); }
#ifndef QZ_SRC_HASH
#define QZ_SRC_HASH "unknown"
#endif
extern "C" const char* qz_version(void) { return "qz_b200 0.2 (sm_100a, FP64) src " QZ_SRC_HASH; }

extern "C" qz_status qz_grid_create(const double* nodes, int M, qz_grid** out) {
    if (!nodes || !out) return fail(QZ_ERR_ARG, "qz_grid_create: null pointer");
    *out = nullptr;
    if (M < 3) return fail(QZ_ERR_ARG, "grid: need at least 2 cells");
    if (std::abs(nodes[0]) > 0) return fail(QZ_ERR_ARG, "grid: first node must be r=0");
    for (int j = 1; j < M; ++j)
        if (!(nodes[j] > nodes[j - 1])) return fail(QZ_ERR_ARG, "grid: nodes must be strictly increasing");
    qz_grid* g = new (std::nothrow) qz_grid;
    if (!g) return fail(QZ_ERR_NOMEM, "qz_grid_create: out of host memory");
    // src/RadialGrid.cpp:106-148
    g->M = M;
    g->N = M - 1;
    const int N = g->N;
    g->r.assign(nodes, nodes + M);
    g->R = g->r[N];
    g->h.resize(N);
    g->rmid.resize(N);
    for (int j = 0; j < N; ++j) {
        g->h[j] = g->r[j + 1] - g->r[j];
        g->rmid[j] = 0.5 * (g->r[j + 1] + g->r[j]);
    }
    g->V.assign(M, 0.0);
    for (int j = 0; j <= N; ++j) {
        double v = 0;
        if (j > 0) v += g->r[j - 1] * g->h[j - 1] / 2 + g->h[j - 1] * g->h[j - 1] / 3;
        if (j < N) v += g->r[j] * g->h[j] / 2 + g->h[j] * g->h[j] / 6;
        g->V[j] = 2 * PI * v;
    }
    g->inv_V.resize(M);
    g->inv_h.resize(N);
    for (int j = 0; j <= N; ++j) g->inv_V[j] = 1.0 / g->V[j];
    for (int j = 0; j < N; ++j) g->inv_h[j] = 1.0 / g->h[j];
    // operators (src/FieldSolver.cpp:117-156)
    {
        std::vector<double>&a = g->opa[0], &b = g->opb[0], &c = g->opc[0];
        a.assign(M, 0.0); b.assign(M, 0.0); c.assign(M, 0.0);
        for (int j = 0; j < N; ++j) {
            const double invV = 2 * PI / g->V[j];
            a[j] = (j > 0) ? g->rmid[j - 1] / g->h[j - 1] * invV : 0.0;
            c[j] = g->rmid[j] / g->h[j] * invV;
            b[j] = -(a[j] + c[j]);
        }
        b[N] = 1.0;
    }
    fv_rows(*g, 1, g->opa[1], g->opb[1], g->opc[1]);
    fv_rows(*g, 1, g->opa[2], g->opb[2], g->opc[2]);
    {
        const double dV = 0.5 * g->h[N - 1];
        const double kp = 1.0 / (g->h[N - 1] * std::pow(g->rmid[N - 1], 2 * 1 - 1));
        const double k = kp / dV;
        g->opa[2][N] = g->r[N - 1] * k;
        g->opb[2][N] = -g->r[N] * k;
        g->flux_coef = 1.0 / dV;
    }
    fv_rows(*g, 2, g->opa[3], g->opb[3], g->opc[3]);
    // gradient stencils and 1/r (src/FieldSolver.cpp:157-176)
    g->gm.assign(M, 0.0); g->g0.assign(M, 0.0); g->gp.assign(M, 0.0); g->ir.assign(M, 0.0);
    for (int j = 1; j < N; ++j) {
        const double hm = g->h[j - 1], hp = g->h[j];
        const double den = hm * hp * (hm + hp);
        g->gp[j] = hm * hm / den;
        g->gm[j] = -hp * hp / den;
        g->g0[j] = (hp * hp - hm * hm) / den;
    }
    {
        const double h1 = g->h[N - 1], h2 = (N >= 2) ? g->h[N - 2] : g->h[N - 1];
        const double s = h1 + h2;
        g->g0[N] = (2 * h1 + h2) / (h1 * s);
        g->gm[N] = -s / (h1 * h2);
        g->gp[N] = h1 / (h2 * s);
    }
    for (int j = 1; j <= N; ++j) g->ir[j] = 1.0 / g->r[j];
    g->ir[0] = 1.0 / g->r[1];
    // per-node constants of the sweep: stencils, 1/r, L0 Thomas factors, L1D and L1F rows
    {
        std::vector<double> cs((size_t)13 * M, 0.0);
        auto put = [&](int k, const std::vector<double>& v) { std::copy(v.begin(), v.end(), cs.begin() + (size_t)k * M); };
        put(0, g->gm); put(1, g->g0); put(2, g->gp); put(3, g->ir);
        // Thomas on L0 with its Dirichlet row N (src/Tridiag.cpp:111-125): u_i = b_i - a_i c_{i-1}/u_{i-1}
        const std::vector<double>&a0 = g->opa[0], &b0 = g->opb[0], &c0 = g->opc[0];
        double cp = 0.0;
        for (int i = 0; i < M; ++i) {
            const double rr = 1.0 / (b0[i] - (i > 0 ? a0[i] * cp : 0.0));
            cp = c0[i] * rr;
            cs[(size_t)4 * M + i] = rr;
            cs[(size_t)5 * M + i] = -rr * a0[i];
            cs[(size_t)6 * M + i] = -cp;
        }
        put(7, g->opa[1]); put(8, g->opb[1]); put(9, g->opc[1]);
        put(10, g->opa[2]); put(11, g->opb[2]); put(12, g->opc[2]);
        g->consts = cs;
        // modes = 1: Thomas factors of L1D (its Dirichlet rows 0 and N are rows b = 1), L0 and L2D rows
        std::vector<double> c1((size_t)9 * M, 0.0);
        const std::vector<double>&a1 = g->opa[1], &b1 = g->opb[1], &cc1 = g->opc[1];
        cp = 0.0;
        for (int i = 0; i < M; ++i) {
            const double rr = 1.0 / (b1[i] - (i > 0 ? a1[i] * cp : 0.0));
            cp = cc1[i] * rr;
            c1[i] = rr;
            c1[(size_t)M + i] = -rr * a1[i];
            c1[(size_t)2 * M + i] = -cp;
        }
        std::copy(a0.begin(), a0.end(), c1.begin() + (size_t)3 * M);
        std::copy(b0.begin(), b0.end(), c1.begin() + (size_t)4 * M);
        std::copy(c0.begin(), c0.end(), c1.begin() + (size_t)5 * M);
        std::copy(g->opa[3].begin(), g->opa[3].end(), c1.begin() + (size_t)6 * M);
        std::copy(g->opb[3].begin(), g->opb[3].end(), c1.begin() + (size_t)7 * M);
        std::copy(g->opc[3].begin(), g->opc[3].end(), c1.begin() + (size_t)8 * M);
        g->consts1 = c1;
    }
    qz_status st;
    if ((st = dev_upload(&g->d_r, g->r)) || (st = dev_upload(&g->d_inv_h, g->inv_h)) ||
        (st = dev_upload(&g->d_inv_V, g->inv_V)) || (st = dev_upload(&g->d_consts, g->consts)) ||
        (st = dev_upload(&g->d_consts1, g->consts1))) {
        delete g;
        return st;
    }
    *out = g;
    return QZ_OK;
}

extern "C" qz_status qz_grid_destroy(qz_grid* g) {
    delete g;
    return QZ_OK;
}

extern "C" qz_status qz_grid_volumes(const qz_grid* g, double* V) {
    if (!g || !V) return fail(QZ_ERR_ARG, "qz_grid_volumes: null pointer");
    std::memcpy(V, g->V.data(), sizeof(double) * g->M);
    return QZ_OK;
}

extern "C" qz_status qz_grid_operator(const qz_grid* g, int op, double* a, double* b, double* c, double* fc) {
    if (!g || !a || !b || !c || op < 0 || op > 3) return fail(QZ_ERR_ARG, "qz_grid_operator: bad argument");
    std::memcpy(a, g->opa[op].data(), sizeof(double) * g->M);
    std::memcpy(b, g->opb[op].data(), sizeof(double) * g->M);
    std::memcpy(c, g->opc[op].data(), sizeof(double) * g->M);
    if (fc) *fc = g->flux_coef;
    return QZ_OK;
}

// ===================================================================== sweep
// node quanta of the exact beam deposits (qz_fx_create): 2^-qe_j (scales) then 2^qe_j (quanta), the split S
struct qz_fx {
    int M = 0;
    int S = 0;
    std::vector<int> qe;
    double* d_q = nullptr;
    ~qz_fx() {
        if (d_q) cudaFree(d_q);
    }
};

struct qz_sweep {
    const qz_grid* g = nullptr;
    const qz_fx* fx = nullptr;            // qz_sweep_set_exact_sources: bsrc in the two-limb format
    qz_sweep_params p{};
    int np = 0, npad = 0, nbg = 0;
    double* d_pinit = nullptr;
    double* d_bg = nullptr;
    double* d_ps = nullptr;
    double* d_bgs = nullptr;              // modes = 1: background (3, M) and two source buffers (2 x 30, M)
    double* d_fconsts = nullptr;          // smoothing filter: Thomas factors of F0, F1, F2 (9 x M)
    unsigned long long* d_cnt = nullptr;
    unsigned long long* d_tim = nullptr;
    bool timing = false;
    qzb::SweepArgs base{};
    ~qz_sweep() {
        for (void* q : {(void*)d_pinit, (void*)d_bg, (void*)d_ps, (void*)d_bgs, (void*)d_cnt, (void*)d_tim,
                        (void*)d_fconsts})
            if (q) cudaFree(q);
    }
};

namespace {

double prof_radial(const qz_species& s, double r) {
    if (r > s.rmax) return 0.0;
    if (s.channel_radius > 0) return 1.0 + s.channel_depth * (r / s.channel_radius) * (r / s.channel_radius);
    return 1.0;
}

// fresh cold plasma rings of one species at the box head (src/PlasmaSpecies.cpp:202-295):
// appends x y px py Delta w per particle
void load_species(const qz_grid& g, const qz_species& sp, std::vector<double> cols[6]) {
    const double fz = 1.0 * sp.density;
    const int ppc = sp.ppc, nth = sp.ntheta;
    for (int j = 0; j < g.N; ++j) {
        const double h = g.h[j];
        for (int m = 0; m < ppc; ++m) {
            const double ra = g.r[j] + m * h / ppc, rb = g.r[j] + (m + 1) * h / ppc;
            const double r = (2.0 / 3.0) * (rb * rb * rb - ra * ra * ra) / (rb * rb - ra * ra);
            const double vring = fz * PI * (rb * rb - ra * ra);
            const double wring = prof_radial(sp, r) * vring;
            const double off = ((j * ppc + m) % 2) * 0.5;
            for (int l = 0; l < nth; ++l) {
                const double th = 2 * PI * (l + off) / nth;
                const double X = (nth == 1) ? r : r * std::cos(th), Y = (nth == 1) ? 0.0 : r * std::sin(th);
                const double W = wring / nth;
                if (W == 0) continue;
                cols[0].push_back(X); cols[1].push_back(Y); cols[2].push_back(0.0); cols[3].push_back(0.0);
                cols[4].push_back(1.0); cols[5].push_back(W);
            }
        }
    }
}

// Thomas factors 1/u, -a/u, -c/u (3 x M) of the smoothing filter F_n with a^2 in every cell
// (FieldSolver::set_filter, src/FieldSolver.cpp:111-146): n = 0 in flux form on the node volumes with a
// zero-flux wall, n = 1, 2 as the finite-volume L_n with a^2 inside the flux and identity rows 0 and N
void filter_factors(const qz_grid& g, double a2, int n, double* out) {
    const int N = g.N, M = N + 1;
    std::vector<double> a(M, 0.0), b(M, 1.0), c(M, 0.0);
    if (n == 0) {
        for (int j = 0; j <= N; ++j) {
            const double invV = 2 * PI / g.V[j];
            const double am = (j > 0) ? a2 * g.rmid[j - 1] / g.h[j - 1] * invV : 0.0;
            const double cp = (j < N) ? a2 * g.rmid[j] / g.h[j] * invV : 0.0;
            a[j] = -am; c[j] = -cp; b[j] = 1 + am + cp;
        }
    } else {
        for (int j = 1; j < N; ++j) {
            const double dV = 0.5 * (g.h[j] + g.h[j - 1]);
            const double pre = std::pow(g.r[j], n - 1) / dV;
            const double kpj = a2 / (g.h[j] * std::pow(g.rmid[j], 2 * n - 1));
            const double kpm = a2 / (g.h[j - 1] * std::pow(g.rmid[j - 1], 2 * n - 1));
            c[j] = -pre * std::pow(g.r[j + 1], n) * kpj;
            a[j] = -pre * std::pow(g.r[j - 1], n) * kpm;
            b[j] = 1 + pre * std::pow(g.r[j], n) * (kpj + kpm);
        }
    }
    double cp = 0.0;
    for (int i = 0; i < M; ++i) {
        const double rr = 1.0 / (b[i] - (i > 0 ? a[i] * cp : 0.0));
        cp = c[i] * rr;
        out[i] = rr;
        out[(size_t)M + i] = -rr * a[i];
        out[(size_t)2 * M + i] = -cp;
    }
}

}  // namespace

extern "C" qz_status qz_sweep_create(const qz_grid* g, const qz_sweep_params* p, qz_sweep** out) {
    if (!g || !p || !out) return fail(QZ_ERR_ARG, "qz_sweep_create: null pointer");
    *out = nullptr;
    if (p->modes != 0 && p->modes != 1) return fail(QZ_ERR_ARG, "qz_sweep_create: modes must be 0 or 1");
    if (p->ab_order < 1 || p->ab_order > 5) return fail(QZ_ERR_ARG, "pusher.ab_order must be 1..5");
    if (p->modes == 1 && p->picard < 1) return fail(QZ_ERR_ARG, "solver.picard must be >= 1");
    if (p->K < 1 || !(p->dxi > 0)) return fail(QZ_ERR_ARG, "xi: need K >= 1 and dxi > 0");
    if (p->nspecies < 0 || p->nspecies > 4) return fail(QZ_ERR_ARG, "nspecies must be 0..4");
    if (!(p->smooth_length >= 0)) return fail(QZ_ERR_ARG, "plasma.smooth_length must be >= 0");
    const bool filter = p->smooth_length > 0;
    const int M = g->M;
    int dev = 0, optin = 0;
    QZ_CUDA(cudaGetDevice(&dev));
    QZ_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    // shared-memory layout: the fastest that fits (double-buffered sources, constants in shared
    // memory), else single-buffered sources and/or constants read from global memory
    static const bool kLayouts[4][2] = {{true, true}, {false, true}, {true, false}, {false, false}};
    int lay = -1;
    for (int i = 0; i < 4 && lay < 0; ++i)
        if (qzb::sweep_m0_smem_bytes(M, kLayouts[i][0], kLayouts[i][1], filter) <= (size_t)optin) lay = i;
    const int rpt = (M + qzb::kSweepThreads - 1) / qzb::kSweepThreads;
    if (!(p->max_cells_per_step >= 0.0) || p->substep_max < 0)
        return fail(QZ_ERR_ARG, "qz_sweep_create: pusher.max_cells_per_step must be >= 0 and substep_max >= 1");
    if (p->max_cells_per_step > 0.0 && (p->modes != 0 || p->smooth_length > 0.0))
        return fail(QZ_ERR_UNSUPPORTED, "qz_sweep_create: adaptive sub-slicing (pusher.max_cells_per_step) runs with "
                                        "modes = 0 and without plasma.smooth_length");
    // modes = 1: one radial node per thread, 512 threads or (513..1024 nodes) 1024
    if (p->modes == 1 && (M > 2 * qzb::kSweepThreads ||
                          (M <= qzb::kSweepThreads ? qzb::sweep_m1_smem_bytes(M) : qzb::sweep_m1w_smem_bytes(M)) >
                              (size_t)optin))
        return fail(QZ_ERR_SIZE, "qz_sweep_create: the modes = 1 sweep holds one radial node per thread: M = " +
                                     std::to_string(M) + " > " + std::to_string(2 * qzb::kSweepThreads));
    if (lay < 0 || rpt > 4)
        return fail(QZ_ERR_SIZE, "qz_sweep_create: M = " + std::to_string(M) + " is too large for one CTA (" +
                                     std::to_string(qzb::sweep_m0_smem_bytes(M, false, false, filter)) + " B of shared memory, "
                                     "the device allows " + std::to_string(optin) + ")");
    qz_sweep* s = new (std::nothrow) qz_sweep;
    if (!s) return fail(QZ_ERR_NOMEM, "qz_sweep_create: out of host memory");
    s->g = g;
    s->p = *p;
    // plasma: mobile species -> particle state, immobile -> background particles
    std::vector<double> mob[6], bg[3];
    qzb::SweepArgs& A = s->base;
    A.nsp = 0;
    A.sp_off[0] = 0;
    for (int i = 0; i < p->nspecies; ++i) {
        const qz_species& sp = p->species[i];
        if (sp.ppc < 1 || sp.ntheta < 1 || !(sp.m > 0)) {
            delete s;
            return fail(QZ_ERR_ARG, "species: ppc, ntheta >= 1 and m > 0 required");
        }
        std::vector<double> cols[6];
        load_species(*g, sp, cols);
        if (sp.mobile) {
            for (int v = 0; v < 6; ++v) mob[v].insert(mob[v].end(), cols[v].begin(), cols[v].end());
            A.sp_q[A.nsp] = sp.q;
            A.sp_qm[A.nsp] = sp.q / sp.m;
            ++A.nsp;
            A.sp_off[A.nsp] = (int)mob[0].size();
        } else {
            bg[0].insert(bg[0].end(), cols[0].begin(), cols[0].end());
            bg[1].insert(bg[1].end(), cols[1].begin(), cols[1].end());
            for (double w : cols[5]) bg[2].push_back(w * sp.q);
        }
    }
    s->np = (int)mob[0].size();
    s->npad = ((s->np + 31) / 32) * 32;
    if (s->npad == 0) s->npad = 32;
    // plasma in global memory (more particles per slice than threads): keep a shared-memory copy of
    // the particles when a layout leaves room for it (the fastest such layout)
    A.pcache = 0;
    if (p->modes == 0 && s->np > qzb::kSweepThreads)
        for (int i = 0; i < 4; ++i)
            if (qzb::sweep_m0_smem_bytes(M, kLayouts[i][0], kLayouts[i][1], filter, s->np) <= (size_t)optin) {
                lay = i;
                A.pcache = s->np;
                break;
            }
    s->nbg = (int)bg[0].size();
    std::vector<double> pinit((size_t)6 * s->npad, 0.0);
    for (int v = 0; v < 6; ++v) std::copy(mob[v].begin(), mob[v].end(), pinit.begin() + (size_t)v * s->npad);
    std::vector<double> bgp;
    for (int v = 0; v < 3; ++v) bgp.insert(bgp.end(), bg[v].begin(), bg[v].end());
    qz_status st;
    if ((st = dev_upload(&s->d_pinit, pinit)) || (st = dev_upload(&s->d_bg, bgp))) {
        delete s;
        return st;
    }
    const size_t nps = (size_t)(6 + 5 * p->ab_order) * s->npad;
    if (cudaMalloc((void**)&s->d_ps, sizeof(double) * nps) != cudaSuccess ||
        cudaMalloc((void**)&s->d_bgs, sizeof(double) * 63 * M) != cudaSuccess ||
        cudaMalloc((void**)&s->d_cnt, sizeof(unsigned long long) * 4) != cudaSuccess ||
        cudaMalloc((void**)&s->d_tim, sizeof(unsigned long long) * 16) != cudaSuccess) {
        delete s;
        return fail(QZ_ERR_NOMEM, "qz_sweep_create: device allocation failed");
    }
    // AB coefficients (src/PlasmaSpecies.cpp:14-28)
    static const double AB[5][5] = {{1, 0, 0, 0, 0},
                                    {1.5, -0.5, 0, 0, 0},
                                    {23. / 12, -16. / 12, 5. / 12, 0, 0},
                                    {55. / 24, -59. / 24, 37. / 24, -9. / 24, 0},
                                    {1901. / 720, -2774. / 720, 2616. / 720, -1274. / 720, 251. / 720}};
    A.M = M;
    A.N = g->N;
    A.K = p->K;
    A.rows_per_thread = rpt;
    A.R = g->R;
    A.dxi = p->dxi;
    A.idxi = 1.0 / p->dxi;
    A.r = g->d_r; A.inv_h = g->d_inv_h; A.inv_V = g->d_inv_V;
    A.consts = g->d_consts;
    A.flux_coef = g->flux_coef;
    A.np = s->np;
    A.npad = s->npad;
    A.ord = p->ab_order;
    for (int m = 0; m < 5; ++m) A.ab[m] = AB[p->ab_order - 1][m];
    A.delta_min = p->delta_min;
    A.max_qsa = p->max_qsa;
    A.max_cells = p->max_cells_per_step;
    A.substep_max = p->substep_max > 0 ? p->substep_max : 64;
    A.p_init = s->d_pinit;
    A.nbg = s->nbg;
    A.bg_p = s->d_bg;
    A.neutralize = p->neutralize;
    A.ps = s->d_ps;
    A.ngp = p->ngp;
    A.counters = s->d_cnt;
    A.timing = nullptr;
    A.dbuf = kLayouts[lay][0];
    A.const_smem = kLayouts[lay][1];
    A.picard = p->picard;
    A.consts1 = g->d_consts1;
    A.bgs = s->d_bgs;
    A.srcs = s->d_bgs + 3 * (size_t)M;
    A.filter = 0;
    A.fconsts = nullptr;
    A.bstat = nullptr;
    if (filter) {
        std::vector<double> fc((size_t)9 * M);
        const double a2 = p->smooth_length * p->smooth_length;
        for (int n = 0; n < 3; ++n) filter_factors(*g, a2, n, fc.data() + (size_t)3 * n * M);
        if ((st = dev_upload(&s->d_fconsts, fc))) {
            delete s;
            return st;
        }
        A.filter = 1;
        A.fconsts = s->d_fconsts;
    }
    *out = s;
    return QZ_OK;
}

extern "C" qz_status qz_sweep_destroy(qz_sweep* s) {
    delete s;
    return QZ_OK;
}

namespace {
// the optional arguments of one sweep: bsrc in the exact two-limb format (qz_sim's m = 0 runs: the
// node quanta bq, 2^S, the offset of the low limbs) and a slab of a staged run (qz_sweep_run_stage)
struct SweepExtra {
    const double* bq = nullptr;
    double bfx_2s = 0.0;
    long bfx_lo = 0;
    const double* pin = nullptr;
    int pin_pushed = 0;
    const double* bguard = nullptr;
    double* pout = nullptr;
    bool accumulate = false;          // add to the sweep's device counters (a run's sweeps), do not clear them
};

// one sweep of s over bsrc
qz_status sweep_launch(qz_sweep* s, const double* bsrc, double* fld, double* diag, qz_counters* cnt,
                       cudaStream_t st, const SweepExtra& x = SweepExtra()) {
    qzb::SweepArgs A = s->base;
    A.bsrc = bsrc;
    A.fld = fld;
    A.diag = diag;
    A.bq = x.bq;
    A.bfx_2s = x.bfx_2s;
    A.bfx_lo = x.bfx_lo;
    if (!x.bq && s->fx && s->p.modes == 0) {          // the caller's sources in the two-limb format
        A.bq = s->fx->d_q + s->g->M;
        A.bfx_2s = std::ldexp(1.0, s->fx->S);
        A.bfx_lo = (long)s->p.K * s->g->M * qzb::B_NC0;
    }
    A.pin = x.pin;
    A.pin_pushed = x.pin_pushed;
    A.bguard = x.bguard;
    A.pout = x.pout;
    if (!x.accumulate) QZ_CUDA(cudaMemsetAsync(s->d_cnt, 0, sizeof(unsigned long long) * 4, st));
    if (s->timing) {
        QZ_CUDA(cudaMemsetAsync(s->d_tim, 0, sizeof(unsigned long long) * 16, st));
        A.timing = s->d_tim;
    }
    QZ_CUDA(s->p.modes == 1 ? qzb::launch_sweep_m1(A, st) : qzb::launch_sweep_m0(A, st));
    if (cnt) {
        unsigned long long h[4];
        QZ_CUDA(cudaMemcpyAsync(h, s->d_cnt, sizeof(h), cudaMemcpyDeviceToHost, st));
        QZ_CUDA(cudaStreamSynchronize(st));
        cnt->lost += h[0];
        cnt->nonfinite += h[1];
        cnt->trapped += h[2];
        cnt->subslices += h[3];
    }
    return QZ_OK;
}
}  // namespace

extern "C" qz_status qz_sweep_run(qz_sweep* s, const double* bsrc, double* fld, double* diag, qz_counters* cnt,
                                  void* stream) {
    if (!s || !bsrc || !fld || !diag) return fail(QZ_ERR_ARG, "qz_sweep_run: null pointer");
    return sweep_launch(s, bsrc, fld, diag, cnt, (cudaStream_t)stream);
}

extern "C" qz_status qz_sweep_state_shape(qz_sweep* s, int* np, int* npad, int* order) {
    if (!s || !np || !npad || !order) return fail(QZ_ERR_ARG, "qz_sweep_state_shape: null pointer");
    *np = s->np;
    *npad = s->npad;
    *order = s->p.ab_order;
    return QZ_OK;
}

extern "C" qz_status qz_sweep_run_stage(qz_sweep* s, const double* bsrc, const double* bguard,
                                        const qz_plasma_state* in, double* fld, double* diag, qz_plasma_state* out,
                                        qz_counters* cnt, void* stream) {
    if (!s || !bsrc || !fld || !diag) return fail(QZ_ERR_ARG, "qz_sweep_run_stage: null pointer");
    if (s->p.modes != 0) return fail(QZ_ERR_UNSUPPORTED, "qz_sweep_run_stage: modes = 0 sweeps only");
    if (s->base.filter || s->base.bstat || s->base.max_cells > 0.0)
        return fail(QZ_ERR_UNSUPPORTED, "qz_sweep_run_stage: no smoothing filter, static beam sources or adaptive "
                                        "sub-slicing in a stage");
    if ((bguard || out) && !s->p.ngp)
        return fail(QZ_ERR_UNSUPPORTED, "qz_sweep_run_stage: slabs that take a guard row or hand their plasma on "
                                        "need the ngp xi shape (the last slice's derivative would need the next slab)");
    auto check_state = [&](const qz_plasma_state* st, const char* what) -> qz_status {
        if (!st->state) return fail(QZ_ERR_ARG, std::string("qz_sweep_run_stage: null ") + what + " state");
        if (st->np != s->np || st->npad != s->npad || st->order != s->p.ab_order)
            return fail(QZ_ERR_ARG, std::string("qz_sweep_run_stage: ") + what + " state of " + std::to_string(st->np) +
                                        " particles (stride " + std::to_string(st->npad) + ", AB order " +
                                        std::to_string(st->order) + "), the sweep has " + std::to_string(s->np) +
                                        " (" + std::to_string(s->npad) + ", " + std::to_string(s->p.ab_order) + ")");
        return QZ_OK;
    };
    SweepExtra x;
    if (in) {
        if (qz_status e = check_state(in, "input")) return e;
        x.pin = in->state;
        x.pin_pushed = in->pushed ? 1 : 0;
    }
    if (out) {
        if (qz_status e = check_state(out, "output")) return e;
        x.pout = out->state;
    }
    x.bguard = bguard;
    if (qz_status e = sweep_launch(s, bsrc, fld, diag, cnt, (cudaStream_t)stream, x)) return e;
    if (out) out->pushed = 1;
    return QZ_OK;
}

extern "C" qz_status qz_sweep_plasma(qz_sweep* s, double* out, int cap, int* n) {
    if (!s || !out || !n) return fail(QZ_ERR_ARG, "qz_sweep_plasma: null pointer");
    *n = s->np;
    if (cap < s->np) return fail(QZ_ERR_SIZE, "qz_sweep_plasma: capacity too small");
    for (int v = 0; v < 6; ++v)
        QZ_CUDA(cudaMemcpy(out + (size_t)v * s->np, s->d_ps + (size_t)v * s->npad, sizeof(double) * s->np,
                           cudaMemcpyDeviceToHost));
    return QZ_OK;
}

extern "C" qz_status qz_sweep_timing(qz_sweep* s, int enable, unsigned long long* cycles6) {
    if (!s) return fail(QZ_ERR_ARG, "qz_sweep_timing: null pointer");
    if (cycles6) QZ_CUDA(cudaMemcpy(cycles6, s->d_tim, sizeof(unsigned long long) * 16, cudaMemcpyDeviceToHost));
    s->timing = enable != 0;
    return QZ_OK;
}

// ===================================================================== beams
namespace {

qzb::BeamArgs beam_args(const qz_grid* g, const qz_beam_view* b, const qz_box* box) {
    qzb::BeamArgs B{};
    B.x = b->x; B.y = b->y; B.px = b->px; B.py = b->py; B.pz = b->pz; B.xi = b->xi; B.w = b->w;
    B.n = (long)b->n;
    B.q = b->q;
    B.m = b->m;
    B.M = g->M;
    B.N = g->N;
    B.R = g->R;
    B.r = g->d_r;
    B.inv_h = g->d_inv_h;
    B.inv_V = g->d_inv_V;
    B.xi_min = box->xi_min;
    B.dxi = box->dxi;
    B.idxi = 1.0 / box->dxi;
    B.K = box->K;
    B.ngp = box->ngp;
    B.modes = box->modes;
    B.pusher = b->pusher;
    return B;
}

qz_status check_beam(const qz_grid* g, const qz_beam_view* b, const qz_box* box) {
    if (!g || !b || !box) return fail(QZ_ERR_ARG, "beam: null pointer");
    if (b->n > 0 && (!b->x || !b->y || !b->px || !b->py || !b->pz || !b->xi || !b->w))
        return fail(QZ_ERR_ARG, "beam: null column");
    if (box->K < 2 || !(box->dxi > 0)) return fail(QZ_ERR_ARG, "beam: box needs K >= 2 and dxi > 0");
    if (box->modes != 0 && box->modes != 1) return fail(QZ_ERR_ARG, "beam: modes must be 0 or 1");
    if (b->pusher < 0 || b->pusher > 3) return fail(QZ_ERR_ARG, "beam: pusher must be 0..3 (vay, boris, hc, imp)");
    return QZ_OK;
}

}  // namespace

extern "C" qz_status qz_beam_deposit(const qz_grid* g, const qz_beam_view* b, const qz_box* box, double* bsrc,
                                     void* stream) {
    if (qz_status st = check_beam(g, b, box)) return st;
    if (!bsrc) return fail(QZ_ERR_ARG, "qz_beam_deposit: null bsrc");
    QZ_CUDA(qzb::launch_beam_deposit(beam_args(g, b, box), bsrc, (cudaStream_t)stream));
    return QZ_OK;
}

namespace {

qz_status analytic_args(const qz_grid* g, const qz_analytic_beam* b, const qz_box* box, qzb::AnalyticArgs& P) {
    if (!g || !b || !box) return fail(QZ_ERR_ARG, "analytic beam: null pointer");
    if (box->modes != 0 && box->modes != 1) return fail(QZ_ERR_ARG, "analytic beam: modes must be 0 or 1");
    if (box->K < 1 || !(box->dxi > 0)) return fail(QZ_ERR_ARG, "analytic beam: need K >= 1 and dxi > 0");
    if (!(b->sigma_r > 0) || !(b->gamma >= 1) || (b->flattop ? !(b->length >= 0) : !(b->sigma_xi > 0)))
        return fail(QZ_ERR_ARG, "analytic beam: need sigma_r > 0, gamma >= 1 and sigma_xi > 0 (or length >= 0)");
    if (box->modes == 0 && (b->x0 != 0 || b->y0 != 0 || b->x_slope != 0 || b->y_slope != 0))
        return fail(QZ_ERR_ARG, "analytic beam: transverse offsets/tilts need azimuthal mode 1 (modes = 1)");
    P.q = b->q; P.n0 = b->n0; P.s2 = b->sigma_r * b->sigma_r;
    P.xi0 = b->xi0; P.sxi = b->sigma_xi; P.len = b->length; P.cut = b->xi_cut;
    P.x0 = b->x0; P.y0 = b->y0; P.xs = b->x_slope; P.ys = b->y_slope;
    P.vz = std::sqrt(1.0 - 1.0 / (b->gamma * b->gamma));
    P.omvz = 1.0 / (b->gamma * b->gamma * (1.0 + P.vz));
    P.flat = b->flattop ? 1 : 0;
    P.m1 = box->modes;
    P.r = g->d_r;
    P.M = g->M;
    P.K = box->K;
    P.bnc = box->modes ? 15 : 5;
    P.xi_min = box->xi_min;
    P.dxi = box->dxi;
    return QZ_OK;
}

}  // namespace

extern "C" qz_status qz_beam_deposit_analytic(const qz_grid* g, const qz_analytic_beam* b, const qz_box* box,
                                              double* bsrc, void* stream) {
    qzb::AnalyticArgs P;
    if (qz_status st = analytic_args(g, b, box, P)) return st;
    if (!bsrc) return fail(QZ_ERR_ARG, "qz_beam_deposit_analytic: null bsrc");
    QZ_CUDA(qzb::launch_deposit_analytic(P, bsrc, (cudaStream_t)stream));
    return QZ_OK;
}

extern "C" qz_status qz_beam_slice_sums(const qz_beam_view* b, double lo, double hi, int nbins, double* out,
                                        void* stream) {
    if (!b || !out || nbins < 1 || !(hi > lo)) return fail(QZ_ERR_ARG, "qz_beam_slice_sums: need nbins >= 1, hi > lo");
    if (b->n > 0 && (!b->x || !b->y || !b->px || !b->py || !b->pz || !b->xi || !b->w))
        return fail(QZ_ERR_ARG, "qz_beam_slice_sums: null column");
    qzb::BeamArgs B{};
    B.x = b->x; B.y = b->y; B.px = b->px; B.py = b->py; B.pz = b->pz; B.xi = b->xi; B.w = b->w;
    B.n = (long)b->n;
    cudaStream_t st = (cudaStream_t)stream;
    QZ_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * 9 * (size_t)nbins, st));
    QZ_CUDA(qzb::launch_slice_sums(B, lo, (hi - lo) / nbins, nbins, out, st));
    return QZ_OK;
}

extern "C" qz_status qz_beam_advance(const qz_grid* g, qz_beam_view* b, const qz_box* box, const double* fld,
                                     double dt_kick, double dt_drift, int move, void* stream) {
    if (qz_status st = check_beam(g, b, box)) return st;
    if (!fld) return fail(QZ_ERR_ARG, "qz_beam_advance: null fld");
    QZ_CUDA(qzb::launch_beam_push(beam_args(g, b, box), fld, dt_kick, dt_drift, move, (cudaStream_t)stream));
    return QZ_OK;
}

extern "C" qz_status qz_beam_push(const qz_grid* g, qz_beam_view* b, const qz_box* box, const double* fld,
                                  double dt_kick, double dt_drift, int* started, void* stream) {
    if (qz_status st = check_beam(g, b, box)) return st;
    if (!fld || !started) return fail(QZ_ERR_ARG, "qz_beam_push: null pointer");
    const qzb::BeamArgs B = beam_args(g, b, box);
    if (!*started) {
        QZ_CUDA(qzb::launch_beam_push(B, fld, -0.5 * dt_kick, -0.5 * dt_kick, 0, (cudaStream_t)stream));
        *started = 1;
    }
    QZ_CUDA(qzb::launch_beam_push(B, fld, dt_kick, dt_drift, 1, (cudaStream_t)stream));
    return QZ_OK;
}

extern "C" qz_status qz_beam_push_deposit(const qz_grid* g, qz_beam_view* b, const qz_box* box, const double* fld,
                                          double dt_kick, double dt_drift, int* started, double* bsrc_next,
                                          void* stream) {
    if (qz_status st = check_beam(g, b, box)) return st;
    if (!fld || !started || !bsrc_next) return fail(QZ_ERR_ARG, "qz_beam_push_deposit: null pointer");
    const qzb::BeamArgs B = beam_args(g, b, box);
    if (!*started) {
        QZ_CUDA(qzb::launch_beam_push(B, fld, -0.5 * dt_kick, -0.5 * dt_kick, 0, (cudaStream_t)stream));
        *started = 1;
    }
    QZ_CUDA(qzb::launch_beam_push_deposit(B, fld, dt_kick, dt_drift, bsrc_next, (cudaStream_t)stream));
    return QZ_OK;
}

namespace {
// partial-sum scratch of qz_beam_sums, per device, grown on demand; kept with the context it was
// allocated in (a cudaDeviceReset frees it with the context, and the next call allocates afresh)
struct SumScratch {
    unsigned long long ctx = 0;
    double* ptr = nullptr;
    int blocks = 0;
};
constexpr int kSumDevices = 64;
SumScratch g_sum_scratch[kSumDevices];
std::mutex g_sum_mu;
}  // namespace

extern "C" qz_status qz_beam_sums(const qz_beam_view* b, double gref, double xiref, double* out17, void* stream) {
    if (!b || !out17) return fail(QZ_ERR_ARG, "qz_beam_sums: null pointer");
    if (b->n < 0) return fail(QZ_ERR_ARG, "qz_beam_sums: negative particle count");
    qzb::BeamArgs B{};
    B.x = b->x; B.y = b->y; B.px = b->px; B.py = b->py; B.pz = b->pz; B.xi = b->xi; B.w = b->w;
    B.n = (long)b->n;
    const int nb = qzb::beam_sums_blocks(B.n);
    int dev = 0;
    QZ_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kSumDevices) return fail(QZ_ERR_ARG, "qz_beam_sums: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_sum_mu);
    SumScratch& sc = g_sum_scratch[dev];
    const unsigned long long ctx = qzb::current_context_id();
    if (sc.ptr && ctx != 0 && ctx != sc.ctx) sc = SumScratch{};   // its context has ended, and the memory with it
    if (nb > sc.blocks) {
        if (sc.ptr) cudaFree(sc.ptr);
        sc = SumScratch{};
        QZ_CUDA(cudaMalloc((void**)&sc.ptr, sizeof(double) * 17 * nb));
        sc.blocks = nb;
        sc.ctx = qzb::current_context_id();
    }
    QZ_CUDA(qzb::launch_beam_sums(B, gref, xiref, sc.ptr, nb, out17, (cudaStream_t)stream));
    return QZ_OK;
}

// The moment sums for callers that must not allocate device memory: a host whose device memory
// is all owned by its own pool (every byte handed out by its arena, so a cudaMalloc behind its back
// can fail or fragment what it reserved), and a step loop that cannot afford the implicit device-
// wide synchronisation of cudaFree when qz_beam_sums grows its scratch. The partial sums live in a
// static device array of 17 x 592 doubles; the first call on each device looks up its address.
extern "C" qz_status qz_beam_sums_noalloc(const qz_beam_view* b, double gref, double xiref, double* out17,
                                          void* stream) {
    if (!b || !out17) return fail(QZ_ERR_ARG, "qz_beam_sums_noalloc: null pointer");
    if (b->n < 0) return fail(QZ_ERR_ARG, "qz_beam_sums_noalloc: negative particle count");
    qzb::BeamArgs B{};
    B.x = b->x; B.y = b->y; B.px = b->px; B.py = b->py; B.pz = b->pz; B.xi = b->xi; B.w = b->w;
    B.n = (long)b->n;
    int need = 0;
    const cudaError_t e = qzb::beam_sums_static(B, gref, xiref, out17, (cudaStream_t)stream, &need);
    if (need > qzb::kSumsStaticBlocks)
        return fail(QZ_ERR_SIZE, "qz_beam_sums_noalloc: needs " + std::to_string(need) +
                                     " partial-sum rows, the static scratch holds " +
                                     std::to_string(qzb::kSumsStaticBlocks));
    if (e != cudaSuccess) return fail(QZ_ERR_CUDA, std::string("qz_beam_sums_noalloc: ") + cudaGetErrorString(e));
    return QZ_OK;
}

extern "C" qz_status qz_sample_gaussian(double n0, double sr, double xi0, double sxi, double gamma0, double espread,
                                        double emit, double cut, double cx0, double cy0, double cxs, double cys,
                                        double xp0, double yp0, int64_t np, int nrot, int mirror, uint64_t seed,
                                        double xcut, double* out, double* gref, double* xiref, int64_t* n) {
    // src/Beam.cpp:483-570, with the same standard-library generators
    if (!out || !gref || !xiref || !n) return fail(QZ_ERR_ARG, "qz_sample_gaussian: null pointer");
    const bool flat = !(sxi > 0);
    const double len = flat ? -sxi : 0.0;
    const int nsym = nrot * (mirror ? 2 : 1);
    if (nrot < 1 || np % nsym != 0) return fail(QZ_ERR_ARG, "nparticles must be a multiple of nsym (x2 with mirror_y)");
    const double Pr = 1.0 - std::exp(-0.5 * cut * cut);
    auto Phi = [](double x) { return 0.5 * (1.0 + std::erf(x / std::sqrt(2.0))); };
    double wtot;
    if (!flat) {
        const double lo = std::max(-cut, (xcut - xi0) / sxi);
        if (lo >= cut) return fail(QZ_ERR_ARG, "xi_cut_head removes the whole beam");
        wtot = n0 * std::pow(2 * PI, 1.5) * sr * sr * sxi * Pr * (Phi(cut) - Phi(lo));
    } else {
        const double lo = std::max(xi0 - 0.5 * len, xcut), hi = xi0 + 0.5 * len;
        if (lo >= hi) return fail(QZ_ERR_ARG, "xi_cut_head removes the whole beam");
        wtot = n0 * 2 * PI * sr * sr * Pr * (hi - lo);
    }
    const double wmac = wtot / np;
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> N01(0.0, 1.0);
    std::uniform_real_distribution<double> U01(0.0, 1.0);
    const double spx = (sr > 0) ? emit / sr : 0.0;
    double aw = 0, awg = 0, awxi = 0;
    int64_t cnt = 0;
    for (int64_t i0 = 0; i0 < np; i0 += nsym) {
        double x, y;
        do { x = sr * N01(rng); y = sr * N01(rng); } while (x * x + y * y > cut * cut * sr * sr);
        double xi;
        do {
            if (!flat) { do { xi = N01(rng); } while (std::abs(xi) > cut); xi = xi0 + sxi * xi; }
            else xi = xi0 + len * (U01(rng) - 0.5);
        } while (xi < xcut);
        double px = spx * N01(rng), py = spx * N01(rng);
        const double gam = gamma0 * (1.0 + espread * N01(rng));
        px += gam * xp0;
        py += gam * yp0;
        const double pz2 = gam * gam - 1.0 - px * px - py * py;
        if (pz2 <= 0) return fail(QZ_ERR_ARG, "gamma too small for the transverse momentum spread");
        const double tpx = px - gam * xp0, tpy = py - gam * yp0;
        for (int l = 0; l < nsym; ++l) {
            const int lr = l % nrot;
            const double sgn = (l >= nrot) ? -1.0 : 1.0;
            const double ph = 2 * PI * lr / nrot, cp = std::cos(ph), sp = std::sin(ph);
            double* q = out + 7 * cnt;
            q[0] = cp * x - sp * y + cx0 + cxs * (xi - xi0);
            q[1] = sgn * (sp * x + cp * y) + cy0 + cys * (xi - xi0);
            q[2] = cp * tpx - sp * tpy + gam * xp0;
            q[3] = sgn * (sp * tpx + cp * tpy) + gam * yp0;
            q[4] = std::sqrt(pz2);
            q[5] = xi;
            q[6] = wmac;
            if (q[6] != 0) {
                const double g = std::sqrt(1 + q[2] * q[2] + q[3] * q[3] + q[4] * q[4]);
                aw += q[6];
                awg += q[6] * g;
                awxi += q[6] * q[5];
            }
            ++cnt;
        }
    }
    *gref = 0;
    *xiref = 0;
    if (aw > 0) { *gref = awg / aw; *xiref = awxi / aw; }
    *n = cnt;
    return QZ_OK;
}

// ===================================================================== time steps
struct qz_sim {
    const qz_grid* g = nullptr;
    qz_sweep* sw = nullptr;
    qz_sweep_params p{};
    int fnc = 6, bnc = 5, dnc = 3;
    double *d_fld = nullptr, *d_diag = nullptr, *d_bsrc[2] = {nullptr, nullptr}, *d_mom = nullptr;
    double* d_bstat = nullptr;   // sources of the analytic rigid beams (K, M, B_NC), added by every sweep
    int nanalytic = 0;
    int ckpt_every = 0;          // qz_sim_set_adjoint_checkpoint (0: ceil(sqrt(K)))
    int cur = 0;
    bool bsrc_valid = false;
    // exact beam deposits of m = 0 runs (BeamArgs::fx_qe): per-node quantum exponents, the limb split,
    // and the offset of the low limbs behind a (K, M, 5) block of high limbs
    struct Fx {
        double* d_q = nullptr;           // 2 M: 2^-qe_j (scales), then 2^qe_j (quanta)
        std::vector<int> qe;
        double* d_wmax = nullptr;
        int S = 0;
        long lo = 0;
        bool on = false;
        bool wanted = true;              // qz_sim_set_exact
    } fx;
    struct Beam {
        double* d = nullptr;     // 7 columns of n (the library's order: sorted by xi cell after a pipelined run)
        double* d2 = nullptr;    // second copy for reordering
        int* orig = nullptr;     // caller's index of each particle of d
        int* orig2 = nullptr;
        bool orig_identity = true;
        int64_t n = 0;
        double q = -1, m = 1, gref = 0, xiref = 0;
        int rigid = 0, started = 0, pusher = 0;
        qz_beam_view view() const {
            qz_beam_view v;
            v.x = d; v.y = d + n; v.px = d + 2 * n; v.py = d + 3 * n; v.pz = d + 4 * n; v.xi = d + 5 * n; v.w = d + 6 * n;
            v.n = n; v.q = q; v.m = m; v.pusher = pusher;
            return v;
        }
    };
    std::vector<Beam> beams;
    qz_counters cnt{};
    // time-step pipeline (qz_pipeline.cu): options, last schedule, buffers kept between runs
    struct Pipe {
        int enabled = 1, sweep_ctas = 0, bucket = 512, span = 1;
        double timeout_s = 20.0;
        int info[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // grid, sweep CTAs, worker CTAs, ring, buckets, bucket size, pipelined
        int trace = 0;                             // record sweep start / end times
        unsigned long long* d_trace = nullptr;
        size_t trace_n = 0;
        std::vector<unsigned long long> h_trace;
        cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};   // start, launch, kernel end, end
        float times[3] = {0, 0, 0};
        double *fld = nullptr, *diag = nullptr, *bsrc = nullptr;
        int ring = 0;
        bool clean = false;                        // every beam-source slot is zero
        double* ps = nullptr;
        size_t ps_n = 0;
        double* m1s = nullptr;                     // modes = 1 scratch of the sweep CTAs
        size_t m1s_n = 0;
        int* sync = nullptr;
        size_t sync_n = 0;
        int* bk = nullptr;                         // beam, start, end, cmax, cmin (5 x nbk), then cnt_le (K)
        size_t bk_n = 0;
        double *pmom = nullptr, *mom = nullptr;
        size_t pmom_n = 0, mom_n = 0;
        qzb::CellSortBuf sort{};
        long sort_n = 0;
        int* cmin = nullptr;                       // group starts of one beam
        size_t cm_n = 0;
    } pipe;
    ~qz_sim() {
        if (fx.d_q) cudaFree(fx.d_q);
        if (fx.d_wmax) cudaFree(fx.d_wmax);
        for (auto& b : beams)
            for (void* q : {(void*)b.d, (void*)b.d2, (void*)b.orig, (void*)b.orig2})
                if (q) cudaFree(q);
        for (double* q : {d_fld, d_diag, d_bsrc[0], d_bsrc[1], d_mom, d_bstat, pipe.fld, pipe.diag, pipe.bsrc, pipe.ps,
                          pipe.m1s, pipe.pmom, pipe.mom})
            if (q) cudaFree(q);
        for (void* q : {(void*)pipe.sync, (void*)pipe.bk, (void*)pipe.sort.keys[0], (void*)pipe.sort.keys[1],
                        (void*)pipe.sort.vals[0], (void*)pipe.sort.vals[1], pipe.sort.tmp, (void*)pipe.sort.nlive,
                        (void*)pipe.cmin, (void*)pipe.d_trace})
            if (q) cudaFree(q);
        for (cudaEvent_t e : pipe.ev)
            if (e) cudaEventDestroy(e);
        qz_sweep_destroy(sw);
    }
};

extern "C" qz_status qz_sim_create(const qz_grid* g, const qz_sweep_params* p, qz_sim** out) {
    if (!g || !p || !out) return fail(QZ_ERR_ARG, "qz_sim_create: null pointer");
    *out = nullptr;
    qz_sim* s = new (std::nothrow) qz_sim;
    if (!s) return fail(QZ_ERR_NOMEM, "qz_sim_create: out of host memory");
    s->g = g;
    s->p = *p;
    if (qz_status st = qz_sweep_create(g, p, &s->sw)) { delete s; return st; }
    s->fnc = p->modes ? 18 : 6;
    s->bnc = p->modes ? 15 : 5;
    s->dnc = p->modes ? 9 : 3;
    const size_t KM = (size_t)p->K * g->M;
    if (cudaMalloc((void**)&s->d_fld, sizeof(double) * KM * s->fnc) != cudaSuccess ||
        cudaMalloc((void**)&s->d_diag, sizeof(double) * KM * s->dnc) != cudaSuccess ||
        cudaMalloc((void**)&s->d_bsrc[0], sizeof(double) * KM * s->bnc * (p->modes ? 1 : 2)) != cudaSuccess ||
        cudaMalloc((void**)&s->d_bsrc[1], sizeof(double) * KM * s->bnc * (p->modes ? 1 : 2)) != cudaSuccess) {
        delete s;
        return fail(QZ_ERR_NOMEM, "qz_sim_create: device allocation failed");
    }
    *out = s;
    return QZ_OK;
}

extern "C" qz_status qz_sim_destroy(qz_sim* s) {
    delete s;
    return QZ_OK;
}

extern "C" qz_status qz_sim_set_beam_pusher(qz_sim* s, int b, int pusher) {
    if (!s || b < 0 || b >= (int)s->beams.size() || pusher < 0 || pusher > 3)
        return fail(QZ_ERR_ARG, "qz_sim_set_beam_pusher: bad beam index or pusher (0..3)");
    s->beams[b].pusher = pusher;
    return QZ_OK;
}

extern "C" qz_status qz_sim_beam_slice_sums(qz_sim* s, int b, double lo, double hi, int nbins, double* out_host) {
    if (!s || b < 0 || b >= (int)s->beams.size() || !out_host || nbins < 1)
        return fail(QZ_ERR_ARG, "qz_sim_beam_slice_sums: bad argument");
    double* d = nullptr;
    if (cudaMalloc((void**)&d, sizeof(double) * 9 * (size_t)nbins) != cudaSuccess)
        return fail(QZ_ERR_NOMEM, "qz_sim_beam_slice_sums: device allocation failed");
    const qz_beam_view v = s->beams[b].view();
    qz_status st = qz_beam_slice_sums(&v, lo, hi, nbins, d, nullptr);
    if (st == QZ_OK && cudaMemcpy(out_host, d, sizeof(double) * 9 * (size_t)nbins, cudaMemcpyDeviceToHost) != cudaSuccess)
        st = fail(QZ_ERR_CUDA, "qz_sim_beam_slice_sums: copy failed");
    cudaFree(d);
    return st;
}

extern "C" qz_status qz_sim_add_analytic_beam(qz_sim* s, const qz_analytic_beam* b) {
    if (!s || !b) return fail(QZ_ERR_ARG, "qz_sim_add_analytic_beam: null pointer");
    qz_box box;
    box.xi_min = s->p.xi_min; box.dxi = s->p.dxi; box.K = s->p.K; box.ngp = s->p.ngp; box.modes = s->p.modes;
    qzb::AnalyticArgs P;
    if (qz_status st = analytic_args(s->g, b, &box, P)) return st;
    const size_t n = (size_t)s->p.K * s->g->M * s->bnc;
    if (!s->d_bstat) {
        if (cudaMalloc((void**)&s->d_bstat, sizeof(double) * n) != cudaSuccess) {
            s->d_bstat = nullptr;
            return fail(QZ_ERR_NOMEM, "qz_sim_add_analytic_beam: device allocation failed");
        }
        QZ_CUDA(cudaMemset(s->d_bstat, 0, sizeof(double) * n));
    }
    QZ_CUDA(qzb::launch_deposit_analytic(P, s->d_bstat, nullptr));
    QZ_CUDA(cudaDeviceSynchronize());
    s->sw->base.bstat = s->d_bstat;
    ++s->nanalytic;
    return QZ_OK;
}

extern "C" qz_status qz_sim_add_beam(qz_sim* s, const double* p7, int64_t n, double q, double m, int rigid,
                                     double gref, double xiref) {
    if (!s || (n > 0 && !p7) || n < 0) return fail(QZ_ERR_ARG, "qz_sim_add_beam: bad argument");
    qz_sim::Beam b;
    b.n = n; b.q = q; b.m = m; b.rigid = rigid; b.gref = gref; b.xiref = xiref;
    std::vector<double> cols((size_t)7 * (n > 0 ? n : 1), 0.0);
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 7; ++c) cols[(size_t)c * n + i] = p7[7 * i + c];
    if (qz_status st = dev_upload(&b.d, cols)) return st;
    const size_t nn = (size_t)(n > 0 ? n : 1);
    if (cudaMalloc((void**)&b.d2, sizeof(double) * 7 * nn) != cudaSuccess ||
        cudaMalloc((void**)&b.orig, sizeof(int) * nn) != cudaSuccess ||
        cudaMalloc((void**)&b.orig2, sizeof(int) * nn) != cudaSuccess) {
        for (void* q : {(void*)b.d, (void*)b.d2, (void*)b.orig, (void*)b.orig2})
            if (q) cudaFree(q);
        return fail(QZ_ERR_NOMEM, "qz_sim_add_beam: device allocation failed");
    }
    if (s->beams.size() >= (size_t)qzb::kMaxBeams && s->pipe.enabled)
        s->pipe.enabled = 0;   // the pipeline handles up to kMaxBeams beams; more run step by step
    s->beams.push_back(b);
    const int nb = (int)s->beams.size();
    if (s->d_mom) cudaFree(s->d_mom);
    s->d_mom = nullptr;
    QZ_CUDA(cudaMalloc((void**)&s->d_mom, sizeof(double) * 17 * nb));
    s->bsrc_valid = false;
    return QZ_OK;
}

namespace {
qz_box sim_box(const qz_sim* s) {
    qz_box box;
    box.xi_min = s->p.xi_min;
    box.dxi = s->p.dxi;
    box.K = s->p.K;
    box.ngp = s->p.ngp;
    box.modes = s->p.modes;
    return box;
}
}  // namespace

namespace {

// The exact beam deposits of an m = 0 run: every contribution to node j is bounded by
// 2 (sum over beams of max |w q|) / V_j / dxi (the weights of the particles do not change during a run;
// |1 - v_z| <= 2 and every other factor is at most 1), so the quantum of node j is that bound / 2^B.
// With at most n contributions per value (n = all beam particles, 2^nbits > n) the limbs split at
// S = 53 - nbits and B = 2 S keep both limb sums integers below 2^53 (exact in FP64, beam_fx_add).
// The run deposits exactly for m = 0 up to 2^25 particles (B >= 56: the quantum is at most 2^-56 of
// the bound); m = 1 runs and larger beams keep FP64 reductions.
// the node quanta for n contributions bounded by wq (sum over beams of max |w q|): every contribution to
// node j is below bound_j = 2 wq / V_j / dxi < 2^(qe_j + B); S = 53 - nbits and B = 2 S with 2^nbits > n.
// False beyond 2^25 contributions (the quantum would exceed 2^-56 of the bound).
bool fx_quanta(const qz_grid* g, double dxi, double wq, long ntot, std::vector<int>& qe, int& S) {
    int nbits = 1;
    while (nbits < 62 && (1L << nbits) <= ntot) ++nbits;
    if (nbits > 25) return false;
    S = 53 - nbits;
    const int B = 2 * S;
    qe.assign(g->M, 0);
    for (int j = 0; j < g->M; ++j) {
        const double bound = 2.0 * wq * g->inv_V[j] / dxi;
        int e = 0;
        if (bound > 0.0 && std::isfinite(bound)) std::frexp(bound, &e);    // bound < 2^e
        qe[j] = e - B;
    }
    return true;
}

qz_status fx_upload(const std::vector<int>& qe, double* d_q) {
    const size_t M = qe.size();
    std::vector<double> q(2 * M);
    for (size_t j = 0; j < M; ++j) {
        q[j] = std::ldexp(1.0, -qe[j]);
        q[M + j] = std::ldexp(1.0, qe[j]);
    }
    QZ_CUDA(cudaMemcpy(d_q, q.data(), sizeof(double) * q.size(), cudaMemcpyHostToDevice));
    return QZ_OK;
}

qz_status fx_prepare(qz_sim* s, cudaStream_t st) {
    auto& F = s->fx;
    const bool was = F.on;
    F.on = false;
    if (was) s->bsrc_valid = false;             // the format of kept sources changes back to doubles
    if (!F.wanted || s->p.modes != 0 || s->beams.empty()) return QZ_OK;
    const int M = s->g->M;
    long ntot = 0;
    for (const auto& b : s->beams) ntot += (long)b.n;
    {
        std::vector<int> probe;
        int Sp = 0;
        if (!fx_quanta(s->g, s->p.dxi, 1.0, ntot, probe, Sp)) return QZ_OK;   // beyond 2^25: FP64 reductions
    }
    if (!F.d_wmax && cudaMalloc((void**)&F.d_wmax, sizeof(double) * qzb::kMaxBeams * 2) != cudaSuccess) {
        F.d_wmax = nullptr;
        return fail(QZ_ERR_NOMEM, "qz_sim_run: device allocation failed (deposit bounds)");
    }
    const qz_box box = sim_box(s);
    const int nb = std::min((int)s->beams.size(), 2 * qzb::kMaxBeams);
    QZ_CUDA(cudaMemsetAsync(F.d_wmax, 0, sizeof(double) * nb, st));
    double wq = 0.0;
    std::vector<double> wm(nb, 0.0);
    for (int b = 0; b < nb; ++b) {
        const qz_beam_view v = s->beams[b].view();
        QZ_CUDA(qzb::launch_beam_wmax(beam_args(s->g, &v, &box), F.d_wmax + b, st));
    }
    QZ_CUDA(cudaMemcpyAsync(wm.data(), F.d_wmax, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
    QZ_CUDA(cudaStreamSynchronize(st));
    if ((int)s->beams.size() > nb) return QZ_OK;    // more beams than bounds: FP64 reductions
    for (int b = 0; b < nb; ++b) wq += wm[b] * std::fabs(s->beams[b].q);
    std::vector<int> qe;
    int S = 0;
    fx_quanta(s->g, s->p.dxi, wq, ntot, qe, S);
    if (!F.d_q && cudaMalloc((void**)&F.d_q, sizeof(double) * 2 * M) != cudaSuccess) {
        F.d_q = nullptr;
        return fail(QZ_ERR_NOMEM, "qz_sim_run: device allocation failed (deposit bounds)");
    }
    if (qe != F.qe || F.S != S) {
        if (qz_status e = fx_upload(qe, F.d_q)) return e;
        F.qe = qe;
        s->bsrc_valid = false;                      // sources kept from the last run used other quanta
    }
    if (!was) s->bsrc_valid = false;
    F.S = S;
    F.lo = (long)s->p.K * M * s->bnc;
    F.on = true;
    return QZ_OK;
}

// BeamArgs of beam b with the exact deposits of the run when they are on
qzb::BeamArgs sim_beam_args(const qz_sim* s, const qz_beam_view* v, const qz_box* box) {
    qzb::BeamArgs B = beam_args(s->g, v, box);
    if (s->fx.on) {
        B.fx_scale = s->fx.d_q;
        B.fx_inv2s = std::ldexp(1.0, -s->fx.S);
        B.fx_2s = std::ldexp(1.0, s->fx.S);
        B.fx_lo = s->fx.lo;
    }
    return B;
}

void sim_sweep_fx(const qz_sim* s, qzb::SweepArgs& A) {
    A.bq = s->fx.on ? s->fx.d_q + s->g->M : nullptr;
    A.bfx_2s = std::ldexp(1.0, s->fx.S);
    A.bfx_lo = s->fx.lo;
}

// the sim's beam-source buffers: doubles for modes = 1, two limbs per value for m = 0
size_t sim_bsrc_doubles(const qz_sim* s) { return (size_t)s->p.K * s->g->M * s->bnc * (s->p.modes ? 1 : 2); }

// the deposit of every beam into bsrc (cleared first), exact when the run's quanta are set
qz_status sim_deposit_all(qz_sim* s, double* bsrc, cudaStream_t st) {
    const qz_box box = sim_box(s);
    QZ_CUDA(cudaMemsetAsync(bsrc, 0, sizeof(double) * sim_bsrc_doubles(s), st));
    for (auto& b : s->beams) {
        const qz_beam_view v = b.view();
        QZ_CUDA(qzb::launch_beam_deposit(sim_beam_args(s, &v, &box), bsrc, st));
    }
    return QZ_OK;
}

// one sweep of a run; its counters add to the sweep's device counters, which the run clears at its start
qz_status sim_sweep(qz_sim* s, const double* bsrc, cudaStream_t st) {
    SweepExtra x;
    x.accumulate = true;
    if (s->fx.on) {
        x.bq = s->fx.d_q + s->g->M;
        x.bfx_2s = std::ldexp(1.0, s->fx.S);
        x.bfx_lo = s->fx.lo;
    }
    return sweep_launch(s->sw, bsrc, s->d_fld, s->d_diag, nullptr, st, x);
}

// one time step's push of beam b with the deposit into bsrc_next (leapfrog start-up first); rigid
// beams only deposit
qz_status sim_push_deposit(qz_sim* s, qz_sim::Beam& b, double dt_kick, double dt_drift, double* bsrc_next,
                           cudaStream_t st) {
    const qz_box box = sim_box(s);
    const qz_beam_view v = b.view();
    const qzb::BeamArgs B = sim_beam_args(s, &v, &box);
    if (b.rigid) {
        QZ_CUDA(qzb::launch_beam_deposit(B, bsrc_next, st));
        return QZ_OK;
    }
    if (!b.started) {
        QZ_CUDA(qzb::launch_beam_push(B, s->d_fld, -0.5 * dt_kick, -0.5 * dt_kick, 0, st));
        b.started = 1;
    }
    if (B.fx_scale) {
        // exact sources: deposit the stored particles with the deposit kernel, so that any path that
        // deposits the same particles (a staged run's slabs, qz_beam_deposit_fx) gives the same limbs (the
        // fused kernel shares subexpressions with the push and rounds the deposit values differently)
        QZ_CUDA(qzb::launch_beam_push(B, s->d_fld, dt_kick, dt_drift, 1, st));
        QZ_CUDA(qzb::launch_beam_deposit(B, bsrc_next, st));
    } else {
        QZ_CUDA(qzb::launch_beam_push_deposit(B, s->d_fld, dt_kick, dt_drift, bsrc_next, st));
    }
    return QZ_OK;
}

template <class T>
qz_status grow(T** p, size_t* have, size_t need, const char* what) {
    if (*have >= need && *p) return QZ_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *have = 0;
    if (cudaMalloc((void**)p, sizeof(T) * (need > 0 ? need : 1)) != cudaSuccess) {
        cudaGetLastError();
        return fail(QZ_ERR_NOMEM, std::string("qz_sim_run: device allocation failed (") + what + ")");
    }
    *have = need;
    return QZ_OK;
}

// Simulation::run for constant dt as one pipelined launch (qz_pipeline.cu): the beams are put in
// xi-cell order (their caller order is kept in orig), cut into buckets, the step-0 beam sources are
// deposited into ring slot 0, then all sweeps and pushes run concurrently.
// what a forward run records for the adjoint (qz_sim_adjoint): the plasma trajectory of every sweep
// and the beams of every step before its push; with it the rings keep every step
struct FwdRecord {
    double* traj = nullptr;
    size_t traj_slot = 0;
    int traj_every = 1;                 // checkpoint slices k = 0, C, 2C, ... only (C > 1)
    double* wrec = nullptr;             // W+ radial field per slice, K M per step
    double* snap = nullptr;
    size_t snap_step = 0;
    long snap_off[qzb::kMaxBeams] = {0, 0, 0, 0};
};

qz_status run_pipelined(qz_sim* s, int nsteps, double dt, double* mom_host, cudaStream_t st,
                        const FwdRecord* rec = nullptr) {
    auto& P_ = s->pipe;
    const int K = s->p.K, M = s->g->M, nb = (int)s->beams.size();
    const qz_box box = sim_box(s);
    if (!P_.ev[0])
        for (auto& e : P_.ev) QZ_CUDA(cudaEventCreate(&e));
    QZ_CUDA(cudaEventRecord(P_.ev[0], st));
    if (qz_status e = fx_prepare(s, st)) return e;
    // 1. order each beam by (xi cell, radial cell); buckets of at most P_.bucket live particles
    if ((unsigned long long)(K + 2) * (unsigned long long)M >= (1ull << 31))
        return fail(QZ_ERR_SIZE, "qz_sim_run: K * M too large for the pipelined run's sort keys");
    long nmax = 1;
    for (auto& b : s->beams) nmax = std::max<long>(nmax, (long)b.n);
    if (P_.sort_n < nmax) {
        for (void* q : {(void*)P_.sort.keys[0], (void*)P_.sort.keys[1], (void*)P_.sort.vals[0],
                        (void*)P_.sort.vals[1], P_.sort.tmp, (void*)P_.sort.nlive})
            if (q) cudaFree(q);
        P_.sort = qzb::CellSortBuf{};
        P_.sort_n = 0;
        P_.sort.tmp_bytes = qzb::cell_sort_temp_bytes(nmax);
        if (cudaMalloc((void**)&P_.sort.keys[0], sizeof(unsigned) * nmax) != cudaSuccess ||
            cudaMalloc((void**)&P_.sort.keys[1], sizeof(unsigned) * nmax) != cudaSuccess ||
            cudaMalloc((void**)&P_.sort.vals[0], sizeof(int) * nmax) != cudaSuccess ||
            cudaMalloc((void**)&P_.sort.vals[1], sizeof(int) * nmax) != cudaSuccess ||
            cudaMalloc(&P_.sort.tmp, P_.sort.tmp_bytes + 16) != cudaSuccess ||
            cudaMalloc((void**)&P_.sort.nlive, sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            return fail(QZ_ERR_NOMEM, "qz_sim_run: device allocation failed (sort buffers)");
        }
        P_.sort_n = nmax;
    }
    const int bk = P_.bucket > 0 ? P_.bucket : 512;
    struct Bucket { int cmin, beam, start, end, cmax; };
    std::vector<Bucket> list;
    for (int q = 0; q < nb; ++q) {
        auto& b = s->beams[q];
        if (b.n <= 0) continue;
        if (b.orig_identity) {
            QZ_CUDA(qzb::fill_iota(b.orig, b.n, st));
            b.orig_identity = false;
        }
        const qz_beam_view v = b.view();
        const qzb::BeamArgs B = beam_args(s->g, &v, &box);
        QZ_CUDA(qzb::cell_sort(B, b.d, b.d2, b.orig, b.orig2, P_.sort, st));
        std::swap(b.d, b.d2);
        std::swap(b.orig, b.orig2);
        int nlive = 0;
        QZ_CUDA(cudaMemcpyAsync(&nlive, P_.sort.nlive, sizeof(int), cudaMemcpyDeviceToHost, st));
        QZ_CUDA(cudaStreamSynchronize(st));
        // buckets: never across a group of span cells, at most bk particles (near-equal parts)
        const int span = P_.span > 0 ? P_.span : 1;
        const int ngroups = (K + 1 + span - 1) / span;
        if (qz_status e = grow(&P_.cmin, &P_.cm_n, (size_t)ngroups + 1, "bucket groups")) return e;
        QZ_CUDA(qzb::group_starts(P_.sort, nlive, span * M, ngroups, P_.cmin, st));
        std::vector<int> gs(ngroups + 1);
        QZ_CUDA(cudaMemcpyAsync(gs.data(), P_.cmin, sizeof(int) * gs.size(), cudaMemcpyDeviceToHost, st));
        QZ_CUDA(cudaStreamSynchronize(st));
        for (int g = 0; g < ngroups; ++g) {
            const int a = gs[g], cnt = gs[g + 1] - gs[g];
            if (cnt <= 0) continue;
            const int parts = (cnt + bk - 1) / bk;
            const int cmin = g * span - 1, cmax = std::min(g * span + span - 2, K - 1);
            for (int i = 0; i < parts; ++i)
                list.push_back({cmin, q, a + (int)((long)cnt * i / parts), a + (int)((long)cnt * (i + 1) / parts), cmax});
        }
    }
    std::stable_sort(list.begin(), list.end(), [](const Bucket& a, const Bucket& b) { return a.cmin < b.cmin; });
    const int nbk = (int)list.size();
    std::vector<int> bkh((size_t)5 * nbk + K);
    for (int i = 0; i < nbk; ++i) {
        bkh[i] = list[i].beam;
        bkh[nbk + i] = list[i].start;
        bkh[2 * nbk + i] = list[i].end;
        bkh[3 * nbk + i] = list[i].cmax;
        bkh[4 * nbk + i] = list[i].cmin;
    }
    for (int r = 0, c = 0; r < K; ++r) {
        while (c < nbk && list[c].cmin <= r) ++c;
        bkh[5 * nbk + r] = c;
    }
    if (qz_status e = grow(&P_.bk, &P_.bk_n, bkh.size(), "buckets")) return e;
    QZ_CUDA(cudaMemcpyAsync(P_.bk, bkh.data(), sizeof(int) * bkh.size(), cudaMemcpyHostToDevice, st));

    // 2. schedule: one CTA per SM; sweeps for every step up to the SMs left after the workers
    qzb::PipeArgs A{};
    A.sw = s->sw->base;
    A.modes = s->p.modes;
    A.bnc = s->bnc;
    A.sw.counters = s->sw->d_cnt;
    A.sw.timing = nullptr;
    if (s->sw->timing) {                               // phase cycles of every sweep (qz_sim_timing)
        QZ_CUDA(cudaMemsetAsync(s->sw->d_tim, 0, sizeof(unsigned long long) * 16, st));
        A.sw.timing = s->sw->d_tim;
    }
    int sms = 0;
    const int grid = qzb::pipeline_max_grid(A, &sms);
    if (grid < 2) return fail(QZ_ERR_UNSUPPORTED, "qz_sim_run: the pipelined kernel cannot be resident here");
    const int g1 = std::min(grid, sms);
    const int wmin = std::max(8, (2 * g1) / 5);             // measured best: ~2/5 of the SMs push
    int nsweep = P_.sweep_ctas > 0 ? P_.sweep_ctas : std::min(nsteps + 1, g1 - wmin);
    nsweep = std::max(1, std::min({nsweep, nsteps + 1, g1 - 1}));
    // 3. buffers
    const size_t KM = (size_t)K * M;
    const size_t bslot = sim_bsrc_doubles(s);           // a beam-source slot: two limbs per value for m = 0
    // ring slots: one per step in flight; one per step of the run when that fits in half the free memory,
    // which lets the push workers read the field rows through L1 (PipeArgs::fld_l1)
    int ring = rec ? std::max(2, nsteps + 1) : std::max(2, std::min(nsteps + 1, nsweep + 2));
    if (ring < nsteps + 1 && P_.ring >= nsteps + 1) {
        ring = nsteps + 1;                              // the rings already hold a slot per step
    } else if (ring < nsteps + 1) {
        size_t fr = 0, tot = 0;
        const size_t per = sizeof(double) * (KM * (s->fnc + s->dnc) + bslot);
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess && (size_t)(nsteps + 1 - std::max(P_.ring, 0)) * per < fr / 2)
            ring = nsteps + 1;
        cudaGetLastError();
    }
    if (P_.ring < ring) {
        for (double* q : {P_.fld, P_.diag, P_.bsrc})
            if (q) cudaFree(q);
        P_.fld = P_.diag = P_.bsrc = nullptr;
        P_.ring = 0;
        if (cudaMalloc((void**)&P_.fld, sizeof(double) * KM * s->fnc * ring) != cudaSuccess ||
            cudaMalloc((void**)&P_.diag, sizeof(double) * KM * s->dnc * ring) != cudaSuccess ||
            cudaMalloc((void**)&P_.bsrc, sizeof(double) * bslot * ring) != cudaSuccess) {
            cudaGetLastError();
            return fail(QZ_ERR_NOMEM, "qz_sim_run: device allocation failed (field rings)");
        }
        P_.ring = ring;
        P_.clean = false;
    }
    if (!P_.clean) QZ_CUDA(cudaMemsetAsync(P_.bsrc, 0, sizeof(double) * bslot * P_.ring, st));
    P_.clean = false;
    const size_t ps_slot = (size_t)(6 + 5 * s->p.ab_order) * std::max(1, s->sw->npad);
    if (qz_status e = grow(&P_.ps, &P_.ps_n, ps_slot * nsweep, "plasma scratch")) return e;
    const size_t m1s_slot = s->p.modes == 1 ? (size_t)63 * M : 0;
    if (m1s_slot)
        if (qz_status e = grow(&P_.m1s, &P_.m1s_n, m1s_slot * nsweep, "mode-1 scratch")) return e;
    const size_t nsync = 4 * (size_t)(nsteps + 1) + nbk + 2;
    if (qz_status e = grow(&P_.sync, &P_.sync_n, nsync, "sync words")) return e;
    QZ_CUDA(cudaMemsetAsync(P_.sync, 0, sizeof(int) * nsync, st));
    int* bdone = P_.sync + 4 * (size_t)(nsteps + 1);
    if (nbk) QZ_CUDA(cudaMemsetAsync(bdone, 0xff, sizeof(int) * nbk, st));
    const bool moms = mom_host != nullptr && nb > 0;
    if (moms) {
        if (qz_status e = grow(&P_.pmom, &P_.pmom_n, (size_t)(nsteps + 1) * std::max(nbk, 1) * 17, "moments"))
            return e;
        if (qz_status e = grow(&P_.mom, &P_.mom_n, (size_t)(nsteps + 1) * nb * 17, "moments")) return e;
        QZ_CUDA(cudaMemsetAsync(P_.mom, 0, sizeof(double) * (nsteps + 1) * nb * 17, st));
    }
    QZ_CUDA(cudaMemsetAsync(s->sw->d_cnt, 0, sizeof(unsigned long long) * 4, st));
    // 4. beam sources of step 0 into slot 0
    for (auto& b : s->beams) {
        const qz_beam_view v = b.view();
        QZ_CUDA(qzb::launch_beam_deposit(sim_beam_args(s, &v, &box), P_.bsrc, st));
    }
    sim_sweep_fx(s, A.sw);
    // 5. launch
    A.nsteps = nsteps;
    A.nsweep = nsweep;
    A.ring = ring;
    A.fld_l1 = (ring >= nsteps + 1 && (M * s->fnc) % 16 == 0) ? 1 : 0;
    A.fld_slot = KM * s->fnc;
    A.diag_slot = KM * s->dnc;
    A.bsrc_slot = bslot;
    A.ps_slot = ps_slot;
    A.fld = P_.fld;
    A.diag = P_.diag;
    A.bsrc = P_.bsrc;
    A.ps = P_.ps;
    A.m1s = P_.m1s;
    A.m1s_slot = m1s_slot;
    A.nbeams = nb;
    for (int q = 0; q < nb; ++q) {
        const auto& b = s->beams[q];
        const qz_beam_view v = b.view();
        A.beam[q] = sim_beam_args(s, &v, &box);
        A.rigid[q] = b.rigid;
        A.startup[q] = b.started ? 0 : 1;
        A.gref[q] = b.gref;
        A.xiref[q] = b.xiref;
    }
    A.dt_kick = dt;
    A.dt_drift = dt;
    A.nbk = nbk;
    A.bk_beam = P_.bk;
    A.bk_start = P_.bk + nbk;
    A.bk_end = P_.bk + 2 * nbk;
    A.bk_cmax = P_.bk + 3 * nbk;
    A.bk_cmin = P_.bk + 4 * nbk;
    A.cnt_le = P_.bk + 5 * nbk;
    A.pmom = moms ? P_.pmom : nullptr;
    A.prog = P_.sync;
    A.sdone = P_.sync + (nsteps + 1);
    A.pdone = P_.sync + 2 * (size_t)(nsteps + 1);
    A.next = P_.sync + 3 * (size_t)(nsteps + 1);
    A.bdone = bdone;
    A.err = bdone + nbk;
    A.lo = bdone + nbk + 1;
    A.timeout_ns = (unsigned long long)(P_.timeout_s * 1e9);
    if (rec) {
        A.traj = rec->traj;
        A.traj_slot = rec->traj_slot;
        A.sw.traj_every = rec->traj_every;
        A.wrec = rec->wrec;
        A.snap = rec->snap;
        A.snap_step = rec->snap_step;
        for (int q = 0; q < qzb::kMaxBeams; ++q) A.snap_off[q] = rec->snap_off[q];
    }
    A.trace = nullptr;
    if (P_.trace) {
        const size_t ntr = (size_t)qzb::kTraceStride * (nsteps + 1) + qzb::kWorkerTotals;
        if (qz_status e = grow(&P_.d_trace, &P_.trace_n, ntr, "trace")) return e;
        QZ_CUDA(cudaMemsetAsync(P_.d_trace, 0, sizeof(unsigned long long) * ntr, st));
        A.trace = P_.d_trace;
    }
    QZ_CUDA(cudaEventRecord(P_.ev[1], st));
    QZ_CUDA(qzb::launch_pipeline(A, g1, st));
    QZ_CUDA(cudaEventRecord(P_.ev[2], st));
    if (moms) QZ_CUDA(qzb::launch_moments_reduce(A, P_.mom, st));
    int err = 0;
    unsigned long long h[4];
    QZ_CUDA(cudaMemcpyAsync(&err, A.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    QZ_CUDA(cudaMemcpyAsync(h, s->sw->d_cnt, sizeof(h), cudaMemcpyDeviceToHost, st));
    if (moms)
        QZ_CUDA(cudaMemcpyAsync(mom_host, P_.mom, sizeof(double) * (nsteps + 1) * nb * 17, cudaMemcpyDeviceToHost, st));
    // the last sweep's fields are what qz_sim_fields returns
    const int last = nsteps % ring;
    QZ_CUDA(cudaMemcpyAsync(s->d_fld, P_.fld + (size_t)last * A.fld_slot, sizeof(double) * A.fld_slot,
                            cudaMemcpyDeviceToDevice, st));
    QZ_CUDA(cudaMemcpyAsync(s->d_diag, P_.diag + (size_t)last * A.diag_slot, sizeof(double) * A.diag_slot,
                            cudaMemcpyDeviceToDevice, st));
    if (P_.trace) {
        P_.h_trace.assign((size_t)qzb::kTraceStride * (nsteps + 1) + qzb::kWorkerTotals, 0ull);
        QZ_CUDA(cudaMemcpyAsync(P_.h_trace.data(), P_.d_trace, sizeof(unsigned long long) * P_.h_trace.size(),
                                cudaMemcpyDeviceToHost, st));
    }
    QZ_CUDA(cudaEventRecord(P_.ev[3], st));
    QZ_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < 3; ++i) QZ_CUDA(cudaEventElapsedTime(&P_.times[i], P_.ev[i], P_.ev[i + 1]));
    s->cnt.lost += h[0];
    s->cnt.nonfinite += h[1];
    s->cnt.trapped += h[2];
    s->cnt.subslices += h[3];
    s->bsrc_valid = false;
    const int info[8] = {g1, nsweep, g1 - nsweep, ring, nbk, bk, 1, P_.span > 0 ? P_.span : 1};
    std::copy(info, info + 8, P_.info);
    if (err) {
        s->cnt.giveup += 1;
        static const char* site[] = {"?", "field ring slot", "beam-source rows", "no push task ready"};
        const int w = (err >> 8) & 0xff;
        return fail(QZ_ERR_CUDA, std::string("qz_sim_run: pipeline wait timed out (") + site[w <= 3 ? w : 0] +
                                     "); results of this call are invalid");
    }
    P_.clean = true;
    if (nsteps > 0)
        for (auto& b : s->beams)
            if (!b.rigid) b.started = 1;
    return QZ_OK;
}

qz_status run_sequential(qz_sim* s, int nsteps, double dt, double* mom_host, cudaStream_t st) {
    void* stream = (void*)st;
    const int nb = (int)s->beams.size();
    if (qz_status e = fx_prepare(s, st)) return e;
    QZ_CUDA(cudaMemsetAsync(s->sw->d_cnt, 0, sizeof(unsigned long long) * 4, st));   // the run's counters
    if (!s->bsrc_valid) {
        if (qz_status e = sim_deposit_all(s, s->d_bsrc[s->cur], st)) return e;
        s->bsrc_valid = true;
    }
    double dt_prev = dt;
    for (int n = 0; n <= nsteps; ++n) {
        if (qz_status e = sim_sweep(s, s->d_bsrc[s->cur], st)) return e;
        if (mom_host) {
            for (int b = 0; b < nb; ++b) {
                const qz_beam_view v = s->beams[b].view();
                if (qz_status e = qz_beam_sums(&v, s->beams[b].gref, s->beams[b].xiref, s->d_mom + 17 * b, stream))
                    return e;
            }
            QZ_CUDA(cudaMemcpyAsync(mom_host + (size_t)n * nb * 17, s->d_mom, sizeof(double) * 17 * nb,
                                    cudaMemcpyDeviceToHost, st));
        }
        if (n < nsteps) {
            const double dkick = 0.5 * (dt_prev + dt), ddrift = dt;
            const int nxt = 1 - s->cur;
            QZ_CUDA(cudaMemsetAsync(s->d_bsrc[nxt], 0, sizeof(double) * sim_bsrc_doubles(s), st));
            for (auto& b : s->beams)
                if (qz_status e = sim_push_deposit(s, b, dkick, ddrift, s->d_bsrc[nxt], st)) return e;
            s->cur = nxt;
            dt_prev = dt;
        }
    }
    unsigned long long h[4];
    QZ_CUDA(cudaMemcpyAsync(h, s->sw->d_cnt, sizeof(h), cudaMemcpyDeviceToHost, st));
    QZ_CUDA(cudaStreamSynchronize(st));
    s->cnt.lost += h[0];
    s->cnt.nonfinite += h[1];
    s->cnt.trapped += h[2];
    s->cnt.subslices += h[3];
    s->pipe.info[6] = 0;
    return QZ_OK;
}

}  // namespace

extern "C" qz_status qz_sim_run(qz_sim* s, int nsteps, double dt, double* mom_host, void* stream) {
    if (!s || nsteps < 0) return fail(QZ_ERR_ARG, "qz_sim_run: bad argument");
    if (!(dt > 0.0)) return fail(QZ_ERR_ARG, "qz_sim_run: dt must be positive");
    cudaStream_t st = (cudaStream_t)stream;
    bool vay_only = true;                 // the pipeline's push workers use Vay
    for (const auto& b : s->beams) vay_only = vay_only && b.pusher == 0;
    // (the pipeline's sweep CTAs have 512 threads: m = 1 runs with more nodes go step by step)
    const bool wide_m1 = s->p.modes == 1 && s->sw->base.M > qzb::kSweepThreads;
    if (s->pipe.enabled && !s->beams.empty() && vay_only && !wide_m1) return run_pipelined(s, nsteps, dt, mom_host, st);
    return run_sequential(s, nsteps, dt, mom_host, st);
}

namespace {
// where the adjoint's seed comes from: given values, or a function of the forward's moment sums
struct AdjSeed {
    const double* fixed = nullptr;
    qz_adjoint_seed_fn fn = nullptr;
    void* user = nullptr;
    // the seed (nb x 17) once the forward's moments (host, (nsteps+1, nb, 17)) are known
    void values(const double* mom, int nsteps, int nb, std::vector<double>& out) const {
        out.assign((size_t)17 * nb, 0.0);
        if (fixed) std::copy(fixed, fixed + 17 * (size_t)nb, out.begin());
        else fn(mom, nsteps, nb, out.data(), user);
    }
};

// The adjoint with both passes pipelined: the forward pipeline records the trajectories and the beams
// of every step (rings of one slot per step), the reverse pipeline runs the reverse sweeps of
// consecutive steps concurrently with the beam adjoint tasks (qz_adjoint.cu).
qz_status adjoint_pipelined(qz_sim* s, int nsteps, double dt, const AdjSeed& seed, double* const* lam_host,
                            double* mom_host, double* ms2, cudaStream_t st) {
    auto& P_ = s->pipe;
    const qzb::SweepArgs& base = s->sw->base;
    const int nb = (int)s->beams.size();
    const int K = s->p.K, M = s->g->M, T = nsteps;
    const size_t KM = (size_t)K * M;
    std::vector<size_t> off(nb + 1, 0);
    for (int b = 0; b < nb; ++b) off[b + 1] = off[b] + (size_t)s->beams[b].n;
    const size_t per = 7 * off[nb];
    // slice checkpointing: the plasma state of every C-th slice per step, C = ceil(sqrt(K)) by default
    const int every = s->ckpt_every > 0 ? std::min(s->ckpt_every, K) : (int)std::ceil(std::sqrt((double)K) - 1e-9);
    const int nck = (K + every - 1) / every;
    const size_t state = (6 + 5 * (size_t)base.ord) * base.npad;
    const size_t traj_slot = (size_t)nck * state;
    double *snap = nullptr, *traj = nullptr, *lam = nullptr, *lam2 = nullptr, *lfld = nullptr, *lbsrc = nullptr,
           *lamS = nullptr, *wrec = nullptr, *seg = nullptr;
    int* ints = nullptr;
    auto release = [&]() {
        for (void* q : {(void*)snap, (void*)traj, (void*)lam, (void*)lam2, (void*)lfld, (void*)lbsrc, (void*)lamS,
                        (void*)ints, (void*)wrec, (void*)seg})
            if (q) cudaFree(q);
    };
    if (cudaMalloc((void**)&snap, sizeof(double) * (per * (T + 1) + 1)) != cudaSuccess ||
        cudaMalloc((void**)&traj, sizeof(double) * traj_slot * (T + 1)) != cudaSuccess ||
        cudaMalloc((void**)&wrec, sizeof(double) * KM * (T + 1)) != cudaSuccess ||
        cudaMalloc((void**)&lam, sizeof(double) * (per + 1)) != cudaSuccess ||
        cudaMalloc((void**)&lam2, sizeof(double) * (per + 1)) != cudaSuccess ||
        cudaMalloc((void**)&lfld, sizeof(double) * KM * 6 * T) != cudaSuccess ||
        cudaMalloc((void**)&lbsrc, sizeof(double) * KM * 5 * T) != cudaSuccess ||
        cudaMalloc((void**)&lamS, sizeof(double) * 17 * (nb + 1)) != cudaSuccess) {
        cudaGetLastError();
        release();
        return fail(QZ_ERR_NOMEM, "qz_sim_adjoint: device allocation failed (records of every step)");
    }
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    auto pass = [&]() -> qz_status {
        for (auto& e : ev) QZ_CUDA(cudaEventCreate(&e));
        QZ_CUDA(cudaEventRecord(ev[0], st));
        // ---- forward with records
        FwdRecord rec;
        rec.traj = traj;
        rec.traj_slot = traj_slot;
        rec.traj_every = every;
        rec.wrec = wrec;
        rec.snap = snap;
        rec.snap_step = per;
        for (int b = 0; b < nb; ++b) rec.snap_off[b] = (long)(7 * off[b]);
        std::vector<double> momv(mom_host ? 0 : (size_t)(T + 1) * nb * 17);
        double* mom = mom_host ? mom_host : momv.data();
        if (qz_status e = run_pipelined(s, T, dt, mom, st, &rec)) return e;     // (synchronises)
        std::vector<double> seedv;
        seed.values(mom, T, nb, seedv);
        for (int b = 0; b < nb; ++b)                   // the beams after the last push
            QZ_CUDA(cudaMemcpyAsync(snap + per * T + 7 * off[b], s->beams[b].d, sizeof(double) * 7 * s->beams[b].n,
                                    cudaMemcpyDeviceToDevice, st));
        QZ_CUDA(cudaEventRecord(ev[1], st));
        // ---- reverse
        const int nbk = P_.info[4];
        const size_t nints = (size_t)(T + 1) * nbk * 2 + (size_t)T * nbk + T + nbk + (T + 1) + 2;
        QZ_CUDA(cudaMalloc((void**)&ints, sizeof(int) * (nints + 1)));
        int* cmin = ints;
        int* cmax = cmin + (size_t)(T + 1) * nbk;
        int* pmax = cmax + (size_t)(T + 1) * nbk;
        int* sync = pmax + (size_t)T * nbk;
        qzb::AdjPipeArgs A{};
        A.sw = base;
        A.sw.timing = nullptr;
        A.nsteps = T;
        A.fld = P_.fld;
        A.fld_slot = KM * 6;
        A.traj = traj;
        A.traj_slot = traj_slot;
        A.sw.traj_every = every;
        A.wrec = wrec;
        A.lfld = lfld;
        A.lfld_slot = KM * 6;
        A.lbsrc = lbsrc;
        A.lbsrc_slot = KM * 5;
        A.nbeams = nb;
        const qz_box box = sim_box(s);
        for (int q = 0; q < nb; ++q) {
            const qz_beam_view v = s->beams[q].view();
            A.beam[q] = beam_args(s->g, &v, &box);
            A.rigid[q] = s->beams[q].rigid;
            A.startup[q] = s->beams[q].rigid ? 0 : 1;
            A.snap_off[q] = (long)(7 * off[q]);
            A.lam_off[q] = (long)(7 * off[q]);
        }
        A.snap = snap;
        A.snap_step = per;
        A.lam = lam;
        A.dt = dt;
        A.nbk = nbk;
        A.bk_beam = P_.bk;
        A.bk_start = P_.bk + nbk;
        A.bk_end = P_.bk + 2 * nbk;
        A.cmin = cmin;
        A.pmax = pmax;
        A.prog = sync;
        A.bdone = sync + T;
        A.next = sync + T + nbk;
        A.err = A.next + (T + 1);
        A.lo = A.err + 1;
        A.timeout_ns = (unsigned long long)(P_.timeout_s * 1e9);
        QZ_CUDA(qzb::launch_bucket_cells(A, cmin, cmax, pmax, st));
        {
            std::vector<int> init((size_t)T + nbk + (T + 1) + 2, 0);
            for (int n = 0; n < T; ++n) init[n] = K;
            for (int b = 0; b < nbk; ++b) init[T + b] = T;
            QZ_CUDA(cudaMemcpyAsync(sync, init.data(), sizeof(int) * init.size(), cudaMemcpyHostToDevice, st));
            QZ_CUDA(cudaStreamSynchronize(st));          // init is a host temporary
        }
        QZ_CUDA(cudaMemsetAsync(lfld, 0, sizeof(double) * KM * 6 * T, st));
        QZ_CUDA(cudaMemsetAsync(lbsrc, 0, sizeof(double) * KM * 5 * T, st));
        QZ_CUDA(cudaMemsetAsync(lam, 0, sizeof(double) * per, st));
        QZ_CUDA(cudaMemcpyAsync(lamS, seedv.data(), sizeof(double) * 17 * nb, cudaMemcpyHostToDevice, st));
        for (int b = 0; b < nb; ++b) {
            qz_beam_view v = s->beams[b].view();
            double* d = snap + per * T + 7 * off[b];
            v.x = d; v.y = d + v.n; v.px = d + 2 * v.n; v.py = d + 3 * v.n; v.pz = d + 4 * v.n; v.xi = d + 5 * v.n;
            v.w = d + 6 * v.n;
            QZ_CUDA(qzb::launch_sums_back(beam_args(s->g, &v, &box), s->beams[b].gref, s->beams[b].xiref, lamS + 17 * b,
                                          lam + 7 * off[b], st));
        }
        int sms = 0;
        const int grid = qzb::adjoint_pipeline_max_grid(A, &sms);
        if (grid < 2) return fail(QZ_ERR_UNSUPPORTED, "qz_sim_adjoint: the reverse pipeline cannot be resident here");
        const int g1 = std::min(grid, sms);
        const int wmin = std::max(8, (2 * g1) / 5);
        A.nsweep = std::max(1, std::min(T, g1 - wmin));
        if (every > 1) {                               // one segment buffer per reverse-sweep CTA
            A.seg_slot = (size_t)every * state;
            if (cudaMalloc((void**)&seg, sizeof(double) * A.seg_slot * A.nsweep) != cudaSuccess) {
                cudaGetLastError();
                return fail(QZ_ERR_NOMEM, "qz_sim_adjoint: device allocation failed (checkpoint segments)");
            }
            A.seg = seg;
        }
        QZ_CUDA(qzb::launch_adjoint_pipeline(A, g1, st));
        int err = 0;
        QZ_CUDA(cudaMemcpyAsync(&err, A.err, sizeof(int), cudaMemcpyDeviceToHost, st));
        QZ_CUDA(cudaEventRecord(ev[2], st));
        // the caller's particle order
        for (int b = 0; b < nb; ++b) {
            const auto& B = s->beams[b];
            if (B.orig_identity)
                QZ_CUDA(cudaMemcpyAsync(lam2 + 7 * off[b], lam + 7 * off[b], sizeof(double) * 7 * B.n,
                                        cudaMemcpyDeviceToDevice, st));
            else
                QZ_CUDA(qzb::unpermute7(lam + 7 * off[b], lam2 + 7 * off[b], B.orig, B.n, st));
            QZ_CUDA(cudaMemcpyAsync(lam_host[b], lam2 + 7 * off[b], sizeof(double) * 7 * B.n, cudaMemcpyDeviceToHost,
                                    st));
        }
        QZ_CUDA(cudaStreamSynchronize(st));
        if (err) {
            static const char* site[] = {"?", "beam adjoint rows", "no beam adjoint task ready"};
            const int w = (err >> 8) & 0xff;
            return fail(QZ_ERR_CUDA, std::string("qz_sim_adjoint: reverse pipeline wait timed out (") +
                                         site[w <= 2 ? w : 0] + "); results of this call are invalid");
        }
        float t0 = 0, t1 = 0;
        QZ_CUDA(cudaEventElapsedTime(&t0, ev[0], ev[1]));
        QZ_CUDA(cudaEventElapsedTime(&t1, ev[1], ev[2]));
        if (ms2) { ms2[0] = t0; ms2[1] = t1; }
        return QZ_OK;
    };
    const qz_status status = pass();
    cudaStreamSynchronize(st);
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    release();
    s->bsrc_valid = false;
    return status;
}
}  // namespace

// The adjoint of a run (qz_adjoint.cu). Forward: step by step like run_sequential, keeping the
// beams of every step on the device. Reverse, for n = nsteps-1 .. 0: the beam deposit and the sweep
// of step n again (recording the plasma trajectory), the beam pushes in reverse (field-store
// adjoint), the sweep in reverse (beam-source adjoint), the beam deposits in reverse.
namespace {
qz_status sim_adjoint(qz_sim* s, int nsteps, double dt, const AdjSeed& seed, double* const* lam_host,
                      double* mom_host, double* ms2, void* stream) {
    if (!s || nsteps < 1 || !(dt > 0.0) || (!seed.fixed && !seed.fn) || (!s->beams.empty() && !lam_host))
        return fail(QZ_ERR_ARG, "qz_sim_adjoint: bad argument");
    const qzb::SweepArgs& base = s->sw->base;
    if (s->p.modes != 0 || s->p.K < 2 || base.max_cells > 0.0)
        return fail(QZ_ERR_UNSUPPORTED, "qz_sim_adjoint: built for modes = 0, K >= 2, without adaptive sub-slicing");
    if (base.M > qzb::kSweepThreads || base.np > qzb::kSweepThreads || base.nsp != 1)
        return fail(QZ_ERR_UNSUPPORTED, "qz_sim_adjoint: needs M <= 512, one mobile species, <= 512 plasma "
                                        "particles per slice");
    for (size_t b = 0; b < s->beams.size(); ++b) {
        if (s->beams[b].pusher != 0)
            return fail(QZ_ERR_UNSUPPORTED, "qz_sim_adjoint: built for the Vay pusher");
        if (s->beams[b].started)
            return fail(QZ_ERR_ARG, "qz_sim_adjoint: the beams were pushed already (the adjoint starts a run)");
        if (!lam_host[b]) return fail(QZ_ERR_ARG, "qz_sim_adjoint: null adjoint buffer");
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (s->pipe.enabled && s->beams.size() <= (size_t)qzb::kMaxBeams)
        return adjoint_pipelined(s, nsteps, dt, seed, lam_host, mom_host, ms2, st);
    void* sv = (void*)st;
    const int nb = (int)s->beams.size();
    for (auto& b : s->beams)                         // the caller's particle order
        if (!b.orig_identity) {
            QZ_CUDA(qzb::unpermute7(b.d, b.d2, b.orig, b.n, st));
            std::swap(b.d, b.d2);
            b.orig_identity = true;
        }
    std::vector<size_t> off(nb + 1, 0);
    for (int b = 0; b < nb; ++b) off[b + 1] = off[b] + (size_t)s->beams[b].n;
    const size_t per = 7 * off[nb];
    const int K = s->p.K, M = s->g->M;
    const size_t KM = (size_t)K * M;
    const size_t nv = 6 + 5 * (size_t)base.ord;
    double *snap = nullptr, *traj = nullptr, *lfld = nullptr, *lbsrc = nullptr, *lam = nullptr, *lamS = nullptr;
    auto release = [&]() {
        for (double* q : {snap, traj, lfld, lbsrc, lam, lamS})
            if (q) cudaFree(q);
    };
    std::vector<double> momv(mom_host ? 0 : (size_t)(nsteps + 1) * nb * 17);
    if (!mom_host) mom_host = momv.data();
    if (cudaMalloc((void**)&snap, sizeof(double) * (per * (nsteps + 1) + 1)) != cudaSuccess ||
        cudaMalloc((void**)&traj, sizeof(double) * (size_t)K * nv * base.npad) != cudaSuccess ||
        cudaMalloc((void**)&lfld, sizeof(double) * KM * 6) != cudaSuccess ||
        cudaMalloc((void**)&lbsrc, sizeof(double) * KM * 5) != cudaSuccess ||
        cudaMalloc((void**)&lam, sizeof(double) * (per + 1)) != cudaSuccess ||
        cudaMalloc((void**)&lamS, sizeof(double) * 17 * (nb + 1)) != cudaSuccess) {
        cudaGetLastError();
        release();
        return fail(QZ_ERR_NOMEM, "qz_sim_adjoint: device allocation failed (beams of every step, trajectory)");
    }
    const qz_box box = sim_box(s);
    double* bsrc = s->d_bsrc[0];
    auto view_at = [&](int b, double* base_ptr) {
        const auto& B = s->beams[b];
        qz_beam_view v = B.view();
        double* d = base_ptr + 7 * off[b];
        v.x = d; v.y = d + B.n; v.px = d + 2 * B.n; v.py = d + 3 * B.n; v.pz = d + 4 * B.n; v.xi = d + 5 * B.n;
        v.w = d + 6 * B.n;
        return v;
    };
    auto deposit_all = [&](double* beams_ptr) -> qz_status {
        QZ_CUDA(cudaMemsetAsync(bsrc, 0, sizeof(double) * KM * 5, st));
        for (int b = 0; b < nb; ++b) {
            const qz_beam_view v = view_at(b, beams_ptr);
            if (qz_status e = qz_beam_deposit(s->g, &v, &box, bsrc, sv)) return e;
        }
        return QZ_OK;
    };
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    // the whole pass; QZ_CUDA returns from it, the buffers are released below in every case
    auto pass = [&]() -> qz_status {
        qz_status status = QZ_OK;
        for (auto& e : ev) QZ_CUDA(cudaEventCreate(&e));
        QZ_CUDA(cudaEventRecord(ev[0], st));
        // ---- forward, keeping the beams of every step
        for (int n = 0; n <= nsteps && status == QZ_OK; ++n) {
            double* sn = snap + per * n;
            for (int b = 0; b < nb; ++b)
                QZ_CUDA(cudaMemcpyAsync(sn + 7 * off[b], s->beams[b].d, sizeof(double) * 7 * s->beams[b].n,
                                        cudaMemcpyDeviceToDevice, st));
            if ((status = deposit_all(sn))) break;
            if ((status = qz_sweep_run(s->sw, bsrc, s->d_fld, s->d_diag, nullptr, sv))) break;
            if (mom_host) {
                for (int b = 0; b < nb; ++b) {
                    const qz_beam_view v = s->beams[b].view();
                    if ((status = qz_beam_sums(&v, s->beams[b].gref, s->beams[b].xiref, s->d_mom + 17 * b, sv))) break;
                }
                if (status) return status;
                QZ_CUDA(cudaMemcpyAsync(mom_host + (size_t)n * nb * 17, s->d_mom, sizeof(double) * 17 * nb,
                                        cudaMemcpyDeviceToHost, st));
            }
            if (n < nsteps)
                for (int b = 0; b < nb && status == QZ_OK; ++b) {
                    auto& B = s->beams[b];
                    if (B.rigid) continue;
                    qz_beam_view v = B.view();
                    status = qz_beam_push(s->g, &v, &box, s->d_fld, dt, dt, &B.started, sv);
                }
        }
        if (status) return status;
        QZ_CUDA(cudaEventRecord(ev[1], st));
        // ---- seed: the last step's moment sums
        QZ_CUDA(cudaMemsetAsync(lam, 0, sizeof(double) * per, st));
        QZ_CUDA(cudaStreamSynchronize(st));              // the moments are on the host
        std::vector<double> seedv;
        seed.values(mom_host, nsteps, nb, seedv);
        QZ_CUDA(cudaMemcpyAsync(lamS, seedv.data(), sizeof(double) * 17 * nb, cudaMemcpyHostToDevice, st));
        for (int b = 0; b < nb; ++b) {
            const qz_beam_view v = view_at(b, snap + per * nsteps);
            const qzb::BeamArgs BA = beam_args(s->g, &v, &box);
            QZ_CUDA(qzb::launch_sums_back(BA, s->beams[b].gref, s->beams[b].xiref, lamS + 17 * b, lam + 7 * off[b], st));
        }
        // ---- reverse
        qzb::SweepArgs A = base;
        if (s->sw->timing) A.timing = s->sw->d_tim;     // phase cycles (qz_sim_timing)
        A.traj = traj;
        A.bsrc = bsrc;
        A.fld = s->d_fld;
        A.diag = s->d_diag;
        for (int n = nsteps - 1; n >= 0 && status == QZ_OK; --n) {
            double* sn = snap + per * n;
            if ((status = deposit_all(sn))) break;
            QZ_CUDA(qzb::launch_sweep_m0(A, st));
            QZ_CUDA(cudaMemsetAsync(lfld, 0, sizeof(double) * KM * 6, st));
            for (int b = 0; b < nb; ++b) {
                if (s->beams[b].rigid) continue;
                const qz_beam_view v = view_at(b, sn);
                QZ_CUDA(qzb::launch_push_back(beam_args(s->g, &v, &box), s->d_fld, lam + 7 * off[b], lfld, dt, dt,
                                              n == 0 ? 1 : 0, st));
            }
            QZ_CUDA(cudaMemsetAsync(lbsrc, 0, sizeof(double) * KM * 5, st));
            QZ_CUDA(qzb::launch_sweep_back(A, traj, s->d_fld, lfld, lbsrc, st));
            for (int b = 0; b < nb; ++b) {
                const qz_beam_view v = view_at(b, sn);
                QZ_CUDA(qzb::launch_deposit_back(beam_args(s->g, &v, &box), lbsrc, lam + 7 * off[b], st));
            }
        }
        if (status) return status;
        QZ_CUDA(cudaEventRecord(ev[2], st));
        for (int b = 0; b < nb; ++b)
            QZ_CUDA(cudaMemcpyAsync(lam_host[b], lam + 7 * off[b], sizeof(double) * 7 * s->beams[b].n,
                                    cudaMemcpyDeviceToHost, st));
        // leave the fields of the last step, as qz_sim_run does
        if ((status = deposit_all(snap + per * nsteps))) return status;
        A.traj = nullptr;
        A.timing = nullptr;
        QZ_CUDA(qzb::launch_sweep_m0(A, st));
        QZ_CUDA(cudaStreamSynchronize(st));
        float t0 = 0, t1 = 0;
        QZ_CUDA(cudaEventElapsedTime(&t0, ev[0], ev[1]));
        QZ_CUDA(cudaEventElapsedTime(&t1, ev[1], ev[2]));
        if (ms2) { ms2[0] = t0; ms2[1] = t1; }
        return QZ_OK;
    };
    const qz_status status = pass();
    cudaStreamSynchronize(st);
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    release();
    s->bsrc_valid = false;
    return status;
}

}  // namespace

extern "C" qz_status qz_sim_adjoint(qz_sim* s, int nsteps, double dt, const double* lamS_host, double* const* lam_host,
                                    double* mom_host, double* ms2, void* stream) {
    AdjSeed seed;
    seed.fixed = lamS_host;
    return sim_adjoint(s, nsteps, dt, seed, lam_host, mom_host, ms2, stream);
}

extern "C" qz_status qz_sim_adjoint_fn(qz_sim* s, int nsteps, double dt, qz_adjoint_seed_fn fn, void* user,
                                       double* const* lam_host, double* mom_host, double* ms2, void* stream) {
    AdjSeed seed;
    seed.fn = fn;
    seed.user = user;
    return sim_adjoint(s, nsteps, dt, seed, lam_host, mom_host, ms2, stream);
}

extern "C" qz_status qz_sim_timing(qz_sim* s, int enable, unsigned long long* cycles16) {
    if (!s) return fail(QZ_ERR_ARG, "qz_sim_timing: null pointer");
    return qz_sweep_timing(s->sw, enable, cycles16);
}

extern "C" qz_status qz_sim_restart(qz_sim* s) {
    if (!s) return fail(QZ_ERR_ARG, "qz_sim_restart: null pointer");
    for (auto& b : s->beams) b.started = 0;
    s->bsrc_valid = false;
    return QZ_OK;
}

extern "C" qz_status qz_sim_set_adjoint_checkpoint(qz_sim* s, int every) {
    if (!s || every < 0) return fail(QZ_ERR_ARG, "qz_sim_set_adjoint_checkpoint: bad argument");
    s->ckpt_every = every;
    return QZ_OK;
}

extern "C" qz_status qz_fx_create(const qz_grid* g, double dxi, double wq, int64_t nparticles, qz_fx** out) {
    if (!g || !out || !(dxi > 0.0) || !(wq >= 0.0) || nparticles < 0) return fail(QZ_ERR_ARG, "qz_fx_create: bad argument");
    auto* f = new (std::nothrow) qz_fx;
    if (!f) return fail(QZ_ERR_NOMEM, "qz_fx_create: out of host memory");
    f->M = g->M;
    if (!fx_quanta(g, dxi, wq, (long)nparticles, f->qe, f->S)) {
        delete f;
        return fail(QZ_ERR_UNSUPPORTED, "qz_fx_create: exact deposits take at most 2^25 beam particles");
    }
    if (cudaMalloc((void**)&f->d_q, sizeof(double) * 2 * g->M) != cudaSuccess) {
        cudaGetLastError();
        f->d_q = nullptr;
        delete f;
        return fail(QZ_ERR_NOMEM, "qz_fx_create: device allocation failed");
    }
    if (qz_status e = fx_upload(f->qe, f->d_q)) { delete f; return e; }
    *out = f;
    return QZ_OK;
}

extern "C" qz_status qz_fx_destroy(qz_fx* f) {
    delete f;
    return QZ_OK;
}

extern "C" qz_status qz_beam_deposit_fx(const qz_grid* g, const qz_beam_view* b, const qz_box* box, const qz_fx* fx,
                                        double* bsrc2, void* stream) {
    if (qz_status st = check_beam(g, b, box)) return st;
    if (!fx || !bsrc2) return fail(QZ_ERR_ARG, "qz_beam_deposit_fx: null pointer");
    if (box->modes != 0 || fx->M != g->M) return fail(QZ_ERR_ARG, "qz_beam_deposit_fx: modes = 0 and the grid of fx");
    qzb::BeamArgs B = beam_args(g, b, box);
    B.fx_scale = fx->d_q;
    B.fx_inv2s = std::ldexp(1.0, -fx->S);
    B.fx_2s = std::ldexp(1.0, fx->S);
    B.fx_lo = (long)box->K * g->M * qzb::B_NC0;
    QZ_CUDA(qzb::launch_beam_deposit(B, bsrc2, (cudaStream_t)stream));
    return QZ_OK;
}

extern "C" qz_status qz_sweep_set_exact_sources(qz_sweep* s, const qz_fx* fx) {
    if (!s) return fail(QZ_ERR_ARG, "qz_sweep_set_exact_sources: null pointer");
    if (fx && (s->p.modes != 0 || fx->M != s->g->M))
        return fail(QZ_ERR_ARG, "qz_sweep_set_exact_sources: modes = 0 and the grid of fx");
    s->fx = fx;
    return QZ_OK;
}

extern "C" qz_status qz_sim_set_exact(qz_sim* s, int exact) {
    if (!s) return fail(QZ_ERR_ARG, "qz_sim_set_exact: null pointer");
    s->fx.wanted = exact != 0;
    return QZ_OK;
}

extern "C" qz_status qz_sim_set_schedule(qz_sim* s, int pipelined, int sweep_ctas, int bucket, int span,
                                         double timeout_s) {
    if (!s || sweep_ctas < 0 || bucket < 0 || span < 0 || timeout_s < 0)
        return fail(QZ_ERR_ARG, "qz_sim_set_schedule: bad argument");
    if (pipelined && s->beams.size() > (size_t)qzb::kMaxBeams)
        return fail(QZ_ERR_UNSUPPORTED, "qz_sim_set_schedule: the pipelined run handles at most 4 beams");
    s->pipe.enabled = pipelined ? 1 : 0;
    s->pipe.sweep_ctas = sweep_ctas;
    s->pipe.bucket = bucket > 0 ? bucket : 512;
    s->pipe.span = span > 0 ? span : 1;
    if (timeout_s > 0) s->pipe.timeout_s = timeout_s;
    return QZ_OK;
}

extern "C" qz_status qz_sim_schedule(qz_sim* s, int* info8) {
    if (!s || !info8) return fail(QZ_ERR_ARG, "qz_sim_schedule: null pointer");
    std::copy(s->pipe.info, s->pipe.info + 8, info8);
    return QZ_OK;
}

extern "C" qz_status qz_sim_times(qz_sim* s, double* ms3) {
    if (!s || !ms3) return fail(QZ_ERR_ARG, "qz_sim_times: null pointer");
    for (int i = 0; i < 3; ++i) ms3[i] = s->pipe.times[i];
    return QZ_OK;
}

extern "C" qz_status qz_sim_set_beam(qz_sim* s, int b, const double* cols7, int on_device, void* stream) {
    if (!s || !cols7 || b < 0 || b >= (int)s->beams.size()) return fail(QZ_ERR_ARG, "qz_sim_set_beam: bad argument");
    auto& B = s->beams[b];
    QZ_CUDA(cudaMemcpyAsync(B.d, cols7, sizeof(double) * 7 * B.n,
                            on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, (cudaStream_t)stream));
    B.orig_identity = true;
    s->bsrc_valid = false;
    return QZ_OK;
}

extern "C" qz_status qz_sim_trace(qz_sim* s, int enable, unsigned long long* out, int cap, int* n) {
    if (!s || cap < 0 || (cap > 0 && !out)) return fail(QZ_ERR_ARG, "qz_sim_trace: bad argument");
    const int have = (int)s->pipe.h_trace.size();
    if (n) *n = have;
    for (int i = 0; i < std::min(cap, have); ++i) out[i] = s->pipe.h_trace[i];
    s->pipe.trace = enable ? 1 : 0;
    return QZ_OK;
}

extern "C" qz_status qz_sim_run_host(qz_sim* s, int nsteps, double dt, double* const* cols, double* mom_host,
                                     void* stream) {
    if (!s || nsteps < 0 || (!s->beams.empty() && !cols)) return fail(QZ_ERR_ARG, "qz_sim_run_host: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    for (auto& b : s->beams) {
        const size_t i = &b - s->beams.data();
        if (!cols[i]) return fail(QZ_ERR_ARG, "qz_sim_run_host: null beam buffer");
        QZ_CUDA(cudaMemcpyAsync(b.d, cols[i], sizeof(double) * 7 * b.n, cudaMemcpyHostToDevice, st));
        b.orig_identity = true;
    }
    s->bsrc_valid = false;
    if (qz_status e = qz_sim_run(s, nsteps, dt, mom_host, stream)) return e;
    for (auto& b : s->beams) {
        const size_t i = &b - s->beams.data();
        if (!b.orig_identity) {
            QZ_CUDA(qzb::unpermute7(b.d, b.d2, b.orig, b.n, st));
            std::swap(b.d, b.d2);
            b.orig_identity = true;
        }
        QZ_CUDA(cudaMemcpyAsync(cols[i], b.d, sizeof(double) * 7 * b.n, cudaMemcpyDeviceToHost, st));
    }
    QZ_CUDA(cudaStreamSynchronize(st));
    return QZ_OK;
}

extern "C" qz_status qz_sim_fields(qz_sim* s, double* fld, double* diag) {
    if (!s) return fail(QZ_ERR_ARG, "qz_sim_fields: null pointer");
    const size_t KM = (size_t)s->p.K * s->g->M;
    if (fld) QZ_CUDA(cudaMemcpy(fld, s->d_fld, sizeof(double) * KM * s->fnc, cudaMemcpyDeviceToHost));
    if (diag) QZ_CUDA(cudaMemcpy(diag, s->d_diag, sizeof(double) * KM * s->dnc, cudaMemcpyDeviceToHost));
    return QZ_OK;
}

// ===================================================================== field files
namespace {

// Simulation::field_table / write_fields (src/Simulation.cpp:878-993) for this path: no ion, laser or
// output-group columns, every slice and node. Layout (version 3): int32 {3, M, K, mode1}, float64 t,
// float64 r[M], float64 xi[K] (user xi, increasing: slice k is row K-1-k), int32 ncomp, then per component
// char name[16] and float64 data[K][M].
qz_status write_fields_host(const char* path, const double* nodes, int M, const qz_box* box, double t,
                            const double* F, const double* D, const double* B) {
    const int K = box->K, m1 = box->modes == 1;
    const int fnc = m1 ? 18 : 6, dnc = m1 ? 9 : 3, bnc = m1 ? 15 : 5;
    // every written component is s0 * a[kj * na + ca] + s1 * b[kj * nb + cb] of the stored arrays (one
    // or two columns), copied by a plain strided loop
    struct Col { const double* p; int n, c; double s; };
    struct Comp { std::string name; Col a, b; };
    std::vector<Comp> comps;
    const Col none{nullptr, 1, 0, 0.0};
    auto f = [&](int c, double sc = 1.0) { return Col{F, fnc, c, sc}; };
    auto d = [&](int c, double sc = 1.0) { return Col{D, dnc, c, sc}; };
    auto b = [&](int c, double sc = 1.0) { return Col{B, bnc, c, sc}; };     // B == nullptr: zero
    using namespace qzb;
    comps.push_back({"psi", d(D_PSI0), none});
    comps.push_back({"ez", f(F_EZ0), none});
    comps.push_back({"er", f(F_EP1R), none});
    comps.push_back({"eth", f(F_EP1I), none});
    comps.push_back({"br", f(F_BP1R), none});
    comps.push_back({"bth", f(F_BP1I), none});
    comps.push_back({"bz", f(F_BZ0), none});
    comps.push_back({"ne", d(D_NE0), none});
    comps.push_back({"ni", d(D_NI0), none});
    comps.push_back({"rhob", b(B_RHO0), none});
    if (m1) {   // f = f0 + 2 Re[f1 e^{i th}]: f_c = 2 Re f1, f_s = -2 Im f1; vectors from the V+ modes 0 and 2
        const std::pair<const char*, std::pair<Col, Col>> sc[] = {
            {"psi", {d(D_PSI1R), d(D_PSI1I)}}, {"ez", {f(F_EZ1R), f(F_EZ1I)}}, {"bz", {f(F_BZ1R), f(F_BZ1I)}},
            {"ne", {d(D_NE1R), d(D_NE1I)}}, {"ni", {d(D_NI1R), d(D_NI1I)}}, {"rhob", {b(B_RHO1R), b(B_RHO1I)}}};
        for (const auto& e : sc) {
            Col re = e.second.first, im = e.second.second;
            re.s = 2.0;
            im.s = -2.0;
            comps.push_back({std::string(e.first) + "_c", re, none});
            comps.push_back({std::string(e.first) + "_s", im, none});
        }
        const int vr[2][4] = {{F_EP0R, F_EP0I, F_EP2R, F_EP2I}, {F_BP0R, F_BP0I, F_BP2R, F_BP2I}};
        const char* nm[2][2] = {{"er", "eth"}, {"br", "bth"}};
        for (int v = 0; v < 2; ++v) {
            comps.push_back({std::string(nm[v][0]) + "_c", f(vr[v][0]), f(vr[v][2])});
            comps.push_back({std::string(nm[v][0]) + "_s", f(vr[v][1]), f(vr[v][3], -1.0)});
            comps.push_back({std::string(nm[v][1]) + "_c", f(vr[v][1]), f(vr[v][3])});
            comps.push_back({std::string(nm[v][1]) + "_s", f(vr[v][2]), f(vr[v][0], -1.0)});
        }
    }
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(QZ_ERR_ARG, std::string("qz_write_fields: cannot open ") + path);
    const int32_t hdr[4] = {3, M, K, m1};
    bool ok = std::fwrite(hdr, sizeof(hdr), 1, fp) == 1 && std::fwrite(&t, 8, 1, fp) == 1 &&
              std::fwrite(nodes, 8, (size_t)M, fp) == (size_t)M;
    std::vector<double> xi(K);
    for (int k = 0; k < K; ++k) xi[k] = 0.0 - (box->xi_min + (K - 1 - k) * box->dxi);
    const int32_t nc = (int32_t)comps.size();
    ok = ok && std::fwrite(xi.data(), 8, (size_t)K, fp) == (size_t)K && std::fwrite(&nc, 4, 1, fp) == 1;
    std::vector<double> v((size_t)K * M);
    for (const auto& c : comps) {
        char name[16] = {0};
        std::strncpy(name, c.name.c_str(), 15);
        for (int k = 0; k < K; ++k) {
            double* row = v.data() + (size_t)(K - 1 - k) * M;             // file rows: the box head last
            const size_t kj0 = (size_t)k * M;
            if (!c.a.p) {
                std::fill(row, row + M, 0.0);
            } else if (!c.b.p) {
                for (int j = 0; j < M; ++j) row[j] = c.a.s * c.a.p[(kj0 + j) * c.a.n + c.a.c];
            } else {
                for (int j = 0; j < M; ++j)
                    row[j] = c.a.s * c.a.p[(kj0 + j) * c.a.n + c.a.c] + c.b.s * c.b.p[(kj0 + j) * c.b.n + c.b.c];
            }
        }
        ok = ok && std::fwrite(name, 16, 1, fp) == 1 && std::fwrite(v.data(), 8, v.size(), fp) == v.size();
    }
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? QZ_OK : fail(QZ_ERR_ARG, std::string("qz_write_fields: write failed: ") + path);
}

}  // namespace

extern "C" qz_status qz_write_fields(const char* path, const double* nodes, int M, const qz_box* box, double t,
                                     const double* fld, const double* diag, const double* bsrc, int on_device) {
    if (!path || !nodes || !box || !fld || !diag) return fail(QZ_ERR_ARG, "qz_write_fields: null pointer");
    if ((box->modes != 0 && box->modes != 1) || box->K < 1 || M < 2) return fail(QZ_ERR_ARG, "qz_write_fields: bad size");
    if (!on_device) return write_fields_host(path, nodes, M, box, t, fld, diag, bsrc);
    const size_t KM = (size_t)box->K * M;
    const int m1 = box->modes == 1;
    std::vector<double> F(KM * (m1 ? 18 : 6)), D(KM * (m1 ? 9 : 3)), B(bsrc ? KM * (m1 ? 15 : 5) : 0);
    QZ_CUDA(cudaMemcpy(F.data(), fld, sizeof(double) * F.size(), cudaMemcpyDeviceToHost));
    QZ_CUDA(cudaMemcpy(D.data(), diag, sizeof(double) * D.size(), cudaMemcpyDeviceToHost));
    if (bsrc) QZ_CUDA(cudaMemcpy(B.data(), bsrc, sizeof(double) * B.size(), cudaMemcpyDeviceToHost));
    return write_fields_host(path, nodes, M, box, t, F.data(), D.data(), bsrc ? B.data() : nullptr);
}

extern "C" qz_status qz_sim_write_fields(qz_sim* s, double t, const char* path) {
    if (!s || !path) return fail(QZ_ERR_ARG, "qz_sim_write_fields: null pointer");
    const qz_box box = sim_box(s);
    const size_t nb = (size_t)s->p.K * s->g->M * s->bnc;
    double* d = nullptr;
    if (cudaMalloc((void**)&d, sizeof(double) * nb) != cudaSuccess)
        return fail(QZ_ERR_NOMEM, "qz_sim_write_fields: device allocation failed");
    // the beam sources of the last sweep: the beams as they stand (not pushed after it) and the static ones
    qz_status st = QZ_OK;
    if (s->d_bstat) {
        if (cudaMemcpy(d, s->d_bstat, sizeof(double) * nb, cudaMemcpyDeviceToDevice) != cudaSuccess)
            st = fail(QZ_ERR_CUDA, "qz_sim_write_fields: copy failed");
    } else if (cudaMemset(d, 0, sizeof(double) * nb) != cudaSuccess) {
        st = fail(QZ_ERR_CUDA, "qz_sim_write_fields: memset failed");
    }
    for (size_t b = 0; st == QZ_OK && b < s->beams.size(); ++b) {
        const qz_beam_view v = s->beams[b].view();
        st = qz_beam_deposit(s->g, &v, &box, d, nullptr);
    }
    if (st == QZ_OK) st = qz_write_fields(path, s->g->r.data(), s->g->M, &box, t, s->d_fld, s->d_diag, d, 1);
    cudaFree(d);
    return st;
}

extern "C" qz_status qz_sim_beam(qz_sim* s, int b, double* p7) {
    if (!s || !p7 || b < 0 || b >= (int)s->beams.size()) return fail(QZ_ERR_ARG, "qz_sim_beam: bad argument");
    const auto& B = s->beams[b];
    std::vector<double> cols((size_t)7 * B.n);
    std::vector<int> orig(B.orig_identity ? 0 : (size_t)B.n);
    if (B.n > 0) QZ_CUDA(cudaMemcpy(cols.data(), B.d, sizeof(double) * cols.size(), cudaMemcpyDeviceToHost));
    if (!orig.empty()) QZ_CUDA(cudaMemcpy(orig.data(), B.orig, sizeof(int) * orig.size(), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < B.n; ++i) {
        const int64_t o = orig.empty() ? i : orig[i];     // the caller's index of this particle
        for (int c = 0; c < 7; ++c) p7[7 * o + c] = cols[(size_t)c * B.n + i];
    }
    return QZ_OK;
}

extern "C" qz_status qz_sim_counters(qz_sim* s, qz_counters* out) {
    if (!s || !out) return fail(QZ_ERR_ARG, "qz_sim_counters: null pointer");
    *out = s->cnt;
    return QZ_OK;
}

extern "C" qz_status qz_sim_step_host(qz_sim* s, double* const* cols, double dt_kick, double dt_drift, int push,
                                      double* mom_host, void* stream) {
    if (!s || (!s->beams.empty() && !cols)) return fail(QZ_ERR_ARG, "qz_sim_step_host: null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    const qz_box box = sim_box(s);
    const int nb = (int)s->beams.size();
    for (int b = 0; b < nb; ++b) {
        if (!cols[b]) return fail(QZ_ERR_ARG, "qz_sim_step_host: null beam buffer");
        QZ_CUDA(cudaMemcpyAsync(s->beams[b].d, cols[b], sizeof(double) * 7 * s->beams[b].n, cudaMemcpyHostToDevice,
                                st));
        s->beams[b].orig_identity = true;
    }
    if (qz_status e = fx_prepare(s, st)) return e;
    QZ_CUDA(cudaMemsetAsync(s->sw->d_cnt, 0, sizeof(unsigned long long) * 4, st));
    if (qz_status e = sim_deposit_all(s, s->d_bsrc[s->cur], st)) return e;
    if (qz_status e = sim_sweep(s, s->d_bsrc[s->cur], st)) return e;
    for (int b = 0; b < nb; ++b) {
        const qz_beam_view v = s->beams[b].view();
        if (qz_status e = qz_beam_sums(&v, s->beams[b].gref, s->beams[b].xiref, s->d_mom + 17 * b, stream)) return e;
    }
    if (push)
        for (auto& b : s->beams) {
            if (b.rigid) continue;
            qz_beam_view v = b.view();
            if (qz_status e = qz_beam_push(s->g, &v, &box, s->d_fld, dt_kick, dt_drift, &b.started, stream)) return e;
        }
    for (int b = 0; b < nb; ++b)
        QZ_CUDA(cudaMemcpyAsync(cols[b], s->beams[b].d, sizeof(double) * 7 * s->beams[b].n, cudaMemcpyDeviceToHost,
                                st));
    if (mom_host && nb > 0)
        QZ_CUDA(cudaMemcpyAsync(mom_host, s->d_mom, sizeof(double) * 17 * nb, cudaMemcpyDeviceToHost, st));
    QZ_CUDA(cudaStreamSynchronize(st));
    s->bsrc_valid = false;
    return QZ_OK;
}

// ===================================================================== batched independent runs
// A parameter scan: many small runs, each with its own grid, box, plasma and beams, in one persistent
// launch (qz_batch.cu). No counterpart in the reference, which runs one deck per process.
struct qz_batch {
    struct Inst {
        qz_grid* g = nullptr;
        qz_sweep* sw = nullptr;
        std::vector<double*> beam_d;       // 7 columns of n per beam
        std::vector<int64_t> beam_n;
        qzb::BatchInst dev{};
        double cost = 0;
        ~Inst() {
            for (double* d : beam_d)
                if (d) cudaFree(d);
            qz_sweep_destroy(sw);
            qz_grid_destroy(g);
        }
    };
    std::vector<Inst*> inst;
    int ord = 0;
    qzb::BatchInst* d_inst = nullptr;
    int* d_order = nullptr;
    int* d_next = nullptr;
    double *d_fld = nullptr, *d_diag = nullptr, *d_bsrc = nullptr, *d_mom = nullptr;
    size_t fld_alloc = 0, diag_alloc = 0, bsrc_alloc = 0, mom_alloc = 0;   // doubles
    float last_ms = 0;
    int last_grid = 0;
    bool trace = false;                          // qz_batch_set_trace
    unsigned long long* d_trace = nullptr;
    size_t trace_n = 0;
    std::vector<unsigned long long> h_trace;     // the last traced run, kBatchTrace words per instance
    ~qz_batch() {
        for (Inst* i : inst) delete i;
        for (void* q : {(void*)d_inst, (void*)d_order, (void*)d_next, (void*)d_fld, (void*)d_diag, (void*)d_bsrc,
                        (void*)d_mom, (void*)d_trace})
            if (q) cudaFree(q);
    }
};

extern "C" qz_status qz_batch_create(qz_batch** out) {
    if (!out) return fail(QZ_ERR_ARG, "qz_batch_create: null pointer");
    *out = new (std::nothrow) qz_batch;
    return *out ? QZ_OK : fail(QZ_ERR_NOMEM, "qz_batch_create: out of host memory");
}

extern "C" qz_status qz_batch_destroy(qz_batch* b) {
    delete b;
    return QZ_OK;
}

extern "C" qz_status qz_batch_add(qz_batch* b, const double* nodes, int M, const qz_sweep_params* p, int nbeams,
                                  const double* const* p7_host, const int64_t* n, const double* q, const double* m,
                                  const int* rigid, const double* gref, const double* xiref, int* index) {
    if (!b || !nodes || !p || nbeams < 0 || nbeams > qzb::kBatchBeams || (nbeams > 0 && (!p7_host || !n || !q ||
        !m || !rigid || !gref || !xiref)))
        return fail(QZ_ERR_ARG, "qz_batch_add: bad argument (at most 2 beams per instance)");
    if (p->modes != 0 && p->modes != 1) return fail(QZ_ERR_ARG, "qz_batch_add: modes must be 0 or 1");
    if (p->modes == 1 && M > 2 * qzb::kSweepThreads)
        return fail(QZ_ERR_SIZE, "qz_batch_add: modes = 1 instances need M <= 1024 (one radial row per thread)");
    if (b->ord && p->ab_order != b->ord) return fail(QZ_ERR_ARG, "qz_batch_add: every instance needs the same AB order");
    auto* I = new (std::nothrow) qz_batch::Inst;
    if (!I) return fail(QZ_ERR_NOMEM, "qz_batch_add: out of host memory");
    if (qz_status st = qz_grid_create(nodes, M, &I->g)) { delete I; return st; }
    if (qz_status st = qz_sweep_create(I->g, p, &I->sw)) { delete I; return st; }
    qzb::BatchInst& D = I->dev;
    D.sw = I->sw->base;
    {
        // the batch kernel holds the instance record and a reduction scratch in static shared memory:
        // the sweep's layout must leave room for them
        int dev = 0, optin = 0;
        QZ_CUDA(cudaGetDevice(&dev));
        QZ_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        const size_t reserve = sizeof(qzb::BatchInst) + sizeof(double) * 17 * (qzb::kSweepThreads / 32) + 256;
        if (p->modes == 1) {
            const bool wide = M > qzb::kSweepThreads;     // the 1024-thread batch kernel (qz_batch_m1w.cu)
            if ((wide ? qzb::sweep_m1w_smem_bytes(M) + qzb::batch_m1w_static_bytes()
                      : qzb::sweep_m1_smem_bytes(M) + reserve) > (size_t)optin) {
                delete I;
                return fail(QZ_ERR_SIZE, "qz_batch_add: M too large for the batched sweep");
            }
        } else {
            static const bool kLay[4][2] = {{true, true}, {false, true}, {true, false}, {false, false}};
            const bool filt = p->smooth_length > 0;
            int lay = -1, pc = 0;
            // with plasma in global memory, the fastest layout that also holds the particle copy, if any
            if (D.sw.np > qzb::kSweepThreads)
                for (int l = 0; l < 4 && lay < 0; ++l)
                    if (qzb::sweep_m0_smem_bytes(M, kLay[l][0], kLay[l][1], filt, D.sw.np) + reserve <= (size_t)optin) {
                        lay = l;
                        pc = D.sw.np;
                    }
            for (int l = 0; l < 4 && lay < 0; ++l)
                if (qzb::sweep_m0_smem_bytes(M, kLay[l][0], kLay[l][1], filt) + reserve <= (size_t)optin) lay = l;
            if (lay < 0) { delete I; return fail(QZ_ERR_SIZE, "qz_batch_add: M too large for the batched sweep"); }
            D.sw.dbuf = kLay[lay][0];
            D.sw.const_smem = kLay[lay][1];
            D.sw.pcache = pc;
        }
    }
    D.modes = p->modes;
    D.nbeams = nbeams;
    qz_box box;
    box.xi_min = p->xi_min; box.dxi = p->dxi; box.K = p->K; box.ngp = p->ngp; box.modes = p->modes;
    long ntot = 0;
    for (int k = 0; k < nbeams; ++k) {
        if (n[k] < 0 || (n[k] > 0 && !p7_host[k])) { delete I; return fail(QZ_ERR_ARG, "qz_batch_add: bad beam"); }
        std::vector<double> cols((size_t)7 * (n[k] > 0 ? n[k] : 1), 0.0);
        for (int64_t i = 0; i < n[k]; ++i)
            for (int c = 0; c < 7; ++c) cols[(size_t)c * n[k] + i] = p7_host[k][7 * i + c];
        double* d = nullptr;
        if (qz_status st = dev_upload(&d, cols)) { delete I; return st; }
        I->beam_d.push_back(d);
        I->beam_n.push_back(n[k]);
        qz_beam_view v;
        v.x = d; v.y = d + n[k]; v.px = d + 2 * n[k]; v.py = d + 3 * n[k]; v.pz = d + 4 * n[k];
        v.xi = d + 5 * n[k]; v.w = d + 6 * n[k]; v.n = n[k]; v.q = q[k]; v.m = m[k];
        v.pusher = 0;                                   // the batched runs push with Vay
        D.beam[k] = beam_args(I->g, &v, &box);
        D.rigid[k] = rigid[k];
        D.gref[k] = gref[k];
        D.xiref[k] = xiref[k];
        ntot += n[k];
    }
    // cost estimate (queue order): the sweeps plus the beam work
    // (the m = 1 slice costs about 7x the m = 0 one at the same M and particles)
    I->cost = (p->modes ? 7.0 : 1.0) * (double)p->K * (M + 4.0 * I->sw->np) + 2.0 * ntot * (p->modes ? 3.0 : 1.0);
    b->ord = p->ab_order;
    b->inst.push_back(I);
    if (index) *index = (int)b->inst.size() - 1;
    return QZ_OK;
}

extern "C" qz_status qz_batch_run(qz_batch* b, int nsteps, double dt, double* mom_host, void* stream) {
    if (!b || nsteps < 0 || !(dt > 0)) return fail(QZ_ERR_ARG, "qz_batch_run: bad argument");
    const int ni = (int)b->inst.size();
    if (ni == 0) return QZ_OK;
    cudaStream_t st = (cudaStream_t)stream;
    // two groups: the 512-thread batch kernel takes every m = 0 instance and the m = 1 ones with up to 512
    // nodes; m = 1 instances with more nodes (wide) run after it in the 1024-thread kernel (qz_batch_m1w.cu).
    // Per group the slot sizes and shared memory of its largest instance; the two launches run one after
    // the other on the stream and share the slot buffers.
    struct Group {
        size_t fmax = 0, dmax = 0, bmax = 0, smem = 0;
        bool with_m1 = false, with_ext = false;
        int n = 0, grid = 0;
    } gr[2];
    size_t mom_total = 0;
    std::vector<size_t> mom_off(ni);
    std::vector<int> grp(ni);
    for (int i = 0; i < ni; ++i) {
        const auto& A = b->inst[i]->dev.sw;
        const bool m1 = b->inst[i]->dev.modes == 1;
        grp[i] = (m1 && A.M > qzb::kSweepThreads) ? 1 : 0;
        Group& G = gr[grp[i]];
        ++G.n;
        G.with_m1 = G.with_m1 || m1;
        G.with_ext = G.with_ext || A.filter;
        const size_t km = (size_t)A.K * A.M;
        G.fmax = std::max(G.fmax, km * (m1 ? 18 : 6));        // fld (K, M, 18 / 6)
        G.dmax = std::max(G.dmax, km * (m1 ? 9 : 3));         // diag (K, M, 9 / 3)
        G.bmax = std::max(G.bmax, km * (m1 ? 15 : 5));        // bsrc (K, M, 15 / 5)
        G.smem = std::max(G.smem, grp[i] ? qzb::sweep_m1w_smem_bytes(A.M)
                                  : m1 ? qzb::sweep_m1_smem_bytes(A.M)
                                       : qzb::sweep_m0_smem_bytes(A.M, A.dbuf, A.const_smem, A.filter != 0, A.pcache));
        mom_off[i] = mom_total;
        mom_total += (size_t)(nsteps + 1) * std::max(1, b->inst[i]->dev.nbeams) * 17;
    }
    int sms = 0;
    if (gr[0].n) {
        gr[0].grid = std::min(qzb::batch_max_grid(b->ord, gr[0].with_m1, gr[0].with_ext, gr[0].smem, &sms), gr[0].n);
        if (gr[0].grid < 1) return fail(QZ_ERR_UNSUPPORTED, "qz_batch_run: the batch kernel cannot be resident here");
    }
    if (gr[1].n) {
        int dev = 0, per = 0;
        QZ_CUDA(cudaGetDevice(&dev));
        QZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        qzb::BatchArgs probe{};
        probe.ord = b->ord;
        probe.with_m1 = 1;
        probe.with_ext = gr[1].with_ext ? 1 : 0;
        QZ_CUDA(qzb::launch_batch_m1w(&probe, sizeof(probe), 0, gr[1].smem, st, &per));
        gr[1].grid = std::min(per * sms, gr[1].n);
        if (gr[1].grid < 1)
            return fail(QZ_ERR_UNSUPPORTED, "qz_batch_run: the 1024-thread batch kernel cannot be resident here");
    }
    const size_t fneed = std::max((size_t)gr[0].grid * gr[0].fmax, (size_t)gr[1].grid * gr[1].fmax);
    const size_t dneed = std::max((size_t)gr[0].grid * gr[0].dmax, (size_t)gr[1].grid * gr[1].dmax);
    const size_t bneed = std::max((size_t)gr[0].grid * gr[0].bmax, (size_t)gr[1].grid * gr[1].bmax);
    if (b->fld_alloc < fneed || b->diag_alloc < dneed || b->bsrc_alloc < bneed) {
        for (double* q : {b->d_fld, b->d_diag, b->d_bsrc})
            if (q) cudaFree(q);
        b->d_fld = b->d_diag = b->d_bsrc = nullptr;
        b->fld_alloc = b->diag_alloc = b->bsrc_alloc = 0;
        if (cudaMalloc((void**)&b->d_fld, sizeof(double) * fneed) != cudaSuccess ||
            cudaMalloc((void**)&b->d_diag, sizeof(double) * dneed) != cudaSuccess ||
            cudaMalloc((void**)&b->d_bsrc, sizeof(double) * bneed) != cudaSuccess) {
            cudaGetLastError();
            return fail(QZ_ERR_NOMEM, "qz_batch_run: device allocation failed (slot buffers)");
        }
        b->fld_alloc = fneed;
        b->diag_alloc = dneed;
        b->bsrc_alloc = bneed;
    }
    if (b->mom_alloc < mom_total) {
        if (b->d_mom) cudaFree(b->d_mom);
        b->d_mom = nullptr;
        QZ_CUDA(cudaMalloc((void**)&b->d_mom, sizeof(double) * mom_total));
        b->mom_alloc = mom_total;
    }
    std::vector<qzb::BatchInst> hi(ni);
    for (int i = 0; i < ni; ++i) {
        hi[i] = b->inst[i]->dev;
        hi[i].mom = b->d_mom + mom_off[i];
    }
    // the queue: the 512-thread group, then the wide group, each largest first
    std::vector<int> order(ni);
    for (int i = 0; i < ni; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return grp[x] != grp[y] ? grp[x] < grp[y] : b->inst[x]->cost > b->inst[y]->cost;
    });
    if (!b->d_inst) {
        QZ_CUDA(cudaMalloc((void**)&b->d_next, sizeof(int)));
    }
    if (b->d_inst) cudaFree(b->d_inst);
    if (b->d_order) cudaFree(b->d_order);
    b->d_inst = nullptr;
    b->d_order = nullptr;
    QZ_CUDA(cudaMalloc((void**)&b->d_inst, sizeof(qzb::BatchInst) * ni));
    QZ_CUDA(cudaMalloc((void**)&b->d_order, sizeof(int) * ni));
    QZ_CUDA(cudaMemcpyAsync(b->d_inst, hi.data(), sizeof(qzb::BatchInst) * ni, cudaMemcpyHostToDevice, st));
    QZ_CUDA(cudaMemcpyAsync(b->d_order, order.data(), sizeof(int) * ni, cudaMemcpyHostToDevice, st));
    qzb::BatchArgs B{};
    B.inst = b->d_inst;
    B.order = b->d_order;
    B.ninst = gr[0].n;
    B.nsteps = nsteps;
    B.dt = dt;
    B.ord = b->ord;
    B.with_m1 = gr[0].with_m1 ? 1 : 0;
    B.with_ext = gr[0].with_ext ? 1 : 0;
    B.fld = b->d_fld; B.diag = b->d_diag; B.bsrc = b->d_bsrc;
    B.fld_slot = gr[0].fmax; B.diag_slot = gr[0].dmax; B.bsrc_slot = gr[0].bmax;
    B.next = b->d_next;
    B.trace = nullptr;
    if (b->trace) {
        const size_t nt = (size_t)ni * qzb::kBatchTrace;
        if (b->trace_n < nt) {
            if (b->d_trace) cudaFree(b->d_trace);
            b->d_trace = nullptr;
            b->trace_n = 0;
            QZ_CUDA(cudaMalloc((void**)&b->d_trace, sizeof(unsigned long long) * nt));
            b->trace_n = nt;
        }
        QZ_CUDA(cudaMemsetAsync(b->d_trace, 0, sizeof(unsigned long long) * nt, st));
        B.trace = b->d_trace;
    }
    cudaEvent_t e0, e1;
    QZ_CUDA(cudaEventCreate(&e0));
    QZ_CUDA(cudaEventCreate(&e1));
    QZ_CUDA(cudaEventRecord(e0, st));
    if (gr[0].n) {
        QZ_CUDA(cudaMemsetAsync(b->d_next, 0, sizeof(int), st));
        QZ_CUDA(qzb::launch_batch(B, gr[0].grid, gr[0].smem, st));
    }
    if (gr[1].n) {
        qzb::BatchArgs W = B;
        W.order = b->d_order + gr[0].n;
        W.ninst = gr[1].n;
        W.with_m1 = 1;
        W.with_ext = gr[1].with_ext ? 1 : 0;
        W.fld_slot = gr[1].fmax; W.diag_slot = gr[1].dmax; W.bsrc_slot = gr[1].bmax;
        QZ_CUDA(cudaMemsetAsync(b->d_next, 0, sizeof(int), st));
        QZ_CUDA(qzb::launch_batch_m1w(&W, sizeof(W), gr[1].grid, gr[1].smem, st, nullptr));
    }
    QZ_CUDA(cudaEventRecord(e1, st));
    if (mom_host) QZ_CUDA(cudaMemcpyAsync(mom_host, b->d_mom, sizeof(double) * mom_total, cudaMemcpyDeviceToHost, st));
    if (B.trace) {
        b->h_trace.resize((size_t)ni * qzb::kBatchTrace);
        QZ_CUDA(cudaMemcpyAsync(b->h_trace.data(), B.trace, sizeof(unsigned long long) * b->h_trace.size(),
                                cudaMemcpyDeviceToHost, st));
    }
    QZ_CUDA(cudaStreamSynchronize(st));
    QZ_CUDA(cudaEventElapsedTime(&b->last_ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->last_grid = gr[0].n ? gr[0].grid : gr[1].grid;
    return QZ_OK;
}

extern "C" qz_status qz_batch_set_tuning(qz_batch* b, int index, int layout, double cost) {
    if (!b || index < 0 || index >= (int)b->inst.size()) return fail(QZ_ERR_ARG, "qz_batch_set_tuning: bad index");
    auto* I = b->inst[index];
    if (cost > 0.0) I->cost = cost;
    if (layout < 0) return QZ_OK;
    qzb::SweepArgs& A = I->dev.sw;
    if (I->dev.modes != 0 || layout > 7) return fail(QZ_ERR_ARG, "qz_batch_set_tuning: layouts are for modes = 0 (0..7)");
    const bool dbuf = layout & 1, cs = (layout >> 1) & 1, pc = (layout >> 2) & 1;
    if (pc && A.np <= qzb::kSweepThreads)
        return fail(QZ_ERR_ARG, "qz_batch_set_tuning: the particle copy is for plasma in global memory (np > 512)");
    int dev = 0, optin = 0;
    QZ_CUDA(cudaGetDevice(&dev));
    QZ_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t reserve = sizeof(qzb::BatchInst) + sizeof(double) * 17 * (qzb::kSweepThreads / 32) + 256;
    if (qzb::sweep_m0_smem_bytes(A.M, dbuf, cs, A.filter != 0, pc ? A.np : 0) + reserve > (size_t)optin)
        return fail(QZ_ERR_SIZE, "qz_batch_set_tuning: layout " + std::to_string(layout) + " does not fit M = " +
                                     std::to_string(A.M));
    A.dbuf = dbuf;
    A.const_smem = cs;
    A.pcache = pc ? A.np : 0;
    return QZ_OK;
}

extern "C" qz_status qz_batch_tuning(qz_batch* b, int index, int* layout, double* cost) {
    if (!b || index < 0 || index >= (int)b->inst.size() || !layout || !cost)
        return fail(QZ_ERR_ARG, "qz_batch_tuning: bad argument");
    const auto* I = b->inst[index];
    const qzb::SweepArgs& A = I->dev.sw;
    *layout = I->dev.modes ? -1 : (A.dbuf ? 1 : 0) | (A.const_smem ? 2 : 0) | (A.pcache ? 4 : 0);
    *cost = I->cost;
    return QZ_OK;
}

extern "C" qz_status qz_batch_set_trace(qz_batch* b, int enable) {
    if (!b) return fail(QZ_ERR_ARG, "qz_batch_set_trace: null pointer");
    b->trace = enable != 0;
    return QZ_OK;
}

extern "C" qz_status qz_batch_trace(qz_batch* b, double* out, int n) {
    if (!b || !out || n < 0) return fail(QZ_ERR_ARG, "qz_batch_trace: bad argument");
    const size_t ni = b->h_trace.size() / qzb::kBatchTrace;
    if ((size_t)n < ni) return fail(QZ_ERR_SIZE, "qz_batch_trace: out holds fewer instances than the last run");
    unsigned long long t0 = ~0ull;
    for (size_t i = 0; i < ni; ++i) t0 = std::min(t0, b->h_trace[i * qzb::kBatchTrace + 1]);
    for (size_t i = 0; i < ni; ++i) {
        const unsigned long long* t = b->h_trace.data() + i * qzb::kBatchTrace;
        double* o = out + i * 5;
        o[0] = (double)t[0];
        o[1] = 1e-6 * (double)(t[1] - t0);
        o[2] = 1e-6 * (double)(t[2] - t0);
        o[3] = 1e-6 * (double)t[3];
        o[4] = 1e-6 * (double)t[4];
    }
    return QZ_OK;
}

extern "C" qz_status qz_batch_info(qz_batch* b, double* out4) {
    if (!b || !out4) return fail(QZ_ERR_ARG, "qz_batch_info: null pointer");
    out4[0] = (double)b->inst.size();
    out4[1] = b->last_grid;
    out4[2] = b->last_ms;
    out4[3] = 0;
    return QZ_OK;
}
