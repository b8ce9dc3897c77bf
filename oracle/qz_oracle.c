/* qz_oracle.c -- CPU restatement of the QUARZ hot path (TEST INFRASTRUCTURE, see qz_oracle.h).
 *
 * Every routine follows the reference's arithmetic expression by expression (same operand
 * order, same rounding points) and sums in particle-index order, the order of the reference's
 * serial build. Compiled with -ffp-contract=off.
 */
#include "qz_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI 3.14159265358979323846

/* ===================================================================== random numbers */
/* mt19937_64 (Matsumoto & Nishimura, 64-bit Mersenne twister, published parameters) */
#define MT_N 312
#define MT_M 156
void qzo_rng_seed(qzo_rng* g, uint64_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < MT_N; ++i)
        g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->idx = MT_N;
    g->have_saved = 0;
    g->saved = 0;
}

static void mt_twist(qzo_rng* g) {
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL, A = 0xB5026F5AA96619E9ULL;
    for (int i = 0; i < MT_N; ++i) {
        const uint64_t x = (g->mt[i] & UM) | (g->mt[(i + 1) % MT_N] & LM);
        uint64_t xa = x >> 1;
        if (x & 1ULL) xa ^= A;
        g->mt[i] = g->mt[(i + MT_M) % MT_N] ^ xa;
    }
    g->idx = 0;
}

uint64_t qzo_rng_u64(qzo_rng* g) {
    if (g->idx >= MT_N) mt_twist(g);
    uint64_t y = g->mt[g->idx++];
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= y >> 43;
    return y;
}

/* 53-bit canonical variate from one 64-bit draw: u / 2^64 (rounded to double), kept below 1 */
double qzo_rng_canonical(qzo_rng* g) {
    const double u = (double)qzo_rng_u64(g);
    double r = u / 18446744073709551616.0;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    return r;
}

/* Marsaglia-Bray polar method; the pair's second member is cached for the next call.
   The variate returned first is the one built from the second uniform. */
double qzo_rng_normal(qzo_rng* g) {
    if (g->have_saved) { g->have_saved = 0; return g->saved; }
    double x, y, r2;
    do {
        x = 2.0 * qzo_rng_canonical(g) - 1.0;
        y = 2.0 * qzo_rng_canonical(g) - 1.0;
        r2 = x * x + y * y;
    } while (r2 > 1.0 || r2 == 0.0);
    const double mult = sqrt(-2 * log(r2) / r2);
    g->saved = x * mult;
    g->have_saved = 1;
    return y * mult;
}

/* ===================================================================== grid */
/* src/RadialGrid.cpp:139-145 */
int qzo_make_uniform(double R, double dr, double* out, int cap) {
    if (R <= 0 || dr <= 0) return -1;
    long n = lround(R / dr);
    if (n < 1) n = 1;
    if (n + 1 > cap) return -(int)(n + 1);
    for (long j = 0; j <= n; ++j) out[j] = R * (double)j / (double)n;
    return (int)(n + 1);
}

/* src/RadialGrid.cpp:27-71 */
static double regions_target(double x, const double* ends, const double* hs, int nreg, double g) {
    double ht = hs[nreg - 1];
    for (int i = 0; i < nreg; ++i)
        if (x < ends[i]) { ht = hs[i]; break; }
    double start = 0;
    for (int i = 0; i < nreg; ++i) {
        if (start > x && g > 0) { const double v = hs[i] + g * (start - x); if (v < ht) ht = v; }
        if (start > x && g == 0) { if (hs[i] < ht) ht = hs[i]; }
        start = ends[i];
    }
    return ht;
}

int qzo_make_regions(double R, const double* ends, const double* hs, int nreg, double max_ratio, double* out,
                     int cap) {
    if (nreg < 1 || max_ratio < 1.0) return -1;
    const double g = max_ratio - 1.0;
    int n = 0;
    out[n++] = 0.0;
    double x = 0, hprev = regions_target(0, ends, hs, nreg, g);
    while (x < R * (1 - 1e-12)) {
        const double ht = regions_target(x + 0.5 * hprev, ends, hs, nreg, g);
        double lo = hprev / max_ratio, hi = hprev * max_ratio;
        double hnew = ht < lo ? lo : (hi < ht ? hi : ht);
        if (n == 1) hnew = regions_target(0, ends, hs, nreg, g);
        x += hnew;
        if (n >= cap) return -2;
        out[n++] = x;
        hprev = hnew;
    }
    if (n >= 3 && (out[n - 1] - R) > (R - out[n - 2])) --n;
    const double scale = R / out[n - 1];
    for (int i = 0; i < n; ++i) out[i] *= scale;
    out[n - 1] = R;
    return n;
}

typedef struct {
    int N;
    double R;
    double *r, *h, *rmid, *V, *inv_h, *inv_V;
} grid_t;

/* src/RadialGrid.cpp:106-148 */
static int grid_init(grid_t* g, const double* nodes, int M) {
    if (M < 3 || nodes[0] != 0.0) return -1;
    for (int j = 1; j < M; ++j)
        if (!(nodes[j] > nodes[j - 1])) return -1;
    const int N = M - 1;
    g->N = N;
    g->r = (double*)malloc(sizeof(double) * M);
    g->V = (double*)malloc(sizeof(double) * M);
    g->inv_V = (double*)malloc(sizeof(double) * M);
    g->h = (double*)malloc(sizeof(double) * N);
    g->rmid = (double*)malloc(sizeof(double) * N);
    g->inv_h = (double*)malloc(sizeof(double) * N);
    memcpy(g->r, nodes, sizeof(double) * M);
    g->R = g->r[N];
    for (int j = 0; j < N; ++j) {
        g->h[j] = g->r[j + 1] - g->r[j];
        g->rmid[j] = 0.5 * (g->r[j + 1] + g->r[j]);
    }
    for (int j = 0; j <= N; ++j) {
        double v = 0;
        if (j > 0) v += g->r[j - 1] * g->h[j - 1] / 2 + g->h[j - 1] * g->h[j - 1] / 3;
        if (j < N) v += g->r[j] * g->h[j] / 2 + g->h[j] * g->h[j] / 6;
        g->V[j] = 2 * PI * v;
    }
    for (int j = 0; j <= N; ++j) g->inv_V[j] = 1.0 / g->V[j];
    for (int j = 0; j < N; ++j) g->inv_h[j] = 1.0 / g->h[j];
    return 0;
}

static void grid_free(grid_t* g) {
    free(g->r); free(g->V); free(g->inv_V); free(g->h); free(g->rmid); free(g->inv_h);
}

/* src/RadialGrid.hpp:35-50 */
static inline int grid_locate(const grid_t* g, double x) {
    if (x <= 0.0) return 0;
    if (x >= g->R) return g->N - 1;
    int lo = 0, hi = g->N;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (g->r[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

static inline void grid_weights(const grid_t* g, double x, int* j, double* t) {
    *j = grid_locate(g, x);
    double tt = (x - g->r[*j]) * g->inv_h[*j];
    tt = tt < 0.0 ? 0.0 : (tt > 1.0 ? 1.0 : tt);
    *t = tt;
}

/* ===================================================================== tridiagonal */
/* src/Tridiag.cpp:111-125 */
static void thomas(int M, const double* a, const double* b, const double* c, const double* d, double* x,
                   double* cp, double* dp) {
    cp[0] = c[0] / b[0];
    dp[0] = d[0] / b[0];
    for (int i = 1; i < M; ++i) {
        const double m = 1.0 / (b[i] - a[i] * cp[i - 1]);
        cp[i] = c[i] * m;
        dp[i] = (d[i] - a[i] * dp[i - 1]) * m;
    }
    x[M - 1] = dp[M - 1];
    for (int i = M - 2; i >= 0; --i) x[i] = dp[i] - cp[i] * x[i + 1];
}

/* src/Tridiag.cpp:127-162: PCR over the whole system (work: 8*M doubles) */
static void pcr(int M, const double* a, const double* b, const double* c, const double* d, double* x,
                double* work) {
    double *pa[2], *pb[2], *pc[2], *pd[2];
    for (int q = 0; q < 2; ++q) {
        pa[q] = work + (0 + 4 * q) * M; pb[q] = work + (1 + 4 * q) * M;
        pc[q] = work + (2 + 4 * q) * M; pd[q] = work + (3 + 4 * q) * M;
    }
    memcpy(pa[0], a, sizeof(double) * M); memcpy(pb[0], b, sizeof(double) * M);
    memcpy(pc[0], c, sizeof(double) * M); memcpy(pd[0], d, sizeof(double) * M);
    int src = 0;
    for (int s = 1; s < M; s *= 2) {
        const int dst = 1 - src;
        for (int i = 0; i < M; ++i) {
            const int lo = (i - s >= 0), hi = (i + s < M);
            const double alpha = lo ? -pa[src][i] / pb[src][i - s] : 0.0;
            const double gamma = hi ? -pc[src][i] / pb[src][i + s] : 0.0;
            pa[dst][i] = lo ? alpha * pa[src][i - s] : 0.0;
            pc[dst][i] = hi ? gamma * pc[src][i + s] : 0.0;
            pb[dst][i] = pb[src][i] + (lo ? alpha * pc[src][i - s] : 0.0) + (hi ? gamma * pa[src][i + s] : 0.0);
            pd[dst][i] = pd[src][i] + (lo ? alpha * pd[src][i - s] : 0.0) + (hi ? gamma * pd[src][i + s] : 0.0);
        }
        src = dst;
    }
    for (int i = 0; i < M; ++i) x[i] = pd[src][i] / pb[src][i];
}

/* src/Tridiag.cpp:30-109: Laszlo-Giles-Appleyard partition, P = min(256, M/8) chunks */
static void partition(int M, const double* a, const double* b, const double* c, const double* d, double* x,
                      double* work) {
    const int P = M / 8 < 256 ? M / 8 : 256, R = 2 * P;
    double *qa = work, *qc = work + M, *qd = work + 2 * M;
    double* r0[4]; double* r1[4];
    for (int q = 0; q < 4; ++q) { r0[q] = work + 3 * M + q * R; r1[q] = work + 3 * M + (4 + q) * R; }
    for (int t = 0; t < P; ++t) {
        const int s = (int)((long)t * M / P), e = (int)((long)(t + 1) * M / P);
        double r = 1.0 / b[s + 1];
        qa[s + 1] = a[s + 1] * r;
        qc[s + 1] = c[s + 1] * r;
        qd[s + 1] = d[s + 1] * r;
        for (int i = s + 2; i < e; ++i) {
            const double ci = (i == M - 1) ? 0.0 : c[i];
            r = 1.0 / (b[i] - a[i] * qc[i - 1]);
            qd[i] = r * (d[i] - a[i] * qd[i - 1]);
            qa[i] = -r * a[i] * qa[i - 1];
            qc[i] = r * ci;
        }
        for (int i = e - 3; i > s; --i) {
            const double cn = qc[i];
            qd[i] -= cn * qd[i + 1];
            qa[i] -= cn * qa[i + 1];
            qc[i] = -cn * qc[i + 1];
        }
        const double as = (s == 0) ? 0.0 : a[s];
        r0[0][2 * t] = as;
        r0[1][2 * t] = b[s] - c[s] * qa[s + 1];
        r0[2][2 * t] = -c[s] * qc[s + 1];
        r0[3][2 * t] = d[s] - c[s] * qd[s + 1];
        r0[0][2 * t + 1] = qa[e - 1];
        r0[1][2 * t + 1] = 1.0;
        r0[2][2 * t + 1] = qc[e - 1];
        r0[3][2 * t + 1] = qd[e - 1];
    }
    int flip = 0;
    for (int st = 1; st < R; st *= 2) {
        double** S = flip ? r1 : r0;
        double** D = flip ? r0 : r1;
        for (int i = 0; i < R; ++i) {
            const int lo = (i - st >= 0), hi = (i + st < R);
            const double alpha = lo ? -S[0][i] / S[1][i - st] : 0.0;
            const double gamma = hi ? -S[2][i] / S[1][i + st] : 0.0;
            D[0][i] = lo ? alpha * S[0][i - st] : 0.0;
            D[2][i] = hi ? gamma * S[2][i + st] : 0.0;
            D[1][i] = S[1][i] + (lo ? alpha * S[2][i - st] : 0.0) + (hi ? gamma * S[0][i + st] : 0.0);
            D[3][i] = S[3][i] + (lo ? alpha * S[3][i - st] : 0.0) + (hi ? gamma * S[3][i + st] : 0.0);
        }
        flip = !flip;
    }
    double** F = flip ? r1 : r0;
    for (int t = 0; t < P; ++t) {
        const int s = (int)((long)t * M / P), e = (int)((long)(t + 1) * M / P);
        const double xs = F[3][2 * t] / F[1][2 * t], xe = F[3][2 * t + 1] / F[1][2 * t + 1];
        x[s] = xs;
        x[e - 1] = xe;
        for (int i = s + 1; i < e - 1; ++i) x[i] = qd[i] - qa[i] * xs - qc[i] * xe;
    }
}

static int tridiag_work_size(int M) { return 3 * M + 8 * 512 + 8 * M; }

static void tridiag_any(int method, int M, const double* a, const double* b, const double* c, const double* d,
                        double* x, double* work) {
    if (method == QZO_PARTITION && M < 16) method = QZO_THOMAS;
    if (method == QZO_PCR) pcr(M, a, b, c, d, x, work);
    else if (method == QZO_PARTITION) partition(M, a, b, c, d, x, work);
    else thomas(M, a, b, c, d, x, work, work + M);
}

int qzo_tridiag(int method, int M, const double* a, const double* b, const double* c, const double* d, double* x) {
    double* work = (double*)malloc(sizeof(double) * tridiag_work_size(M));
    if (!work) return -1;
    tridiag_any(method, M, a, b, c, d, x, work);
    free(work);
    return 0;
}

/* ===================================================================== field solver */
typedef struct { double *a, *b, *c; int flux, regular; } op_t;

typedef struct {
    grid_t g;
    int method;
    op_t L[4];             /* L0, L1D, L1F, L2D */
    double flux_coef;
    double *gm, *g0, *gp, *ir;
    double *bw, *dw, *work;
    op_t F[3];             /* smoothing filter operators, angular number n = 0, 1, 2 */
    int filter_on;
    double* fw;
} solver_t;

enum { OP_L0 = 0, OP_L1D = 1, OP_L1F = 2, OP_L2D = 3 };

/* src/FieldSolver.cpp:90-103 */
static void fv_rows(const grid_t* g, int n, double* a, double* b, double* c) {
    const int N = g->N, M = N + 1;
    for (int j = 0; j < M; ++j) { a[j] = 0; b[j] = 0; c[j] = 0; }
    b[0] = 1.0;
    b[N] = 1.0;
    for (int j = 1; j < N; ++j) {
        const double dV = 0.5 * (g->h[j] + g->h[j - 1]);
        const double pre = pow(g->r[j], n - 1) / dV;
        const double kpj = 1.0 / (g->h[j] * pow(g->rmid[j], 2 * n - 1));
        const double kpm = 1.0 / (g->h[j - 1] * pow(g->rmid[j - 1], 2 * n - 1));
        c[j] = pre * pow(g->r[j + 1], n) * kpj;
        a[j] = pre * pow(g->r[j - 1], n) * kpm;
        b[j] = -pre * pow(g->r[j], n) * (kpj + kpm);
    }
}

/* src/FieldSolver.cpp:113-179 */
static int solver_init(solver_t* s, const double* nodes, int M, int method) {
    s->filter_on = 0;
    s->fw = NULL;
    for (int n = 0; n < 3; ++n) s->F[n].a = s->F[n].b = s->F[n].c = NULL;
    if (grid_init(&s->g, nodes, M)) return -1;
    const grid_t* g = &s->g;
    const int N = g->N;
    s->method = method;
    for (int k = 0; k < 4; ++k) {
        s->L[k].a = (double*)calloc(M, sizeof(double));
        s->L[k].b = (double*)calloc(M, sizeof(double));
        s->L[k].c = (double*)calloc(M, sizeof(double));
    }
    {   /* L0: lumped-mass FEM, Dirichlet at N */
        double *a = s->L[OP_L0].a, *b = s->L[OP_L0].b, *c = s->L[OP_L0].c;
        for (int j = 0; j < N; ++j) {
            const double invV = 2 * PI / g->V[j];
            a[j] = (j > 0) ? g->rmid[j - 1] / g->h[j - 1] * invV : 0.0;
            c[j] = g->rmid[j] / g->h[j] * invV;
            b[j] = -(a[j] + c[j]);
        }
        b[N] = 1.0;
        s->L[OP_L0].regular = 1;
        s->L[OP_L0].flux = 0;
    }
    fv_rows(g, 1, s->L[OP_L1D].a, s->L[OP_L1D].b, s->L[OP_L1D].c);
    s->L[OP_L1D].regular = 0; s->L[OP_L1D].flux = 0;
    fv_rows(g, 1, s->L[OP_L1F].a, s->L[OP_L1F].b, s->L[OP_L1F].c);
    {
        const double dV = 0.5 * g->h[N - 1];
        const double kp = 1.0 / (g->h[N - 1] * pow(g->rmid[N - 1], 2 * 1 - 1));
        const double k = kp / dV;
        s->L[OP_L1F].a[N] = g->r[N - 1] * k;
        s->L[OP_L1F].b[N] = -g->r[N] * k;
        s->flux_coef = 1.0 / dV;
    }
    s->L[OP_L1F].regular = 0; s->L[OP_L1F].flux = 1;
    fv_rows(g, 2, s->L[OP_L2D].a, s->L[OP_L2D].b, s->L[OP_L2D].c);
    s->L[OP_L2D].regular = 0; s->L[OP_L2D].flux = 0;

    s->gm = (double*)calloc(M, sizeof(double));
    s->g0 = (double*)calloc(M, sizeof(double));
    s->gp = (double*)calloc(M, sizeof(double));
    s->ir = (double*)calloc(M, sizeof(double));
    for (int j = 1; j < N; ++j) {
        const double hm = g->h[j - 1], hp = g->h[j];
        const double den = hm * hp * (hm + hp);
        s->gp[j] = hm * hm / den;
        s->gm[j] = -hp * hp / den;
        s->g0[j] = (hp * hp - hm * hm) / den;
    }
    {
        const double h1 = g->h[N - 1], h2 = (N >= 2) ? g->h[N - 2] : g->h[N - 1];
        const double sm = h1 + h2;
        s->g0[N] = (2 * h1 + h2) / (h1 * sm);
        s->gm[N] = -sm / (h1 * h2);
        s->gp[N] = h1 / (h2 * sm);
    }
    for (int j = 1; j <= N; ++j) s->ir[j] = 1.0 / g->r[j];
    s->ir[0] = 1.0 / g->r[1];
    s->bw = (double*)malloc(sizeof(double) * M);
    s->dw = (double*)malloc(sizeof(double) * M);
    s->work = (double*)malloc(sizeof(double) * tridiag_work_size(M));
    return 0;
}

static void solver_free(solver_t* s) {
    for (int k = 0; k < 4; ++k) { free(s->L[k].a); free(s->L[k].b); free(s->L[k].c); }
    for (int n = 0; n < 3; ++n) { free(s->F[n].a); free(s->F[n].b); free(s->F[n].c); }
    free(s->fw);
    free(s->gm); free(s->g0); free(s->gp); free(s->ir); free(s->bw); free(s->dw); free(s->work);
    grid_free(&s->g);
}

/* src/FieldSolver.cpp:172-191 */
static void solver_solve(solver_t* s, int k, const double* rhs, double* f, const double* chi, const double* wall,
                         double scale) {
    const op_t* o = &s->L[k];
    const int N = s->g.N;
    for (int j = 0; j <= N; ++j) {
        const int dirichlet = (j == N && !o->flux) || (j == 0 && !o->regular);
        if (dirichlet) { s->bw[j] = o->b[j]; s->dw[j] = 0.0; continue; }
        s->bw[j] = chi ? o->b[j] - chi[j] : o->b[j];
        s->dw[j] = scale * rhs[j];
        if (j == N && o->flux) s->dw[j] -= s->flux_coef * wall[N];
    }
    tridiag_any(s->method, N + 1, o->a, s->bw, o->c, s->dw, f, s->work);
}

/* FieldSolver::set_filter (src/FieldSolver.cpp:111-146): the implicit radial diffusion
   1 - div a^2 grad of angular number n with a^2 = a2[j] in cell j. n = 0 in flux form on the node
   volumes with a zero-flux wall (charge conserving); n = 1, 2 as the finite-volume L_n with a^2 inside
   the flux, identity rows on the axis and at the wall. */
static void solver_set_filter(solver_t* s, const double* a2) {
    const grid_t* g = &s->g;
    const int N = g->N, M = N + 1;
    s->filter_on = 0;
    for (int j = 0; j < N; ++j)
        if (a2[j] > 0) s->filter_on = 1;
    if (!s->filter_on) return;
    for (int n = 0; n < 3; ++n) {
        s->F[n].a = (double*)calloc(M, sizeof(double));
        s->F[n].b = (double*)calloc(M, sizeof(double));
        s->F[n].c = (double*)calloc(M, sizeof(double));
        for (int j = 0; j < M; ++j) s->F[n].b[j] = 1.0;
    }
    s->fw = (double*)calloc(M, sizeof(double));
    for (int j = 0; j <= N; ++j) {
        const double invV = 2 * PI / g->V[j];
        const double am = (j > 0) ? a2[j - 1] * g->rmid[j - 1] / g->h[j - 1] * invV : 0.0;
        const double cp = (j < N) ? a2[j] * g->rmid[j] / g->h[j] * invV : 0.0;
        s->F[0].a[j] = -am;
        s->F[0].c[j] = -cp;
        s->F[0].b[j] = 1 + am + cp;
    }
    for (int n = 1; n <= 2; ++n)
        for (int j = 1; j < N; ++j) {
            const double dV = 0.5 * (g->h[j] + g->h[j - 1]);
            const double pre = pow(g->r[j], n - 1) / dV;
            const double kpj = a2[j] / (g->h[j] * pow(g->rmid[j], 2 * n - 1));
            const double kpm = a2[j - 1] / (g->h[j - 1] * pow(g->rmid[j - 1], 2 * n - 1));
            s->F[n].c[j] = -pre * pow(g->r[j + 1], n) * kpj;
            s->F[n].a[j] = -pre * pow(g->r[j - 1], n) * kpm;
            s->F[n].b[j] = 1 + pre * pow(g->r[j], n) * (kpj + kpm);
        }
}

/* FieldSolver::filter (src/FieldSolver.cpp:148-161): f <- F_n^{-1} f */
static void solver_filter(solver_t* s, int n, double* f) {
    if (!s->filter_on) return;
    const op_t* o = &s->F[n];
    const int M = s->g.N + 1;
    for (int j = 0; j < M; ++j) { s->bw[j] = o->b[j]; s->dw[j] = f[j]; }
    tridiag_any(s->method, M, o->a, s->bw, o->c, s->dw, s->fw, s->work);
    memcpy(f, s->fw, sizeof(double) * M);
}

int qzo_filter(const double* nodes, int M, double a2, int n, double* f) {
    if (n < 0 || n > 2) return -1;
    solver_t s;
    memset(&s, 0, sizeof(s));
    if (solver_init(&s, nodes, M, QZO_THOMAS)) return -1;
    double* a = (double*)malloc(sizeof(double) * M);
    for (int j = 0; j < M; ++j) a[j] = a2;
    solver_set_filter(&s, a);
    solver_filter(&s, n, f);
    free(a);
    solver_free(&s);
    return 0;
}

/* src/FieldSolver.cpp:193-219 */
static void solver_gradient(const solver_t* s, const double* f, double* df) {
    const int N = s->g.N;
    for (int j = 0; j <= N; ++j) {
        if (j == 0) { df[0] = 0.0; continue; }
        if (j == N) { df[N] = s->g0[N] * f[N] + s->gm[N] * f[N - 1] + s->gp[N] * f[N - 2]; continue; }
        df[j] = s->gm[j] * f[j - 1] + s->g0[j] * f[j] + s->gp[j] * f[j + 1];
    }
}
static void solver_gradient_odd(const solver_t* s, const double* f, double* df) {
    const int N = s->g.N;
    for (int j = 0; j <= N; ++j) {
        if (j == 0) { df[0] = f[1] * s->ir[0]; continue; }
        if (j == N) { df[N] = s->g0[N] * f[N] + s->gm[N] * f[N - 1] + s->gp[N] * f[N - 2]; continue; }
        df[j] = s->gm[j] * f[j - 1] + s->g0[j] * f[j] + s->gp[j] * f[j + 1];
    }
}
static void solver_over_r(const solver_t* s, const double* f, double* out) {
    const int N = s->g.N;
    for (int j = 0; j <= N; ++j) out[j] = (j == 0 ? f[1] : f[j]) * s->ir[j];
}

int qzo_field_solve(const double* nodes, int M, int op, int method, const double* rhs, const double* chi,
                    const double* wall, double scale, double* f) {
    solver_t s;
    if (solver_init(&s, nodes, M, method)) return -1;
    solver_solve(&s, op, rhs, f, chi, wall, scale);
    solver_free(&s);
    return 0;
}

int qzo_operator_rows(const double* nodes, int M, int op, double* a, double* b, double* c, double* flux_coef) {
    solver_t s;
    if (solver_init(&s, nodes, M, QZO_THOMAS)) return -1;
    memcpy(a, s.L[op].a, sizeof(double) * M);
    memcpy(b, s.L[op].b, sizeof(double) * M);
    memcpy(c, s.L[op].c, sizeof(double) * M);
    if (flux_coef) *flux_coef = s.flux_coef;
    solver_free(&s);
    return 0;
}

int qzo_stencils(const double* nodes, int M, double* gm, double* g0, double* gp, double* ir) {
    solver_t s;
    if (solver_init(&s, nodes, M, QZO_THOMAS)) return -1;
    memcpy(gm, s.gm, sizeof(double) * M); memcpy(g0, s.g0, sizeof(double) * M);
    memcpy(gp, s.gp, sizeof(double) * M); memcpy(ir, s.ir, sizeof(double) * M);
    solver_free(&s);
    return 0;
}

int qzo_grid_volumes(const double* nodes, int M, double* V) {
    grid_t g;
    if (grid_init(&g, nodes, M)) return -1;
    memcpy(V, g.V, sizeof(double) * M);
    grid_free(&g);
    return 0;
}

/* ===================================================================== pushers (src/Pushers.hpp:36-68) */
typedef struct { double x, y, z; } v3;
static inline v3 v3add(v3 a, v3 b) { v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static inline v3 v3mul(double s, v3 a) { v3 r = {s * a.x, s * a.y, s * a.z}; return r; }
static inline double v3dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 v3cross(v3 a, v3 b) {
    v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static inline double gamma2_root(double x, double c) {
    const double s = sqrt(x * x + c);
    return x >= 0.0 ? x + s : (s > -x ? c / (s - x) : 1.0);
}
static inline v3 solve_implicit(v3 a, v3 b) {
    const double b2 = v3dot(b, b), ab = v3dot(a, b);
    const double g2 = gamma2_root(0.5 * (1.0 + v3dot(a, a) - b2), b2 + ab * ab);
    const double g = sqrt(g2);
    const v3 axb = v3cross(a, b);
    const double inv = 1.0 / (g2 + b2);
    v3 r = {inv * (g2 * a.x + g * axb.x + ab * b.x), inv * (g2 * a.y + g * axb.y + ab * b.y),
            inv * (g2 * a.z + g * axb.z + ab * b.z)};
    return r;
}
static inline v3 vay(v3 u, v3 E, v3 B, double eps) {
    const double g0 = sqrt(1.0 + v3dot(u, u));
    const v3 up = v3add(v3add(u, v3mul(2.0 * eps, E)), v3mul(eps / g0, v3cross(u, B)));
    return solve_implicit(up, v3mul(eps, B));
}
void qzo_vay(const double u[3], const double E[3], const double B[3], double eps, double out[3]) {
    v3 uu = {u[0], u[1], u[2]}, EE = {E[0], E[1], E[2]}, BB = {B[0], B[1], B[2]};
    v3 r = vay(uu, EE, BB, eps);
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

/* src/Pushers.hpp:64-95, the other beam pushers. Boris (1970): half electric kick, rotation by
   t = eps B / gamma(u-), half kick. */
static inline v3 boris(v3 u, v3 E, v3 B, double eps) {
    const v3 um = v3add(u, v3mul(eps, E));
    const double g = sqrt(1.0 + v3dot(um, um));
    const v3 t = v3mul(eps / g, B);
    const v3 s = v3mul(2.0 / (1.0 + v3dot(t, t)), t);
    const v3 up = v3add(um, v3cross(v3add(um, v3cross(um, t)), s));
    return v3add(up, v3mul(eps, E));
}
/* Higuera & Cary (2017): the rotation with the gamma of the time-centred momentum, from the
   quadratic for gamma+^2 */
static inline v3 higuera_cary(v3 u, v3 E, v3 B, double eps) {
    const v3 um = v3add(u, v3mul(eps, E));
    const v3 tau = v3mul(eps, B);
    const double us = v3dot(um, tau), tt = v3dot(tau, tau);
    const double sig = 1.0 + v3dot(um, um) - tt;
    const double gp = sqrt(0.5 * (sig + sqrt(sig * sig + 4.0 * (tt + us * us))));
    const v3 t = v3mul(1.0 / gp, tau);
    const double s = 1.0 / (1.0 + v3dot(t, t));
    const v3 upl = v3mul(s, v3add(v3add(um, v3mul(v3dot(um, t), t)), v3cross(um, t)));
    return v3add(v3add(upl, v3mul(eps, E)), v3cross(upl, t));
}
/* the implicit midpoint push: ubar = (u + eps E) + (ubar / gamma(ubar)) x eps B solved exactly,
   u+ = 2 ubar - u */
static inline v3 imp(v3 u, v3 E, v3 B, double eps) {
    const v3 ub = solve_implicit(v3add(u, v3mul(eps, E)), v3mul(eps, B));
    return v3add(v3mul(2.0, ub), v3mul(-1.0, u));
}
/* pusher kinds of <beam>.pusher: 0 vay, 1 boris, 2 hc, 3 imp (src/Beam.cpp:72-78) */
static inline v3 push_u(int kind, v3 u, v3 E, v3 B, double eps) {
    switch (kind) {
        case 1: return boris(u, E, B, eps);
        case 2: return higuera_cary(u, E, B, eps);
        case 3: return imp(u, E, B, eps);
        default: return vay(u, E, B, eps);
    }
}
int qzo_push(int kind, long n, const double* u, const double* E, const double* B, const double* eps, double* out) {
    if (kind < 0 || kind > 3) return -1;
    for (long i = 0; i < n; ++i) {
        const v3 uu = {u[3 * i], u[3 * i + 1], u[3 * i + 2]}, EE = {E[3 * i], E[3 * i + 1], E[3 * i + 2]};
        const v3 BB = {B[3 * i], B[3 * i + 1], B[3 * i + 2]};
        const v3 r = push_u(kind, uu, EE, BB, eps[i]);
        out[3 * i] = r.x; out[3 * i + 1] = r.y; out[3 * i + 2] = r.z;
    }
    return 0;
}

/* ===================================================================== Adams-Bashforth (src/PlasmaSpecies.cpp:14-48) */
int qzo_ab_coeffs(int order, double* c) {
    for (int m = 0; m < 5; ++m) c[m] = 0;
    switch (order) {
        case 1: c[0] = 1; break;
        case 2: c[0] = 1.5; c[1] = -0.5; break;
        case 3: c[0] = 23. / 12; c[1] = -16. / 12; c[2] = 5. / 12; break;
        case 4: c[0] = 55. / 24; c[1] = -59. / 24; c[2] = 37. / 24; c[3] = -9. / 24; break;
        case 5: c[0] = 1901. / 720; c[1] = -2774. / 720; c[2] = 2616. / 720; c[3] = -1274. / 720; c[4] = 251. / 720;
            break;
        default: return -1;
    }
    return 0;
}

int qzo_ab_variable(int order, const double* t, double h, double* c) {
    const double gx[3] = {-0.7745966692414834, 0.0, 0.7745966692414834};
    const double gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    for (int m = 0; m < 5; ++m) c[m] = 0;
    for (int m = 0; m < order; ++m) {
        double s = 0;
        for (int q = 0; q < 3; ++q) {
            const double tt = t[0] + 0.5 * h * (1.0 + gx[q]);
            double l = 1;
            for (int n = 0; n < order; ++n)
                if (n != m) l *= (tt - t[n]) / (t[m] - t[n]);
            s += 0.5 * gw[q] * l;
        }
        c[m] = s;
    }
    return 0;
}

/* Timing build (the reference's OpenMP backend stand-in): compiled with -fopenmp, the per-particle
   loops run on all host threads with atomic source updates; without it these expand to the serial
   code, whose fixed summation order is the oracle's. */
#ifdef _OPENMP
#define QZO_ADD(x, v) do { _Pragma("omp atomic") (x) += (v); } while (0)
#define QZO_PFOR _Pragma("omp parallel for schedule(static)")
#else
#define QZO_ADD(x, v) ((x) += (v))
#define QZO_PFOR
#endif

/* ===================================================================== simulation */
/* field / beam-source / diagnostic components (src/FieldStore.hpp:9-21, src/Simulation.hpp:44) */
enum { F_EP1R = 0, F_EP1I, F_BP1R, F_BP1I, F_EZ0, F_BZ0, F_EP0R, F_EP0I, F_EP2R, F_EP2I, F_BP0R, F_BP0I, F_BP2R,
       F_BP2I, F_EZ1R, F_EZ1I, F_BZ1R, F_BZ1I };
enum { B_RT0 = 0, B_JZ0, B_JP1R, B_JP1I, B_RHO0, B_RT1R, B_RT1I, B_JZ1R, B_JZ1I, B_JP0R, B_JP0I, B_JP2R, B_JP2I,
       B_RHO1R, B_RHO1I };
enum { D_PSI0 = 0, D_NE0, D_NI0, D_PSI1R, D_PSI1I, D_NE1R, D_NE1I, D_NI1R, D_NI1I };

typedef struct { double *a0, *ar, *ai; } msc_t;
typedef struct { double *r0, *i0, *r1, *i1, *r2, *i2; } mvec_t;

typedef struct {
    qzo_species_params p;
    int Np, cap;
    double *x, *y, *px, *py, *dl, *w;
    double* hist;          /* (order, 5, cap) */
    long npush;
    double xi_cur, xi_slot[5];
    double ab[5];
} species_t;

typedef struct {
    double q, m;
    int rigid, started;
    long n;
    double *x, *y, *px, *py, *pz, *xi, *w;
    double gref, xiref;
    int pusher;            /* 0 vay, 1 boris, 2 hc, 3 imp */
    /* analytic rigid beam (no particles): src/Beam.hpp:153-160 */
    int analytic, an_flat;
    double an_n0, an_sr, an_xi0, an_sxi, an_len, an_cut, an_x0, an_y0, an_xs, an_ys, an_gamma;
} beam_t;

struct qzo_sim {
    qzo_params p;
    solver_t fs;
    int M, m1;
    int nsp, nb;
    species_t sp[4];
    beam_t bm[8];
    /* sources */
    msc_t rhot, drho, jz, chi, rho, ne, ni;
    mvec_t jp, S;
    /* fields */
    msc_t psi, ez, bz;
    mvec_t wp, bp, bprev;
    double *t1, *t2, *t3, *t4, *rhs;
    msc_t bg_rhot, bg_rho;
    mvec_t gz;
    double* bguard;        /* (M, 15) */
    double *fld, *bsrc, *diag;
    int fnc, bnc, dnc;
    long lost;
    long nsub_extra;       /* sub-slices beyond the regular slices, all sweeps */
    double* pool;
    /* optional (the adjoint's recomputation): the mobile species' state at the start of every
       slice, (K, 6 + 5 * ab_order, cap) -- x y px py dl w, then the AB history */
    double* traj;
};

static double* take(double** cur, int M) { double* r = *cur; *cur += M; return r; }
static void msc_take(msc_t* m, double** cur, int M) { m->a0 = take(cur, M); m->ar = take(cur, M); m->ai = take(cur, M); }
static void mvec_take(mvec_t* v, double** cur, int M) {
    v->r0 = take(cur, M); v->i0 = take(cur, M); v->r1 = take(cur, M);
    v->i1 = take(cur, M); v->r2 = take(cur, M); v->i2 = take(cur, M);
}
static void msc_zero(msc_t* m, int M) {
    memset(m->a0, 0, sizeof(double) * M); memset(m->ar, 0, sizeof(double) * M); memset(m->ai, 0, sizeof(double) * M);
}
static void mvec_zero(mvec_t* v, int M) {
    memset(v->r0, 0, sizeof(double) * M); memset(v->i0, 0, sizeof(double) * M); memset(v->r1, 0, sizeof(double) * M);
    memset(v->i1, 0, sizeof(double) * M); memset(v->r2, 0, sizeof(double) * M); memset(v->i2, 0, sizeof(double) * M);
}

qzo_sim* qzo_sim_create(const qzo_params* p, const double* nodes, int M) {
    qzo_sim* s = (qzo_sim*)calloc(1, sizeof(qzo_sim));
    s->p = *p;
    if (solver_init(&s->fs, nodes, M, p->tridiag)) { free(s); return NULL; }
    s->M = M;
    s->m1 = p->modes == 1;
    if (p->smooth_length < 0) { solver_free(&s->fs); free(s); return NULL; }
    if (p->smooth_length > 0) {   /* src/Simulation.cpp:63-66: a^2 in every cell */
        double* a2 = (double*)malloc(sizeof(double) * M);
        for (int j = 0; j < M; ++j) a2[j] = p->smooth_length * p->smooth_length;
        solver_set_filter(&s->fs, a2);
        free(a2);
    }
    const int narr = 7 * 3 + 2 * 6 + 3 * 3 + 3 * 6 + 5 + 2 * 3 + 6;
    s->pool = (double*)calloc((size_t)narr * M + 15 * (size_t)M, sizeof(double));
    double* cur = s->pool;
    msc_take(&s->rhot, &cur, M); msc_take(&s->drho, &cur, M); msc_take(&s->jz, &cur, M);
    msc_take(&s->chi, &cur, M); msc_take(&s->rho, &cur, M); msc_take(&s->ne, &cur, M); msc_take(&s->ni, &cur, M);
    mvec_take(&s->jp, &cur, M); mvec_take(&s->S, &cur, M);
    msc_take(&s->psi, &cur, M); msc_take(&s->ez, &cur, M); msc_take(&s->bz, &cur, M);
    mvec_take(&s->wp, &cur, M); mvec_take(&s->bp, &cur, M); mvec_take(&s->bprev, &cur, M);
    s->t1 = take(&cur, M); s->t2 = take(&cur, M); s->t3 = take(&cur, M); s->t4 = take(&cur, M); s->rhs = take(&cur, M);
    msc_take(&s->bg_rhot, &cur, M); msc_take(&s->bg_rho, &cur, M);
    mvec_take(&s->gz, &cur, M);
    s->bguard = cur;
    s->fnc = s->m1 ? 18 : 6;
    s->bnc = s->m1 ? 15 : 5;
    s->dnc = s->m1 ? 9 : 3;
    const size_t KM = (size_t)p->K * M;
    s->fld = (double*)calloc(KM * s->fnc, sizeof(double));
    s->bsrc = (double*)calloc(KM * s->bnc, sizeof(double));
    s->diag = (double*)calloc(KM * s->dnc, sizeof(double));
    if (!s->fld || !s->bsrc || !s->diag) { qzo_sim_destroy(s); return NULL; }
    return s;
}

void qzo_sim_destroy(qzo_sim* s) {
    if (!s) return;
    for (int i = 0; i < s->nsp; ++i) {
        species_t* q = &s->sp[i];
        free(q->x); free(q->y); free(q->px); free(q->py); free(q->dl); free(q->w); free(q->hist);
    }
    for (int b = 0; b < s->nb; ++b) {
        beam_t* B = &s->bm[b];
        free(B->x); free(B->y); free(B->px); free(B->py); free(B->pz); free(B->xi); free(B->w);
    }
    free(s->fld); free(s->bsrc); free(s->diag); free(s->pool);
    solver_free(&s->fs);
    free(s);
}

int qzo_sim_add_species(qzo_sim* s, const qzo_species_params* sp) {
    if (s->nsp >= 4) return -1;
    species_t* q = &s->sp[s->nsp++];
    memset(q, 0, sizeof(*q));
    q->p = *sp;
    const int N = s->fs.g.N;
    q->cap = N * sp->ppc * sp->ntheta;
    if (q->cap < 1) q->cap = 1;
    q->x = (double*)calloc(q->cap, sizeof(double)); q->y = (double*)calloc(q->cap, sizeof(double));
    q->px = (double*)calloc(q->cap, sizeof(double)); q->py = (double*)calloc(q->cap, sizeof(double));
    q->dl = (double*)calloc(q->cap, sizeof(double)); q->w = (double*)calloc(q->cap, sizeof(double));
    q->hist = (double*)calloc((size_t)s->p.ab_order * 5 * q->cap, sizeof(double));
    qzo_ab_coeffs(s->p.ab_order, q->ab);
    return 0;
}

int qzo_sim_add_beam(qzo_sim* s, const double* p7, long n, double q, double m, int rigid, double gref, double xiref) {
    if (s->nb >= 8) return -1;
    beam_t* B = &s->bm[s->nb++];
    memset(B, 0, sizeof(*B));
    B->q = q; B->m = m; B->rigid = rigid; B->n = n; B->gref = gref; B->xiref = xiref;
    double** cols[7] = {&B->x, &B->y, &B->px, &B->py, &B->pz, &B->xi, &B->w};
    for (int c = 0; c < 7; ++c) {
        *cols[c] = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
        for (long i = 0; i < n; ++i) (*cols[c])[i] = p7[7 * i + c];
    }
    return 0;
}

int qzo_sim_set_beam_pusher(qzo_sim* s, int b, int kind) {
    if (b < 0 || b >= s->nb || kind < 0 || kind > 3) return -1;
    s->bm[b].pusher = kind;
    return 0;
}

int qzo_sim_add_analytic_beam(qzo_sim* s, double q, double n0, double sigma_r, double xi0, double sigma_xi,
                              int flattop, double length, double xi_cut, double x0, double y0, double xs,
                              double ys, double gamma) {
    if (s->nb >= 8 || !(sigma_r > 0) || !(gamma >= 1) || (!flattop && !(sigma_xi > 0))) return -1;
    if (!s->m1 && (x0 != 0 || y0 != 0 || xs != 0 || ys != 0)) return -1;   /* src/Beam.cpp:197-198 */
    beam_t* B = &s->bm[s->nb++];
    memset(B, 0, sizeof(*B));
    B->q = q; B->m = 1.0; B->rigid = 1; B->n = 0; B->analytic = 1;
    double** cols[7] = {&B->x, &B->y, &B->px, &B->py, &B->pz, &B->xi, &B->w};
    for (int c = 0; c < 7; ++c) *cols[c] = (double*)malloc(sizeof(double));
    B->an_flat = flattop; B->an_n0 = n0; B->an_sr = sigma_r; B->an_xi0 = xi0; B->an_sxi = sigma_xi;
    B->an_len = length; B->an_cut = xi_cut; B->an_x0 = x0; B->an_y0 = y0; B->an_xs = xs; B->an_ys = ys;
    B->an_gamma = gamma;
    return 0;
}

/* Abramowitz & Stegun 9.8.1-9.8.4: I0, I1 as polynomials in (z / 3.75)^2 below 3.75, and
   sqrt(z) e^{-z} I0,1 as polynomials in 3.75 / z above (relative error below 2e-7) */
void qzo_bessel_i01_scaled(double z, double* i0, double* i1) {
    if (z < 3.75) {
        const double t = (z / 3.75) * (z / 3.75);
        const double I0 = 1.0 + t * (3.5156229 + t * (3.0899424 + t * (1.2067492 + t * (0.2659732
                          + t * (0.0360768 + t * 0.0045813)))));
        const double I1 = z * (0.5 + t * (0.87890594 + t * (0.51498869 + t * (0.15084934 + t * (0.02658733
                          + t * (0.00301532 + t * 0.00032411))))));
        const double e = exp(-z);
        *i0 = I0 * e;
        *i1 = I1 * e;
    } else {
        const double u = 3.75 / z, sq = 1.0 / sqrt(z);
        *i0 = sq * (0.39894228 + u * (0.01328592 + u * (0.00225319 + u * (-0.00157565 + u * (0.00916281
              + u * (-0.02057706 + u * (0.02635537 + u * (-0.01647633 + u * 0.00392377))))))));
        *i1 = sq * (0.39894228 + u * (-0.03988024 + u * (-0.00362018 + u * (0.00163801 + u * (-0.01031555
              + u * (0.02282967 + u * (-0.02895312 + u * (0.01787654 - u * 0.00420059))))))));
    }
}

/* src/Beam.cpp:236-279: rho = q n0 f(xi) exp(-|x_perp - c(xi)|^2 / 2 sigma_r^2) moving at v_z(gamma), its
   azimuthal modes at every node through the scaled Bessel functions of z = r d / sigma_r^2 */
static void deposit_analytic(qzo_sim* s, const beam_t* B) {
    const grid_t* g = &s->fs.g;
    const int M = s->M, K = s->p.K, bnc = s->bnc, m1 = s->m1;
    const double s2 = B->an_sr * B->an_sr;
    const double gam = B->an_gamma;
    const double vz = sqrt(1.0 - 1.0 / (gam * gam));
    const double omvz = 1.0 / (gam * gam * (1.0 + vz));
    for (int k = 0; k < K; ++k) {
        const double xi = s->p.xi_min + k * s->p.dxi;
        if (xi < B->an_cut) continue;
        double fxi;
        if (B->an_flat) fxi = (fabs(xi - B->an_xi0) <= 0.5 * B->an_len) ? 1.0 : 0.0;
        else fxi = exp(-0.5 * (xi - B->an_xi0) * (xi - B->an_xi0) / (B->an_sxi * B->an_sxi));
        if (fxi == 0.0) continue;
        const double cx = B->an_x0 + B->an_xs * (xi - B->an_xi0), cy = B->an_y0 + B->an_ys * (xi - B->an_xi0);
        const double d = sqrt(cx * cx + cy * cy);
        for (int j = 0; j < M; ++j) {
            const double r = g->r[j];
            double i0, i1;
            qzo_bessel_i01_scaled(r * d / s2, &i0, &i1);
            const double env = B->q * B->an_n0 * fxi * exp(-0.5 * (r - d) * (r - d) / s2);
            const double rho0 = env * i0;
            double* o = s->bsrc + ((size_t)k * M + j) * bnc;
            o[B_RHO0] += rho0;
            o[B_RT0] += rho0 * omvz;
            o[B_JZ0] += rho0 * vz;
            if (m1 && d > 0.0) {
                const double f1r = env * i1 * (cx / d), f1i = -env * i1 * (cy / d);
                o[B_RHO1R] += f1r; o[B_RHO1I] += f1i;
                o[B_RT1R] += f1r * omvz; o[B_RT1I] += f1i * omvz;
                o[B_JZ1R] += f1r * vz; o[B_JZ1I] += f1i * vz;
            }
        }
    }
}

/* ---- plasma ---- */
static double prof_radial(const qzo_species_params* p, double r) {
    if (r > p->rmax) return 0.0;
    if (p->channel_radius > 0) return 1.0 + p->channel_depth * (r / p->channel_radius) * (r / p->channel_radius);
    return 1.0;
}

/* src/PlasmaSpecies.cpp:202-295 (cold plasma, built-in radial profiles) */
static void species_load(qzo_sim* s, species_t* q) {
    const grid_t* g = &s->fs.g;
    const double fz = 1.0 * q->p.density;
    const int ppc = q->p.ppc, nth = q->p.ntheta;
    int i = 0;
    for (int j = 0; j < g->N; ++j) {
        const double h = g->h[j];
        for (int m = 0; m < ppc; ++m) {
            const double ra = g->r[j] + m * h / ppc, rb = g->r[j] + (m + 1) * h / ppc;
            const double r = (2.0 / 3.0) * (rb * rb * rb - ra * ra * ra) / (rb * rb - ra * ra);
            const double vring = fz * PI * (rb * rb - ra * ra);
            const double wring = prof_radial(&q->p, r) * vring;
            const double off = ((j * ppc + m) % 2) * 0.5;
            for (int l = 0; l < nth; ++l, ++i) {
                const double th = 2 * PI * (l + off) / nth;
                const double px = 0, py = 0, pz = 0;
                const double gam = sqrt(1 + px * px + py * py + pz * pz);
                const double X = (nth == 1) ? r : r * cos(th), Y = (nth == 1) ? 0.0 : r * sin(th);
                const double W = wring / nth;
                if (W == 0) { --i; continue; }
                q->x[i] = X; q->y[i] = Y; q->px[i] = px; q->py[i] = py; q->dl[i] = gam - pz; q->w[i] = W;
            }
        }
    }
    memset(q->hist, 0, sizeof(double) * (size_t)s->p.ab_order * 5 * q->cap);
    q->Np = i;
    q->npush = 0;
    q->xi_cur = 0;
}

typedef struct { double r, c, s; int j; double W[2], dW[2], Wor[2]; } pgeo_t;

/* src/PlasmaSpecies.cpp:57-70 */
static inline pgeo_t geometry(const grid_t* g, double x, double y) {
    pgeo_t p;
    p.r = sqrt(x * x + y * y);
    if (p.r > 0.0) { p.c = x / p.r; p.s = y / p.r; } else { p.c = 1.0; p.s = 0.0; }
    double t;
    grid_weights(g, p.r, &p.j, &t);
    const double ih = g->inv_h[p.j];
    p.W[0] = 1.0 - t; p.W[1] = t;
    p.dW[0] = -ih; p.dW[1] = ih;
    const double ir = p.r > 0.0 ? 1.0 / p.r : 0.0;
    p.Wor[0] = (p.j == 0) ? 0.0 : p.W[0] * ir;
    p.Wor[1] = (p.j == 0) ? ih : p.W[1] * ir;
    return p;
}
static inline double lin(const double* f, const pgeo_t* p) { return p->W[0] * f[p->j] + p->W[1] * f[p->j + 1]; }

/* src/SliceData.hpp:70-83 */
static inline double eval_scalar(double f0, double fr, double fi, double c, double s, int m1) {
    return m1 ? f0 + 2.0 * (fr * c - fi * s) : f0;
}
static inline void eval_vector(double r0, double i0, double r1, double i1, double r2, double i2, double c, double s,
                               int m1, double* vx, double* vy) {
    *vx = r1 * c - i1 * s;
    *vy = r1 * s + i1 * c;
    if (m1) {
        const double c2 = c * c - s * s, s2 = 2.0 * c * s;
        *vx += r0 + r2 * c2 - i2 * s2;
        *vy += i0 + r2 * s2 + i2 * c2;
    }
}

typedef struct { double Wx, Wy, Bx, By, Bz, Ez; } pfld_t;
/* src/PlasmaSpecies.cpp:75-89 (no laser) */
static inline pfld_t gather(const qzo_sim* s, const pgeo_t* p, int m1, int needB) {
    pfld_t o;
    eval_vector(lin(s->wp.r0, p), lin(s->wp.i0, p), lin(s->wp.r1, p), lin(s->wp.i1, p), lin(s->wp.r2, p),
                lin(s->wp.i2, p), p->c, p->s, m1, &o.Wx, &o.Wy);
    o.Ez = eval_scalar(lin(s->ez.a0, p), lin(s->ez.ar, p), lin(s->ez.ai, p), p->c, p->s, m1);
    o.Bz = eval_scalar(lin(s->bz.a0, p), lin(s->bz.ar, p), lin(s->bz.ai, p), p->c, p->s, m1);
    if (needB)
        eval_vector(lin(s->bp.r0, p), lin(s->bp.i0, p), lin(s->bp.r1, p), lin(s->bp.i1, p), lin(s->bp.r2, p),
                    lin(s->bp.i2, p), p->c, p->s, m1, &o.Bx, &o.By);
    else
        o.Bx = o.By = 0.0;
    return o;
}

/* src/PlasmaSpecies.cpp:409-478 */
static void species_deposit(qzo_sim* s, const species_t* q) {
    const grid_t* g = &s->fs.g;
    const double q0 = q->p.q, qm = q->p.q / q->p.m;
    const int neg = q->p.q < 0;
    const int m1 = s->m1;
    const double chif = 1.0;
    msc_t* dens = neg ? &s->ne : &s->ni;
    QZO_PFOR
    for (int i = 0; i < q->Np; ++i) {
        const double wi = q->w[i];
        if (wi == 0.0) continue;
        const double PX = q->px[i], PY = q->py[i], D = q->dl[i];
        const pgeo_t p = geometry(g, q->x[i], q->y[i]);
        const double A = 0.0;
        const double gam = (1.0 + PX * PX + PY * PY + A + D * D) / (2.0 * D);
        const double invd = 1.0 / D;
        const double pz = gam - D;
        const double ux = PX * invd, uy = PY * invd;
        const double ur = p.c * ux + p.s * uy, uth = p.c * uy - p.s * ux;
        const double wq = wi * q0;
        for (int cc = 0; cc < 2; ++cc) {
            const int jj = p.j + cc;
            const double iv = g->inv_V[jj];
            const double a = wq * p.W[cc] * iv;
            const double dr = wq * ur * p.dW[cc] * iv;
            const double vjz = a * pz * invd, vchi = chif * a * qm * invd, vrho = a * gam * invd;
            const double vn = wi * p.W[cc] * iv * gam * invd;
            QZO_ADD(s->rhot.a0[jj], a);
            QZO_ADD(s->drho.a0[jj], dr);
            QZO_ADD(s->jz.a0[jj], vjz);
            QZO_ADD(s->chi.a0[jj], vchi);
            QZO_ADD(s->rho.a0[jj], vrho);
            QZO_ADD(dens->a0[jj], vn);
            QZO_ADD(s->jp.r1[jj], a * ur);
            QZO_ADD(s->jp.i1[jj], a * uth);
            if (m1) {
                const double c = p.c, sn = p.s;
                QZO_ADD(s->rhot.ar[jj], a * c);
                QZO_ADD(s->rhot.ai[jj], -a * sn);
                const double th = wq * uth * p.Wor[cc] * iv;
                QZO_ADD(s->drho.ar[jj], dr * c - th * sn);
                QZO_ADD(s->drho.ai[jj], -dr * sn - th * c);
                QZO_ADD(s->jz.ar[jj], vjz * c);
                QZO_ADD(s->jz.ai[jj], -vjz * sn);
                QZO_ADD(s->chi.ar[jj], vchi * c);
                QZO_ADD(s->chi.ai[jj], -vchi * sn);
                QZO_ADD(s->rho.ar[jj], vrho * c);
                QZO_ADD(s->rho.ai[jj], -vrho * sn);
                QZO_ADD(dens->ar[jj], vn * c);
                QZO_ADD(dens->ai[jj], -vn * sn);
                QZO_ADD(s->jp.r0[jj], a * ux);
                QZO_ADD(s->jp.i0[jj], a * uy);
                const double c2 = c * c - sn * sn, s2 = 2.0 * c * sn;
                QZO_ADD(s->jp.r2[jj], a * (ux * c2 + uy * s2));
                QZO_ADD(s->jp.i2[jj], a * (uy * c2 - ux * s2));
            }
        }
    }
}

/* src/PlasmaSpecies.cpp:480-506 */
static void species_deposit_rho(qzo_sim* s, const species_t* q, msc_t* rhot, msc_t* rho) {
    const grid_t* g = &s->fs.g;
    const double q0 = q->p.q;
    for (int i = 0; i < q->Np; ++i) {
        const double wi = q->w[i];
        if (wi == 0.0) continue;
        const pgeo_t p = geometry(g, q->x[i], q->y[i]);
        for (int cc = 0; cc < 2; ++cc) {
            const int jj = p.j + cc;
            const double a = wi * q0 * p.W[cc] * g->inv_V[jj];
            rhot->a0[jj] += a;
            rho->a0[jj] += a;
            if (s->m1) {
                rhot->ar[jj] += a * p.c;
                rhot->ai[jj] += -a * p.s;
                rho->ar[jj] += a * p.c;
                rho->ai[jj] += -a * p.s;
            }
        }
    }
}

/* src/PlasmaSpecies.cpp:508-559 */
static void add_mode_S(const grid_t* g, const pgeo_t* p, int k, double* Sr, double* Si, double ck, double sk,
                       double wq, double ax, double ay, double ux, double uy, double ur, double uth) {
    for (int cc = 0; cc < 2; ++cc) {
        const int jj = p->j + cc;
        const double iv = g->inv_V[jj] * wq;
        double Ar = ax * p->W[cc] + ux * ur * p->dW[cc];
        double Ai = ay * p->W[cc] + uy * ur * p->dW[cc];
        if (k != 0) {
            const double f2 = k * uth * p->Wor[cc];
            Ar += f2 * uy;
            Ai -= f2 * ux;
        }
        QZO_ADD(Sr[jj], iv * (Ar * ck + Ai * sk));
        QZO_ADD(Si[jj], iv * (Ai * ck - Ar * sk));
    }
}

static void species_deposit_S(qzo_sim* s, const species_t* q) {
    if (!q->p.mobile) return;
    const grid_t* g = &s->fs.g;
    const double q0 = q->p.q, qm = q->p.q / q->p.m;
    const int m1 = s->m1;
    QZO_PFOR
    for (int i = 0; i < q->Np; ++i) {
        const double wi = q->w[i];
        if (wi == 0.0) continue;
        const double PX = q->px[i], PY = q->py[i], D = q->dl[i];
        const pgeo_t p = geometry(g, q->x[i], q->y[i]);
        const pfld_t F = gather(s, &p, m1, 0);
        const double gam = (1.0 + PX * PX + PY * PY + qm * qm * 0.0 + D * D) / (2.0 * D);
        const double invd = 1.0 / D;
        const double ux = PX * invd, uy = PY * invd;
        const double ur = p.c * ux + p.s * uy, uth = p.c * uy - p.s * ux;
        const double dD = qm * ((PX * F.Wx + PY * F.Wy) * invd - F.Ez);
        const double ax = (qm * (gam * F.Wx + PY * F.Bz) * invd) * invd - PX * dD * invd * invd;
        const double ay = (qm * (gam * F.Wy - PX * F.Bz) * invd) * invd - PY * dD * invd * invd;
        const double wq = wi * q0;
        add_mode_S(g, &p, 1, s->S.r1, s->S.i1, p.c, p.s, wq, ax, ay, ux, uy, ur, uth);
        if (m1) {
            add_mode_S(g, &p, 0, s->S.r0, s->S.i0, 1.0, 0.0, wq, ax, ay, ux, uy, ur, uth);
            add_mode_S(g, &p, 2, s->S.r2, s->S.i2, p.c * p.c - p.s * p.s, 2.0 * p.c * p.s, wq, ax, ay, ux, uy, ur, uth);
        }
    }
}

/* src/PlasmaSpecies.cpp:561-668 (no ionization, no trapping records, no laser) */
static void species_push(qzo_sim* s, species_t* q, double dxi) {
    if (!q->p.mobile) return;
    const int ord = s->p.ab_order;
    const int k = (int)(q->npush % ord);
    const int first = (q->npush == 0);
    if (first)
        for (int m = 0; m < ord; ++m) q->xi_slot[(k - m + ord) % ord] = q->xi_cur - m * dxi;
    else
        q->xi_slot[k] = q->xi_cur;
    double tn[5], ab[5];
    int uniform = 1;
    for (int m = 0; m < ord; ++m) {
        tn[m] = q->xi_slot[(k - m + ord) % ord];
        if (m > 0 && fabs((tn[m - 1] - tn[m]) - dxi) > 1e-9 * dxi) uniform = 0;
    }
    if (uniform) memcpy(ab, q->ab, sizeof(ab));
    else qzo_ab_variable(ord, tn, dxi, ab);
    ++q->npush;
    q->xi_cur += dxi;
    const grid_t* g = &s->fs.g;
    const double qm = q->p.q / q->p.m;
    const double dmin = s->p.delta_min, qsamax = s->p.max_qsa;
    const double R = g->R;
    const int m1 = s->m1;
    const int cap = q->cap;
    QZO_PFOR
    for (int i = 0; i < q->Np; ++i) {
        const double wi = q->w[i];
        if (wi == 0.0) continue;
        const double X = q->x[i], Y = q->y[i], PX = q->px[i], PY = q->py[i], D = q->dl[i];
        const pgeo_t p = geometry(g, X, Y);
        const pfld_t F = gather(s, &p, m1, 1);
        const double gam = (1.0 + PX * PX + PY * PY + qm * qm * 0.0 + D * D) / (2.0 * D);
        const double invd = 1.0 / D;
        double fv[5];
        fv[0] = PX * invd;
        fv[1] = PY * invd;
        fv[2] = qm * (gam * F.Wx * invd + F.By + PY * F.Bz * invd);
        fv[3] = qm * (gam * F.Wy * invd - F.Bx - PX * F.Bz * invd);
        fv[4] = qm * ((PX * F.Wx + PY * F.Wy) * invd - F.Ez);
#define H(sl, v) q->hist[((size_t)(sl) * 5 + (v)) * cap + i]
        if (first) {
            for (int sl = 0; sl < ord; ++sl)
                for (int v = 0; v < 5; ++v) H(sl, v) = fv[v];
        } else {
            for (int v = 0; v < 5; ++v) H(k, v) = fv[v];
        }
        double sum[5] = {0, 0, 0, 0, 0};
        for (int m = 0; m < ord; ++m) {
            const int sl = (k - m + ord) % ord;
            for (int v = 0; v < 5; ++v) sum[v] += ab[m] * H(sl, v);
        }
        double xn = X + dxi * sum[0], yn = Y + dxi * sum[1];
        double pxn = PX + dxi * sum[2], pyn = PY + dxi * sum[3];
        const double dn = D + dxi * sum[4];
        const double gn = (1.0 + pxn * pxn + pyn * pyn + dn * dn) / (2.0 * dn);
        if (!(dn > dmin) || gn > qsamax * dn) {
            q->w[i] = 0.0;
            QZO_ADD(s->lost, 1);
            continue;
        }
        const double rn = sqrt(xn * xn + yn * yn);
        if (rn > R) {
            const double nx = xn / rn, ny = yn / rn;
            const double rr = 2.0 * R - rn;
            if (rr < 0.0) { q->w[i] = 0.0; QZO_ADD(s->lost, 1); continue; }
            xn = nx * rr; yn = ny * rr;
            const double pn = pxn * nx + pyn * ny;
            pxn -= 2.0 * pn * nx; pyn -= 2.0 * pn * ny;
            for (int sl = 0; sl < ord; ++sl) {
                const double a = H(sl, 0) * nx + H(sl, 1) * ny;
                H(sl, 0) -= 2.0 * a * nx; H(sl, 1) -= 2.0 * a * ny;
                const double b = H(sl, 2) * nx + H(sl, 3) * ny;
                H(sl, 2) -= 2.0 * b * nx; H(sl, 3) -= 2.0 * b * ny;
            }
        }
#undef H
        q->x[i] = xn; q->y[i] = yn; q->px[i] = pxn; q->py[i] = pyn; q->dl[i] = dn;
    }
}

/* src/PlasmaSpecies.cpp:814-830: the most radial cells a particle would cross in a step of dxi, its
   straight path's length over the cell size at the path's closest approach to the axis */
static double species_max_cells(const qzo_sim* s, const species_t* q, double dxi) {
    if (!q->p.mobile || q->Np == 0) return 0.0;
    const grid_t* g = &s->fs.g;
    double mx = 0.0;
    for (int i = 0; i < q->Np; ++i) {
        if (q->w[i] == 0.0) continue;
        const double X = q->x[i], Y = q->y[i], D = q->dl[i];
        const double X1 = X + dxi * q->px[i] / D, Y1 = Y + dxi * q->py[i] / D;
        const double dx = X1 - X, dy = Y1 - Y, l2 = dx * dx + dy * dy;
        double t = l2 > 0.0 ? -(X * dx + Y * dy) / l2 : 0.0;
        t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
        const double xm = X + t * dx, ym = Y + t * dy;
        const double c = sqrt(l2) * g->inv_h[grid_locate(g, sqrt(xm * xm + ym * ym))];
        if (c > mx) mx = c;
    }
    return mx;
}

/* src/PlasmaSpecies.hpp:63: the last push's step */
static double species_last_step(const qzo_sim* s, const species_t* q) {
    const int ord = s->p.ab_order;
    return q->npush > 0 ? q->xi_cur - q->xi_slot[(q->npush - 1) % ord] : 0.0;
}

/* src/Simulation.cpp:837-847: sub-slices of the coming step */
static int subslices(const qzo_sim* s, double dxi) {
    if (!(s->p.max_cells > 0.0)) return 1;
    double c = 0.0, hlast = 0.0;
    for (int i = 0; i < s->nsp; ++i)
        if (s->sp[i].p.mobile) {
            const double ci = species_max_cells(s, &s->sp[i], dxi), hi = species_last_step(s, &s->sp[i]);
            if (ci > c) c = ci;
            if (hi > hlast) hlast = hi;
        }
    int n = c <= s->p.max_cells ? 1 : (int)ceil(c / s->p.max_cells);
    if (hlast > 0.0) {
        const int m = (int)ceil(dxi / (2.0 * hlast) - 1e-9);
        if (m > n) n = m;
    }
    const int nmax = s->p.substep_max > 0 ? s->p.substep_max : 64;
    return n < nmax ? n : nmax;
}

/* ---- slice steps (src/Simulation.cpp) ---- */
static void zero_sources(qzo_sim* s) {
    const int M = s->M;
    msc_t* sc[7] = {&s->rhot, &s->drho, &s->jz, &s->chi, &s->rho, &s->ne, &s->ni};
    for (int c = 0; c < 7; ++c) msc_zero(sc[c], M);
    mvec_zero(&s->jp, M);
    mvec_zero(&s->S, M);
}

#define BS(k, j, c) s->bsrc[((size_t)(k) * M + (j)) * bnc + (c)]
/* src/Simulation.cpp:408-457; ds != 0 (a sub-slice at xi_k + ds): the beam sources extrapolated linearly
   with their xi-derivative */
static void combine_sources(qzo_sim* s, int k, double ds) {
    const int M = s->M, KL = s->p.K, bnc = s->bnc;
    const double idxi = 1.0 / s->p.dxi;
    const int m1 = s->m1, ngp = s->p.ngp, sub = ds != 0.0;
    for (int j = 0; j < M; ++j) {
#define DXI_B(comp) ( ngp ? (BS(k, j, comp) - ((k > 0) ? BS(k - 1, j, comp) : s->bguard[15 * j + (comp)])) * idxi \
            : (KL == 1 ? 0.0 : (k == 0 ? (BS(1, j, comp) - BS(0, j, comp)) * idxi \
            : (k == KL - 1 ? (BS(KL - 1, j, comp) - BS(KL - 2, j, comp)) * idxi \
            : 0.5 * (BS(k + 1, j, comp) - BS(k - 1, j, comp)) * idxi))) )
#define BV(comp) (sub ? BS(k, j, comp) + ds * DXI_B(comp) : BS(k, j, comp))
        s->rhot.a0[j] += s->bg_rhot.a0[j] + BV(B_RT0);
        s->drho.a0[j] += DXI_B(B_RT0);
        s->jz.a0[j] += BV(B_JZ0);
        s->jp.r1[j] += BV(B_JP1R);
        s->jp.i1[j] += BV(B_JP1I);
        s->rho.a0[j] += s->bg_rho.a0[j] + BV(B_RHO0);
        if (s->bg_rho.a0[j] > 0.0) s->ni.a0[j] += s->bg_rho.a0[j];
        if (m1) {
            s->rhot.ar[j] += s->bg_rhot.ar[j] + BV(B_RT1R);
            s->rhot.ai[j] += s->bg_rhot.ai[j] + BV(B_RT1I);
            s->drho.ar[j] += DXI_B(B_RT1R);
            s->drho.ai[j] += DXI_B(B_RT1I);
            s->jz.ar[j] += BV(B_JZ1R);
            s->jz.ai[j] += BV(B_JZ1I);
            s->jp.r0[j] += BV(B_JP0R);
            s->jp.i0[j] += BV(B_JP0I);
            s->jp.r2[j] += BV(B_JP2R);
            s->jp.i2[j] += BV(B_JP2I);
            s->rho.ar[j] += s->bg_rho.ar[j] + BV(B_RHO1R);
            s->rho.ai[j] += s->bg_rho.ai[j] + BV(B_RHO1I);
        }
#undef BV
#undef DXI_B
    }
}
#undef BS

static void compute_wplus(qzo_sim* s) {
    const int M = s->M, m1 = s->m1;
    solver_gradient(&s->fs, s->psi.a0, s->t1);
    if (m1) {
        solver_gradient_odd(&s->fs, s->psi.ar, s->t2);
        solver_over_r(&s->fs, s->psi.ar, s->t3);
        solver_gradient_odd(&s->fs, s->psi.ai, s->t4);
        solver_over_r(&s->fs, s->psi.ai, s->rhs);
    }
    for (int j = 0; j < M; ++j) {
        s->wp.r1[j] = -s->t1[j];
        s->wp.i1[j] = 0.0;
        if (m1) {
            s->wp.r2[j] = -(s->t2[j] - s->t3[j]);
            s->wp.i2[j] = -(s->t4[j] - s->rhs[j]);
            s->wp.r0[j] = -(s->t2[j] + s->t3[j]);
            s->wp.i0[j] = (s->t4[j] + s->rhs[j]);
        }
    }
}

static void compute_bz(qzo_sim* s) {
    const int M = s->M, m1 = s->m1;
    mvec_t* g = &s->gz;
    solver_gradient_odd(&s->fs, s->jp.i1, s->t1);
    solver_over_r(&s->fs, s->jp.i1, s->t2);
    if (m1) {
        solver_gradient_odd(&s->fs, s->jp.r2, g->r0);
        solver_over_r(&s->fs, s->jp.r2, g->i0);
        solver_gradient_odd(&s->fs, s->jp.i2, g->r1);
        solver_over_r(&s->fs, s->jp.i2, g->i1);
        solver_gradient(&s->fs, s->jp.r0, g->r2);
        solver_gradient(&s->fs, s->jp.i0, g->i2);
    }
    for (int j = 0; j < M; ++j) {
        s->t3[j] = -(s->t1[j] + s->t2[j]);
        if (m1) {
            const double D1r = g->r0[j] + 2.0 * g->i0[j], D1i = g->r1[j] + 2.0 * g->i1[j];
            const double Dmr = g->r2[j], Dmi = g->i2[j];
            s->t4[j] = -0.5 * (D1i + Dmi);
            s->rhs[j] = 0.5 * (D1r - Dmr);
        }
    }
    solver_solve(&s->fs, OP_L0, s->t3, s->bz.a0, NULL, NULL, 1.0);
    if (m1) {
        solver_solve(&s->fs, OP_L1D, s->t4, s->bz.ar, NULL, NULL, 1.0);
        solver_solve(&s->fs, OP_L1D, s->rhs, s->bz.ai, NULL, NULL, 1.0);
    }
}

static void solve_bplus(qzo_sim* s) {
    const int M = s->M, m1 = s->m1;
    mvec_t* g = &s->gz;
    solver_gradient(&s->fs, s->jz.a0, s->t1);
    if (m1) {
        solver_gradient_odd(&s->fs, s->jz.ar, s->t2);
        solver_over_r(&s->fs, s->jz.ar, s->t3);
        solver_gradient_odd(&s->fs, s->jz.ai, s->t4);
        solver_over_r(&s->fs, s->jz.ai, s->rhs);
    }
    for (int j = 0; j < M; ++j) {
        g->r1[j] = s->t1[j] + s->S.r1[j];
        g->i1[j] = s->S.i1[j];
        if (m1) {
            g->r2[j] = (s->t2[j] - s->t3[j]) + s->S.r2[j];
            g->i2[j] = (s->t4[j] - s->rhs[j]) + s->S.i2[j];
            g->r0[j] = (s->t2[j] + s->t3[j]) + s->S.r0[j];
            g->i0[j] = -(s->t4[j] + s->rhs[j]) + s->S.i0[j];
        }
    }
    mvec_t* rb = &s->bprev;
    const int niter = m1 ? s->p.picard : 1;
    for (int it = 0; it < niter; ++it) {
        for (int j = 0; j < M; ++j) {
            double r1 = -g->i1[j], i1 = g->r1[j];
            if (m1) {
                double r0 = -g->i0[j], i0 = g->r0[j], r2 = -g->i2[j], i2 = g->r2[j];
                const double cr = s->chi.ar[j], ci = s->chi.ai[j];
                const double b0r = s->bp.r0[j], b0i = s->bp.i0[j], b1r = s->bp.r1[j], b1i = s->bp.i1[j];
                const double b2r = s->bp.r2[j], b2i = s->bp.i2[j];
                r0 += cr * b1r + ci * b1i;  i0 += cr * b1i - ci * b1r;
                r1 += cr * b0r - ci * b0i + cr * b2r + ci * b2i;
                i1 += cr * b0i + ci * b0r + cr * b2i - ci * b2r;
                r2 += cr * b1r - ci * b1i;  i2 += cr * b1i + ci * b1r;
                rb->r0[j] = r0; rb->i0[j] = i0; rb->r2[j] = r2; rb->i2[j] = i2;
            }
            rb->r1[j] = r1; rb->i1[j] = i1;
        }
        solver_solve(&s->fs, OP_L1D, rb->r1, s->bp.r1, s->chi.a0, NULL, 1.0);
        solver_solve(&s->fs, OP_L1F, rb->i1, s->bp.i1, s->chi.a0, s->jz.a0, 1.0);
        if (m1) {
            solver_solve(&s->fs, OP_L0, rb->r0, s->bp.r0, s->chi.a0, NULL, 1.0);
            solver_solve(&s->fs, OP_L0, rb->i0, s->bp.i0, s->chi.a0, NULL, 1.0);
            solver_solve(&s->fs, OP_L2D, rb->r2, s->bp.r2, s->chi.a0, NULL, 1.0);
            solver_solve(&s->fs, OP_L2D, rb->i2, s->bp.i2, s->chi.a0, NULL, 1.0);
        }
    }
}

static void store_slice(qzo_sim* s, int k) {
    const int M = s->M, m1 = s->m1, fnc = s->fnc, dnc = s->dnc;
    for (int j = 0; j < M; ++j) {
        double* F = s->fld + ((size_t)k * M + j) * fnc;
        double* D = s->diag + ((size_t)k * M + j) * dnc;
        F[F_EP1R] = s->wp.r1[j] + s->bp.i1[j];
        F[F_EP1I] = s->wp.i1[j] - s->bp.r1[j];
        F[F_BP1R] = s->bp.r1[j];
        F[F_BP1I] = s->bp.i1[j];
        F[F_EZ0] = s->ez.a0[j];
        F[F_BZ0] = s->bz.a0[j];
        D[D_PSI0] = s->psi.a0[j];
        D[D_NE0] = s->ne.a0[j];
        D[D_NI0] = s->ni.a0[j];
        if (m1) {
            F[F_EP0R] = s->wp.r0[j] + s->bp.i0[j];
            F[F_EP0I] = s->wp.i0[j] - s->bp.r0[j];
            F[F_EP2R] = s->wp.r2[j] + s->bp.i2[j];
            F[F_EP2I] = s->wp.i2[j] - s->bp.r2[j];
            F[F_BP0R] = s->bp.r0[j];
            F[F_BP0I] = s->bp.i0[j];
            F[F_BP2R] = s->bp.r2[j];
            F[F_BP2I] = s->bp.i2[j];
            F[F_EZ1R] = s->ez.ar[j];
            F[F_EZ1I] = s->ez.ai[j];
            F[F_BZ1R] = s->bz.ar[j];
            F[F_BZ1I] = s->bz.ai[j];
            D[D_PSI1R] = s->psi.ar[j];
            D[D_PSI1I] = s->psi.ai[j];
            D[D_NE1R] = s->ne.ar[j];
            D[D_NE1I] = s->ne.ai[j];
            D[D_NI1R] = s->ni.ar[j];
            D[D_NI1I] = s->ni.ai[j];
        }
    }
}

static void solve_slice_fields(qzo_sim* s) {
    solver_solve(&s->fs, OP_L0, s->rhot.a0, s->psi.a0, NULL, NULL, -1.0);
    solver_solve(&s->fs, OP_L0, s->drho.a0, s->ez.a0, NULL, NULL, -1.0);
    if (s->m1) {
        solver_solve(&s->fs, OP_L1D, s->rhot.ar, s->psi.ar, NULL, NULL, -1.0);
        solver_solve(&s->fs, OP_L1D, s->rhot.ai, s->psi.ai, NULL, NULL, -1.0);
        solver_solve(&s->fs, OP_L1D, s->drho.ar, s->ez.ar, NULL, NULL, -1.0);
        solver_solve(&s->fs, OP_L1D, s->drho.ai, s->ez.ai, NULL, NULL, -1.0);
    }
    compute_wplus(s);
    compute_bz(s);
    for (int i = 0; i < s->nsp; ++i)
        if (s->sp[i].p.mobile) species_deposit_S(s, &s->sp[i]);
    if (s->fs.filter_on) {   /* src/Simulation.cpp:810-816 */
        solver_filter(&s->fs, 1, s->S.r1); solver_filter(&s->fs, 1, s->S.i1);
        if (s->m1) {
            solver_filter(&s->fs, 0, s->S.r0); solver_filter(&s->fs, 0, s->S.i0);
            solver_filter(&s->fs, 2, s->S.r2); solver_filter(&s->fs, 2, s->S.i2);
        }
    }
    solve_bplus(s);
}

/* ---- beams ---- */
/* src/Beam.cpp:725-785 */
static void beam_deposit(qzo_sim* s, const beam_t* B) {
    const grid_t* g = &s->fs.g;
    const int M = s->M, bnc = s->bnc, m1 = s->m1, ngp = s->p.ngp;
    const double q = B->q;
    const double xmin = s->p.xi_min, idxi = 1.0 / s->p.dxi;
    const int k0 = 0, nloc = s->p.K;
    const double R = g->R;
    QZO_PFOR
    for (long i = 0; i < B->n; ++i) {
        const double wi = B->w[i];
        if (wi == 0.0) continue;
        const double X = B->x[i], Y = B->y[i];
        const double r = sqrt(X * X + Y * Y);
        if (r > R) continue;
        const double c = r > 0.0 ? X / r : 1.0, sn = r > 0.0 ? Y / r : 0.0;
        const double sx = (B->xi[i] - xmin) * idxi;
        const int k = ngp ? (int)floor(sx + 0.5) : (int)floor(sx);
        if (k < k0 - 1 || k >= k0 + nloc) continue;
        const double tk = ngp ? 0.0 : sx - k;
        const double PX = B->px[i], PY = B->py[i], PZ = B->pz[i];
        const double p2 = PX * PX + PY * PY;
        const double gam = sqrt(1.0 + p2 + PZ * PZ);
        const double omvz = (1.0 + p2) / (gam * (gam + PZ));
        const double vz = PZ / gam, vx = PX / gam, vy = PY / gam;
        const double vr = c * vx + sn * vy, vt = c * vy - sn * vx;
        int j; double t;
        grid_weights(g, r, &j, &t);
        const double Wr[2] = {1.0 - t, t};
        const double Wk[2] = {1.0 - tk, tk};
        for (int a = 0; a < (ngp ? 1 : 2); ++a) {
            const int kk = k + a - k0;
            if (kk < 0 || kk >= nloc) continue;
            for (int b = 0; b < 2; ++b) {
                const int jj = j + b;
                double* o = s->bsrc + ((size_t)kk * M + jj) * bnc;
                const double d = wi * q * Wk[a] * Wr[b] * g->inv_V[jj] * idxi;
                QZO_ADD(o[B_RT0], d * omvz);
                QZO_ADD(o[B_JZ0], d * vz);
                QZO_ADD(o[B_JP1R], d * vr);
                QZO_ADD(o[B_JP1I], d * vt);
                QZO_ADD(o[B_RHO0], d);
                if (m1) {
                    QZO_ADD(o[B_RT1R], d * omvz * c);
                    QZO_ADD(o[B_RT1I], -d * omvz * sn);
                    QZO_ADD(o[B_JZ1R], d * vz * c);
                    QZO_ADD(o[B_JZ1I], -d * vz * sn);
                    QZO_ADD(o[B_RHO1R], d * c);
                    QZO_ADD(o[B_RHO1I], -d * sn);
                    QZO_ADD(o[B_JP0R], d * vx);
                    QZO_ADD(o[B_JP0I], d * vy);
                    const double c2 = c * c - sn * sn, s2 = 2.0 * c * sn;
                    QZO_ADD(o[B_JP2R], d * (vx * c2 + vy * s2));
                    QZO_ADD(o[B_JP2I], d * (vy * c2 - vx * s2));
                }
            }
        }
    }
}

/* src/Beam.cpp:948-1131: gather + Vay + drift (no laser, spin, scattering or radiation) */
static void beam_advance(qzo_sim* s, beam_t* B, double dt_kick, double dt, int move) {
    const grid_t* g = &s->fs.g;
    const int M = s->M, fnc = s->fnc, m1 = s->m1, ngp = s->p.ngp;
    const double qm = B->q / B->m;
    const double xmin = s->p.xi_min, idxi = 1.0 / s->p.dxi;
    const double xmax = s->p.xi_min + (s->p.K - 1) * s->p.dxi;
    const int k0 = 0, nloc = s->p.K;
    const double R = g->R;
    const double* fld = s->fld;
    QZO_PFOR
    for (long i = 0; i < B->n; ++i) {
        if (B->w[i] == 0.0) continue;
        const double X = B->x[i], Y = B->y[i];
        const double r = sqrt(X * X + Y * Y);
        const double c = r > 0.0 ? X / r : 1.0, sn = r > 0.0 ? Y / r : 0.0;
        double sl = (B->xi[i] - xmin) * idxi - k0;
        int k;
        double tk;
        if (ngp) {
            k = (int)floor(sl + 0.5);
            k = k < 0 ? 0 : (k > nloc - 1 ? nloc - 1 : k);
            tk = 0.0;
        } else {
            k = (int)floor(sl);
            if (k < 0) { k = 0; sl = 0; }
            if (k > nloc - 2) { k = nloc - 2; sl = nloc - 1; }
            tk = sl - k;
        }
        const int k1 = ngp ? k : k + 1;
        int j; double t;
        grid_weights(g, r, &j, &t);
#define FL(kk, jj, comp) fld[((size_t)(kk) * M + (jj)) * fnc + (comp)]
#define BIL(comp) ((1.0 - tk) * ((1.0 - t) * FL(k, j, comp) + t * FL(k, j + 1, comp)) + \
                   tk * ((1.0 - t) * FL(k1, j, comp) + t * FL(k1, j + 1, comp)))
        double Ex, Ey, Bx, By, Ez, Bz;
        if (m1) {
            eval_vector(BIL(F_EP0R), BIL(F_EP0I), BIL(F_EP1R), BIL(F_EP1I), BIL(F_EP2R), BIL(F_EP2I), c, sn, 1, &Ex, &Ey);
            eval_vector(BIL(F_BP0R), BIL(F_BP0I), BIL(F_BP1R), BIL(F_BP1I), BIL(F_BP2R), BIL(F_BP2I), c, sn, 1, &Bx, &By);
            Ez = eval_scalar(BIL(F_EZ0), BIL(F_EZ1R), BIL(F_EZ1I), c, sn, 1);
            Bz = eval_scalar(BIL(F_BZ0), BIL(F_BZ1R), BIL(F_BZ1I), c, sn, 1);
        } else {
            eval_vector(0.0, 0.0, BIL(F_EP1R), BIL(F_EP1I), 0.0, 0.0, c, sn, 0, &Ex, &Ey);
            eval_vector(0.0, 0.0, BIL(F_BP1R), BIL(F_BP1I), 0.0, 0.0, c, sn, 0, &Bx, &By);
            Ez = BIL(F_EZ0);
            Bz = BIL(F_BZ0);
        }
#undef BIL
#undef FL
        const v3 E = {Ex, Ey, Ez}, Bf = {Bx, By, Bz};
        v3 u = {B->px[i], B->py[i], B->pz[i]};
        const double h = 0.5 * qm * dt_kick;
        if (!move) {
            const double g0 = sqrt(1.0 + v3dot(u, u));
            u = v3add(u, v3mul(2.0 * h, v3add(E, v3cross(v3mul(1.0 / g0, u), Bf))));
            B->px[i] = u.x; B->py[i] = u.y; B->pz[i] = u.z;
            continue;
        }
        u = push_u(B->pusher, u, E, Bf, h);
        const double p2 = u.x * u.x + u.y * u.y;
        const double gam = sqrt(1.0 + p2 + u.z * u.z);
        const double omvz = (1.0 + p2) / (gam * (gam + u.z));
        const double xn = X + u.x / gam * dt, yn = Y + u.y / gam * dt;
        B->x[i] = xn; B->y[i] = yn;
        B->px[i] = u.x; B->py[i] = u.y; B->pz[i] = u.z;
        B->xi[i] += omvz * dt;
        if (xn * xn + yn * yn >= R * R || B->xi[i] < xmin || B->xi[i] > xmax) B->w[i] = 0.0;
    }
}

int qzo_sim_deposit_beams(qzo_sim* s) {
    memset(s->bsrc, 0, sizeof(double) * (size_t)s->p.K * s->M * s->bnc);
    for (int b = 0; b < s->nb; ++b) {
        if (s->bm[b].analytic) deposit_analytic(s, &s->bm[b]);
        else beam_deposit(s, &s->bm[b]);
    }
    return 0;
}

/* Simulation::filter_plasma_sources (src/Simulation.cpp:821-835): the plasma deposit of the slice, before
   the beams and the background are added */
static void filter_plasma_sources(qzo_sim* s) {
    if (!s->fs.filter_on) return;
    msc_t* sc[7] = {&s->rhot, &s->drho, &s->jz, &s->chi, &s->rho, &s->ne, &s->ni};
    for (int c = 0; c < 7; ++c) {
        solver_filter(&s->fs, 0, sc[c]->a0);
        if (s->m1) { solver_filter(&s->fs, 1, sc[c]->ar); solver_filter(&s->fs, 1, sc[c]->ai); }
    }
    solver_filter(&s->fs, 1, s->jp.r1);
    solver_filter(&s->fs, 1, s->jp.i1);
    if (s->m1) {
        solver_filter(&s->fs, 0, s->jp.r0); solver_filter(&s->fs, 0, s->jp.i0);
        solver_filter(&s->fs, 2, s->jp.r2); solver_filter(&s->fs, 2, s->jp.i2);
    }
}

/* src/Simulation.cpp:636-795 (single rank: bguard = 0, B+ starts at 0, one sub-slice) */
int qzo_sim_step_fields(qzo_sim* s, double t) {
    (void)t;
    const int M = s->M, K = s->p.K;
    qzo_sim_deposit_beams(s);
    msc_zero(&s->bg_rhot, M);
    msc_zero(&s->bg_rho, M);
    for (int i = 0; i < s->nsp; ++i) species_load(s, &s->sp[i]);
    for (int i = 0; i < s->nsp; ++i)
        if (!s->sp[i].p.mobile) species_deposit_rho(s, &s->sp[i], &s->bg_rhot, &s->bg_rho);
    if (s->p.neutralize) {
        msc_zero(&s->rhot, M);
        msc_zero(&s->rho, M);
        for (int i = 0; i < s->nsp; ++i)
            if (s->sp[i].p.mobile) species_deposit_rho(s, &s->sp[i], &s->rhot, &s->rho);
        for (int j = 0; j < M; ++j) {
            s->bg_rhot.a0[j] -= s->rhot.a0[j]; s->bg_rhot.ar[j] -= s->rhot.ar[j]; s->bg_rhot.ai[j] -= s->rhot.ai[j];
            s->bg_rho.a0[j] -= s->rho.a0[j]; s->bg_rho.ar[j] -= s->rho.ar[j]; s->bg_rho.ai[j] -= s->rho.ai[j];
        }
    }
    if (s->fs.filter_on)   /* src/Simulation.cpp:685-690 */
        for (int c = 0; c < 2; ++c) {
            msc_t* m = c == 0 ? &s->bg_rhot : &s->bg_rho;
            solver_filter(&s->fs, 0, m->a0);
            if (s->m1) { solver_filter(&s->fs, 1, m->ar); solver_filter(&s->fs, 1, m->ai); }
        }
    mvec_zero(&s->bp, M);
    memset(s->bguard, 0, sizeof(double) * 15 * M);
    const double dxi = s->p.dxi;
    for (int k = 0; k < K; ++k) {
        if (s->traj)
            for (int i = 0; i < s->nsp; ++i)
                if (s->sp[i].p.mobile) {
                    const species_t* q = &s->sp[i];
                    const size_t cap = (size_t)q->cap, nv = 6 + 5 * (size_t)s->p.ab_order;
                    double* o = s->traj + (size_t)k * nv * cap;
                    const double* cols[6] = {q->x, q->y, q->px, q->py, q->dl, q->w};
                    for (int c = 0; c < 6; ++c) memcpy(o + c * cap, cols[c], sizeof(double) * cap);
                    memcpy(o + 6 * cap, q->hist, sizeof(double) * (nv - 6) * cap);
                    break;
                }
        zero_sources(s);
        for (int i = 0; i < s->nsp; ++i)
            if (s->sp[i].p.mobile) species_deposit(s, &s->sp[i]);
        filter_plasma_sources(s);
        combine_sources(s, k, 0.0);
        solve_slice_fields(s);
        store_slice(s, k);
        if (k < K - 1) {
            /* src/Simulation.cpp:755-781: adaptive sub-slicing, each sub-slice with its own deposit and
               field solve (the beam sources extrapolated from this slice); only the slices are stored */
            const int nsub = subslices(s, dxi);
            const double h = dxi / nsub;
            for (int ss = 0; ss < nsub; ++ss) {
                if (ss > 0) {
                    zero_sources(s);
                    for (int i = 0; i < s->nsp; ++i)
                        if (s->sp[i].p.mobile) species_deposit(s, &s->sp[i]);
                    filter_plasma_sources(s);
                    combine_sources(s, k, ss * h);
                    solve_slice_fields(s);
                }
                for (int i = 0; i < s->nsp; ++i)
                    if (s->sp[i].p.mobile) species_push(s, &s->sp[i], h);
            }
            s->nsub_extra += nsub - 1;
        }
    }
    return 0;
}

long qzo_sim_subslices(const qzo_sim* s) { return s->nsub_extra; }

/* src/Beam.cpp:900-905 */
int qzo_sim_push_beams(qzo_sim* s, double dt_kick, double dt_drift) {
    for (int b = 0; b < s->nb; ++b) {
        beam_t* B = &s->bm[b];
        if (B->rigid) continue;
        if (!B->started) { beam_advance(s, B, -0.5 * dt_kick, -0.5 * dt_kick, 0); B->started = 1; }
        beam_advance(s, B, dt_kick, dt_drift, 1);
    }
    return 0;
}

/* src/Beam.cpp:1133-1155 */
int qzo_sim_beam_sums(const qzo_sim* s, int b, double S[17]) {
    if (b < 0 || b >= s->nb) return -1;
    const beam_t* B = &s->bm[b];
    for (int c = 0; c < 17; ++c) S[c] = 0;
#ifdef _OPENMP
#pragma omp parallel for reduction(+ : S[:17])
#endif
    for (long i = 0; i < B->n; ++i) {
        const double w = B->w[i];
        if (w == 0) continue;
        S[16] += 1;
        const double g = sqrt(1 + B->px[i] * B->px[i] + B->py[i] * B->py[i] + B->pz[i] * B->pz[i]);
        const double X = B->x[i], Y = B->y[i], PX = B->px[i], PY = B->py[i];
        const double G = g - B->gref, XI = B->xi[i] - B->xiref;
        const double v[15] = {G, G * G, XI, XI * XI, X * X + Y * Y, X, Y, X * X, Y * Y, PX, PY, PX * PX, PY * PY,
                              X * PX, Y * PY};
        S[0] += w;
        for (int c = 0; c < 15; ++c) S[c + 1] += w * v[c];
    }
    return 0;
}

/* src/Beam.cpp:1195-1217: per-bin sums over [lo, hi) of the USER xi (= -internal xi), nbins bins, 9 per bin:
   w, w x, w y, w x^2, w y^2, w gamma, w px, w px^2, w x px */
int qzo_slice_sums(const double* p7, long n, double lo, double hi, int nbins, double* out) {
    if (nbins < 1 || !(hi > lo)) return -1;
    for (long c = 0; c < 9L * nbins; ++c) out[c] = 0.0;
    const double db = (hi - lo) / nbins;
    for (long i = 0; i < n; ++i) {
        const double* p = p7 + 7 * i;
        const double w = p[6];
        if (w == 0) continue;
        const int b = (int)floor(((0.0 - p[5]) - lo) / db);
        if (b < 0 || b >= nbins) continue;
        const double g = sqrt(1 + p[2] * p[2] + p[3] * p[3] + p[4] * p[4]);
        const double v[9] = {1.0, p[0], p[1], p[0] * p[0], p[1] * p[1], g, p[2], p[2] * p[2], p[0] * p[2]};
        for (int c = 0; c < 9; ++c) out[9 * b + c] += w * v[c];
    }
    return 0;
}

int qzo_sim_beam_get(const qzo_sim* s, int b, double* p7) {
    if (b < 0 || b >= s->nb) return -1;
    const beam_t* B = &s->bm[b];
    const double* cols[7] = {B->x, B->y, B->px, B->py, B->pz, B->xi, B->w};
    for (long i = 0; i < B->n; ++i)
        for (int c = 0; c < 7; ++c) p7[7 * i + c] = cols[c][i];
    return 0;
}

long qzo_sim_beam_count(const qzo_sim* s, int b) { return (b >= 0 && b < s->nb) ? s->bm[b].n : -1; }
const double* qzo_sim_fld(const qzo_sim* s) { return s->fld; }
const double* qzo_sim_bsrc(const qzo_sim* s) { return s->bsrc; }
const double* qzo_sim_diag(const qzo_sim* s) { return s->diag; }
long qzo_sim_lost(const qzo_sim* s) { return s->lost; }

int qzo_sim_plasma_get(const qzo_sim* s, int sp, double* out6, int cap) {
    if (sp < 0 || sp >= s->nsp) return -1;
    const species_t* q = &s->sp[sp];
    if (q->Np > cap) return -q->Np;
    const double* cols[6] = {q->x, q->y, q->px, q->py, q->dl, q->w};
    for (int c = 0; c < 6; ++c) memcpy(out6 + (size_t)c * q->Np, cols[c], sizeof(double) * q->Np);
    return q->Np;
}

/* src/Simulation.cpp:1370-1448 (constant dt) */
int qzo_sim_run(qzo_sim* s, int nsteps, double dt, double* mom) {
    double t = 0.0, dt_prev = dt;
    for (int n = 0; n <= nsteps; ++n) {
        qzo_sim_step_fields(s, t);
        if (mom)
            for (int b = 0; b < s->nb; ++b) qzo_sim_beam_sums(s, b, mom + ((size_t)n * s->nb + b) * 17);
        if (n < nsteps) {
            const double dkick = 0.5 * (dt_prev + dt), ddrift = dt;
            qzo_sim_push_beams(s, dkick, ddrift);
            t += dt;
            dt_prev = dt;
        }
    }
    return 0;
}

/* src/Beam.cpp:483-570 (gaussian longitudinal profile; flattop when sxi <= 0 uses len = -sxi) */
long qzo_sample_gaussian(double n0, double sr, double xi0, double sxi, double gamma0, double espread, double emit,
                         double cut, double cx0, double cy0, double cxs, double cys, double xp0, double yp0, long np,
                         int nrot, int mirror, uint64_t seed, double xcut, double* out, double* gref,
                         double* xiref) {
    const int flat = !(sxi > 0);
    const double len = flat ? -sxi : 0.0;
    const int nsym = nrot * (mirror ? 2 : 1);
    if (nrot < 1 || np % nsym != 0) return -1;
    const double Pr = 1.0 - exp(-0.5 * cut * cut);
#define PHI(x) (0.5 * (1.0 + erf((x) / sqrt(2.0))))
    double wtot;
    if (!flat) {
        const double lo0 = (xcut - xi0) / sxi;
        const double lo = -cut > lo0 ? -cut : lo0;
        if (lo >= cut) return -2;
        wtot = n0 * pow(2 * PI, 1.5) * sr * sr * sxi * Pr * (PHI(cut) - PHI(lo));
    } else {
        const double lo = (xi0 - 0.5 * len) > xcut ? (xi0 - 0.5 * len) : xcut, hi = xi0 + 0.5 * len;
        if (lo >= hi) return -2;
        wtot = n0 * 2 * PI * sr * sr * Pr * (hi - lo);
    }
#undef PHI
    const double wmac = wtot / np;
    qzo_rng rng;
    qzo_rng_seed(&rng, seed);
    const double spx = (sr > 0) ? emit / sr : 0.0;
    double aw = 0, awg = 0, awxi = 0;
    long n = 0;
    for (long i0 = 0; i0 < np; i0 += nsym) {
        double x, y;
        do { x = sr * qzo_rng_normal(&rng); y = sr * qzo_rng_normal(&rng); } while (x * x + y * y > cut * cut * sr * sr);
        double xi;
        do {
            if (!flat) {
                do { xi = qzo_rng_normal(&rng); } while (fabs(xi) > cut);
                xi = xi0 + sxi * xi;
            } else {
                xi = xi0 + len * (qzo_rng_canonical(&rng) * (1.0 - 0.0) + 0.0 - 0.5);
            }
        } while (xi < xcut);
        double px = spx * qzo_rng_normal(&rng), py = spx * qzo_rng_normal(&rng);
        const double gam = gamma0 * (1.0 + espread * qzo_rng_normal(&rng));
        px += gam * xp0;
        py += gam * yp0;
        const double pz2 = gam * gam - 1.0 - px * px - py * py;
        if (pz2 <= 0) return -3;
        const double tpx = px - gam * xp0, tpy = py - gam * yp0;
        for (int l = 0; l < nsym; ++l) {
            const int lr = l % nrot;
            const double sgn = (l >= nrot) ? -1.0 : 1.0;
            const double ph = 2 * PI * lr / nrot, cp = cos(ph), sp = sin(ph);
            double* q = out + 7 * n;
            q[0] = cp * x - sp * y + cx0 + cxs * (xi - xi0);
            q[1] = sgn * (sp * x + cp * y) + cy0 + cys * (xi - xi0);
            q[2] = cp * tpx - sp * tpy + gam * xp0;
            q[3] = sgn * (sp * tpx + cp * tpy) + gam * yp0;
            q[4] = sqrt(pz2);
            q[5] = xi;
            q[6] = wmac;
            if (q[6] != 0) {
                const double g = sqrt(1 + q[2] * q[2] + q[3] * q[3] + q[4] * q[4]);
                aw += q[6];
                awg += q[6] * g;
                awxi += q[6] * q[5];
            }
            ++n;
        }
    }
    *gref = 0; *xiref = 0;
    if (aw > 0) { *gref = awg / aw; *xiref = awxi / aw; }
    return n;
}
