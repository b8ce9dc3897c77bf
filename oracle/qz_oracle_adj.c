/* qz_oracle_adj.c -- the hand-written adjoint (reverse mode) of the m = 0 run: the FP64 reference
 * gradient that the CUDA adjoint is checked against.
 *
 * TEST INFRASTRUCTURE, like the rest of oracle/ (see qz_oracle.h). The reference has no
 * gradients; this file differentiates the forward restatement of qz_oracle.c exactly, running its
 * discrete operations in reverse order, and the tests pin it against central finite differences of
 * that forward. It is compiled as one translation unit with the forward (it includes qz_oracle.c),
 * so that it uses the same grid, geometry, gather and solver helpers.
 *
 * What it differentiates (QUARZ file:line of the forward steps, in reverse order):
 *   beam moment sums         src/Beam.cpp:1133-1155
 *   beam push                src/Beam.cpp:900-905 (start-up half kick), :948-1131 (gather, Vay, drift)
 *   Vay                      src/Pushers.hpp:36-68
 *   slice store              src/Simulation.cpp:594-633
 *   plasma push (AB, wall)   src/PlasmaSpecies.cpp:561-668
 *   B+ solves with chi       src/Simulation.cpp:535-591, src/FieldSolver.cpp:172-191
 *   S deposit                src/PlasmaSpecies.cpp:508-559
 *   B_z, W+, psi, E_z        src/Simulation.cpp:477-532, :797-819
 *   combine sources          src/Simulation.cpp:408-457
 *   plasma deposit           src/PlasmaSpecies.cpp:409-478
 *   beam deposit             src/Beam.cpp:725-785
 *
 * Scope: modes = 0, linear or nearest-grid-point beam shape in xi, one mobile plasma species
 * (immobile ones only add a constant background), constant AB coefficients, constant dt. Particle
 * removal, cell changes, clamps and the nearest-slice choice are piecewise constant, so their
 * derivative is taken as zero.
 *
 * Storage: the beams of every step are kept; the sweep of step n is recomputed in the reverse pass
 * from the beams of step n, recording the plasma state at the start of every slice.
 */
#include "qz_oracle.c"

/* ------------------------------------------------------------------ linear-algebra transposes */
/* A^T mu = lam for the tridiagonal A = (a, bw, c) that solver_solve builds for operator op (with
   chi on the non-Dirichlet rows); returns mu, and whether row j is Dirichlet in dir[] */
static void solve_T(solver_t* s, int op, const double* chi, const double* lam, double* mu, int* dir) {
    const op_t* o = &s->L[op];
    const int N = s->g.N, M = N + 1;
    double* at = (double*)malloc(sizeof(double) * M);
    double* ct = (double*)malloc(sizeof(double) * M);
    double* bw = (double*)malloc(sizeof(double) * M);
    double* cp = (double*)malloc(sizeof(double) * M);
    double* dp = (double*)malloc(sizeof(double) * M);
    for (int j = 0; j <= N; ++j) {
        dir[j] = (j == N && !o->flux) || (j == 0 && !o->regular);
        bw[j] = (dir[j] || !chi) ? o->b[j] : o->b[j] - chi[j];
        at[j] = j > 0 ? o->c[j - 1] : 0.0;      /* row j of A^T: c_{j-1}, b_j, a_{j+1} */
        ct[j] = j < N ? o->a[j + 1] : 0.0;
    }
    thomas(M, at, bw, ct, lam, mu, cp, dp);
    free(at); free(ct); free(bw); free(cp); free(dp);
}

/* the smoothing filter in reverse: lam <- F_n^-T lam in place (solver_filter builds x = F_n^-1 f with
   every row of F_n, identity rows included, so the transpose is the transposed Thomas solve) */
static void filter_T(solver_t* s, int n, double* lam) {
    if (!s->filter_on) return;
    const op_t* o = &s->F[n];
    const int N = s->g.N, M = N + 1;
    double* at = (double*)malloc(sizeof(double) * M);
    double* ct = (double*)malloc(sizeof(double) * M);
    double* mu = (double*)malloc(sizeof(double) * M);
    double* cp = (double*)malloc(sizeof(double) * M);
    double* dp = (double*)malloc(sizeof(double) * M);
    for (int j = 0; j <= N; ++j) {
        at[j] = j > 0 ? o->c[j - 1] : 0.0;
        ct[j] = j < N ? o->a[j + 1] : 0.0;
    }
    thomas(M, at, o->b, ct, lam, mu, cp, dp);
    memcpy(lam, mu, sizeof(double) * M);
    free(at); free(ct); free(mu); free(cp); free(dp);
}

/* lam_f += grad^T lam_df (solver_gradient) */
static void gradient_T(const solver_t* s, const double* ldf, double* lf) {
    const int N = s->g.N;
    for (int j = 1; j < N; ++j) {
        lf[j - 1] += s->gm[j] * ldf[j];
        lf[j] += s->g0[j] * ldf[j];
        lf[j + 1] += s->gp[j] * ldf[j];
    }
    lf[N] += s->g0[N] * ldf[N];
    lf[N - 1] += s->gm[N] * ldf[N];
    lf[N - 2] += s->gp[N] * ldf[N];
}
/* lam_f += grad_odd^T lam_df */
static void gradient_odd_T(const solver_t* s, const double* ldf, double* lf) {
    gradient_T(s, ldf, lf);                 /* identical except row 0 */
    lf[1] += s->ir[0] * ldf[0];
}
/* lam_f += over_r^T lam_out */
static void over_r_T(const solver_t* s, const double* lo, double* lf) {
    const int N = s->g.N;
    lf[1] += s->ir[0] * lo[0];
    for (int j = 1; j <= N; ++j) lf[j] += s->ir[j] * lo[j];
}

/* ------------------------------------------------------------------ geometry adjoint */
/* the adjoints of the geometry outputs a particle's computation used */
typedef struct { double r, c, s, W[2], Wor[2]; } geo_adj_t;

/* lam (X, Y) from the adjoints of r, c, s, W, Wor at a particle (pgeo_t of geometry()) */
static void geo_back(const grid_t* g, const pgeo_t* p, geo_adj_t* a, double* lX, double* lY) {
    const double ih = g->inv_h[p->j];
    if (p->j > 0 && p->r > 0.0) {            /* Wor = W / r */
        for (int cc = 0; cc < 2; ++cc) {
            a->W[cc] += a->Wor[cc] / p->r;
            a->r -= a->Wor[cc] * p->W[cc] / (p->r * p->r);
        }
    }
    /* W1 = t, W0 = 1 - t, t = (r - r_j) / h_j inside the cell (clamped outside: no derivative) */
    const double tt = (p->r - g->r[p->j]) * ih;
    if (tt > 0.0 && tt < 1.0) a->r += (a->W[1] - a->W[0]) * ih;
    if (p->r > 0.0) {
        const double c = p->c, s = p->s, r = p->r;
        *lX += a->r * c + a->c * s * s / r - a->s * c * s / r;
        *lY += a->r * s - a->c * c * s / r + a->s * c * c / r;
    }
}

/* value of lin(f) and its adjoint: lam_f[j], [j+1] += l * W; the W adjoints += l * f */
static inline void lin_back(const pgeo_t* p, const double* f, double l, double* lf, geo_adj_t* a) {
    lf[p->j] += l * p->W[0];
    lf[p->j + 1] += l * p->W[1];
    a->W[0] += l * f[p->j];
    a->W[1] += l * f[p->j + 1];
}

/* ------------------------------------------------------------------ slice-level adjoint buffers */
typedef struct {
    double *wpr, *ez, *bz, *bpr, *bpi;      /* field arrays of the slice */
    double *chi;                            /* plasma chi of the slice (forward value) */
    double *l_wpr, *l_ez, *l_bz, *l_bpr, *l_bpi;
    double *l_rhot, *l_drho, *l_jz, *l_chi, *l_jpr, *l_jpi, *l_Sr, *l_Si;
    double *l_psi, *l_t, *mu;
    int* dir;
    double* pool;
} slice_adj_t;

static void slice_adj_init(slice_adj_t* A, int M) {
    const int n = 22;
    A->pool = (double*)calloc((size_t)n * M, sizeof(double));
    double* p = A->pool;
    double** arr[] = {&A->wpr, &A->ez, &A->bz, &A->bpr, &A->bpi, &A->chi, &A->l_wpr, &A->l_ez, &A->l_bz,
                      &A->l_bpr, &A->l_bpi, &A->l_rhot, &A->l_drho, &A->l_jz, &A->l_chi, &A->l_jpr, &A->l_jpi,
                      &A->l_Sr, &A->l_Si, &A->l_psi, &A->l_t, &A->mu};
    for (size_t i = 0; i < sizeof(arr) / sizeof(arr[0]); ++i) { *arr[i] = p; p += M; }
    A->dir = (int*)calloc(M, sizeof(int));
}
static void slice_adj_free(slice_adj_t* A) { free(A->pool); free(A->dir); }
static void slice_adj_zero_l(slice_adj_t* A, int M) {
    /* every adjoint array (from l_wpr on) */
    memset(A->l_wpr, 0, sizeof(double) * (size_t)M * 16);
}

/* ------------------------------------------------------------------ plasma particle adjoints */
typedef struct { double X, Y, PX, PY, D; } pst_t;

/* the S deposit of one particle (species_deposit_S, m = 0) in reverse: lam of its state and of the
   gathered fields (scattered into l_wpr, l_ez, l_bz) from l_Sr, l_Si */
static void S_back(qzo_sim* s, const species_t* q, slice_adj_t* A, const pst_t* P, double w, double* lst) {
    const grid_t* g = &s->fs.g;
    const double q0 = q->p.q, qm = q->p.q / q->p.m;
    const pgeo_t p = geometry(g, P->X, P->Y);
    const double R1 = lin(A->wpr, &p), Ez = lin(A->ez, &p), Bz = lin(A->bz, &p);
    const double Wx = R1 * p.c, Wy = R1 * p.s;
    const double PX = P->PX, PY = P->PY, D = P->D;
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D, invd2 = invd * invd;
    const double ux = PX * invd, uy = PY * invd;
    const double ur = p.c * ux + p.s * uy, uth = p.c * uy - p.s * ux;
    const double dD = qm * ((PX * Wx + PY * Wy) * invd - Ez);
    const double nx_ = qm * (gam * Wx + PY * Bz) - PX * dD, ny_ = qm * (gam * Wy - PX * Bz) - PY * dD;
    const double ax = nx_ * invd2, ay = ny_ * invd2;
    const double wq = w * q0;
    geo_adj_t ga = {0};
    double l_ax = 0, l_ay = 0, l_ux = 0, l_uy = 0, l_ur = 0, l_uth = 0;
    for (int cc = 0; cc < 2; ++cc) {
        const int jj = p.j + cc;
        const double iv = g->inv_V[jj] * wq;
        const double f2 = uth * p.Wor[cc];
        const double Ar = ax * p.W[cc] + ux * ur * p.dW[cc] + f2 * uy;
        const double Ai = ay * p.W[cc] + uy * ur * p.dW[cc] - f2 * ux;
        const double LSr = A->l_Sr[jj], LSi = A->l_Si[jj];
        const double lAr = iv * (LSr * p.c - LSi * p.s);
        const double lAi = iv * (LSr * p.s + LSi * p.c);
        ga.c += iv * (LSr * Ar + LSi * Ai);
        ga.s += iv * (LSr * Ai - LSi * Ar);
        l_ax += lAr * p.W[cc];
        l_ay += lAi * p.W[cc];
        ga.W[cc] += lAr * ax + lAi * ay;
        l_ux += lAr * ur * p.dW[cc] - lAi * f2;
        l_uy += lAr * f2 + lAi * ur * p.dW[cc];
        l_ur += (lAr * ux + lAi * uy) * p.dW[cc];
        const double l_f2 = lAr * uy - lAi * ux;
        l_uth += l_f2 * p.Wor[cc];
        ga.Wor[cc] += l_f2 * uth;
    }
    double l_PX = 0, l_PY = 0, l_D = 0, l_gam = 0, l_invd = 0, l_Wx = 0, l_Wy = 0, l_Ez = 0, l_Bz = 0, l_dD = 0;
    /* ax = nx_ invd2, ay = ny_ invd2 */
    l_invd += (l_ax * nx_ + l_ay * ny_) * 2.0 * invd;
    {
        const double lnx = l_ax * invd2, lny = l_ay * invd2;
        l_gam += qm * (lnx * Wx + lny * Wy);
        l_Wx += lnx * qm * gam;
        l_Wy += lny * qm * gam;
        l_PY += lnx * qm * Bz;
        l_PX -= lny * qm * Bz;
        l_Bz += qm * (lnx * PY - lny * PX);
        l_PX -= lnx * dD;
        l_PY -= lny * dD;
        l_dD -= lnx * PX + lny * PY;
    }
    /* dD = qm ((PX Wx + PY Wy) invd - Ez) */
    l_PX += l_dD * qm * Wx * invd;
    l_PY += l_dD * qm * Wy * invd;
    l_Wx += l_dD * qm * PX * invd;
    l_Wy += l_dD * qm * PY * invd;
    l_invd += l_dD * qm * (PX * Wx + PY * Wy);
    l_Ez -= l_dD * qm;
    /* ur, uth */
    ga.c += l_ur * ux + l_uth * uy;
    ga.s += l_ur * uy - l_uth * ux;
    l_ux += l_ur * p.c - l_uth * p.s;
    l_uy += l_ur * p.s + l_uth * p.c;
    l_PX += l_ux * invd; l_invd += l_ux * PX;
    l_PY += l_uy * invd; l_invd += l_uy * PY;
    /* gam = (1 + PX^2 + PY^2 + D^2) / (2 D) */
    l_PX += l_gam * PX * invd;
    l_PY += l_gam * PY * invd;
    l_D += l_gam * (0.5 - (1.0 + PX * PX + PY * PY) * 0.5 * invd2);
    l_D -= l_invd * invd2;
    /* gathered fields: Wx = R1 c, Wy = R1 s */
    const double l_R1 = l_Wx * p.c + l_Wy * p.s;
    ga.c += l_Wx * R1;
    ga.s += l_Wy * R1;
    lin_back(&p, A->wpr, l_R1, A->l_wpr, &ga);
    lin_back(&p, A->ez, l_Ez, A->l_ez, &ga);
    lin_back(&p, A->bz, l_Bz, A->l_bz, &ga);
    geo_back(g, &p, &ga, &lst[0], &lst[1]);
    lst[2] += l_PX; lst[3] += l_PY; lst[4] += l_D;
}

/* the plasma deposit of one particle (species_deposit, m = 0) in reverse: lam of its state from the
   adjoints of rhot, drho, jz, chi, jp.r1, jp.i1 (rho and the densities feed nothing downstream) */
static void deposit_back(qzo_sim* s, const species_t* q, slice_adj_t* A, const pst_t* P, double w, double* lst) {
    const grid_t* g = &s->fs.g;
    const double q0 = q->p.q, qm = q->p.q / q->p.m;
    const pgeo_t p = geometry(g, P->X, P->Y);
    const double PX = P->PX, PY = P->PY, D = P->D;
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D;
    const double pz = gam - D;
    const double ux = PX * invd, uy = PY * invd;
    const double ur = p.c * ux + p.s * uy, uth = p.c * uy - p.s * ux;
    const double wq = w * q0;
    geo_adj_t ga = {0};
    double l_pzd = 0, l_invd = 0, l_ur = 0, l_uth = 0;
    for (int cc = 0; cc < 2; ++cc) {
        const int jj = p.j + cc;
        const double iv = g->inv_V[jj];
        const double a = wq * p.W[cc] * iv;
        const double la = A->l_rhot[jj] + A->l_jz[jj] * pz * invd + A->l_chi[jj] * qm * invd +
                          A->l_jpr[jj] * ur + A->l_jpi[jj] * uth;
        l_pzd += A->l_jz[jj] * a;
        l_invd += A->l_chi[jj] * a * qm;
        l_ur += A->l_jpr[jj] * a + A->l_drho[jj] * wq * p.dW[cc] * iv;
        l_uth += A->l_jpi[jj] * a;
        ga.W[cc] += la * wq * iv;
    }
    double l_PX = 0, l_PY = 0, l_D = 0;
    /* pz / D = (1 + PX^2 + PY^2) / (2 D^2) - 1/2 */
    l_PX += l_pzd * PX * invd * invd;
    l_PY += l_pzd * PY * invd * invd;
    l_D -= l_pzd * (1.0 + PX * PX + PY * PY) * invd * invd * invd;
    ga.c += l_ur * ux + l_uth * uy;
    ga.s += l_ur * uy - l_uth * ux;
    const double l_ux = l_ur * p.c - l_uth * p.s, l_uy = l_ur * p.s + l_uth * p.c;
    l_PX += l_ux * invd; l_invd += l_ux * PX;
    l_PY += l_uy * invd; l_invd += l_uy * PY;
    l_D -= l_invd * invd * invd;
    geo_back(g, &p, &ga, &lst[0], &lst[1]);
    lst[2] += l_PX; lst[3] += l_PY; lst[4] += l_D;
}

/* the push of one particle at slice k (species_push, uniform AB) in reverse.
   H: its AB history before the push ((ord, 5) for this particle, read with stride cap);
   lnext: lam of its state after the push (5) and of the history after the push (ord * 5);
   out lst: lam of the state before (5, accumulated), lH: lam of the history before (ord * 5, set).
   Returns 0 when the particle was removed by this push (no adjoint flows through it). */
static int push_back(qzo_sim* s, const species_t* q, slice_adj_t* A, int k, const pst_t* P, const double* H,
                     size_t cap, const double* lnext, double* lst, double* lH) {
    const grid_t* g = &s->fs.g;
    const int ord = s->p.ab_order;
    const int slot = k % ord, first = (k == 0);
    const double dxi = s->p.dxi, qm = q->p.q / q->p.m;
    const double R = g->R;
    const pgeo_t p = geometry(g, P->X, P->Y);
    const double R1 = lin(A->wpr, &p), Ez = lin(A->ez, &p), Bz = lin(A->bz, &p);
    const double BR = lin(A->bpr, &p), BI = lin(A->bpi, &p);
    const double Wx = R1 * p.c, Wy = R1 * p.s;
    const double Bx = BR * p.c - BI * p.s, By = BR * p.s + BI * p.c;
    const double PX = P->PX, PY = P->PY, D = P->D;
    const double gam = (1.0 + PX * PX + PY * PY + D * D) / (2.0 * D);
    const double invd = 1.0 / D;
    double fv[5];
    fv[0] = PX * invd;
    fv[1] = PY * invd;
    fv[2] = qm * (gam * Wx * invd + By + PY * Bz * invd);
    fv[3] = qm * (gam * Wy * invd - Bx - PX * Bz * invd);
    fv[4] = qm * ((PX * Wx + PY * Wy) * invd - Ez);
    double Hc[5][5];                             /* history after writing fv (before reflection) */
    for (int sl = 0; sl < ord; ++sl)
        for (int v = 0; v < 5; ++v) Hc[sl][v] = (first || sl == slot) ? fv[v] : H[((size_t)sl * 5 + v) * cap];
    double sum[5] = {0, 0, 0, 0, 0};
    for (int m = 0; m < ord; ++m) {
        const int sl = (slot - m + ord) % ord;
        for (int v = 0; v < 5; ++v) sum[v] += q->ab[m] * Hc[sl][v];
    }
    const double xn = P->X + dxi * sum[0], yn = P->Y + dxi * sum[1];
    const double pxn = PX + dxi * sum[2], pyn = PY + dxi * sum[3];
    const double dn = D + dxi * sum[4];
    const double gn = (1.0 + pxn * pxn + pyn * pyn + dn * dn) / (2.0 * dn);
    if (!(dn > s->p.delta_min) || gn > s->p.max_qsa * dn) return 0;
    const double rn = sqrt(xn * xn + yn * yn);
    double l_pre[4] = {lnext[0], lnext[1], lnext[2], lnext[3]};     /* lam of xn yn pxn pyn */
    double lHc[5][5];
    for (int sl = 0; sl < ord; ++sl)
        for (int v = 0; v < 5; ++v) lHc[sl][v] = lnext[5 + sl * 5 + v];
    if (rn > R) {                                /* specular reflection at the wall */
        const double rr = 2.0 * R - rn;
        if (rr < 0.0) return 0;
        const double nx = xn / rn, ny = yn / rn;
        double lnx = 0, lny = 0, lrn = 0;
        /* position: x' = nx rr, y' = ny rr */
        lnx += lnext[0] * rr;
        lny += lnext[1] * rr;
        lrn -= lnext[0] * nx + lnext[1] * ny;
        /* pairs v' = v - 2 (v.n) n: lam_v = lam' - 2 (lam'.n) n; lam_n += -2 ((lam'.n) v + (v.n) lam') */
#define REFL_BACK(v0, v1, l0, l1, o0, o1)                                             \
        do {                                                                          \
            const double ln_ = (l0) * nx + (l1) * ny, vn_ = (v0) * nx + (v1) * ny;   \
            o0 = (l0) - 2.0 * ln_ * nx;                                               \
            o1 = (l1) - 2.0 * ln_ * ny;                                               \
            lnx += -2.0 * (ln_ * (v0) + vn_ * (l0));                                  \
            lny += -2.0 * (ln_ * (v1) + vn_ * (l1));                                  \
        } while (0)
        REFL_BACK(pxn, pyn, lnext[2], lnext[3], l_pre[2], l_pre[3]);
        for (int sl = 0; sl < ord; ++sl) {
            const double l0 = lnext[5 + sl * 5 + 0], l1 = lnext[5 + sl * 5 + 1];
            const double l2 = lnext[5 + sl * 5 + 2], l3 = lnext[5 + sl * 5 + 3];
            REFL_BACK(Hc[sl][0], Hc[sl][1], l0, l1, lHc[sl][0], lHc[sl][1]);
            REFL_BACK(Hc[sl][2], Hc[sl][3], l2, l3, lHc[sl][2], lHc[sl][3]);
        }
#undef REFL_BACK
        const double ldot = lnx * nx + lny * ny;
        l_pre[0] = (lnx - nx * ldot) / rn + lrn * nx;
        l_pre[1] = (lny - ny * ldot) / rn + lrn * ny;
    }
    /* AB update: xn = X + dxi sum0 ... dn = D + dxi sum4 */
    const double lsum[5] = {dxi * l_pre[0], dxi * l_pre[1], dxi * l_pre[2], dxi * l_pre[3], dxi * lnext[4]};
    for (int m = 0; m < ord; ++m) {
        const int sl = (slot - m + ord) % ord;
        for (int v = 0; v < 5; ++v) lHc[sl][v] += q->ab[m] * lsum[v];
    }
    double lfv[5] = {0, 0, 0, 0, 0};
    for (int sl = 0; sl < ord; ++sl)
        for (int v = 0; v < 5; ++v) {
            const int written = first || sl == slot;
            if (written) lfv[v] += lHc[sl][v];
            lH[sl * 5 + v] = written ? 0.0 : lHc[sl][v];
        }
    double l_X = l_pre[0], l_Y = l_pre[1], l_PX = l_pre[2], l_PY = l_pre[3], l_D = lnext[4];
    /* fv in reverse */
    double l_gam = 0, l_invd = 0, l_Wx = 0, l_Wy = 0, l_Ez = 0, l_Bz = 0, l_Bx = 0, l_By = 0;
    l_PX += lfv[0] * invd; l_invd += lfv[0] * PX;
    l_PY += lfv[1] * invd; l_invd += lfv[1] * PY;
    l_gam += lfv[2] * qm * Wx * invd;
    l_Wx += lfv[2] * qm * gam * invd;
    l_invd += lfv[2] * qm * (gam * Wx + PY * Bz);
    l_By += lfv[2] * qm;
    l_PY += lfv[2] * qm * Bz * invd;
    l_Bz += lfv[2] * qm * PY * invd;
    l_gam += lfv[3] * qm * Wy * invd;
    l_Wy += lfv[3] * qm * gam * invd;
    l_invd += lfv[3] * qm * (gam * Wy - PX * Bz);
    l_Bx -= lfv[3] * qm;
    l_PX -= lfv[3] * qm * Bz * invd;
    l_Bz -= lfv[3] * qm * PX * invd;
    l_PX += lfv[4] * qm * Wx * invd;
    l_PY += lfv[4] * qm * Wy * invd;
    l_Wx += lfv[4] * qm * PX * invd;
    l_Wy += lfv[4] * qm * PY * invd;
    l_invd += lfv[4] * qm * (PX * Wx + PY * Wy);
    l_Ez -= lfv[4] * qm;
    l_PX += l_gam * PX * invd;
    l_PY += l_gam * PY * invd;
    l_D += l_gam * (0.5 - (1.0 + PX * PX + PY * PY) * 0.5 * invd * invd);
    l_D -= l_invd * invd * invd;
    geo_adj_t ga = {0};
    const double l_R1 = l_Wx * p.c + l_Wy * p.s;
    ga.c += l_Wx * R1 + l_Bx * BR + l_By * BI;
    ga.s += l_Wy * R1 - l_Bx * BI + l_By * BR;
    const double l_BR = l_Bx * p.c + l_By * p.s, l_BI = -l_Bx * p.s + l_By * p.c;
    lin_back(&p, A->wpr, l_R1, A->l_wpr, &ga);
    lin_back(&p, A->ez, l_Ez, A->l_ez, &ga);
    lin_back(&p, A->bz, l_Bz, A->l_bz, &ga);
    lin_back(&p, A->bpr, l_BR, A->l_bpr, &ga);
    lin_back(&p, A->bpi, l_BI, A->l_bpi, &ga);
    geo_back(g, &p, &ga, &l_X, &l_Y);
    lst[0] += l_X; lst[1] += l_Y; lst[2] += l_PX; lst[3] += l_PY; lst[4] += l_D;
    return 1;
}

/* ------------------------------------------------------------------ the reverse sweep */
/* From the adjoint of the step's field store (lfld: (K, M, 6)) to the adjoint of its beam sources
   (lbsrc: (K, M, 5), accumulated). Needs s->fld of this step and s->traj recorded by the same
   sweep (s->sp[isp] the mobile species). */
static void sweep_back(qzo_sim* s, int isp, const double* lfld, double* lbsrc) {
    const int M = s->M, K = s->p.K, N = M - 1, ord = s->p.ab_order;
    species_t* q = &s->sp[isp];
    const size_t cap = (size_t)q->cap, nv = 6 + 5 * (size_t)ord;
    const int np = q->Np;
    const double idxi = 1.0 / s->p.dxi;
    const double qm = q->p.q / q->p.m;
    slice_adj_t A;
    slice_adj_init(&A, M);
    const int nl = 5 + 5 * ord;
    double* lam = (double*)calloc((size_t)np * nl, sizeof(double));     /* lam of P_{k+1} */
    double* lam2 = (double*)calloc((size_t)np * nl, sizeof(double));    /* lam of P_k */
    const grid_t* g = &s->fs.g;
#define LB(k, j, c) lbsrc[((size_t)(k) * M + (j)) * 5 + (c)]
    for (int k = K - 1; k >= 0; --k) {
        const double* F = s->fld + (size_t)k * M * 6;
        const double* LF = lfld + (size_t)k * M * 6;
        const double* T = s->traj + (size_t)k * nv * cap;
        for (int j = 0; j < M; ++j) {
            A.wpr[j] = F[j * 6 + F_EP1R] - F[j * 6 + F_BP1I];
            A.bpr[j] = F[j * 6 + F_BP1R];
            A.bpi[j] = F[j * 6 + F_BP1I];
            A.ez[j] = F[j * 6 + F_EZ0];
            A.bz[j] = F[j * 6 + F_BZ0];
            A.chi[j] = 0.0;
        }
        slice_adj_zero_l(&A, M);
        /* chi of the slice: the plasma deposit of P_k */
        for (int i = 0; i < np; ++i) {
            const double w = T[5 * cap + i];
            if (w == 0.0) continue;
            const double PX = T[2 * cap + i], PY = T[3 * cap + i], D = T[4 * cap + i];
            const pgeo_t p = geometry(g, T[i], T[cap + i]);
            (void)PX; (void)PY;
            for (int cc = 0; cc < 2; ++cc) {
                const int jj = p.j + cc;
                const double a = w * q->p.q * p.W[cc] * g->inv_V[jj];
                A.chi[jj] += a * qm / D;
            }
        }
        solver_filter(&s->fs, 0, A.chi);             /* B+ saw the smoothed chi (src/Simulation.cpp:823-835) */
        /* store (src/Simulation.cpp:594-633): EP1R = wp.r1 + bp.i1, EP1I = -bp.r1, BP1R, BP1I, EZ0, BZ0 */
        for (int j = 0; j < M; ++j) {
            A.l_wpr[j] += LF[j * 6 + F_EP1R];
            A.l_bpi[j] += LF[j * 6 + F_EP1R] + LF[j * 6 + F_BP1I];
            A.l_bpr[j] += -LF[j * 6 + F_EP1I] + LF[j * 6 + F_BP1R];
            A.l_ez[j] += LF[j * 6 + F_EZ0];
            A.l_bz[j] += LF[j * 6 + F_BZ0];
        }
        /* push of slice k (P_k -> P_{k+1}) */
        memset(lam2, 0, sizeof(double) * (size_t)np * nl);
        if (k < K - 1)
            for (int i = 0; i < np; ++i) {
                if (T[5 * cap + i] == 0.0) continue;
                const pst_t P = {T[i], T[cap + i], T[2 * cap + i], T[3 * cap + i], T[4 * cap + i]};
                push_back(s, q, &A, k, &P, T + 6 * cap + i, cap, lam + (size_t)i * nl, lam2 + (size_t)i * nl,
                          lam2 + (size_t)i * nl + 5);
            }
        /* B+ (src/Simulation.cpp:535-591, m = 0): bp.r1 = (L1D - chi)^-1 (-S.i1), bp.i1 = (L1F - chi)^-1
           (grad jz + S.r1, wall flux - fc jz[N]) */
        {
            solve_T(&s->fs, OP_L1D, A.chi, A.l_bpr, A.mu, A.dir);
            for (int j = 0; j <= N; ++j) {
                if (A.dir[j]) continue;
                A.l_chi[j] += A.mu[j] * A.bpr[j];
                A.l_Si[j] -= A.mu[j];
            }
            solve_T(&s->fs, OP_L1F, A.chi, A.l_bpi, A.mu, A.dir);
            for (int j = 0; j <= N; ++j) A.l_t[j] = 0.0;
            for (int j = 0; j <= N; ++j) {
                if (A.dir[j]) continue;
                A.l_chi[j] += A.mu[j] * A.bpi[j];
                A.l_t[j] = A.mu[j];                  /* lam of rb.i1 */
            }
            A.l_jz[N] -= s->fs.flux_coef * A.mu[N];
            for (int j = 0; j <= N; ++j) A.l_Sr[j] += A.l_t[j];
            gradient_T(&s->fs, A.l_t, A.l_jz);
        }
        /* the S+ filter (src/Simulation.cpp:810-812) in reverse */
        filter_T(&s->fs, 1, A.l_Sr);
        filter_T(&s->fs, 1, A.l_Si);
        /* S deposit (needs lam_S; adds to lam of W+, E_z, B_z) */
        for (int i = 0; i < np; ++i) {
            const double w = T[5 * cap + i];
            if (w == 0.0) continue;
            const pst_t P = {T[i], T[cap + i], T[2 * cap + i], T[3 * cap + i], T[4 * cap + i]};
            S_back(s, q, &A, &P, w, lam2 + (size_t)i * nl);
        }
        /* B_z = L0^-1 (-(grad_odd + over_r) jp.i1) */
        solve_T(&s->fs, OP_L0, NULL, A.l_bz, A.mu, A.dir);
        for (int j = 0; j <= N; ++j) A.l_t[j] = A.dir[j] ? 0.0 : -A.mu[j];
        gradient_odd_T(&s->fs, A.l_t, A.l_jpi);
        over_r_T(&s->fs, A.l_t, A.l_jpi);
        /* W+ = -grad psi */
        for (int j = 0; j <= N; ++j) A.l_t[j] = -A.l_wpr[j];
        gradient_T(&s->fs, A.l_t, A.l_psi);
        /* psi = L0^-1 (-rhot), E_z = L0^-1 (-drho) */
        solve_T(&s->fs, OP_L0, NULL, A.l_psi, A.mu, A.dir);
        for (int j = 0; j <= N; ++j) A.l_rhot[j] += A.dir[j] ? 0.0 : -A.mu[j];
        solve_T(&s->fs, OP_L0, NULL, A.l_ez, A.mu, A.dir);
        for (int j = 0; j <= N; ++j) A.l_drho[j] += A.dir[j] ? 0.0 : -A.mu[j];
        /* combine sources (src/Simulation.cpp:408-457): beam rows k (and k +- 1 through d/dxi) */
        for (int j = 0; j < M; ++j) {
            LB(k, j, B_RT0) += A.l_rhot[j];
            LB(k, j, B_JZ0) += A.l_jz[j];
            LB(k, j, B_JP1R) += A.l_jpr[j];
            LB(k, j, B_JP1I) += A.l_jpi[j];
            const double ld = A.l_drho[j] * idxi;
            if (s->p.ngp) {      /* ngp: the backward difference of rho - J_z (no row ahead of the box head) */
                LB(k, j, B_RT0) += ld;
                if (k > 0) LB(k - 1, j, B_RT0) -= ld;
                continue;
            }
            if (K == 1) continue;
            if (k == 0) { LB(1, j, B_RT0) += ld; LB(0, j, B_RT0) -= ld; }
            else if (k == K - 1) { LB(K - 1, j, B_RT0) += ld; LB(K - 2, j, B_RT0) -= ld; }
            else { LB(k + 1, j, B_RT0) += 0.5 * ld; LB(k - 1, j, B_RT0) -= 0.5 * ld; }
        }
        /* the filter of the plasma deposit (src/Simulation.cpp:823-835) in reverse: the beams were added after
           it, so their adjoints above are those of the combined sources */
        filter_T(&s->fs, 0, A.l_rhot);
        filter_T(&s->fs, 0, A.l_drho);
        filter_T(&s->fs, 0, A.l_jz);
        filter_T(&s->fs, 0, A.l_chi);
        filter_T(&s->fs, 1, A.l_jpr);
        filter_T(&s->fs, 1, A.l_jpi);
        /* plasma deposit of P_k */
        for (int i = 0; i < np; ++i) {
            const double w = T[5 * cap + i];
            if (w == 0.0) continue;
            const pst_t P = {T[i], T[cap + i], T[2 * cap + i], T[3 * cap + i], T[4 * cap + i]};
            deposit_back(s, q, &A, &P, w, lam2 + (size_t)i * nl);
        }
        double* tmp = lam; lam = lam2; lam2 = tmp;
    }
#undef LB
    free(lam); free(lam2);
    slice_adj_free(&A);
}

/* ------------------------------------------------------------------ beam adjoints */
/* reverse of solve_implicit(a, b) -> r: lam_a, lam_b += from lam_r */
static void solve_implicit_back(v3 a, v3 b, v3 lr, v3* la, v3* lb) {
    const double b2 = v3dot(b, b), ab = v3dot(a, b);
    const double X = 0.5 * (1.0 + v3dot(a, a) - b2), Cc = b2 + ab * ab;
    const double g2 = gamma2_root(X, Cc);
    const double g = sqrt(g2);
    const v3 axb = v3cross(a, b);
    const double inv = 1.0 / (g2 + b2);
    const v3 qv = {g2 * a.x + g * axb.x + ab * b.x, g2 * a.y + g * axb.y + ab * b.y, g2 * a.z + g * axb.z + ab * b.z};
    const v3 lq = v3mul(inv, lr);
    const double l_inv = v3dot(lr, qv);
    double l_g2 = -l_inv * inv * inv, l_b2 = -l_inv * inv * inv;
    l_g2 += v3dot(lq, a);
    *la = v3add(*la, v3mul(g2, lq));
    const double l_g = v3dot(lq, axb);
    const v3 laxb = v3mul(g, lq);
    double l_ab = v3dot(lq, b);
    *lb = v3add(*lb, v3mul(ab, lq));
    *la = v3add(*la, v3cross(b, laxb));
    *lb = v3add(*lb, v3cross(laxb, a));
    l_g2 += l_g / (2.0 * g);
    const double sq = sqrt(X * X + Cc);
    const double l_X = l_g2 * (1.0 + X / sq), l_C = l_g2 / (2.0 * sq);
    *la = v3add(*la, v3mul(l_X, a));
    l_b2 -= 0.5 * l_X;
    l_b2 += l_C;
    l_ab += 2.0 * ab * l_C;
    *la = v3add(*la, v3mul(l_ab, b));
    *lb = v3add(*lb, v3mul(l_ab, a));
    *lb = v3add(*lb, v3mul(2.0 * l_b2, b));
}

/* reverse of vay(u, E, B, eps): lam_u, lam_E, lam_B += from lam_out */
static void vay_back(v3 u, v3 E, v3 B, double eps, v3 lout, v3* lu, v3* lE, v3* lB) {
    const double g0 = sqrt(1.0 + v3dot(u, u));
    const v3 uxB = v3cross(u, B);
    const v3 up = v3add(v3add(u, v3mul(2.0 * eps, E)), v3mul(eps / g0, uxB));
    v3 lup = {0, 0, 0}, lb = {0, 0, 0};
    solve_implicit_back(up, v3mul(eps, B), lout, &lup, &lb);
    *lB = v3add(*lB, v3mul(eps, lb));
    *lu = v3add(*lu, lup);
    *lE = v3add(*lE, v3mul(2.0 * eps, lup));
    const v3 lc = v3mul(eps / g0, lup);
    *lu = v3add(*lu, v3cross(B, lc));
    *lB = v3add(*lB, v3cross(lc, u));
    const double l_ig0 = eps * v3dot(lup, uxB);
    *lu = v3add(*lu, v3mul(-l_ig0 / (g0 * g0 * g0), u));
}

/* reverse of omvz(p) = (1 + px^2 + py^2) / (gam (gam + pz)), gam = sqrt(1 + |p|^2): lam_p += */
static void omvz_back(double px, double py, double pz, double l, double* lp) {
    const double A = 1.0 + px * px + py * py;
    const double G = sqrt(A + pz * pz);
    const double den = G * (G + pz);
    const double lA = l / den;
    const double lG = -l * A * (2.0 * G + pz) / (den * den);
    const double lpz = -l * A * G / (den * den);
    lp[0] += lA * 2.0 * px + lG * px / G;
    lp[1] += lA * 2.0 * py + lG * py / G;
    lp[2] += lpz + lG * pz / G;
}

/* the push of one beam (beam_advance with move, preceded by the start-up half kick when startup) in
   reverse; lam7: in = lam after the push, out = lam before (x y px py pz xi w); lfld accumulates */
static void beam_push_back(qzo_sim* s, const beam_t* B, long i, double dt_kick, double dt, int startup,
                           double* lam7, double* lfld) {
    const grid_t* g = &s->fs.g;
    const int M = s->M, nloc = s->p.K;
    const double qm = B->q / B->m;
    const double xmin = s->p.xi_min, idxi = 1.0 / s->p.dxi;
    const double xmax = s->p.xi_min + (s->p.K - 1) * s->p.dxi;
    const double R = g->R;
    const double* fld = s->fld;
    if (B->w[i] == 0.0) { for (int c = 0; c < 7; ++c) lam7[c] = 0.0; return; }
    const double X = B->x[i], Y = B->y[i];
    const double r = sqrt(X * X + Y * Y);
    const double c = r > 0.0 ? X / r : 1.0, sn = r > 0.0 ? Y / r : 0.0;
    double sl = (B->xi[i] - xmin) * idxi;
    int k, kclamp = 0;
    double tk;
    if (s->p.ngp) {          /* the slice nearest to the particle, no xi interpolation (src/Beam.cpp:980-983) */
        k = (int)floor(sl + 0.5);
        k = k < 0 ? 0 : (k > nloc - 1 ? nloc - 1 : k);
        tk = 0.0;
        kclamp = 1;          /* piecewise constant in xi: no xi derivative */
    } else {
        k = (int)floor(sl);
        if (k < 0) { k = 0; sl = 0; kclamp = 1; }
        if (k > nloc - 2) { k = nloc - 2; sl = nloc - 1; kclamp = 1; }
        tk = sl - k;
    }
    const int k1 = s->p.ngp ? k : k + 1;
    int j; double t;
    grid_weights(g, r, &j, &t);
#define FL(kk, jj, comp) fld[((size_t)(kk) * M + (jj)) * 6 + (comp)]
#define BIL(comp) ((1.0 - tk) * ((1.0 - t) * FL(k, j, comp) + t * FL(k, j + 1, comp)) + \
                   tk * ((1.0 - t) * FL(k1, j, comp) + t * FL(k1, j + 1, comp)))
    const double er = BIL(F_EP1R), ei = BIL(F_EP1I), br = BIL(F_BP1R), bi = BIL(F_BP1I);
    const v3 E = {er * c - ei * sn, er * sn + ei * c, BIL(F_EZ0)};
    const v3 Bf = {br * c - bi * sn, br * sn + bi * c, BIL(F_BZ0)};
    const v3 u0 = {B->px[i], B->py[i], B->pz[i]};
    /* forward */
    v3 u1 = u0;
    const double hs = 0.5 * qm * (-0.5 * dt_kick);
    double g00 = 0.0;
    if (startup) {
        g00 = sqrt(1.0 + v3dot(u0, u0));
        u1 = v3add(u0, v3mul(2.0 * hs, v3add(E, v3cross(v3mul(1.0 / g00, u0), Bf))));
    }
    const double h = 0.5 * qm * dt_kick;
    const v3 u2 = vay(u1, E, Bf, h);
    const double p2 = u2.x * u2.x + u2.y * u2.y;
    const double gam = sqrt(1.0 + p2 + u2.z * u2.z);
    const double omvz = (1.0 + p2) / (gam * (gam + u2.z));
    const double xn = X + u2.x / gam * dt, yn = Y + u2.y / gam * dt;
    const double xin = B->xi[i] + omvz * dt;
    if (xn * xn + yn * yn >= R * R || xin < xmin || xin > xmax) { for (int cc = 0; cc < 7; ++cc) lam7[cc] = 0.0; return; }
    /* reverse */
    const double lxn = lam7[0], lyn = lam7[1], lxin = lam7[5];
    v3 lu2 = {lam7[2], lam7[3], lam7[4]};
    double lX = lxn, lY = lyn, lxi = lxin;
    double lgam = -(lxn * u2.x + lyn * u2.y) * dt / (gam * gam);
    lu2.x += lxn * dt / gam;
    lu2.y += lyn * dt / gam;
    double lp[3] = {0, 0, 0};
    omvz_back(u2.x, u2.y, u2.z, lxin * dt, lp);
    lu2.x += lp[0] + lgam * u2.x / gam;
    lu2.y += lp[1] + lgam * u2.y / gam;
    lu2.z += lp[2] + lgam * u2.z / gam;
    v3 lu1 = {0, 0, 0}, lE = {0, 0, 0}, lB = {0, 0, 0};
    vay_back(u1, E, Bf, h, lu2, &lu1, &lE, &lB);
    v3 lu0 = lu1;
    if (startup) {
        const v3 lw = v3mul(2.0 * hs, lu1);                 /* w = E + (u0 x B) / g00 */
        lE = v3add(lE, lw);
        const v3 lcr = v3mul(1.0 / g00, lw);
        lu0 = v3add(lu0, v3cross(Bf, lcr));
        lB = v3add(lB, v3cross(lcr, u0));
        const double l_ig = v3dot(lw, v3cross(u0, Bf));
        lu0 = v3add(lu0, v3mul(-l_ig / (g00 * g00 * g00), u0));
    }
    /* fields: E = (er c - ei s, er s + ei c, ez), B likewise */
    const double l_er = lE.x * c + lE.y * sn, l_ei = -lE.x * sn + lE.y * c;
    const double l_br = lB.x * c + lB.y * sn, l_bi = -lB.x * sn + lB.y * c;
    double l_c = lE.x * er + lE.y * ei + lB.x * br + lB.y * bi;
    double l_s = -lE.x * ei + lE.y * er - lB.x * bi + lB.y * br;
    const double lcomp[6] = {l_er, l_ei, l_br, l_bi, lE.z, lB.z};
    const int comp[6] = {F_EP1R, F_EP1I, F_BP1R, F_BP1I, F_EZ0, F_BZ0};
    double l_tk = 0.0, l_t = 0.0;
#define LFL(kk, jj, cmp) lfld[((size_t)(kk) * M + (jj)) * 6 + (cmp)]
    for (int q = 0; q < 6; ++q) {
        const int cm = comp[q];
        const double l = lcomp[q];
        LFL(k, j, cm) += l * (1.0 - tk) * (1.0 - t);
        LFL(k, j + 1, cm) += l * (1.0 - tk) * t;
        LFL(k1, j, cm) += l * tk * (1.0 - t);
        LFL(k1, j + 1, cm) += l * tk * t;
        l_tk += l * (((1.0 - t) * FL(k1, j, cm) + t * FL(k1, j + 1, cm)) - ((1.0 - t) * FL(k, j, cm) + t * FL(k, j + 1, cm)));
        l_t += l * ((1.0 - tk) * (FL(k, j + 1, cm) - FL(k, j, cm)) + tk * (FL(k1, j + 1, cm) - FL(k1, j, cm)));
    }
#undef LFL
#undef BIL
#undef FL
    if (!kclamp) lxi += l_tk * idxi;
    const double tt = (r - g->r[j]) * g->inv_h[j];
    double l_r = (tt > 0.0 && tt < 1.0) ? l_t * g->inv_h[j] : 0.0;
    if (r > 0.0) {
        lX += l_r * c + l_c * sn * sn / r - l_s * c * sn / r;
        lY += l_r * sn - l_c * c * sn / r + l_s * c * c / r;
    }
    lam7[0] = lX; lam7[1] = lY; lam7[2] = lu0.x; lam7[3] = lu0.y; lam7[4] = lu0.z; lam7[5] = lxi;
    /* lam7[6] (w) passes through: the weight is carried unchanged */
}

/* the deposit of one beam particle (beam_deposit, m = 0, linear in xi) in reverse: lam7 += */
static void beam_deposit_back(qzo_sim* s, const beam_t* B, long i, const double* lbsrc, double* lam7) {
    const grid_t* g = &s->fs.g;
    const int M = s->M;
    const double q = B->q;
    const double xmin = s->p.xi_min, idxi = 1.0 / s->p.dxi;
    const int nloc = s->p.K;
    const double R = g->R;
    const double wi = B->w[i];
    if (wi == 0.0) return;
    const double X = B->x[i], Y = B->y[i];
    const double r = sqrt(X * X + Y * Y);
    if (r > R) return;
    const double c = r > 0.0 ? X / r : 1.0, sn = r > 0.0 ? Y / r : 0.0;
    const double sx = (B->xi[i] - xmin) * idxi;
    const int ngp = s->p.ngp;
    const int k = ngp ? (int)floor(sx + 0.5) : (int)floor(sx);
    if (k < -1 || k >= nloc) return;
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
    double l_omvz = 0, l_vz = 0, l_vr = 0, l_vt = 0, l_w = 0, lWk[2] = {0, 0}, lWr[2] = {0, 0};
    for (int a = 0; a < (ngp ? 1 : 2); ++a) {
        const int kk = k + a;
        if (kk < 0 || kk >= nloc) continue;
        for (int b = 0; b < 2; ++b) {
            const int jj = j + b;
            const double* L = lbsrc + ((size_t)kk * M + jj) * 5;
            const double base = q * g->inv_V[jj] * idxi;
            const double d = wi * Wk[a] * Wr[b] * base;
            const double ld = L[B_RT0] * omvz + L[B_JZ0] * vz + L[B_JP1R] * vr + L[B_JP1I] * vt + L[B_RHO0];
            l_omvz += L[B_RT0] * d;
            l_vz += L[B_JZ0] * d;
            l_vr += L[B_JP1R] * d;
            l_vt += L[B_JP1I] * d;
            l_w += ld * Wk[a] * Wr[b] * base;
            lWk[a] += ld * wi * Wr[b] * base;
            lWr[b] += ld * wi * Wk[a] * base;
        }
    }
    lam7[6] += l_w;
    if (!ngp) lam7[5] += (lWk[1] - lWk[0]) * idxi;
    const double tt = (r - g->r[j]) * g->inv_h[j];
    const double l_r = (tt > 0.0 && tt < 1.0) ? (lWr[1] - lWr[0]) * g->inv_h[j] : 0.0;
    const double l_vx = l_vr * c - l_vt * sn, l_vy = l_vr * sn + l_vt * c;
    const double l_c = l_vr * vx + l_vt * vy, l_s = l_vr * vy - l_vt * vx;
    if (r > 0.0) {
        lam7[0] += l_r * c + l_c * sn * sn / r - l_s * c * sn / r;
        lam7[1] += l_r * sn - l_c * c * sn / r + l_s * c * c / r;
    }
    /* v = p / gam */
    double lp[3] = {l_vx / gam, l_vy / gam, l_vz / gam};
    const double l_g = -(l_vx * PX + l_vy * PY + l_vz * PZ) / (gam * gam);
    lp[0] += l_g * PX / gam; lp[1] += l_g * PY / gam; lp[2] += l_g * PZ / gam;
    omvz_back(PX, PY, PZ, l_omvz, lp);
    lam7[2] += lp[0]; lam7[3] += lp[1]; lam7[4] += lp[2];
}

/* the moment sums of one particle in reverse: lam7 += from lamS (17) */
static void sums_back(const beam_t* B, long i, const double* lS, double* lam7) {
    const double w = B->w[i];
    if (w == 0.0) return;
    const double PX = B->px[i], PY = B->py[i], PZ = B->pz[i], X = B->x[i], Y = B->y[i];
    const double g = sqrt(1 + PX * PX + PY * PY + PZ * PZ);
    const double G = g - B->gref, XI = B->xi[i] - B->xiref;
    const double v[15] = {G, G * G, XI, XI * XI, X * X + Y * Y, X, Y, X * X, Y * Y, PX, PY, PX * PX, PY * PY,
                          X * PX, Y * PY};
    double lw = lS[0];
    for (int c = 0; c < 15; ++c) lw += lS[c + 1] * v[c];
    lam7[6] += lw;
    const double* lv = lS + 1;     /* lam of v[c] is w * lS[c + 1] */
    const double lG = w * (lv[0] + 2.0 * G * lv[1]);
    lam7[2] += lG * PX / g + w * (lv[9] + 2.0 * PX * lv[11] + X * lv[13]);
    lam7[3] += lG * PY / g + w * (lv[10] + 2.0 * PY * lv[12] + Y * lv[14]);
    lam7[4] += lG * PZ / g;
    lam7[5] += w * (lv[2] + 2.0 * XI * lv[3]);
    lam7[0] += w * (2.0 * X * lv[4] + lv[5] + 2.0 * X * lv[7] + PX * lv[13]);
    lam7[1] += w * (2.0 * Y * lv[4] + lv[6] + 2.0 * Y * lv[8] + PY * lv[14]);
}

/* ------------------------------------------------------------------ the whole run */
static void beams_save(const qzo_sim* s, double* out) {
    size_t off = 0;
    for (int b = 0; b < s->nb; ++b) {
        const beam_t* B = &s->bm[b];
        const double* cols[7] = {B->x, B->y, B->px, B->py, B->pz, B->xi, B->w};
        for (int c = 0; c < 7; ++c) { memcpy(out + off, cols[c], sizeof(double) * B->n); off += B->n; }
    }
}
static void beams_load(qzo_sim* s, const double* in) {
    size_t off = 0;
    for (int b = 0; b < s->nb; ++b) {
        beam_t* B = &s->bm[b];
        double* cols[7] = {B->x, B->y, B->px, B->py, B->pz, B->xi, B->w};
        for (int c = 0; c < 7; ++c) { memcpy(cols[c], in + off, sizeof(double) * B->n); off += B->n; }
    }
}

/* Runs nsteps like qzo_sim_run (from the sim's current beams, which must not have been pushed yet),
   then the adjoint: lamS (nb, 17) is the adjoint of the last step's moment sums; lam_out receives
   for every beam in order its (n, 7) rows (x y px py pz xi w) = d(J)/d(initial particle), where
   J = sum lamS * sums. mom (optional): the forward's moment sums ((nsteps + 1), nb, 17).
   Returns 0, or -2 when the deck is outside the adjoint's scope. The sim ends at the last step. */
int qzo_sim_adjoint(qzo_sim* s, int nsteps, double dt, const double* lamS, double* lam_out, double* mom) {
    if (s->m1 || nsteps < 1) return -2;
    int isp = -1;
    for (int i = 0; i < s->nsp; ++i)
        if (s->sp[i].p.mobile) { if (isp >= 0) return -2; isp = i; }
    if (isp < 0) return -2;
    for (int b = 0; b < s->nb; ++b)
        if (s->bm[b].started || s->bm[b].pusher != 0) return -2;
    size_t ntot = 0;
    for (int b = 0; b < s->nb; ++b) ntot += (size_t)s->bm[b].n;
    const size_t per = 7 * ntot;
    double* hist = (double*)malloc(sizeof(double) * per * (nsteps + 1));
    /* forward, keeping the beams of every step */
    for (int n = 0; n <= nsteps; ++n) {
        beams_save(s, hist + per * n);
        qzo_sim_step_fields(s, 0.0);
        if (mom)
            for (int b = 0; b < s->nb; ++b) qzo_sim_beam_sums(s, b, mom + ((size_t)n * s->nb + b) * 17);
        if (n < nsteps) qzo_sim_push_beams(s, dt, dt);
    }
    const int M = s->M, K = s->p.K;
    species_t* q = &s->sp[isp];
    const size_t nv = 6 + 5 * (size_t)s->p.ab_order;
    s->traj = (double*)malloc(sizeof(double) * (size_t)K * nv * q->cap);
    double* lfld = (double*)malloc(sizeof(double) * (size_t)K * M * 6);
    double* lbsrc = (double*)malloc(sizeof(double) * (size_t)K * M * 5);
    double* lam = (double*)calloc(per, sizeof(double));       /* (particle, 7) rows, beams in order */
    /* seed: the moment sums of the last step */
    {
        beams_load(s, hist + per * nsteps);
        size_t off = 0;
        for (int b = 0; b < s->nb; ++b) {
            for (long i = 0; i < s->bm[b].n; ++i) sums_back(&s->bm[b], i, lamS + 17 * b, lam + 7 * (off + i));
            off += s->bm[b].n;
        }
    }
    for (int n = nsteps - 1; n >= 0; --n) {
        beams_load(s, hist + per * n);
        qzo_sim_step_fields(s, 0.0);                  /* fields of step n, plasma trajectory recorded */
        memset(lfld, 0, sizeof(double) * (size_t)K * M * 6);
        memset(lbsrc, 0, sizeof(double) * (size_t)K * M * 5);
        size_t off = 0;
        for (int b = 0; b < s->nb; ++b) {
            const beam_t* B = &s->bm[b];
            if (!B->rigid)
                for (long i = 0; i < B->n; ++i) beam_push_back(s, B, i, dt, dt, n == 0, lam + 7 * (off + i), lfld);
            off += B->n;
        }
        sweep_back(s, isp, lfld, lbsrc);
        off = 0;
        for (int b = 0; b < s->nb; ++b) {
            for (long i = 0; i < s->bm[b].n; ++i) beam_deposit_back(s, &s->bm[b], i, lbsrc, lam + 7 * (off + i));
            off += s->bm[b].n;
        }
    }
    memcpy(lam_out, lam, sizeof(double) * per);
    free(s->traj);
    s->traj = NULL;
    /* leave the sim at the last step, as qzo_sim_run would */
    beams_load(s, hist + per * nsteps);
    for (int b = 0; b < s->nb; ++b) s->bm[b].started = !s->bm[b].rigid;
    qzo_sim_step_fields(s, 0.0);
    free(hist); free(lfld); free(lbsrc); free(lam);
    return 0;
}
