/* CPU restatement of REEF3D's level-set transport path.  TEST
 * INFRASTRUCTURE ONLY (see ls_oracle.h): the shipped library never links or
 * calls this file.  Every function cites the reference code it restates;
 * arithmetic is written in the reference's operation order so that, built
 * with -O2 -ffp-contract=off, results are bit-identical to the reference
 * compiled the same way (checked against oracle/_ref through
 * tests/golden/).
 */
#include "ls_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* the reference's truncated pi (src/definitions.h:37) */
#define LSO_PI 3.14159265359

#define MINV(a, b) ((a) < (b) ? (a) : (b))
#define MIN3V(a, b, c) (MINV(a, b) < (c) ? MINV(a, b) : (c))

long lso_index(const lso_grid* g, int i, int j, int k) {
    return (long)(i + LSO_MARGIN) * g->jmax * g->kmax + (long)(j + LSO_MARGIN) * g->kmax + (k + LSO_MARGIN);
}

/* ------------------------------------------------------------------ metrics
 * src/grid.cpp:55-100 (gridspacing): cell centres, node and centre spacing. */
static void spacing_1d(int n, const double* xn, double* xp, double* dxn, double* dxp) {
    for (int i = -LSO_MARGE; i < n + LSO_MARGE; ++i) {
        int t = i + LSO_MARGE;
        xp[t] = 0.5 * (xn[t] + xn[t + 1]);
        dxn[t] = xn[t + 1] - xn[t];
        dxp[t] = 0.5 * (xn[t + 2] + xn[t + 1]) - 0.5 * (xn[t + 1] + xn[t]);
    }
}

/* Non-uniform WENO5 node tables for one axis, index t = i+marge for
 * i = -1..n (src/weno_nug_func_precalc_qf.cpp:28-80,
 * src/weno_nug_func_precalc_cf.cpp:27-56,
 * src/weno_nug_func_precalc_isf.cpp:27-176; identical for x, y and z).
 * Layout qf[t][side*3+r][2], cf[t][side*3+r], isf[t][side*3+r][3] with
 * side 0 = upwind from the minus side, 1 = from the plus side. */
static void weno_tables_1d(int n, const double* X, double* qf, double* cf, double* isf) {
    for (int i = -1; i < n + 1; ++i) {
        const int t = i + LSO_MARGE;
        const double Xm2 = X[t - 2], Xm1 = X[t - 1], X0 = X[t], X1 = X[t + 1];
        const double X2 = X[t + 2], X3 = X[t + 3], X4 = X[t + 4];
        double* q = qf + (long)t * 12;
        double* c = cf + (long)t * 6;
        double* s = isf + (long)t * 18;
        double fac;

        q[0] = ((X2 - X1) / (X3 - X0)) * ((X3 - X1) / (X2 - X0));
        q[1] = ((X2 - X1) / (X3 - X0)) * ((X1 - X0) / (X3 - X1));
        q[2] = ((X1 - X0) / (X2 - Xm1)) * ((X1 - Xm1) / (X2 - X0));
        q[3] = ((X1 - X0) / (X2 - Xm1)) * ((X2 - X1) / (X1 - Xm1));
        q[4] = ((X1 - X0) / (X0 - Xm2)) * ((X1 - Xm1) / (X1 - Xm2));
        q[5] = (1.0 + (X1 - X0) / (X1 - Xm1) + (X1 - X0) / (X1 - Xm2));
        q[6] = (1.0 + (X2 - X1) / (X3 - X1) + (X2 - X1) / (X4 - X1));
        q[7] = ((X2 - X1) / (X4 - X1)) * ((X3 - X1) / (X4 - X2));
        q[8] = ((X2 - X1) / (X3 - X0)) * ((X3 - X1) / (X2 - X0));
        q[9] = ((X2 - X1) / (X3 - X0)) * ((X1 - X0) / (X3 - X1));
        q[10] = ((X1 - X0) / (X2 - Xm1)) * ((X1 - Xm1) / (X2 - X0));
        q[11] = ((X1 - X0) / (X2 - Xm1)) * ((X2 - X1) / (X1 - Xm1));

        c[0] = ((X1 - Xm2) / (X3 - Xm2)) * ((X1 - Xm1) / (X3 - Xm1));
        c[1] = ((X1 - Xm2) / (X3 - Xm2)) * ((X3 - X1) / (X3 - Xm1)) * ((X3 - Xm1) / (X2 - Xm2) + 1.0);
        c[2] = ((X2 - X1) / (X3 - Xm2)) * ((X3 - X1) / (X2 - Xm2));
        c[3] = ((X1 - X0) / (X4 - Xm1)) * ((X1 - Xm1) / (X4 - X0));
        c[4] = ((X1 - Xm1) / (X4 - Xm1)) * ((X4 - X1) / (X4 - X0)) * ((X4 - X0) / (X3 - Xm1) + 1.0);
        c[5] = ((X3 - X1) / (X4 - Xm1)) * ((X4 - X1) / (X3 - Xm1));

        /* minus side */
        fac = 4.0 * pow((X1 - X0) / (X3 - X0), 2.0);
        s[0] = fac * ((10.0 * pow(X1 - X0, 2.0) + (X2 - X0) * (X2 - X1)) / pow(X3 - X1, 2.0));
        s[1] = fac * ((20.0 * pow(X1 - X0, 2.0) + 2.0 * (X2 - X0) * (X2 - X1) + (X3 - X0) * (2.0 * X2 - X1 - X0)) /
                      ((X3 - X1) * (X2 - X0)));
        s[2] = fac * ((10.0 * pow(X1 - X0, 2.0) + (X3 + X2 - 2.0 * X0) * (X3 + X2 - X1 - X0)) / pow(X2 - X0, 2.0));

        fac = 4.0 * pow((X1 - X0) / (X2 - Xm1), 2.0);
        s[3] = fac * ((10.0 * pow(X1 - X0, 2.0) + (X2 - X0) * (X2 - X1)) / pow(X1 - Xm1, 2.0));
        s[4] = fac * ((20.0 * pow(X1 - X0, 2.0) - (X2 - X1) * (X0 - Xm1) - (X2 - X0) * (X1 - Xm1)) /
                      ((X2 - X0) * (X1 - Xm1)));
        s[5] = fac * ((10.0 * pow(X1 - X0, 2.0) + (X0 - Xm1) * (X1 - Xm1)) / pow(X2 - X0, 2.0));

        fac = 4.0 * pow((X1 - X0) / (X1 - Xm2), 2.0);
        s[6] = fac * ((10.0 * pow(X1 - X0, 2.0) + (X1 - Xm1) * (X0 - Xm1)) / pow(X0 - Xm2, 2.0));
        s[7] = fac * ((20.0 * pow(X1 - X0, 2.0) + 2.0 * (X1 - Xm1) * (X0 - Xm1) + (X1 - Xm2) * (X1 + X0 - 2.0 * Xm1)) /
                      ((X1 - Xm1) * (X0 - Xm2)));
        s[8] = fac * ((10.0 * pow(X1 - X0, 2.0) + (2.0 * X1 - Xm2 - Xm1) * (X1 + X0 - Xm1 - Xm2)) / pow(X1 - Xm1, 2.0));

        /* plus side */
        fac = 4.0 * pow((X2 - X1) / (X4 - X1), 2.0);
        s[9] = fac * ((10.0 * pow(X2 - X1, 2.0) + (X3 - X1) * (X3 - X2)) / pow(X4 - X2, 2.0));
        s[10] = fac * ((20.0 * pow(X2 - X1, 2.0) + 2.0 * (X3 - X1) * (X3 - X2) + (X4 - X1) * (2.0 * X3 - X2 - X1)) /
                       ((X4 - X2) * (X3 - X1)));
        s[11] = fac * ((10.0 * pow(X2 - X1, 2.0) + (X4 + X3 - 2.0 * X1) * (X4 + X3 - X2 - X1)) / pow(X3 - X1, 2.0));

        fac = 4.0 * pow((X2 - X1) / (X3 - X0), 2.0);
        s[12] = fac * ((10.0 * pow(X2 - X1, 2.0) + (X3 - X1) * (X3 - X2)) / pow(X2 - X0, 2.0));
        s[13] = fac * ((20.0 * pow(X2 - X1, 2.0) - (X3 - X2) * (X1 - X0) - (X3 - X1) * (X2 - X0)) /
                       ((X3 - X1) * (X2 - X0)));
        s[14] = fac * ((10.0 * pow(X2 - X1, 2.0) + (X1 - X0) * (X2 - X0)) / pow(X3 - X1, 2.0));

        fac = 4.0 * pow((X2 - X1) / (X2 - Xm1), 2.0);
        s[15] = fac * ((10.0 * pow(X2 - X1, 2.0) + (X2 - X0) * (X1 - X0)) / pow(X1 - Xm1, 2.0));
        s[16] = fac * ((20.0 * pow(X2 - X1, 2.0) + 2.0 * (X2 - X0) * (X1 - X0) + (X2 - Xm1) * (X2 + X1 - 2.0 * X0)) /
                       ((X2 - X0) * (X1 - Xm1)));
        s[17] = fac * ((10.0 * pow(X2 - X1, 2.0) + (2.0 * X2 - Xm1 - X0) * (X2 + X1 - X0 - Xm1)) / pow(X2 - X0, 2.0));
    }
}

int lso_grid_init(lso_grid* g, int nx, int ny, int nz, const double* xn, const double* yn,
                  const double* zn, double f43, int f44, double f45, int f49, double n47) {
    memset(g, 0, sizeof(*g));
    if (nx < 1 || ny < 1 || nz < 1) return -1;
    g->nx = nx; g->ny = ny; g->nz = nz;
    g->jdir = ny > 1 ? 1 : 0;
    g->imax = nx + 2 * LSO_MARGIN;
    g->jmax = ny + 2 * LSO_MARGIN;
    g->kmax = nz + 2 * LSO_MARGIN;
    g->ncell = (long)g->imax * g->jmax * g->kmax;
    g->f43 = f43; g->f44 = f44; g->f45 = f45; g->f49 = f49; g->n47 = n47;
    int n[3] = {nx, ny, nz};
    const double* src[3] = {xn, yn, zn};
    double** nodes[3] = {&g->xn, &g->yn, &g->zn};
    double** cp[3] = {&g->xp, &g->yp, &g->zp};
    double** dn[3] = {&g->dxn, &g->dyn, &g->dzn};
    double** dp[3] = {&g->dxp, &g->dyp, &g->dzp};
    for (int a = 0; a < 3; ++a) {
        long len = n[a] + 1 + 4 * LSO_MARGE;  /* src/read_grid.cpp:404-406 */
        *nodes[a] = (double*)calloc(len, sizeof(double));
        *cp[a] = (double*)calloc(len, sizeof(double));
        *dn[a] = (double*)calloc(len, sizeof(double));
        *dp[a] = (double*)calloc(len, sizeof(double));
        memcpy(*nodes[a], src[a], sizeof(double) * (n[a] + 1 + 2 * LSO_MARGE));
        spacing_1d(n[a], *nodes[a], *cp[a], *dn[a], *dp[a]);
        g->qf[a] = (double*)calloc((long)(n[a] + 8) * 12, sizeof(double));
        g->cf[a] = (double*)calloc((long)(n[a] + 8) * 6, sizeof(double));
        g->isf[a] = (double*)calloc((long)(n[a] + 8) * 18, sizeof(double));
        weno_tables_1d(n[a], *nodes[a], g->qf[a], g->cf[a], g->isf[a]);
    }
    /* header means (first spacing) and the gridspacing mean
     * (src/grid.cpp:102-148, one rank) */
    g->dxm = xn[LSO_MARGE + 1] - xn[LSO_MARGE];
    g->dym = yn[LSO_MARGE + 1] - yn[LSO_MARGE];
    g->dzm = zn[LSO_MARGE + 1] - zn[LSO_MARGE];
    {
        double m = 0.0;
        int count = 0;
        for (int i = 0; i < nx; ++i) { m += g->dxp[i + LSO_MARGE]; ++count; }
        if (g->jdir == 1)
            for (int j = 0; j < ny; ++j) { m += g->dyp[j + LSO_MARGE]; ++count; }
        for (int k = 0; k < nz; ++k) { m += g->dzp[k + LSO_MARGE]; ++count; }
        m /= (double)count;
        g->dxm_mean = m;
    }
    /* src/ini_psi.cpp:33-37 (DXM is the gridspacing mean by then) */
    if (g->jdir == 0) g->psi = g->f45 * (1.0 / 2.0) * (g->dxm_mean + g->dzm);
    else g->psi = g->f45 * (1.0 / 3.0) * (g->dxm_mean + g->dym + g->dzm);
    return 0;
}

void lso_grid_free(lso_grid* g) {
    double* p[] = {g->xn, g->yn, g->zn, g->xp, g->yp, g->zp, g->dxn, g->dyn, g->dzn, g->dxp, g->dyp, g->dzp};
    for (unsigned t = 0; t < sizeof(p) / sizeof(p[0]); ++t) free(p[t]);
    for (int a = 0; a < 3; ++a) { free(g->qf[a]); free(g->cf[a]); free(g->isf[a]); }
    memset(g, 0, sizeof(*g));
}

/* ------------------------------------------------------------ WENO5 kernel
 * One-axis WENO5 derivative from the five divided differences q1..q5 of the
 * upwind set, with the node tables of index t.
 *   minus side (upwind from the left): IS src/weno_nug_func.h:48-60,
 *     weights :133-143, reconstruction src/weno_hj_df_nug.cpp:155-159;
 *   plus side: IS :61-73, weights :144-153, reconstruction :186-190.
 * epsilon = 0, psi = 1e-6 (src/weno_nug_func.cpp:26). */
static double weno_axis(const double* qf, const double* cf, const double* isf, int t, int plus,
                        double q1, double q2, double q3, double q4, double q5) {
    const double psi = 1.0e-6, eps = 0.0;
    const double* Q = qf + (long)t * 12 + (plus ? 6 : 0);
    const double* C = cf + (long)t * 6 + (plus ? 3 : 0);
    const double* S = isf + (long)t * 18 + (plus ? 9 : 0);
    const double dq12 = q1 - q2, dq23 = q2 - q3, dq32 = q3 - q2;
    const double dq34 = q3 - q4, dq43 = q4 - q3, dq54 = q5 - q4;
    const double is1 = S[0] * dq54 * dq54 + S[1] * (dq54) * (dq34) + S[2] * dq34 * dq34;
    const double is2 = S[3] * dq23 * dq23 + S[4] * (dq43) * (dq23) + S[5] * dq43 * dq43;
    const double is3 = S[6] * dq12 * dq12 + S[7] * (dq32) * (dq12) + S[8] * dq32 * dq32;
    const double a = is1 + psi, b = is2 + psi, c = is3 + psi;
    const double w1 = C[0] / (eps + (a * a) * (C[0] / (a * a) + C[1] / (b * b) + C[2] / (c * c)));
    const double w2 = C[1] / (eps + (b * b) * (C[0] / (a * a) + C[1] / (b * b) + C[2] / (c * c)));
    const double w3 = C[2] / (eps + (c * c) * (C[0] / (a * a) + C[1] / (b * b) + C[2] / (c * c)));
    if (!plus)
        return w1 * (q4 + Q[0] * (q3 - q4) - Q[1] * (q5 - q4))
             + w2 * (q3 + Q[2] * (q4 - q3) - Q[3] * (q2 - q3))
             + w3 * (q2 + Q[4] * (q1 - q2) + Q[5] * (q3 - q2));
    return w1 * (q4 + Q[0] * (q3 - q4) + Q[1] * (q5 - q4))
         + w2 * (q3 + Q[2] * (q2 - q3) - Q[3] * (q4 - q3))
         + w3 * (q2 + Q[4] * (q3 - q2) - Q[5] * (q1 - q2));
}

/* Upwind-biased derivative of f along one axis at the cell with linear
 * index c and stride s, axis metric dp (DXP-like) and table index t:
 * minus stencil src/weno_hj_df_nug.cpp:344-351, plus stencil :371-378 (the
 * same stencils as src/ddweno_nug_sf.cpp:225-277). */
static double weno_deriv(const double* f, long c, long s, const double* dp, const double* qf,
                         const double* cf, const double* isf, int t, int plus) {
    double q1, q2, q3, q4, q5;
    if (!plus) {
        q1 = (f[c - 2 * s] - f[c - 3 * s]) / dp[t - 3];
        q2 = (f[c - s] - f[c - 2 * s]) / dp[t - 2];
        q3 = (f[c] - f[c - s]) / dp[t - 1];
        q4 = (f[c + s] - f[c]) / dp[t];
        q5 = (f[c + 2 * s] - f[c + s]) / dp[t + 1];
    } else {
        q1 = (f[c - s] - f[c - 2 * s]) / dp[t - 2];
        q2 = (f[c] - f[c - s]) / dp[t - 1];
        q3 = (f[c + s] - f[c]) / dp[t];
        q4 = (f[c + 2 * s] - f[c + s]) / dp[t + 1];
        q5 = (f[c + 3 * s] - f[c + 2 * s]) / dp[t + 2];
    }
    return weno_axis(qf, cf, isf, t, plus, q1, q2, q3, q4, q5);
}

/* Direct-forcing divided difference of the cell pair (a, b = a + s) of the
 * X45 stencils (src/weno_hj_df_nug.cpp:398-987; the i, j, k variants and
 * both sides follow one rule per X45): 1 zero unless |fb| > 0.6 DXM at both
 * cells, 2 weighted by the mean fbh5 of the pair, 3 zero unless fbh4 < 0.5
 * at both, 4 weighted by fbh5 at the cell `w` (the pair's lower cell on the
 * minus side, its upper cell on the plus side), 5 zero unless solid > 0 and
 * topo > 0 at both, 6 like 3 but 1e20 where masked. */
static double df_q(const lso_grid* g, const double* f, long a, long b, long w, double d) {
    const double* h = g->body1;
    switch (g->x45) {
        case 1:
            if (fabs(h[b]) > 0.6 * g->dxm_mean && fabs(h[a]) > 0.6 * g->dxm_mean) return (f[b] - f[a]) / d;
            return 0.0;
        case 2: return 0.5 * (h[b] + h[a]) * (f[b] - f[a]) / d;
        case 3:
            if (h[b] < 0.5 && h[a] < 0.5) return (f[b] - f[a]) / d;
            return 0.0;
        case 4: return (h[w]) * (f[b] - f[a]) / d;
        case 5:
            if (h[b] > 0.0 && g->body2[b] > 0.0 && h[a] > 0.0 && g->body2[a] > 0.0) return (f[b] - f[a]) / d;
            return 0.0;
        case 6:
            if (h[b] < 0.5 && h[a] < 0.5) return (f[b] - f[a]) / d;
            return 1.0e20;
        default: return (f[b] - f[a]) / d;
    }
}

/* weno_deriv with the X45 differences: q_m from the pair (m-1, m) of the
 * six upwind points. */
static double weno_deriv_df(const lso_grid* g, const double* f, long c, long s, const double* dp, const double* qf,
                            const double* cf, const double* isf, int t, int plus) {
    const int o = plus ? -2 : -3;
    double q[5];
    for (int m = 1; m <= 5; ++m) {
        const long a = c + (o + m - 1) * s, b = c + (o + m) * s;
        q[m - 1] = df_q(g, f, a, b, plus ? b : a, dp[t + o + m - 1]);
    }
    return weno_axis(qf, cf, isf, t, plus, q[0], q[1], q[2], q[3], q[4]);
}

/* ghostcell::solid_forcing_lsm (src/gc_solid_forcing_lsm.cpp:27-78): for
 * each entry in list order with side > 0, the two cells beyond the side
 * take the entry cell's value. */
static void solid_forcing(const lso_grid* g, double* f) {
    for (int n = 0; n < g->nsf; ++n) {
        const int* e = g->sf + 4 * n;
        const int i = e[0], j = e[1], k = e[2], side = e[3];
        if (side <= 0) continue;
        const double v = f[lso_index(g, i, j, k)];
        if (side == 1) { f[lso_index(g, i - 1, j, k)] = v; f[lso_index(g, i - 2, j, k)] = v; }
        if (side == 4) { f[lso_index(g, i + 1, j, k)] = v; f[lso_index(g, i + 2, j, k)] = v; }
        if (side == 3) { f[lso_index(g, i, j - 1, k)] = v; f[lso_index(g, i, j - 2, k)] = v; }
        if (side == 2) { f[lso_index(g, i, j + 1, k)] = v; f[lso_index(g, i, j + 2, k)] = v; }
        if (side == 5) { f[lso_index(g, i, j, k - 1)] = v; f[lso_index(g, i, j, k - 2)] = v; }
        if (side == 6) { f[lso_index(g, i, j, k + 1)] = v; f[lso_index(g, i, j, k + 2)] = v; }
    }
}

void lso_set_solid_forcing(lso_grid* g, int n, const int* cells) {
    g->nsf = n;
    g->sf = cells;
}

void lso_set_direct_forcing(lso_grid* g, int x45, const double* body1, const double* body2) {
    g->x45 = x45;
    g->body1 = body1;
    g->body2 = body2;
}

/* ------------------------------------------------------------- convection
 * src/weno_hj_df_nug.cpp:84-111 (ipol 4) with the cell-centre velocities of
 * src/flux_HJ_CDS2.cpp:59-64,90-95,122-127 (2D: src/flux_HJ_CDS2_2D.cpp,
 * no y term). */
void lso_weno_L(const lso_grid* g, const double* phi, const double* u, const double* v,
                const double* w, double* L) {
    const long si = (long)g->jmax * g->kmax, sj = g->kmax, sk = 1;
#define DERIV(...) (g->x45 ? weno_deriv_df(g, __VA_ARGS__) : weno_deriv(__VA_ARGS__))
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const long c = lso_index(g, i, j, k);
                const double iadvec = 0.5 * (u[c] + u[c - si]);
                const double jadvec = 0.5 * (v[c] + v[c - sj]);
                const double kadvec = 0.5 * (w[c] + w[c - sk]);
                double grad, l;
                grad = 0.0;
                if (iadvec > 0.0) grad = DERIV(phi, c, si, g->dxp, g->qf[0], g->cf[0], g->isf[0], i + LSO_MARGE, 0);
                if (iadvec < 0.0) grad = DERIV(phi, c, si, g->dxp, g->qf[0], g->cf[0], g->isf[0], i + LSO_MARGE, 1);
                l = -iadvec * grad;
                if (g->jdir == 1) {
                    grad = 0.0;
                    if (jadvec > 0.0) grad = DERIV(phi, c, sj, g->dyp, g->qf[1], g->cf[1], g->isf[1], j + LSO_MARGE, 0);
                    if (jadvec < 0.0) grad = DERIV(phi, c, sj, g->dyp, g->qf[1], g->cf[1], g->isf[1], j + LSO_MARGE, 1);
                    l -= jadvec * grad;
                }
                grad = 0.0;
                if (kadvec > 0.0) grad = DERIV(phi, c, sk, g->dzp, g->qf[2], g->cf[2], g->isf[2], k + LSO_MARGE, 0);
                if (kadvec < 0.0) grad = DERIV(phi, c, sk, g->dzp, g->qf[2], g->cf[2], g->isf[2], k + LSO_MARGE, 1);
                l -= kadvec * grad;
                L[c] = 0.0;
                L[c] += l;  /* a->L(i,j,k) += aij(...) on a zeroed L */
            }
#undef DERIV
}

/* --------------------------------------------------------- reinitialisation
 * src/reinidisc_f.cpp:58-127 (F49=1, every cell) and
 * src/reinidisc_fsf.cpp:66-141 (F49=0, only cells whose 7-point stencil has
 * one sign; the others keep L=0). */
static double reini_cell(const lso_grid* g, const double* f, int i, int j, int k) {
    const long si = (long)g->jmax * g->kmax, sj = g->kmax, sk = 1;
    const long c = lso_index(g, i, j, k);
    const int ti = i + LSO_MARGE, tj = j + LSO_MARGE, tk = k + LSO_MARGE;
    double dx = 0.0, dy = 0.0, dz = 0.0;
    const double lsv = f[c];
    double lsSig = lsv / sqrt(lsv * lsv);
    if (fabs(lsv) < 1.0e-8) lsSig = 1.0;

    double xmin = (lsv - f[c - si]) / g->dxp[ti - 1];
    double xplus = (f[c + si] - lsv) / g->dxp[ti];
    if (xmin * lsSig > 0.0 && xplus * lsSig > -xmin * lsSig)
        dx = weno_deriv(f, c, si, g->dxp, g->qf[0], g->cf[0], g->isf[0], ti, 0);
    if (xplus * lsSig < 0.0 && xmin * lsSig < -xplus * lsSig)
        dx = weno_deriv(f, c, si, g->dxp, g->qf[0], g->cf[0], g->isf[0], ti, 1);
    if (xplus * lsSig > 0.0 && xmin * lsSig < 0.0) dx = 0.0;

    if (g->jdir == 1) {
        double ymin = (lsv - f[c - sj]) / g->dyp[tj - 1];
        double yplus = (f[c + sj] - lsv) / g->dyp[tj];
        if (ymin * lsSig > 0.0 && yplus * lsSig > -ymin * lsSig)
            dy = weno_deriv(f, c, sj, g->dyp, g->qf[1], g->cf[1], g->isf[1], tj, 0);
        if (yplus * lsSig < 0.0 && ymin * lsSig < -yplus * lsSig)
            dy = weno_deriv(f, c, sj, g->dyp, g->qf[1], g->cf[1], g->isf[1], tj, 1);
        if (yplus * lsSig > 0.0 && ymin * lsSig < 0.0) dy = 0.0;
    }

    double zmin = (lsv - f[c - sk]) / g->dzp[tk - 1];
    double zplus = (f[c + sk] - lsv) / g->dzp[tk];
    if (zmin * lsSig > 0.0 && zplus * lsSig > -zmin * lsSig)
        dz = weno_deriv(f, c, sk, g->dzp, g->qf[2], g->cf[2], g->isf[2], tk, 0);
    if (zplus * lsSig < 0.0 && zmin * lsSig < -zplus * lsSig)
        dz = weno_deriv(f, c, sk, g->dzp, g->qf[2], g->cf[2], g->isf[2], tk, 1);
    if (zplus * lsSig > 0.0 && zmin * lsSig < 0.0) dz = 0.0;

    const double dnorm = sqrt(dx * dx + dy * dy + dz * dz);
    double deltax;
    if (g->jdir == 0) deltax = (1.0 / 2.0) * (g->dxn[ti] + g->dzn[tk]);
    else deltax = (1.0 / 3.0) * (g->dxn[ti] + g->dyn[tj] + g->dzn[tk]);
    double sign = lsv / sqrt(lsv * lsv + dnorm * dnorm * deltax * deltax);
    if (sign != sign) sign = 1.0;
    return -(sign * dnorm - sign);
}

/* F49=0 interface test (src/reinidisc_fsf.cpp:70-72).  In 2D the y
 * neighbours are ghost cells of the degenerate axis that nothing on the path
 * writes; they read as stored (zero in every field the reference allocates). */
static int same_sign_stencil(const lso_grid* g, const double* f, long c) {
    const long si = (long)g->jmax * g->kmax, sj = g->kmax, sk = 1;
    return (f[c] >= 0.0 && f[c + si] >= 0.0 && f[c - si] >= 0.0 && f[c + sj] >= 0.0 && f[c - sj] >= 0.0 &&
            f[c + sk] >= 0.0 && f[c - sk] >= 0.0) ||
           (f[c] < 0.0 && f[c + si] < 0.0 && f[c - si] < 0.0 && f[c + sj] < 0.0 && f[c - sj] < 0.0 &&
            f[c + sk] < 0.0 && f[c - sk] < 0.0);
}

void lso_reinidisc_L(const lso_grid* g, const double* f, double* L) {
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const long c = lso_index(g, i, j, k);
                L[c] = 0.0;
                if (g->f49 == 1 || same_sign_stencil(g, f, c)) L[c] = reini_cell(g, f, i, j, k);
            }
}

/* --------------------------------------------------------------- ghost fill
 * ghostcell::start4 for the level set on wall faces: gceval4 maps walls to
 * gclabel_lsm=4 (src/gc_epol4.cpp:26-31, src/ghostcell.cpp:116), i.e. the
 * Neumann copy of src/gc_neumann.cpp:29-54 into the three face ghost layers.
 * 2D skips the y sides (src/gc_neumann.cpp:34-40). */
/* Ghost label of an x face for the level-set gcval 50+f50
 * (src/gc_epol4.cpp:26-58): walls (type 21) always 4 (Neumann copy);
 * inflow (type 1) 4 for gcv 52/54, else 0 (untouched); outflow (type 2) 4
 * for gcv 51/54 and for 52 with B77 = 1, else 0. */
static int x_face_filled(const lso_grid* g, int side) {
    if (!g->io_on) return 1;
    const int gcv = 50 + g->f50;
    if (side == 1 && g->io_in) return gcv == 52 || gcv == 54;
    if (side == 4 && g->io_out) return gcv == 51 || gcv == 54 || (gcv == 52 && g->b77 == 1);
    return 1;
}

static void ghost_fill_gcv(const lso_grid* g, double* f, int level_set);

void lso_ghost_fill(const lso_grid* g, double* f) { ghost_fill_gcv(g, f, 1); }

/* level_set 0: gcval 1 of ro/visc, a Neumann copy on every face
 * (src/gc_epol4.cpp:90-93), whatever the boundary type. */
static void ghost_fill_gcv(const lso_grid* g, double* f, int level_set) {
    const int fill_lo = !level_set || x_face_filled(g, 1), fill_hi = !level_set || x_face_filled(g, 4);
    for (int j = 0; j < g->ny; ++j)
        for (int k = 0; k < g->nz; ++k)
            for (int q = 0; q < LSO_MARGIN; ++q) {
                if (fill_lo) f[lso_index(g, -q - 1, j, k)] = f[lso_index(g, 0, j, k)];
                if (fill_hi) f[lso_index(g, g->nx + q, j, k)] = f[lso_index(g, g->nx - 1, j, k)];
            }
    if (g->jdir == 1)
        for (int i = 0; i < g->nx; ++i)
            for (int k = 0; k < g->nz; ++k)
                for (int q = 0; q < LSO_MARGIN; ++q) {
                    f[lso_index(g, i, -q - 1, k)] = f[lso_index(g, i, 0, k)];
                    f[lso_index(g, i, g->ny + q, k)] = f[lso_index(g, i, g->ny - 1, k)];
                }
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int q = 0; q < LSO_MARGIN; ++q) {
                f[lso_index(g, i, j, -q - 1)] = f[lso_index(g, i, j, 0)];
                f[lso_index(g, i, j, g->nz + q)] = f[lso_index(g, i, j, g->nz - 1)];
            }
    /* With an inflow face, fsfinflow reads the edge ghost (-1, j, nz) above
     * the top inflow cell; start4 leaves there the copy of cell (0, j, nz-1)
     * that dgcpol4 writes into the first diagonal ghost layer
     * (src/gc_dgcpol4.cpp:28-50, Y40 = 3). */
    if (level_set && g->io_on && g->io_in)
        for (int j = 0; j < g->ny; ++j) f[lso_index(g, -1, j, g->nz)] = f[lso_index(g, 0, j, g->nz - 1)];
}

/* ------------------------------------------------------------ ioflow hooks
 * ioflow_f::fsfinflow (src/ioflow_waterlevel.cpp:29-141): the water level
 * at the inflow from the zero crossings of the first ghost column over the
 * inflow cells (list order: j outer, k inner, the order of the boundary
 * list), imposed on the inflow ghosts for F50 = 2 or 4; the outflow level
 * from the last interior column; with F62 set and B77 = 2 the outflow
 * ghosts take the (ramped) outflow level. */
static void io_fsfinflow(lso_grid* g, double* phi) {
    g->phimean = g->f56;
    if (g->f60 > -1.0e20) { g->phimean = g->f60; g->phiout = g->f60; }
    if (g->f62 > -1.0e20) g->phiout = g->f62;
    int count = 0;
    double zval = 0.0;
    if (g->io_in) {
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const double a = phi[lso_index(g, -1, j, k)], b = phi[lso_index(g, -1, j, k + 1)];
                if (a >= 0.0 && b < 0.0) {
                    zval += -(a * g->dzp[k + LSO_MARGE]) / (b - a) + g->zp[k + LSO_MARGE];
                    ++count;
                }
            }
        if (count > 0) {
            g->phimean = zval / (double)count;
            if (g->f50 == 2 || g->f50 == 4)
                for (int j = 0; j < g->ny; ++j)
                    for (int k = 0; k < g->nz; ++k)
                        for (int q = 1; q <= 3; ++q) phi[lso_index(g, -q, j, k)] = g->phimean - g->zp[k + LSO_MARGE];
        }
    }
    count = 0;
    zval = 0.0;
    if (g->io_out) {
        const int i = g->nx - 1;
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const double a = phi[lso_index(g, i, j, k)], b = phi[lso_index(g, i, j, k + 1)];
                if (a >= 0.0 && b < 0.0) {
                    zval += -(a * g->dzp[k + LSO_MARGE]) / (b - a) + g->zp[k + LSO_MARGE];
                    ++count;
                }
            }
        if (count > 0) g->phiout = zval / (double)count;
    }
    double wsfout = g->phimean;
    if (g->f62 > 1.0e-20) {
        if (g->f64 == 0) wsfout = g->f62;
        if (g->f64 > 0) {
            double f = 1.0;
            if (g->count < g->f64) f = 0.5 * cos(LSO_PI + LSO_PI * (double)g->count / (double)g->f64) + 0.5;
            wsfout = f * g->f62 + (1.0 - f) * g->f60;
        }
    }
    if (g->io_out && g->f62 > -1.0e20 && g->b77 == 2)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k)
                for (int q = 1; q <= 3; ++q) phi[lso_index(g, g->nx - 1 + q, j, k)] = wsfout - g->zp[k + LSO_MARGE];
}

/* ioflow_f::fsfrkin and fsfrkout (src/ioflow_waterlevel.cpp:143-177): the
 * RK buffer's inflow ghosts copy phi's; its outflow ghosts copy phi's, or
 * hold F62 - z with F62 set and B77 = 2. */
static void io_fsfrk(const lso_grid* g, const double* phi, double* f) {
    if (!g->io_on) return;
    for (int j = 0; j < g->ny; ++j)
        for (int k = 0; k < g->nz; ++k)
            for (int q = 1; q <= 3; ++q) {
                if (g->io_in) f[lso_index(g, -q, j, k)] = phi[lso_index(g, -q, j, k)];
                if (g->io_out) {
                    const long c = lso_index(g, g->nx - 1 + q, j, k);
                    if (g->f62 < -1.0e19 || g->b77 != 2) f[c] = phi[c];
                    if (g->f62 > -1.0e20 && g->b77 == 2) f[c] = g->f62 - g->zp[k + LSO_MARGE];
                }
            }
}

/* iowave::fsfrkin / fsfrkout (src/iowave_waterlevel.cpp:37-63): the RK
 * buffer's inflow and outflow ghosts copy phi's. */
static void io_fsfrk_waves(const lso_grid* g, const double* phi, double* f) {
    for (int j = 0; j < g->ny; ++j)
        for (int k = 0; k < g->nz; ++k)
            for (int q = 1; q <= 3; ++q) {
                if (g->io_in) f[lso_index(g, -q, j, k)] = phi[lso_index(g, -q, j, k)];
                if (g->io_out) {
                    const long c = lso_index(g, g->nx - 1 + q, j, k);
                    f[c] = phi[c];
                }
            }
}

/* iowave::phi_relax (src/iowave_relax.cpp:346-378) over LOOP (i, j, k): the
 * generation zone (distgen < 1e20) blends towards ramp * lsval[count] with
 * count running over the zone's cells in LOOP order, then the beach
 * (distbeach < 1e20) towards phimean - z. */
static void phi_relax(const lso_grid* g, double* f) {
    if (!g->rz_wg && !g->rz_wb) return;
    long count = 0;
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const long c = lso_index(g, i, j, k);
                const double wg = g->rz_wg ? g->rz_wg[(long)i * g->ny + j] : -1.0;
                const double wb = g->rz_wb ? g->rz_wb[(long)i * g->ny + j] : -1.0;
                if (wg >= 0.0) {
                    f[c] = (1.0 - wg) * g->rz_ramp * g->rz_lsval[count] + wg * f[c];
                    ++count;
                }
                if (wb >= 0.0) f[c] = (1.0 - wb) * (g->rz_phimean - g->zp[k + LSO_MARGE]) + wb * f[c];
            }
}

void lso_set_io_waves(lso_grid* g, int on) { g->io_waves = on; }

void lso_set_relaxation(lso_grid* g, const double* wg, const double* wb, double phimean) {
    g->rz_wg = wg;
    g->rz_wb = wb;
    g->rz_phimean = phimean;
}

void lso_set_relaxation_target(lso_grid* g, const double* lsval, double ramp) {
    g->rz_lsval = lsval;
    g->rz_ramp = ramp;
}

void lso_set_ioflow(lso_grid* g, int inflow, int outflow, int f50, int b77, double f56, double f60, double f61,
                    double f62, int f64, double qi, double qo) {
    g->io_on = 1;
    g->io_in = inflow;
    g->io_out = outflow;
    g->f50 = f50;
    g->b77 = b77;
    g->f56 = f56;
    g->f60 = f60;
    g->f61 = f61;
    g->f62 = f62;
    g->f64 = f64;
    g->qi = qi;
    g->qo = qo;
}

void lso_io_levels(const lso_grid* g, double* out) {
    out[0] = g->phimean;
    out[1] = g->phiout;
}

void lso_set_count(lso_grid* g, int count) { g->count = count - 1; }

/* reinit pseudo time step per cell (src/reini_RK3.cpp:150-160) */
static double reini_dt(const lso_grid* g, int i, int j, int k) {
    const int ti = i + LSO_MARGE, tj = j + LSO_MARGE, tk = k + LSO_MARGE;
    if (g->jdir == 0) return g->f43 * MINV(g->dxp[ti], g->dzp[tk]);
    return g->f43 * MIN3V(g->dxp[ti], g->dyp[tj], g->dzp[tk]);
}

/* --------------------------------------------------- picard mass correction
 * src/picard_f.cpp:36-56 (volcalc, volcalc2): volume of the smoothed
 * Heaviside with epsi = F45*DXM and cell volume DXM^3, LOOP order. */
static double picard_volume(const lso_grid* g, const double* f) {
    const double epsi = g->f45 * g->dxm_mean;
    double vol = 0.0, H = 0.0;
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const double b = f[lso_index(g, i, j, k)];
                if (b > epsi) H = 1.0;
                if (b < -epsi) H = 0.0;
                if (fabs(b) <= epsi) H = 0.5 * (1.0 + b / epsi + (1.0 / LSO_PI) * sin((LSO_PI * b) / epsi));
                vol += pow(g->dxm_mean, 3.0) * H;
            }
    return vol;
}

/* src/picard_f.cpp:82-113 (correct_ls): F47 uniform shifts of the interior
 * by the difference of the equivalent-sphere radii; ghosts untouched. */
static void picard_correct(const lso_grid* g, double* f, double vol1) {
    for (int n = 0; n < g->f47; ++n) {
        const double vol2 = picard_volume(g, f);
        const double r1 = pow((0.75 / LSO_PI) * vol1, 1.0 / 3.0);
        const double r2 = pow((0.75 / LSO_PI) * vol2, 1.0 / 3.0);
        const double w = r1 - r2;
        for (int i = 0; i < g->nx; ++i)
            for (int j = 0; j < g->ny; ++j)
                for (int k = 0; k < g->nz; ++k) f[lso_index(g, i, j, k)] += w;
    }
}

void lso_set_picard(lso_grid* g, int f46, int f47) {
    g->f46 = f46;
    g->f47 = f47;
    g->count = 0;
    g->netvol = 0.0;
}

/* src/reini_RK3.cpp:113-138 (with picard_f when F46=1, :92 and :140) */
void lso_reini(const lso_grid* g, double* f, double* a1, double* a2, double* L, int iters) {
    const double vol1 = g->f46 == 1 ? picard_volume(g, f) : 0.0;
    if (g->io_on && g->io_waves) {
        io_fsfrk_waves(g, f, a1);
        io_fsfrk_waves(g, f, a2);
    } else {
        io_fsfrk(g, f, a1);
        io_fsfrk(g, f, a2);
    }
    for (int q = 0; q < iters; ++q) {
        lso_reinidisc_L(g, f, L);
        for (int i = 0; i < g->nx; ++i)
            for (int j = 0; j < g->ny; ++j)
                for (int k = 0; k < g->nz; ++k) {
                    const long c = lso_index(g, i, j, k);
                    a1[c] = f[c] + reini_dt(g, i, j, k) * L[c];
                }
        lso_ghost_fill(g, a1);
        lso_reinidisc_L(g, a1, L);
        for (int i = 0; i < g->nx; ++i)
            for (int j = 0; j < g->ny; ++j)
                for (int k = 0; k < g->nz; ++k) {
                    const long c = lso_index(g, i, j, k);
                    a2[c] = 0.75 * f[c] + 0.25 * a1[c] + 0.25 * reini_dt(g, i, j, k) * L[c];
                }
        lso_ghost_fill(g, a2);
        lso_reinidisc_L(g, a2, L);
        for (int i = 0; i < g->nx; ++i)
            for (int j = 0; j < g->ny; ++j)
                for (int k = 0; k < g->nz; ++k) {
                    const long c = lso_index(g, i, j, k);
                    f[c] = (1.0 / 3.0) * f[c] + (2.0 / 3.0) * a2[c] + (2.0 / 3.0) * reini_dt(g, i, j, k) * L[c];
                }
        lso_ghost_fill(g, f);
    }
    if (g->f46 == 1) picard_correct(g, f, vol1);
}

/* src/levelset_RK3.cpp:112-161 then reini_RK3::start (F44 steps), with
 * picard_f around them when F46=2 (:110 and :171).  F46=3 (picard_lsm,
 * src/picard_lsm.cpp:36-116): the target volume is the one of the first step
 * (count == 1), carried as netvol; netvol += Qi*dt - Qo*dt (zero discharges
 * for the closed box).  g->count counts the steps like lexer::count.  With
 * inflow / outflow faces the ioflow_f hooks run first (:105-109). */
void lso_ls_step(lso_grid* g, double* phi, const double* u, const double* v, const double* w,
                 double dt, double* a1, double* a2, double* L) {
    g->count += 1;
    if (g->io_on && g->io_waves) {
        io_fsfrk_waves(g, phi, a1);
        io_fsfrk_waves(g, phi, a2);
    } else if (g->io_on) {
        io_fsfinflow(g, phi);
        io_fsfrk(g, phi, a1);
        io_fsfrk(g, phi, a2);
    }
    double vol1 = g->f46 >= 2 ? picard_volume(g, phi) : 0.0;
    if (g->f46 == 3) {
        if (g->count == 1) g->netvol = vol1;
        g->netvol = g->netvol + g->qi * dt - g->qo * dt;
    }
    lso_weno_L(g, phi, u, v, w, L);
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const long c = lso_index(g, i, j, k);
                a1[c] = phi[c] + dt * L[c];
            }
    phi_relax(g, a1);
    lso_ghost_fill(g, a1);
    solid_forcing(g, a1);
    lso_weno_L(g, a1, u, v, w, L);
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const long c = lso_index(g, i, j, k);
                a2[c] = 0.75 * phi[c] + 0.25 * a1[c] + 0.25 * dt * L[c];
            }
    phi_relax(g, a2);
    lso_ghost_fill(g, a2);
    solid_forcing(g, a2);
    lso_weno_L(g, a2, u, v, w, L);
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const long c = lso_index(g, i, j, k);
                phi[c] = (1.0 / 3.0) * phi[c] + (2.0 / 3.0) * a2[c] + (2.0 / 3.0) * dt * L[c];
            }
    phi_relax(g, phi);
    lso_ghost_fill(g, phi);
    solid_forcing(g, phi);
    lso_reini(g, phi, a1, a2, L, g->f44);
    if (g->f46 == 2) picard_correct(g, phi, vol1);
    if (g->f46 == 3) picard_correct(g, phi, g->netvol);
}

/* src/fluid_update_fsf.cpp:50-74 (porosity 1, every interior cell) */
void lso_volume(const lso_grid* g, const double* phi, double* vol1, double* vol2) {
    double v1 = 0.0, v2 = 0.0, H = 0.0;
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const double p = phi[lso_index(g, i, j, k)];
                if (p > g->psi) H = 1.0;
                if (p < -g->psi) H = 0.0;
                if (fabs(p) <= g->psi) H = 0.5 * (1.0 + p / g->psi + (1.0 / LSO_PI) * sin((LSO_PI * p) / g->psi));
                const double vol = g->dxn[i + LSO_MARGE] * g->dyn[j + LSO_MARGE] * g->dzn[k + LSO_MARGE];
                v1 += vol * (H - (1.0 - 1.0));
                v2 += vol * (1.0 - H - (1.0 - 1.0));
            }
    *vol1 = v1;
    *vol2 = v2;
}

/* src/fluid_update_fsf.cpp:39-104: density and viscosity from the smoothed
 * Heaviside on every interior cell (BASELOOP), then the wall ghost fill of
 * both (gcval 1, a Neumann copy like the level set's, src/gc_epol4.cpp:90-93).
 * W1 ro_water, W2 visc_water, W3 ro_air, W4 visc_air. */
void lso_fluid(const lso_grid* g, const double* phi, double* ro, double* visc, double w1, double w2, double w3,
               double w4) {
    double H = 0.0;
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const long c = lso_index(g, i, j, k);
                const double p = phi[c];
                if (p > g->psi) H = 1.0;
                if (p < -g->psi) H = 0.0;
                if (fabs(p) <= g->psi) H = 0.5 * (1.0 + p / g->psi + (1.0 / LSO_PI) * sin((LSO_PI * p) / g->psi));
                ro[c] = w1 * H + w3 * (1.0 - H);
                visc[c] = w2 * H + w4 * (1.0 - H);
            }
    ghost_fill_gcv(g, ro, 0);
    ghost_fill_gcv(g, visc, 0);
}

/* src/ietimestep.cpp:38-188 for a prescribed velocity (N50=1, no source
 * term): face maxima over ULOOP/VLOOP/WLOOP with wall boundaries
 * (ulast=vlast=wlast=1, src/lexer_gridsize.cpp:74-77). */
double lso_cfl_dt(const lso_grid* g, const double* u, const double* v, const double* w) {
    double umax = 0.0, vmax = 0.0, wmax = 0.0;
    for (int i = 0; i < g->nx - 1; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const double a = fabs(u[lso_index(g, i, j, k)]);
                umax = umax > a ? umax : a;
            }
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny - 1; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const double a = fabs(v[lso_index(g, i, j, k)]);
                vmax = vmax > a ? vmax : a;
            }
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz - 1; ++k) {
                const double a = fabs(w[lso_index(g, i, j, k)]);
                wmax = wmax > a ? wmax : a;
            }
    double cu = 1.0e10;
    for (int i = 0; i < g->nx; ++i)
        for (int j = 0; j < g->ny; ++j)
            for (int k = 0; k < g->nz; ++k) {
                const double dx = MIN3V(g->dxn[i + LSO_MARGE], g->dyn[j + LSO_MARGE], g->dzn[k + LSO_MARGE]);
                const double cand = 2.0 / ((sqrt(umax * umax + vmax * vmax + wmax * wmax)) / dx
                                           + sqrt((4.0 * fabs(0.0)) / dx));
                cu = MINV(cu, cand);
            }
    return g->n47 * cu;
}

/* ------------------------------------------------- opaque handle for ctypes */
lso_grid* lso_new(int nx, int ny, int nz, const double* xn, const double* yn, const double* zn,
                  double f43, int f44, double f45, int f49, double n47) {
    lso_grid* g = (lso_grid*)calloc(1, sizeof(lso_grid));
    if (!g) return NULL;
    if (lso_grid_init(g, nx, ny, nz, xn, yn, zn, f43, f44, f45, f49, n47) != 0) { free(g); return NULL; }
    return g;
}
void lso_delete(lso_grid* g) { if (g) { lso_grid_free(g); free(g); } }
long lso_ncell(const lso_grid* g) { return g->ncell; }
double lso_psi(const lso_grid* g) { return g->psi; }
double lso_dxm(const lso_grid* g) { return g->dxm_mean; }
int lso_get_metric(const lso_grid* g, int which, double* dst, int n) {
    const double* src[9] = {g->dxn, g->dyn, g->dzn, g->dxp, g->dyp, g->dzp, g->xp, g->yp, g->zp};
    if (which < 0 || which > 8) return -1;
    memcpy(dst, src[which], sizeof(double) * (size_t)n);
    return 0;
}
/* tables in the harness order: qf [t][6][2], cf [t][6], isf [t][6][3] */
int lso_get_weno_tables(const lso_grid* g, int axis, double* qf, double* cf, double* isf, int n) {
    memcpy(qf, g->qf[axis], sizeof(double) * (size_t)n * 12);
    memcpy(cf, g->cf[axis], sizeof(double) * (size_t)n * 6);
    memcpy(isf, g->isf[axis], sizeof(double) * (size_t)n * 18);
    return 0;
}
