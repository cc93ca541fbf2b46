// Grid metrics and WENO coefficient tables of an instance, built on the host
// in the reference's operation order so that the FP64 device path sees
// bit-identical coefficients.  Compiled with -ffp-contract=off.
#include <cmath>

#include "r3d_internal.h"

namespace r3d {

namespace {

constexpr int kMarge = 5;  // 1D offset of the reference (src/iterators1D.h)

// src/grid.cpp:55-100: cell centres, node spacing DXN and centre spacing DXP.
void spacing(int n, const std::vector<double>& xn, std::vector<double>& xp, std::vector<double>& dxn,
             std::vector<double>& dxp) {
    const size_t len = n + 1 + 4 * kMarge;  // src/read_grid.cpp:404-406
    xp.assign(len, 0.0);
    dxn.assign(len, 0.0);
    dxp.assign(len, 0.0);
    for (int i = -kMarge; i < n + kMarge; ++i) {
        const int t = i + kMarge;
        xp[t] = 0.5 * (xn[t] + xn[t + 1]);
        dxn[t] = xn[t + 1] - xn[t];
        dxp[t] = 0.5 * (xn[t + 2] + xn[t + 1]) - 0.5 * (xn[t + 1] + xn[t]);
    }
}

inline double sq(double x) { return std::pow(x, 2.0); }  // the reference calls pow(x, 2.0)

// Non-uniform WENO5 node tables (uf=0) for one axis, for the index range
// IBLOOP i = -1..n (src/weno_nug_func_precalc_qf.cpp:28-80,
// src/weno_nug_func_precalc_cf.cpp:27-56, src/weno_nug_func_precalc_isf.cpp:27-176;
// the y and z sections of those files are the same formulas).  Per index t:
// qf[12] = {side,r,coef} with side 0 = upwind from the minus side,
// cf[6] = {side,r}, isf[18] = {side,r,coef}.
void weno_tables(int n, const std::vector<double>& X, std::vector<double>& qf, std::vector<double>& cf,
                 std::vector<double>& isf) {
    qf.assign((size_t)(n + 8) * 12, 0.0);
    cf.assign((size_t)(n + 8) * 6, 0.0);
    isf.assign((size_t)(n + 8) * 18, 0.0);
    for (int i = -1; i < n + 1; ++i) {
        const int t = i + kMarge;
        const double Xm2 = X[t - 2], Xm1 = X[t - 1], X0 = X[t], X1 = X[t + 1];
        const double X2 = X[t + 2], X3 = X[t + 3], X4 = X[t + 4];
        double* q = &qf[(size_t)t * 12];
        double* c = &cf[(size_t)t * 6];
        double* s = &isf[(size_t)t * 18];

        // reconstruction weights of the three candidate stencils
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

        // linear (ideal) weights
        c[0] = ((X1 - Xm2) / (X3 - Xm2)) * ((X1 - Xm1) / (X3 - Xm1));
        c[1] = ((X1 - Xm2) / (X3 - Xm2)) * ((X3 - X1) / (X3 - Xm1)) * ((X3 - Xm1) / (X2 - Xm2) + 1.0);
        c[2] = ((X2 - X1) / (X3 - Xm2)) * ((X3 - X1) / (X2 - Xm2));
        c[3] = ((X1 - X0) / (X4 - Xm1)) * ((X1 - Xm1) / (X4 - X0));
        c[4] = ((X1 - Xm1) / (X4 - Xm1)) * ((X4 - X1) / (X4 - X0)) * ((X4 - X0) / (X3 - Xm1) + 1.0);
        c[5] = ((X3 - X1) / (X4 - Xm1)) * ((X4 - X1) / (X3 - Xm1));

        // smoothness-indicator quadratic forms, minus side
        double fac = 4.0 * sq((X1 - X0) / (X3 - X0));
        s[0] = fac * ((10.0 * sq(X1 - X0) + (X2 - X0) * (X2 - X1)) / sq(X3 - X1));
        s[1] = fac * ((20.0 * sq(X1 - X0) + 2.0 * (X2 - X0) * (X2 - X1) + (X3 - X0) * (2.0 * X2 - X1 - X0)) /
                      ((X3 - X1) * (X2 - X0)));
        s[2] = fac * ((10.0 * sq(X1 - X0) + (X3 + X2 - 2.0 * X0) * (X3 + X2 - X1 - X0)) / sq(X2 - X0));
        fac = 4.0 * sq((X1 - X0) / (X2 - Xm1));
        s[3] = fac * ((10.0 * sq(X1 - X0) + (X2 - X0) * (X2 - X1)) / sq(X1 - Xm1));
        s[4] = fac * ((20.0 * sq(X1 - X0) - (X2 - X1) * (X0 - Xm1) - (X2 - X0) * (X1 - Xm1)) /
                      ((X2 - X0) * (X1 - Xm1)));
        s[5] = fac * ((10.0 * sq(X1 - X0) + (X0 - Xm1) * (X1 - Xm1)) / sq(X2 - X0));
        fac = 4.0 * sq((X1 - X0) / (X1 - Xm2));
        s[6] = fac * ((10.0 * sq(X1 - X0) + (X1 - Xm1) * (X0 - Xm1)) / sq(X0 - Xm2));
        s[7] = fac * ((20.0 * sq(X1 - X0) + 2.0 * (X1 - Xm1) * (X0 - Xm1) + (X1 - Xm2) * (X1 + X0 - 2.0 * Xm1)) /
                      ((X1 - Xm1) * (X0 - Xm2)));
        s[8] = fac * ((10.0 * sq(X1 - X0) + (2.0 * X1 - Xm2 - Xm1) * (X1 + X0 - Xm1 - Xm2)) / sq(X1 - Xm1));
        // plus side
        fac = 4.0 * sq((X2 - X1) / (X4 - X1));
        s[9] = fac * ((10.0 * sq(X2 - X1) + (X3 - X1) * (X3 - X2)) / sq(X4 - X2));
        s[10] = fac * ((20.0 * sq(X2 - X1) + 2.0 * (X3 - X1) * (X3 - X2) + (X4 - X1) * (2.0 * X3 - X2 - X1)) /
                       ((X4 - X2) * (X3 - X1)));
        s[11] = fac * ((10.0 * sq(X2 - X1) + (X4 + X3 - 2.0 * X1) * (X4 + X3 - X2 - X1)) / sq(X3 - X1));
        fac = 4.0 * sq((X2 - X1) / (X3 - X0));
        s[12] = fac * ((10.0 * sq(X2 - X1) + (X3 - X1) * (X3 - X2)) / sq(X2 - X0));
        s[13] = fac * ((20.0 * sq(X2 - X1) - (X3 - X2) * (X1 - X0) - (X3 - X1) * (X2 - X0)) /
                       ((X3 - X1) * (X2 - X0)));
        s[14] = fac * ((10.0 * sq(X2 - X1) + (X1 - X0) * (X2 - X0)) / sq(X3 - X1));
        fac = 4.0 * sq((X2 - X1) / (X2 - Xm1));
        s[15] = fac * ((10.0 * sq(X2 - X1) + (X2 - X0) * (X1 - X0)) / sq(X1 - Xm1));
        s[16] = fac * ((20.0 * sq(X2 - X1) + 2.0 * (X2 - X0) * (X1 - X0) + (X2 - Xm1) * (X2 + X1 - 2.0 * X0)) /
                       ((X2 - X0) * (X1 - Xm1)));
        s[17] = fac * ((10.0 * sq(X2 - X1) + (2.0 * X2 - Xm1 - X0) * (X2 + X1 - X0 - Xm1)) / sq(X2 - X0));
    }
}

}  // namespace

Layout make_layout(int nx, int ny, int nz) {
    Layout L{};
    L.nx = nx; L.ny = ny; L.nz = nz;
    L.two_d = (ny == 1);
    L.gx = 4;
    L.gy = L.two_d ? 0 : 3;
    L.gz = 3;
    L.px = ((nx + L.gx + 3) + 7) / 8 * 8;  // row pitch: multiple of 8 elements (32 B)
    L.py = L.two_d ? 1 : ny + 6;
    L.pz = nz + 6;
    L.sy = L.px;
    L.sz = (long long)L.px * L.py;
    L.ncell = L.sz * L.pz;
    return L;
}

void build_metrics(int nx, int ny, int nz, const double* xn, const double* yn, const double* zn, double f45,
                   HostMetrics& m) {
    const int n[3] = {nx, ny, nz};
    const double* src[3] = {xn, yn, zn};
    for (int a = 0; a < 3; ++a) {
        m.n[a] = n[a];
        m.xn[a].assign((size_t)n[a] + 1 + 4 * kMarge, 0.0);
        for (int t = 0; t < n[a] + 1 + 2 * kMarge; ++t) m.xn[a][t] = src[a][t];
        spacing(n[a], m.xn[a], m.xp[a], m.dxn[a], m.dxp[a]);
        weno_tables(n[a], m.xn[a], m.qf[a], m.cf[a], m.isf[a]);
    }
    const bool two_d = (ny == 1);
    // src/grid.cpp:102-148 (one rank)
    double dxm = 0.0;
    int count = 0;
    for (int i = 0; i < nx; ++i) { dxm += m.dxp[0][i + kMarge]; ++count; }
    if (!two_d)
        for (int j = 0; j < ny; ++j) { dxm += m.dxp[1][j + kMarge]; ++count; }
    for (int k = 0; k < nz; ++k) { dxm += m.dxp[2][k + kMarge]; ++count; }
    dxm /= double(count);
    m.dxm_mean = dxm;
    m.dym = yn[kMarge + 1] - yn[kMarge];
    m.dzm = zn[kMarge + 1] - zn[kMarge];
    // src/ini_psi.cpp:33-37
    if (two_d) m.psi = f45 * (1.0 / 2.0) * (m.dxm_mean + m.dzm);
    else m.psi = f45 * (1.0 / 3.0) * (m.dxm_mean + m.dym + m.dzm);

    // CFL length: the reference takes MIN over cells of MIN3(DXN,DYN,DZN) of
    // 2/(|u|/dx); that expression is non-decreasing in dx under correct
    // rounding, so its minimum sits at the smallest MIN3 over the cells.
    double dmin[3];
    for (int a = 0; a < 3; ++a) {
        dmin[a] = m.dxn[a][kMarge];
        for (int c = 0; c < n[a]; ++c) dmin[a] = std::fmin(dmin[a], m.dxn[a][c + kMarge]);
    }
    double d = dmin[0] < dmin[1] ? dmin[0] : dmin[1];
    m.dxmin_cfl = d < dmin[2] ? d : dmin[2];

    m.uniform = true;
    for (int a = 0; a < 3; ++a) {
        m.h[a] = m.dxn[a][kMarge];
        for (int c = -kMarge; c < n[a] + kMarge; ++c) {
            const double e = std::fabs(m.dxn[a][c + kMarge] - m.h[a]);
            if (e > 1e-12 * std::fabs(m.h[a])) m.uniform = false;
        }
    }
}

}  // namespace r3d
