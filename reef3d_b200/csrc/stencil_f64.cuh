// FP64 stencil arithmetic of the level-set path, written in the reference's
// operation order.  Included only by translation units compiled with
// -fmad=false, so every product and sum rounds separately as in the
// reference built without FMA contraction; double division and sqrt are
// IEEE round-to-nearest on the device as on the host (the divisions by grid
// spacings through div_rn, which forms the same quotient).
#pragma once

#include "r3d_internal.h"


namespace r3d {
namespace f64 {

// a / b rounded to nearest from r = 1/b rounded to nearest (the IEEE
// reciprocal, tabulated per grid spacing): q0 = a r, then two residual
// corrections with fused multiply-adds (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990).  The first correction makes the quotient faithful; a
// faithful quotient corrected once more with the correctly rounded
// reciprocal is the correctly rounded quotient (Markstein's theorem), i.e.
// the IEEE a / b.  Valid when the residual neither overflows nor underflows,
// which holds for level-set differences over grid spacings.  A zero
// numerator gives +0 where the IEEE quotient of -0 is -0.
__device__ __forceinline__ double div_rn(double a, double b, double r) {
    const double q0 = a * r;
    const double q1 = fma(fma(-b, q0, a), r, q0);
    return fma(fma(-b, q1, a), r, q1);
}

// WENO5 derivative from the divided differences q1..q5 of the upwind set,
// node tables of index t and the side: the record W = wt + 18 (2t + side)
// holds Q0..Q5, C0..C2, S0..S8 (16-byte aligned: nine 16-byte loads).
// Minus side: IS src/weno_nug_func.h:48-60, weights :133-143,
// reconstruction src/weno_hj_df_nug.cpp:155-159.  Plus side: :61-73,
// :144-153, :186-190.  epsilon = 0, psi = 1e-6 (src/weno_nug_func.cpp:26).
__device__ __forceinline__ double2 ldg2(const double* p) { return __ldg(reinterpret_cast<const double2*>(p)); }

__device__ __forceinline__ double weno5(const double* __restrict__ W, bool plus, double q1, double q2, double q3,
                                        double q4, double q5) {
    const double2 w01 = ldg2(W + 0), w23 = ldg2(W + 2), w45 = ldg2(W + 4), w67 = ldg2(W + 6);
    const double2 w89 = ldg2(W + 8), wab = ldg2(W + 10), wcd = ldg2(W + 12), wef = ldg2(W + 14);
    const double2 wgh = ldg2(W + 16);
    const double S[9] = {w89.y, wab.x, wab.y, wcd.x, wcd.y, wef.x, wef.y, wgh.x, wgh.y};
    const double psi = 1.0e-6, eps = 0.0;
    const double dq12 = q1 - q2, dq23 = q2 - q3, dq32 = q3 - q2;
    const double dq34 = q3 - q4, dq43 = q4 - q3, dq54 = q5 - q4;
    const double is1 = S[0] * dq54 * dq54 + S[1] * (dq54) * (dq34) + S[2] * dq34 * dq34;
    const double is2 = S[3] * dq23 * dq23 + S[4] * (dq43) * (dq23) + S[5] * dq43 * dq43;
    const double is3 = S[6] * dq12 * dq12 + S[7] * (dq32) * (dq12) + S[8] * dq32 * dq32;
    const double a = is1 + psi, b = is2 + psi, c = is3 + psi;
    const double c0 = w67.x, c1 = w67.y, c2 = w89.x;
    const double sum = c0 / (a * a) + c1 / (b * b) + c2 / (c * c);
    const double w1 = c0 / (eps + (a * a) * sum);
    const double w2 = c1 / (eps + (b * b) * sum);
    const double w3 = c2 / (eps + (c * c) * sum);
    const double Q0 = w01.x, Q1 = w01.y, Q2 = w23.x, Q3 = w23.y, Q4 = w45.x, Q5 = w45.y;
    // The two sides' reconstructions differ only in which differences enter
    // and in two signs (minus side :155-159, plus side :186-190); selecting
    // those operands keeps every rounding of either side:
    //   w1 (q4 + Q0 (q3-q4) -+ Q1 (q5-q4))
    //   w2 (q3 + Q2 x2 - Q3 y2)   x2, y2 = (q4-q3), (q2-q3)  [plus: swapped]
    //   w3 (q2 + Q4 x3 +- Q5 y3)  x3, y3 = (q1-q2), (q3-q2)  [plus: swapped]
    const double t1 = Q1 * (q5 - q4);
    const double x2 = plus ? (q2 - q3) : (q4 - q3), y2 = plus ? (q4 - q3) : (q2 - q3);
    const double x3 = plus ? (q3 - q2) : (q1 - q2), y3 = plus ? (q1 - q2) : (q3 - q2);
    const double t3 = Q5 * y3;
    return w1 * (q4 + Q0 * (q3 - q4) + (plus ? t1 : -t1))
         + w2 * (q3 + Q2 * x2 - Q3 * y2)
         + w3 * (q2 + Q4 * x3 + (plus ? -t3 : t3));
}

// Upwind-biased derivative along one axis (stride s) at linear index c,
// cell index t = idx+5.  Minus stencil src/weno_hj_df_nug.cpp:344-351, plus
// stencil :371-378 (shared with src/ddweno_nug_sf.cpp:225-277): the six
// points f[c+(o+m)s], m = 0..5, with o = -3 (minus) or -2 (plus), and
// q_m = (f_m - f_{m-1}) / DXP[t+o+m-1], the IEEE quotient formed by div_rn
// from the reciprocal table rp of dp.  The side is a runtime value, so a
// warp whose cells take different sides runs one evaluation, not both.
__device__ __forceinline__ double deriv(const double* __restrict__ f, long long c, long long s,
                                        const double* __restrict__ dpr, const double* __restrict__ wt, int t,
                                        bool plus) {
    const int o = plus ? -2 : -3;
    const double* p = f + c + o * s;
    const double* d = dpr + 2 * (t + o);
    const double f0 = __ldg(p), f1 = __ldg(p + s), f2 = __ldg(p + 2 * s);
    const double f3 = __ldg(p + 3 * s), f4 = __ldg(p + 4 * s), f5 = __ldg(p + 5 * s);
    const double2 e1 = ldg2(d), e2 = ldg2(d + 2), e3 = ldg2(d + 4), e4 = ldg2(d + 6), e5 = ldg2(d + 8);
    const double q1 = div_rn(f1 - f0, e1.x, e1.y);
    const double q2 = div_rn(f2 - f1, e2.x, e2.y);
    const double q3 = div_rn(f3 - f2, e3.x, e3.y);
    const double q4 = div_rn(f4 - f3, e4.x, e4.y);
    const double q5 = div_rn(f5 - f4, e5.x, e5.y);
    return weno5(wt + 18 * (2 * (long long)t + (plus ? 1 : 0)), plus, q1, q2, q3, q4, q5);
}

// deriv from precomputed face differences: Q[m] = (f_{c+m-2} - f_{c+m-3}) /
// DXP[t+m-3], m = 0..5, i.e. the divided differences of the six faces
// around the cell (face m lies between cells c+m-3 and c+m-2).  The minus
// stencil reads faces 0..4, the plus stencil faces 1..5, in the order deriv
// forms them; each face value is the same IEEE operation whichever cell
// computes it, so the result is deriv's bit for bit.
__device__ __forceinline__ double deriv_q(const double* Q, const double* __restrict__ wt, int t, bool plus) {
    return weno5(wt + 18 * (2 * (long long)t + (plus ? 1 : 0)), plus, plus ? Q[1] : Q[0], plus ? Q[2] : Q[1],
                 plus ? Q[3] : Q[2], plus ? Q[4] : Q[3], plus ? Q[5] : Q[4]);
}

// Direct-forcing divided difference of the cell pair (a, b = a + s) of the
// X45 stencils (src/weno_hj_df_nug.cpp:398-987; one rule per X45 for the
// three axes and both sides), with ha, hb the body field at the two cells:
//  1 zero unless |fb| > 0.6 DXM at both (body = fb),
//  2 weighted by 0.5 (fbh5(b) + fbh5(a)),
//  3 zero unless fbh4 < 0.5 at both,
//  4 weighted by fbh5 at hw: the pair's lower cell on the minus side, its
//    upper cell on the plus side,
//  5 zero unless solid > 0 and topo > 0 at both (body = min(solid, topo),
//    which is > 0 exactly when both are),
//  6 like 3 but 1e20 where masked.
__device__ __forceinline__ double df_q(int x45, double thr, double fa, double fb, double ha, double hb, double hw,
                                       double d) {
    switch (x45) {
        case 1: return (fabs(hb) > thr && fabs(ha) > thr) ? (fb - fa) / d : 0.0;
        case 2: return 0.5 * (hb + ha) * (fb - fa) / d;
        case 3: return (hb < 0.5 && ha < 0.5) ? (fb - fa) / d : 0.0;
        case 4: return hw * (fb - fa) / d;
        case 5: return (hb > 0.0 && ha > 0.0) ? (fb - fa) / d : 0.0;
        default: return (hb < 0.5 && ha < 0.5) ? (fb - fa) / d : 1.0e20;
    }
}

// deriv with the direct-forcing differences of df_q.
__device__ __forceinline__ double deriv_df(const double* __restrict__ f, const double* __restrict__ h, long long c,
                                           long long s, const double* __restrict__ dp,
                                           const double* __restrict__ wt, int t, bool plus, int x45, double thr) {
    const int o = plus ? -2 : -3;
    const long long b0 = c + o * s;
    const double* d = dp + t + o;
    double fv[6], hv[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        fv[m] = __ldg(f + b0 + m * s);
        hv[m] = __ldg(h + b0 + m * s);
    }
    double q[5];
#pragma unroll
    for (int m = 1; m <= 5; ++m)
        q[m - 1] = df_q(x45, thr, fv[m - 1], fv[m], hv[m - 1], hv[m], plus ? hv[m] : hv[m - 1], __ldg(d + m - 1));
    return weno5(wt + 18 * (2 * (long long)t + (plus ? 1 : 0)), plus, q[0], q[1], q[2], q[3], q[4]);
}

// -u.grad(f) at interior cell (i,j,k): src/weno_hj_df_nug.cpp:93-111 with the
// cell-centre velocities of src/flux_HJ_CDS2.cpp:59-127 (2D: no y term,
// src/flux_HJ_CDS2_2D.cpp).  Returned as the reference's a->L value
// (0.0 + L).
// The stored face velocities are multiplied by vs (1 leaves them exact).
// DF: the direct-forcing stencils of g.x45 (g.body) replace the plain ones.
template <bool TWO_D, bool DF = false>
__device__ __forceinline__ double conv_L(const KGrid<double>& g, const double* __restrict__ f,
                                         const double* __restrict__ u, const double* __restrict__ v,
                                         const double* __restrict__ w, long long c, int i, int j, int k,
                                         double vs) {
    const long long sy = g.L.sy, sz = g.L.sz;
    const double iadvec = 0.5 * (vs * __ldg(u + c) + vs * __ldg(u + c - 1));
    const double kadvec = 0.5 * (vs * __ldg(w + c) + vs * __ldg(w + c - sz));
    auto axis = [&](long long s, int a, int t, bool plus) {
        if (DF) return deriv_df(f, g.body, c, s, g.dxp[a], g.wt[a], t, plus, g.x45, g.df_thr);
        return deriv(f, c, s, g.dpr[a], g.wt[a], t, plus);
    };
    // advec > 0: minus side, < 0: plus side, == 0: no contribution (grad 0)
    double grad = axis(1, 0, i + 5, iadvec < 0.0);
    if (iadvec == 0.0) grad = 0.0;
    double l = -iadvec * grad;
    if (!TWO_D) {
        const double jadvec = 0.5 * (vs * __ldg(v + c) + vs * __ldg(v + c - sy));
        grad = axis(sy, 1, j + 5, jadvec < 0.0);
        if (jadvec == 0.0) grad = 0.0;
        l -= jadvec * grad;
    }
    grad = axis(sz, 2, k + 5, kadvec < 0.0);
    if (kadvec == 0.0) grad = 0.0;
    l -= kadvec * grad;
    double acc = 0.0;
    acc += l;
    return acc;
}

// F49=0 interface test (src/reinidisc_fsf.cpp:70-72).  In 2D the y
// neighbours are ghost planes the reference never writes (zero).
template <bool TWO_D>
__device__ __forceinline__ bool same_sign(const double* __restrict__ f, long long c, long long sy,
                                          long long sz) {
    const double f0 = __ldg(f + c), xp = __ldg(f + c + 1), xm = __ldg(f + c - 1);
    const double yp = TWO_D ? 0.0 : __ldg(f + c + sy), ym = TWO_D ? 0.0 : __ldg(f + c - sy);
    const double zp = __ldg(f + c + sz), zm = __ldg(f + c - sz);
    return (f0 >= 0.0 && xp >= 0.0 && xm >= 0.0 && yp >= 0.0 && ym >= 0.0 && zp >= 0.0 && zm >= 0.0) ||
           (f0 < 0.0 && xp < 0.0 && xm < 0.0 && yp < 0.0 && ym < 0.0 && zp < 0.0 && zm < 0.0);
}

// The six face divided differences around the cell along one axis (stride
// s, cell index t = idx + 5): Q[m] = (f[c+(m-2)s] - f[c+(m-3)s]) /
// DXP[t+m-3] (div_rn with the (DXP, 1/DXP) pairs dpr), the layout deriv_q
// reads.  Each is the quotient deriv forms for that face, and faces 2 and 3
// are the backward and forward differences of the reinitialisation's
// Godunov test.
__device__ __forceinline__ void faces6(const double* __restrict__ f, long long c, long long s,
                                       const double* __restrict__ dpr, int t, double* Q) {
    double fv[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) fv[m] = __ldg(f + c + (m - 3) * s);
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        const double2 e = ldg2(dpr + 2 * (t + m - 3));
        Q[m] = div_rn(fv[m + 1] - fv[m], e.x, e.y);
    }
}

// One axis of the reinitialisation right-hand side: the Godunov selection
// of src/reinidisc_f.cpp:70-109 on the backward / forward differences (faces
// 2, 3), then the one-sided WENO derivative of the selected side from the
// same faces (src/ddweno_nug_sf.cpp), or 0.
__device__ __forceinline__ double reini_axis(const double* Q, double lsSig, const double* __restrict__ wt, int t) {
    const double xmin = Q[2], xplus = Q[3];
    // minus side if c1, plus side if c2 (the later test wins, as there), else 0
    const bool c1 = xmin * lsSig > 0.0 && xplus * lsSig > -xmin * lsSig;
    const bool c2 = xplus * lsSig < 0.0 && xmin * lsSig < -xplus * lsSig;
    double d = deriv_q(Q, wt, t, c2);
    if (!(c1 || c2)) d = 0.0;
    if (xplus * lsSig > 0.0 && xmin * lsSig < 0.0) d = 0.0;
    return d;
}

// Reinitialisation right-hand side at (i,j,k): src/reinidisc_f.cpp:58-127
// (and the body of src/reinidisc_fsf.cpp:74-139).  Each axis's six face
// differences are formed once and serve the Godunov test and the WENO
// stencil (the reference divides the two Godunov faces a second time; the
// quotients are the same).
template <bool TWO_D>
__device__ __forceinline__ double reini_L(const KGrid<double>& g, const double* __restrict__ f, long long c,
                                          int i, int j, int k) {
    const long long sy = g.L.sy, sz = g.L.sz;
    const int ti = i + 5, tj = j + 5, tk = k + 5;
    double dx = 0.0, dy = 0.0, dz = 0.0;
    const double lsv = __ldg(f + c);
    // lsv / sqrt(lsv * lsv): the square root of a correctly rounded square
    // is |lsv| exactly (binary arithmetic, round to nearest, no overflow), so
    // the quotient is the sign; the formula itself where the square overflows
    // (or lsv is NaN)
    double lsSig = lsv > 0.0 ? 1.0 : -1.0;
    if (!(fabs(lsv) < 1.0e150)) lsSig = lsv / sqrt(lsv * lsv);
    if (fabs(lsv) < 1.0e-8) lsSig = 1.0;
    double Q[6];
    faces6(f, c, 1, g.dpr[0], ti, Q);
    dx = reini_axis(Q, lsSig, g.wt[0], ti);
    if (!TWO_D) {
        faces6(f, c, sy, g.dpr[1], tj, Q);
        dy = reini_axis(Q, lsSig, g.wt[1], tj);
    }
    faces6(f, c, sz, g.dpr[2], tk, Q);
    dz = reini_axis(Q, lsSig, g.wt[2], tk);

    const double dnorm = sqrt(dx * dx + dy * dy + dz * dz);
    double deltax;
    if (TWO_D) deltax = (1.0 / 2.0) * (__ldg(g.dxn[0] + ti) + __ldg(g.dxn[2] + tk));
    else deltax = (1.0 / 3.0) * (__ldg(g.dxn[0] + ti) + __ldg(g.dxn[1] + tj) + __ldg(g.dxn[2] + tk));
    double sign = lsv / sqrt(lsv * lsv + dnorm * dnorm * deltax * deltax);
    if (sign != sign) sign = 1.0;
    return -(sign * dnorm - sign);
}

// Reinit pseudo time step of a cell (src/reini_RK3.cpp:150-160).
template <bool TWO_D>
__device__ __forceinline__ double reini_dt(const KGrid<double>& g, int i, int j, int k) {
    const double a = __ldg(g.dxp[0] + i + 5), c = __ldg(g.dxp[2] + k + 5);
    if (TWO_D) return g.f43 * (a < c ? a : c);
    const double b = __ldg(g.dxp[1] + j + 5);
    const double m = a < b ? a : b;
    return g.f43 * (m < c ? m : c);
}

}  // namespace f64
}  // namespace r3d
