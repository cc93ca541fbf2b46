// FP32 form of the level-set stencils.
//
// Uniform grids (the common case) use undivided differences: with
// q = (f[m+1]-f[m]) instead of (f[m+1]-f[m])/h, every smoothness indicator
// scales by h^2, so the WENO psi of the reference (1e-6,
// src/weno_nug_func.cpp:26) is rescaled to 1e-6*h^2 and the nonlinear
// weights come out identical in exact arithmetic; the reconstruction is
// divided by h once.  The classic Jiang-Peng coefficients used here are the
// values the reference's node tables take on a uniform grid (ideal weights
// 0.3/0.6/0.1, IS forms 10/3, 11/3, 4/3 of the q differences).
// Non-uniform grids use the reference's node tables in FP32 with divided
// differences.  The same templates run in FP64 for the interface band of
// the reinitialisation (see kernels_f32.cu).
#pragma once

#include "r3d_internal.h"

namespace r3d {
namespace f32 {

template <typename R>
__device__ __forceinline__ R rcp(R x) { return R(1) / x; }
template <>
__device__ __forceinline__ float rcp<float>(float x) { return __frcp_rn(x); }
template <typename R>
__device__ __forceinline__ R rsqrt_r(R x) { return rsqrt(x); }
template <>
__device__ __forceinline__ float rsqrt_r<float>(float x) { return rsqrtf(x); }

// WENO5-HJ derivative on a uniform grid from the undivided differences
// d1..d5 of the upwind set; eps = 1e-6*h^2.  Returns h * derivative.
template <typename R>
__device__ __forceinline__ R weno5_uniform(bool plus, R d1, R d2, R d3, R d4, R d5, R eps) {
    // IS of the stencils (d3,d4,d5), (d2,d3,d4), (d1,d2,d3):
    // 10/3 a^2 + 11/3 ab + 4/3 b^2 with a, b the differences to the middle q
    const R a1 = d3 - d4, b1 = d5 - d4;
    const R a2 = d4 - d3, b2 = d2 - d3;
    const R a3 = d3 - d2, b3 = d1 - d2;
    const R k10 = R(10.0 / 3.0), k11 = R(11.0 / 3.0), k4 = R(4.0 / 3.0);
    const R is1 = (k10 * a1 + k11 * b1) * a1 + k4 * b1 * b1;
    const R is2 = (k4 * a2 + R(5.0 / 3.0) * b2) * a2 + k4 * b2 * b2;
    const R is3 = (k10 * a3 + k11 * b3) * a3 + k4 * b3 * b3;
    const R s1 = is1 + eps, s2 = is2 + eps, s3 = is3 + eps;
    const R r1 = rcp(s1), r2 = rcp(s2), r3 = rcp(s3);
    R c1, c2, c3;
    if (!plus) { c1 = R(0.3); c2 = R(0.6); c3 = R(0.1); }
    else { c1 = R(0.1); c2 = R(0.6); c3 = R(0.3); }
    const R al1 = c1 * r1 * r1, al2 = c2 * r2 * r2, al3 = c3 * r3 * r3;
    const R inv = rcp(al1 + al2 + al3);
    R p1, p2, p3;
    if (!plus) {
        p1 = d4 + R(1.0 / 3.0) * a1 - R(1.0 / 6.0) * b1;
        p2 = d3 + R(1.0 / 3.0) * a2 - R(1.0 / 6.0) * b2;
        p3 = d2 + R(1.0 / 3.0) * b3 + R(11.0 / 6.0) * a3;
    } else {
        p1 = d4 + R(11.0 / 6.0) * a1 + R(1.0 / 3.0) * b1;
        p2 = d3 + R(1.0 / 3.0) * b2 - R(1.0 / 6.0) * a2;
        p3 = d2 + R(1.0 / 3.0) * a3 - R(1.0 / 6.0) * b3;
    }
    return (al1 * p1 + al2 * p2 + al3 * p3) * inv;
}

// The reference's non-uniform form (tables, divided differences) in FP32.
// zero1..zero3: the weight of stencil (q3,q4,q5) / (q2,q3,q4) / (q1,q2,q3)
// is set to 0 (the X45 = 6 masked differences; at least one stays on).
__device__ __forceinline__ float weno5_tables(const float* __restrict__ Q, const float* __restrict__ C,
                                              const float* __restrict__ S, bool plus, float q1, float q2,
                                              float q3, float q4, float q5, bool zero1 = false,
                                              bool zero2 = false, bool zero3 = false) {
    const float dq12 = q1 - q2, dq23 = q2 - q3, dq32 = q3 - q2;
    const float dq34 = q3 - q4, dq43 = q4 - q3, dq54 = q5 - q4;
    const float is1 = __ldg(S + 0) * dq54 * dq54 + __ldg(S + 1) * dq54 * dq34 + __ldg(S + 2) * dq34 * dq34;
    const float is2 = __ldg(S + 3) * dq23 * dq23 + __ldg(S + 4) * dq43 * dq23 + __ldg(S + 5) * dq43 * dq43;
    const float is3 = __ldg(S + 6) * dq12 * dq12 + __ldg(S + 7) * dq32 * dq12 + __ldg(S + 8) * dq32 * dq32;
    const float r1 = __frcp_rn(is1 + 1.0e-6f), r2 = __frcp_rn(is2 + 1.0e-6f), r3 = __frcp_rn(is3 + 1.0e-6f);
    float al1 = __ldg(C + 0) * r1 * r1, al2 = __ldg(C + 1) * r2 * r2, al3 = __ldg(C + 2) * r3 * r3;
    if (zero1) al1 = 0.0f;
    if (zero2) al2 = 0.0f;
    if (zero3) al3 = 0.0f;
    const float inv = __frcp_rn(al1 + al2 + al3);
    float p1, p2, p3;
    if (!plus) {
        p1 = q4 + __ldg(Q + 0) * (q3 - q4) - __ldg(Q + 1) * (q5 - q4);
        p2 = q3 + __ldg(Q + 2) * (q4 - q3) - __ldg(Q + 3) * (q2 - q3);
        p3 = q2 + __ldg(Q + 4) * (q1 - q2) + __ldg(Q + 5) * (q3 - q2);
    } else {
        p1 = q4 + __ldg(Q + 0) * (q3 - q4) + __ldg(Q + 1) * (q5 - q4);
        p2 = q3 + __ldg(Q + 2) * (q2 - q3) - __ldg(Q + 3) * (q4 - q3);
        p3 = q2 + __ldg(Q + 4) * (q3 - q2) - __ldg(Q + 5) * (q1 - q2);
    }
    return (al1 * p1 + al2 * p2 + al3 * p3) * inv;
}

// Derivative along an axis from the 7 values f[-3..3] around the cell.
// Uniform: returns the derivative (already divided by h).
template <typename R>
__device__ __forceinline__ R deriv_uniform(const R* fv, bool plus, R rh, R eps) {
    // fv[0..6] = f[-3..3]
    if (!plus)
        return rh * weno5_uniform<R>(false, fv[1] - fv[0], fv[2] - fv[1], fv[3] - fv[2], fv[4] - fv[3],
                                     fv[5] - fv[4], eps);
    return rh * weno5_uniform<R>(true, fv[2] - fv[1], fv[3] - fv[2], fv[4] - fv[3], fv[5] - fv[4],
                                 fv[6] - fv[5], eps);
}

__device__ __forceinline__ float deriv_tables(const float* fv, bool plus, const float* __restrict__ dp,
                                              const float* __restrict__ qf, const float* __restrict__ cf,
                                              const float* __restrict__ isf, int t) {
    float q1, q2, q3, q4, q5;
    if (!plus) {
        q1 = __fdividef(fv[1] - fv[0], __ldg(dp + t - 3));
        q2 = __fdividef(fv[2] - fv[1], __ldg(dp + t - 2));
        q3 = __fdividef(fv[3] - fv[2], __ldg(dp + t - 1));
        q4 = __fdividef(fv[4] - fv[3], __ldg(dp + t));
        q5 = __fdividef(fv[5] - fv[4], __ldg(dp + t + 1));
    } else {
        q1 = __fdividef(fv[2] - fv[1], __ldg(dp + t - 2));
        q2 = __fdividef(fv[3] - fv[2], __ldg(dp + t - 1));
        q3 = __fdividef(fv[4] - fv[3], __ldg(dp + t));
        q4 = __fdividef(fv[5] - fv[4], __ldg(dp + t + 1));
        q5 = __fdividef(fv[6] - fv[5], __ldg(dp + t + 2));
    }
    const int side = plus ? 1 : 0;
    return weno5_tables(qf + t * 12 + side * 6, cf + t * 6 + side * 3, isf + t * 18 + side * 9, plus, q1, q2, q3,
                        q4, q5);
}

// Reinitialisation right-hand side from the axis stencils (7 values per
// axis, centre at [3]); the Godunov selection and smoothed sign of
// src/reinidisc_f.cpp:58-127 on a uniform grid.  rh[a] = 1/h_a,
// hh[a] = h_a^2, eps = the reference's WENO psi (1e-6).
template <typename R, bool TWO_D>
__device__ __forceinline__ R reini_rhs_uniform(const R* fx, const R* fy, const R* fz, const R* rh, const R* hh,
                                               R eps, R deltax) {
    const R lsv = fx[3];
    const R lsSig = (fabs((double)lsv) < 1.0e-8) ? R(1) : (lsv > R(0) ? R(1) : R(-1));
    R g[3] = {R(0), R(0), R(0)};
    const R* fa[3] = {fx, fy, fz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (TWO_D && a == 1) continue;
        const R* f = fa[a];
        const R xmin = (lsv - f[2]) * rh[a];
        const R xplus = (f[4] - lsv) * rh[a];
        R d = R(0);
        if (xmin * lsSig > R(0) && xplus * lsSig > -xmin * lsSig) d = deriv_uniform<R>(f, false, rh[a], eps * hh[a]);
        if (xplus * lsSig < R(0) && xmin * lsSig < -xplus * lsSig) d = deriv_uniform<R>(f, true, rh[a], eps * hh[a]);
        if (xplus * lsSig > R(0) && xmin * lsSig < R(0)) d = R(0);
        g[a] = d;
    }
    const R dnorm = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    R sign = lsv * rsqrt_r(lsv * lsv + dnorm * dnorm * deltax * deltax);
    if (sign != sign) sign = R(1);
    return -(sign * dnorm - sign);
}

}  // namespace f32
}  // namespace r3d
