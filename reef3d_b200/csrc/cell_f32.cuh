// FP32 cell operators shared by the per-instance kernels (kernels_f32.cu)
// and the batched persistent kernels (kernels_batch.cu): one cell per call,
// stencils read through the read-only cache.
#pragma once

#include "stencil_f32.cuh"

namespace r3d {
namespace f32c {

__device__ __forceinline__ void load7(const float* __restrict__ f, long long c, long long s, float* o) {
#pragma unroll
    for (int m = 0; m < 7; ++m) o[m] = __ldg(f + c + (m - 3) * s);
}

// Direct-forcing divided difference of the X45 stencils
// (src/weno_hj_df_nug.cpp:398-987) in the FP32 form: the mask decisions on
// the FP64 body field (the reference's), the difference in FP32.  X45 6
// (masked differences 1e20) is handled by deriv_tables_df6.
__device__ __forceinline__ float df_q32(int x45, double thr, float fa, float fb, double ha, double hb, double hw,
                                        float d) {
    switch (x45) {
        case 1: return (fabs(hb) > thr && fabs(ha) > thr) ? __fdividef(fb - fa, d) : 0.0f;
        case 2: return __fdividef((float)(0.5 * (hb + ha)) * (fb - fa), d);
        case 3: return (hb < 0.5 && ha < 0.5) ? __fdividef(fb - fa, d) : 0.0f;
        case 4: return __fdividef((float)hw * (fb - fa), d);
        default: return (hb > 0.0 && ha > 0.0) ? __fdividef(fb - fa, d) : 0.0f;
    }
}

// X45 = 6 (src/weno_hj_df_nug.cpp:868-987): a difference whose pair of
// cells is not all fluid (fbh4 >= 0.5 at either) is 1e20 in the reference,
// and 1e20 squared overflows FP32.  In the reference's FP64 a stencil that
// holds such a difference has a smoothness indicator ~1e40, hence a weight
// ~1e-80 relative to any stencil without one: here that weight is exactly 0.
// When all three stencils hold one (the upwind face of the cell is masked,
// or one face on each side), or the FP32 weights leave the FP32 range (the
// 1e20-scale values such cells feed into the next stages), the reference's
// arithmetic runs in FP64 on the FP32 values and tables and is rounded to
// FP32.
__device__ __forceinline__ float deriv_tables_df6(const float* fv, const double* hv, bool plus,
                                                  const float* __restrict__ dp, const float* __restrict__ qf,
                                                  const float* __restrict__ cf, const float* __restrict__ isf, int t) {
    const int off = plus ? 1 : 0;
    float q[5];
    bool masked[5];
#pragma unroll
    for (int m = 1; m <= 5; ++m) {
        const int a = m - 1 + off, b = m + off;
        masked[m - 1] = !(hv[b] < 0.5 && hv[a] < 0.5);
        q[m - 1] = masked[m - 1] ? 0.0f : __fdividef(fv[b] - fv[a], __ldg(dp + t - 4 + m + off));
    }
    const int side = plus ? 1 : 0;
    const float* Q = qf + t * 12 + side * 6;
    const float* C = cf + t * 6 + side * 3;
    const float* S = isf + t * 18 + side * 9;
    const bool z1 = masked[2] || masked[3] || masked[4];  // stencil (q3, q4, q5)
    const bool z2 = masked[1] || masked[2] || masked[3];  // (q2, q3, q4)
    const bool z3 = masked[0] || masked[1] || masked[2];  // (q1, q2, q3)
    if (!(z1 && z2 && z3)) {
        const float r = f32::weno5_tables(Q, C, S, plus, q[0], q[1], q[2], q[3], q[4], z1, z2, z3);
        if (isfinite(r)) return r;
    }
    // the reference's weighting (src/weno_nug_func.h:48-73, 133-153) in FP64
    double d[5];
#pragma unroll
    for (int m = 0; m < 5; ++m)
        d[m] = masked[m] ? 1.0e20 : (double)(fv[m + 1 + off] - fv[m + off]) / (double)__ldg(dp + t - 3 + m + off);
    const double dq12 = d[0] - d[1], dq23 = d[1] - d[2], dq32 = d[2] - d[1];
    const double dq34 = d[2] - d[3], dq43 = d[3] - d[2], dq54 = d[4] - d[3];
    const double is1 = (double)__ldg(S + 0) * dq54 * dq54 + (double)__ldg(S + 1) * dq54 * dq34 +
                       (double)__ldg(S + 2) * dq34 * dq34 + 1.0e-6;
    const double is2 = (double)__ldg(S + 3) * dq23 * dq23 + (double)__ldg(S + 4) * dq43 * dq23 +
                       (double)__ldg(S + 5) * dq43 * dq43 + 1.0e-6;
    const double is3 = (double)__ldg(S + 6) * dq12 * dq12 + (double)__ldg(S + 7) * dq32 * dq12 +
                       (double)__ldg(S + 8) * dq32 * dq32 + 1.0e-6;
    const double al1 = (double)__ldg(C + 0) / (is1 * is1), al2 = (double)__ldg(C + 1) / (is2 * is2),
                 al3 = (double)__ldg(C + 2) / (is3 * is3);
    double p1, p2, p3;
    if (!plus) {
        p1 = d[3] + (double)__ldg(Q + 0) * (d[2] - d[3]) - (double)__ldg(Q + 1) * (d[4] - d[3]);
        p2 = d[2] + (double)__ldg(Q + 2) * (d[3] - d[2]) - (double)__ldg(Q + 3) * (d[1] - d[2]);
        p3 = d[1] + (double)__ldg(Q + 4) * (d[0] - d[1]) + (double)__ldg(Q + 5) * (d[2] - d[1]);
    } else {
        p1 = d[3] + (double)__ldg(Q + 0) * (d[2] - d[3]) + (double)__ldg(Q + 1) * (d[4] - d[3]);
        p2 = d[2] + (double)__ldg(Q + 2) * (d[1] - d[2]) - (double)__ldg(Q + 3) * (d[3] - d[2]);
        p3 = d[1] + (double)__ldg(Q + 4) * (d[2] - d[1]) - (double)__ldg(Q + 5) * (d[0] - d[1]);
    }
    return (float)((al1 * p1 + al2 * p2 + al3 * p3) / (al1 + al2 + al3));
}

// deriv_tables with the X45 differences: fv, hv the 7-point windows of the
// level set and the body field (centre at [3]); q_m from the pair
// (m-1, m) of the six upwind points, the X45 4 weight at the pair's
// upwind-most cell.
__device__ __forceinline__ float deriv_tables_df(const float* fv, const double* hv, bool plus,
                                                 const float* __restrict__ dp, const float* __restrict__ qf,
                                                 const float* __restrict__ cf, const float* __restrict__ isf, int t,
                                                 int x45, double thr) {
    const int off = plus ? 1 : 0;
    float q[5];
#pragma unroll
    for (int m = 1; m <= 5; ++m) {
        const int a = m - 1 + off, b = m + off;
        q[m - 1] = df_q32(x45, thr, fv[a], fv[b], hv[a], hv[b], plus ? hv[b] : hv[a], __ldg(dp + t - 4 + m + off));
    }
    const int side = plus ? 1 : 0;
    return f32::weno5_tables(qf + t * 12 + side * 6, cf + t * 6 + side * 3, isf + t * 18 + side * 9, plus, q[0], q[1],
                             q[2], q[3], q[4]);
}

__device__ __forceinline__ void load7d(const double* __restrict__ f, long long c, long long s, double* o) {
#pragma unroll
    for (int m = 0; m < 7; ++m) o[m] = __ldg(f + c + (m - 3) * s);
}

// DF: the direct-forcing stencils of g.x45 over g.body (table form).
template <bool TWO_D, bool UNIFORM, bool DF = false>
__device__ __forceinline__ float conv_L(const KGrid<float>& g, const float* __restrict__ f,
                                        const float* __restrict__ u, const float* __restrict__ v,
                                        const float* __restrict__ w, long long c, int i, int j, int k, float vs) {
    const long long sy = g.L.sy, sz = g.L.sz;
    const float ia = 0.5f * vs * (__ldg(u + c) + __ldg(u + c - 1));
    const float ka = 0.5f * vs * (__ldg(w + c) + __ldg(w + c - sz));
    float fv[7];
    double hv[7];
    auto axis = [&](long long s, int a, int t, bool plus) {
        if (DF) {
            load7d(g.body, c, s, hv);
            if (g.x45 == 6) return deriv_tables_df6(fv, hv, plus, g.dxp[a], g.qf[a], g.cf[a], g.isf[a], t);
            return deriv_tables_df(fv, hv, plus, g.dxp[a], g.qf[a], g.cf[a], g.isf[a], t, g.x45, g.df_thr);
        }
        return UNIFORM ? f32::deriv_uniform<float>(fv, plus, g.rh[a], g.eps_u * g.h[a] * g.h[a])
                       : f32::deriv_tables(fv, plus, g.dxp[a], g.qf[a], g.cf[a], g.isf[a], t);
    };
    float l = 0.0f;
    if (ia != 0.0f) {
        load7(f, c, 1, fv);
        l -= ia * axis(1, 0, i + 5, ia < 0.0f);
    }
    if (!TWO_D) {
        const float ja = 0.5f * vs * (__ldg(v + c) + __ldg(v + c - sy));
        if (ja != 0.0f) {
            load7(f, c, sy, fv);
            l -= ja * axis(sy, 1, j + 5, ja < 0.0f);
        }
    }
    if (ka != 0.0f) {
        load7(f, c, sz, fv);
        l -= ka * axis(sz, 2, k + 5, ka < 0.0f);
    }
    return l;
}

// Non-uniform reinitialisation RHS in FP32 with the node tables.
template <bool TWO_D>
__device__ __forceinline__ float reini_tables(const KGrid<float>& g, const float* fx, const float* fy,
                                              const float* fz, int i, int j, int k) {
    const float lsv = fx[3];
    const float lsSig = (fabsf(lsv) < 1.0e-8f) ? 1.0f : (lsv > 0.0f ? 1.0f : -1.0f);
    const float* fa[3] = {fx, fy, fz};
    const int t[3] = {i + 5, j + 5, k + 5};
    float gsum = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (TWO_D && a == 1) continue;
        const float* f = fa[a];
        const float xmin = __fdividef(lsv - f[2], __ldg(g.dxp[a] + t[a] - 1));
        const float xplus = __fdividef(f[4] - lsv, __ldg(g.dxp[a] + t[a]));
        float d = 0.0f;
        if (xmin * lsSig > 0.0f && xplus * lsSig > -xmin * lsSig)
            d = f32::deriv_tables(f, false, g.dxp[a], g.qf[a], g.cf[a], g.isf[a], t[a]);
        if (xplus * lsSig < 0.0f && xmin * lsSig < -xplus * lsSig)
            d = f32::deriv_tables(f, true, g.dxp[a], g.qf[a], g.cf[a], g.isf[a], t[a]);
        if (xplus * lsSig > 0.0f && xmin * lsSig < 0.0f) d = 0.0f;
        gsum += d * d;
    }
    const float dnorm = sqrtf(gsum);
    const float deltax = TWO_D ? 0.5f * (__ldg(g.dxn[0] + t[0]) + __ldg(g.dxn[2] + t[2]))
                               : (1.0f / 3.0f) * (__ldg(g.dxn[0] + t[0]) + __ldg(g.dxn[1] + t[1]) + __ldg(g.dxn[2] + t[2]));
    float sign = lsv * rsqrtf(lsv * lsv + dnorm * dnorm * deltax * deltax);
    if (sign != sign) sign = 1.0f;
    return -(sign * dnorm - sign);
}

template <bool TWO_D, bool UNIFORM>
__device__ __forceinline__ float reini_L(const KGrid<float>& g, const float* __restrict__ f, long long c, int i,
                                         int j, int k) {
    float fx[7], fy[7], fz[7];
    load7(f, c, 1, fx);
    load7(f, c, g.L.sz, fz);
    if (!TWO_D) load7(f, c, g.L.sy, fy);
    else {
#pragma unroll
        for (int m = 0; m < 7; ++m) fy[m] = 0.0f;
        fy[3] = fx[3];
    }
    const float f0 = fx[3];
    const bool pos = f0 >= 0.0f && fx[2] >= 0.0f && fx[4] >= 0.0f && fz[2] >= 0.0f && fz[4] >= 0.0f &&
                     (TWO_D || (fy[2] >= 0.0f && fy[4] >= 0.0f));
    const bool neg = f0 < 0.0f && fx[2] < 0.0f && fx[4] < 0.0f && fz[2] < 0.0f && fz[4] < 0.0f &&
                     (TWO_D || (fy[2] < 0.0f && fy[4] < 0.0f));
    const bool band = !(pos || neg);  // the zero level set crosses the 7-point stencil
    // F49=0 freezes band cells (src/reinidisc_fsf.cpp:70-72); in 2D the
    // reference's test also reads the never-written y ghost planes (zero),
    // so no negative cell passes it there.
    if (g.f49 == 0 && (band || (TWO_D && neg))) return 0.0f;
    if (!UNIFORM) return reini_tables<TWO_D>(g, fx, fy, fz, i, j, k);
    const float deltax = TWO_D ? 0.5f * (g.h[0] + g.h[2]) : (1.0f / 3.0f) * (g.h[0] + g.h[1] + g.h[2]);
    if (band) {
        // interface band: FP64 re-anchoring of the zero level set
        double dx[7], dy[7], dz[7];
#pragma unroll
        for (int m = 0; m < 7; ++m) { dx[m] = fx[m]; dy[m] = fy[m]; dz[m] = fz[m]; }
        const double rh[3] = {1.0 / g.h[0], 1.0 / g.h[1], 1.0 / g.h[2]};
        const double hh[3] = {(double)g.h[0] * g.h[0], (double)g.h[1] * g.h[1], (double)g.h[2] * g.h[2]};
        const double dlt = TWO_D ? 0.5 * ((double)g.h[0] + g.h[2]) : (1.0 / 3.0) * ((double)g.h[0] + g.h[1] + g.h[2]);
        return (float)f32::reini_rhs_uniform<double, TWO_D>(dx, dy, dz, rh, hh, 1.0e-6, dlt);
    }
    const float hh[3] = {g.h[0] * g.h[0], g.h[1] * g.h[1], g.h[2] * g.h[2]};
    return f32::reini_rhs_uniform<float, TWO_D>(fx, fy, fz, g.rh, hh, 1.0e-6f, deltax);
}

template <bool TWO_D>
__device__ __forceinline__ float reini_dt32(const KGrid<float>& g, int i, int j, int k) {
    const float a = __ldg(g.dxp[0] + i + 5), c = __ldg(g.dxp[2] + k + 5);
    if (TWO_D) return (float)g.f43 * fminf(a, c);
    const float b = __ldg(g.dxp[1] + j + 5);
    return (float)g.f43 * fminf(fminf(a, b), c);
}

}  // namespace f32c
}  // namespace r3d
