// FP32 form: stencils and RK stages in FP32, the volume integral in FP64,
// and the reinitialisation of interface-band cells (cells whose 7-point
// stencil changes sign) re-anchored in FP64 so the zero level set is moved
// with FP64 arithmetic.  One fused pass per RK stage as in the FP64 path.
#include "stencil_f32.cuh"

namespace r3d {
namespace {

constexpr int kBX = 32, kBY = 4;

struct StageArgs32 {
    const float* fn;
    const float* fs;
    float* out;
    const float* u;
    const float* v;
    const float* w;
    const double* dt;
    const double* vscale;
    double* partial;
};

__device__ __forceinline__ void load7(const float* __restrict__ f, long long c, long long s, float* o) {
#pragma unroll
    for (int m = 0; m < 7; ++m) o[m] = __ldg(f + c + (m - 3) * s);
}

template <bool TWO_D, bool UNIFORM>
__device__ __forceinline__ float conv_L(const KGrid<float>& g, const float* __restrict__ f,
                                        const float* __restrict__ u, const float* __restrict__ v,
                                        const float* __restrict__ w, long long c, int i, int j, int k, float vs) {
    const long long sy = g.L.sy, sz = g.L.sz;
    const float ia = 0.5f * vs * (__ldg(u + c) + __ldg(u + c - 1));
    const float ka = 0.5f * vs * (__ldg(w + c) + __ldg(w + c - sz));
    float fv[7];
    float l = 0.0f;
    if (ia != 0.0f) {
        load7(f, c, 1, fv);
        const float d = UNIFORM ? f32::deriv_uniform<float>(fv, ia < 0.0f, g.rh[0], g.eps_u * g.h[0] * g.h[0])
                                : f32::deriv_tables(fv, ia < 0.0f, g.dxp[0], g.qf[0], g.cf[0], g.isf[0], i + 5);
        l -= ia * d;
    }
    if (!TWO_D) {
        const float ja = 0.5f * vs * (__ldg(v + c) + __ldg(v + c - sy));
        if (ja != 0.0f) {
            load7(f, c, sy, fv);
            const float d = UNIFORM ? f32::deriv_uniform<float>(fv, ja < 0.0f, g.rh[1], g.eps_u * g.h[1] * g.h[1])
                                    : f32::deriv_tables(fv, ja < 0.0f, g.dxp[1], g.qf[1], g.cf[1], g.isf[1], j + 5);
            l -= ja * d;
        }
    }
    if (ka != 0.0f) {
        load7(f, c, sz, fv);
        const float d = UNIFORM ? f32::deriv_uniform<float>(fv, ka < 0.0f, g.rh[2], g.eps_u * g.h[2] * g.h[2])
                                : f32::deriv_tables(fv, ka < 0.0f, g.dxp[2], g.qf[2], g.cf[2], g.isf[2], k + 5);
        l -= ka * d;
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

__device__ __forceinline__ void block_sum2(double a, double b, double* dst) {
    __shared__ double sa[32], sb[32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31;
    const int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
    const int nwarp = (blockDim.x * blockDim.y) >> 5;
    if (lane == 0) { sa[warp] = a; sb[warp] = b; }
    __syncthreads();
    if (warp == 0) {
        a = lane < nwarp ? sa[lane] : 0.0;
        b = lane < nwarp ? sb[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (lane == 0) { dst[0] = a; dst[1] = b; }
    }
}

template <bool TWO_D, int STAGE, bool REINI, bool VOLUME, bool UNIFORM>
__global__ void __launch_bounds__(kBX * kBY) stage_kernel32(KGrid<float> g, StageArgs32 a) {
    const int i = blockIdx.x * kBX + threadIdx.x;
    const int j = TWO_D ? 0 : blockIdx.y * kBY + threadIdx.y;
    const int k = TWO_D ? blockIdx.z * kBY + threadIdx.y : blockIdx.z;
    const bool active = i < g.L.nx && j < g.L.ny && k < g.L.nz;
    double v1 = 0.0, v2 = 0.0;
    if (active) {
        const long long c = (long long)(k + g.L.gz) * g.L.sz + (long long)(j + g.L.gy) * g.L.sy + (i + g.L.gx);
        float Lc, dtc;
        if (REINI) {
            Lc = reini_L<TWO_D, UNIFORM>(g, a.fs, c, i, j, k);
            dtc = reini_dt32<TWO_D>(g, i, j, k);
        } else {
            Lc = conv_L<TWO_D, UNIFORM>(g, a.fs, a.u, a.v, a.w, c, i, j, k, (float)*a.vscale);
            dtc = (float)*a.dt;
        }
        const float fn = a.fn[c];
        float val;
        if (STAGE == 1) val = fn + dtc * Lc;
        else if (STAGE == 2) val = 0.75f * fn + 0.25f * (__ldg(a.fs + c) + dtc * Lc);
        else val = (1.0f / 3.0f) * fn + (2.0f / 3.0f) * (__ldg(a.fs + c) + dtc * Lc);
        a.out[c] = val;
        if (i == 0) { a.out[c - 1] = val; a.out[c - 2] = val; a.out[c - 3] = val; }
        if (i == g.L.nx - 1) { a.out[c + 1] = val; a.out[c + 2] = val; a.out[c + 3] = val; }
        if (!TWO_D) {
            const long long sy = g.L.sy;
            if (j == 0) { a.out[c - sy] = val; a.out[c - 2 * sy] = val; a.out[c - 3 * sy] = val; }
            if (j == g.L.ny - 1) { a.out[c + sy] = val; a.out[c + 2 * sy] = val; a.out[c + 3 * sy] = val; }
        }
        const long long sz = g.L.sz;
        if (k == 0) { a.out[c - sz] = val; a.out[c - 2 * sz] = val; a.out[c - 3 * sz] = val; }
        if (k == g.L.nz - 1) { a.out[c + sz] = val; a.out[c + 2 * sz] = val; a.out[c + 3 * sz] = val; }
        if (VOLUME) {
            const double PI_REF = 3.14159265359;  // src/definitions.h:37
            const double p = val, psi = g.psi;
            double H = 0.0;
            if (p > psi) H = 1.0;
            if (p < -psi) H = 0.0;
            if (fabs(p) <= psi) H = 0.5 * (1.0 + p / psi + (1.0 / PI_REF) * sin((PI_REF * p) / psi));
            const double vol = (double)__ldg(g.dxn[0] + i + 5) * (double)__ldg(g.dxn[1] + j + 5) *
                               (double)__ldg(g.dxn[2] + k + 5);
            v1 = vol * H;
            v2 = vol * (1.0 - H);
        }
    }
    if (VOLUME) {
        const long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        block_sum2(v1, v2, a.partial + 2 * b);
    }
}

template <bool TWO_D, bool REINI, bool UNIFORM>
__global__ void __launch_bounds__(kBX * kBY) operator_kernel32(KGrid<float> g, StageArgs32 a) {
    const int i = blockIdx.x * kBX + threadIdx.x;
    const int j = TWO_D ? 0 : blockIdx.y * kBY + threadIdx.y;
    const int k = TWO_D ? blockIdx.z * kBY + threadIdx.y : blockIdx.z;
    if (i >= g.L.nx || j >= g.L.ny || k >= g.L.nz) return;
    const long long c = (long long)(k + g.L.gz) * g.L.sz + (long long)(j + g.L.gy) * g.L.sy + (i + g.L.gx);
    a.out[c] = REINI ? reini_L<TWO_D, UNIFORM>(g, a.fs, c, i, j, k)
                     : conv_L<TWO_D, UNIFORM>(g, a.fs, a.u, a.v, a.w, c, i, j, k, (float)*a.vscale);
}

dim3 grid_of32(const Layout& L) {
    if (L.two_d) return dim3((L.nx + kBX - 1) / kBX, 1, (L.nz + kBY - 1) / kBY);
    return dim3((L.nx + kBX - 1) / kBX, (L.ny + kBY - 1) / kBY, L.nz);
}

template <bool TWO_D, bool REINI, bool UNIFORM>
void launch_t(const KGrid<float>& g, const StageArgs32& a, int stage, bool volume, cudaStream_t st) {
    const dim3 grid = grid_of32(g.L), block(kBX, kBY);
#define R3D_L32(S, V) stage_kernel32<TWO_D, S, REINI, V, UNIFORM><<<grid, block, 0, st>>>(g, a)
    if (stage == 1) { if (volume) R3D_L32(1, true); else R3D_L32(1, false); }
    else if (stage == 2) { if (volume) R3D_L32(2, true); else R3D_L32(2, false); }
    else { if (volume) R3D_L32(3, true); else R3D_L32(3, false); }
#undef R3D_L32
}

template <bool REINI>
void launch_any(const KGrid<float>& g, const StageArgs32& a, int stage, bool volume, bool uniform, cudaStream_t st) {
    if (g.L.two_d) {
        if (uniform) launch_t<true, REINI, true>(g, a, stage, volume, st);
        else launch_t<true, REINI, false>(g, a, stage, volume, st);
    } else {
        if (uniform) launch_t<false, REINI, true>(g, a, stage, volume, st);
        else launch_t<false, REINI, false>(g, a, stage, volume, st);
    }
}

StageArgs32 args32(const Fields& f, int stage, const Scratch& s) {
    StageArgs32 a{};
    const float* phi = static_cast<const float*>(f.phi);
    a.fn = phi;
    a.fs = stage == 1 ? phi : stage == 2 ? static_cast<const float*>(f.a1) : static_cast<const float*>(f.a2);
    a.out = stage == 1 ? static_cast<float*>(f.a1) : stage == 2 ? static_cast<float*>(f.a2) : static_cast<float*>(f.phi);
    a.u = static_cast<const float*>(f.u);
    a.v = static_cast<const float*>(f.v);
    a.w = static_cast<const float*>(f.w);
    a.dt = s.dt;
    a.vscale = s.vscale;
    a.partial = s.partial;
    return a;
}

bool is_uniform(const KGrid<float>& g) { return g.h[0] > 0.0f; }

}  // namespace

int launch_conv_stage_f32(const KGrid<float>& g, const Fields& f, int stage, const Scratch& s, bool volume,
                          cudaStream_t st) {
    launch_any<false>(g, args32(f, stage, s), stage, volume, is_uniform(g), st);
    return 1;
}

int launch_reini_stage_f32(const KGrid<float>& g, const Fields& f, int stage, const Scratch& s, bool volume,
                           cudaStream_t st) {
    launch_any<true>(g, args32(f, stage, s), stage, volume, is_uniform(g), st);
    return 1;
}

template <bool REINI>
static void launch_op(const KGrid<float>& g, const StageArgs32& a, cudaStream_t st) {
    const dim3 grid = grid_of32(g.L), block(kBX, kBY);
    const bool u = is_uniform(g);
    if (g.L.two_d) {
        if (u) operator_kernel32<true, REINI, true><<<grid, block, 0, st>>>(g, a);
        else operator_kernel32<true, REINI, false><<<grid, block, 0, st>>>(g, a);
    } else {
        if (u) operator_kernel32<false, REINI, true><<<grid, block, 0, st>>>(g, a);
        else operator_kernel32<false, REINI, false><<<grid, block, 0, st>>>(g, a);
    }
}

int launch_conv_L_f32(const KGrid<float>& g, const void* in, const Fields& f, const Scratch& s, cudaStream_t st) {
    StageArgs32 a{};
    a.vscale = s.vscale;
    a.fs = static_cast<const float*>(in);
    a.out = static_cast<float*>(f.L);
    a.u = static_cast<const float*>(f.u);
    a.v = static_cast<const float*>(f.v);
    a.w = static_cast<const float*>(f.w);
    launch_op<false>(g, a, st);
    return 1;
}

int launch_reini_L_f32(const KGrid<float>& g, const void* in, const Fields& f, cudaStream_t st) {
    StageArgs32 a{};
    a.fs = static_cast<const float*>(in);
    a.out = static_cast<float*>(f.L);
    launch_op<true>(g, a, st);
    return 1;
}

}  // namespace r3d
