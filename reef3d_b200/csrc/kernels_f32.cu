// FP32 form: stencils and RK stages in FP32, the volume integral in FP64,
// and the reinitialisation of interface-band cells (cells whose 7-point
// stencil changes sign) re-anchored in FP64 so the zero level set is moved
// with FP64 arithmetic.  One fused pass per RK stage as in the FP64 path.
#include "cell_f32.cuh"

namespace r3d {
namespace {
using namespace f32c;

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

template <bool TWO_D, int STAGE, bool REINI, bool VOLUME, bool UNIFORM, bool DF = false>
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
            Lc = conv_L<TWO_D, UNIFORM, DF>(g, a.fs, a.u, a.v, a.w, c, i, j, k, (float)*a.vscale);
            dtc = (float)*a.dt;
        }
        const float fn = a.fn[c];
        float val;
        if (STAGE == 1) val = fn + dtc * Lc;
        else if (STAGE == 2) val = 0.75f * fn + 0.25f * (__ldg(a.fs + c) + dtc * Lc);
        else val = (1.0f / 3.0f) * fn + (2.0f / 3.0f) * (__ldg(a.fs + c) + dtc * Lc);
        a.out[c] = val;
        // x faces: inflow / outflow faces with ghost label 0 keep their
        // ghosts; an inflow face also gets the edge ghost (-1, j, nz)
        if (i == 0 && !(g.L.io & kIoSkipLo)) { a.out[c - 1] = val; a.out[c - 2] = val; a.out[c - 3] = val; }
        if (i == g.L.nx - 1 && !(g.L.io & kIoSkipHi)) { a.out[c + 1] = val; a.out[c + 2] = val; a.out[c + 3] = val; }
        if ((g.L.io & kIoEdge) && i == 0 && k == g.L.nz - 1) a.out[c - 1 + g.L.sz] = val;
        if (!TWO_D) {
            const long long sy = g.L.sy;
            if (j == 0) { a.out[c - sy] = val; a.out[c - 2 * sy] = val; a.out[c - 3 * sy] = val; }
            if (j == g.L.ny - 1) { a.out[c + sy] = val; a.out[c + 2 * sy] = val; a.out[c + 3 * sy] = val; }
        }
        const long long sz = g.L.sz;
        if (k == 0 && !(g.L.io & kHaloZLo)) { a.out[c - sz] = val; a.out[c - 2 * sz] = val; a.out[c - 3 * sz] = val; }
        if (k == g.L.nz - 1 && !(g.L.io & kHaloZHi)) {
            a.out[c + sz] = val; a.out[c + 2 * sz] = val; a.out[c + 3 * sz] = val;
        }
        if (VOLUME) {
            const double PI_REF = 3.14159265359;  // src/definitions.h:37
            const double p = val, psi = g.psi;
            double H = 0.0;
            if (p > psi) H = 1.0;
            if (p < -psi) H = 0.0;
            if (fabs(p) <= psi) H = 0.5 * (1.0 + p / psi + (1.0 / PI_REF) * sin((PI_REF * p) / psi));
            const double vol = __ldg(g.dxn_d[0] + i + 5) * __ldg(g.dxn_d[1] + j + 5) * __ldg(g.dxn_d[2] + k + 5);
            v1 = vol * H;
            v2 = vol * (1.0 - H);
        }
    }
    if (VOLUME) {
        const long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        block_sum2(v1, v2, a.partial + 2 * b);
    }
}

template <bool TWO_D, bool REINI, bool UNIFORM, bool DF = false>
__global__ void __launch_bounds__(kBX * kBY) operator_kernel32(KGrid<float> g, StageArgs32 a) {
    const int i = blockIdx.x * kBX + threadIdx.x;
    const int j = TWO_D ? 0 : blockIdx.y * kBY + threadIdx.y;
    const int k = TWO_D ? blockIdx.z * kBY + threadIdx.y : blockIdx.z;
    if (i >= g.L.nx || j >= g.L.ny || k >= g.L.nz) return;
    const long long c = (long long)(k + g.L.gz) * g.L.sz + (long long)(j + g.L.gy) * g.L.sy + (i + g.L.gx);
    a.out[c] = REINI ? reini_L<TWO_D, UNIFORM>(g, a.fs, c, i, j, k)
                     : conv_L<TWO_D, UNIFORM, DF>(g, a.fs, a.u, a.v, a.w, c, i, j, k, (float)*a.vscale);
}

dim3 grid_of32(const Layout& L) {
    if (L.two_d) return dim3((L.nx + kBX - 1) / kBX, 1, (L.nz + kBY - 1) / kBY);
    return dim3((L.nx + kBX - 1) / kBX, (L.ny + kBY - 1) / kBY, L.nz);
}

template <bool TWO_D, bool REINI, bool UNIFORM, bool DF = false>
void launch_t(const KGrid<float>& g, const StageArgs32& a, int stage, bool volume, cudaStream_t st) {
    const dim3 grid = grid_of32(g.L), block(kBX, kBY);
#define R3D_L32(S, V) stage_kernel32<TWO_D, S, REINI, V, UNIFORM, DF><<<grid, block, 0, st>>>(g, a)
    if (stage == 1) { if (volume) R3D_L32(1, true); else R3D_L32(1, false); }
    else if (stage == 2) { if (volume) R3D_L32(2, true); else R3D_L32(2, false); }
    else { if (volume) R3D_L32(3, true); else R3D_L32(3, false); }
#undef R3D_L32
}

template <bool REINI>
void launch_any(const KGrid<float>& g, const StageArgs32& a, int stage, bool volume, bool uniform, cudaStream_t st) {
    if (!REINI && g.x45) {  // direct-forcing stencils (table form)
        if (g.L.two_d) launch_t<true, false, false, true>(g, a, stage, volume, st);
        else launch_t<false, false, false, true>(g, a, stage, volume, st);
        return;
    }
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
    if (!REINI && g.x45) {
        if (g.L.two_d) operator_kernel32<true, false, false, true><<<grid, block, 0, st>>>(g, a);
        else operator_kernel32<false, false, false, true><<<grid, block, 0, st>>>(g, a);
        return;
    }
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
