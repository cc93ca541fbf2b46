// FP64 plain path: one fused pass per RK stage.  Each pass computes the
// operator (WENO5-HJ convection or the reinitialisation right-hand side)
// from the stage input, combines it with the step's start value as the
// reference's Shu-Osher stage does, writes the stage output and its wall
// ghost copies, and in the last pass of a step adds the cell's share of the
// FP64 volume integral.  Compiled with -fmad=false (see stencil_f64.cuh).
#include "stencil_f64.cuh"

namespace r3d {
namespace {

constexpr int kBX = 32, kBY = 4;
// resident blocks per SM the stage kernels are register-limited for
#ifndef R3D_F64_MINB
#define R3D_F64_MINB 8
#endif

struct StageArgs {
    const double* fn;   // step start value (phi^n / f): read at the cell only
    const double* fs;   // stage input: read with the stencil
    double* out;        // stage output (may alias fn in the last stage)
    const double* u;
    const double* v;
    const double* w;
    const double* dt;   // device time step (convection stages)
    const double* vscale;  // device factor of the stored velocities
    double* partial;    // volume partials, 2 per block
};

__device__ __forceinline__ void cell_of_thread(const Layout& L, bool two_d, int& i, int& j, int& k) {
    i = blockIdx.x * kBX + threadIdx.x;
    if (two_d) {
        j = 0;
        k = blockIdx.z * kBY + threadIdx.y;
    } else {
        j = blockIdx.y * kBY + threadIdx.y;
        k = blockIdx.z;
    }
}

// Wall ghost copy of the cell value into the three face ghost layers
// (src/gc_neumann.cpp:29-54; 2D skips y, src/gc_start.cpp:160).  Inflow /
// outflow x faces whose ghost label is 0 keep their ghosts; with an inflow
// face the top inflow cell also fills the edge ghost (-1, j, nz) as
// dgcpol4 does (src/gc_dgcpol4.cpp:28-50).
template <typename T>
__device__ __forceinline__ void write_ghosts(const Layout& L, T* out, long long c, int i, int j, int k, T val) {
    if (i == 0 && !(L.io & kIoSkipLo)) { out[c - 1] = val; out[c - 2] = val; out[c - 3] = val; }
    if (i == L.nx - 1 && !(L.io & kIoSkipHi)) { out[c + 1] = val; out[c + 2] = val; out[c + 3] = val; }
    if ((L.io & kIoEdge) && i == 0 && k == L.nz - 1) out[c - 1 + L.sz] = val;
    if (!L.two_d) {
        if (j == 0) { out[c - L.sy] = val; out[c - 2 * L.sy] = val; out[c - 3 * L.sy] = val; }
        if (j == L.ny - 1) { out[c + L.sy] = val; out[c + 2 * L.sy] = val; out[c + 3 * L.sy] = val; }
    }
    if (k == 0 && !(L.io & kHaloZLo)) { out[c - L.sz] = val; out[c - 2 * L.sz] = val; out[c - 3 * L.sz] = val; }
    if (k == L.nz - 1 && !(L.io & kHaloZHi)) { out[c + L.sz] = val; out[c + 2 * L.sz] = val; out[c + 3 * L.sz] = val; }
}

// Deterministic block sum of two doubles (fixed shuffle tree, fixed warp
// order); thread 0 writes the block's pair.
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

// Smoothed Heaviside and cell volume (src/fluid_update_fsf.cpp:50-71,
// porosity 1, the reference's PI of src/definitions.h:37).
__device__ __forceinline__ void heaviside_volume(const KGrid<double>& g, double p, int i, int j, int k,
                                                 double& v1, double& v2) {
    const double PI_REF = 3.14159265359;
    const double psi = g.psi;
    double H = 0.0;
    if (p > psi) H = 1.0;
    if (p < -psi) H = 0.0;
    if (fabs(p) <= psi) H = 0.5 * (1.0 + p / psi + (1.0 / PI_REF) * sin((PI_REF * p) / psi));
    const double vol = __ldg(g.dxn[0] + i + 5) * __ldg(g.dxn[1] + j + 5) * __ldg(g.dxn[2] + k + 5);
    v1 = vol * (H - (1.0 - 1.0));
    v2 = vol * (1.0 - H - (1.0 - 1.0));
}

// Convection stage s of src/levelset_RK3.cpp:112-159:
//   s=1: out = fn + dt L(fn)
//   s=2: out = 0.75 fn + 0.25 fs + 0.25 dt L(fs)
//   s=3: out = 1/3 fn + 2/3 fs + 2/3 dt L(fs)
// Reinit stage s of src/reini_RK3.cpp:113-137: the same with the per-cell
// pseudo time step.
template <bool TWO_D, int STAGE, bool REINI, bool VOLUME, bool DF = false>
__global__ void __launch_bounds__(kBX * kBY, R3D_F64_MINB) stage_kernel(KGrid<double> g, StageArgs a) {
    int i, j, k;
    cell_of_thread(g.L, TWO_D, i, j, k);
    const bool active = i < g.L.nx && j < g.L.ny && k < g.L.nz;
    double v1 = 0.0, v2 = 0.0;
    if (active) {
        const long long c = (long long)(k + g.L.gz) * g.L.sz + (long long)(j + g.L.gy) * g.L.sy + (i + g.L.gx);
        double Lc, dtc;
        if (REINI) {
            if (g.f49 == 1 || f64::same_sign<TWO_D>(a.fs, c, g.L.sy, g.L.sz))
                Lc = f64::reini_L<TWO_D>(g, a.fs, c, i, j, k);
            else
                Lc = 0.0;
            dtc = f64::reini_dt<TWO_D>(g, i, j, k);
        } else {
            Lc = f64::conv_L<TWO_D, DF>(g, a.fs, a.u, a.v, a.w, c, i, j, k, *a.vscale);
            dtc = *a.dt;
        }
        const double fn = a.fn[c];
        double val;
        if (STAGE == 1) val = fn + dtc * Lc;
        else if (STAGE == 2) val = 0.75 * fn + 0.25 * __ldg(a.fs + c) + 0.25 * dtc * Lc;
        else val = (1.0 / 3.0) * fn + (2.0 / 3.0) * __ldg(a.fs + c) + (2.0 / 3.0) * dtc * Lc;
        a.out[c] = val;
        write_ghosts(g.L, a.out, c, i, j, k, val);
        if (VOLUME) heaviside_volume(g, val, i, j, k, v1, v2);
    }
    if (VOLUME) {
        const long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        block_sum2(v1, v2, a.partial + 2 * b);
    }
}

// Operator only (drop-ins for convection::start / reinidisc::start): L of
// `fs` into `out` on interior cells.
template <bool TWO_D, bool REINI, bool DF = false>
__global__ void __launch_bounds__(kBX * kBY) operator_kernel(KGrid<double> g, StageArgs a) {
    int i, j, k;
    cell_of_thread(g.L, TWO_D, i, j, k);
    if (i >= g.L.nx || j >= g.L.ny || k >= g.L.nz) return;
    const long long c = (long long)(k + g.L.gz) * g.L.sz + (long long)(j + g.L.gy) * g.L.sy + (i + g.L.gx);
    double Lc;
    if (REINI) {
        if (g.f49 == 1 || f64::same_sign<TWO_D>(a.fs, c, g.L.sy, g.L.sz)) Lc = f64::reini_L<TWO_D>(g, a.fs, c, i, j, k);
        else Lc = 0.0;
    } else {
        Lc = f64::conv_L<TWO_D, DF>(g, a.fs, a.u, a.v, a.w, c, i, j, k, *a.vscale);
    }
    a.out[c] = Lc;
}

dim3 grid_of(const Layout& L) {
    if (L.two_d) return dim3((L.nx + kBX - 1) / kBX, 1, (L.nz + kBY - 1) / kBY);
    return dim3((L.nx + kBX - 1) / kBX, (L.ny + kBY - 1) / kBY, L.nz);
}

template <bool TWO_D, bool REINI, bool DF = false>
void launch_stage_t(const KGrid<double>& g, const StageArgs& a, int stage, bool volume, cudaStream_t st) {
    const dim3 grid = grid_of(g.L), block(kBX, kBY);
    if (stage == 1) {
        if (volume) stage_kernel<TWO_D, 1, REINI, true, DF><<<grid, block, 0, st>>>(g, a);
        else stage_kernel<TWO_D, 1, REINI, false, DF><<<grid, block, 0, st>>>(g, a);
    } else if (stage == 2) {
        if (volume) stage_kernel<TWO_D, 2, REINI, true, DF><<<grid, block, 0, st>>>(g, a);
        else stage_kernel<TWO_D, 2, REINI, false, DF><<<grid, block, 0, st>>>(g, a);
    } else {
        if (volume) stage_kernel<TWO_D, 3, REINI, true, DF><<<grid, block, 0, st>>>(g, a);
        else stage_kernel<TWO_D, 3, REINI, false, DF><<<grid, block, 0, st>>>(g, a);
    }
}

StageArgs stage_args(const Fields& f, int stage, const Scratch& s) {
    StageArgs a{};
    const double* phi = static_cast<const double*>(f.phi);
    a.fn = phi;
    a.fs = stage == 1 ? phi : stage == 2 ? static_cast<const double*>(f.a1) : static_cast<const double*>(f.a2);
    a.out = stage == 1 ? static_cast<double*>(f.a1) : stage == 2 ? static_cast<double*>(f.a2) : static_cast<double*>(f.phi);
    a.u = static_cast<const double*>(f.u);
    a.v = static_cast<const double*>(f.v);
    a.w = static_cast<const double*>(f.w);
    a.dt = s.dt;
    a.vscale = s.vscale;
    a.partial = s.partial;
    return a;
}

}  // namespace

int launch_conv_stage_f64(const KGrid<double>& g, const Fields& f, int stage, const Scratch& s, bool volume,
                          cudaStream_t st) {
    const StageArgs a = stage_args(f, stage, s);
    if (g.x45) {  // direct-forcing stencils (X45 1..6)
        if (g.L.two_d) launch_stage_t<true, false, true>(g, a, stage, volume, st);
        else launch_stage_t<false, false, true>(g, a, stage, volume, st);
    } else {
        if (g.L.two_d) launch_stage_t<true, false>(g, a, stage, volume, st);
        else launch_stage_t<false, false>(g, a, stage, volume, st);
    }
    return 1;
}

int launch_reini_stage_f64(const KGrid<double>& g, const Fields& f, int stage, const Scratch& s, bool volume,
                           cudaStream_t st) {
    const StageArgs a = stage_args(f, stage, s);
    if (g.L.two_d) launch_stage_t<true, true>(g, a, stage, volume, st);
    else launch_stage_t<false, true>(g, a, stage, volume, st);
    return 1;
}

int launch_conv_L_f64(const KGrid<double>& g, const void* in, const Fields& f, const Scratch& s, cudaStream_t st) {
    StageArgs a{};
    a.vscale = s.vscale;
    a.fs = static_cast<const double*>(in);
    a.out = static_cast<double*>(f.L);
    a.u = static_cast<const double*>(f.u);
    a.v = static_cast<const double*>(f.v);
    a.w = static_cast<const double*>(f.w);
    const dim3 grid = grid_of(g.L), block(kBX, kBY);
    if (g.x45) {
        if (g.L.two_d) operator_kernel<true, false, true><<<grid, block, 0, st>>>(g, a);
        else operator_kernel<false, false, true><<<grid, block, 0, st>>>(g, a);
    } else {
        if (g.L.two_d) operator_kernel<true, false><<<grid, block, 0, st>>>(g, a);
        else operator_kernel<false, false><<<grid, block, 0, st>>>(g, a);
    }
    return 1;
}

int launch_reini_L_f64(const KGrid<double>& g, const void* in, const Fields& f, cudaStream_t st) {
    StageArgs a{};
    a.fs = static_cast<const double*>(in);
    a.out = static_cast<double*>(f.L);
    const dim3 grid = grid_of(g.L), block(kBX, kBY);
    if (g.L.two_d) operator_kernel<true, true><<<grid, block, 0, st>>>(g, a);
    else operator_kernel<false, true><<<grid, block, 0, st>>>(g, a);
    return 1;
}

long long volume_blocks(const Layout& L) {
    const dim3 g = grid_of(L);
    return (long long)g.x * g.y * g.z;
}



}  // namespace r3d
