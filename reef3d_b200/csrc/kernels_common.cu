// Kernels shared by both arithmetic forms: host-layout import/export, the
// standalone wall ghost fill, the FP64 CFL reduction and time step, and the
// deterministic second pass of the FP64 volume integral.
#include "r3d_internal.h"

namespace r3d {
namespace {

// ---------------------------------------------------------------- layouts
// REEF3D padded layout: (i+3)*(ny+6)*(nz+6) + (j+3)*(nz+6) + (k+3) with j
// spanning the 6 y ghost planes also in 2D (src/field_base.h:32-47).
// Dense layout: interior only, i + nx*(j + ny*k).
// One thread per device cell of the interior plus the stencil-visible face
// ghosts (cells with at most one index outside the interior).

__device__ __forceinline__ bool visible(const Layout& L, int i, int j, int k) {
    const int out = (i < 0 || i >= L.nx) + (j < 0 || j >= L.ny) + (k < 0 || k >= L.nz);
    return out <= 1;
}

template <typename T>
__global__ void import_kernel(Layout L, const double* __restrict__ src, int layout, T* __restrict__ dst) {
    const int gyp = L.two_d ? 0 : 3;
    const int i = blockIdx.x * blockDim.x + threadIdx.x - 3;
    const int j = blockIdx.y - gyp;
    const int k = blockIdx.z - 3;
    if (i >= L.nx + 3) return;
    const long long d = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx);
    if (layout == 0) {
        const long long jm = L.ny + 6, km = L.nz + 6;
        const long long s = (long long)(i + 3) * jm * km + (long long)(j + 3) * km + (k + 3);
        dst[d] = (T)src[s];
    } else {
        if (i < 0 || i >= L.nx || j < 0 || j >= L.ny || k < 0 || k >= L.nz) return;
        dst[d] = (T)src[i + (long long)L.nx * (j + (long long)L.ny * k)];
    }
}

template <typename T>
__global__ void export_kernel(Layout L, const T* __restrict__ src, int layout, double* __restrict__ dst) {
    const int gyp = L.two_d ? 0 : 3;
    const int i = blockIdx.x * blockDim.x + threadIdx.x - 3;
    const int j = blockIdx.y - gyp;
    const int k = blockIdx.z - 3;
    if (i >= L.nx + 3) return;
    const long long d = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx);
    if (layout == 0) {
        const long long jm = L.ny + 6, km = L.nz + 6;
        const long long s = (long long)(i + 3) * jm * km + (long long)(j + 3) * km + (k + 3);
        dst[s] = visible(L, i, j, k) ? (double)src[d] : 0.0;
    } else {
        if (i < 0 || i >= L.nx || j < 0 || j >= L.ny || k < 0 || k >= L.nz) return;
        dst[i + (long long)L.nx * (j + (long long)L.ny * k)] = (double)src[d];
    }
}

// ------------------------------------------------------------- ghost fill
// ghostcell::start4 with a level-set gcv (src/gc_start.cpp:146-185): the
// Neumann copy on every face whose ghost label is 4 (all walls; inflow /
// outflow faces as Layout::io says) and the inflow edge ghost of dgcpol4.
template <typename T>
__global__ void ghost_kernel(Layout L, T* f) {
    // one thread per interior cell on any face
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= L.nx) return;
    const bool face = i == 0 || i == L.nx - 1 || k == 0 || k == L.nz - 1 ||
                      (!L.two_d && (j == 0 || j == L.ny - 1));
    if (!face) return;
    const long long c = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx);
    const T val = f[c];
    if ((L.io & kIoEdge) && i == 0 && k == L.nz - 1) f[c - 1 + L.sz] = val;
    for (int q = 1; q <= 3; ++q) {
        if (i == 0 && !(L.io & kIoSkipLo)) f[c - q] = val;
        if (i == L.nx - 1 && !(L.io & kIoSkipHi)) f[c + q] = val;
        if (!L.two_d && j == 0) f[c - q * L.sy] = val;
        if (!L.two_d && j == L.ny - 1) f[c + q * L.sy] = val;
        if (k == 0 && !(L.io & kHaloZLo)) f[c - q * L.sz] = val;
        if (k == L.nz - 1 && !(L.io & kHaloZHi)) f[c + q * L.sz] = val;
    }
}

// ------------------------------------------------------------------- CFL
// Face maxima over ULOOP/VLOOP/WLOOP with wall boundaries: x faces
// i = 0..nx-2, y faces j = 0..ny-2, z faces k = 0..nz-2
// (src/ietimestep.cpp:72-88, ulast=vlast=wlast=1 src/lexer_gridsize.cpp:74).
// Non-negative doubles order like their bit patterns, so an atomicMax on the
// bits is an exact, order-independent max.
template <typename T>
__global__ void __launch_bounds__(256) vmax_kernel(Layout L, const T* __restrict__ u, const T* __restrict__ v,
                                                   const T* __restrict__ w, unsigned long long* out) {
    // grid-stride over the (j,k) rows; one atomic per block and component
    double mu = 0.0, mv = 0.0, mw = 0.0;
    const long long rows = (long long)L.ny * L.nz;
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        const int j = (int)(r % L.ny), k = (int)(r / L.ny);
        const long long base = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + L.gx;
        for (int i = threadIdx.x; i < L.nx; i += blockDim.x) {
            if (i < L.nx - 1) mu = fmax(mu, fabs((double)u[base + i]));
            if (j < L.ny - 1) mv = fmax(mv, fabs((double)v[base + i]));
            if (k < L.nz - 1 || (L.io & kHaloZHi)) mw = fmax(mw, fabs((double)w[base + i]));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        mu = fmax(mu, __shfl_down_sync(0xffffffffu, mu, o));
        mv = fmax(mv, __shfl_down_sync(0xffffffffu, mv, o));
        mw = fmax(mw, __shfl_down_sync(0xffffffffu, mw, o));
    }
    __shared__ double s[3][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { s[0][warp] = mu; s[1][warp] = mv; s[2][warp] = mw; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
            mu = fmax(mu, s[0][q]);
            mv = fmax(mv, s[1][q]);
            mw = fmax(mw, s[2][q]);
        }
        atomicMax(out + 0, (unsigned long long)__double_as_longlong(mu));
        atomicMax(out + 1, (unsigned long long)__double_as_longlong(mv));
        atomicMax(out + 2, (unsigned long long)__double_as_longlong(mw));
    }
}

// FP32 fields: the same face maxima over float4 chunks of the rows.  |x| of
// a float compared as its bit pattern with the sign cleared is exact, and the
// largest magnitude converted to double equals the maximum of the converted
// magnitudes, so the result is the one vmax_kernel<float> gives.  Rows start
// 16-byte aligned; a chunk past the last cell reads the row's padding, which
// the masks discard.
__global__ void __launch_bounds__(256) vmax_f32_kernel(Layout L, const float* __restrict__ u,
                                                       const float* __restrict__ v, const float* __restrict__ w,
                                                       unsigned long long* out) {
    const int nq = (L.nx + 3) >> 2;
    const long long items = (long long)L.ny * L.nz * nq;
    unsigned mu = 0u, mv = 0u, mw = 0u;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < items;
         t += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(t % nq);
        const long long r = t / nq;
        const int j = (int)(r % L.ny), k = (int)(r / L.ny);
        const long long c = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + L.gx + 4 * q;
        const float4 a = __ldg(reinterpret_cast<const float4*>(u + c));
        const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (4 * q + e < L.nx - 1) mu = max(mu, __float_as_uint(av[e]) & 0x7fffffffu);
        if (j < L.ny - 1) {
            const float4 b = __ldg(reinterpret_cast<const float4*>(v + c));
            const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (4 * q + e < L.nx) mv = max(mv, __float_as_uint(bv[e]) & 0x7fffffffu);
        }
        if (k < L.nz - 1 || (L.io & kHaloZHi)) {
            const float4 d = __ldg(reinterpret_cast<const float4*>(w + c));
            const float dv[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (4 * q + e < L.nx) mw = max(mw, __float_as_uint(dv[e]) & 0x7fffffffu);
        }
    }
    mu = __reduce_max_sync(0xffffffffu, mu);
    mv = __reduce_max_sync(0xffffffffu, mv);
    mw = __reduce_max_sync(0xffffffffu, mw);
    __shared__ unsigned s[3][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { s[0][warp] = mu; s[1][warp] = mv; s[2][warp] = mw; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
            mu = max(mu, s[0][q]);
            mv = max(mv, s[1][q]);
            mw = max(mw, s[2][q]);
        }
        atomicMax(out + 0, (unsigned long long)__double_as_longlong((double)__uint_as_float(mu)));
        atomicMax(out + 1, (unsigned long long)__double_as_longlong((double)__uint_as_float(mv)));
        atomicMax(out + 2, (unsigned long long)__double_as_longlong((double)__uint_as_float(mw)));
    }
}

// dt = N47 * MIN(1e10, 2/(sqrt(umax^2+vmax^2+wmax^2)/dx + sqrt(0/dx)))
// (src/ietimestep.cpp:160-188 with maxF=maxG=maxH=0, evaluated at the
// smallest cell length, where the reference's minimum over cells sits).
__global__ void dt_kernel(const unsigned long long* vm, const double* vscale, double dxmin, double n47, double* dt) {
    // max |s*u| = |s| * max |u| exactly: rounding is monotone
    const double sc = fabs(*vscale);
    const double umax = sc * __longlong_as_double((long long)vm[0]);
    const double vmax = sc * __longlong_as_double((long long)vm[1]);
    const double wmax = sc * __longlong_as_double((long long)vm[2]);
    double cu = 1.0e10;
    const double cand = 2.0 / ((sqrt(umax * umax + vmax * vmax + wmax * wmax)) / dxmin + sqrt((4.0 * fabs(0.0)) / dxmin));
    cu = cu < cand ? cu : cand;
    *dt = n47 * cu;
}

// --------------------------------------------------------------- volume
// Second pass: one block sums the per-block partials in a fixed order.
__global__ void volume_reduce_kernel(const double* __restrict__ partial, long long n, double* out, double* t,
                                     double* vscale, const double* dt, double period) {
    __shared__ double sa[1024], sb[1024];
    double a = 0.0, b = 0.0;
    for (long long t = threadIdx.x; t < n; t += blockDim.x) {
        a += partial[2 * t];
        b += partial[2 * t + 1];
    }
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sa[threadIdx.x] += sa[threadIdx.x + s];
            sb[threadIdx.x] += sb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sa[0];
        out[1] = sb[0];
        if (t) {
            *t += *dt;
            if (period > 0.0) *vscale = cos(3.141592653589793 * *t / period);
        }
    }
}

// Standalone volume of a field (first pass), one block per (j,k) row group.
template <typename T>
__global__ void volume_direct_kernel(Layout L, const T* __restrict__ phi, const double* __restrict__ dxn,
                                     const double* __restrict__ dyn, const double* __restrict__ dzn, double psi,
                                     double* partial) {
    const double PI_REF = 3.14159265359;  // src/definitions.h:37
    const int j = blockIdx.y, k = blockIdx.z;
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < L.nx; i += blockDim.x) {
        const long long c = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx);
        const double p = (double)phi[c];
        double H = 0.0;
        if (p > psi) H = 1.0;
        if (p < -psi) H = 0.0;
        if (fabs(p) <= psi) H = 0.5 * (1.0 + p / psi + (1.0 / PI_REF) * sin((PI_REF * p) / psi));
        const double vol = dxn[i + 5] * dyn[j + 5] * dzn[k + 5];
        a += vol * (H - (1.0 - 1.0));
        b += vol * (1.0 - H - (1.0 - 1.0));
    }
    __shared__ double sa[256], sb[256];
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sa[threadIdx.x] += sa[threadIdx.x + s];
            sb[threadIdx.x] += sb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const long long blk = (long long)k * gridDim.y + j;
        partial[2 * blk] = sa[0];
        partial[2 * blk + 1] = sb[0];
    }
}

// ------------------------------------------------------- Airy velocity
// Linear (Airy) wave orbital velocity at the device clock t, written on
// every stored cell (interior and ghost layers):
//   u = a cosh(kw z_c) cos(kw x_f - om t)   (x faces, cell-centre z)
//   w = a sinh(kw z_f) sin(kw x_c - om t)   (z faces, cell-centre x)
// with a = amp om / sinh(kw depth), the bed at z = 0, and z limited to the
// still-water depth (the field above it is the one at the surface, instead of
// the exponential growth of the linear solution into the air).  The field is
// separable, so each block first tabulates the x and z factors in shared
// memory (coord: x centres, x faces, z centres, z faces of padded indices
// -3..n+2) and then writes rows with two multiplies per value.
template <typename T>
__global__ void __launch_bounds__(256) airy_kernel(Layout L, T* __restrict__ u, T* __restrict__ w,
                                                   const double* __restrict__ coord, const double* __restrict__ t,
                                                   AiryParams ap) {
    extern __shared__ double tab[];
    const int nx6 = L.nx + 6, nz6 = L.nz + 6;
    double* xu = tab;
    double* xw = tab + nx6;
    double* zu = tab + 2 * nx6;
    double* zw = tab + 2 * nx6 + nz6;
    const double tt = *t;
    for (int i = threadIdx.x; i < nx6; i += blockDim.x) {
        xu[i] = cos(ap.kw * coord[nx6 + i] - ap.om * tt);
        xw[i] = sin(ap.kw * coord[i] - ap.om * tt);
    }
    for (int k = threadIdx.x; k < nz6; k += blockDim.x) {
        // above the still-water level the surface value is carried upward
        zu[k] = ap.a * cosh(ap.kw * fmin(coord[2 * nx6 + k], ap.depth));
        zw[k] = ap.a * sinh(ap.kw * fmin(coord[2 * nx6 + nz6 + k], ap.depth));
    }
    __syncthreads();
    const int py = L.two_d ? 1 : L.ny + 6;
    const long long rows = (long long)py * nz6;
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        const int jj = (int)(r % py), kk = (int)(r / py);
        const long long base = (long long)kk * L.sz + (long long)jj * L.sy + (L.gx - 3);
        for (int i = threadIdx.x; i < nx6; i += blockDim.x) {
            u[base + i] = static_cast<T>(zu[kk] * xu[i]);
            w[base + i] = static_cast<T>(zw[kk] * xw[i]);
        }
    }
}

// --------------------------------------------------------- fluid update
// fluid_update_fsf::start (src/fluid_update_fsf.cpp:39-104) on one (j,k)
// row per block: smoothed Heaviside of phi, ro = W1 H + W3 (1-H),
// visc = W2 H + W4 (1-H) on the interior, the wall ghost layers of both
// (gcval 1: a Neumann copy into the three layers, src/gc_epol4.cpp:90-93,
// src/gc_neumann.cpp:29-54; 2D skips y), and the volume partials of
// volume_direct_kernel.
template <typename T>
__global__ void fluid_kernel(Layout L, const T* __restrict__ phi, T* __restrict__ ro, T* __restrict__ visc,
                             const double* __restrict__ dxn, const double* __restrict__ dyn,
                             const double* __restrict__ dzn, double psi, FluidConst fc, double* partial) {
    const double PI_REF = 3.14159265359;  // src/definitions.h:37
    const int j = blockIdx.y, k = blockIdx.z;
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < L.nx; i += blockDim.x) {
        const long long c = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx);
        const double p = (double)phi[c];
        double H = 0.0;
        if (p > psi) H = 1.0;
        if (p < -psi) H = 0.0;
        if (fabs(p) <= psi) H = 0.5 * (1.0 + p / psi + (1.0 / PI_REF) * sin((PI_REF * p) / psi));
        const T r = static_cast<T>(fc.ro_water * H + fc.ro_air * (1.0 - H));
        const T m = static_cast<T>(fc.visc_water * H + fc.visc_air * (1.0 - H));
        ro[c] = r;
        visc[c] = m;
        for (int q = 1; q <= 3; ++q) {
            if (i == 0) { ro[c - q] = r; visc[c - q] = m; }
            if (i == L.nx - 1) { ro[c + q] = r; visc[c + q] = m; }
            if (!L.two_d && j == 0) { ro[c - q * L.sy] = r; visc[c - q * L.sy] = m; }
            if (!L.two_d && j == L.ny - 1) { ro[c + q * L.sy] = r; visc[c + q * L.sy] = m; }
            if (k == 0 && !(L.io & kHaloZLo)) { ro[c - q * L.sz] = r; visc[c - q * L.sz] = m; }
            if (k == L.nz - 1 && !(L.io & kHaloZHi)) { ro[c + q * L.sz] = r; visc[c + q * L.sz] = m; }
        }
        const double vol = dxn[i + 5] * dyn[j + 5] * dzn[k + 5];
        a += vol * (H - (1.0 - 1.0));
        b += vol * (1.0 - H - (1.0 - 1.0));
    }
    __shared__ double sa[256], sb[256];
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sa[threadIdx.x] += sa[threadIdx.x + s];
            sb[threadIdx.x] += sb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const long long blk = (long long)k * gridDim.y + j;
        partial[2 * blk] = sa[0];
        partial[2 * blk + 1] = sb[0];
    }
}

// --------------------------------------------------------------- picard
// One pass of the picard mass correction over the interior, one block per
// (j,k) row (src/picard_f.cpp:36-113).  SHIFT: the row is first moved by
// s.pic[1] (correct_ls's "LOOP b += w", :109-110; the ghost cells keep their
// values as there).  SUM: the row's smoothed-Heaviside volume of the (moved)
// values goes to partial[row] (volcalc/volcalc2, :36-76).  One pass thus
// serves one iteration's update and the next iteration's volume.
template <typename T, bool SHIFT, bool SUM>
__global__ void __launch_bounds__(256) picard_row_kernel(Layout L, T* __restrict__ phi,
                                                         const double* __restrict__ pic, double epsi,
                                                         double cellvol, double* __restrict__ partial) {
    const double PI_REF = 3.14159265359;  // src/definitions.h:37
    const int j = blockIdx.y, k = blockIdx.z;
    const double w = SHIFT ? pic[1] : 0.0;
    double a = 0.0;
    for (int i = threadIdx.x; i < L.nx; i += blockDim.x) {
        const long long c = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx);
        T v = phi[c];
        if (SHIFT) {
            v = static_cast<T>(static_cast<double>(v) + w);
            phi[c] = v;
        }
        if (SUM) {
            const double b = static_cast<double>(v);
            double H = 0.0;
            if (b > epsi) H = 1.0;
            if (b < -epsi) H = 0.0;
            if (fabs(b) <= epsi) H = 0.5 * (1.0 + b / epsi + (1.0 / PI_REF) * sin((PI_REF * b) / epsi));
            a += cellvol * H;
        }
    }
    if (!SUM) return;
    __shared__ double sa[256];
    sa[threadIdx.x] = a;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sa[threadIdx.x] += sa[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[(long long)k * gridDim.y + j] = sa[0];
}

// Fixed-order sum of the row volumes.  mode 0: pic[0] = volume (vol1 of
// volcalc); with lsm (picard_lsm, src/picard_lsm.cpp:36-61) the step
// counter pic[3] advances and the first step's volume becomes the target
// netvol pic[2] (netvol += (Qi - Qo) dt is zero for a closed box).
// mode 1: volume is vol2, pic[1] = w = r1 - r2 with the equivalent-sphere
// radii r = ((3/4pi) vol)^(1/3) of the target (pic[0], or pic[2] with lsm)
// and of vol2 (src/picard_f.cpp:99-102, src/picard_lsm.cpp:102-105).
__global__ void picard_reduce_kernel(const double* __restrict__ partial, long long n, double* pic, int mode,
                                     int lsm) {
    const double PI_REF = 3.14159265359;
    __shared__ double sa[1024];
    double a = 0.0;
    for (long long t = threadIdx.x; t < n; t += blockDim.x) a += partial[t];
    sa[threadIdx.x] = a;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sa[threadIdx.x] += sa[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (mode == 0) {
            pic[0] = sa[0];
            if (lsm) {
                pic[3] += 1.0;
                if (pic[3] == 1.0) pic[2] = sa[0];
            }
        } else if (mode == 1) {
            const double r1 = pow((0.75 / PI_REF) * (lsm ? pic[2] : pic[0]), 1.0 / 3.0);
            const double r2 = pow((0.75 / PI_REF) * sa[0], 1.0 / 3.0);
            pic[1] = r1 - r2;
        } else {
            pic[4] = sa[0];  // mode 2: this subdomain's share only (the grid's sum follows)
        }
    }
}

// Picard over the slabs of a decomposed grid (the globalsum of
// src/picard_f.cpp:53 and :75): p holds each slab's pic[0..4], gathered.
// mode 0 (after volcalc): every slab's step-start volume becomes the grid's,
// and picard_lsm's first-step target too; mode 1 (after an iteration's
// volume): w = r(target) - r(grid's vol2) for every slab.
__global__ void domain_picard_kernel(double* p, int n, int mode, int lsm) {
    const double PI_REF = 3.14159265359;
    double v = 0.0;
    for (int s = 0; s < n; ++s) v += p[5 * s + (mode == 0 ? 0 : 4)];
    if (mode == 0) {
        for (int s = 0; s < n; ++s) {
            p[5 * s] = v;
            if (lsm && p[5 * s + 3] == 1.0) p[5 * s + 2] = v;
        }
    } else {
        const double r1 = pow((0.75 / PI_REF) * (lsm ? p[2] : p[0]), 1.0 / 3.0);
        const double r2 = pow((0.75 / PI_REF) * v, 1.0 / 3.0);
        for (int s = 0; s < n; ++s) p[5 * s + 1] = r1 - r2;
    }
}

template <typename T, bool SHIFT, bool SUM>
void picard_pass(const Layout& L, void* phi, double epsi, double cellvol, const Scratch& s, cudaStream_t st) {
    const dim3 grid(1, L.ny, L.nz), block(256);
    picard_row_kernel<T, SHIFT, SUM><<<grid, block, 0, st>>>(L, static_cast<T*>(phi), s.pic, epsi, cellvol, s.partial);
}

template <bool SHIFT, bool SUM>
void picard_pass(const Layout& L, void* phi, bool fp32, double epsi, double cellvol, const Scratch& s,
                 cudaStream_t st) {
    if (fp32) picard_pass<float, SHIFT, SUM>(L, phi, epsi, cellvol, s, st);
    else picard_pass<double, SHIFT, SUM>(L, phi, epsi, cellvol, s, st);
}

// --------------------------------------------------------- ioflow hooks
constexpr int kIoThreads = 1024;

// Zero-crossing water level of column i over the face's cells
// (src/ioflow_waterlevel.cpp:48-58 inflow, :84-91 outflow): a cell counts
// when phi(i,j,k) >= 0 > phi(i,j,k+1), with the height
//     -(phi(i,j,k) DZP[k]) / (phi(i,j,k+1) - phi(i,j,k)) + ZP[k].
// The cells are visited in the order of the reference's boundary list
// (j outer, k inner); every thread forms the height of one cell, the block
// compacts the crossings in that order and thread 0 adds them one by one,
// so the FP64 sum rounds exactly as the reference's loop does.  zval is
// valid in thread 0, count in every thread.
template <typename T>
__device__ __forceinline__ bool crossing_height(const Layout& L, const T* __restrict__ phi, int i, const IoParams& p,
                                                int j, int k, double& h) {
    const long long c = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx);
    const double a = static_cast<double>(phi[c]), b = static_cast<double>(phi[c + L.sz]);
    if (!(a >= 0.0 && b < 0.0)) return false;
    h = -(a * p.dzp[k + 5]) / (b - a) + p.zp[k + 5];
    return true;
}

// The face's cells of one grid (the crossing heights formed on the spot).
template <typename T>
struct CellHeights {
    Layout L;
    const T* phi;
    IoParams p;
    int i;
    __device__ int size() const { return L.ny * L.nz; }
    __device__ bool at(int e, double& h) const {
        const int j = e / L.nz, k = e - j * L.nz;
        return crossing_height(L, phi, i, p, j, k, h);
    }
};

// Heights gathered from the slabs of a decomposed grid, in the order
// j * nz + k of the whole grid (NaN: no crossing in that cell).
struct GatheredHeights {
    const double* h;
    int n;
    __device__ int size() const { return n; }
    __device__ bool at(int e, double& v) const {
        v = h[e];
        return !isnan(v);
    }
};

template <typename Src>
__device__ void crossing_sum(const Src& src, double& zval, int& count) {
    __shared__ double vals[kIoThreads];
    __shared__ int wc[kIoThreads / 32];
    const int n = src.size();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    zval = 0.0;
    count = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        const int e = base + threadIdx.x;
        bool hit = false;
        double h = 0.0;
        if (e < n) hit = src.at(e, h);
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) wc[warp] = __popc(m);
        __syncthreads();
        int off = __popc(m & ((1u << lane) - 1u)), total = 0;
        for (int w = 0; w < nwarp; ++w) {
            if (w < warp) off += wc[w];
            total += wc[w];
        }
        if (hit) vals[off] = h;
        __syncthreads();
        if (threadIdx.x == 0)
            for (int q = 0; q < total; ++q) zval += vals[q];
        count += total;
        __syncthreads();
    }
}

// ioflow_f::fsfinflow, the measuring half (src/ioflow_waterlevel.cpp:29-125):
// advances the step count (lexer::count of this step), sets phimean from
// F56/F60 or the inflow crossings, phiout from F60/F62 or the outflow
// crossings, and the outflow level wsfout (F62, or its ramp from F60 over
// F64 steps).  One block.
template <typename In, typename Out>
__device__ void io_levels(const In& in, const Out& out, const IoParams& p) {
    double* st = p.state;
    double phimean = p.f56, phiout = st[kIoPhiout];
    if (p.f60 > -1.0e20) {
        phimean = p.f60;
        phiout = p.f60;
    }
    if (p.f62 > -1.0e20) phiout = p.f62;
    double zval = 0.0;
    int count = 0, found = 0;
    if (p.inflow) {
        crossing_sum(in, zval, count);
        if (count > 0) {
            phimean = zval / static_cast<double>(count);
            found = 1;
        }
    }
    if (p.outflow) {
        crossing_sum(out, zval, count);
        if (count > 0) phiout = zval / static_cast<double>(count);
    }
    if (threadIdx.x != 0) return;
    const double cnt = st[kIoCount] + 1.0;
    double wsfout = phimean;
    if (p.f62 > 1.0e-20) {
        if (p.f64 == 0) wsfout = p.f62;
        if (p.f64 > 0) {
            // f = 0.5 cos(PI + PI count/F64) + 0.5 below F64 (tabulated on the host)
            const double f = cnt < static_cast<double>(p.f64) ? p.ramp[static_cast<int>(cnt)] : 1.0;
            wsfout = f * p.f62 + (1.0 - f) * p.f60;
        }
    }
    st[kIoCount] = cnt;
    st[kIoPhimean] = phimean;
    st[kIoPhiout] = phiout;
    st[kIoWsfout] = wsfout;
    st[kIoFound] = found;
}

template <typename T>
__global__ void __launch_bounds__(kIoThreads) io_level_kernel(Layout L, const T* __restrict__ phi, IoParams p) {
    io_levels(CellHeights<T>{L, phi, p, -1}, CellHeights<T>{L, phi, p, L.nx - 1}, p);
}

// One slab's crossing heights (NaN where none) of the inflow column (out[0,
// ny nz)) and the outflow column (out[ny nz, 2 ny nz)), j-major over its own
// cells, for the gather into the whole grid's order.
template <typename T>
__global__ void __launch_bounds__(256) io_heights_kernel(Layout L, const T* __restrict__ phi, IoParams p,
                                                         double* __restrict__ out) {
    const int n = L.ny * L.nz;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 2 * n) return;
    const int f = e / n, r = e - f * n, j = r / L.nz, k = r - j * L.nz;
    double h = 0.0;
    const bool on = f == 0 ? p.inflow : p.outflow;
    out[e] = on && crossing_height(L, phi, f == 0 ? -1 : L.nx - 1, p, j, k, h) ? h : nan("");
}

// The measuring half of fsfinflow for a decomposed grid: the gathered
// heights folded in the undivided grid's order, so the levels are the
// undivided grid's bit for bit.  p.state: the grid's state (one copy).
__global__ void __launch_bounds__(kIoThreads) io_fold_kernel(const double* __restrict__ heights, int n, IoParams p) {
    io_levels(GatheredHeights{heights, n}, GatheredHeights{heights + n, n}, p);
}

// The imposing half of fsfinflow (step == 1): inflow ghosts of phi =
// phimean - ZP when a crossing was found and F50 is 2 or 4 (:60-73),
// outflow ghosts = wsfout - ZP with F62 set and B77 = 2 (:119-130).  Then
// fsfrkin / fsfrkout (:143-177) on both RK buffers: inflow ghosts copy
// phi's, outflow ghosts copy phi's or hold F62 - ZP (F62 set, B77 = 2).
// One thread per (j,k) of the x faces.
template <typename T>
__global__ void __launch_bounds__(256) io_ghost_kernel(Layout L, T* __restrict__ phi, T* __restrict__ a1,
                                                       T* __restrict__ a2, IoParams p, int step) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= L.ny * L.nz) return;
    const int j = e / L.nz, k = e - j * L.nz;
    const double zc = p.zp[k + 5];
    const long long row = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + L.gx;
    if (p.inflow) {
        if (step && !p.waves && p.state[kIoFound] != 0.0 && (p.f50 == 2 || p.f50 == 4)) {
            const T v = static_cast<T>(p.state[kIoPhimean] - zc);
            for (int q = 1; q <= 3; ++q) phi[row - q] = v;
        }
        for (int q = 1; q <= 3; ++q) {
            const T v = phi[row - q];
            a1[row - q] = v;
            a2[row - q] = v;
        }
    }
    if (p.outflow) {
        const long long c = row + L.nx - 1;
        const bool fixed = !p.waves && p.f62 > -1.0e20 && p.b77 == 2;
        if (step && fixed) {
            const T v = static_cast<T>(p.state[kIoWsfout] - zc);
            for (int q = 1; q <= 3; ++q) phi[c + q] = v;
        }
        for (int q = 1; q <= 3; ++q) {
            const T v = fixed ? static_cast<T>(p.f62 - zc) : phi[c + q];
            a1[c + q] = v;
            a2[c + q] = v;
        }
    }
}

// ------------------------------------------------------ VTU point data
// Cell value as the reference's fields hold it around the interior: face
// ghosts as stored (the y face ghosts of a 2D field, which start4 skips, as
// zero), the first diagonal (edge) ghosts as the copy of the diagonal
// interior cell that dgcpol4 writes (src/gc_dgcpol4.cpp:28-50, also in 2D);
// the eight triple-corner ghosts, which nothing in the reference writes, as
// the corner cell.
template <typename T>
__device__ __forceinline__ double vtu_cell(const Layout& L, const T* f, int i, int j, int k) {
    const int out = (i < 0 || i >= L.nx) + (j < 0 || j >= L.ny) + (k < 0 || k >= L.nz);
    if (out == 1 && L.two_d && j != 0) return 0.0;
    if (out >= 2) {
        i = i < 0 ? 0 : (i >= L.nx ? L.nx - 1 : i);
        j = j < 0 ? 0 : (j >= L.ny ? L.ny - 1 : j);
        k = k < 0 ? 0 : (k >= L.nz ? L.nz - 1 : k);
    }
    return static_cast<double>(f[(long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx)]);
}

// Point data of the reference's VTU printer at the grid nodes (TPLOOP:
// node (i,j,k) for i,j,k = -1..n-1, between cells i and i+1; i fastest),
// src/printer_CFD.cpp:678-727:
//   phi: ipol4phi, the mean of the 8 surrounding cells
//        (src/interpolation_ipol.cpp:480-541);
//   rho: ipol4_a, 8 cells (2D: the 4 of the j = 0 plane) (:543-559);
//   viscosity: ipol4, the surrounding interior cells only (flag4 > 0),
//        divided by 8 (2D: 4) all the same (:326-372).
// Computed in FP64 in the reference's operation order, stored as float.
template <typename T>
__global__ void __launch_bounds__(256) vtu_node_kernel(Layout L, const T* __restrict__ phi, const T* __restrict__ ro,
                                                       const T* __restrict__ visc, float* __restrict__ out,
                                                       long long npoints) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= npoints) return;
    const int nyp = L.two_d ? 2 : L.ny + 1;
    const int i = (int)(n % (L.nx + 1)) - 1;
    const int j = (int)((n / (L.nx + 1)) % nyp) - 1;
    const int k = (int)(n / ((long long)(L.nx + 1) * nyp)) - 1;
    auto b = [&](const T* f, int di, int dj, int dk) { return vtu_cell(L, f, i + di, j + dj, k + dk); };
    out[n] = (float)(0.125 * (b(phi, 0, 0, 0) + b(phi, 0, 1, 0) + b(phi, 1, 0, 0) + b(phi, 1, 1, 0) +
                              b(phi, 0, 0, 1) + b(phi, 0, 1, 1) + b(phi, 1, 0, 1) + b(phi, 1, 1, 1)));
    if (!ro) return;
    double r, m;
    auto in = [&](int di, int dj, int dk) {
        const int ii = i + di, jj = j + dj, kk = k + dk;
        return ii >= 0 && ii < L.nx && jj >= 0 && jj < L.ny && kk >= 0 && kk < L.nz;
    };
    if (L.two_d) {
        // ipol4_a and ipol4 evaluate at j = 0 in 2D
        const int jj = -j;
        r = 0.25 * (b(ro, 0, jj, 0) + b(ro, 1, jj, 0) + b(ro, 0, jj, 1) + b(ro, 1, jj, 1));
        const double v1 = in(0, jj, 0) ? b(visc, 0, jj, 0) : 0.0, v2 = in(1, jj, 0) ? b(visc, 1, jj, 0) : 0.0;
        const double v3 = in(0, jj, 1) ? b(visc, 0, jj, 1) : 0.0, v4 = in(1, jj, 1) ? b(visc, 1, jj, 1) : 0.0;
        m = 0.25 * (v1 + v2 + v3 + v4);
    } else {
        r = 0.125 * (b(ro, 0, 0, 0) + b(ro, 0, 1, 0) + b(ro, 1, 0, 0) + b(ro, 1, 1, 0) + b(ro, 0, 0, 1) +
                     b(ro, 0, 1, 1) + b(ro, 1, 0, 1) + b(ro, 1, 1, 1));
        double v[8];
        const int d[8][3] = {{0, 0, 0}, {0, 1, 0}, {1, 0, 0}, {1, 1, 0}, {0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = in(d[q][0], d[q][1], d[q][2]) ? b(visc, d[q][0], d[q][1], d[q][2]) : 0.0;
        m = 0.125 * (v[0] + v[1] + v[2] + v[3] + v[4] + v[5] + v[6] + v[7]);
    }
    out[npoints + n] = (float)r;
    out[2 * npoints + n] = (float)m;
}

// --------------------------------------------------------- solid forcing
// One dependency level of ghostcell::solid_forcing_lsm
// (src/gc_solid_forcing_lsm.cpp:27-78): ops[3q..3q+2] = the entry cell and
// the two cells beyond its side (device indices); the host puts every entry
// after the earlier entries whose cells it writes or reads, so the entries
// of one level touch disjoint cells and the result is the reference's
// sequential one.
template <typename T>
__global__ void __launch_bounds__(256) solid_forcing_kernel(T* __restrict__ f, const long long* __restrict__ ops,
                                                            int n) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const T v = f[ops[3 * q]];
    f[ops[3 * q + 1]] = v;
    f[ops[3 * q + 2]] = v;
}

// picard_lsm::correct_ls's target update netvol = netvol + Qi dt - Qo dt
// (src/picard_lsm.cpp:93), before its iterations.
__global__ void netvol_kernel(double* pic, const double* dt, double qi, double qo) {
    pic[2] = pic[2] + qi * *dt - qo * *dt;
}

}  // namespace

int launch_io_hooks(const Layout& L, void* phi, void* a1, void* a2, bool fp32, const IoParams& p, bool step,
                    cudaStream_t st) {
    const int rows = L.ny * L.nz;
    const int blocks = (rows + 255) / 256;
    int n = 0;
    if (step && !p.waves) {
        if (fp32) io_level_kernel<float><<<1, kIoThreads, 0, st>>>(L, static_cast<const float*>(phi), p);
        else io_level_kernel<double><<<1, kIoThreads, 0, st>>>(L, static_cast<const double*>(phi), p);
        ++n;
    }
    if (fp32)
        io_ghost_kernel<float><<<blocks, 256, 0, st>>>(L, static_cast<float*>(phi), static_cast<float*>(a1),
                                                       static_cast<float*>(a2), p, step ? 1 : 0);
    else
        io_ghost_kernel<double><<<blocks, 256, 0, st>>>(L, static_cast<double*>(phi), static_cast<double*>(a1),
                                                        static_cast<double*>(a2), p, step ? 1 : 0);
    return n + 1;
}

int launch_io_heights(const Layout& L, const void* phi, bool fp32, const IoParams& p, double* out, cudaStream_t st) {
    const int blocks = (2 * L.ny * L.nz + 255) / 256;
    if (fp32) io_heights_kernel<float><<<blocks, 256, 0, st>>>(L, static_cast<const float*>(phi), p, out);
    else io_heights_kernel<double><<<blocks, 256, 0, st>>>(L, static_cast<const double*>(phi), p, out);
    return 1;
}

int launch_io_fold(const double* heights, int n, const IoParams& p, cudaStream_t st) {
    io_fold_kernel<<<1, kIoThreads, 0, st>>>(heights, n, p);
    return 1;
}

int launch_io_ghosts(const Layout& L, void* phi, void* a1, void* a2, bool fp32, const IoParams& p, cudaStream_t st) {
    const int blocks = (L.ny * L.nz + 255) / 256;
    if (fp32)
        io_ghost_kernel<float><<<blocks, 256, 0, st>>>(L, static_cast<float*>(phi), static_cast<float*>(a1),
                                                       static_cast<float*>(a2), p, 1);
    else
        io_ghost_kernel<double><<<blocks, 256, 0, st>>>(L, static_cast<double*>(phi), static_cast<double*>(a1),
                                                        static_cast<double*>(a2), p, 1);
    return 1;
}

int launch_dt_from_max(double dxmin, double n47, const Scratch& s, cudaStream_t st) {
    dt_kernel<<<1, 1, 0, st>>>(s.vmax, s.vscale, dxmin, n47, s.dt);
    return 1;
}

int launch_vtu_nodes(const Layout& L, const void* phi, const void* ro, const void* visc, bool fp32, float* out,
                     long long npoints, cudaStream_t st) {
    const unsigned blocks = (unsigned)((npoints + 255) / 256);
    if (fp32)
        vtu_node_kernel<float><<<blocks, 256, 0, st>>>(L, static_cast<const float*>(phi), static_cast<const float*>(ro),
                                                       static_cast<const float*>(visc), out, npoints);
    else
        vtu_node_kernel<double><<<blocks, 256, 0, st>>>(L, static_cast<const double*>(phi),
                                                        static_cast<const double*>(ro),
                                                        static_cast<const double*>(visc), out, npoints);
    return 1;
}

// Relaxation zones (iowave::phi_relax, src/iowave_relax.cpp:346-378), one
// thread per (zone column, k).  In the generation zone
//   f = (1 - relax4_wg) ramp lsval + relax4_wg f,
// then in the beach zone
//   f = (1 - relax4_nb) (phimean - z) + relax4_nb f,
// in the reference's operation order (FP64; the FP32 form rounds the
// result), and the relaxed value goes into the cell's wall ghost layers as
// ghostcell::start4 afterwards does (src/levelset_RK3.cpp:125-127).
template <typename T>
__global__ void relax_kernel(Layout L, T* f, RelaxZones z) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)z.ncol * L.nz) return;
    const int q = (int)(t / L.nz), k = (int)(t % L.nz);
    const int i = z.col[4 * q], j = z.col[4 * q + 1], zone = z.col[4 * q + 2], off = z.col[4 * q + 3];
    const long long c = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx);
    double v = (double)f[c];
    if (zone & 1) {
        const double w = z.w[2 * q];
        v = (1.0 - w) * (*z.ramp) * z.lsval[off + k] + w * v;
    }
    if (zone & 2) {
        const double w = z.w[2 * q + 1];
        v = (1.0 - w) * (z.phimean - z.zc[k]) + w * v;
    }
    const T val = (T)v;
    f[c] = val;
    if ((L.io & kIoEdge) && i == 0 && k == L.nz - 1) f[c - 1 + L.sz] = val;
    for (int r = 1; r <= 3; ++r) {
        if (i == 0 && !(L.io & kIoSkipLo)) f[c - r] = val;
        if (i == L.nx - 1 && !(L.io & kIoSkipHi)) f[c + r] = val;
        if (!L.two_d && j == 0) f[c - r * L.sy] = val;
        if (!L.two_d && j == L.ny - 1) f[c + r * L.sy] = val;
        if (k == 0 && !(L.io & kHaloZLo)) f[c - r * L.sz] = val;
        if (k == L.nz - 1 && !(L.io & kHaloZHi)) f[c + r * L.sz] = val;
    }
}

int launch_relax(const Layout& L, void* f, bool fp32, const RelaxZones& z, cudaStream_t st) {
    const long long n = (long long)z.ncol * L.nz;
    if (n <= 0) return 0;
    const unsigned g = (unsigned)((n + 255) / 256);
    if (fp32) relax_kernel<float><<<g, 256, 0, st>>>(L, static_cast<float*>(f), z);
    else relax_kernel<double><<<g, 256, 0, st>>>(L, static_cast<double*>(f), z);
    return 1;
}

int launch_solid_forcing(void* f, bool fp32, const long long* ops, const std::vector<int>& level_off,
                         cudaStream_t st) {
    int n = 0;
    for (size_t l = 0; l + 1 < level_off.size(); ++l) {
        const int cnt = level_off[l + 1] - level_off[l];
        if (cnt <= 0) continue;
        const long long* o = ops + 3LL * level_off[l];
        if (fp32) solid_forcing_kernel<float><<<(cnt + 255) / 256, 256, 0, st>>>(static_cast<float*>(f), o, cnt);
        else solid_forcing_kernel<double><<<(cnt + 255) / 256, 256, 0, st>>>(static_cast<double*>(f), o, cnt);
        ++n;
    }
    return n;
}

// One time step for every slab of a decomposed grid: the maxima over the
// slabs' CFL maxima (gathered into vm[3 n], pgc->globalmax,
// src/ietimestep.cpp) and the expression of dt_kernel at the smallest cell
// of the whole grid.
__global__ void domain_dt_kernel(const unsigned long long* vm, int n, const double* vscale, double dxmin, double n47,
                                 double* dt) {
    unsigned long long m[3] = {0, 0, 0};
    for (int s = 0; s < n; ++s)
        for (int a = 0; a < 3; ++a) m[a] = vm[3 * s + a] > m[a] ? vm[3 * s + a] : m[a];
    const double sc = fabs(*vscale);
    const double umax = sc * __longlong_as_double((long long)m[0]);
    const double vmax = sc * __longlong_as_double((long long)m[1]);
    const double wmax = sc * __longlong_as_double((long long)m[2]);
    double cu = 1.0e10;
    const double cand = 2.0 / ((sqrt(umax * umax + vmax * vmax + wmax * wmax)) / dxmin + sqrt((4.0 * fabs(0.0)) / dxmin));
    cu = cu < cand ? cu : cand;
    *dt = n47 * cu;
}

int launch_domain_dt(const unsigned long long* vm, int n, const double* vscale, double dxmin, double n47, double* dt,
                     cudaStream_t st) {
    domain_dt_kernel<<<1, 1, 0, st>>>(vm, n, vscale, dxmin, n47, dt);
    return 1;
}

int launch_picard_local(const Layout& L, void* phi, bool fp32, double epsi, double cellvol, bool shift, bool sum,
                        int mode, bool lsm, const Scratch& s, cudaStream_t st) {
    if (shift && sum) picard_pass<true, true>(L, phi, fp32, epsi, cellvol, s, st);
    else if (shift) picard_pass<true, false>(L, phi, fp32, epsi, cellvol, s, st);
    else picard_pass<false, true>(L, phi, fp32, epsi, cellvol, s, st);
    if (!sum) return 1;
    picard_reduce_kernel<<<1, 1024, 0, st>>>(s.partial, (long long)L.ny * L.nz, s.pic, mode, lsm ? 1 : 0);
    return 2;
}

int launch_domain_picard(double* gathered, int n, int mode, bool lsm, cudaStream_t st) {
    domain_picard_kernel<<<1, 1, 0, st>>>(gathered, n, mode, lsm ? 1 : 0);
    return 1;
}

int launch_netvol(const Scratch& s, double qi, double qo, cudaStream_t st) {
    netvol_kernel<<<1, 1, 0, st>>>(s.pic, s.dt, qi, qo);
    return 1;
}

size_t airy_smem_bytes(const Layout& L) { return (size_t)(2 * (L.nx + 6) + 2 * (L.nz + 6)) * sizeof(double); }

int launch_airy(const Layout& L, void* u, void* w, bool fp32, const double* coord, const double* t,
                const AiryParams& ap, int sms, cudaStream_t st) {
    const long long rows = (long long)(L.two_d ? 1 : L.ny + 6) * (L.nz + 6);
    const int grid = (int)(rows < 4LL * sms ? rows : 4LL * sms);
    const size_t smem = airy_smem_bytes(L);
    if (fp32)
        airy_kernel<float><<<grid, 256, smem, st>>>(L, static_cast<float*>(u), static_cast<float*>(w), coord, t, ap);
    else
        airy_kernel<double><<<grid, 256, smem, st>>>(L, static_cast<double*>(u), static_cast<double*>(w), coord, t,
                                                     ap);
    return 1;
}

int airy_prepare(const Layout& L) {
    const size_t smem = airy_smem_bytes(L);
    if (smem > 227 * 1024) return 1;
    if (smem > 48 * 1024) {
        if (cudaFuncSetAttribute(airy_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                cudaSuccess ||
            cudaFuncSetAttribute(airy_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                cudaSuccess)
            return 1;
    }
    return 0;
}

int launch_fluid_update(const Layout& L, const void* phi, void* ro, void* visc, bool fp32, const double* dxn,
                        const double* dyn, const double* dzn, double psi, const FluidConst& fc, bool clock,
                        double period, const Scratch& s, cudaStream_t st) {
    const dim3 grid(1, L.ny, L.nz), block(256);
    if (fp32)
        fluid_kernel<float><<<grid, block, 0, st>>>(L, static_cast<const float*>(phi), static_cast<float*>(ro),
                                                    static_cast<float*>(visc), dxn, dyn, dzn, psi, fc, s.partial);
    else
        fluid_kernel<double><<<grid, block, 0, st>>>(L, static_cast<const double*>(phi), static_cast<double*>(ro),
                                                     static_cast<double*>(visc), dxn, dyn, dzn, psi, fc, s.partial);
    if (clock)
        volume_reduce_kernel<<<1, 1024, 0, st>>>(s.partial, (long long)L.ny * L.nz, s.vol, s.t, s.vscale, s.dt,
                                                 period);
    else
        volume_reduce_kernel<<<1, 1024, 0, st>>>(s.partial, (long long)L.ny * L.nz, s.vol, nullptr, nullptr,
                                                 nullptr, 0.0);
    return 2;
}

int launch_picard_volcalc(const Layout& L, const void* phi, bool fp32, double epsi, double cellvol, bool lsm,
                          const Scratch& s, cudaStream_t st) {
    picard_pass<false, true>(L, const_cast<void*>(phi), fp32, epsi, cellvol, s, st);
    picard_reduce_kernel<<<1, 1024, 0, st>>>(s.partial, (long long)L.ny * L.nz, s.pic, 0, lsm);
    return 2;
}

int launch_picard_correct(const Layout& L, void* phi, bool fp32, double epsi, double cellvol, int f47, bool lsm,
                          const Scratch& s, cudaStream_t st) {
    if (f47 <= 0) return 0;
    const long long rows = (long long)L.ny * L.nz;
    picard_pass<false, true>(L, phi, fp32, epsi, cellvol, s, st);
    picard_reduce_kernel<<<1, 1024, 0, st>>>(s.partial, rows, s.pic, 1, lsm);
    for (int n = 1; n < f47; ++n) {
        picard_pass<true, true>(L, phi, fp32, epsi, cellvol, s, st);
        picard_reduce_kernel<<<1, 1024, 0, st>>>(s.partial, rows, s.pic, 1, lsm);
    }
    picard_pass<true, false>(L, phi, fp32, epsi, cellvol, s, st);
    return 2 * f47 + 1;
}

int launch_import(const Layout& L, const double* staging, int layout, void* dst, bool fp32, cudaStream_t st) {
    const int py = L.two_d ? 1 : L.ny + 6;
    const dim3 grid((L.nx + 6 + 127) / 128, py, L.nz + 6), block(128);
    if (fp32) import_kernel<float><<<grid, block, 0, st>>>(L, staging, layout, static_cast<float*>(dst));
    else import_kernel<double><<<grid, block, 0, st>>>(L, staging, layout, static_cast<double*>(dst));
    return 1;
}

int launch_export(const Layout& L, const void* src, bool fp32, int layout, double* staging, cudaStream_t st) {
    const int py = L.two_d ? 1 : L.ny + 6;
    const dim3 grid((L.nx + 6 + 127) / 128, py, L.nz + 6), block(128);
    if (fp32) export_kernel<float><<<grid, block, 0, st>>>(L, static_cast<const float*>(src), layout, staging);
    else export_kernel<double><<<grid, block, 0, st>>>(L, static_cast<const double*>(src), layout, staging);
    return 1;
}

int launch_ghost_fill(const Layout& L, void* f, bool fp32, cudaStream_t st) {
    const dim3 grid((L.nx + 127) / 128, L.ny, L.nz), block(128);
    if (fp32) ghost_kernel<float><<<grid, block, 0, st>>>(L, static_cast<float*>(f));
    else ghost_kernel<double><<<grid, block, 0, st>>>(L, static_cast<double*>(f));
    return 1;
}

int launch_cfl(const Layout& L, const void* u, const void* v, const void* w, bool fp32, double dxmin, double n47,
               const Scratch& s, cudaStream_t st) {
    cudaMemsetAsync(s.vmax, 0, 3 * sizeof(unsigned long long), st);
    const long long rows = (long long)L.ny * L.nz;
    const dim3 grid((unsigned)(rows < 1184 ? rows : 1184)), block(256);
    if (fp32) {
        const long long items = rows * ((L.nx + 3) / 4);
        const long long blocks = (items + 255) / 256;
        vmax_f32_kernel<<<(unsigned)(blocks < 148 * 8 ? blocks : 148 * 8), 256, 0, st>>>(
            L, static_cast<const float*>(u), static_cast<const float*>(v), static_cast<const float*>(w), s.vmax);
    } else
        vmax_kernel<double><<<grid, block, 0, st>>>(L, static_cast<const double*>(u), static_cast<const double*>(v),
                                                    static_cast<const double*>(w), s.vmax);
    dt_kernel<<<1, 1, 0, st>>>(s.vmax, s.vscale, dxmin, n47, s.dt);
    return 2;
}

int launch_volume_reduce(const Layout&, const Scratch& s, long long nblocks, double period, cudaStream_t st) {
    volume_reduce_kernel<<<1, 1024, 0, st>>>(s.partial, nblocks, s.vol, s.t, s.vscale, s.dt, period);
    return 1;
}

int launch_volume_direct(const Layout& L, const void* phi, bool fp32, const double* dxn, const double* dyn,
                         const double* dzn, double psi, const Scratch& s, cudaStream_t st) {
    const dim3 grid(1, L.ny, L.nz), block(256);
    if (fp32)
        volume_direct_kernel<float><<<grid, block, 0, st>>>(L, static_cast<const float*>(phi), dxn, dyn, dzn, psi,
                                                            s.partial);
    else
        volume_direct_kernel<double><<<grid, block, 0, st>>>(L, static_cast<const double*>(phi), dxn, dyn, dzn, psi,
                                                             s.partial);
    volume_reduce_kernel<<<1, 1024, 0, st>>>(s.partial, (long long)L.ny * L.nz, s.vol, nullptr, nullptr, nullptr,
                                             0.0);
    return 2;
}

int launch_volume_direct_clock(const Layout& L, const void* phi, bool fp32, const double* dxn, const double* dyn,
                               const double* dzn, double psi, double period, const Scratch& s, cudaStream_t st) {
    const dim3 grid(1, L.ny, L.nz), block(256);
    if (fp32)
        volume_direct_kernel<float><<<grid, block, 0, st>>>(L, static_cast<const float*>(phi), dxn, dyn, dzn, psi,
                                                            s.partial);
    else
        volume_direct_kernel<double><<<grid, block, 0, st>>>(L, static_cast<const double*>(phi), dxn, dyn, dzn, psi,
                                                             s.partial);
    volume_reduce_kernel<<<1, 1024, 0, st>>>(s.partial, (long long)L.ny * L.nz, s.vol, s.t, s.vscale, s.dt, period);
    return 2;
}

namespace {
__global__ void set_scalar_kernel(double* dst, double value) { *dst = value; }

// Initial fields of a sphere-union / Taylor-Green case on every stored cell
// (interior and ghosts): phi = min over spheres of |x - c| - r (circles in
// the x-z plane in 2D) at cell centres; u, v, w = sum of Taylor-Green modes
// at the x, y, z faces.  xc/xf hold, per axis, the centre and face
// coordinates of padded indices -3..n+2.
template <typename T>
__global__ void init_kernel(Layout L, const double* __restrict__ xc, const double* __restrict__ xf, int ns,
                            const double* __restrict__ sph, int nm, const double* __restrict__ modes, T* phi, T* u,
                            T* v, T* w) {
    const int gyp = L.two_d ? 0 : 3;
    const int i = blockIdx.x * blockDim.x + threadIdx.x - 3;
    const int j = blockIdx.y - gyp;
    const int k = blockIdx.z - 3;
    if (i >= L.nx + 3) return;
    const int nx6 = L.nx + 6, ny6 = L.ny + 6;
    const double* cx = xc;
    const double* cy = xc + nx6;
    const double* cz = xc + nx6 + ny6;
    const double* fx = xf;
    const double* fy = xf + nx6;
    const double* fz = xf + nx6 + ny6;
    const double X = cx[i + 3], Y = cy[j + 3], Z = cz[k + 3];
    double d = 1e30;
    for (int s = 0; s < ns; ++s) {
        const double ex = X - sph[4 * s], ey = Y - sph[4 * s + 1], ez = Z - sph[4 * s + 2];
        const double e = (L.two_d ? sqrt(ex * ex + ez * ez) : sqrt(ex * ex + ey * ey + ez * ez)) - sph[4 * s + 3];
        d = e < d ? e : d;
    }
    double uu = 0.0, vv = 0.0, ww = 0.0;
    for (int m = 0; m < nm; ++m) {
        const double kk = modes[2 * m] * 3.141592653589793, A = modes[2 * m + 1];
        if (L.two_d) {
            uu += A * sin(kk * fx[i + 3]) * cos(kk * Z);
            ww += -A * cos(kk * X) * sin(kk * fz[k + 3]);
        } else {
            uu += A * sin(kk * fx[i + 3]) * cos(kk * Y) * cos(kk * Z);
            vv += -A * cos(kk * X) * sin(kk * fy[j + 3]) * cos(kk * Z);
        }
    }
    const long long c = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx);
    phi[c] = (T)d;
    u[c] = (T)uu;
    v[c] = (T)vv;
    w[c] = (T)ww;
}
}  // namespace

int launch_init_fields(const Layout& L, const double* xc, const double* xf, int ns, const double* sph, int nm,
                       const double* modes, bool fp32, void* phi, void* u, void* v, void* w, cudaStream_t st) {
    const int py = L.two_d ? 1 : L.ny + 6;
    const dim3 grid((L.nx + 6 + 127) / 128, py, L.nz + 6), block(128);
    if (fp32)
        init_kernel<float><<<grid, block, 0, st>>>(L, xc, xf, ns, sph, nm, modes, (float*)phi, (float*)u, (float*)v,
                                                   (float*)w);
    else
        init_kernel<double><<<grid, block, 0, st>>>(L, xc, xf, ns, sph, nm, modes, (double*)phi, (double*)u,
                                                    (double*)v, (double*)w);
    return 1;
}

// Writes a scalar into device memory as a kernel argument, so the value is
// captured at enqueue time (also inside a CUDA graph).
int launch_set_scalar(double* dst, double value, cudaStream_t st) {
    set_scalar_kernel<<<1, 1, 0, st>>>(dst, value);
    return 1;
}

int launch_zero(void* p, size_t bytes, cudaStream_t st) {
    cudaMemsetAsync(p, 0, bytes, st);
    return 0;
}

}  // namespace r3d
