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
    for (int q = 1; q <= 3; ++q) {
        if (i == 0) f[c - q] = val;
        if (i == L.nx - 1) f[c + q] = val;
        if (!L.two_d && j == 0) f[c - q * L.sy] = val;
        if (!L.two_d && j == L.ny - 1) f[c + q * L.sy] = val;
        if (k == 0) f[c - q * L.sz] = val;
        if (k == L.nz - 1) f[c + q * L.sz] = val;
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
            if (k < L.nz - 1) mw = fmax(mw, fabs((double)w[base + i]));
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

}  // namespace

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
    if (fp32)
        vmax_kernel<float><<<grid, block, 0, st>>>(L, static_cast<const float*>(u), static_cast<const float*>(v),
                                                   static_cast<const float*>(w), s.vmax);
    else
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
