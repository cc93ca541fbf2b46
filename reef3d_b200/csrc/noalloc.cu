// Volume integral of a level set that allocates nothing.
//
// Some callers cannot allocate device memory when they call us: a host
// application that reserves all of the GPU's memory for its own pool at
// start-up and hands out pieces itself, or a time loop that must not pay
// cudaMalloc's implicit device-wide synchronisation in the middle of a step.
// For them this variant of the volume reduction keeps its per-row partial
// sums in a fixed, file-scope device array instead of instance scratch: the
// caller passes the level set and the two-double result in device memory it
// owns, and the call performs no allocation of any kind.
//
// Limits and sharing: the array holds 2 partial sums for each (j,k) row of
// the field, at most kMaxRows = 65536 rows (ny*nz <= 65536, e.g. a 256^3
// grid), 1 MiB that every GPU which loads the library keeps until the process
// exits.  All calls share that array and it keeps the last call's contents;
// every call writes each partial it reads before reading it, so nothing needs
// clearing, but two calls whose kernels overlap on a GPU (different streams,
// or different host threads on one device) race on it and must be ordered by
// the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "reef3d_b200.h"

namespace r3d {
void set_thread_error(const char* msg);  // the text r3d_last_error(NULL) returns (api.cpp)
}

namespace {

constexpr int kMaxRows = 65536;
constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;

// the scratch: 2 doubles per (j,k) row
__device__ __align__(256) double g_row_partials[2 * kMaxRows];

std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {nullptr};

// One block per (j,k) row: smoothed Heaviside of src/fluid_update_fsf.cpp:50-71
// (porosity 1, the reference's PI of src/definitions.h:37) times the cell
// volume, summed over the row in a fixed order.
__global__ void __launch_bounds__(kThreads) row_partials_kernel(const double* __restrict__ phi, int nx, int ny,
                                                                double cellvol, double psi, double* scratch) {
    const double PI_REF = 3.14159265359;
    const int row = blockIdx.x;  // row = j + ny*k
    const double* p = phi + (long long)row * nx;
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < nx; i += kThreads) {
        const double v = p[i];
        double H = 0.0;
        if (v > psi) H = 1.0;
        if (v < -psi) H = 0.0;
        if (fabs(v) <= psi) H = 0.5 * (1.0 + v / psi + (1.0 / PI_REF) * sin((PI_REF * v) / psi));
        a += cellvol * (H - (1.0 - 1.0));
        b += cellvol * (1.0 - H - (1.0 - 1.0));
    }
    __shared__ double sa[kThreads], sb[kThreads];
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sa[threadIdx.x] += sa[threadIdx.x + s];
            sb[threadIdx.x] += sb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        scratch[2 * row] = sa[0];
        scratch[2 * row + 1] = sb[0];
    }
    (void)ny;
}

// One block: the row partials in a fixed order into out[0..1].
__global__ void __launch_bounds__(1024) rows_total_kernel(const double* __restrict__ scratch, int nrows,
                                                          double* out) {
    __shared__ double sa[1024], sb[1024];
    double a = 0.0, b = 0.0;
    for (int r = threadIdx.x; r < nrows; r += blockDim.x) {
        a += scratch[2 * r];
        b += scratch[2 * r + 1];
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
    }
}

// Device address of the scratch array on the current device, looked up
// once per device (host code may not use g_row_partials itself: on the host
// that name is only a stand-in for the device symbol).
int scratch_address(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        r3d::set_thread_error((std::string("cudaGetDevice: ") + cudaGetErrorString(e)).c_str());
        return R3D_EDEVICE;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        r3d::set_thread_error("device ordinal beyond the supported range");
        return R3D_EDEVICE;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_row_partials);
        if (e != cudaSuccess || !p) {
            r3d::set_thread_error((std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)).c_str());
            return R3D_EDEVICE;
        }
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return R3D_OK;
}

}  // namespace

extern "C" int r3d_volume_dense_noalloc(const double* phi, int nx, int ny, int nz, double dx, double dy, double dz,
                                        double psi, double* out, void* stream) {
    if (!phi || !out) {
        r3d::set_thread_error("null device pointer");
        return R3D_EINVAL;
    }
    if (nx < 1 || ny < 1 || nz < 1) {
        r3d::set_thread_error("grid sizes must be >= 1");
        return R3D_EINVAL;
    }
    if ((long long)ny * nz > kMaxRows) {
        r3d::set_thread_error("ny*nz exceeds the 65536 rows the fixed scratch array holds");
        return R3D_EINVAL;
    }
    if (!(dx > 0.0) || !(dy > 0.0) || !(dz > 0.0) || !(psi > 0.0)) {
        r3d::set_thread_error("spacings and psi must be positive");
        return R3D_EINVAL;
    }
    double* scratch = nullptr;
    if (int rc = scratch_address(&scratch)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nrows = ny * nz;
    row_partials_kernel<<<nrows, kThreads, 0, st>>>(phi, nx, ny, dx * dy * dz, psi, scratch);
    rows_total_kernel<<<1, 1024, 0, st>>>(scratch, nrows, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        r3d::set_thread_error((std::string("launch: ") + cudaGetErrorString(e)).c_str());
        return R3D_EDEVICE;
    }
    return R3D_OK;
}
