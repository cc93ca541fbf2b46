// C-ABI of libreef3d_b200.so (declared in include/reef3d_b200.h).
#include "reef3d_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "handle.h"

using namespace r3d;

namespace {

thread_local std::string g_thread_err;

int fail(r3d_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    else g_thread_err = msg;
    return code;
}

int cuda_fail(r3d_handle* h, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(h, R3D_EDEVICE, m);
}

#define R3D_CUDA(h, call)                                  \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

bool fp32(const r3d_handle* h) { return h->desc.precision == R3D_FP32; }
size_t elem(const r3d_handle* h) { return fp32(h) ? sizeof(float) : sizeof(double); }

int check_desc(const r3d_grid_desc* d, std::string& why) {
    if (!d) { why = "null descriptor"; return R3D_EINVAL; }
    if (d->nx < 1 || d->ny < 1 || d->nz < 1) { why = "grid sizes must be >= 1"; return R3D_EINVAL; }
    if (d->nx > 65535 * 32 || d->ny > 65535 || d->nz > 65535) { why = "grid size beyond launch limits"; return R3D_EINVAL; }
    if (!d->xn || !d->yn || !d->zn) { why = "node coordinates missing"; return R3D_EINVAL; }
    if (d->precision != R3D_FP64 && d->precision != R3D_FP32) { why = "precision must be R3D_FP64 or R3D_FP32"; return R3D_EINVAL; }
    if (d->f44 < 0) { why = "f44 must be >= 0"; return R3D_EINVAL; }
    if (d->f49 != 0 && d->f49 != 1) { why = "f49 must be 0 or 1"; return R3D_EINVAL; }
    if (d->f46 < 0 || d->f46 > 3) { why = "f46 must be 0, 1, 2 or 3"; return R3D_EINVAL; }
    if (d->f46 != 0 && d->f47 < 0) { why = "f47 must be >= 0"; return R3D_EINVAL; }
    const int n[3] = {d->nx, d->ny, d->nz};
    const double* x[3] = {d->xn, d->yn, d->zn};
    for (int a = 0; a < 3; ++a)
        for (int t = 0; t < n[a] + 10; ++t)
            if (!(x[a][t + 1] > x[a][t])) { why = "node coordinates must increase strictly"; return R3D_EINVAL; }
    return R3D_OK;
}

// device bytes: 7 fields + metric tables + scratch (staging excluded: it is
// allocated on first host copy)
size_t footprint(const r3d_grid_desc* d, const Layout& L) {
    const size_t e = d->precision == R3D_FP32 ? 4 : 8;
    size_t b = 7 * (size_t)L.ncell * e;
    size_t tab = 0;
    const int n[3] = {d->nx, d->ny, d->nz};
    for (int a = 0; a < 3; ++a) tab += 4 * (size_t)(n[a] + 21) + 2 * (size_t)(n[a] + 8) * 36 + 8;
    b += tab * (8 + 4);
    const long long blocks = (long long)((d->nx + 31) / 32) * ((d->ny + 3) / 4 + 4) * (d->nz + 4);
    b += (size_t)(blocks + (long long)d->ny * d->nz + 64) * 16 + 256;
    return b;
}

template <typename T>
void fill_kgrid(r3d_handle* h, KGrid<T>& g, T* base, std::vector<T>& host) {
    g.L = h->L;
    size_t off = 0;
    host.clear();
    for (int a = 0; a < 3; ++a) {
        const size_t o_dxp = off;
        for (double v : h->M.dxp[a]) host.push_back((T)v);
        off = host.size();
        const size_t o_dxn = off;
        for (double v : h->M.dxn[a]) host.push_back((T)v);
        off = host.size();
        const size_t o_qf = off;
        for (double v : h->M.qf[a]) host.push_back((T)v);
        off = host.size();
        const size_t o_cf = off;
        for (double v : h->M.cf[a]) host.push_back((T)v);
        off = host.size();
        const size_t o_isf = off;
        for (double v : h->M.isf[a]) host.push_back((T)v);
        off = host.size();
        g.dxp[a] = base + o_dxp;
        g.dxn[a] = base + o_dxn;
        g.qf[a] = base + o_qf;
        g.cf[a] = base + o_cf;
        g.isf[a] = base + o_isf;
    }
    // packed forms read by the FP64 stencils, each 16-byte aligned
    for (int a = 0; a < 3; ++a) {
        while (host.size() % 4) host.push_back((T)0);
        g.dpr[a] = base + host.size();
        for (double v : h->M.dxp[a]) {
            host.push_back((T)v);
            host.push_back((T)(1.0 / v));
        }
        while (host.size() % 4) host.push_back((T)0);
        g.wt[a] = base + host.size();
        const size_t nt = h->M.cf[a].size() / 6;
        for (size_t t = 0; t < nt; ++t)
            for (int side = 0; side < 2; ++side) {
                for (int m = 0; m < 6; ++m) host.push_back((T)h->M.qf[a][t * 12 + side * 6 + m]);
                for (int m = 0; m < 3; ++m) host.push_back((T)h->M.cf[a][t * 6 + side * 3 + m]);
                for (int m = 0; m < 9; ++m) host.push_back((T)h->M.isf[a][t * 18 + side * 9 + m]);
            }
    }
    g.f43 = h->desc.f43;
    g.f49 = h->desc.f49;
    g.psi = h->M.psi;
    for (int a = 0; a < 3; ++a) {
        g.h[a] = h->M.uniform ? (float)h->M.h[a] : 0.0f;
        g.rh[a] = h->M.uniform ? (float)(1.0 / h->M.h[a]) : 0.0f;
    }
    g.eps_u = 1.0e-6f;
}

size_t metric_count(const r3d_handle* h) {
    size_t c = 0;
    for (int a = 0; a < 3; ++a)
        c += h->M.dxp[a].size() + h->M.dxn[a].size() + h->M.qf[a].size() + h->M.cf[a].size() + h->M.isf[a].size()
             + 2 * h->M.dxp[a].size() + 6 * h->M.cf[a].size() + 8;  // packed pairs and records, padding
    return c;
}

void release(r3d_handle* h) {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
    for (void*& p : h->field) { if (p) cudaFree(p); p = nullptr; }
    if (h->metrics64) cudaFree(h->metrics64);
    if (h->metrics32) cudaFree(h->metrics32);
    if (h->S.partial) cudaFree(h->S.partial);
    if (h->S.vmax) cudaFree(h->S.vmax);
    if (h->staging) cudaFree(h->staging);
    if (h->coord) cudaFree(h->coord);
    if (h->io_buf) cudaFree(h->io_buf);
    if (h->sf_ops) cudaFree(h->sf_ops);
    if (h->rz_col) cudaFree(h->rz_col);
    if (h->rz_buf) cudaFree(h->rz_buf);
    if (h->stream) cudaStreamDestroy(h->stream);
    cudaSetDevice(cur);
}

Fields fields_of(r3d_handle* h) {
    Fields f{};
    f.phi = h->field[R3D_PHI];
    f.u = h->field[R3D_U];
    f.v = h->field[R3D_V];
    f.w = h->field[R3D_W];
    f.L = h->field[R3D_L];
    f.a1 = h->field[R3D_WORK1];
    f.a2 = h->field[R3D_WORK2];
    return f;
}

int ensure_staging(r3d_handle* h) {
    const size_t need = sizeof(double) * (size_t)(h->L.nx + 6) * (h->L.ny + 6) * (h->L.nz + 6);
    if (h->staging_bytes >= need) return R3D_OK;
    if (h->staging) cudaFree(h->staging);
    if (h->coord) cudaFree(h->coord);
    h->staging = nullptr;
    h->staging_bytes = 0;
    if (cudaMalloc(&h->staging, need) != cudaSuccess) {
        cudaGetLastError();
        return fail(h, R3D_ENOMEM, "staging allocation failed");
    }
    h->staging_bytes = need;
    return R3D_OK;
}

size_t host_count(const r3d_handle* h, int layout) {
    if (layout == R3D_LAYOUT_REEF3D) return (size_t)(h->L.nx + 6) * (h->L.ny + 6) * (h->L.nz + 6);
    return (size_t)h->L.nx * h->L.ny * h->L.nz;
}

// Makes the instance's device current for the call; if the instance is a
// batch member, its work queued on the batch's stream completes first.
struct DeviceGuard {
    int prev = 0;
    DeviceGuard(int dev, cudaStream_t batch = nullptr) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
        if (batch) cudaStreamSynchronize(batch);
    }
    ~DeviceGuard() { int cur = 0; cudaGetDevice(&cur); if (cur != prev) cudaSetDevice(prev); }
};

// The tiled kernels fill every face as a wall and know only the plain
// stencils: instances with inflow / outflow faces or direct forcing run the
// one-cell-per-thread kernels.
// the volume partials of a tiled stage (one pair per CTA) must fit the
// scratch buffer sized at creation for the cell kernels
bool tile_fits(const r3d_handle* h, int kc, int cfg) { return tile_items_of(h->L, kc, cfg) <= h->S.npartial; }
bool tiled(const r3d_handle* h) {
    return h->tile_ok && h->use_tile && !h->io && !h->g64.x45 && tile_fits(h, h->kc, h->tile_cfg) &&
           tile_fits(h, h->kc_r, h->tile_cfg_r);
}

// The body field of the direct-forcing stencils is FP64 in both forms.
size_t field_elem(const r3d_handle* h, int id) { return id == R3D_BODY ? sizeof(double) : elem(h); }
bool field_fp32(const r3d_handle* h, int id) { return fp32(h) && id != R3D_BODY; }

}  // namespace

namespace r3d {
// Tiled-kernel arguments of an instance for stage 1..3 (also used by batches).
TileArgs make_tile_args(r3d_handle* h, int stage) {
    TileArgs a{};
    a.L = h->L;
    a.fn = static_cast<const float*>(h->field[R3D_PHI]);
    a.out = static_cast<float*>(stage == 1 ? h->field[R3D_WORK1] : stage == 2 ? h->field[R3D_WORK2] : h->field[R3D_PHI]);
    a.u = static_cast<const float*>(h->field[R3D_U]);
    a.v = static_cast<const float*>(h->field[R3D_V]);
    a.w = static_cast<const float*>(h->field[R3D_W]);
    a.dt = h->S.dt;
    a.vscale = h->S.vscale;
    a.partial = h->S.partial;
    a.err = h->S.err;
    double hmin = h->M.h[0];
    for (int d = 0; d < 3; ++d) {
        a.rh[d] = (float)(1.0 / h->M.h[d]);
        a.eps[d] = (float)(1.0 / (h->M.h[d] * h->M.h[d]));
        const double hb = 1.0 / (double)a.rh[d];
        a.beps[d] = 1.0e-6 * hb * hb;
        hmin = std::fmin(hmin, h->M.h[d]);
    }
    a.dtr = (float)(h->desc.f43 * hmin);
    a.deltax = (float)((1.0 / 3.0) * (h->M.h[0] + h->M.h[1] + h->M.h[2]));
    a.f49 = h->desc.f49;
    a.band64 = h->band64;
    a.wait_test = h->wait_test;
    a.spin = h->wait_test ? (1ll << 12) : 0;
    a.psi = h->M.psi;
    a.cellvol = h->M.h[0] * h->M.h[1] * h->M.h[2];
    a.kc = h->kc;
    return a;
}
}  // namespace r3d

namespace {
TileArgs tile_args(r3d_handle* h, int stage) { return r3d::make_tile_args(h, stage); }

long long stage_launch_plain(r3d_handle* h, bool reini, int s, bool vol) {
    const Fields f = fields_of(h);
    if (tiled(h)) {
        TileArgs a = tile_args(h, s);
        a.kc = reini ? h->kc_r : h->kc;
        return launch_tile_stage(reini ? h->map_r[s - 1] : h->map[s - 1], a, reini ? h->tile_cfg_r : h->tile_cfg,
                                 reini, s, vol, h->stream);
    }
    if (fp32(h))
        return reini ? launch_reini_stage_f32(h->g32, f, s, h->S, vol, h->stream)
                     : launch_conv_stage_f32(h->g32, f, s, h->S, vol, h->stream);
    return reini ? launch_reini_stage_f64(h->g64, f, s, h->S, vol, h->stream)
                 : launch_conv_stage_f64(h->g64, f, s, h->S, vol, h->stream);
}

RelaxZones relax_zones(const r3d_handle* h) {
    RelaxZones z{};
    z.col = h->rz_col;
    z.ncol = h->rz_ncol;
    z.w = h->rz_buf;
    z.zc = h->rz_buf + 2 * (size_t)h->rz_ncol;
    z.ramp = z.zc + h->L.nz;
    z.lsval = z.ramp + 1;
    z.phimean = h->rz_phimean;
    return z;
}

// A stage; a convection stage is followed by the relaxation zones
// (src/levelset_RK3.cpp:125,142,158) and the solid forcing of its output
// (:128,145,160) when enabled.
long long stage_launch(r3d_handle* h, bool reini, int s, bool vol) {
    long long n = stage_launch_plain(h, reini, s, vol);
    if (reini) return n;
    void* out = h->field[s == 1 ? R3D_WORK1 : s == 2 ? R3D_WORK2 : R3D_PHI];
    if (h->relax) n += launch_relax(h->L, out, fp32(h), relax_zones(h), h->stream);
    if (h->sf_ops) n += launch_solid_forcing(out, fp32(h), h->sf_ops, h->sf_levels, h->stream);
    return n;
}

long long volume_block_count(const r3d_handle* h) {
    if (tiled(h)) {
        // the step's last stage writes the partials: reinitialisation stage
        // 3, or convection stage 3 without reinitialisation
        const bool r = h->desc.f44 > 0;
        const dim3 g = tile_grid(h->L, r ? h->kc_r : h->kc, r ? h->tile_cfg_r : h->tile_cfg);
        return (long long)g.x * g.y * g.z;
    }
    return volume_blocks(h->L);
}

int check_field(r3d_handle* h, int field) {
    if (field < 0 || field > R3D_BODY) return fail(h, R3D_EINVAL, "bad field id");
    if (!h->field[field])
        return fail(h, R3D_ESTATE, field == R3D_BODY ? "the body field exists once r3d_set_direct_forcing enabled it"
                                                     : "ro/visc exist once r3d_set_fluid enabled them");
    return R3D_OK;
}

// Airy velocity at the device clock (no-op unless r3d_set_velocity_airy).
long long refresh_velocity(r3d_handle* h) {
    if (!h->airy) return 0;
    return launch_airy(h->L, h->field[R3D_U], h->field[R3D_W], fp32(h), h->coord, h->S.t, h->ap, h->sms,
                       h->stream);
}

long long fluid_update(r3d_handle* h, bool clock) {
    return launch_fluid_update(h->L, h->field[R3D_PHI], h->field[R3D_RO], h->field[R3D_VISC], fp32(h),
                               h->g64.dxn[0], h->g64.dxn[1], h->g64.dxn[2], h->M.psi, h->fc, clock, h->period,
                               h->S, h->stream);
}

// Picard constants (src/picard_f.cpp:30, :51): epsi = F45*DXM, cell volume DXM^3.
double picard_epsi(const r3d_handle* h) { return h->desc.f45 * h->M.dxm_mean; }
double picard_cellvol(const r3d_handle* h) { return std::pow(h->M.dxm_mean, 3.0); }

long long picard_volcalc(r3d_handle* h) {
    return launch_picard_volcalc(h->L, h->field[R3D_PHI], fp32(h), picard_epsi(h), picard_cellvol(h),
                                 h->desc.f46 == 3, h->S, h->stream);
}

long long picard_correct(r3d_handle* h) {
    return launch_picard_correct(h->L, h->field[R3D_PHI], fp32(h), picard_epsi(h), picard_cellvol(h),
                                 h->desc.f47, h->desc.f46 == 3, h->S, h->stream);
}

// reini_RK3::start (src/reini_RK3.cpp:84-160): iters pseudo-steps of three
// stages, inside picard volcalc/correct_ls when f46 == 1 (:92, :140).
// fuse_volume: the last stage also writes the volume partials.
// ioflow_f hooks (no-op for the closed box): step = fsfinflow + fsfrkin/out
// at the start of levelset_RK3::start, else fsfrkin/out alone as at the
// start of reini_RK3::start.
long long io_hooks(r3d_handle* h, bool step) {
    if (!h->io) return 0;
    return launch_io_hooks(h->L, h->field[R3D_PHI], h->field[R3D_WORK1], h->field[R3D_WORK2], fp32(h), h->iop,
                           step, h->stream);
}

long long enqueue_reinit(r3d_handle* h, int iters, bool fuse_volume) {
    long long n = 0;
    if (h->desc.f46 == 1) n += picard_volcalc(h);
    n += io_hooks(h, false);
    for (int q = 0; q < iters; ++q)
        for (int s = 1; s <= 3; ++s) n += stage_launch(h, true, s, fuse_volume && q == iters - 1 && s == 3);
    if (h->desc.f46 == 1) n += picard_correct(h);
    return n;
}

// levelset_RK3::start (src/levelset_RK3.cpp:103-174).  Without picard or
// fluid update the volume partials come from the last stage; with picard
// (f46 = 1, 2 or 3) the volume pass follows the correction, and with the
// fluid update enabled that pass is fluid_update_fsf::start (:174), which
// also writes ro and visc.  f46 = 2 (picard_f) and 3 (picard_lsm) wrap the
// step (:84-91, :110, :171).
int enqueue_step(r3d_handle* h) {
    const int f44 = h->desc.f44;
    const bool pic = h->desc.f46 != 0 || h->fluid;
    long long n = 0;
    const bool step_picard = h->desc.f46 >= 2;
    n += io_hooks(h, true);
    if (step_picard) n += picard_volcalc(h);
    for (int s = 1; s <= 3; ++s) n += stage_launch(h, false, s, !pic && f44 == 0 && s == 3);
    n += enqueue_reinit(h, f44, !pic);
    if (h->desc.f46 == 3 && h->io) n += launch_netvol(h->S, h->iod.qi, h->iod.qo, h->stream);
    if (step_picard) n += picard_correct(h);
    if (h->fluid)
        n += fluid_update(h, true);
    else if (pic)
        n += launch_volume_direct_clock(h->L, h->field[R3D_PHI], fp32(h), h->g64.dxn[0], h->g64.dxn[1],
                                        h->g64.dxn[2], h->M.psi, h->period, h->S, h->stream);
    else
        n += launch_volume_reduce(h->L, h->S, volume_block_count(h), h->period, h->stream);
    h->launches += n;
    h->have_last_volume = true;
    return R3D_OK;
}

// Reads and clears the device error flag raised by a bounded wait.
int check_device_flag(r3d_handle* h) {
    int flag = 0;
    if (cudaMemcpy(&flag, h->S.err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaError_t e = cudaGetLastError();
        return cuda_fail(h, e, "reading the device error flag");
    }
    if (flag) {
        cudaMemset(h->S.err, 0, sizeof(int));
        return fail(h, R3D_ETIMEOUT, "a device wait gave up (TMA copy did not complete)");
    }
    return R3D_OK;
}

}  // namespace

namespace r3d {
// Error text of calls that have no handle (returned by r3d_last_error(NULL)).
void set_thread_error(const char* msg) { g_thread_err = msg ? msg : ""; }
}  // namespace r3d

extern "C" {

const char* r3d_last_error(const r3d_handle* h) { return h ? h->err.c_str() : g_thread_err.c_str(); }

int r3d_footprint(const r3d_grid_desc* desc, size_t* bytes) {
    std::string why;
    if (int rc = check_desc(desc, why)) return fail(nullptr, rc, why);
    if (!bytes) return fail(nullptr, R3D_EINVAL, "null output");
    *bytes = footprint(desc, make_layout(desc->nx, desc->ny, desc->nz));
    return R3D_OK;
}

int r3d_create(const r3d_grid_desc* desc, r3d_handle** out) {
    std::string why;
    if (!out) return fail(nullptr, R3D_EINVAL, "null output handle");
    *out = nullptr;
    if (int rc = check_desc(desc, why)) return fail(nullptr, rc, why);
    r3d_handle* h = new (std::nothrow) r3d_handle();
    if (!h) return fail(nullptr, R3D_ENOMEM, "host allocation failed");
    h->desc = *desc;
    h->desc.xn = h->desc.yn = h->desc.zn = nullptr;
    cudaGetDevice(&h->device);
    h->L = make_layout(desc->nx, desc->ny, desc->nz);
    build_metrics(desc->nx, desc->ny, desc->nz, desc->xn, desc->yn, desc->zn, desc->f45, h->M);

    auto bail = [&](int code, const std::string& m) {
        g_thread_err = m;
        release(h);
        delete h;
        return code;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return bail(R3D_EDEVICE, "stream creation failed (no usable CUDA device?)");
    }
    const size_t fbytes = (size_t)h->L.ncell * elem(h);
    for (int id = 0; id < 7; ++id) {
        if (cudaMalloc(&h->field[id], fbytes) != cudaSuccess) {
            cudaGetLastError();
            return bail(R3D_ENOMEM, "device field allocation failed");
        }
        cudaMemsetAsync(h->field[id], 0, fbytes, h->stream);
    }
    const size_t mc = metric_count(h);
    if (cudaMalloc(&h->metrics64, mc * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->metrics32, mc * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return bail(R3D_ENOMEM, "metric allocation failed");
    }
    std::vector<double> m64;
    std::vector<float> m32;
    fill_kgrid<double>(h, h->g64, h->metrics64, m64);
    fill_kgrid<float>(h, h->g32, h->metrics32, m32);
    for (int a = 0; a < 3; ++a) h->g64.dxn_d[a] = h->g32.dxn_d[a] = h->g64.dxn[a];
    cudaMemcpy(h->metrics64, m64.data(), m64.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(h->metrics32, m32.data(), m32.size() * sizeof(float), cudaMemcpyHostToDevice);

    const long long nb = volume_blocks(h->L);
    const long long np = (nb > (long long)h->L.ny * h->L.nz ? nb : (long long)h->L.ny * h->L.nz) + 64;
    if (cudaMalloc(&h->S.partial, (size_t)np * 2 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->S.vmax, 256) != cudaSuccess) {
        cudaGetLastError();
        return bail(R3D_ENOMEM, "scratch allocation failed");
    }
    h->S.npartial = np;
    h->S.dt = reinterpret_cast<double*>(reinterpret_cast<char*>(h->S.vmax) + 64);
    h->S.vol = reinterpret_cast<double*>(reinterpret_cast<char*>(h->S.vmax) + 128);
    h->S.t = reinterpret_cast<double*>(reinterpret_cast<char*>(h->S.vmax) + 160);
    h->S.vscale = reinterpret_cast<double*>(reinterpret_cast<char*>(h->S.vmax) + 168);
    h->S.pic = reinterpret_cast<double*>(reinterpret_cast<char*>(h->S.vmax) + 208);
    h->S.err = reinterpret_cast<int*>(reinterpret_cast<char*>(h->S.vmax) + 192);
    cudaMemsetAsync(h->S.vmax, 0, 256, h->stream);
    launch_set_scalar(h->S.vscale, 1.0, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return bail(R3D_EDEVICE, std::string("initialisation: ") + cudaGetErrorString(e));
    // the tiled kernels index a field with 32-bit offsets
    if (fp32(h) && !h->L.two_d && h->M.uniform && h->L.ncell < (1ll << 31)) {
        std::string why;
        const int ids[3] = {R3D_PHI, R3D_WORK1, R3D_WORK2};
        bool ok = true;
        for (int q = 0; q < 3 && ok; ++q)
            ok = encode_plane_map(h->L, static_cast<const float*>(h->field[ids[q]]), h->tile_cfg, &h->map[q], &why) == 0 &&
                 encode_plane_map(h->L, static_cast<const float*>(h->field[ids[q]]), h->tile_cfg_r, &h->map_r[q], &why) == 0;
        h->tile_ok = ok && tile_prepare();
    }
    *out = h;
    return R3D_OK;
}

int r3d_destroy(r3d_handle* h) {
    if (!h) return R3D_OK;
    release(h);
    delete h;
    return R3D_OK;
}

int r3d_upload(r3d_handle* h, int field, const double* host, int layout) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (int rc = check_field(h, field)) return rc;
    if (layout != R3D_LAYOUT_REEF3D && layout != R3D_LAYOUT_DENSE) return fail(h, R3D_EINVAL, "bad layout");
    if (!host) return fail(h, R3D_EINVAL, "null host pointer");
    DeviceGuard dg(h->device, h->batch_stream);
    if (int rc = ensure_staging(h)) return rc;
    const size_t n = host_count(h, layout);
    R3D_CUDA(h, cudaMemcpyAsync(h->staging, host, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    h->launches += launch_import(h->L, h->staging, layout, h->field[field], field_fp32(h, field), h->stream);
    R3D_CUDA(h, cudaGetLastError());
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    return R3D_OK;
}

int r3d_download(r3d_handle* h, int field, double* host, int layout) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (int rc = check_field(h, field)) return rc;
    if (layout != R3D_LAYOUT_REEF3D && layout != R3D_LAYOUT_DENSE) return fail(h, R3D_EINVAL, "bad layout");
    if (!host) return fail(h, R3D_EINVAL, "null host pointer");
    DeviceGuard dg(h->device, h->batch_stream);
    if (int rc = ensure_staging(h)) return rc;
    const size_t n = host_count(h, layout);
    if (layout == R3D_LAYOUT_REEF3D) R3D_CUDA(h, cudaMemsetAsync(h->staging, 0, n * sizeof(double), h->stream));
    h->launches += launch_export(h->L, h->field[field], field_fp32(h, field), layout, h->staging, h->stream);
    R3D_CUDA(h, cudaGetLastError());
    R3D_CUDA(h, cudaMemcpyAsync(host, h->staging, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    return check_device_flag(h);
}

int r3d_set_dt(r3d_handle* h, double dt) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(h, R3D_EINVAL, "dt must be positive and finite");
    DeviceGuard dg(h->device, h->batch_stream);
    h->dt_host = dt;
    h->launches += launch_set_scalar(h->S.dt, dt, h->stream);
    R3D_CUDA(h, cudaGetLastError());
    return R3D_OK;
}

int r3d_cfl_dt(r3d_handle* h, double* dt) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    DeviceGuard dg(h->device, h->batch_stream);
    h->launches += refresh_velocity(h);
    h->launches += launch_cfl(h->L, h->field[R3D_U], h->field[R3D_V], h->field[R3D_W], fp32(h), h->M.dxmin_cfl,
                              h->desc.n47, h->S, h->stream);
    R3D_CUDA(h, cudaGetLastError());
    double v = 0.0;
    R3D_CUDA(h, cudaMemcpyAsync(&v, h->S.dt, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    h->dt_host = v;
    if (dt) *dt = v;
    return R3D_OK;
}

int r3d_ls_step(r3d_handle* h, double dt) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    DeviceGuard dg(h->device, h->batch_stream);
    if (dt > 0.0) {
        if (int rc = r3d_set_dt(h, dt)) return rc;
    } else if (!(h->dt_host > 0.0)) {
        return fail(h, R3D_ESTATE, "no time step set (pass dt > 0, r3d_set_dt or r3d_cfl_dt first)");
    }
    h->launches += refresh_velocity(h);
    enqueue_step(h);
    h->wait_test = 0;  // a timeout-path test covers one step
    R3D_CUDA(h, cudaGetLastError());
    return R3D_OK;
}

// The launches of one step of r3d_ls_run (CFL first when adaptive).
void enqueue_run_step(r3d_handle* h, int adaptive) {
    h->launches += refresh_velocity(h);
    if (adaptive)
        h->launches += launch_cfl(h->L, h->field[R3D_U], h->field[R3D_V], h->field[R3D_W], fp32(h), h->M.dxmin_cfl,
                                  h->desc.n47, h->S, h->stream);
    enqueue_step(h);
}

long long run_graph_key(const r3d_handle* h, int adaptive) {
    long long k = adaptive ? 1 : 0;
    k = k * 2 + (tiled(h) ? 1 : 0);
    k = k * 2 + (h->band64 ? 1 : 0);
    k = k * 8192 + h->kc;
    k = k * 8192 + h->kc_r;
    return k;
}

void drop_step_graph(r3d_handle* h) {
    if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
    h->step_graph = nullptr;
    h->graph_key = -1;
    ++h->config_gen;
}

// Captures one step into a CUDA graph (the step reads dt, the clock and the
// velocity factor from device memory, so the same graph serves every step).
int capture_step(r3d_handle* h, int adaptive) {
    drop_step_graph(h);
    cudaGraph_t g = nullptr;
    R3D_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const long long before = h->launches;
    enqueue_run_step(h, adaptive);
    h->graph_launches = h->launches - before;
    h->launches = before;
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (e != cudaSuccess) return cuda_fail(h, e, "step graph capture");
    e = cudaGraphInstantiate(&h->step_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        h->step_graph = nullptr;
        return cuda_fail(h, e, "step graph instantiate");
    }
    h->graph_key = run_graph_key(h, adaptive);
    return R3D_OK;
}

int r3d_ls_run(r3d_handle* h, int nsteps, int adaptive) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (nsteps < 0) return fail(h, R3D_EINVAL, "nsteps must be >= 0");
    DeviceGuard dg(h->device, h->batch_stream);
    if (!adaptive && !(h->dt_host > 0.0)) return fail(h, R3D_ESTATE, "no time step set");
    const bool use_graph = nsteps >= 2 || (h->step_graph && h->graph_key == run_graph_key(h, adaptive));
    if (use_graph && !(h->step_graph && h->graph_key == run_graph_key(h, adaptive)))
        if (int rc = capture_step(h, adaptive)) return rc;
    for (int n = 0; n < nsteps; ++n) {
        if (use_graph) {
            R3D_CUDA(h, cudaGraphLaunch(h->step_graph, h->stream));
            h->launches += h->graph_launches;
            h->have_last_volume = true;
        } else {
            enqueue_run_step(h, adaptive);
        }
    }
    R3D_CUDA(h, cudaGetLastError());
    return R3D_OK;
}

int r3d_reinit(r3d_handle* h, int iters) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    DeviceGuard dg(h->device, h->batch_stream);
    const int it = iters > 0 ? iters : h->desc.f44;
    h->launches += enqueue_reinit(h, it, false);
    R3D_CUDA(h, cudaGetLastError());
    return R3D_OK;
}

int r3d_convection_L(r3d_handle* h, int field_in) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (field_in != R3D_PHI && field_in != R3D_WORK1 && field_in != R3D_WORK2)
        return fail(h, R3D_EINVAL, "convection input must be a level-set field");
    DeviceGuard dg(h->device, h->batch_stream);
    const Fields f = fields_of(h);
    h->launches += fp32(h) ? launch_conv_L_f32(h->g32, h->field[field_in], f, h->S, h->stream)
                           : launch_conv_L_f64(h->g64, h->field[field_in], f, h->S, h->stream);
    R3D_CUDA(h, cudaGetLastError());
    return R3D_OK;
}

int r3d_reinidisc_L(r3d_handle* h, int field_in) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (field_in != R3D_PHI && field_in != R3D_WORK1 && field_in != R3D_WORK2)
        return fail(h, R3D_EINVAL, "reinitialisation input must be a level-set field");
    DeviceGuard dg(h->device, h->batch_stream);
    const Fields f = fields_of(h);
    h->launches += fp32(h) ? launch_reini_L_f32(h->g32, h->field[field_in], f, h->stream)
                           : launch_reini_L_f64(h->g64, h->field[field_in], f, h->stream);
    R3D_CUDA(h, cudaGetLastError());
    return R3D_OK;
}

int r3d_ghost_fill(r3d_handle* h, int field) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (int rc = check_field(h, field)) return rc;
    DeviceGuard dg(h->device, h->batch_stream);
    h->launches += launch_ghost_fill(h->L, h->field[field], fp32(h), h->stream);
    R3D_CUDA(h, cudaGetLastError());
    return R3D_OK;
}

int r3d_write_vtu(r3d_handle* h, const char* path) {
    if (!h || !path) return fail(h, R3D_EINVAL, "null argument");
    DeviceGuard dg(h->device, h->batch_stream);
    const Layout& L = h->L;
    const long long nyp = L.two_d ? 2 : L.ny + 1;
    const long long np = (long long)(L.nx + 1) * nyp * (L.nz + 1);
    const long long nc = (long long)L.nx * L.ny * L.nz;
    if (32 * nc > 0xffffffffLL || 12 * np > 0xffffffffLL)
        return fail(h, R3D_EINVAL, "grid too large for a VTU file with 32-bit block sizes");
    const int nf = h->fluid ? 3 : 1;
    float* dev = nullptr;
    if (cudaMalloc(&dev, (size_t)nf * np * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return fail(h, R3D_ENOMEM, "VTU point data buffer");
    }
    h->launches += launch_vtu_nodes(L, h->field[R3D_PHI], h->fluid ? h->field[R3D_RO] : nullptr,
                                    h->fluid ? h->field[R3D_VISC] : nullptr, fp32(h), dev, np, h->stream);
    std::vector<float> pd((size_t)nf * np);
    double t = 0.0;
    cudaMemcpyAsync(pd.data(), dev, pd.size() * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(&t, h->S.t, sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    cudaFree(dev);
    if (e != cudaSuccess) return cuda_fail(h, e, "VTU point data");

    // The reference's printer layout (src/printer_CFD.cpp:356-600,
    // src/vtu3D.cpp:63-101,125-225): point data at the TPLOOP nodes, then the
    // node coordinates, hexahedral cells in k, j, i order with the node
    // numbering of initialize::nodecalc (src/initialize.cpp:118-131),
    // appended raw blocks each preceded by its byte count.
    const char* names[3] = {"phi", "rho", "viscosity"};
    std::ostringstream x;
    long long off = 0;
    x << "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\">\n"
      << "<UnstructuredGrid>\n<FieldData>\n<DataArray type=\"Float64\" Name=\"TimeValue\" NumberOfTuples=\"1\"> "
      << t << "\n</DataArray>\n</FieldData>\n<Piece NumberOfPoints=\"" << np << "\" NumberOfCells=\"" << nc
      << "\">\n<PointData>\n";
    for (int q = 0; q < nf; ++q) {
        x << "<DataArray type=\"Float32\" Name=\"" << names[q] << "\" format=\"appended\" offset=\"" << off
          << "\"/>\n";
        off += 4 + 4 * np;
    }
    x << "</PointData>\n<CellData>\n</CellData>\n<Points>\n<DataArray type=\"Float32\" NumberOfComponents=\"3\" "
      << "format=\"appended\" offset=\"" << off << "\"/>\n</Points>\n<Cells>\n";
    off += 4 + 12 * np;
    x << "<DataArray type=\"Int32\" Name=\"connectivity\" format=\"appended\" offset=\"" << off << "\"/>\n";
    off += 4 + 32 * nc;
    x << "<DataArray type=\"Int32\" Name=\"offsets\" format=\"appended\" offset=\"" << off << "\"/>\n";
    off += 4 + 4 * nc;
    x << "<DataArray type=\"Int32\" Name=\"types\" format=\"appended\" offset=\"" << off << "\"/>\n"
      << "</Cells>\n</Piece>\n</UnstructuredGrid>\n<AppendedData encoding=\"raw\">\n_";

    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(h, R3D_EINVAL, std::string("cannot open ") + path);
    const std::string head = x.str();
    bool ok = std::fwrite(head.data(), 1, head.size(), fp) == head.size();
    auto block = [&](const void* data, long long bytes) {
        const unsigned n = (unsigned)bytes;
        ok = ok && std::fwrite(&n, sizeof n, 1, fp) == 1;
        ok = ok && (bytes == 0 || std::fwrite(data, 1, (size_t)bytes, fp) == (size_t)bytes);
    };
    for (int q = 0; q < nf; ++q) block(pd.data() + (size_t)q * np, 4 * np);
    {
        std::vector<float> xyz((size_t)3 * np);
        size_t m = 0;
        for (long long k = -1; k < L.nz; ++k)
            for (long long j = -1; j < nyp - 1; ++j)
                for (long long i = -1; i < L.nx; ++i) {
                    xyz[m++] = (float)h->M.xn[0][i + 6];
                    xyz[m++] = (float)h->M.xn[1][j + 6];
                    xyz[m++] = (float)h->M.xn[2][k + 6];
                }
        block(xyz.data(), 12 * np);
    }
    {
        std::vector<int> con((size_t)8 * nc);
        const long long sx = L.nx + 1, sy = sx * nyp;
        auto id = [&](long long i, long long j, long long k) { return (int)((k + 1) * sy + (j + 1) * sx + (i + 1)); };
        size_t m = 0;
        for (long long k = 0; k < L.nz; ++k)
            for (long long j = 0; j < L.ny; ++j)
                for (long long i = 0; i < L.nx; ++i) {
                    con[m++] = id(i - 1, j - 1, k - 1);
                    con[m++] = id(i, j - 1, k - 1);
                    con[m++] = id(i, j, k - 1);
                    con[m++] = id(i - 1, j, k - 1);
                    con[m++] = id(i - 1, j - 1, k);
                    con[m++] = id(i, j - 1, k);
                    con[m++] = id(i, j, k);
                    con[m++] = id(i - 1, j, k);
                }
        block(con.data(), 32 * nc);
        for (long long c = 0; c < nc; ++c) con[(size_t)c] = (int)((c + 1) * 8);
        block(con.data(), 4 * nc);
        for (long long c = 0; c < nc; ++c) con[(size_t)c] = 12;  // VTK_HEXAHEDRON
        block(con.data(), 4 * nc);
    }
    const char tail[] = "\n</AppendedData>\n</VTKFile>";
    ok = ok && std::fwrite(tail, 1, sizeof tail - 1, fp) == sizeof tail - 1;
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return fail(h, R3D_EINVAL, std::string("writing ") + path + " failed");
    return R3D_OK;
}

// ---------------------------------------------------------- checkpoint
namespace {
constexpr char kStateMagic[8] = {'R', '3', 'D', 'S', 'T', 'A', 'T', 'E'};
constexpr unsigned kStateVersion = 1;

// FNV-1a over the node coordinates: a state loads only into the grid it
// was written from.
unsigned long long grid_hash(const r3d_handle* h) {
    unsigned long long x = 1469598103934665603ULL;
    for (int a = 0; a < 3; ++a)
        for (int t = 0; t < h->M.n[a] + 11; ++t) {
            unsigned long long b;
            std::memcpy(&b, &h->M.xn[a][t], sizeof b);
            for (int q = 0; q < 8; ++q) {
                x ^= (b >> (8 * q)) & 0xffULL;
                x *= 1099511628211ULL;
            }
        }
    return x;
}

struct StateHead {
    char magic[8];
    unsigned version;
    int nx, ny, nz, precision;
    int fluid, x45, io;
    unsigned long long grid;
    double scalars[32];  // dt, t, vscale, picard (4), hook state (8), volumes (2)
};
}  // namespace

int r3d_save_state(r3d_handle* h, const char* path) {
    if (!h || !path) return fail(h, R3D_EINVAL, "null argument");
    DeviceGuard dg(h->device, h->batch_stream);
    StateHead hd{};
    std::memcpy(hd.magic, kStateMagic, 8);
    hd.version = kStateVersion;
    hd.nx = h->L.nx;
    hd.ny = h->L.ny;
    hd.nz = h->L.nz;
    hd.precision = h->desc.precision;
    hd.fluid = h->fluid ? 1 : 0;
    hd.x45 = h->g64.x45;
    hd.io = h->io ? 1 : 0;
    hd.grid = grid_hash(h);
    double* sc = hd.scalars;
    cudaMemcpyAsync(sc + 0, h->S.dt, sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(sc + 1, h->S.t, sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(sc + 2, h->S.vscale, sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(sc + 3, h->S.pic, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (h->io) cudaMemcpyAsync(sc + 7, h->io_buf, kIoStateLen * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(sc + 15, h->S.vol, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    std::vector<char> buf((size_t)h->L.ncell * sizeof(double));
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(h, R3D_EINVAL, std::string("cannot open ") + path);
    bool ok = true;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    ok = e == cudaSuccess && std::fwrite(&hd, sizeof hd, 1, fp) == 1;
    for (int id = 0; id <= R3D_BODY && ok; ++id) {
        if (!h->field[id] || id == R3D_L) continue;
        const size_t bytes = (size_t)h->L.ncell * field_elem(h, id);
        e = cudaMemcpy(buf.data(), h->field[id], bytes, cudaMemcpyDeviceToHost);
        ok = e == cudaSuccess && std::fwrite(&id, sizeof id, 1, fp) == 1 && std::fwrite(buf.data(), 1, bytes, fp) == bytes;
    }
    ok = (std::fclose(fp) == 0) && ok;
    if (e != cudaSuccess) return cuda_fail(h, e, "reading the state");
    if (!ok) return fail(h, R3D_EINVAL, std::string("writing ") + path + " failed");
    return R3D_OK;
}

int r3d_load_state(r3d_handle* h, const char* path) {
    if (!h || !path) return fail(h, R3D_EINVAL, "null argument");
    DeviceGuard dg(h->device, h->batch_stream);
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return fail(h, R3D_EINVAL, std::string("cannot open ") + path);
    StateHead hd{};
    const bool got = std::fread(&hd, sizeof hd, 1, fp) == 1;
    auto bad = [&](const char* why) {
        std::fclose(fp);
        return fail(h, R3D_EINVAL, std::string(path) + ": " + why);
    };
    if (!got || std::memcmp(hd.magic, kStateMagic, 8) != 0 || hd.version != kStateVersion)
        return bad("not a state file of this version");
    if (hd.nx != h->L.nx || hd.ny != h->L.ny || hd.nz != h->L.nz || hd.precision != h->desc.precision ||
        hd.grid != grid_hash(h))
        return bad("written from another grid or precision");
    if (hd.fluid != (h->fluid ? 1 : 0) || hd.x45 != h->g64.x45 || hd.io != (h->io ? 1 : 0))
        return bad("written with another fluid / direct-forcing / inflow-outflow configuration");
    std::vector<char> buf((size_t)h->L.ncell * sizeof(double));
    int id = -1;
    while (std::fread(&id, sizeof id, 1, fp) == 1) {
        if (id < 0 || id > R3D_BODY || !h->field[id]) return bad("unexpected field");
        const size_t bytes = (size_t)h->L.ncell * field_elem(h, id);
        if (std::fread(buf.data(), 1, bytes, fp) != bytes) return bad("truncated");
        R3D_CUDA(h, cudaMemcpy(h->field[id], buf.data(), bytes, cudaMemcpyHostToDevice));
    }
    std::fclose(fp);
    const double* sc = hd.scalars;
    R3D_CUDA(h, cudaMemcpy(h->S.dt, sc + 0, sizeof(double), cudaMemcpyHostToDevice));
    R3D_CUDA(h, cudaMemcpy(h->S.t, sc + 1, sizeof(double), cudaMemcpyHostToDevice));
    R3D_CUDA(h, cudaMemcpy(h->S.vscale, sc + 2, sizeof(double), cudaMemcpyHostToDevice));
    R3D_CUDA(h, cudaMemcpy(h->S.pic, sc + 3, 4 * sizeof(double), cudaMemcpyHostToDevice));
    if (h->io) R3D_CUDA(h, cudaMemcpy(h->io_buf, sc + 7, kIoStateLen * sizeof(double), cudaMemcpyHostToDevice));
    R3D_CUDA(h, cudaMemcpy(h->S.vol, sc + 15, 2 * sizeof(double), cudaMemcpyHostToDevice));
    h->dt_host = sc[0];
    return R3D_OK;
}

int r3d_volume(r3d_handle* h, double* volume1, double* volume2) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    DeviceGuard dg(h->device, h->batch_stream);
    const double* dxn = h->g64.dxn[0];
    const double* dyn = h->g64.dxn[1];
    const double* dzn = h->g64.dxn[2];
    h->launches += launch_volume_direct(h->L, h->field[R3D_PHI], fp32(h), dxn, dyn, dzn, h->M.psi, h->S, h->stream);
    R3D_CUDA(h, cudaGetLastError());
    double v[2] = {0.0, 0.0};
    R3D_CUDA(h, cudaMemcpyAsync(v, h->S.vol, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    if (volume1) *volume1 = v[0];
    if (volume2) *volume2 = v[1];
    return R3D_OK;
}

int r3d_set_fluid(r3d_handle* h, double ro_water, double visc_water, double ro_air, double visc_air) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (h->batch_stream) return fail(h, R3D_ESTATE, "the instance is a batch member");
    DeviceGuard dg(h->device, h->batch_stream);
    if (!h->fluid) {
        const size_t fbytes = (size_t)h->L.ncell * elem(h);
        for (int id : {R3D_RO, R3D_VISC}) {
            if (cudaMalloc(&h->field[id], fbytes) != cudaSuccess) {
                cudaGetLastError();
                return fail(h, R3D_ENOMEM, "ro/visc allocation failed");
            }
            R3D_CUDA(h, cudaMemsetAsync(h->field[id], 0, fbytes, h->stream));
        }
    }
    h->fc = r3d::FluidConst{ro_water, visc_water, ro_air, visc_air};
    h->fluid = true;
    drop_step_graph(h);
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    return R3D_OK;
}

int r3d_fluid_update(r3d_handle* h, double* volume1, double* volume2) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (!h->fluid) return fail(h, R3D_ESTATE, "r3d_set_fluid has not enabled the fluid update");
    DeviceGuard dg(h->device, h->batch_stream);
    h->launches += fluid_update(h, false);
    R3D_CUDA(h, cudaGetLastError());
    double v[2] = {0.0, 0.0};
    R3D_CUDA(h, cudaMemcpyAsync(v, h->S.vol, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    if (volume1) *volume1 = v[0];
    if (volume2) *volume2 = v[1];
    return R3D_OK;
}

int r3d_last_volume(r3d_handle* h, double* volume1, double* volume2) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (!h->have_last_volume) return fail(h, R3D_ESTATE, "no step has run yet");
    DeviceGuard dg(h->device, h->batch_stream);
    double v[2] = {0.0, 0.0};
    R3D_CUDA(h, cudaMemcpyAsync(v, h->S.vol, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    if (volume1) *volume1 = v[0];
    if (volume2) *volume2 = v[1];
    return R3D_OK;
}

int r3d_set_velocity_scale(r3d_handle* h, double scale) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (!std::isfinite(scale)) return fail(h, R3D_EINVAL, "velocity scale must be finite");
    DeviceGuard dg(h->device, h->batch_stream);
    h->launches += launch_set_scalar(h->S.vscale, scale, h->stream);
    R3D_CUDA(h, cudaGetLastError());
    return R3D_OK;
}

namespace {
void set_layout_io(r3d_handle* h, int mask) {
    h->L.io = mask;
    h->g64.L.io = mask;
    h->g32.L.io = mask;
}
}  // namespace

int r3d_set_ioflow(r3d_handle* h, const r3d_ioflow_desc* io) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (h->batch_stream) return fail(h, R3D_ESTATE, "the instance is a batch member");
    DeviceGuard dg(h->device, h->batch_stream);
    if (!io) {
        drop_step_graph(h);
        h->io = false;
        set_layout_io(h, h->L.io & (kHaloZLo | kHaloZHi));
        return R3D_OK;
    }
    if ((io->inflow != 0 && io->inflow != 1) || (io->outflow != 0 && io->outflow != 1))
        return fail(h, R3D_EINVAL, "inflow and outflow must be 0 or 1");
    if (io->f50 < 1 || io->f50 > 4) return fail(h, R3D_EINVAL, "f50 must be 1..4");
    if (io->b77 != 1 && io->b77 != 2) return fail(h, R3D_EINVAL, "b77 must be 1 or 2");
    if (io->f64 < 0 || io->f64 > (1 << 24)) return fail(h, R3D_EINVAL, "f64 must be 0..2^24");
    if ((h->L.io & (kHaloZLo | kHaloZHi)) && !h->domain_slab)
        return fail(h, R3D_EINVAL, "subdomain instances have no inflow/outflow faces");
    drop_step_graph(h);
    // state, ZP (index k + 5), ramp table of the outflow level (F64 > 0)
    const std::vector<double>& zp = h->M.xp[2];
    const size_t ramp_at = kIoStateLen + zp.size();
    const size_t len = ramp_at + (size_t)std::max(io->f64, 1);
    std::vector<double> host(len, 0.0);
    if (h->io_buf) {  // keep the step count and levels of an earlier configuration
        R3D_CUDA(h, cudaMemcpyAsync(host.data(), h->io_buf, kIoStateLen * sizeof(double), cudaMemcpyDeviceToHost,
                                    h->stream));
        R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    } else {
        host[kIoCount] = (double)(h->next_count - 1);
    }
    for (size_t t = 0; t < zp.size(); ++t) host[kIoStateLen + t] = zp[t];
    const double PI_REF = 3.14159265359;  // src/definitions.h:37
    for (int c = 0; c < io->f64; ++c)  // src/ioflow_waterlevel.cpp:110-111
        host[ramp_at + c] = 0.5 * std::cos(PI_REF + PI_REF * double(c) / double(io->f64)) + 0.5;
    if (len > h->io_buf_len) {
        if (h->io_buf) cudaFree(h->io_buf);
        h->io_buf = nullptr;
        h->io_buf_len = 0;
        if (cudaMalloc(&h->io_buf, len * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            h->io = false;
            set_layout_io(h, h->L.io & (kHaloZLo | kHaloZHi));
            return fail(h, R3D_ENOMEM, "ioflow state allocation failed");
        }
        h->io_buf_len = len;
    }
    R3D_CUDA(h, cudaMemcpyAsync(h->io_buf, host.data(), len * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    h->iod = *io;
    h->io = true;
    IoParams p{};
    p.inflow = io->inflow;
    p.outflow = io->outflow;
    p.f50 = io->f50;
    p.b77 = io->b77;
    p.f64 = io->f64;
    p.f56 = io->f56;
    p.f60 = io->f60;
    p.f62 = io->f62;
    p.zp = h->io_buf + kIoStateLen;
    p.dzp = h->g64.dxp[2];
    p.ramp = h->io_buf + ramp_at;
    p.state = h->io_buf;
    h->iop = p;
    // ghost labels of gcval 50+f50 on the two x faces (src/gc_epol4.cpp:26-58)
    const int gcv = 50 + io->f50;
    int mask = 0;
    if (io->inflow && !(gcv == 52 || gcv == 54)) mask |= kIoSkipLo;
    if (io->outflow && !(gcv == 51 || gcv == 54 || (gcv == 52 && io->b77 == 1))) mask |= kIoSkipHi;
    if (io->inflow) mask |= kIoEdge;
    set_layout_io(h, mask | (h->L.io & (kHaloZLo | kHaloZHi)));
    return R3D_OK;
}

int r3d_set_ioflow_waves(r3d_handle* h, const r3d_ioflow_desc* io) {
    if (int rc = r3d_set_ioflow(h, io)) return rc;
    if (io) h->iop.waves = 1;
    return R3D_OK;
}

// ------------------------------------------------ grid spacing constants
int r3d_grid_spacing(const r3d_grid_desc* desc, double* out) {
    std::string why;
    if (int rc = check_desc(desc, why)) return fail(nullptr, rc, why);
    if (!out) return fail(nullptr, R3D_EINVAL, "null output");
    HostMetrics m;
    build_metrics(desc->nx, desc->ny, desc->nz, desc->xn, desc->yn, desc->zn, desc->f45, m);
    out[0] = m.dxm_mean;
    out[1] = m.dym;
    out[2] = m.dzm;
    out[3] = m.psi;
    return R3D_OK;
}

int r3d_set_grid_spacing(r3d_handle* h, double dxm, double dym, double dzm) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (!(dxm > 0.0) || !(dym > 0.0) || !(dzm > 0.0)) return fail(h, R3D_EINVAL, "spacings must be > 0");
    DeviceGuard dg(h->device, h->batch_stream);
    drop_step_graph(h);
    h->M.dxm_mean = dxm;
    h->M.dym = dym;
    h->M.dzm = dzm;
    // src/ini_psi.cpp:33-37, as build_metrics
    if (h->L.two_d) h->M.psi = h->desc.f45 * (1.0 / 2.0) * (dxm + dzm);
    else h->M.psi = h->desc.f45 * (1.0 / 3.0) * (dxm + dym + dzm);
    h->g64.psi = h->M.psi;
    h->g32.psi = h->M.psi;
    h->g64.df_thr = h->g32.df_thr = 0.6 * dxm;
    return R3D_OK;
}

// ------------------------------------------------ subdomain (slab) halos
int r3d_set_halo(r3d_handle* h, int zlo, int zhi) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (h->batch_stream) return fail(h, R3D_ESTATE, "the instance is a batch member");
    if ((zlo != 0 && zlo != 1) || (zhi != 0 && zhi != 1)) return fail(h, R3D_EINVAL, "zlo and zhi must be 0 or 1");
    if ((zlo || zhi) && h->desc.f46 != 0)
        return fail(h, R3D_EINVAL, "subdomain instances run without the picard correction (f46 = 0)");
    if ((zlo || zhi) && h->io) return fail(h, R3D_EINVAL, "subdomain instances have no inflow/outflow faces");
    DeviceGuard dg(h->device, h->batch_stream);
    drop_step_graph(h);
    const int mask = (h->L.io & ~(kHaloZLo | kHaloZHi)) | (zlo ? kHaloZLo : 0) | (zhi ? kHaloZHi : 0);
    set_layout_io(h, mask);
    return R3D_OK;
}

int r3d_halo_bytes(const r3d_handle* h, size_t* bytes) {
    if (!h || !bytes) return fail(nullptr, R3D_EINVAL, "null argument");
    *bytes = (size_t)3 * (size_t)h->L.sz * elem(h);
    return R3D_OK;
}

int r3d_halo_copy(r3d_handle* h, int field, int side, int dir, void* buf) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (int rc = check_field(h, field)) return rc;
    if ((side != 0 && side != 1) || (dir != 0 && dir != 1) || !buf)
        return fail(h, R3D_EINVAL, "side 0 (z-min) or 1 (z-max), dir 0 (pack) or 1 (unpack), device buffer");
    if (h->L.nz < 3) return fail(h, R3D_EINVAL, "a subdomain needs at least 3 cells in z");
    DeviceGuard dg(h->device, h->batch_stream);
    const size_t e = field_elem(h, field), plane = (size_t)h->L.sz;
    // planes k = 0..2 / nz-3..nz-1 (pack) and -3..-1 / nz..nz+2 (unpack);
    // plane k starts at (k + gz) * sz
    const long long k0 = dir == 0 ? (side == 0 ? 0 : h->L.nz - 3) : (side == 0 ? -3 : h->L.nz);
    char* f = static_cast<char*>(h->field[field]) + (size_t)(k0 + h->L.gz) * plane * e;
    if (dir == 0)
        R3D_CUDA(h, cudaMemcpyAsync(buf, f, 3 * plane * e, cudaMemcpyDeviceToDevice, h->stream));
    else
        R3D_CUDA(h, cudaMemcpyAsync(f, buf, 3 * plane * e, cudaMemcpyDeviceToDevice, h->stream));
    return R3D_OK;
}

int r3d_cfl_max(r3d_handle* h, double* vmax) {
    if (!h || !vmax) return fail(h, R3D_EINVAL, "null argument");
    DeviceGuard dg(h->device, h->batch_stream);
    h->launches += refresh_velocity(h);
    h->launches += launch_cfl(h->L, h->field[R3D_U], h->field[R3D_V], h->field[R3D_W], fp32(h), h->M.dxmin_cfl,
                              h->desc.n47, h->S, h->stream);
    unsigned long long bits[3] = {0, 0, 0};
    R3D_CUDA(h, cudaMemcpyAsync(bits, h->S.vmax, sizeof bits, cudaMemcpyDeviceToHost, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    for (int a = 0; a < 3; ++a) std::memcpy(&vmax[a], &bits[a], sizeof(double));
    return R3D_OK;
}

int r3d_cfl_dt_from_max(r3d_handle* h, const double* vmax, double* dt) {
    if (!h || !vmax) return fail(h, R3D_EINVAL, "null argument");
    for (int a = 0; a < 3; ++a)
        if (!(vmax[a] >= 0.0)) return fail(h, R3D_EINVAL, "velocity maxima must be >= 0");
    DeviceGuard dg(h->device, h->batch_stream);
    unsigned long long bits[3];
    for (int a = 0; a < 3; ++a) std::memcpy(&bits[a], &vmax[a], sizeof(double));
    R3D_CUDA(h, cudaMemcpyAsync(h->S.vmax, bits, sizeof bits, cudaMemcpyHostToDevice, h->stream));
    h->launches += launch_dt_from_max(h->M.dxmin_cfl, h->desc.n47, h->S, h->stream);
    double v = 0.0;
    R3D_CUDA(h, cudaMemcpyAsync(&v, h->S.dt, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    h->dt_host = v;
    if (dt) *dt = v;
    return R3D_OK;
}

int r3d_set_solid_forcing(r3d_handle* h, int n, const int* cells) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (h->batch_stream) return fail(h, R3D_ESTATE, "the instance is a batch member");
    if (n < 0 || (n > 0 && !cells)) return fail(h, R3D_EINVAL, "n >= 0 entries of (i, j, k, side)");
    const Layout& L = h->L;
    // device index of cell (i,j,k); ops skip sides <= 0 (GCDF4CHECK) and > 6
    auto idx = [&](long long i, long long j, long long k) { return (k + L.gz) * L.sz + (j + L.gy) * L.sy + (i + L.gx); };
    struct Op { long long c[3]; };
    std::vector<Op> ops;
    std::vector<int> level;
    std::unordered_map<long long, int> wl, rl;  // last level that wrote / read a cell
    for (int q = 0; q < n; ++q) {
        const int i = cells[4 * q], j = cells[4 * q + 1], k = cells[4 * q + 2], side = cells[4 * q + 3];
        if (side <= 0 || side > 6) continue;
        if (i < 0 || i >= L.nx || j < 0 || j >= L.ny || k < 0 || k >= L.nz)
            return fail(h, R3D_EINVAL, "solid-forcing entry outside the interior");
        if (L.two_d && (side == 2 || side == 3))
            return fail(h, R3D_EINVAL, "a 2D instance holds no y ghost planes for y sides");
        const int di = side == 1 ? -1 : side == 4 ? 1 : 0, dj = side == 3 ? -1 : side == 2 ? 1 : 0;
        const int dk = side == 5 ? -1 : side == 6 ? 1 : 0;
        Op o{{idx(i, j, k), idx(i + di, j + dj, k + dk), idx(i + 2 * di, j + 2 * dj, k + 2 * dk)}};
        // after every earlier entry that wrote a cell this one touches or read a cell it writes
        int lv = 0;
        for (int t = 0; t < 3; ++t) {
            auto w = wl.find(o.c[t]);
            if (w != wl.end()) lv = std::max(lv, w->second + 1);
            if (t > 0) {
                auto r = rl.find(o.c[t]);
                if (r != rl.end()) lv = std::max(lv, r->second + 1);
            }
        }
        rl[o.c[0]] = std::max(rl.count(o.c[0]) ? rl[o.c[0]] : 0, lv);
        for (int t = 1; t < 3; ++t) wl[o.c[t]] = std::max(wl.count(o.c[t]) ? wl[o.c[t]] : 0, lv);
        ops.push_back(o);
        level.push_back(lv);
    }
    DeviceGuard dg(h->device, h->batch_stream);
    drop_step_graph(h);
    if (h->sf_ops) cudaFree(h->sf_ops);
    h->sf_ops = nullptr;
    h->sf_levels.clear();
    if (ops.empty()) return R3D_OK;
    const int nl = *std::max_element(level.begin(), level.end()) + 1;
    std::vector<int> off(nl + 1, 0);
    for (int lv : level) ++off[lv + 1];
    for (int l = 0; l < nl; ++l) off[l + 1] += off[l];
    std::vector<long long> flat(3 * ops.size());
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (size_t q = 0; q < ops.size(); ++q) {
        const int at = fill[level[q]]++;
        for (int t = 0; t < 3; ++t) flat[3 * (size_t)at + t] = ops[q].c[t];
    }
    if (cudaMalloc(&h->sf_ops, flat.size() * sizeof(long long)) != cudaSuccess) {
        cudaGetLastError();
        h->sf_ops = nullptr;
        return fail(h, R3D_ENOMEM, "solid-forcing list allocation failed");
    }
    R3D_CUDA(h, cudaMemcpy(h->sf_ops, flat.data(), flat.size() * sizeof(long long), cudaMemcpyHostToDevice));
    h->sf_levels = off;
    return R3D_OK;
}

int r3d_set_relaxation(r3d_handle* h, const double* w_gen, const double* w_beach, double phimean) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (h->batch_stream) return fail(h, R3D_ESTATE, "the instance is a batch member");
    if (h->domain_slab) return fail(h, R3D_ESTATE, "relaxation zones are not supported on slabs of a domain");
    DeviceGuard dg(h->device, h->batch_stream);
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    drop_step_graph(h);
    if (h->rz_col) cudaFree(h->rz_col);
    if (h->rz_buf) cudaFree(h->rz_buf);
    h->rz_col = nullptr;
    h->rz_buf = nullptr;
    h->relax = false;
    h->rz_ncol = 0;
    h->rz_ntarget = 0;
    if (!w_gen && !w_beach) return R3D_OK;
    if (!std::isfinite(phimean)) return fail(h, R3D_EINVAL, "phimean must be finite");
    const int nx = h->L.nx, ny = h->L.ny, nz = h->L.nz;
    // zone columns in the reference's LOOP order (i outer, j inner), the
    // generation targets of a column at nz consecutive offsets
    std::vector<int> col;
    std::vector<double> w;
    int ngen = 0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            const double wg = w_gen ? w_gen[(size_t)i * ny + j] : -1.0;
            const double wb = w_beach ? w_beach[(size_t)i * ny + j] : -1.0;
            const bool g = wg >= 0.0, b = wb >= 0.0;
            if ((g && !(wg <= 1.0)) || (b && !(wb <= 1.0)))
                return fail(h, R3D_EINVAL, "relaxation weights must lie in [0, 1] (negative: outside the zone)");
            if (!g && !b) continue;
            col.insert(col.end(), {i, j, (g ? 1 : 0) | (b ? 2 : 0), g ? ngen * nz : 0});
            w.push_back(g ? wg : 0.0);
            w.push_back(b ? wb : 0.0);
            if (g) ++ngen;
        }
    if (col.empty()) return R3D_OK;
    const int ncol = (int)(col.size() / 4);
    const long long ntarget = (long long)ngen * nz;
    std::vector<double> buf(w);
    for (int k = 0; k < nz; ++k) buf.push_back(h->M.xp[2][k + 5]);  // cell-centre z
    buf.push_back(0.0);                                             // ramp
    buf.resize(buf.size() + (size_t)ntarget, 0.0);                  // targets
    if (cudaMalloc(&h->rz_col, col.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&h->rz_buf, buf.size() * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        if (h->rz_col) cudaFree(h->rz_col);
        h->rz_col = nullptr;
        return fail(h, R3D_ENOMEM, "relaxation zone allocation failed");
    }
    R3D_CUDA(h, cudaMemcpy(h->rz_col, col.data(), col.size() * sizeof(int), cudaMemcpyHostToDevice));
    R3D_CUDA(h, cudaMemcpy(h->rz_buf, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice));
    h->rz_ncol = ncol;
    h->rz_ntarget = ntarget;
    h->rz_phimean = phimean;
    h->relax = true;
    return R3D_OK;
}

int r3d_set_relaxation_target(r3d_handle* h, const double* lsval, long long n, double ramp) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (!h->relax) return fail(h, R3D_ESTATE, "no relaxation zones (r3d_set_relaxation)");
    if (n != h->rz_ntarget) return fail(h, R3D_EINVAL, "target count must be nz x the generation zone's columns");
    if (n > 0 && !lsval) return fail(h, R3D_EINVAL, "null targets");
    if (!std::isfinite(ramp)) return fail(h, R3D_EINVAL, "ramp must be finite");
    DeviceGuard dg(h->device, h->batch_stream);
    const RelaxZones z = relax_zones(h);
    h->launches += launch_set_scalar(const_cast<double*>(z.ramp), ramp, h->stream);
    if (n > 0)
        R3D_CUDA(h, cudaMemcpyAsync(const_cast<double*>(z.lsval), lsval, (size_t)n * sizeof(double),
                                    cudaMemcpyHostToDevice, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    return R3D_OK;
}

int r3d_set_direct_forcing(r3d_handle* h, int x45) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (h->batch_stream) return fail(h, R3D_ESTATE, "the instance is a batch member");
    if (x45 < 0 || x45 > 6) return fail(h, R3D_EINVAL, "x45 must be 0..6");
    DeviceGuard dg(h->device, h->batch_stream);
    if (x45 != 0 && !h->field[R3D_BODY]) {
        const size_t bytes = (size_t)h->L.ncell * sizeof(double);
        if (cudaMalloc(&h->field[R3D_BODY], bytes) != cudaSuccess) {
            cudaGetLastError();
            h->field[R3D_BODY] = nullptr;
            return fail(h, R3D_ENOMEM, "body field allocation failed");
        }
        R3D_CUDA(h, cudaMemsetAsync(h->field[R3D_BODY], 0, bytes, h->stream));
    }
    drop_step_graph(h);
    h->g64.x45 = h->g32.x45 = x45;
    h->g64.df_thr = h->g32.df_thr = 0.6 * h->M.dxm_mean;  // 0.6*p->DXM, src/weno_hj_df_nug.cpp:402
    h->g64.body = h->g32.body = static_cast<const double*>(h->field[R3D_BODY]);
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    return R3D_OK;
}

int r3d_io_levels(r3d_handle* h, double* phimean, double* phiout) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (!h->io) return fail(h, R3D_ESTATE, "r3d_set_ioflow has not set inflow/outflow faces");
    DeviceGuard dg(h->device, h->batch_stream);
    double v[2] = {0.0, 0.0};
    R3D_CUDA(h, cudaMemcpyAsync(v, h->io_buf, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    if (phimean) *phimean = v[kIoPhimean];
    if (phiout) *phiout = v[kIoPhiout];
    return R3D_OK;
}

int r3d_set_step_count(r3d_handle* h, long long count) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (count < 0 || count > (1LL << 50)) return fail(h, R3D_EINVAL, "count out of range");
    DeviceGuard dg(h->device, h->batch_stream);
    h->next_count = count;
    const double c = (double)(count - 1);
    // picard_lsm's step counter (s.pic[3]) and the hooks' one count the steps taken
    launch_set_scalar(h->S.pic + 3, c, h->stream);
    if (h->io_buf) launch_set_scalar(h->io_buf + kIoCount, c, h->stream);
    h->launches += h->io_buf ? 2 : 1;
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    return R3D_OK;
}

int r3d_set_velocity_airy(r3d_handle* h, double amplitude, double wavelength, double depth, double gravity) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (h->batch_stream) return fail(h, R3D_ESTATE, "the instance is a batch member");
    DeviceGuard dg(h->device, h->batch_stream);
    drop_step_graph(h);
    if (!(wavelength > 0.0)) {
        h->airy = false;
        return R3D_OK;
    }
    if (!(depth > 0.0) || !(gravity > 0.0) || !std::isfinite(amplitude) || !std::isfinite(wavelength))
        return fail(h, R3D_EINVAL, "Airy wave needs depth > 0, gravity > 0 and finite amplitude/wavelength");
    if (airy_prepare(h->L)) return fail(h, R3D_EINVAL, "grid too long in x or z for the Airy generator");
    if (!h->coord) {
        std::vector<double> c;
        for (int a : {0, 2}) {
            const int n = h->M.n[a];
            for (int i = -3; i < n + 3; ++i) c.push_back(h->M.xp[a][i + 5]);  // centres
            for (int i = -3; i < n + 3; ++i) c.push_back(h->M.xn[a][i + 6]);  // faces i+1/2
        }
        // order expected by the kernel: x centres, x faces, z centres, z faces
        if (cudaMalloc(&h->coord, c.size() * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            h->coord = nullptr;
            return fail(h, R3D_ENOMEM, "coordinate table allocation failed");
        }
        R3D_CUDA(h, cudaMemcpy(h->coord, c.data(), c.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device) == cudaSuccess && sms > 0)
        h->sms = sms;
    const double kw = 2.0 * 3.141592653589793 / wavelength;
    const double om = std::sqrt(gravity * kw * std::tanh(kw * depth));
    h->ap = r3d::AiryParams{amplitude * om / std::sinh(kw * depth), kw, om, depth};
    h->airy = true;
    h->period = 0.0;
    h->launches += launch_set_scalar(h->S.vscale, 1.0, h->stream);
    R3D_CUDA(h, cudaMemsetAsync(h->field[R3D_V], 0, (size_t)h->L.ncell * elem(h), h->stream));
    h->launches += refresh_velocity(h);
    R3D_CUDA(h, cudaGetLastError());
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    return R3D_OK;
}

int r3d_set_velocity_period(r3d_handle* h, double period) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (!(period >= 0.0) || !std::isfinite(period)) return fail(h, R3D_EINVAL, "period must be >= 0");
    if (h->airy && period > 0.0) return fail(h, R3D_ESTATE, "the Airy generator sets the velocity itself");
    if (h->period != period) drop_step_graph(h);
    h->period = period;
    return R3D_OK;
}

int r3d_set_time(r3d_handle* h, double t) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (!std::isfinite(t)) return fail(h, R3D_EINVAL, "time must be finite");
    DeviceGuard dg(h->device, h->batch_stream);
    h->launches += launch_set_scalar(h->S.t, t, h->stream);
    if (h->period > 0.0) h->launches += launch_set_scalar(h->S.vscale, std::cos(3.141592653589793 * t / h->period), h->stream);
    R3D_CUDA(h, cudaGetLastError());
    return R3D_OK;
}

int r3d_get_time(r3d_handle* h, double* t) {
    if (!h || !t) return fail(h, R3D_EINVAL, "null argument");
    DeviceGuard dg(h->device, h->batch_stream);
    R3D_CUDA(h, cudaMemcpyAsync(t, h->S.t, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    return R3D_OK;
}

int r3d_stage(r3d_handle* h, int kind, int stage) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if ((kind != R3D_STAGE_CONVECTION && kind != R3D_STAGE_REINIT) || stage < 1 || stage > 3)
        return fail(h, R3D_EINVAL, "kind must be R3D_STAGE_CONVECTION or R3D_STAGE_REINIT, stage 1..3");
    if (kind == R3D_STAGE_CONVECTION && !(h->dt_host > 0.0)) return fail(h, R3D_ESTATE, "no time step set");
    DeviceGuard dg(h->device, h->batch_stream);
    h->launches += stage_launch(h, kind == R3D_STAGE_REINIT, stage, false);
    R3D_CUDA(h, cudaGetLastError());
    return R3D_OK;
}

int r3d_init_spheres_tg(r3d_handle* h, int nspheres, const double* spheres, int nmodes, const double* modes) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    if (nspheres < 1 || nspheres > 64 || nmodes < 0 || nmodes > 64 || !spheres || (nmodes && !modes))
        return fail(h, R3D_EINVAL, "1..64 spheres and 0..64 modes");
    DeviceGuard dg(h->device, h->batch_stream);
    // centre and face coordinates of padded indices -3..n+2 per axis
    std::vector<double> xc, xf;
    for (int a = 0; a < 3; ++a) {
        const int n = h->M.n[a];
        for (int i = -3; i < n + 3; ++i) {
            xc.push_back(h->M.xp[a][i + 5]);
            xf.push_back(h->M.xn[a][i + 6]);
        }
    }
    std::vector<double> buf;
    buf.insert(buf.end(), xc.begin(), xc.end());
    buf.insert(buf.end(), xf.begin(), xf.end());
    buf.insert(buf.end(), spheres, spheres + 4 * nspheres);
    if (nmodes) buf.insert(buf.end(), modes, modes + 2 * nmodes);
    double* d = nullptr;
    R3D_CUDA(h, cudaMallocAsync((void**)&d, buf.size() * sizeof(double), h->stream));
    R3D_CUDA(h, cudaMemcpyAsync(d, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    const double* dxc = d;
    const double* dxf = d + xc.size();
    const double* dsp = dxf + xf.size();
    const double* dmo = dsp + 4 * nspheres;
    h->launches += launch_init_fields(h->L, dxc, dxf, nspheres, dsp, nmodes, dmo, fp32(h), h->field[R3D_PHI],
                                      h->field[R3D_U], h->field[R3D_V], h->field[R3D_W], h->stream);
    R3D_CUDA(h, cudaGetLastError());
    R3D_CUDA(h, cudaFreeAsync(d, h->stream));
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    return R3D_OK;
}

int r3d_sync(r3d_handle* h) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    DeviceGuard dg(h->device, h->batch_stream);
    R3D_CUDA(h, cudaStreamSynchronize(h->stream));
    return check_device_flag(h);
}

int r3d_set_option(r3d_handle* h, int option, int value) {
    if (!h) return fail(nullptr, R3D_EINVAL, "null handle");
    switch (option) {
        case R3D_OPT_TILED:
            if (h->use_tile != (value ? 1 : 0)) drop_step_graph(h);
            h->use_tile = value ? 1 : 0;
            return R3D_OK;
        case R3D_OPT_CHUNK:
        case R3D_OPT_CHUNK_REINIT:
            if (value < 1 || value > 4096) return fail(h, R3D_EINVAL, "chunk must be 1..4096 planes");
            drop_step_graph(h);
            if (option == R3D_OPT_CHUNK) h->kc = value;
            h->kc_r = value;
            return R3D_OK;
        case R3D_OPT_BAND64:
            if (h->band64 != (value ? 1 : 0)) drop_step_graph(h);
            h->band64 = value ? 1 : 0;
            return R3D_OK;
        case R3D_OPT_WAIT_TEST: h->wait_test = value ? 1 : 0; return R3D_OK;
        case R3D_OPT_TILE_CFG:
        case R3D_OPT_TILE_CFG_REINIT: {
            if (value < 0 || value >= tile_cfg_count()) return fail(h, R3D_EINVAL, "unknown tile configuration");
            CUtensorMap m[3];
            if (h->tile_ok) {
                // the stage inputs' tensor maps carry the configuration's box
                const int ids[3] = {R3D_PHI, R3D_WORK1, R3D_WORK2};
                std::string why;
                for (int q = 0; q < 3; ++q)
                    if (encode_plane_map(h->L, static_cast<const float*>(h->field[ids[q]]), value, &m[q], &why))
                        return fail(h, R3D_EDEVICE, why);
            }
            drop_step_graph(h);
            for (int q = 0; q < 3 && h->tile_ok; ++q) {
                if (option == R3D_OPT_TILE_CFG) h->map[q] = m[q];
                h->map_r[q] = m[q];
            }
            if (option == R3D_OPT_TILE_CFG) h->tile_cfg = value;
            h->tile_cfg_r = value;
            return R3D_OK;
        }
        default: return fail(h, R3D_EINVAL, "unknown option");
    }
}

int r3d_get_option(r3d_handle* h, int option, int* value) {
    if (!h || !value) return fail(h, R3D_EINVAL, "null argument");
    switch (option) {
        case R3D_OPT_TILED: *value = tiled(h) ? 1 : 0; return R3D_OK;
        case R3D_OPT_CHUNK: *value = h->kc; return R3D_OK;
        case R3D_OPT_BAND64: *value = h->band64; return R3D_OK;
        case R3D_OPT_WAIT_TEST: *value = h->wait_test; return R3D_OK;
        case R3D_OPT_TILE_CFG: *value = h->tile_cfg; return R3D_OK;
        case R3D_OPT_TILE_CFG_REINIT: *value = h->tile_cfg_r; return R3D_OK;
        case R3D_OPT_CHUNK_REINIT: *value = h->kc_r; return R3D_OK;
        default: return fail(h, R3D_EINVAL, "unknown option");
    }
}

int r3d_tile_config_count(void) { return tile_cfg_count(); }

int r3d_tile_config_describe(int cfg, int* tx, int* ty, int* rows_per_thread, int* ring, int* threads) {
    return tile_cfg_describe(cfg, tx, ty, rows_per_thread, ring, threads) ? R3D_EINVAL : R3D_OK;
}

int r3d_stream(r3d_handle* h, void** stream) {
    if (!h || !stream) return fail(h, R3D_EINVAL, "null argument");
    *stream = (void*)h->stream;
    return R3D_OK;
}

int r3d_launch_count(const r3d_handle* h, long long* count) {
    if (!h || !count) return fail(nullptr, R3D_EINVAL, "null argument");
    *count = h->launches;
    return R3D_OK;
}

}  // extern "C"

// ----------------------------------------------------------- slab domain
// One grid split along z into slabs, on one device or several, stepped as
// one: every RK stage runs on all slabs (each on its own stream), then the
// halo planes move between neighbours by peer copies (the role of
// ghostcell::gcparax, src/gcx_parax.cpp), then the next stage; the CFL step
// takes the maxima over all slabs; the whole step is captured in one CUDA
// graph.
struct r3d_domain {
    std::vector<r3d_handle*> slab;
    std::vector<int> k0, k1;
    int nx = 0, ny = 0, nz = 0;
    int f44 = 0;
    int f46 = 0, f47 = 0;  // picard correction of the whole grid (the slabs run with f46 = 0)
    double n47 = 0.0;
    double dxmin = 0.0;
    cudaStream_t main = nullptr;
    std::vector<cudaEvent_t> ev;  // one per slab, reused per stage
    cudaEvent_t fork = nullptr, xdone = nullptr;
    int dev0 = 0;                          // device of slab 0: main stream, gather buffers
    unsigned long long* gather = nullptr;  // the slabs' CFL maxima, 3 per slab (on dev0)
    double* dtbuf = nullptr;               // the grid's time step (on dev0)
    double* pgather = nullptr;             // the slabs' picard slots, 5 per slab (on dev0)
    bool io = false;                       // inflow/outflow faces (r3d_domain_set_ioflow)
    std::vector<double*> iol;              // each slab's crossing heights, 2 ny n (on its device)
    double* iog = nullptr;                 // the grid's heights, 2 ny nz, and state (on dev0)
    cudaGraphExec_t graph = nullptr;
    // what the captured step was built from: adaptive time step, the faces,
    // and each slab's configuration generation (r3d_handle::config_gen)
    int graph_adaptive = -1;
    bool graph_io = false;
    std::vector<unsigned long long> graph_gen;
    bool ran = false;
    std::string err;
};

namespace {

int dfail(r3d_domain* d, int code, const std::string& m) {
    if (d) d->err = m;
    return code;
}

// all slab streams wait for work recorded on the main stream
void domain_fork(r3d_domain* d) {
    cudaSetDevice(d->dev0);
    cudaEventRecord(d->fork, d->main);
    for (r3d_handle* h : d->slab) {
        cudaSetDevice(h->device);
        cudaStreamWaitEvent(h->stream, d->fork, 0);
    }
    cudaSetDevice(d->dev0);
}

// the main stream waits for every slab stream
void domain_join(r3d_domain* d) {
    for (size_t s = 0; s < d->slab.size(); ++s) {
        cudaSetDevice(d->slab[s]->device);
        cudaEventRecord(d->ev[s], d->slab[s]->stream);
    }
    cudaSetDevice(d->dev0);
    for (size_t s = 0; s < d->slab.size(); ++s) cudaStreamWaitEvent(d->main, d->ev[s], 0);
}

// Halo exchange of `field` on the main stream: slab r's top three interior
// planes into slab r+1's bottom ghost planes, and back.
void domain_exchange(r3d_domain* d, int field) {
    domain_join(d);
    for (size_t r = 0; r + 1 < d->slab.size(); ++r) {
        r3d_handle* lo = d->slab[r];
        r3d_handle* hi = d->slab[r + 1];
        const size_t e = field_elem(lo, field), plane = (size_t)lo->L.sz * e;
        char* flo = static_cast<char*>(lo->field[field]);
        char* fhi = static_cast<char*>(hi->field[field]);
        // unified addressing: the copy engine moves the planes between the
        // slabs' devices (peer copies over NVLink) or within one
        cudaMemcpyAsync(fhi, flo + (size_t)lo->L.nz * plane, 3 * plane, cudaMemcpyDefault, d->main);
        cudaMemcpyAsync(flo + (size_t)(lo->L.nz + 3) * plane, fhi + 3 * plane, 3 * plane, cudaMemcpyDefault,
                        d->main);
    }
    domain_fork(d);
}

// One picard volume of the whole grid: every slab's row pass and ordered
// reduce (mode 0: volcalc; 2: an iteration's vol2 share, after the shift by
// the current w when `shift`), then on slab 0's device the sum over the
// slabs in slab order (the role of ghostcell::globalsum,
// src/picard_f.cpp:53, :75) and the grid's w, written back into every
// slab's picard slots.
void domain_picard_sum(r3d_domain* d, bool shift, int mode) {
    const bool lsm = d->f46 == 3;
    for (r3d_handle* h : d->slab) {
        cudaSetDevice(h->device);
        h->launches += launch_picard_local(h->L, h->field[R3D_PHI], fp32(h), picard_epsi(h), picard_cellvol(h), shift,
                                           true, mode, lsm, h->S, h->stream);
    }
    domain_join(d);
    const int n = (int)d->slab.size();
    for (int s = 0; s < n; ++s)
        cudaMemcpyAsync(d->pgather + 5 * s, d->slab[s]->S.pic, 5 * sizeof(double), cudaMemcpyDefault, d->main);
    launch_domain_picard(d->pgather, n, mode == 0 ? 0 : 1, lsm, d->main);
    for (int s = 0; s < n; ++s)
        cudaMemcpyAsync(d->slab[s]->S.pic, d->pgather + 5 * s, 5 * sizeof(double), cudaMemcpyDefault, d->main);
    domain_fork(d);
}

// picard_f / picard_lsm correct_ls over the slabs (src/picard_f.cpp:79-113,
// src/picard_lsm.cpp:88-115): F47 iterations of grid volume, w and shift,
// the last shift alone.  The phi halo planes then follow the shifted
// interiors, so that the next stage reads what the undivided grid reads
// (the reference's decomposed run calls no ghostcell::start4 there and
// keeps the neighbours' pre-shift values in its halos).
void domain_picard_correct(r3d_domain* d) {
    if (d->f47 <= 0) return;
    for (int n = 0; n < d->f47; ++n) domain_picard_sum(d, n > 0, 2);
    for (r3d_handle* h : d->slab) {
        cudaSetDevice(h->device);
        h->launches += launch_picard_local(h->L, h->field[R3D_PHI], fp32(h), picard_epsi(h), picard_cellvol(h), true,
                                           false, 0, d->f46 == 3, h->S, h->stream);
    }
    domain_exchange(d, R3D_PHI);
}

// fsfinflow + fsfrkin/fsfrkout of a decomposed grid (src/ioflow_waterlevel.cpp
// :29-177): the slabs' crossing heights gathered on slab 0's device into the
// whole grid's order (a strided copy per slab and face), one fold into the
// grid's levels and step count (from slab 0's state), the state copied back
// to every slab, then each slab's ghosts.
void domain_io_step(r3d_domain* d) {
    const int n = (int)d->slab.size();
    const size_t plane = (size_t)d->ny * d->nz;
    double* state = d->iog + 2 * plane;
    for (int s = 0; s < n; ++s) {
        r3d_handle* h = d->slab[s];
        cudaSetDevice(h->device);
        h->launches += launch_io_heights(h->L, h->field[R3D_PHI], fp32(h), h->iop, d->iol[s], h->stream);
    }
    domain_join(d);
    cudaMemcpyAsync(state, d->slab[0]->iop.state, kIoStateLen * sizeof(double), cudaMemcpyDefault, d->main);
    for (int s = 0; s < n; ++s) {
        const size_t ns = (size_t)(d->k1[s] - d->k0[s]);
        for (int f = 0; f < 2; ++f)
            cudaMemcpy2DAsync(d->iog + f * plane + d->k0[s], d->nz * sizeof(double), d->iol[s] + f * d->ny * ns,
                              ns * sizeof(double), ns * sizeof(double), d->ny, cudaMemcpyDefault, d->main);
    }
    IoParams p = d->slab[0]->iop;
    p.state = state;
    launch_io_fold(d->iog, (int)plane, p, d->main);
    for (int s = 0; s < n; ++s)
        cudaMemcpyAsync(d->slab[s]->iop.state, state, kIoStateLen * sizeof(double), cudaMemcpyDefault, d->main);
    domain_fork(d);
    for (r3d_handle* h : d->slab) {
        cudaSetDevice(h->device);
        h->launches += launch_io_ghosts(h->L, h->field[R3D_PHI], h->field[R3D_WORK1], h->field[R3D_WORK2], fp32(h),
                                        h->iop, h->stream);
    }
}

void domain_stage(r3d_domain* d, bool reini, int s, bool vol) {
    for (r3d_handle* h : d->slab) {
        cudaSetDevice(h->device);
        h->launches += stage_launch(h, reini, s, vol);
    }
    domain_exchange(d, s == 1 ? R3D_WORK1 : s == 2 ? R3D_WORK2 : R3D_PHI);
}

// One step of every slab (levelset_RK3::start with the inflow/outflow hooks
// and the picard correction F46 selects: 2 or 3 around the step, 1 around
// the reinitialisation, src/reini_RK3.cpp:92, :140), enqueued from the main
// stream back to it.
void domain_enqueue_step(r3d_domain* d, bool adaptive) {
    domain_fork(d);
    for (r3d_handle* h : d->slab) {
        cudaSetDevice(h->device);
        h->launches += refresh_velocity(h);
        if (adaptive)
            h->launches += launch_cfl(h->L, h->field[R3D_U], h->field[R3D_V], h->field[R3D_W], fp32(h),
                                      h->M.dxmin_cfl, h->desc.n47, h->S, h->stream);
    }
    if (adaptive) {
        // gather the maxima on slab 0's device, one dt, back to every slab
        domain_join(d);
        const int n = (int)d->slab.size();
        for (int s = 0; s < n; ++s)
            cudaMemcpyAsync(d->gather + 3 * s, d->slab[s]->S.vmax, 3 * sizeof(unsigned long long), cudaMemcpyDefault,
                            d->main);
        launch_domain_dt(d->gather, n, d->slab[0]->S.vscale, d->dxmin, d->n47, d->dtbuf, d->main);
        for (int s = 0; s < n; ++s)
            cudaMemcpyAsync(d->slab[s]->S.dt, d->dtbuf, sizeof(double), cudaMemcpyDefault, d->main);
        domain_fork(d);
    }
    const bool fluid = d->slab[0]->fluid;
    const bool fused = !fluid && d->f46 == 0;  // volume partials from the last stage
    if (d->io) domain_io_step(d);
    if (d->f46 >= 2) domain_picard_sum(d, false, 0);
    for (int s = 1; s <= 3; ++s) domain_stage(d, false, s, fused && d->f44 == 0 && s == 3);
    if (d->f46 == 1) domain_picard_sum(d, false, 0);
    for (r3d_handle* h : d->slab) {  // fsfrkin/fsfrkout at the start of reini_RK3::start
        cudaSetDevice(h->device);
        h->launches += io_hooks(h, false);
    }
    for (int q = 0; q < d->f44; ++q)
        for (int s = 1; s <= 3; ++s) domain_stage(d, true, s, fused && q == d->f44 - 1 && s == 3);
    if (d->f46 == 3 && d->io)
        for (r3d_handle* h : d->slab) {  // picard_lsm's netvol += (Qi - Qo) dt
            cudaSetDevice(h->device);
            h->launches += launch_netvol(h->S, h->iod.qi, h->iod.qo, h->stream);
        }
    if (d->f46 != 0) domain_picard_correct(d);
    for (r3d_handle* h : d->slab) {
        cudaSetDevice(h->device);
        if (fluid)  // fluid_update_fsf: ro, visc and the volume sums (src/levelset_RK3.cpp:174)
            h->launches += fluid_update(h, true);
        else if (!fused)
            h->launches += launch_volume_direct_clock(h->L, h->field[R3D_PHI], fp32(h), h->g64.dxn[0], h->g64.dxn[1],
                                                      h->g64.dxn[2], h->M.psi, h->period, h->S, h->stream);
        else
            h->launches += launch_volume_reduce(h->L, h->S, volume_block_count(h), h->period, h->stream);
    }
    if (fluid) {
        domain_exchange(d, R3D_RO);
        domain_exchange(d, R3D_VISC);
    }
    domain_join(d);
}

}  // namespace

extern "C" {

int r3d_domain_create(const r3d_grid_desc* desc, int nslabs, const int* devices, r3d_domain** out) {
    std::string why;
    if (!out) return fail(nullptr, R3D_EINVAL, "null output");
    *out = nullptr;
    if (int rc = check_desc(desc, why)) return fail(nullptr, rc, why);
    if (nslabs < 1 || desc->nz < 3 * nslabs) return fail(nullptr, R3D_EINVAL, "every slab needs >= 3 z cells");
    r3d_domain* d = new (std::nothrow) r3d_domain();
    if (!d) return fail(nullptr, R3D_ENOMEM, "host allocation failed");
    d->nx = desc->nx;
    d->ny = desc->ny;
    d->nz = desc->nz;
    d->f44 = desc->f44;
    d->f46 = desc->f46;
    d->f47 = desc->f47;
    d->n47 = desc->n47;
    double out4[4];
    if (int rc = r3d_grid_spacing(desc, out4)) {
        delete d;
        return rc;
    }
    const int base = desc->nz / nslabs, extra = desc->nz % nslabs;
    int k = 0;
    d->dxmin = 1.0e300;
    int rc = R3D_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    d->dev0 = devices ? devices[0] : cur;
    for (int r = 0; r < nslabs && !rc; ++r) {
        const int n = base + (r < extra ? 1 : 0);
        r3d_grid_desc sd = *desc;
        sd.nz = n;
        sd.f46 = 0;  // the grid's picard runs over all slabs at once
        sd.zn = desc->zn + k;  // node indices -5..n+5 of the slab
        r3d_handle* h = nullptr;
        if (cudaSetDevice(devices ? devices[r] : cur) != cudaSuccess) {
            rc = R3D_EINVAL;
            break;
        }
        rc = r3d_create(&sd, &h);
        if (h) h->domain_slab = true;
        if (!rc) rc = r3d_set_halo(h, k > 0 ? 1 : 0, k + n < desc->nz ? 1 : 0);
        if (!rc) rc = r3d_set_grid_spacing(h, out4[0], out4[1], out4[2]);
        if (h) {
            d->slab.push_back(h);
            d->k0.push_back(k);
            d->k1.push_back(k + n);
            d->dxmin = std::min(d->dxmin, h->M.dxmin_cfl);
        }
        k += n;
    }
    auto bail = [&](int code, const std::string& m) {
        r3d_domain_destroy(d);
        return fail(nullptr, code, m);
    };
    if (rc) {
        cudaSetDevice(cur);
        return bail(rc, "creating the slabs");
    }
    // halo, CFL and picard copies go between neighbouring slabs and to slab
    // 0's device: let those devices address each other's memory directly
    // (without it a copy between two GPUs is staged through the host)
    for (size_t r = 0; r < d->slab.size(); ++r) {
        const int a = d->slab[r]->device;
        std::vector<int> peers = {d->dev0};
        if (r + 1 < d->slab.size()) peers.push_back(d->slab[r + 1]->device);
        for (int b : peers) {
            if (a == b) continue;
            for (int pass = 0; pass < 2; ++pass) {
                const int from = pass ? b : a, to = pass ? a : b;
                int can = 0;
                if (cudaDeviceCanAccessPeer(&can, from, to) != cudaSuccess || !can) continue;
                cudaSetDevice(from);
                const cudaError_t e = cudaDeviceEnablePeerAccess(to, 0);
                if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled) {
                    cudaGetLastError();
                    cudaSetDevice(cur);
                    return bail(R3D_EDEVICE, std::string("peer access: ") + cudaGetErrorString(e));
                }
                cudaGetLastError();  // clear cudaErrorPeerAccessAlreadyEnabled
            }
        }
    }
    cudaSetDevice(cur);
    d->ev.resize(d->slab.size(), nullptr);
    for (size_t r = 0; r < d->slab.size(); ++r) {  // each event on its slab's device
        cudaSetDevice(d->slab[r]->device);
        if (cudaEventCreateWithFlags(&d->ev[r], cudaEventDisableTiming) != cudaSuccess) {
            cudaSetDevice(cur);
            return bail(R3D_EDEVICE, "domain events");
        }
    }
    cudaSetDevice(d->dev0);
    const bool ok = cudaStreamCreateWithFlags(&d->main, cudaStreamNonBlocking) == cudaSuccess &&
                    cudaEventCreateWithFlags(&d->fork, cudaEventDisableTiming) == cudaSuccess &&
                    cudaEventCreateWithFlags(&d->xdone, cudaEventDisableTiming) == cudaSuccess &&
                    cudaMalloc(&d->gather, 3 * d->slab.size() * sizeof(unsigned long long)) == cudaSuccess &&
                    cudaMalloc(&d->dtbuf, sizeof(double)) == cudaSuccess &&
                    cudaMalloc(&d->pgather, 5 * d->slab.size() * sizeof(double)) == cudaSuccess;
    cudaSetDevice(cur);
    if (!ok) return bail(R3D_EDEVICE, "domain stream, events and buffers");
    *out = d;
    return R3D_OK;
}

int r3d_domain_destroy(r3d_domain* d) {
    if (!d) return R3D_EINVAL;
    if (d->main) cudaStreamSynchronize(d->main);
    if (d->graph) cudaGraphExecDestroy(d->graph);
    for (r3d_handle* h : d->slab) r3d_destroy(h);
    for (auto e : d->ev)
        if (e) cudaEventDestroy(e);
    if (d->fork) cudaEventDestroy(d->fork);
    if (d->xdone) cudaEventDestroy(d->xdone);
    if (d->gather) cudaFree(d->gather);
    if (d->dtbuf) cudaFree(d->dtbuf);
    if (d->pgather) cudaFree(d->pgather);
    for (size_t s = 0; s < d->iol.size(); ++s)
        if (d->iol[s]) cudaFree(d->iol[s]);
    if (d->iog) cudaFree(d->iog);
    if (d->main) cudaStreamDestroy(d->main);
    delete d;
    return R3D_OK;
}

const char* r3d_domain_last_error(const r3d_domain* d) { return d ? d->err.c_str() : ""; }

int r3d_domain_slab(r3d_domain* d, int s, r3d_handle** h, int* k0, int* k1) {
    if (!d || s < 0 || s >= (int)d->slab.size()) return dfail(d, R3D_EINVAL, "bad slab index");
    if (h) *h = d->slab[s];
    if (k0) *k0 = d->k0[s];
    if (k1) *k1 = d->k1[s];
    return R3D_OK;
}

int r3d_domain_upload(r3d_domain* d, int field, const double* host) {
    if (!d || !host) return dfail(d, R3D_EINVAL, "null argument");
    const long long jm = d->ny + 6, km = d->nz + 6;
    for (size_t s = 0; s < d->slab.size(); ++s) {
        const int n = d->k1[s] - d->k0[s];
        std::vector<double> part((size_t)(d->nx + 6) * jm * (n + 6));
        for (long long i = 0; i < d->nx + 6; ++i)
            for (long long j = 0; j < jm; ++j)
                std::memcpy(&part[((size_t)i * jm + j) * (n + 6)], host + (i * jm + j) * km + d->k0[s],
                            sizeof(double) * (n + 6));
        if (int rc = r3d_upload(d->slab[s], field, part.data(), R3D_LAYOUT_REEF3D))
            return dfail(d, rc, r3d_last_error(d->slab[s]));
    }
    return R3D_OK;
}

int r3d_domain_download(r3d_domain* d, int field, double* host) {
    if (!d || !host) return dfail(d, R3D_EINVAL, "null argument");
    const long long jm = d->ny + 6, km = d->nz + 6;
    const size_t ns = d->slab.size();
    for (size_t s = 0; s < ns; ++s) {
        const int n = d->k1[s] - d->k0[s];
        std::vector<double> part((size_t)(d->nx + 6) * jm * (n + 6));
        if (int rc = r3d_download(d->slab[s], field, part.data(), R3D_LAYOUT_REEF3D))
            return dfail(d, rc, r3d_last_error(d->slab[s]));
        // interior planes of the slab; the outer ghost planes from the end slabs
        const int lo = s == 0 ? 0 : 3, hi = s + 1 == ns ? n + 6 : n + 3;
        for (long long i = 0; i < d->nx + 6; ++i)
            for (long long j = 0; j < jm; ++j)
                std::memcpy(host + (i * jm + j) * km + d->k0[s] + lo, &part[((size_t)i * jm + j) * (n + 6) + lo],
                            sizeof(double) * (hi - lo));
    }
    return R3D_OK;
}

int r3d_domain_run(r3d_domain* d, int nsteps, double dt) {
    if (!d || nsteps < 0) return dfail(d, R3D_EINVAL, "bad argument");
    DeviceGuard dg(d->dev0);  // restores the caller's device
    const bool adaptive = !(dt > 0.0);
    for (r3d_handle* h : d->slab)
        if (h->io != d->io || h->fluid != d->slab[0]->fluid)
            return dfail(d, R3D_EINVAL, "inflow/outflow faces only through r3d_domain_set_ioflow; fluid update on all "
                                        "slabs or none");
    if (!adaptive)
        for (r3d_handle* h : d->slab)
            if (int rc = r3d_set_dt(h, dt)) return dfail(d, rc, r3d_last_error(h));
    for (r3d_handle* h : d->slab) cudaStreamSynchronize(h->stream);
    // the captured step bakes in the slabs' configuration (velocity
    // generator and its parameters, forcing lists, fluid constants, options):
    // recapture when any slab's configuration generation moved
    std::vector<unsigned long long> gen;
    for (r3d_handle* h : d->slab) gen.push_back(h->config_gen);
    if (!d->graph || d->graph_adaptive != (adaptive ? 1 : 0) || d->graph_io != d->io || d->graph_gen != gen) {
        if (d->graph) cudaGraphExecDestroy(d->graph);
        d->graph = nullptr;
        cudaGraph_t g = nullptr;
        cudaSetDevice(d->dev0);
        if (cudaStreamBeginCapture(d->main, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return dfail(d, R3D_EDEVICE, "domain capture");
        domain_enqueue_step(d, adaptive);
        cudaError_t e = cudaStreamEndCapture(d->main, &g);
        if (e == cudaSuccess) e = cudaGraphInstantiate(&d->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            d->graph = nullptr;
            cudaGetLastError();  // leave no capture error behind for later calls
            return dfail(d, R3D_EDEVICE, std::string("domain step graph: ") + cudaGetErrorString(e));
        }
        d->graph_adaptive = adaptive ? 1 : 0;
        d->graph_io = d->io;
        d->graph_gen = gen;
    }
    cudaSetDevice(d->dev0);
    for (int n = 0; n < nsteps; ++n)
        if (cudaGraphLaunch(d->graph, d->main) != cudaSuccess) return dfail(d, R3D_EDEVICE, "domain step launch");
    const cudaError_t e = cudaStreamSynchronize(d->main);
    if (e != cudaSuccess) return dfail(d, R3D_EDEVICE, cudaGetErrorString(e));
    for (r3d_handle* h : d->slab) {
        h->have_last_volume = true;
        if (int rc = check_device_flag(h)) return dfail(d, rc, r3d_last_error(h));
    }
    d->ran = d->ran || nsteps > 0;
    return R3D_OK;
}

int r3d_domain_last_volume(r3d_domain* d, double* volume1, double* volume2) {
    if (!d) return R3D_EINVAL;
    if (!d->ran) return dfail(d, R3D_ESTATE, "no step has run yet");
    double a = 0.0, b = 0.0;
    for (r3d_handle* h : d->slab) {
        double v1 = 0.0, v2 = 0.0;
        if (int rc = r3d_last_volume(h, &v1, &v2)) return dfail(d, rc, r3d_last_error(h));
        a += v1;
        b += v2;
    }
    if (volume1) *volume1 = a;
    if (volume2) *volume2 = b;
    return R3D_OK;
}

int r3d_domain_set_ioflow(r3d_domain* d, const r3d_ioflow_desc* io) {
    if (!d) return R3D_EINVAL;
    if (d->graph) {  // the captured step holds the faces' parameters
        cudaGraphExecDestroy(d->graph);
        d->graph = nullptr;
    }
    for (r3d_handle* h : d->slab)
        if (int rc = r3d_set_ioflow(h, io)) {
            for (r3d_handle* g : d->slab) r3d_set_ioflow(g, nullptr);
            d->io = false;
            return dfail(d, rc, r3d_last_error(h));
        }
    d->io = io != nullptr;
    if (!d->io || d->iog) return R3D_OK;
    // crossing heights: per slab on its device, the grid's on slab 0's
    DeviceGuard dg(d->dev0);
    d->iol.assign(d->slab.size(), nullptr);
    bool ok = true;
    for (size_t s = 0; s < d->slab.size() && ok; ++s) {
        cudaSetDevice(d->slab[s]->device);
        ok = cudaMalloc(&d->iol[s], 2 * (size_t)d->ny * (d->k1[s] - d->k0[s]) * sizeof(double)) == cudaSuccess;
    }
    cudaSetDevice(d->dev0);
    ok = ok && cudaMalloc(&d->iog, (2 * (size_t)d->ny * d->nz + kIoStateLen) * sizeof(double)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        for (size_t s = 0; s < d->iol.size(); ++s)
            if (d->iol[s]) cudaFree(d->iol[s]);
        d->iol.clear();
        if (d->iog) cudaFree(d->iog);
        d->iog = nullptr;
        for (r3d_handle* g : d->slab) r3d_set_ioflow(g, nullptr);
        d->io = false;
        return dfail(d, R3D_ENOMEM, "inflow/outflow buffers");
    }
    return R3D_OK;
}

int r3d_domain_set_fluid(r3d_domain* d, double ro_water, double visc_water, double ro_air, double visc_air) {
    if (!d) return R3D_EINVAL;
    if (d->graph) {  // the captured step holds the fluid constants
        cudaGraphExecDestroy(d->graph);
        d->graph = nullptr;
    }
    for (r3d_handle* h : d->slab)
        if (int rc = r3d_set_fluid(h, ro_water, visc_water, ro_air, visc_air)) return dfail(d, rc, r3d_last_error(h));
    return R3D_OK;
}

int r3d_domain_fluid_update(r3d_domain* d, double* volume1, double* volume2) {
    if (!d) return R3D_EINVAL;
    double a = 0.0, b = 0.0;
    for (r3d_handle* h : d->slab) {
        double v1 = 0.0, v2 = 0.0;
        if (int rc = r3d_fluid_update(h, &v1, &v2)) return dfail(d, rc, r3d_last_error(h));
        a += v1;
        b += v2;
    }
    {
        DeviceGuard dg(d->dev0);
        domain_exchange(d, R3D_RO);
        domain_exchange(d, R3D_VISC);
        domain_join(d);
        if (cudaStreamSynchronize(d->main) != cudaSuccess) return dfail(d, R3D_EDEVICE, "domain halo copies");
    }
    if (volume1) *volume1 = a;
    if (volume2) *volume2 = b;
    return R3D_OK;
}

int r3d_domain_get_dt(r3d_domain* d, double* dt) {
    if (!d || !dt) return R3D_EINVAL;
    if (cudaMemcpy(dt, d->slab[0]->S.dt, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return dfail(d, R3D_EDEVICE, "reading dt");
    return R3D_OK;
}

}  // extern "C"
