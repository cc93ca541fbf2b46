// Internal declarations shared by the host API (api.cpp) and the kernel
// translation units.  Not part of the public C-ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace r3d {

// Device field layout: x contiguous ("i-contiguous"), padded by ghost cells.
// A cell (i,j,k) of the interior lives at
//     (k + gz) * sz + (j + gy) * sy + (i + gx)
// with gx = 4 (3 ghost cells plus one slot so the interior starts 16-byte
// aligned for FP32 and FP64 alike), gy = gz = 3.  A 2D grid (ny == 1) keeps
// no y ghost planes (gy = 0, py = 1): the reference never writes them on
// this path.  Faces: u(i) is the x face i+1/2, v(j) the y face j+1/2, w(k)
// the z face k+1/2 (the staggering of src/flux_HJ_CDS2.cpp:59-127).
struct Layout {
    int nx, ny, nz;
    int gx, gy, gz;
    int px, py, pz;
    long long sy, sz;
    long long ncell;  // px*py*pz
    bool two_d;
    // faces whose ghosts the stage kernels do not write (0 for the closed
    // box).  Inflow / outflow: kIoSkipLo / kIoSkipHi leave the x-min / x-max
    // face ghosts of a level-set field untouched (ghost label 0 of
    // src/gc_epol4.cpp:26-58); kIoEdge also writes the edge ghost
    // (-1, j, nz) of each inflow column, which the inflow water level reads
    // (src/ioflow_waterlevel.cpp:55).  Subdomain (slab) boundaries:
    // kHaloZLo / kHaloZHi mark z faces whose ghost planes a neighbour's
    // halo fills (src/gcx_parax.cpp) -- no wall copy there, for any field,
    // and the z faces at nz-1 belong to the CFL maximum (wlast = 0 with a
    // neighbour above, src/lexer_gridsize.cpp:78-79).
    int io;
};
constexpr int kIoSkipLo = 1, kIoSkipHi = 2, kIoEdge = 4, kHaloZLo = 8, kHaloZHi = 16;

Layout make_layout(int nx, int ny, int nz);

// Per-axis metric and WENO table offsets inside one device buffer of
// doubles (FP64) and one of floats (FP32).  Index t = cell index + 5, the
// reference's 1D indexing (src/iterators1D.h:25-60).
struct AxisTables {
    long long dxp, dxn;          // n + 21 entries each
    long long qf, cf, isf;       // (n+8)*12, (n+8)*6, (n+8)*18 entries
};

struct HostMetrics {
    int n[3];
    std::vector<double> xn[3], xp[3], dxn[3], dxp[3];
    std::vector<double> qf[3], cf[3], isf[3];
    double dxm_mean;   // src/grid.cpp:102-148
    double dym, dzm;   // DIVEMesh header spacings (first node spacing)
    double psi;        // src/ini_psi.cpp:33-37
    double dxmin_cfl;  // min over cells of MIN3(DXN,DYN,DZN) (src/ietimestep.cpp:160-166)
    bool uniform;      // every spacing equal to the first within 1e-12 relative
    double h[3];       // uniform spacing per axis
};

// Builds the metrics exactly as the reference does (src/grid.cpp:55-148,
// src/weno_nug_func_precalc_qf.cpp, _cf.cpp, _isf.cpp, src/ini_psi.cpp).
void build_metrics(int nx, int ny, int nz, const double* xn, const double* yn, const double* zn,
                   double f45, HostMetrics& m);

// Kernel-side view of an instance (passed by value).
template <typename T>
struct KGrid {
    Layout L;
    const T* dxp[3];
    // (DXP, 1/DXP) pairs per index, 1/DXP the IEEE quotient (the FP64 face
    // divisions, div_rn), 16-byte aligned
    const T* dpr[3];
    // the WENO node tables of one (index, side) in one record of 18 values:
    // Q0..Q5, C0..C2, S0..S8 (record 2t + side), 16-byte aligned
    const T* wt[3];
    const T* dxn[3];
    const T* qf[3];
    const T* cf[3];
    const T* isf[3];
    double f43;
    int f49;
    double psi;
    // FP64 cell sizes DXN, DYN, DZN for the volume sums (the FP32 form
    // sums in FP64 with the exact cell volumes)
    const double* dxn_d[3];
    // direct-forcing convection stencils (X45 1..6; 1..5 in the FP32 form):
    // the body field they read (FP64 in both forms, so that every mask
    // decision is the reference's) and 0.6 DXM, the fb threshold of X45 = 1
    int x45;
    double df_thr;
    const double* body;
    // uniform-grid FP32 form
    float h[3], rh[3];
    float eps_u;  // WENO psi (1e-6); rescaled by h^2 per axis for undivided differences
};

struct Fields {
    void* phi;
    void* a1;
    void* a2;
    void* L;
    void* u;
    void* v;
    void* w;
};

// Scratch in device memory: FP64 reduction partials and scalars.
struct Scratch {
    double* partial;        // per-block volume partial sums (2 per block)
    long long npartial;     // capacity in blocks
    unsigned long long* vmax;  // |u|,|v|,|w| maxima as ordered bit patterns
    double* dt;             // current time step (read by the stage kernels)
    double* vol;            // volume1, volume2
    double* t;              // simulated time (advanced by each step)
    double* vscale;         // factor applied to the stored face velocities
    int* err;               // set by a kernel whose bounded wait gave up
    double* pic;            // picard: step-start volume, shift w, picard_lsm target, step count
};

// ---- launchers (kernels_f64.cu / kernels_f32.cu / kernels_common.cu)
// All launchers enqueue on `st` and return the number of kernels launched.
int launch_conv_stage_f64(const KGrid<double>& g, const Fields& f, int stage, const Scratch& s,
                          bool volume, cudaStream_t st);
int launch_reini_stage_f64(const KGrid<double>& g, const Fields& f, int stage, const Scratch& s,
                           bool volume, cudaStream_t st);
int launch_conv_L_f64(const KGrid<double>& g, const void* in, const Fields& f, const Scratch& s, cudaStream_t st);
int launch_reini_L_f64(const KGrid<double>& g, const void* in, const Fields& f, cudaStream_t st);

int launch_conv_stage_f32(const KGrid<float>& g, const Fields& f, int stage, const Scratch& s,
                          bool volume, cudaStream_t st);
int launch_reini_stage_f32(const KGrid<float>& g, const Fields& f, int stage, const Scratch& s,
                           bool volume, cudaStream_t st);
int launch_conv_L_f32(const KGrid<float>& g, const void* in, const Fields& f, const Scratch& s, cudaStream_t st);
int launch_reini_L_f32(const KGrid<float>& g, const void* in, const Fields& f, cudaStream_t st);

long long volume_blocks(const Layout& L);

// also advances the device clock by dt and, with period > 0, sets the
// velocity factor cos(pi t / period)
int launch_volume_reduce(const Layout& L, const Scratch& s, long long nblocks, double period, cudaStream_t st);
int launch_volume_direct(const Layout& L, const void* phi, bool fp32, const double* dxn,
                         const double* dyn, const double* dzn, double psi, const Scratch& s,
                         cudaStream_t st);
// Relaxation zones of the wave generator and the numerical beach on the
// level set (iowave::phi_relax, src/iowave_relax.cpp:346-378), device side:
// col[4 q .. 4 q + 3] = (i, j, zone bits: 1 generation, 2 beach, offset of
// the column's first generation target) for each zone column q; w[2 q],
// w[2 q + 1] = its generation and beach weights relax4_wg(i,j),
// relax4_nb(i,j); zc the cell-centre z of k = 0..nz-1; lsval the
// generation zone's targets (the wave theory's level set, LOOP order);
// *ramp the wave generation ramp of the step.
struct RelaxZones {
    const int* col;
    const double* w;
    const double* zc;
    const double* lsval;
    const double* ramp;
    int ncol;
    double phimean;
};
int launch_relax(const Layout& L, void* f, bool fp32, const RelaxZones& z, cudaStream_t st);

// Airy wave velocity generator: a = amp om / sinh(kw depth), kw = 2 pi /
// wavelength, om = sqrt(g kw tanh(kw depth)).
struct AiryParams {
    double a, kw, om, depth;
};
// Writes u and w of the Airy field at the device time *t on every stored
// cell; coord = x centres, x faces, z centres, z faces (padded indices
// -3..n+2).  airy_prepare sets the kernels' shared-memory limit (nonzero:
// the grid is too long in x or z for the shared-memory tables).
int airy_prepare(const Layout& L);
int launch_airy(const Layout& L, void* u, void* w, bool fp32, const double* coord, const double* t,
                const AiryParams& ap, int sms, cudaStream_t st);

// Fluid constants of fluid_update_fsf (W1..W4, src/ini.cpp:831-834).
struct FluidConst {
    double ro_water, visc_water, ro_air, visc_air;
};
// Density/viscosity update with volume sums (src/fluid_update_fsf.cpp:39-104);
// clock: the volume pass also advances the device clock like
// launch_volume_reduce.
int launch_fluid_update(const Layout& L, const void* phi, void* ro, void* visc, bool fp32, const double* dxn,
                        const double* dyn, const double* dzn, double psi, const FluidConst& fc, bool clock,
                        double period, const Scratch& s, cudaStream_t st);

// Picard mass correction (src/picard_f.cpp:36-113; lsm: src/picard_lsm.cpp)
// on the interior of phi: epsi = f45*DXM, cellvol = DXM^3 (host pow).
// launch_picard_volcalc stores the smoothed-Heaviside volume in s.pic[0]
// (lsm: the first step's one also in s.pic[2]); launch_picard_correct runs
// f47 iterations of "volume, w = r(target) - r(vol2), phi += w".
int launch_picard_volcalc(const Layout& L, const void* phi, bool fp32, double epsi, double cellvol, bool lsm,
                          const Scratch& s, cudaStream_t st);
int launch_picard_correct(const Layout& L, void* phi, bool fp32, double epsi, double cellvol, int f47, bool lsm,
                          const Scratch& s, cudaStream_t st);
// Volume pass of r3d_volume that also advances the device clock like
// launch_volume_reduce (used when the step's last stage cannot fuse it).
int launch_volume_direct_clock(const Layout& L, const void* phi, bool fp32, const double* dxn,
                               const double* dyn, const double* dzn, double psi, double period,
                               const Scratch& s, cudaStream_t st);
int launch_cfl(const Layout& L, const void* u, const void* v, const void* w, bool fp32,
               double dxmin, double n47, const Scratch& s, cudaStream_t st);
int launch_ghost_fill(const Layout& L, void* f, bool fp32, cudaStream_t st);

// ioflow_f level-set hooks (src/ioflow_waterlevel.cpp:29-177) on an
// inflow x-min face and an outflow x-max face.
struct IoParams {
    int inflow, outflow;  // faces present
    int f50, b77, f64;
    double f56, f60, f62;
    const double* zp;     // cell-centre z (ZP), index k + 5
    const double* dzp;    // centre spacing (DZP), index k + 5
    const double* ramp;   // outflow level ramp for count = 0 .. f64-1
    double* state;        // kIo* slots below
    // the faces belong to REEF3D's wave generator (iowave): its fsfinflow
    // imposes nothing (src/iowave_waterlevel.cpp:29-35 without flow files or
    // patch boundaries) and its fsfrkin / fsfrkout copy the level set's
    // ghost layers into the stage buffers (:37-63)
    int waves;
};
constexpr int kIoPhimean = 0, kIoPhiout = 1, kIoCount = 2, kIoWsfout = 3, kIoFound = 4, kIoStateLen = 8;
// fsfinflow: advances the step count, measures the water levels, imposes
// the inflow / outflow ghosts of phi; then fsfrkin/fsfrkout on a1 and a2.
// step == false: fsfrkin/fsfrkout only (the start of reini_RK3::start).
int launch_io_hooks(const Layout& L, void* phi, void* a1, void* a2, bool fp32, const IoParams& p, bool step,
                    cudaStream_t st);
// The same split for a decomposed grid: every slab's crossing heights
// (2 ny nz doubles, NaN where none), the fold of the gathered heights of the
// whole grid (n = ny nz per face) into p.state, then every slab's imposing
// half of fsfinflow with fsfrkin/fsfrkout.
int launch_io_heights(const Layout& L, const void* phi, bool fp32, const IoParams& p, double* out, cudaStream_t st);
int launch_io_fold(const double* heights, int n, const IoParams& p, cudaStream_t st);
int launch_io_ghosts(const Layout& L, void* phi, void* a1, void* a2, bool fp32, const IoParams& p, cudaStream_t st);
// VTU point data at the grid nodes: out[0..n) phi, then rho and viscosity
// when ro != nullptr (3 n floats).
int launch_vtu_nodes(const Layout& L, const void* phi, const void* ro, const void* visc, bool fp32, float* out,
                     long long npoints, cudaStream_t st);
// One picard pass of one subdomain (row pass with the shift and/or the
// volume; with sum, the reduce in `mode`: 0 volcalc, 2 this slab's vol2 into
// s.pic[4]); and the grid-wide step over the gathered pic[0..4] of n slabs.
int launch_picard_local(const Layout& L, void* phi, bool fp32, double epsi, double cellvol, bool shift, bool sum,
                        int mode, bool lsm, const Scratch& s, cudaStream_t st);
int launch_domain_picard(double* gathered, int n, int mode, bool lsm, cudaStream_t st);
// dt of a decomposed grid from the slabs' maxima gathered into vm[3 n], at
// the grid's smallest cell.
int launch_domain_dt(const unsigned long long* vm, int n, const double* vscale, double dxmin, double n47, double* dt,
                     cudaStream_t st);
// dt from the velocity maxima already in s.vmax (the CFL's second kernel).
int launch_dt_from_max(double dxmin, double n47, const Scratch& s, cudaStream_t st);
// Solid forcing of a field (src/gc_solid_forcing_lsm.cpp): one launch per
// dependency level [level_off[l], level_off[l+1]) of the device op list.
int launch_solid_forcing(void* f, bool fp32, const long long* ops, const std::vector<int>& level_off,
                         cudaStream_t st);
// picard_lsm's netvol = netvol + Qi dt - Qo dt (src/picard_lsm.cpp:93)
int launch_netvol(const Scratch& s, double qi, double qo, cudaStream_t st);
// host layout <-> device layout (src is a device staging copy of the host array)
int launch_import(const Layout& L, const double* staging, int layout, void* dst, bool fp32,
                  cudaStream_t st);
int launch_export(const Layout& L, const void* src, bool fp32, int layout, double* staging,
                  cudaStream_t st);
int launch_zero(void* p, size_t bytes, cudaStream_t st);

// TMA-tiled FP32 stage kernels (kernels_f32_tile.cu), 3D uniform grids
struct TileArgs;
size_t tile_smem_bytes(int cfg);
dim3 tile_grid(const Layout& L, int kc, int cfg);
int launch_set_scalar(double* dst, double value, cudaStream_t st);
int launch_init_fields(const Layout& L, const double* xc, const double* xf, int ns, const double* sph, int nm,
                       const double* modes, bool fp32, void* phi, void* u, void* v, void* w, cudaStream_t st);

}  // namespace r3d
