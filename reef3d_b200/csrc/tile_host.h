// Host side of the TMA-tiled FP32 stage kernels.
#pragma once

#include <cuda.h>

#include "r3d_internal.h"

namespace r3d {

struct TileArgs {
    Layout L;
    const float* fn;
    float* out;
    const float* u;
    const float* v;
    const float* w;
    const double* dt;
    const double* vscale;
    double* partial;
    int* err;
    float rh[3];
    float eps[3];    // 1/h^2 per axis
    double beps[3];  // FP64 interface band: 1e-6 h^2 per axis, h = 1/(double)rh
    float dtr;
    float deltax;
    int f49;
    int band64;
    int wait_test;   // nonzero: each item first waits for a copy that is never issued (timeout-path test)
    long long spin;  // iteration limit of a bounded wait (0: the default)
    double psi;
    double cellvol;
    int kc;
};

// True when the three axes' spacing constants are bitwise equal (cubic
// cells): the kernels then hold one set for all axes, with the same results.
inline bool tile_args_iso(const TileArgs& a) {
    return a.rh[0] == a.rh[1] && a.rh[1] == a.rh[2] && a.eps[0] == a.eps[1] && a.eps[1] == a.eps[2];
}

// A member of a batch that runs on the tiled kernels (3D, uniform, FP32).
struct TiledMember {
    TileArgs args;  // fn, u, v, w, dt, vscale, err, metrics, kc; out set per stage
    float* phi;
    float* a1;
    float* a2;
    int f44;
};

// Tile configurations of the tiled kernels (tile shape, rows per thread,
// ring depth); id 0 .. tile_cfg_count()-1.  describe: returns 0 for a valid id.
int tile_cfg_count();
int tile_cfg_describe(int cfg, int* tx, int* ty, int* ry, int* ring, int* threads);
// Encodes the 3D tensor map of a padded FP32 field for the (TX+8) x (TY+6) x 1
// plane boxes configuration `cfg` loads.  Returns 0 on success.
int encode_plane_map(const Layout& L, const float* base, int cfg, CUtensorMap* out, std::string* why);
int launch_tile_stage(const CUtensorMap& map, const TileArgs& a, int cfg, bool reini, int stage, bool volume,
                      cudaStream_t st);
// Sets the tiled kernels' shared-memory attributes on the current device
// (once per device); false when the device refuses them.
bool tile_prepare();
// CTAs per SM configuration `cfg` is built to co-reside (persistent grids)
int tile_ctas_per_sm(int cfg);
long long tile_items_of(const Layout& L, int kc, int cfg);
// Batched persistent tiled stage over the items of nm tiled members, whose
// maps were encoded for configuration `cfg`.
// work: two zero-initialised counters the launch takes items from (it leaves
// them at zero for the next launch on the same stream).
// iso: every member's spacing constants satisfy tile_args_iso.
int launch_batch_tile_stage(const TiledMember* members, const CUtensorMap* maps, const long long* tile0, int nm,
                            int cfg, bool iso, bool reini, int stage, int q, double* vol_part, unsigned* work,
                            unsigned grid, cudaStream_t st);
// Per-item face maxima of the tiled members (3 doubles per item).
int launch_batch_tile_vmax(const TiledMember* members, const long long* tile0, int nm, int cfg, double* vmax_part,
                           unsigned grid, cudaStream_t st);

}  // namespace r3d
