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
    float eps[3];  // 1/h^2 per axis
    float dtr;
    float deltax;
    int f49;
    int band64;
    double psi;
    double cellvol;
    int kc;
};

// Encodes the 3D tensor map of a padded FP32 field for the 72 x 14 x 1
// plane boxes the tile kernels load.  Returns 0 on success.
int encode_plane_map(const Layout& L, const float* base, CUtensorMap* out, std::string* why);
int launch_tile_stage(const CUtensorMap& map, const TileArgs& a, bool reini, int stage, bool volume, cudaStream_t st);

}  // namespace r3d
