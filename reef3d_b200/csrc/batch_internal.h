// Batched execution of many FP32 instances (kernels_batch.cu, batch.cpp).
#pragma once

#include "r3d_internal.h"

namespace r3d {

// Everything a batched kernel needs about one member instance.
struct MemberDesc {
    KGrid<float> g;
    float* phi;
    float* a1;
    float* a2;
    const float* u;
    const float* v;
    const float* w;
    double* dt;
    double* vscale;
    double* t;
    double* vol;
    double n47;
    double dxmin;
    double period;
    int f44;
};

struct BatchLaunch {
    const MemberDesc* members;
    const long long* tile0;  // first tile of each member, nm+1 entries
    int nm;
    long long t_begin;       // first tile of these members in the batch's tile space
    long long ntiles;        // one past the last tile
    double* vol_part;        // 2 per tile
    double* vmax_part;       // 3 per tile
    int rows;                // tile rows (2, 4 or 8); 32*rows threads per CTA
    unsigned grid;           // persistent CTAs
};

long long batch_tiles_of(const Layout& L, int rows);
int launch_batch_stage(const BatchLaunch& b, int conv, int stage, int q, cudaStream_t st);
int launch_batch_cfl(const BatchLaunch& b, cudaStream_t st);
int launch_batch_vmax(const BatchLaunch& b, cudaStream_t st);   // per-tile maxima only
int launch_batch_dt(const BatchLaunch& b, cudaStream_t st);     // per-member dt from the maxima
int launch_batch_finish(const BatchLaunch& b, cudaStream_t st);

}  // namespace r3d
