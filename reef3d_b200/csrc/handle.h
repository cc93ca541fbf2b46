// The instance handle behind the C-ABI (shared by api.cpp and batch.cpp).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "reef3d_b200.h"
#include "r3d_internal.h"
#include "tile_host.h"

struct r3d_handle {
    r3d::Layout L{};
    r3d_grid_desc desc{};
    r3d::HostMetrics M;
    int device = 0;
    cudaStream_t stream = nullptr;
    // fields 0..6 always; 7 (ro) and 8 (visc) once r3d_set_fluid enabled
    // them, 9 (body) once r3d_set_direct_forcing did
    void* field[10] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    bool fluid = false;
    r3d::FluidConst fc{};
    // Airy wave velocity regenerated at the device clock before every step
    bool airy = false;
    r3d::AiryParams ap{};
    double* coord = nullptr;  // x centres, x faces, z centres, z faces
    // inflow / outflow faces with ioflow_f's hooks (r3d_set_ioflow)
    bool io = false;
    bool domain_slab = false;  // a slab of an r3d_domain (its io levels are the grid's)
    r3d_ioflow_desc iod{};
    double* io_buf = nullptr;  // hook state, ZP, ramp table (r3d::IoParams)
    size_t io_buf_len = 0;
    r3d::IoParams iop{};
    long long next_count = 1;  // lexer::count of the next step, for r3d_set_ioflow's first state
    // relaxation zones after each convection stage (r3d_set_relaxation)
    bool relax = false;
    int* rz_col = nullptr;       // 4 ints per zone column
    double* rz_buf = nullptr;    // weights (2 per column), z centres (nz), ramp (1), targets
    int rz_ncol = 0;
    long long rz_ntarget = 0;    // generation targets: nz x generation columns
    double rz_phimean = 0.0;
    // solid forcing after each convection stage (r3d_set_solid_forcing)
    long long* sf_ops = nullptr;     // device: (entry cell, two target cells) per op, by level
    std::vector<int> sf_levels;      // op offsets of the dependency levels
    int sms = 148;
    double* metrics64 = nullptr;
    float* metrics32 = nullptr;
    r3d::KGrid<double> g64{};
    r3d::KGrid<float> g32{};
    r3d::Scratch S{};
    double* staging = nullptr;
    size_t staging_bytes = 0;
    long long launches = 0;
    double dt_host = 0.0;
    double period = 0.0;
    bool have_last_volume = false;
    // TMA-tiled FP32 path (3D uniform grids)
    bool tile_ok = false;
    int use_tile = 1;
    // tile configuration (shape, rows per thread, ring depth) and z chunk of
    // the convection stages; *_r: of the reinitialisation stages
    int kc = 16;
    int tile_cfg = 0;
    int kc_r = 16;
    int tile_cfg_r = 0;
    int band64 = 1;
    int wait_test = 0;  // R3D_OPT_WAIT_TEST: armed for the next r3d_ls_step
    CUtensorMap map[3];    // stage inputs phi, WORK1, WORK2 for tile_cfg
    CUtensorMap map_r[3];  // the same for tile_cfg_r
    // set while the instance is a member of a batch: calls on the handle
    // first wait for the batch's stream
    cudaStream_t batch_stream = nullptr;
    // one captured step (CFL when adaptive + the step) replayed by r3d_ls_run;
    // rebuilt when anything baked into it changes
    cudaGraphExec_t step_graph = nullptr;
    long long graph_key = -1;
    // bumped whenever something a captured step bakes in changes (kernel
    // arguments by value, device pointers, options): graphs that hold this
    // instance's work (its own step graph, a slab domain's) compare it
    unsigned long long config_gen = 0;
    long long graph_launches = 0;
    std::string err;
};

namespace r3d {
TileArgs make_tile_args(r3d_handle* h, int stage);
}
