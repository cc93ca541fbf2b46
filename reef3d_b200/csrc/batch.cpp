// Batched execution of many FP32 instances: one persistent launch per RK
// stage over a packed tile list of all members, the whole step captured in
// a CUDA graph and replayed, the tile shape and grid size picked by an
// autotuner whose choice is cached per size class.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "batch_internal.h"
#include "handle.h"

using namespace r3d;

struct r3d_batch {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    // the cell-kernel members run beside the tiled ones on this stream,
    // forked from and joined back into `stream` by the two events
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    std::vector<r3d_handle*> members;
    // device state, rebuilt when the membership or the configuration changes
    MemberDesc* d_members = nullptr;
    long long* d_tile0 = nullptr;
    TiledMember* d_tiled = nullptr;   // members on the tiled kernels come first
    CUtensorMap* d_maps = nullptr;    // 3 per tiled member
    size_t cap_tiled = 0;
    int n_tiled = 0;
    long long t_tiled = 0;            // items of the tiled members: tiles [0, t_tiled)
    double* d_vol = nullptr;
    double* d_vmax = nullptr;
    unsigned* d_work = nullptr;       // item counters of the persistent tiled launches
    size_t cap_members = 0, cap_tiles = 0;
    long long ntiles = 0;
    int max_f44 = 0;
    int rows = 4;
    int ctas_per_sm = 8;
    // tile configuration and z chunk of the tiled members' launches (the
    // batch encodes its own tensor maps of their fields for it)
    int tile_cfg = 0;
    bool tile_iso = false;  // every tiled member has cubic cells (tile_args_iso)
    int tile_kc = 16;
    bool tuned = false;  // rows/ctas set explicitly or by the autotuner
    bool dirty = true;
    bool use_graph = true;
    cudaGraphExec_t graph = nullptr;
    long long launches = 0;
    long long steps = 0;
    std::string err;
};

namespace {

thread_local std::string g_batch_err;

int bfail(r3d_batch* b, int code, const std::string& m) {
    if (b) b->err = m;
    else g_batch_err = m;
    return code;
}

#define B_CUDA(b, call)                                                                      \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) return bfail(b, R3D_EDEVICE, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

void drop_graph(r3d_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

MemberDesc describe(const r3d_handle* h) {
    MemberDesc m{};
    m.g = h->g32;
    m.phi = static_cast<float*>(h->field[R3D_PHI]);
    m.a1 = static_cast<float*>(h->field[R3D_WORK1]);
    m.a2 = static_cast<float*>(h->field[R3D_WORK2]);
    m.u = static_cast<const float*>(h->field[R3D_U]);
    m.v = static_cast<const float*>(h->field[R3D_V]);
    m.w = static_cast<const float*>(h->field[R3D_W]);
    m.dt = h->S.dt;
    m.vscale = h->S.vscale;
    m.t = h->S.t;
    m.vol = h->S.vol;
    m.n47 = h->desc.n47;
    m.dxmin = h->M.dxmin_cfl;
    m.period = h->period;
    m.f44 = h->desc.f44;
    return m;
}

bool on_tiles(const r3d_handle* h) { return h->tile_ok && h->use_tile; }

int rebuild(r3d_batch* b) {
    drop_graph(b);
    const size_t nm = b->members.size();
    // members on the tiled kernels first, the others after them
    std::vector<r3d_handle*> order;
    for (r3d_handle* h : b->members)
        if (on_tiles(h)) order.push_back(h);
    b->n_tiled = (int)order.size();
    for (r3d_handle* h : b->members)
        if (!on_tiles(h)) order.push_back(h);
    std::vector<MemberDesc> desc(nm);
    std::vector<long long> tile0(nm + 1, 0);
    std::vector<TiledMember> tiled(b->n_tiled);
    std::vector<CUtensorMap> maps(3 * (size_t)b->n_tiled);
    b->max_f44 = 0;
    bool iso = true;
    for (size_t q = 0; q < nm; ++q) {
        r3d_handle* h = order[q];
        desc[q] = describe(h);
        const bool t = (int)q < b->n_tiled;
        tile0[q + 1] = tile0[q] + (t ? tile_items_of(h->L, b->tile_kc, b->tile_cfg) : batch_tiles_of(h->L, b->rows));
        b->max_f44 = std::max(b->max_f44, h->desc.f44);
        if (t) {
            TiledMember& m = tiled[q];
            m.args = make_tile_args(h, 1);
            m.args.kc = b->tile_kc;
            iso = iso && tile_args_iso(m.args);
            m.phi = static_cast<float*>(h->field[R3D_PHI]);
            m.a1 = static_cast<float*>(h->field[R3D_WORK1]);
            m.a2 = static_cast<float*>(h->field[R3D_WORK2]);
            m.f44 = h->desc.f44;
            const float* src[3] = {m.phi, m.a1, m.a2};
            std::string why;
            for (int s = 0; s < 3; ++s)
                if (encode_plane_map(h->L, src[s], b->tile_cfg, &maps[3 * q + s], &why))
                    return bfail(b, R3D_EDEVICE, why);
        }
    }
    b->t_tiled = tile0[b->n_tiled];
    b->tile_iso = iso;
    b->ntiles = tile0[nm];
    if ((size_t)b->n_tiled > b->cap_tiled) {
        if (b->d_tiled) cudaFree(b->d_tiled);
        if (b->d_maps) cudaFree(b->d_maps);
        b->d_tiled = nullptr;
        b->d_maps = nullptr;
        const size_t cap = std::max<size_t>((size_t)b->n_tiled, 2 * b->cap_tiled);
        if (cudaMalloc(&b->d_tiled, cap * sizeof(TiledMember)) != cudaSuccess ||
            cudaMalloc(&b->d_maps, 3 * cap * sizeof(CUtensorMap)) != cudaSuccess) {
            cudaGetLastError();
            b->cap_tiled = 0;
            return bfail(b, R3D_ENOMEM, "batch tiled-member allocation failed");
        }
        b->cap_tiled = cap;
    }
    if (b->n_tiled) {
        B_CUDA(b, cudaMemcpyAsync(b->d_tiled, tiled.data(), tiled.size() * sizeof(TiledMember),
                                  cudaMemcpyHostToDevice, b->stream));
        B_CUDA(b, cudaMemcpyAsync(b->d_maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice,
                                  b->stream));
    }
    if (nm > b->cap_members) {
        if (b->d_members) cudaFree(b->d_members);
        if (b->d_tile0) cudaFree(b->d_tile0);
        b->d_members = nullptr;
        b->d_tile0 = nullptr;
        const size_t cap = std::max<size_t>(nm, 2 * b->cap_members);
        if (cudaMalloc(&b->d_members, cap * sizeof(MemberDesc)) != cudaSuccess ||
            cudaMalloc(&b->d_tile0, (cap + 1) * sizeof(long long)) != cudaSuccess) {
            cudaGetLastError();
            b->cap_members = 0;
            return bfail(b, R3D_ENOMEM, "batch descriptor allocation failed");
        }
        b->cap_members = cap;
    }
    if ((size_t)b->ntiles > b->cap_tiles) {
        if (b->d_vol) cudaFree(b->d_vol);
        if (b->d_vmax) cudaFree(b->d_vmax);
        b->d_vol = b->d_vmax = nullptr;
        const size_t cap = std::max<size_t>((size_t)b->ntiles, 2 * b->cap_tiles);
        if (cudaMalloc(&b->d_vol, cap * 2 * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&b->d_vmax, cap * 3 * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            b->cap_tiles = 0;
            return bfail(b, R3D_ENOMEM, "batch reduction scratch allocation failed");
        }
        b->cap_tiles = cap;
    }
    if (nm) {
        B_CUDA(b, cudaMemcpyAsync(b->d_members, desc.data(), nm * sizeof(MemberDesc), cudaMemcpyHostToDevice, b->stream));
        B_CUDA(b, cudaMemcpyAsync(b->d_tile0, tile0.data(), (nm + 1) * sizeof(long long), cudaMemcpyHostToDevice, b->stream));
        B_CUDA(b, cudaStreamSynchronize(b->stream));
    }
    b->dirty = false;
    return R3D_OK;
}

// All members (for the per-member reductions).
BatchLaunch launch_of(const r3d_batch* b) {
    BatchLaunch l{};
    l.members = b->d_members;
    l.tile0 = b->d_tile0;
    l.nm = (int)b->members.size();
    l.t_begin = 0;
    l.ntiles = b->ntiles;
    l.vol_part = b->d_vol;
    l.vmax_part = b->d_vmax;
    l.rows = b->rows;
    const long long want = (long long)b->ctas_per_sm * b->sms;
    l.grid = (unsigned)std::max<long long>(1, std::min<long long>(want, b->ntiles));
    return l;
}

// The members on the one-cell-per-thread kernels: tiles [t_tiled, ntiles).
BatchLaunch cell_launch_of(const r3d_batch* b) {
    BatchLaunch l = launch_of(b);
    l.members = b->d_members + b->n_tiled;
    l.tile0 = b->d_tile0 + b->n_tiled;
    l.nm = (int)b->members.size() - b->n_tiled;
    l.t_begin = b->t_tiled;
    return l;
}

unsigned tiled_grid(const r3d_batch* b) {
    const long long want = (long long)tile_ctas_per_sm(b->tile_cfg) * b->sms;  // the co-resident CTAs
    return (unsigned)std::max<long long>(1, std::min<long long>(want, b->t_tiled));
}

// Enqueues the tiled members' launch on the batch stream and the cell-kernel
// members' launch on the side stream, so the two (independent) groups run at
// the same time; the side stream forks from and joins back into the batch
// stream (also inside a graph capture).
template <typename T, typename C>
long long fork_join(r3d_batch* b, T tiled, C cells) {
    const bool has_t = b->n_tiled > 0, has_c = (size_t)b->n_tiled < b->members.size();
    if (has_t && has_c) {
        cudaEventRecord(b->fork, b->stream);
        cudaStreamWaitEvent(b->side, b->fork, 0);
        const long long n = cells(b->side) + tiled(b->stream);
        cudaEventRecord(b->join, b->side);
        cudaStreamWaitEvent(b->stream, b->join, 0);
        return n;
    }
    return (has_t ? tiled(b->stream) : 0) + (has_c ? cells(b->stream) : 0);
}

long long enqueue_stage(r3d_batch* b, bool reini, int s, int q) {
    return fork_join(
        b,
        [&](cudaStream_t st) {
            return (long long)launch_batch_tile_stage(b->d_tiled, b->d_maps, b->d_tile0, b->n_tiled, b->tile_cfg,
                                                      b->tile_iso, reini, s, q, b->d_vol, b->d_work, tiled_grid(b), st);
        },
        [&](cudaStream_t st) { return (long long)launch_batch_stage(cell_launch_of(b), reini ? 0 : 1, s, q, st); });
}

long long enqueue_vmax(r3d_batch* b) {
    return fork_join(
        b,
        [&](cudaStream_t st) {
            return (long long)launch_batch_tile_vmax(b->d_tiled, b->d_tile0, b->n_tiled, b->tile_cfg, b->d_vmax,
                                                     tiled_grid(b), st);
        },
        [&](cudaStream_t st) { return (long long)launch_batch_vmax(cell_launch_of(b), st); });
}

// CFL, 3 convection stages, max(f44) reinit pseudo-steps, volume + clock.
long long enqueue_batch_step(r3d_batch* b) {
    long long n = 0;
    n += enqueue_vmax(b);
    n += launch_batch_dt(launch_of(b), b->stream);
    for (int s = 1; s <= 3; ++s) n += enqueue_stage(b, false, s, 0);
    for (int q = 0; q < b->max_f44; ++q)
        for (int s = 1; s <= 3; ++s) n += enqueue_stage(b, true, s, q);
    n += launch_batch_finish(launch_of(b), b->stream);
    return n;
}

int capture(r3d_batch* b) {
    drop_graph(b);
    cudaGraph_t g = nullptr;
    B_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_batch_step(b);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess) return bfail(b, R3D_EDEVICE, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->graph = nullptr;
        return bfail(b, R3D_EDEVICE, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    return R3D_OK;
}

// ---------------------------------------------------------------- autotuner
std::mutex g_tune_mu;
// size class -> (rows, CTAs per SM, tile configuration, z chunk) of a
// batch, or (convection tile configuration, chunk, reinitialisation tile
// configuration, chunk) of an instance ("inst-" keys)
std::map<std::string, std::vector<int>> g_tune_cache;

std::string size_class(const r3d_batch* b) {
    double c3 = 0, c2 = 0;
    for (const r3d_handle* h : b->members) {
        const double c = (double)h->L.nx * h->L.ny * h->L.nz;
        (h->L.two_d ? c2 : c3) += c;
    }
    const double tot = c2 + c3;
    std::ostringstream os;
    os << (c3 >= c2 ? "3d" : "2d") << "-c" << (int)std::floor(std::log2(std::max(1.0, tot))) << "-m"
       << (int)std::floor(std::log2(std::max<size_t>(1, b->members.size())));
    return os.str();
}

// One line per size class: the key and four integers.
void load_cache(const char* path) {
    if (!path || !*path) return;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        std::string key;
        std::vector<int> v(4, 0);
        if (is >> key >> v[0] >> v[1] >> v[2] >> v[3]) g_tune_cache[key] = v;
    }
}

void save_cache(const char* path) {
    if (!path || !*path) return;
    std::ofstream f(path, std::ios::trunc);
    for (auto& kv : g_tune_cache) {
        f << kv.first;
        for (int x : kv.second) f << " " << x;
        f << "\n";
    }
}

// The z chunks and the (tile configuration, z chunk) candidates of the
// autotuners.
constexpr int kChunks[] = {6, 7, 8, 10, 12, 16, 32};

std::vector<std::pair<int, int>> tile_candidates() {
    std::vector<std::pair<int, int>> out;
    for (int c = 0; c < tile_cfg_count(); ++c)
        for (int kc : kChunks) out.push_back({c, kc});
    return out;
}

}  // namespace

extern "C" {

int r3d_tile_chunk_candidates(int* out, int max) {
    const int n = (int)(sizeof(kChunks) / sizeof(kChunks[0]));
    for (int q = 0; q < n && q < max && out; ++q) out[q] = kChunks[q];
    return n;
}

const char* r3d_batch_last_error(const r3d_batch* b) { return b ? b->err.c_str() : g_batch_err.c_str(); }

int r3d_batch_create(r3d_batch** out) {
    if (!out) return bfail(nullptr, R3D_EINVAL, "null output");
    *out = nullptr;
    r3d_batch* b = new (std::nothrow) r3d_batch();
    if (!b) return bfail(nullptr, R3D_ENOMEM, "host allocation failed");
    cudaGetDevice(&b->device);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    if (cudaMalloc(&b->d_work, 4 * sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(b->d_work, 0, 4 * sizeof(unsigned)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (b->join) cudaEventDestroy(b->join);
        if (b->fork) cudaEventDestroy(b->fork);
        if (b->side) cudaStreamDestroy(b->side);
        if (b->stream) cudaStreamDestroy(b->stream);
        if (b->d_work) cudaFree(b->d_work);
        delete b;
        return bfail(nullptr, R3D_EDEVICE, "stream creation failed");
    }
    *out = b;
    return R3D_OK;
}

int r3d_batch_destroy(r3d_batch* b) {
    if (!b) return R3D_OK;
    cudaStreamSynchronize(b->stream);
    for (r3d_handle* h : b->members) h->batch_stream = nullptr;
    drop_graph(b);
    if (b->d_members) cudaFree(b->d_members);
    if (b->d_tile0) cudaFree(b->d_tile0);
    if (b->d_vol) cudaFree(b->d_vol);
    if (b->d_vmax) cudaFree(b->d_vmax);
    if (b->d_tiled) cudaFree(b->d_tiled);
    if (b->d_maps) cudaFree(b->d_maps);
    cudaStreamSynchronize(b->side);
    cudaEventDestroy(b->join);
    cudaEventDestroy(b->fork);
    cudaStreamDestroy(b->side);
    cudaStreamDestroy(b->stream);
    cudaFree(b->d_work);
    delete b;
    return R3D_OK;
}

int r3d_batch_add(r3d_batch* b, r3d_handle* h) {
    if (!b || !h) return bfail(b, R3D_EINVAL, "null argument");
    if (h->desc.precision != R3D_FP32) return bfail(b, R3D_EINVAL, "batches hold FP32 instances");
    if (h->desc.f46 != 0) return bfail(b, R3D_EINVAL, "batches hold instances without picard mass correction (f46 = 0)");
    if (h->fluid) return bfail(b, R3D_EINVAL, "batches hold instances without the fluid update");
    if (h->airy) return bfail(b, R3D_EINVAL, "batches hold instances without the Airy velocity generator");
    if (h->io || h->L.io) return bfail(b, R3D_EINVAL, "batches hold closed-box instances (no inflow/outflow or halo faces)");
    if (h->g64.x45 || h->sf_ops) return bfail(b, R3D_EINVAL, "batches hold instances without direct or solid forcing");
    if (h->device != b->device) return bfail(b, R3D_EINVAL, "instance lives on another device");
    if (h->batch_stream) return bfail(b, R3D_ESTATE, "instance already in a batch");
    // the member's own queued work (uploads, settings) completes first
    B_CUDA(b, cudaStreamSynchronize(h->stream));
    b->members.push_back(h);
    h->batch_stream = b->stream;
    b->dirty = true;
    return R3D_OK;
}

int r3d_batch_remove(r3d_batch* b, r3d_handle* h) {
    if (!b || !h) return bfail(b, R3D_EINVAL, "null argument");
    auto it = std::find(b->members.begin(), b->members.end(), h);
    if (it == b->members.end()) return bfail(b, R3D_EINVAL, "not a member");
    B_CUDA(b, cudaStreamSynchronize(b->stream));
    b->members.erase(it);
    h->batch_stream = nullptr;
    b->dirty = true;
    return R3D_OK;
}

int r3d_batch_size(const r3d_batch* b, int* n) {
    if (!b || !n) return bfail(nullptr, R3D_EINVAL, "null argument");
    *n = (int)b->members.size();
    return R3D_OK;
}

int r3d_batch_set_config(r3d_batch* b, int rows, int ctas_per_sm) {
    if (!b) return bfail(nullptr, R3D_EINVAL, "null batch");
    if (rows != 2 && rows != 4 && rows != 8) return bfail(b, R3D_EINVAL, "rows must be 2, 4 or 8");
    if (ctas_per_sm < 1 || ctas_per_sm * 32 * rows > 2048) return bfail(b, R3D_EINVAL, "ctas_per_sm out of range");
    b->rows = rows;
    b->ctas_per_sm = ctas_per_sm;
    b->tuned = true;
    b->dirty = true;
    return R3D_OK;
}

int r3d_batch_get_config(const r3d_batch* b, int* rows, int* ctas_per_sm) {
    if (!b || !rows || !ctas_per_sm) return bfail(nullptr, R3D_EINVAL, "null argument");
    *rows = b->rows;
    *ctas_per_sm = b->ctas_per_sm;
    return R3D_OK;
}

int r3d_batch_use_graph(r3d_batch* b, int on) {
    if (!b) return bfail(nullptr, R3D_EINVAL, "null batch");
    b->use_graph = on != 0;
    drop_graph(b);
    return R3D_OK;
}

int r3d_batch_set_tile_config(r3d_batch* b, int cfg, int kc) {
    if (!b) return bfail(nullptr, R3D_EINVAL, "null batch");
    if (cfg < 0 || cfg >= tile_cfg_count()) return bfail(b, R3D_EINVAL, "unknown tile configuration");
    if (kc < 1 || kc > 4096) return bfail(b, R3D_EINVAL, "chunk must be 1..4096 planes");
    b->tile_cfg = cfg;
    b->tile_kc = kc;
    b->dirty = true;
    drop_graph(b);
    return R3D_OK;
}

int r3d_batch_get_tile_config(const r3d_batch* b, int* cfg, int* kc) {
    if (!b || !cfg || !kc) return bfail(nullptr, R3D_EINVAL, "null argument");
    *cfg = b->tile_cfg;
    *kc = b->tile_kc;
    return R3D_OK;
}

// Picks the tiled members' (tile configuration, z chunk) and the cell
// members' (rows, CTAs per SM) for the batch's size class by timing the
// first convection and reinitialisation stages (they write only the stage
// buffer WORK1, so the members' state is untouched): first the tile
// configurations with the cell members at their current choice, then the
// cell choices with the best tile configuration.  The choice is cached per
// size class in memory and in `cache_path` (a text file; may be NULL).
int r3d_batch_autotune(r3d_batch* b, const char* cache_path, int* rows_out, int* ctas_out) {
    if (!b) return bfail(nullptr, R3D_EINVAL, "null batch");
    if (b->members.empty()) return bfail(b, R3D_ESTATE, "empty batch");
    const std::string key = size_class(b);
    auto finish = [&](int r, int c, int cfg, int kc) {
        int rc = r3d_batch_set_config(b, r, c);
        if (!rc) rc = r3d_batch_set_tile_config(b, cfg, kc);
        if (rows_out) *rows_out = b->rows;
        if (ctas_out) *ctas_out = b->ctas_per_sm;
        return rc;
    };
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        if (g_tune_cache.empty()) load_cache(cache_path);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end() && it->second.size() == 4 && it->second[2] < tile_cfg_count() &&
            it->second[3] > 0)
            return finish(it->second[0], it->second[1], it->second[2], it->second[3]);
    }
    cudaEvent_t e0, e1;
    B_CUDA(b, cudaEventCreate(&e0));
    B_CUDA(b, cudaEventCreate(&e1));
    // the stages read dt: give every member a valid one first
    b->rows = 4;
    b->ctas_per_sm = 8;
    b->tile_cfg = 0;
    b->tile_kc = 16;
    if (int rc = rebuild(b)) return rc;
    enqueue_vmax(b);
    launch_batch_dt(launch_of(b), b->stream);
    int err = R3D_OK;
    auto time_now = [&]() -> float {
        if (int rc = rebuild(b)) {
            err = rc;
            return 1e30f;
        }
        enqueue_stage(b, false, 1, 0);  // warm
        cudaEventRecord(e0, b->stream);
        for (int rep = 0; rep < 3; ++rep) {
            enqueue_stage(b, false, 1, 0);
            enqueue_stage(b, true, 1, 0);
        }
        cudaEventRecord(e1, b->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            err = bfail(b, R3D_EDEVICE, "autotune timing");
            return 1e30f;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms;
    };
    float best = 1e30f;
    int bcfg = 0, bkc = 16;
    if (b->n_tiled > 0)
        for (auto [cfg, kc] : tile_candidates()) {
            b->tile_cfg = cfg;
            b->tile_kc = kc;
            const float ms = time_now();
            if (err) break;
            if (ms < best) { best = ms; bcfg = cfg; bkc = kc; }
        }
    b->tile_cfg = bcfg;
    b->tile_kc = bkc;
    best = 1e30f;
    int br = 4, bc = 8;
    const int cand_rows[3] = {2, 4, 8};
    const int cand_ctas[4] = {4, 8, 16, 32};
    if (!err && (size_t)b->n_tiled < b->members.size())
        for (int r : cand_rows)
            for (int c : cand_ctas) {
                if (c * 32 * r > 2048) continue;
                b->rows = r;
                b->ctas_per_sm = c;
                const float ms = time_now();
                if (err) break;
                if (ms < best) { best = ms; br = r; bc = c; }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err) return err;
    B_CUDA(b, cudaGetLastError());
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = {br, bc, bcfg, bkc};
        save_cache(cache_path);
    }
    return finish(br, bc, bcfg, bkc);
}

// Picks the tile configuration and z chunk of one instance on the tiled
// path for its grid size, for the convection and the reinitialisation
// stages separately, by timing stage 2 of each kind under every candidate
// (stage 2 reads phi and WORK1 and writes only WORK2, so the level set is
// untouched), and caches the choice per grid size like r3d_batch_autotune
// (cache line: key, convection configuration and chunk, reinitialisation
// configuration and chunk).
int r3d_autotune(r3d_handle* h, const char* cache_path, int* cfg_out, int* kc_out) {
    if (!h) return R3D_EINVAL;
    int on = 0;
    if (int rc = r3d_get_option(h, R3D_OPT_TILED, &on)) return rc;
    auto report = [&]() {
        if (cfg_out) *cfg_out = h->tile_cfg;
        if (kc_out) *kc_out = h->kc;
    };
    if (!on) {  // not on the tiled kernels: nothing to choose
        report();
        return R3D_OK;
    }
    std::ostringstream os;
    os << "inst-" << h->L.nx << "x" << h->L.ny << "x" << h->L.nz;
    const std::string key = os.str();
    auto finish = [&](int c, int k, int cr, int kr) {
        int rc = r3d_set_option(h, R3D_OPT_TILE_CFG, c);
        if (!rc) rc = r3d_set_option(h, R3D_OPT_CHUNK, k);
        if (!rc) rc = r3d_set_option(h, R3D_OPT_TILE_CFG_REINIT, cr);
        if (!rc) rc = r3d_set_option(h, R3D_OPT_CHUNK_REINIT, kr);
        report();
        return rc;
    };
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        if (g_tune_cache.empty()) load_cache(cache_path);
        auto it = g_tune_cache.find(key);
        const int n = tile_cfg_count();
        if (it != g_tune_cache.end() && it->second.size() == 4 && it->second[0] < n && it->second[2] < n &&
            it->second[1] > 0 && it->second[3] > 0)
            return finish(it->second[0], it->second[1], it->second[2], it->second[3]);
    }
    double dt = 0.0;
    if (int rc = r3d_cfl_dt(h, &dt)) return rc;
    if (int rc = r3d_set_dt(h, dt)) return rc;
    const int c0 = h->tile_cfg, k0 = h->kc, cr0 = h->tile_cfg_r, kr0 = h->kc_r;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return R3D_EDEVICE;
    int rc = R3D_OK;
    // ms per launch of one kind under (cfg, kc), timed over pairs of stage 1
    // and stage 2 as a step runs them (stage 2 reading the output stage 1
    // just wrote; the level set itself, which stage 3 writes, is left as it
    // is); < 0: not tiled
    auto time_stage = [&](int cfg, int kc, int kind, int reps) -> float {
        if ((rc = r3d_set_option(h, R3D_OPT_TILE_CFG, cfg)) || (rc = r3d_set_option(h, R3D_OPT_CHUNK, kc)))
            return -1.f;
        if ((rc = r3d_get_option(h, R3D_OPT_TILED, &on)) || !on) return -1.f;  // e.g. more items than scratch
        const int st = kind ? R3D_STAGE_REINIT : R3D_STAGE_CONVECTION;
        if ((rc = r3d_stage(h, st, 1)) || (rc = r3d_stage(h, st, 2))) return -1.f;  // warm
        cudaEventRecord(e0, h->stream);
        for (int rep = 0; rep < reps && !rc; ++rep)
            if (!(rc = r3d_stage(h, st, 1))) rc = r3d_stage(h, st, 2);
        cudaEventRecord(e1, h->stream);
        if (rc || cudaEventSynchronize(e1) != cudaSuccess) {
            if (!rc) rc = R3D_EDEVICE;
            return -1.f;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms / (2 * reps);
    };
    // a sweep of every candidate, then the three fastest of each kind timed
    // again, longer and interleaved, so that run-to-run noise of a few per
    // cent does not pick a slower configuration
    std::vector<std::tuple<float, int, int>> seen[2];
    for (auto [cfg, kc] : tile_candidates()) {
        for (int kind = 0; kind < 2 && !rc; ++kind) {
            const float ms = time_stage(cfg, kc, kind, 5);
            if (ms >= 0.f) seen[kind].emplace_back(ms, cfg, kc);
        }
        if (rc) break;
    }
    float best[2] = {1e30f, 1e30f};
    int bc[2] = {c0, cr0}, bk[2] = {k0, kr0};
    for (int kind = 0; kind < 2 && !rc; ++kind) {
        std::sort(seen[kind].begin(), seen[kind].end());
        const size_t top = std::min<size_t>(3, seen[kind].size());
        std::vector<float> t(top, 1e30f);
        for (int round = 0; round < 3 && !rc; ++round)
            for (size_t q = 0; q < top && !rc; ++q) {
                const float ms = time_stage(std::get<1>(seen[kind][q]), std::get<2>(seen[kind][q]), kind, 10);
                if (ms >= 0.f) t[q] = std::min(t[q], ms);
            }
        for (size_t q = 0; q < top; ++q)
            if (t[q] < best[kind]) {
                best[kind] = t[q];
                bc[kind] = std::get<1>(seen[kind][q]);
                bk[kind] = std::get<2>(seen[kind][q]);
            }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) {
        finish(c0, k0, cr0, kr0);
        return rc;
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = {bc[0], bk[0], bc[1], bk[1]};
        save_cache(cache_path);
    }
    return finish(bc[0], bk[0], bc[1], bk[1]);
}

// nsteps physical steps of every member: per member the CFL time step from
// its velocities, the three convection stages, its f44 reinitialisation
// pseudo-steps, the volume integral and its clock (src/levelset_RK3.cpp
// for every member at once).  Asynchronous on the batch's stream.
int r3d_batch_step(r3d_batch* b, int nsteps) {
    if (!b) return bfail(nullptr, R3D_EINVAL, "null batch");
    if (nsteps < 0) return bfail(b, R3D_EINVAL, "nsteps must be >= 0");
    if (b->members.empty() || nsteps == 0) return R3D_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != b->device) cudaSetDevice(b->device);
    int rc = R3D_OK;
    if (b->dirty) rc = rebuild(b);
    if (!rc && b->use_graph && !b->graph) rc = capture(b);
    if (!rc) {
        for (int s = 0; s < nsteps; ++s) {
            if (b->graph) {
                if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) {
                    rc = bfail(b, R3D_EDEVICE, "graph launch failed");
                    break;
                }
            } else {
                b->launches += enqueue_batch_step(b) - 0;
            }
        }
        if (!rc) {
            if (b->graph) {
                const int kinds = (b->n_tiled ? 1 : 0) + ((size_t)b->n_tiled < b->members.size() ? 1 : 0);
                const long long per = kinds + 1 + kinds * (3 + 3 * b->max_f44) + 1;
                b->launches += per * nsteps;
            }
            b->steps += nsteps;
            for (r3d_handle* h : b->members) h->have_last_volume = true;
        }
    }
    cudaError_t e = cudaGetLastError();
    if (!rc && e != cudaSuccess) rc = bfail(b, R3D_EDEVICE, cudaGetErrorString(e));
    if (cur != b->device) cudaSetDevice(cur);
    return rc;
}

int r3d_batch_sync(r3d_batch* b) {
    if (!b) return bfail(nullptr, R3D_EINVAL, "null batch");
    B_CUDA(b, cudaStreamSynchronize(b->stream));
    return R3D_OK;
}

int r3d_batch_stream(r3d_batch* b, void** stream) {
    if (!b || !stream) return bfail(b, R3D_EINVAL, "null argument");
    *stream = (void*)b->stream;
    return R3D_OK;
}

int r3d_batch_launch_count(const r3d_batch* b, long long* count) {
    if (!b || !count) return bfail(nullptr, R3D_EINVAL, "null argument");
    *count = b->launches;
    return R3D_OK;
}

}  // extern "C"
