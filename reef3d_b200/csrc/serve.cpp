// Continuous-batching job server behind the C-ABI (r3d_serve_*): transport
// jobs wait in arrival order until their device footprint fits the HBM
// budget, every admitted job stays resident on the device, and all active
// jobs advance together -- FP32 jobs as members of one batch (one persistent
// launch per RK stage over every member, the step replayed from a CUDA
// graph), FP64 jobs each on its own instance.  Jobs join and leave between
// steps; a job's result does not depend on which others shared its steps.
#include <cuda_runtime.h>

#include "reef3d_b200.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <map>
#include <new>
#include <string>
#include <vector>

struct r3d_server {
    struct Job {
        int nx, ny, nz, steps, f44;
        double n47;
        std::vector<double> spheres, modes;
        r3d_handle* h = nullptr;
        int done_steps = 0;
        int state = 0;  // 0 queued, 1 active, 2 finished, 3 released
        size_t bytes = 0;
        double t_submit = 0.0, t_admit = -1.0, t_done = -1.0;
        double volume[2] = {0.0, 0.0};
        double time = 0.0;
    };
    double budget = 0.0;
    int precision = R3D_FP32;
    int keep = 0;
    r3d_batch* batch = nullptr;
    double used = 0.0, peak = 0.0;
    int max_active = 0;
    long long next_id = 0;
    std::map<long long, Job> jobs;
    std::deque<long long> queue;
    std::vector<long long> active;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::string err;
    // the batch stream's progress at the end of each of the last two polls:
    // a poll returns once the work of the poll before it is done, so the
    // host runs at most one poll ahead of the device and jobs that arrive
    // meanwhile are admitted at the next step, not after a long queue of
    // steps already issued for the jobs before them
    cudaEvent_t done_ev[2] = {nullptr, nullptr};
    int ev_next = 0;
    bool ev_pending[2] = {false, false};

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

int sfail(r3d_server* s, int code, const std::string& m) {
    if (s) s->err = m;
    return code;
}

std::vector<double> nodes(int n) {
    // x_i = i / n for node indices -5..n+5, as a DIVEMesh grid of the unit box
    std::vector<double> x;
    const double h = 1.0 / n;
    for (int i = -5; i <= n + 5; ++i) x.push_back(i * h);
    return x;
}

r3d_grid_desc job_desc(const r3d_server::Job& j, int precision, std::vector<double>* xs) {
    xs[0] = nodes(j.nx);
    xs[1] = nodes(j.ny);
    xs[2] = nodes(j.nz);
    r3d_grid_desc d{};
    d.nx = j.nx;
    d.ny = j.ny;
    d.nz = j.nz;
    d.xn = xs[0].data();
    d.yn = xs[1].data();
    d.zn = xs[2].data();
    d.f43 = 0.5;
    d.f44 = j.f44;
    d.f45 = 2.1;
    d.f49 = 1;
    d.n47 = j.n47;
    d.precision = precision;
    return d;
}

int admit(r3d_server* s, long long id) {
    r3d_server::Job& j = s->jobs[id];
    std::vector<double> xs[3];
    const r3d_grid_desc d = job_desc(j, s->precision, xs);
    r3d_handle* h = nullptr;
    if (int rc = r3d_create(&d, &h)) return sfail(s, rc, std::string("job instance: ") + r3d_last_error(nullptr));
    int rc = r3d_init_spheres_tg(h, (int)(j.spheres.size() / 4), j.spheres.data(), (int)(j.modes.size() / 2),
                                 j.modes.data());
    if (!rc) rc = r3d_set_time(h, 0.0);
    if (!rc && s->batch) rc = r3d_batch_add(s->batch, h);
    if (rc) {
        const std::string m = s->batch && rc == R3D_EINVAL ? r3d_batch_last_error(s->batch) : r3d_last_error(h);
        r3d_destroy(h);
        return sfail(s, rc, "admitting a job: " + m);
    }
    j.h = h;
    j.state = 1;
    j.t_admit = s->now();
    s->used += (double)j.bytes;
    s->peak = std::max(s->peak, s->used);
    s->active.push_back(id);
    s->max_active = std::max(s->max_active, (int)s->active.size());
    return R3D_OK;
}

int retire(r3d_server* s, long long id) {
    r3d_server::Job& j = s->jobs[id];
    if (s->batch) {
        if (int rc = r3d_batch_remove(s->batch, j.h)) return sfail(s, rc, r3d_batch_last_error(s->batch));
    }
    if (int rc = r3d_last_volume(j.h, &j.volume[0], &j.volume[1])) return sfail(s, rc, r3d_last_error(j.h));
    if (int rc = r3d_get_time(j.h, &j.time)) return sfail(s, rc, r3d_last_error(j.h));
    j.t_done = s->now();
    j.state = 2;
    s->used -= (double)j.bytes;
    if (!s->keep) {
        r3d_destroy(j.h);
        j.h = nullptr;
    }
    return R3D_OK;
}

}  // namespace

extern "C" {

int r3d_serve_create(double budget_bytes, int precision, int keep_fields, r3d_server** out) {
    if (!out || !(budget_bytes > 0.0) || (precision != R3D_FP32 && precision != R3D_FP64))
        return R3D_EINVAL;
    r3d_server* s = new (std::nothrow) r3d_server();
    if (!s) return R3D_ENOMEM;
    s->budget = budget_bytes;
    s->precision = precision;
    s->keep = keep_fields ? 1 : 0;
    if (precision == R3D_FP32) {
        int rc = r3d_batch_create(&s->batch);
        if (!rc) rc = r3d_batch_use_graph(s->batch, 1);
        if (rc) {
            if (s->batch) r3d_batch_destroy(s->batch);
            delete s;
            return rc;
        }
    }
    *out = s;
    return R3D_OK;
}

int r3d_serve_destroy(r3d_server* s) {
    if (!s) return R3D_EINVAL;
    for (auto& kv : s->jobs)
        if (kv.second.h) {
            if (s->batch && kv.second.state == 1) r3d_batch_remove(s->batch, kv.second.h);
            r3d_destroy(kv.second.h);
        }
    if (s->batch) r3d_batch_destroy(s->batch);
    for (cudaEvent_t ev : s->done_ev)
        if (ev) cudaEventDestroy(ev);
    delete s;
    return R3D_OK;
}

const char* r3d_serve_last_error(const r3d_server* s) { return s ? s->err.c_str() : ""; }

int r3d_serve_submit(r3d_server* s, const r3d_job_desc* job, long long* id) {
    if (!s || !job || !id) return sfail(s, R3D_EINVAL, "null argument");
    if (job->nx < 1 || job->ny < 1 || job->nz < 1 || job->steps < 1 || job->f44 < 0 || !(job->n47 > 0.0) ||
        job->nspheres < 1 || job->nspheres > 64 || !job->spheres || job->nmodes < 0 || job->nmodes > 64 ||
        (job->nmodes && !job->modes))
        return sfail(s, R3D_EINVAL, "bad job description");
    r3d_server::Job j;
    j.nx = job->nx;
    j.ny = job->ny;
    j.nz = job->nz;
    j.steps = job->steps;
    j.f44 = job->f44;
    j.n47 = job->n47;
    j.spheres.assign(job->spheres, job->spheres + 4 * job->nspheres);
    if (job->nmodes) j.modes.assign(job->modes, job->modes + 2 * job->nmodes);
    std::vector<double> xs[3];
    const r3d_grid_desc d = job_desc(j, s->precision, xs);
    if (int rc = r3d_footprint(&d, &j.bytes)) return sfail(s, rc, r3d_last_error(nullptr));
    if ((double)j.bytes > s->budget) return sfail(s, R3D_ENOMEM, "the job alone exceeds the HBM budget");
    j.t_submit = s->now();
    *id = s->next_id++;
    s->jobs.emplace(*id, std::move(j));
    s->queue.push_back(*id);
    return R3D_OK;
}

int r3d_serve_poll(r3d_server* s, int max_steps, int* nfinished) {
    if (!s || max_steps < 0) return sfail(s, R3D_EINVAL, "bad argument");
    if (nfinished) *nfinished = 0;
    // admission in arrival order while the head of the queue fits
    while (!s->queue.empty() && s->used + (double)s->jobs[s->queue.front()].bytes <= s->budget) {
        const long long id = s->queue.front();
        s->queue.pop_front();
        if (int rc = admit(s, id)) return rc;
    }
    if (s->active.empty() || max_steps == 0) return R3D_OK;
    // advance up to max_steps, stopping at the first job that completes
    int n = max_steps;
    for (long long id : s->active) n = std::min(n, s->jobs[id].steps - s->jobs[id].done_steps);
    if (s->batch) {
        if (int rc = r3d_batch_step(s->batch, n)) return sfail(s, rc, r3d_batch_last_error(s->batch));
        void* st = nullptr;
        r3d_batch_stream(s->batch, &st);
        cudaEvent_t& ev = s->done_ev[s->ev_next];
        if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
            return sfail(s, R3D_EDEVICE, "event creation failed");
        if (cudaEventRecord(ev, (cudaStream_t)st) != cudaSuccess) return sfail(s, R3D_EDEVICE, "event record failed");
        s->ev_pending[s->ev_next] = true;
        s->ev_next ^= 1;
        // the previous poll's work
        if (s->ev_pending[s->ev_next]) {
            if (cudaEventSynchronize(s->done_ev[s->ev_next]) != cudaSuccess)
                return sfail(s, R3D_EDEVICE, "batch step failed on the device");
            s->ev_pending[s->ev_next] = false;
        }
    } else {
        for (long long id : s->active)
            if (int rc = r3d_ls_run(s->jobs[id].h, n, 1)) return sfail(s, rc, r3d_last_error(s->jobs[id].h));
        // FP64 steps take milliseconds each: wait for this poll's (the
        // instances run on their own streams)
        for (long long id : s->active)
            if (int rc = r3d_sync(s->jobs[id].h)) return sfail(s, rc, r3d_last_error(s->jobs[id].h));
    }
    std::vector<long long> still;
    int fin = 0;
    for (long long id : s->active) {
        r3d_server::Job& j = s->jobs[id];
        j.done_steps += n;
        if (j.done_steps >= j.steps) {
            if (int rc = retire(s, id)) return rc;
            ++fin;
        } else {
            still.push_back(id);
        }
    }
    s->active.swap(still);
    if (nfinished) *nfinished = fin;
    return R3D_OK;
}

int r3d_serve_status(const r3d_server* s, int* queued, int* active, double* used_bytes, double* peak_bytes,
                     int* max_active) {
    if (!s) return R3D_EINVAL;
    if (queued) *queued = (int)s->queue.size();
    if (active) *active = (int)s->active.size();
    if (used_bytes) *used_bytes = s->used;
    if (peak_bytes) *peak_bytes = s->peak;
    if (max_active) *max_active = s->max_active;
    return R3D_OK;
}

int r3d_serve_result(const r3d_server* s, long long id, r3d_job_result* out) {
    if (!s || !out) return R3D_EINVAL;
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return R3D_EINVAL;
    const r3d_server::Job& j = it->second;
    out->state = j.state;
    out->steps_done = j.done_steps;
    out->volume1 = j.volume[0];
    out->volume2 = j.volume[1];
    out->sim_time = j.time;
    out->t_submit = j.t_submit;
    out->t_admit = j.t_admit;
    out->t_done = j.t_done;
    out->instance = j.h;
    return R3D_OK;
}

int r3d_serve_batch(r3d_server* s, r3d_batch** batch) {
    if (!s || !batch) return R3D_EINVAL;
    *batch = s->batch;
    return R3D_OK;
}

int r3d_serve_release(r3d_server* s, long long id) {
    if (!s) return R3D_EINVAL;
    auto it = s->jobs.find(id);
    if (it == s->jobs.end() || it->second.state != 2) return sfail(s, R3D_ESTATE, "not a finished job");
    if (it->second.h) r3d_destroy(it->second.h);
    it->second.h = nullptr;
    it->second.state = 3;
    return R3D_OK;
}

}  // extern "C"
