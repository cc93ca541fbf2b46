"""Continuous-batching server for level-set transport jobs.

Jobs (a sphere-union level set advected by a Taylor-Green velocity for a
given number of steps) arrive over time.  The native serving runtime
(r3d_serve_*, reef3d_b200/csrc/serve.cpp) admits waiting jobs in arrival
order whenever their device footprint fits the HBM budget, keeps every
admitted job's fields resident on the device, and advances all active jobs
together in one batch (one persistent launch per RK stage over every
member, the step replayed from a CUDA graph).  Jobs join and leave between
steps, so work of jobs that arrive while others are on the GPU overlaps
with theirs on the device.  A job's result does not depend on which other
jobs shared its steps.  ``TransportServer`` feeds it a timed job stream.

The FP64 plain path (``precision=FP64``) serves the same stream without
batching: every active job is stepped on its own instance.
"""
import collections
import ctypes
import math
import os
import time

import numpy as np

from . import FP32, FP64, LAYOUT_REEF3D, PHI, R3D_OK, JobDesc, JobResult, R3DError, _check, _dp, load_library

_lib = None  # the loaded libreef3d_b200.so (set by TransportServer)


class Job:
    """One transport job."""

    def __init__(self, jid, edges, spheres, modes, steps, arrival, f44=2, cfl=0.25):
        self.id = jid
        self.nx, self.ny, self.nz = edges
        self.spheres = spheres
        self.modes = modes
        self.steps = steps
        self.arrival = arrival
        self.f44 = f44
        self.n47 = cfl / 2.0
        self.t_admit = None
        self.t_done = None
        self.volume = None
        self.time = None
        self.phi = None

    @property
    def cells(self):
        return self.nx * self.ny * self.nz

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.arrival


def poisson_jobs(seed=1, rate=200.0, njobs=64, edge_lo=32, edge_hi=384, steps_lo=50, steps_hi=500):
    """The serving load: Poisson arrivals at `rate` jobs/s; 3D grids with
    edge log-uniform in [edge_lo, edge_hi]; 1-8 spheres with centres
    U[0.2,0.8] and radii U[0.05,0.2]; 4 Taylor-Green modes with wavenumbers
    in {1,2,3} and amplitudes N(0,0.5); step counts uniform in
    [steps_lo, steps_hi].  Draw order per job: gap, edge, spheres, radii,
    modes, steps."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for q in range(njobs):
        t += rng.exponential(1.0 / rate)
        e = int(round(math.exp(rng.uniform(math.log(edge_lo), math.log(edge_hi)))))
        ns = int(rng.integers(1, 9))
        cs = rng.uniform(0.2, 0.8, size=(ns, 3))
        rs = rng.uniform(0.05, 0.2, size=ns)
        modes = [(int(rng.integers(1, 4)), float(rng.normal(0.0, 0.5))) for _ in range(4)]
        steps = int(rng.integers(steps_lo, steps_hi + 1))
        sph = [(float(c[0]), float(c[1]), float(c[2]), float(r)) for c, r in zip(cs, rs)]
        jobs.append(Job(q, (e, e, e), sph, modes, steps, t))
    return jobs


class TransportServer:
    """Python front of the native serving runtime (r3d_serve_*,
    reef3d_b200/csrc/serve.cpp): admission against the HBM budget in arrival
    order, continuous batching of the active FP32 jobs (per-instance FP64
    runs for precision=FP64), retirement with volume sums and clock.  This
    class feeds it a timed job stream and keeps the per-job record."""

    def __init__(self, budget_bytes=150e9, precision=FP32, graph=True, autotune_cache=None, keep_phi=False,
                 clock=time.perf_counter):
        global _lib
        _lib = load_library()
        self.budget = float(budget_bytes)
        self.precision = precision
        self.autotune_cache = autotune_cache
        self.keep_phi = keep_phi
        self.clock = clock
        s = ctypes.c_void_p()
        rc = _lib.r3d_serve_create(self.budget, precision, 1 if keep_phi else 0, ctypes.byref(s))
        if rc != R3D_OK:
            raise R3DError(rc, "r3d_serve_create failed")
        self.s = s
        self.done = []
        self.peak_used = 0.0
        self.max_active = 0
        self.makespan = 0.0

    def _check(self, rc):
        if rc != R3D_OK:
            msg = _lib.r3d_serve_last_error(self.s)
            raise R3DError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "s", None) is not None and self.s.value:
            _lib.r3d_serve_destroy(self.s)
            self.s = ctypes.c_void_p()

    def _submit(self, job):
        sph = np.ascontiguousarray(np.asarray(job.spheres, dtype=np.float64).reshape(-1))
        mod = np.ascontiguousarray(np.asarray(job.modes, dtype=np.float64).reshape(-1))
        d = JobDesc(job.nx, job.ny, job.nz, job.steps, job.f44, job.n47, len(job.spheres),
                    sph.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(job.modes),
                    mod.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        jid = ctypes.c_longlong()
        self._check(_lib.r3d_serve_submit(self.s, ctypes.byref(d), ctypes.byref(jid)))
        return jid.value

    def _status(self):
        q, a, m = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        used, peak = ctypes.c_double(), ctypes.c_double()
        self._check(_lib.r3d_serve_status(self.s, ctypes.byref(q), ctypes.byref(a), ctypes.byref(used),
                                          ctypes.byref(peak), ctypes.byref(m)))
        return q.value, a.value, peak.value, m.value

    def _collect(self, jid, job, offset):
        r = JobResult()
        self._check(_lib.r3d_serve_result(self.s, jid, ctypes.byref(r)))
        if r.state != 2:
            return False
        job.volume = (r.volume1, r.volume2)
        job.time = r.sim_time
        job.t_admit = r.t_admit + offset
        job.t_done = r.t_done + offset
        if self.keep_phi:
            phi = np.zeros((job.nx + 6, job.ny + 6, job.nz + 6))
            _check(_lib.r3d_download(ctypes.c_void_p(r.instance), PHI, _dp(phi), LAYOUT_REEF3D))
            job.phi = phi
            self._check(_lib.r3d_serve_release(self.s, jid))
        self.done.append(job)
        return True

    def serve(self, jobs, realtime=True):
        """Runs the stream to completion.  With realtime, a job is submitted
        at its arrival time on the wall clock (measured from the start of
        serve) and the runtime advances one step per poll (it returns once
        the previous poll's step is done, so an arrival joins at the next
        step); without realtime, all jobs are submitted at once and each
        poll runs up to the next job completion.  Returns the finished
        jobs."""
        pending = collections.deque(sorted(jobs, key=lambda j: j.arrival))
        out = {}  # server job id -> (job, offset of the server clock)
        t0 = self.clock()
        tuned_for = None
        while pending or out:
            now = self.clock() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                job = pending.popleft()
                jid = self._submit(job)
                r = JobResult()
                self._check(_lib.r3d_serve_result(self.s, jid, ctypes.byref(r)))
                out[jid] = (job, (self.clock() - t0) - r.t_submit)
            queued, active, _, _ = self._status()
            if active == 0 and queued == 0:
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (self.clock() - t0))))
                continue
            if self.autotune_cache is not None and self.precision == FP32 and tuned_for != active:
                b = ctypes.c_void_p()
                self._check(_lib.r3d_serve_batch(self.s, ctypes.byref(b)))
                rows, ctas = ctypes.c_int(), ctypes.c_int()
                _lib.r3d_batch_autotune(b, os.fsencode(self.autotune_cache), ctypes.byref(rows), ctypes.byref(ctas))
                tuned_for = active
            nfin = ctypes.c_int()
            self._check(_lib.r3d_serve_poll(self.s, 1 if realtime else (1 << 30), ctypes.byref(nfin)))
            if nfin.value:
                for jid in [j for j in out if self._collect(j, *out[j])]:
                    del out[jid]
        _, _, self.peak_used, self.max_active = self._status()
        self.makespan = self.clock() - t0
        return self.done


def summarize(jobs, makespan):
    """Latency (arrival to completion) split into queueing delay (arrival to
    admission) and service time (admission to completion), p50 / p99 / mean
    of each, and the throughput over the whole run."""
    lat = np.array([j.latency for j in jobs])
    queue = np.array([j.t_admit - j.arrival for j in jobs])
    service = np.array([j.t_done - j.t_admit for j in jobs])
    cells = sum(j.cells * j.steps for j in jobs)
    out = {"jobs": len(jobs), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
           "mean_s": float(lat.mean()), "makespan_s": makespan, "cell_updates": cells,
           "cell_updates_per_s": cells / makespan}
    for name, a in (("queue", queue), ("service", service)):
        out[name] = {"p50_s": float(np.percentile(a, 50)), "p99_s": float(np.percentile(a, 99)),
                     "mean_s": float(a.mean())}
    return out


def mean_job_cell_updates(edge_lo=32, edge_hi=384, steps_lo=50, steps_hi=500):
    """Expected cell-updates of one job of the serving mix: E[edge^3] of the
    log-uniform edge times the mean step count."""
    e3 = (edge_hi ** 3 - edge_lo ** 3) / (3.0 * math.log(edge_hi / edge_lo))
    return e3 * 0.5 * (steps_lo + steps_hi)
