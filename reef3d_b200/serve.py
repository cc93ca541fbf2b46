"""Continuous-batching server for level-set transport jobs.

Jobs (a sphere-union level set advected by a Taylor-Green velocity for a
given number of steps) arrive over time.  The server admits waiting jobs in
arrival order whenever their device footprint fits the HBM budget, keeps
every admitted job's fields resident on the device, and advances all active
jobs together one step at a time in a ``Batch`` (one persistent launch per
RK stage over every member, the step replayed from a CUDA graph).  Jobs join
and leave between steps, so work of jobs that arrive while others are on
the GPU overlaps with theirs on the device.  A job's result does not depend
on which other jobs shared its steps.

The FP64 plain path (``precision=FP64``) serves the same stream without
batching: every active job is stepped on its own instance.
"""
import collections
import math
import time

import numpy as np

from . import FP32, FP64, PHI, Batch, LevelSet, footprint, uniform_nodes


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
    def __init__(self, budget_bytes=150e9, precision=FP32, graph=True, autotune_cache=None, keep_phi=False,
                 clock=time.perf_counter):
        self.budget = float(budget_bytes)
        self.precision = precision
        self.graph = graph
        self.autotune_cache = autotune_cache
        self.keep_phi = keep_phi
        self.clock = clock
        self.used = 0.0
        self.batch = Batch() if precision == FP32 else None
        if self.batch is not None:
            self.batch.use_graph(graph)
        self.active = {}  # job id -> [job, LevelSet, steps done, bytes]
        self.done = []
        self.peak_used = 0.0
        self.max_active = 0

    def close(self):
        for job, ls, _, _ in list(self.active.values()):
            ls.close()
        self.active.clear()
        if self.batch is not None:
            self.batch.close()

    def _footprint(self, job):
        return float(footprint(job.nx, job.ny, job.nz, self.precision))

    def _admit(self, job, now):
        ls = LevelSet(job.nx, job.ny, job.nz, uniform_nodes(job.nx), uniform_nodes(job.ny), uniform_nodes(job.nz),
                      f43=0.5, f44=job.f44, f45=2.1, f49=1, n47=job.n47, precision=self.precision)
        ls.init_spheres_tg(job.spheres, job.modes)
        ls.set_time(0.0)
        if self.batch is not None:
            self.batch.add(ls)
        fp = self._footprint(job)
        self.used += fp
        self.peak_used = max(self.peak_used, self.used)
        job.t_admit = now
        self.active[job.id] = [job, ls, 0, fp]
        self.max_active = max(self.max_active, len(self.active))

    def _retire(self, jid, t0):
        job, ls, _, fp = self.active.pop(jid)
        if self.batch is not None:
            self.batch.remove(ls)
        job.volume = ls.last_volume()
        job.time = ls.time()
        if self.keep_phi:
            job.phi = ls.download(PHI)
        job.t_done = self.clock() - t0
        ls.close()
        self.used -= fp
        self.done.append(job)

    def serve(self, jobs, realtime=True):
        """Runs the stream to completion.  With realtime, a job becomes
        visible at its arrival time on the wall clock (measured from the
        start of serve); otherwise all jobs are visible at once.  Returns
        the finished jobs."""
        pending = collections.deque(sorted(jobs, key=lambda j: j.arrival))
        queue = collections.deque()
        t0 = self.clock()
        retuned_for = None
        while pending or queue or self.active:
            now = self.clock() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                queue.append(pending.popleft())
            changed = False
            while queue and self.used + self._footprint(queue[0]) <= self.budget:
                self._admit(queue.popleft(), now)
                changed = True
            if queue and not self.active:
                raise RuntimeError(f"job {queue[0].id} alone exceeds the HBM budget")
            if not self.active:
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - now)))
                continue
            if self.batch is not None:
                if changed and self.autotune_cache is not None and retuned_for != len(self.active):
                    self.batch.autotune(self.autotune_cache)
                    retuned_for = len(self.active)
                self.batch.step(1)
            else:
                for job, ls, _, _ in self.active.values():
                    ls.run(1, adaptive=True)
            finished = []
            for jid, rec in self.active.items():
                rec[2] += 1
                if rec[2] >= rec[0].steps:
                    finished.append(jid)
            for jid in finished:
                self._retire(jid, t0)
        self.makespan = self.clock() - t0
        return self.done


def summarize(jobs, makespan):
    lat = np.array([j.latency for j in jobs])
    cells = sum(j.cells * j.steps for j in jobs)
    return {"jobs": len(jobs), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "makespan_s": makespan, "cell_updates": cells,
            "cell_updates_per_s": cells / makespan}
