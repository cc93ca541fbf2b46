"""Continuous-batching server: admission against an HBM budget, jobs joining
and leaving between steps, and each job's result the same alone and in the
mix (bit-identical level set and clock, volume within 1e-12)."""
import numpy as np
import pytest

import reef3d_b200 as r3d
from reef3d_b200.serve import Job, TransportServer, poisson_jobs, summarize

pytestmark = pytest.mark.gpu


def small_stream(n=10, seed=3):
    return poisson_jobs(seed=seed, rate=500.0, njobs=n, edge_lo=12, edge_hi=40, steps_lo=3, steps_hi=12)


def clone(job):
    return Job(job.id, (job.nx, job.ny, job.nz), job.spheres, job.modes, job.steps, 0.0, job.f44)


def serve(jobs, **kw):
    s = TransportServer(keep_phi=True, **kw)
    try:
        done = s.serve(jobs, realtime=False)
        return {j.id: j for j in done}, s
    finally:
        s.close()


def test_result_alone_equals_result_in_mix():
    jobs = small_stream()
    mix, _ = serve([clone(j) for j in jobs], budget_bytes=64e9)
    for q in (0, 4, 9):
        alone, _ = serve([clone(jobs[q])], budget_bytes=64e9)
        a, m = alone[q], mix[q]
        assert np.array_equal(a.phi, m.phi)
        assert a.time == m.time
        assert abs(a.volume[0] - m.volume[0]) <= 1e-12 * abs(m.volume[0])


def test_admission_respects_budget():
    jobs = small_stream(8, seed=4)
    fps = sorted(r3d.footprint(j.nx, j.ny, j.nz, r3d.FP32) for j in jobs)
    budget = fps[-1] + fps[-2] + 1.0  # room for two of the largest at most
    done, s = serve([clone(j) for j in jobs], budget_bytes=budget)
    assert len(done) == len(jobs)
    assert s.peak_used <= budget
    assert s.max_active >= 2
    for j in done.values():
        assert j.t_admit is not None and j.t_done is not None


def test_fp64_plain_path_serves_same_stream():
    jobs = small_stream(5, seed=5)
    s32, _ = serve([clone(j) for j in jobs], budget_bytes=64e9)
    s64, _ = serve([clone(j) for j in jobs], budget_bytes=64e9, precision=r3d.FP64)
    for jid in s32:
        a, b = s32[jid], s64[jid]
        m = np.abs(b.phi) > 0
        err = np.max(np.abs(a.phi[m] - b.phi[m])) / np.max(np.abs(b.phi[m]))
        assert err <= 1e-4


def test_realtime_stream_latency_summary():
    jobs = small_stream(6, seed=6)
    s = TransportServer(budget_bytes=64e9)
    try:
        done = s.serve(jobs, realtime=True)
        out = summarize(done, s.makespan)
    finally:
        s.close()
    assert out["jobs"] == 6 and out["p99_s"] >= out["p50_s"] > 0


def test_native_runtime_refusals_and_release():
    """The C-ABI of the serving runtime: a job larger than the budget is
    refused at submission, an unfinished job cannot be released, a finished
    job's instance stays readable until released."""
    import ctypes
    from reef3d_b200 import JobDesc, JobResult
    lib = r3d.load_library()
    s = ctypes.c_void_p()
    assert lib.r3d_serve_create(1e9, r3d.FP32, 1, ctypes.byref(s)) == r3d.R3D_OK
    try:
        sph = np.array([0.5, 0.5, 0.5, 0.2])
        mod = np.array([1.0, 0.5])
        P = ctypes.POINTER(ctypes.c_double)
        big = JobDesc(512, 512, 512, 5, 2, 0.125, 1, sph.ctypes.data_as(P), 1, mod.ctypes.data_as(P))
        jid = ctypes.c_longlong()
        assert lib.r3d_serve_submit(s, ctypes.byref(big), ctypes.byref(jid)) == r3d.R3D_ENOMEM
        small = JobDesc(24, 24, 24, 4, 2, 0.125, 1, sph.ctypes.data_as(P), 1, mod.ctypes.data_as(P))
        assert lib.r3d_serve_submit(s, ctypes.byref(small), ctypes.byref(jid)) == r3d.R3D_OK
        assert lib.r3d_serve_release(s, jid) == r3d.R3D_ESTATE  # still queued
        nfin = ctypes.c_int()
        assert lib.r3d_serve_poll(s, 100, ctypes.byref(nfin)) == r3d.R3D_OK and nfin.value == 1
        r = JobResult()
        assert lib.r3d_serve_result(s, jid, ctypes.byref(r)) == r3d.R3D_OK
        assert r.state == 2 and r.steps_done == 4 and r.instance and r.t_done >= r.t_admit >= r.t_submit
        assert lib.r3d_serve_release(s, jid) == r3d.R3D_OK
        assert lib.r3d_serve_result(s, jid, ctypes.byref(r)) == r3d.R3D_OK and r.state == 3 and not r.instance
    finally:
        lib.r3d_serve_destroy(s)
