"""The benchmark configurations beyond the headline vortex run: the 2D
slotted-disc revolution, the vortex accuracy run (FP32 form against the FP64
path over a full period), the wave tank with the Airy velocity generator,
the batched ensemble and the serving load test.
Each function runs on the current CUDA device and returns a dict for the
benchmark's JSON line."""
import math
import time

import numpy as np

from . import FP32, FP64, PHI, U, V, W, Batch, LevelSet, setups, uniform_nodes


def _events(stream_ptr):
    import torch
    s = torch.cuda.ExternalStream(stream_ptr)
    return s, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def heaviside(phi, eps):
    return np.where(phi > eps, 1.0, np.where(phi < -eps, 0.0, 0.5 * (1 + phi / eps + np.sin(np.pi * phi / eps) / np.pi)))


def slotted_disk_revolution(n=128, precision=FP64):
    """2D slotted disc, rigid rotation for one period (t = 1): device time,
    cell-updates/s, L1 area error of the returned shape and relative volume
    change."""
    c = setups.slotted_disk(n)
    with LevelSet(n, 1, n, c.xn, c.yn, c.zn, precision=precision, **c.flags()) as ls:
        for f, a in ((PHI, c.phi), (U, c.u), (V, c.v), (W, c.w)):
            ls.upload(f, a)
        v0 = ls.volume()[0]
        # the CFL step is constant (steady velocity): take it once, step to t = 1
        dt = ls.cfl_dt()
        nsteps = int(math.ceil(1.0 / dt - 1e-9))
        dt = 1.0 / nsteps
        ls.set_dt(dt)
        s, e0, e1 = _events(ls.stream())
        ls.sync()
        e0.record(s)
        ls.run(nsteps, adaptive=False)  # one captured step replayed
        e1.record(s)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        phi = ls.download(PHI)
        v1 = ls.volume()[0]
    h = 1.0 / n
    a0 = c.phi[3:3 + n, 3, 3:3 + n]
    a1 = phi[3:3 + n, 3, 3:3 + n]
    l1 = float(np.sum(np.abs(heaviside(a1, 1.5 * h) - heaviside(a0, 1.5 * h))) * h * h)
    return {"workload": f"slotted disc 2D {n}x{n}, one revolution", "steps": nsteps, "ms": ms,
            "cell_updates_per_s": n * n * nsteps / (ms * 1e-3), "l1_area_error": l1,
            "relative_volume_change": abs(v1 - v0) / abs(v0), "precision": "fp64" if precision == FP64 else "fp32"}


def _vortex_period(n, precision, T=3.0, perturb=0.0):
    """Vortex to t = T with the fixed step T/N, N = ceil(T / dt_peak) (dt_peak:
    the CFL step of the peak velocity at t = 0).  perturb > 0 multiplies the
    initial level set by 1 + perturb * N(0,1) (seeded).  Returns (case,
    phi(T), volume1 at 0 and T, steps, device ms)."""
    c = setups.vortex3d(n)
    phi0 = c.phi
    if perturb > 0.0:
        phi0 = np.ascontiguousarray(c.phi * (1.0 + perturb * np.random.default_rng(12).standard_normal(c.phi.shape)))
    with LevelSet(n, n, n, c.xn, c.yn, c.zn, precision=precision, **c.flags()) as ls:
        for f, a in ((PHI, phi0), (U, c.u), (V, c.v), (W, c.w)):
            ls.upload(f, a)
        ls.set_velocity_period(T)
        ls.set_time(0.0)
        v0 = ls.volume()[0]
        nsteps = int(math.ceil(T / ls.cfl_dt() - 1e-9))
        ls.set_dt(T / nsteps)
        s, e0, e1 = _events(ls.stream())
        ls.sync()
        e0.record(s)
        ls.run(nsteps, adaptive=False)
        e1.record(s)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        phi = ls.download(PHI)
        v1 = ls.volume()[0]
    return c, phi, v0, v1, nsteps, ms


def vortex_accuracy(n=128, T=3.0, perturbed=True):
    """Shape error and volume change of the FP32 form and of the FP64 path
    over a full vortex period (the shape returns to the initial sphere at
    t = T), and the FP32 result against the FP64 one: L1 of the smoothed
    Heaviside H(phi; 1.5 h) times the cell volume, L-infinity of phi over the
    band |phi_FP64| < 3h, relative change of volume1."""
    h = 1.0 / n
    res = {}
    runs = {}
    forms = [("fp64", FP64, 0.0), ("fp32", FP32, 0.0)] + ([("fp64_perturbed", FP64, 1e-12)] if perturbed else [])
    for name, prec, eps in forms:
        c, phi, v0, v1, nsteps, ms = _vortex_period(n, prec, T, eps)
        a = phi[3:3 + n, 3:3 + n, 3:3 + n]
        runs[name] = a
        a0 = c.phi[3:3 + n, 3:3 + n, 3:3 + n]
        res[name] = {"steps": nsteps, "ms": ms, "cell_updates_per_s": n ** 3 * nsteps / (ms * 1e-3),
                     "l1_shape_error": float(np.sum(np.abs(heaviside(a, 1.5 * h) - heaviside(a0, 1.5 * h))) * h ** 3),
                     "linf_shape_error_band": float(np.max(np.abs(a - a0)[np.abs(a0) < 3 * h])),
                     "relative_volume_change": abs(v1 - v0) / abs(v0)}
    a32, a64 = runs["fp32"], runs["fp64"]
    band = np.abs(a64) < 3 * h
    res["fp32_vs_fp64"] = {
        "l1_heaviside": float(np.sum(np.abs(heaviside(a32, 1.5 * h) - heaviside(a64, 1.5 * h))) * h ** 3),
        "linf_phi_band": float(np.max(np.abs(a32 - a64)[band])),
        "shape_error_ratio": res["fp32"]["l1_shape_error"] / res["fp64"]["l1_shape_error"],
        "volume_change_diff": abs(res["fp32"]["relative_volume_change"] - res["fp64"]["relative_volume_change"])}
    res["fp32_within_1pct"] = {
        "l1_shape_error": abs(res["fp32"]["l1_shape_error"] - res["fp64"]["l1_shape_error"])
        <= 0.01 * res["fp64"]["l1_shape_error"],
        "relative_volume_change": abs(res["fp32"]["relative_volume_change"] - res["fp64"]["relative_volume_change"])
        <= 0.01 * res["fp64"]["relative_volume_change"]}
    res["workload"] = f"3D single vortex {n}^3 to t = T = {T}, CFL 0.25 of the peak velocity, fixed dt"
    if not perturbed:
        return res
    # the same comparison for an FP64 run whose initial level set differs by
    # 1e-12 relative: the sensitivity of these metrics to any perturbation
    ap = runs["fp64_perturbed"]
    res["fp64_perturbed_vs_fp64"] = {
        "l1_heaviside": float(np.sum(np.abs(heaviside(ap, 1.5 * h) - heaviside(a64, 1.5 * h))) * h ** 3),
        "linf_phi_band": float(np.max(np.abs(ap - a64)[band])),
        "shape_error_ratio": res["fp64_perturbed"]["l1_shape_error"] / res["fp64"]["l1_shape_error"],
        "volume_change_diff": abs(res["fp64_perturbed"]["relative_volume_change"] - res["fp64"]["relative_volume_change"])}
    return res


def wave_tank_run(steps=500, warmup=3, dims=(1024, 128, 256), precision=FP32):
    """Wave tank 1024x128x256 (dx = 0.01 m, depth 0.5 m, wavelength 2 m,
    amplitude 0.05 m), Airy orbital velocity regenerated on the device at the
    start of every step, CFL 0.2, one reinitialisation pseudo-step per step,
    `steps` steps in one captured-graph run: device time, cell-updates/s and
    the relative change of volume1."""
    nx, ny, nz = dims
    c = setups.wave_tank(nx, ny, nz, velocity=False)
    with LevelSet(nx, ny, nz, c.xn, c.yn, c.zn, precision=precision, **c.flags()) as ls:
        ls.upload(PHI, c.phi)
        del c.phi
        ls.set_time(0.0)
        ls.set_velocity_airy(0.05, 2.0, 0.5, 9.81)
        v0 = ls.volume()[0]
        ls.run(warmup, adaptive=True)
        s, e0, e1 = _events(ls.stream())
        ls.sync()
        c0 = ls.launch_count()
        e0.record(s)
        ls.run(steps, adaptive=True)
        e1.record(s)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        launches = ls.launch_count() - c0
        v1 = ls.volume()[0]
        t_end = ls.time()
    cells = nx * ny * nz
    return {"workload": f"wave tank {nx}x{ny}x{nz}, Airy velocity per step, CFL 0.2, F44=1", "steps": steps,
            "ms": ms, "ms_per_step": ms / steps, "cell_updates_per_s": cells * steps / (ms * 1e-3),
            "simulated_s": t_end, "relative_volume_change": abs(v1 - v0) / abs(v0), "launches": launches,
            "precision": "fp32 form" if precision == FP32 else "fp64 plain"}


def _accuracy(a32, a64, a0, h, cellvol, v0s, v1s):
    """FP32 result against the FP64 one on the same grid: L1 of the smoothed
    Heaviside H(phi; 1.5 h) times the cell volume, L-infinity of phi over the
    band |phi_FP64| < 3h, and each run's relative change of volume1; plus the
    FP64 run's L1 distance from the initial shape for scale."""
    band = np.abs(a64) < 3 * h
    return {"l1_heaviside_fp32_vs_fp64": float(np.sum(np.abs(heaviside(a32, 1.5 * h) - heaviside(a64, 1.5 * h))) * cellvol),
            "l1_heaviside_fp64_moved": float(np.sum(np.abs(heaviside(a64, 1.5 * h) - heaviside(a0, 1.5 * h))) * cellvol),
            "linf_phi_band": float(np.max(np.abs(a32 - a64)[band])) if band.any() else 0.0,
            "relative_volume_change_fp32": abs(v1s[0] - v0s[0]) / abs(v0s[0]),
            "relative_volume_change_fp64": abs(v1s[1] - v0s[1]) / abs(v0s[1])}


def wave_tank_accuracy(steps=500, dims=(1024, 128, 256)):
    """The wave tank in the FP32 form and in FP64 with the same fixed step
    (the FP64 CFL step at t = 0), compared after `steps` steps."""
    nx, ny, nz = dims
    c = setups.wave_tank(nx, ny, nz, velocity=False)
    outs, v0s, v1s, dt = [], [], [], None
    for prec in (FP64, FP32):
        with LevelSet(nx, ny, nz, c.xn, c.yn, c.zn, precision=prec, **c.flags()) as ls:
            ls.upload(PHI, c.phi)
            ls.set_time(0.0)
            ls.set_velocity_airy(0.05, 2.0, 0.5, 9.81)
            if dt is None:
                dt = ls.cfl_dt()
            ls.set_dt(dt)
            v0s.append(ls.volume()[0])
            ls.run(steps, adaptive=False)
            v1s.append(ls.volume()[0])
            outs.append(ls.download(PHI)[3:3 + nx, 3:3 + ny, 3:3 + nz].copy())
    h = 0.01
    r = _accuracy(outs[1], outs[0], c.phi[3:3 + nx, 3:3 + ny, 3:3 + nz], h, h ** 3, v0s[::-1], v1s[::-1])
    r.update({"steps": steps, "dt": dt, "workload": f"wave tank {nx}x{ny}x{nz}, fixed dt, FP32 form vs FP64"})
    return r


def ensemble_accuracy(steps=200, seed=0, picks=(2, 2)):
    """Members of the ensemble (the first `picks[0]` 2D and `picks[1]` 3D
    ones of seed 0) run alone in the FP32 form -- the arithmetic of their
    batched steps -- and in FP64 with the same fixed step, compared after
    `steps` steps."""
    specs = ensemble_specs(seed)
    chosen = [s for s in specs if s[0][1] == 1][:picks[0]] + [s for s in specs if s[0][1] > 1][:picks[1]]
    res = []
    for dims, sph, modes in chosen:
        nx, ny, nz = dims
        outs, v0s, v1s, dt = [], [], [], None
        for prec in (FP64, FP32):
            ls = make_instance(dims, sph, modes, precision=prec)
            try:
                if dt is None:
                    dt = ls.cfl_dt()
                ls.set_dt(dt)
                v0s.append(ls.volume()[0])
                if prec == FP64:
                    phi0 = ls.download(PHI)[3:3 + nx, 3:3 + ny, 3:3 + nz].copy()
                ls.run(steps, adaptive=False)
                v1s.append(ls.volume()[0])
                outs.append(ls.download(PHI)[3:3 + nx, 3:3 + ny, 3:3 + nz].copy())
            finally:
                ls.close()
        axes = [nx, nz] if ny == 1 else [nx, ny, nz]
        h = 1.0 / min(axes)                     # the coarsest spacing
        cellvol = float(np.prod([1.0 / n for n in axes]))
        r = _accuracy(outs[1], outs[0], phi0, h, cellvol, v0s[::-1], v1s[::-1])
        r["dims"] = list(dims)
        res.append(r)
    return {"steps": steps, "members": res,
            "workload": f"{picks[0]} 2D + {picks[1]} 3D members of the seed-{seed} ensemble, fixed dt, FP32 vs FP64"}


def ensemble_specs(seed=0, count=64, edges=tuple(range(64, 257, 32))):
    """Parameters of the batched ensemble (same draw order as
    setups.random_instance): 50/50 2D/3D, edges uniform in `edges`, 1-8
    spheres, 4 Taylor-Green modes."""
    rng = np.random.default_rng(seed)
    specs = []
    for q in range(count):
        two_d = bool(rng.integers(0, 2))
        nx = int(rng.choice(edges))
        nz = int(rng.choice(edges))
        ny = 1 if two_d else int(rng.choice(edges))
        ns = int(rng.integers(1, 9))
        cs = rng.uniform(0.2, 0.8, size=(ns, 3))
        rs = rng.uniform(0.05, 0.2, size=ns)
        modes = [(int(rng.integers(1, 4)), float(rng.normal(0.0, 0.5))) for _ in range(4)]
        sph = [(float(c[0]), float(c[1]), float(c[2]), float(r)) for c, r in zip(cs, rs)]
        specs.append(((nx, ny, nz), sph, modes))
    return specs


def make_instance(dims, sph, modes, precision=FP32, f44=2, cfl=0.25):
    nx, ny, nz = dims
    yn = uniform_nodes(1, 1.0 / nx) if ny == 1 else uniform_nodes(ny)
    ls = LevelSet(nx, ny, nz, uniform_nodes(nx), yn, uniform_nodes(nz), f43=0.5, f44=f44, f45=2.1, f49=1,
                  n47=cfl / 2.0, precision=precision)
    ls.init_spheres_tg(sph, modes)
    ls.set_time(0.0)
    return ls


def ensemble(steps=200, seed=0, count=64, autotune_cache=None, graph=True):
    """64 instances (seed 0) advanced `steps` steps in one batch: device
    time, aggregate cell-updates/s, launches per step and the tuned
    configuration."""
    specs = ensemble_specs(seed, count)
    members = [make_instance(d, s, m) for d, s, m in specs]
    cells = sum(d[0] * d[1] * d[2] for d, _, _ in specs)
    with Batch() as b:
        for m in members:
            b.add(m)
        t0 = time.perf_counter()
        cfg = b.autotune(autotune_cache)
        tune_s = time.perf_counter() - t0
        b.use_graph(graph)
        b.step(1)  # warm-up: builds and captures the graph
        b.sync()
        s, e0, e1 = _events(b.stream())
        c0 = b.launch_count()
        e0.record(s)
        b.step(steps)
        e1.record(s)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        launches = b.launch_count() - c0
    for m in members:
        m.close()
    n2 = sum(1 for d, _, _ in specs if d[1] == 1)
    return {"workload": f"ensemble of {count} (seed {seed}), {n2} 2D + {count - n2} 3D, edges 64..256",
            "steps": steps, "cells": cells, "ms": ms, "cell_updates_per_s": cells * steps / (ms * 1e-3),
            "launches": launches, "config_rows_ctas": list(cfg), "autotune_s": tune_s, "graph": graph}


def serving(njobs=48, rate=200.0, seed=1, budget=150e9, precision=FP32, autotune_cache=None):
    from .serve import TransportServer, poisson_jobs, summarize
    jobs = poisson_jobs(seed=seed, rate=rate, njobs=njobs)
    srv = TransportServer(budget_bytes=budget, precision=precision, autotune_cache=autotune_cache)
    try:
        done = srv.serve(jobs, realtime=True)
        out = summarize(done, srv.makespan)
        out.update({"rate_jobs_per_s": rate, "seed": seed, "budget_gb": budget / 1e9,
                    "peak_resident_gb": srv.peak_used / 1e9, "max_active": srv.max_active,
                    "precision": "fp32 batched" if precision == FP32 else "fp64 plain"})
    finally:
        srv.close()
    return out


def serving_loads(burst, fractions=(0.5, 0.9), njobs=200, seed=1, budget=150e9, autotune_cache=None):
    """The serving mix at loads the server can carry: its capacity in jobs/s
    is the cell-updates/s of the saturating burst run (`burst`, the output
    of serving() at 200 jobs/s) over the expected cell-updates of one job;
    `njobs` Poisson arrivals at each fraction of that capacity, with p50/p99
    latency split into queueing delay and service time."""
    from .serve import mean_job_cell_updates
    per_job = mean_job_cell_updates()
    cap = burst["cell_updates_per_s"] / per_job
    out = {"capacity_jobs_per_s": cap, "mean_job_cell_updates": per_job,
           "capacity_from": "cell-updates/s of the 200 jobs/s burst / expected cell-updates per job"}
    for f in fractions:
        r = serving(njobs=njobs, rate=f * cap, seed=seed, budget=budget, autotune_cache=autotune_cache)
        r["load_fraction"] = f
        out[f"load_{f:g}"] = r
    return out


def slab_domain(n=256, nslabs=4, steps=20, warmup=3, precision=FP32):
    """The 256^3 vortex split into z slabs on this GPU and stepped by the
    native runner (r3d_domain_*, one CUDA graph per step with the halo
    copies), beside the undivided instance on the same steps: the cost of
    the decomposition.  Fixed-velocity adaptive steps from t = 0."""
    import time
    from . import PHI, U, V, W, LevelSet
    from .slab import Domain
    c = setups.vortex3d(n)
    res = {}
    d = Domain(n, n, n, c.xn, c.yn, c.zn, nslabs=nslabs, precision=precision, **c.flags())
    try:
        for f, a in ((PHI, c.phi), (U, c.u), (V, c.v), (W, c.w)):
            d.upload(f, a)
        d.run(warmup)
        t0 = time.perf_counter()
        d.run(steps)
        res["domain_ms_per_step"] = 1e3 * (time.perf_counter() - t0) / steps
        phi_d = d.download(PHI)
    finally:
        d.close()
    with LevelSet(n, n, n, c.xn, c.yn, c.zn, precision=precision, **c.flags()) as ls:
        for f, a in ((PHI, c.phi), (U, c.u), (V, c.v), (W, c.w)):
            ls.upload(f, a)
        ls.run(warmup, adaptive=True)
        ls.sync()
        t0 = time.perf_counter()
        ls.run(steps, adaptive=True)
        ls.sync()
        res["single_ms_per_step"] = 1e3 * (time.perf_counter() - t0) / steps
        phi_s = ls.download(PHI)
    cells = n ** 3
    res.update({"workload": f"vortex {n}^3 in {nslabs} z slabs on one GPU (r3d_domain), {steps} adaptive steps",
                "cell_updates_per_s": cells / (res["domain_ms_per_step"] * 1e-3),
                "overhead": res["domain_ms_per_step"] / res["single_ms_per_step"] - 1.0,
                "phi_identical_to_undivided": bool(np.array_equal(phi_d[3:-3, 3:-3, 3:-3], phi_s[3:-3, 3:-3, 3:-3])),
                "precision": "fp32 form" if precision == FP32 else "fp64"})
    return res
