"""Benchmark of the level-set transport path (WENO5-HJ convection in TVD-RK3
stages + PDE reinitialisation) on the 3D single-vortex deformation, 256^3
cells, CFL 0.25, 2 reinitialisation pseudo-steps per step.

One step = one physical time step over the whole grid: the FP64 CFL
reduction, 3 fused convection stages, 2 x 3 fused reinitialisation stages
and the FP64 volume integral, with the vortex velocity following the device
clock (u(x,t) = u(x) cos(pi t / 3)).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs under torchrun, one rank per GPU; every rank advances its own
instance (replicas, no collective on the data path), `value` is the
aggregate over ranks with the max-over-ranks device time.
"""
import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CELLS_EDGE = 256
# ncu summary of the tiled FP32 stage kernels on the vortex: its "traffic:"
# lines carry the DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of
# one launch per (stage kind, grid edge, tile configuration, z chunk), from
# the capture whose command the file gives
TRAFFIC_PROFILE = os.path.join("profiles", "tile_stage_kernels_vortex.txt")
METRIC = "level-set cell-updates/s (RK3+reinit), FP64 plain vs FP32 batched; p50/p99 latency"
WORKLOAD = "3D single-vortex deformation 256^3, CFL 0.25, F44=2 reinit pseudo-steps, T=3"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--edge", type=int, default=N_CELLS_EDGE)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--tile-cache", default=None,
                    help="autotune cache file: a run reuses the tile configuration an earlier run stored there "
                         "(so that a profiled run launches the same kernels as the timed one)")
    ap.add_argument("--tile-sweep", action="store_true",
                    help="launch stage 2 of both kinds once under every tile configuration and z chunk the "
                         "autotuner tries, then exit (the DRAM traffic of each, for the ncu summary the "
                         "roofline's traffic is read from)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other workloads (slotted disc, vortex accuracy, wave tank, ensemble, serving)")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_min_mhz": min(sm) if sm else None,
                "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- CPU side
# resident size of one reference process per padded cell of its grid (the
# reference's fdm/lexer fields, measured: 1.55 GB at 128^3, 12.4 GB at 256^3)
REF_BYTES_PER_CELL = 700.0


def _ref_proc(edge, warm, steps, fast, barrier, queue):
    """One reference process: its own vortex grid at `edge`^3, `warm`
    untimed steps, then (after every process is ready) `steps` timed ones."""
    from oracle.bindings import RefOracle
    from reef3d_b200 import setups
    try:
        c = setups.vortex3d(edge)
        o = RefOracle(edge, edge, edge, c.xn, c.yn, c.zn, f43=c.f43, f44=c.f44, f45=c.f45, f49=c.f49, fast=fast)
        o.set_state(c.phi, c.u, c.v, c.w)
        del c
        dt = o.cfl_dt(0.125)
        o.set_count(1)
        for _ in range(warm):
            o.step(dt)
        barrier.wait()
        per = []
        for _ in range(steps):
            t0 = time.perf_counter()
            o.step(dt)
            per.append(time.perf_counter() - t0)
        queue.put((per, None))
    except Exception as e:  # reported by the parent
        barrier.abort()
        queue.put(([], repr(e)))


def host_cpu():
    """Model name and logical CPU count of the host."""
    model = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return f"{model}, {os.cpu_count()} logical CPUs"


def host_has_avx2_fma():
    try:
        flags = open("/proc/cpuinfo").read()
        return " avx2" in flags and " fma" in flags
    except OSError:
        return False


def mem_available():
    try:
        for ln in open("/proc/meminfo"):
            if ln.startswith("MemAvailable:"):
                return int(ln.split()[1]) * 1024
    except OSError:
        pass
    return None


def reference_procs(edge, steps):
    """Processes for the reference CPU arm: one per host core, no more than
    80 % of the available memory holds (each process owns a whole grid), and
    a divisor of `steps` so every process runs the same number of steps."""
    cap = os.cpu_count() or 1
    avail = mem_available()
    if avail is not None:
        per = REF_BYTES_PER_CELL * (edge + 6) ** 3 + 2e8
        cap = min(cap, max(1, int(0.8 * avail // per)))
    cap = max(1, min(cap, steps))
    return max(p for p in range(1, cap + 1) if steps % p == 0)


def reference_cpu(edge, steps, warmup, procs):
    """The reference's own level-set step (oracle/_ref) on the host cores at
    the benchmark's grid: `procs` single-threaded processes (the reference's
    only parallel mode is MPI, absent here), each advancing its own
    `edge`^3 vortex grid; `steps` timed steps and `warmup` untimed ones in
    all, shared equally.  The timed region starts when every process has
    built its grid and run its warm-up (a barrier) and ends when the last
    process finishes.  Returns (cell-updates/s, info)."""
    from oracle.bindings import REF_LIB, REF_LIB_FAST
    fast = host_has_avx2_fma() and os.path.exists(REF_LIB_FAST)
    if not os.path.exists(REF_LIB) and not fast:
        return None, {"unavailable": "oracle/_ref was not built (needs the reference sources)"}
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs + 1)
    queue = ctx.Queue()
    share = [steps // procs + (1 if r < steps % procs else 0) for r in range(procs)]
    warm = [warmup // procs + (1 if r < warmup % procs else 0) for r in range(procs)]
    ps = [ctx.Process(target=_ref_proc, args=(edge, warm[r], share[r], fast, barrier, queue)) for r in range(procs)]
    t_start = time.perf_counter()
    for p in ps:
        p.start()
    try:
        barrier.wait(timeout=3600)
    except Exception:  # a process failed before its timed steps (it aborted the barrier)
        pass
    t0 = time.perf_counter()
    res = [queue.get(timeout=3600) for _ in ps]
    wall = time.perf_counter() - t0
    for p in ps:
        p.join()
    errs = [e for _, e in res if e]
    if errs:
        return None, {"unavailable": "reference process failed: " + errs[0]}
    per = [t for r, _ in res for t in r]
    cells = edge ** 3 * steps
    return cells / wall, {"cores": procs, "kind": "reference", "host": host_cpu(), "timed_s": wall,
                          "build": "-O3 -mavx2 -mfma" if fast else "-O2 -ffp-contract=off",
                          "steps": steps, "warmup": warmup,
                          "s_per_step_one_core": statistics.mean(per),
                          "sample": f"{procs} processes x vortex {edge}^3 (the benchmark grid itself), {steps} timed "
                                    f"steps in all ({steps // procs} per process), {warmup} untimed; timed region "
                                    f"{wall:.1f}s, set-up {t0 - t_start:.1f}s"}


def _ref_disk_worker(args):
    n, steps, fast = args
    from oracle.bindings import RefOracle
    from reef3d_b200 import setups
    c = setups.slotted_disk(n)
    o = RefOracle(n, 1, n, c.xn, c.yn, c.zn, f43=c.f43, f44=c.f44, f45=c.f45, f49=c.f49, fast=fast)
    o.set_state(c.phi, c.u, c.v, c.w)
    dt = o.cfl_dt(c.n47)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(dt)
    return time.perf_counter() - t0


def reference_disk_cpu(n=128, steps=300):
    """The reference's own step on the 2D slotted disc, one core, a sample of
    `steps` steps (the full revolution is ~5.7k steps)."""
    from oracle.bindings import REF_LIB, REF_LIB_FAST
    fast = host_has_avx2_fma() and os.path.exists(REF_LIB_FAST)
    if not os.path.exists(REF_LIB) and not fast:
        return None
    with mp.get_context("spawn").Pool(1) as pool:
        sec = pool.apply(_ref_disk_worker, ((n, steps, fast),))
    return {"value": n * n * steps / sec, "unit": "cell-updates/s", "cores": 1, "kind": "reference", "host": host_cpu(),
            "sample": f"{steps} steps of the {n}x{n} slotted disc"}


def run_configs(ctx):
    """The other workloads of the path, each on this GPU (rank 0 at N=1),
    each with the SM clocks and throttle reasons sampled while it ran."""
    from reef3d_b200 import FP32, FP64, workloads
    out = {}

    def run(name, fn, *a, **k):
        with ClockSampler(ctx.local) as clk:
            r = fn(*a, **k)
        r["clocks"] = clk.summary()
        out[name] = r
        return r

    disk = run("slotted_disk_fp64", workloads.slotted_disk_revolution, 128, FP64)
    disk["cpu_reference"] = reference_disk_cpu()
    run("slotted_disk_fp32", workloads.slotted_disk_revolution, 128, FP32)
    # the stated size (the 1 % criterion), and 128^3 with the FP64
    # perturbation run that measures the metrics' own sensitivity there
    run("vortex_accuracy_256", workloads.vortex_accuracy, 256, perturbed=False)
    run("vortex_accuracy_128", workloads.vortex_accuracy, 128)
    run("wave_tank", workloads.wave_tank_run, 500)
    run("wave_tank_accuracy", workloads.wave_tank_accuracy, 500)
    run("ensemble", workloads.ensemble, steps=200)
    run("ensemble_accuracy", workloads.ensemble_accuracy, 200)
    # an untimed pass first: the first jobs of a process pay the one-time
    # loading of the batch kernels and graph set-up (~1 s of a 5 s burst)
    workloads.serving(njobs=4)
    burst = run("serving_fp32", workloads.serving, njobs=16)
    run("serving_fp32_loads", workloads.serving_loads, burst)
    run("serving_fp64", workloads.serving, njobs=16, precision=FP64)
    run("slab_domain", workloads.slab_domain)
    return out


def run_reference_arm(args, rank):
    if rank != 0:
        return
    procs = reference_procs(args.edge, args.steps)
    rate, info = reference_cpu(args.edge, args.steps, args.warmup, procs)
    if rate is None:
        print(json.dumps({"impl": "reference", "unavailable": info["unavailable"]}))
        return
    base = {"metric": METRIC, "impl": "reference", "value": rate, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * info["timed_s"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "edge": args.edge, "cells_per_step": args.edge ** 3,
                       "form": "the reference's FP64 code on the host cores"},
            "cpu_baseline": dict(value=rate, unit="cell-updates/s", **info),
            "e2e": {"value": rate, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(base))


# --------------------------------------------------------------- GPU side
def device_time(ls, fn, reps):
    import torch
    s = torch.cuda.ExternalStream(ls.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ls.sync()
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps  # ms


def make_instance(case, precision):
    import reef3d_b200 as r3d
    n = case.nx
    ls = r3d.LevelSet(n, n, n, case.xn, case.yn, case.zn, precision=precision, **case.flags())
    for f, a in ((r3d.PHI, case.phi), (r3d.U, case.u), (r3d.V, case.v), (r3d.W, case.w)):
        ls.upload(f, a)
    ls.set_velocity_period(3.0)
    ls.set_time(0.0)
    return ls


def timed_steps(ls, steps, warmup, dist_ctx):
    """W untimed steps, then K steps between barriers, device-timed with
    CUDA events on the instance's stream; per-step events give p50/p99."""
    import torch
    s = torch.cuda.ExternalStream(ls.stream())
    ls.run(warmup, adaptive=True)
    ls.sync()
    dist_ctx.barrier()
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    c0 = ls.launch_count()
    evs[0].record(s)
    for k in range(steps):
        ls.run(1, adaptive=True)
        evs[k + 1].record(s)
    evs[-1].synchronize()
    torch.cuda.synchronize()
    dist_ctx.barrier()
    launches = ls.launch_count() - c0
    per = [evs[k].elapsed_time(evs[k + 1]) for k in range(steps)]
    total = evs[0].elapsed_time(evs[-1])
    return total, per, launches


def stage_roofline(ls, cells, elem, peak_gbs, reps=20):
    """Average device time of each fused stage kernel launched alone, and the
    HBM roofline of the dominant one.  Algorithmic bytes per cell of a
    stage: convection stage 2/3 reads phi^n, the stage input and u,v,w and
    writes the output (6 words); reinit stage 2/3 reads f and the stage
    input and writes the output (3 words)."""
    import reef3d_b200 as r3d
    ls.set_dt(ls.cfl_dt())
    t_conv = device_time(ls, lambda: ls.stage(r3d.STAGE_CONVECTION, 2), reps)
    t_rein = device_time(ls, lambda: ls.stage(r3d.STAGE_REINIT, 2), reps)
    # one step runs 3 convection and 6 reinit stages
    share_conv, share_rein = 3 * t_conv, 6 * t_rein
    if share_rein >= share_conv:
        name, t, words = "reinit_stage", t_rein, 3
    else:
        name, t, words = "convection_stage", t_conv, 6
    alg = words * elem * cells
    achieved = alg / (t * 1e-3) / 1e9
    return {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak_gbs, "unit": "GB/s",
            "frac": achieved / peak_gbs, "bytes_per_launch": alg, "ms_per_launch": t,
            "conv_stage_ms": t_conv, "reinit_stage_ms": t_rein}


def profiled_traffic(kind, edge, cfg, chunk):
    """DRAM bytes of one launch of the dominant stage kernel from the ncu
    summary committed under profiles/ (None when that file holds no capture
    of this stage kind, grid, tile configuration and chunk).  A line reads
    `traffic: <kind> edge=<n> cfg=<id> chunk=<kc> read=<bytes> write=<bytes>`."""
    try:
        lines = open(os.path.join(ROOT, TRAFFIC_PROFILE)).read().splitlines()
    except OSError:
        return None
    for ln in lines:
        if not ln.startswith("traffic: "):
            continue
        f = ln.split()
        kv = dict(x.split("=", 1) for x in f[2:] if "=" in x)
        if f[1] == kind and int(kv["edge"]) == edge and int(kv["cfg"]) == cfg and int(kv["chunk"]) == chunk:
            rd, wr = float(kv["read"]), float(kv["write"])
            return {"bytes": rd + wr, "read": rd, "write": wr, "source": TRAFFIC_PROFILE,
                    "note": "one ncu capture of a launch; output lines still in L2 when the kernel ends are "
                            "written back after it and are not in its write figure"}
    return None


def tile_variants(ls, reps=10):
    """Stage times of the tiled FP32 kernels under other chunkings (both
    stage kinds on the convection stages' tile configuration) and with the
    FP64 interface band off (information for the tuning of R3D_OPT_*)."""
    import reef3d_b200 as r3d
    if not ls.get_option(r3d.OPT_TILED):
        return None
    out = {}
    base = [ls.get_option(o) for o in (r3d.OPT_CHUNK, r3d.OPT_CHUNK_REINIT)]
    for kc in (8, 16, 32, 64):
        ls.set_option(r3d.OPT_CHUNK, kc)
        out[f"kc{kc}"] = {"conv_ms": device_time(ls, lambda: ls.stage(r3d.STAGE_CONVECTION, 2), reps),
                          "reinit_ms": device_time(ls, lambda: ls.stage(r3d.STAGE_REINIT, 2), reps)}
    ls.set_option(r3d.OPT_CHUNK, base[0])
    ls.set_option(r3d.OPT_CHUNK_REINIT, base[1])
    ls.set_option(r3d.OPT_BAND64, 0)
    out["band64_off_reinit_ms"] = device_time(ls, lambda: ls.stage(r3d.STAGE_REINIT, 2), reps)
    ls.set_option(r3d.OPT_BAND64, 1)
    return out


def e2e_steps(case, precision, steps, warmup):
    """Through the C-ABI with host buffers in the reference's layout, the
    way the levelset_RK3 adapter drives it: the level set
    stays on the device between steps; every step uploads the velocities
    u, v, w the host's momentum solver owns (pinned host memory), runs the
    step (CFL + RK3 convection + reinitialisation + volume) and downloads
    phi for the host's density update."""
    import torch

    import reef3d_b200 as r3d
    n = case.nx
    shape = case.phi.shape
    pinned = {}
    for name, a in (("phi", case.phi), ("u", case.u), ("v", case.v), ("w", case.w)):
        t = torch.empty(shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        pinned[name] = t
    out = torch.empty(shape, dtype=torch.float64, pin_memory=True)
    ls = r3d.LevelSet(n, n, n, case.xn, case.yn, case.zn, precision=precision, **case.flags())
    ids = (("phi", r3d.PHI), ("u", r3d.U), ("v", r3d.V), ("w", r3d.W))

    ls.upload_ptr(r3d.PHI, pinned["phi"].data_ptr())

    def one():
        for name, fid in ids[1:]:
            ls.upload_ptr(fid, pinned[name].data_ptr())
        ls.run(1, adaptive=True)
        ls.download_ptr(r3d.PHI, out.data_ptr())

    for _ in range(warmup):
        one()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    ls.close()
    nbytes = pinned["phi"].numel() * 8
    # the same host<->device traffic alone (three uploads, one download per
    # step, pinned buffers, one stream): the link's share of the step
    dev = torch.empty(shape, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(steps):
        for name in ("u", "v", "w"):
            dev.copy_(pinned[name], non_blocking=True)
        out.copy_(dev, non_blocking=True)
    torch.cuda.synchronize()
    copy_ms = (time.perf_counter() - t1) * 1e3 / steps
    del dev
    return n ** 3 * steps / el, 3 * nbytes, nbytes, copy_ms, el * 1e3 / steps


def tile_sweep(args):
    """One launch of convection and reinitialisation stage 2 per (tile
    configuration, z chunk), in that order, on the benchmark grid."""
    import reef3d_b200 as r3d
    from reef3d_b200 import setups
    case = setups.vortex3d(args.edge)
    ls = make_instance(case, r3d.FP32)
    ls.set_dt(ls.cfl_dt())
    done = []
    for cfg in range(len(r3d.tile_configs())):
        for kc in r3d.tile_chunks():
            ls.set_option(r3d.OPT_TILE_CFG, cfg)
            ls.set_option(r3d.OPT_CHUNK, kc)
            if not ls.get_option(r3d.OPT_TILED):
                continue
            ls.stage(r3d.STAGE_CONVECTION, 2)
            ls.stage(r3d.STAGE_REINIT, 2)
            done.append([cfg, kc])
    ls.sync()
    ls.close()
    print(json.dumps({"tile_sweep": done, "edge": args.edge}))


def run_ours(args):
    import torch

    import reef3d_b200 as r3d
    from reef3d_b200 import setups

    from reef3d_b200.replicas import Replicas
    ctx = Replicas()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak_gbs = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    case = setups.vortex3d(args.edge)
    cells = case.cells

    # FP32 form (headline) -------------------------------------------------
    ls32 = make_instance(case, r3d.FP32)
    # tile configuration and z chunk per stage kind, picked by timing
    # (r3d_autotune; untimed, before the warm-up)
    cfg, kc = ls32.autotune(args.tile_cache)
    tile_cfg = {"convection": {"cfg": cfg, "chunk": kc, "tile": r3d.tile_configs()[cfg]},
                "reinit": {"cfg": ls32.get_option(r3d.OPT_TILE_CFG_REINIT),
                           "chunk": ls32.get_option(r3d.OPT_CHUNK_REINIT),
                           "tile": r3d.tile_configs()[ls32.get_option(r3d.OPT_TILE_CFG_REINIT)]},
                "tile_fields": "(tx, ty, rows per thread, ring slots, threads)"}
    with ClockSampler(ctx.local) as clk:
        total32, per32, launches32 = timed_steps(ls32, args.steps, args.warmup, ctx)
    total32 = ctx.max(total32)
    roof32 = stage_roofline(ls32, cells, 4, peak_gbs)
    variants = tile_variants(ls32)
    ls32.close()
    # FP64 plain -----------------------------------------------------------
    ls64 = make_instance(case, r3d.FP64)
    total64, per64, launches64 = timed_steps(ls64, args.steps, args.warmup, ctx)
    total64 = ctx.max(total64)
    roof64 = stage_roofline(ls64, cells, 8, peak_gbs)
    ls64.close()
    # end to end through the C-ABI with host buffers ------------------------
    e2e = None
    if not args.no_e2e:
        e2e_steps_n = max(2, min(args.steps, 10))
        rate, h2d, d2h, copy_ms, step_ms = e2e_steps(case, r3d.FP32, e2e_steps_n, 1)
        e2e = {"value": rate * ctx.world, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": e2e_steps_n, "ms_per_step": step_ms,
               "copies_alone_ms_per_step": copy_ms,
               "link_gbs": (h2d + d2h) / (copy_ms * 1e-3) / 1e9,
               "path": "r3d_upload(u,v,w) + r3d_ls_run(1) + r3d_download(phi) per step (phi resident), "
                       "pinned host buffers in the reference layout, FP32 form"}
    cpu = None
    if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu:
        # the same processes (cores) as the reference arm, one step each
        procs = reference_procs(args.edge, args.steps)
        rate, info = reference_cpu(args.edge, procs, 0, procs)
        if rate is not None:
            cpu = dict(value=rate, unit="cell-updates/s", **info)
        else:
            cpu = info
    configs = None
    if ctx.rank == 0 and ctx.world == 1 and not args.no_configs:
        configs = run_configs(ctx)
    kind = "reinit" if roof32["kernel"] == "reinit_stage" else "convection"
    traffic = profiled_traffic(kind, args.edge, tile_cfg[kind]["cfg"], tile_cfg[kind]["chunk"])
    value32 = cells * args.steps * ctx.world / (total32 * 1e-3)
    value64 = cells * args.steps * ctx.world / (total64 * 1e-3)
    out = {
        "metric": METRIC, "value": value32, "unit": "cell-updates/s", "n_gpus": ctx.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total32 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "edge": args.edge, "cells_per_gpu": cells,
                   "form": "FP32 stencils/RK, FP64 CFL/volume/interface band",
                   "l2": "working set (phi, 2 stage buffers, u, v, w = 6 x 79 MB) larger than L2; no flush",
                   "parallelism": f"replicas x{ctx.world}"},
        "latency_ms": {"p50": float(np.percentile(per32, 50)), "p99": float(np.percentile(per32, 99)),
                       "what": "per-step device time of the FP32 step"},
        "fp64_plain": {"value": value64, "unit": "cell-updates/s", "ms_per_step": total64 / args.steps,
                       "dtype": "f64", "p50_ms": float(np.percentile(per64, 50)),
                       "p99_ms": float(np.percentile(per64, 99)), "roofline": roof64,
                       "gpu_launches": launches64},
        "fp32_over_fp64": value32 / value64,
        "roofline": dict(roof32, traffic=(traffic or {}).get("bytes"), traffic_detail=traffic, peak_source=peak_src),
        "tile_variants": variants,
        "tile_config": tile_cfg,
        "gpu_launches": launches32,
        "clocks": clk.summary(),
        "e2e": e2e,
        "cpu_baseline": cpu,
        "configs": configs,
    }
    if ctx.rank == 0:
        print(json.dumps(out))
    ctx.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args, int(os.environ.get("RANK", "0")))
        return
    if args.tile_sweep:
        tile_sweep(args)
        return
    run_ours(args)


if __name__ == "__main__":
    main()
