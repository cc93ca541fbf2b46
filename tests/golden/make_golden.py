"""Generates the golden vectors in this folder by running the REFERENCE's own
level-set code (oracle/_ref, built by oracle/Makefile.ref from the reference
sources) on small seeded cases.  One process per case: the reference keeps
its grid tables in static members.

    make -f oracle/Makefile.ref REF=$REEF3D_SRC -j8   (REEF3D_SRC: the reference sources)
    python tests/golden/make_golden.py [case name ...]   # default: every case

Each case file holds the inputs (node coordinates, control flags, phi, u, v,
w in the reference's padded layout) and the reference's outputs: WENO node
tables and metrics, the convection operator L, the reinitialisation operator
L, the wall ghost fill, the CFL time step, one full level-set step (or a
short trajectory with the time step recomputed before every step) and the
volume sums after it, with the density and viscosity fields the step's
fluid update wrote.  The picard cases run with the mass correction on
(f46 = 1 in the reinitialisation, f46 = 2 around the step, f46 = 3 the
picard_lsm form that keeps the first step's volume; f47 iterations).  The
io cases open the x-min face as an inflow and the x-max face as an outflow
boundary with the reference's ioflow_f (B60 = 1) and record the water
levels its fsfinflow measured at every step.  The df cases turn on the
direct-forcing convection stencils (X45 1..6) over random body fields; the
sf cases the solid forcing of the level set after each convection stage
(X48 = 1) over a random direct-forcing boundary list; the wave cases run
REEF3D's wave generator iowave (B90 = 1) with relaxation-zone generation and
beach (B98 = B99 = 2) and record its relaxation weights and each step's
targets and ramp.
"""
import math
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def stretched(n, amp):
    from oracle.bindings import uniform_nodes
    x = uniform_nodes(n)
    return x + amp * np.sin(2 * np.pi * x) / n


def random_case(name, nx, ny, nz, f49, stretch, seed, f46=0, f47=10):
    rng = np.random.default_rng(seed)
    xn, yn, zn = stretched(nx, stretch), stretched(ny, stretch), stretched(nz, stretch)
    shape = (nx + 6, ny + 6, nz + 6)
    ii = 0.5 * (xn[2:-3] + xn[3:-2])
    jj = 0.5 * (yn[2:-3] + yn[3:-2])
    kk = 0.5 * (zn[2:-3] + zn[3:-2])
    X, Y, Z = np.meshgrid(ii, jj, kk, indexing="ij")
    if ny == 1:
        phi = np.sqrt((X - 0.5) ** 2 + (Z - 0.55) ** 2) - 0.23
    else:
        phi = np.sqrt((X - 0.5) ** 2 + (Y - 0.45) ** 2 + (Z - 0.55) ** 2) - 0.23
    phi = phi + 0.01 * rng.standard_normal(shape)
    phi[1 + 3, :, 2 + 3] = 0.0  # exact zeros exercise the sign branches
    if ny == 1:
        # 2D: the y ghost planes of a level set are never written on this
        # path; a field initialised on its cells holds zeros there
        phi[:, :3, :] = 0.0
        phi[:, 4:, :] = 0.0
    u = rng.standard_normal(shape)
    v = rng.standard_normal(shape)
    w = rng.standard_normal(shape)
    u[::3] = 0.0  # exact zero velocity: the advec == 0 branch
    return dict(name=name, nx=nx, ny=ny, nz=nz, xn=xn, yn=yn, zn=zn, phi=phi, u=u, v=v, w=w,
                f43=0.5, f44=2, f45=2.1, f49=f49, n47=0.125, steps=1, vel_scale=None, f46=f46, f47=f47)


def tank_case(name, nx, ny, nz, f49, stretch, seed, steps, io, level=0.5, f46=0, f47=10):
    """A still-water tank with a wavy free surface phi = level + waves - z
    (not a distance: the reinitialisation moves it) and a random mean flow
    towards the outflow, for the inflow / outflow hooks."""
    rng = np.random.default_rng(seed)
    xn, yn, zn = stretched(nx, stretch), stretched(ny, stretch), stretched(nz, stretch)
    shape = (nx + 6, ny + 6, nz + 6)
    ii = 0.5 * (xn[2:-3] + xn[3:-2])
    jj = 0.5 * (yn[2:-3] + yn[3:-2])
    kk = 0.5 * (zn[2:-3] + zn[3:-2])
    X, Y, Z = np.meshgrid(ii, jj, kk, indexing="ij")
    phi = level + 0.05 * np.cos(2 * np.pi * X) + (0.02 * np.sin(2 * np.pi * Y) if ny > 1 else 0.0) - Z
    phi = phi + 0.003 * rng.standard_normal(shape)
    if ny == 1:
        phi[:, :3, :] = 0.0
        phi[:, 4:, :] = 0.0
    u = 0.3 + 0.1 * rng.standard_normal(shape)
    v = 0.1 * rng.standard_normal(shape)
    w = 0.05 * np.sin(2 * np.pi * X) + 0.02 * rng.standard_normal(shape)
    return dict(name=name, nx=nx, ny=ny, nz=nz, xn=xn, yn=yn, zn=zn, phi=phi, u=u, v=v, w=w,
                f43=0.5, f44=2, f45=2.1, f49=f49, n47=0.25, steps=steps, vel_scale=None, f46=f46, f47=f47,
                io=io)


def df_case(name, nx, ny, nz, stretch, seed, x45, steps=2):
    """Direct-forcing convection stencils (X45 1..6) with random body fields:
    body1 = fb (X45 1), fbh5 (2, 4), fbh4 (3, 6) or solid (5), body2 = topo."""
    c = random_case(name, nx, ny, nz, 1, stretch, seed)
    rng = np.random.default_rng(seed + 1000)
    shape = c["phi"].shape
    dxm = 1.0 / nx
    if x45 == 1:
        b1 = rng.uniform(-3 * dxm, 3 * dxm, shape)
    elif x45 in (2, 4):
        b1 = rng.uniform(0.0, 1.0, shape)
        b1[rng.uniform(size=shape) < 0.3] = 1.0
    elif x45 in (3, 6):
        b1 = rng.uniform(0.0, 1.0, shape)
        b1[rng.uniform(size=shape) < 0.5] = 0.0
    else:
        b1 = rng.uniform(-0.3, 1.0, shape)
    b2 = rng.uniform(-0.3, 1.0, shape) if x45 == 5 else np.zeros(shape)
    c.update(x45=x45, body1=b1, body2=b2, steps=steps)
    return c


def sf_case(name, nx, ny, nz, f49, stretch, seed, nsf, steps=2):
    """Solid forcing after each convection stage (X48 = 1) with a random
    gcdf4 list: entries on random interior cells with random sides (some 0:
    skipped), so that entries overwrite each other's targets and read cells
    other entries wrote."""
    c = random_case(name, nx, ny, nz, f49, stretch, seed)
    rng = np.random.default_rng(seed + 2000)
    sides = [1, 4, 5, 6] if ny == 1 else [0, 1, 2, 3, 4, 5, 6]
    cells = np.stack([rng.integers(0, nx, nsf), rng.integers(0, ny, nsf), rng.integers(0, nz, nsf),
                      rng.choice(sides, nsf)], axis=1).astype(np.int32)
    c.update(sf=cells, steps=steps)
    return c


def wave_case(name, nx, ny, nz, f49, steps, wave, seed):
    """A wave tank on the unit box (still water at 0.5) with REEF3D's wave
    generator: linear waves relaxed in over the x-min zone, a relaxation
    beach before the x-max face (iowave, B98 = B99 = 2), and a level set
    slightly off the still water with a random flow."""
    rng = np.random.default_rng(seed)
    xn, yn, zn = stretched(nx, 0.0), stretched(ny, 0.0), stretched(nz, 0.0)
    shape = (nx + 6, ny + 6, nz + 6)
    ii = 0.5 * (xn[2:-3] + xn[3:-2])
    jj = 0.5 * (yn[2:-3] + yn[3:-2])
    kk = 0.5 * (zn[2:-3] + zn[3:-2])
    X, Y, Z = np.meshgrid(ii, jj, kk, indexing="ij")
    phi = wave["phimean"] + 0.02 * np.sin(2 * np.pi * X) - Z + 0.002 * rng.standard_normal(shape)
    if ny == 1:
        phi[:, :3, :] = 0.0
        phi[:, 4:, :] = 0.0
    u = 0.2 * np.cos(2 * np.pi * X) + 0.05 * rng.standard_normal(shape)
    v = 0.05 * rng.standard_normal(shape)
    w = 0.1 * np.sin(2 * np.pi * X) + 0.02 * rng.standard_normal(shape)
    return dict(name=name, nx=nx, ny=ny, nz=nz, xn=xn, yn=yn, zn=zn, phi=phi, u=u, v=v, w=w,
                f43=0.5, f44=2, f45=2.1, f49=f49, n47=0.25, steps=steps, vel_scale=None, f46=0, f47=10,
                wave=wave)


def setup_case(name, which, n, steps, f46=0, f47=10):
    from reef3d_b200 import setups
    c = setups.slotted_disk(n) if which == "disk" else setups.vortex3d(n)
    d = dict(name=name, nx=c.nx, ny=c.ny, nz=c.nz, xn=c.xn, yn=c.yn, zn=c.zn, phi=c.phi, u=c.u, v=c.v,
             w=c.w, f43=c.f43, f44=c.f44, f45=c.f45, f49=c.f49, n47=c.n47, steps=steps,
             vel_scale="vortex" if which == "vortex" else None, f46=f46, f47=f47)
    return d


CASES = [
    lambda: random_case("box3d_uniform_f49_1", 9, 7, 8, 1, 0.0, 1),
    lambda: random_case("box3d_stretched_f49_0", 9, 7, 8, 0, 0.3, 2),
    lambda: random_case("box2d_uniform_f49_1", 12, 1, 10, 1, 0.0, 3),
    lambda: random_case("box2d_stretched_f49_0", 12, 1, 10, 0, 0.3, 4),
    lambda: setup_case("vortex3d_n12_3steps", "vortex", 12, 3),
    lambda: setup_case("slotted2d_n24_3steps", "disk", 24, 3),
    lambda: random_case("picard2_box3d_stretched_f49_1", 9, 7, 8, 1, 0.3, 5, f46=2, f47=10),
    lambda: setup_case("picard2_vortex3d_n12_3steps", "vortex", 12, 3, f46=2, f47=10),
    lambda: setup_case("picard1_slotted2d_n24_3steps", "disk", 24, 3, f46=1, f47=4),
    lambda: setup_case("picard3_vortex3d_n12_3steps", "vortex", 12, 3, f46=3, f47=10),
    lambda: tank_case("io_tank3d_f50_2", 20, 6, 16, 1, 0.0, 11, 4, dict(f50=2, b77=1)),
    lambda: tank_case("io_tank2d_f50_2_b77_2_ramp", 24, 1, 18, 0, 0.0, 12, 4,
                      dict(f50=2, b77=2, f60=0.5, f62=0.52, f64=3)),
    lambda: tank_case("io_tank3d_f50_3_lsm_discharge", 18, 5, 14, 1, 0.3, 13, 4,
                      dict(f50=3, b77=2, f62=0.53, qi=0.01, qo=0.02), f46=3, f47=4),
    lambda: tank_case("io_tank3d_f50_4_top_edge", 16, 5, 16, 0, 0.0, 14, 3, dict(f50=4), level=0.955),
    lambda: tank_case("io_tank2d_f50_1_outflow_only", 22, 1, 16, 1, 0.3, 15, 3,
                      dict(f50=1, inflow=0, b77=2, f62=-0.1)),
    lambda: tank_case("io_tank3d_inflow_only_picard2", 16, 6, 14, 1, 0.0, 16, 3,
                      dict(f50=2, outflow=0), f46=2, f47=3),
    lambda: df_case("df1_box3d_stretched", 9, 7, 8, 0.3, 21, 1),
    lambda: df_case("df2_box2d_uniform", 12, 1, 10, 0.0, 22, 2),
    lambda: df_case("df3_box3d_uniform", 9, 7, 8, 0.0, 23, 3),
    lambda: df_case("df4_box3d_stretched", 9, 7, 8, 0.3, 24, 4),
    lambda: df_case("df5_box2d_stretched", 12, 1, 10, 0.3, 25, 5),
    lambda: df_case("df6_box3d_uniform", 9, 7, 8, 0.0, 26, 6),
    lambda: sf_case("sf_box3d_stretched_f49_1", 9, 7, 8, 1, 0.3, 31, 60),
    lambda: sf_case("sf_box2d_uniform_f49_0", 12, 1, 10, 0, 0.0, 32, 40),
    lambda: wave_case("wave_tank2d_relax", 32, 1, 16, 1, 4,
                      dict(b92=2, amp=0.03, period=0.8, depth=0.5, b96_1=0.25, b96_2=0.25, phimean=0.5,
                           b101=0, b102=1.0), 41),
    lambda: wave_case("wave_tank3d_relax_ramp", 24, 5, 14, 0, 3,
                      dict(b92=2, amp=0.04, period=0.7, depth=0.5, b96_1=0.3, b96_2=0.2, phimean=0.5,
                           b101=1, b102=2.0), 42),
]


def run_case(idx):
    from oracle.bindings import RefOracle
    c = CASES[idx]()
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    io = c.get("io")
    x45 = c.get("x45", 0)
    wave = c.get("wave")
    ref = RefOracle(nx, ny, nz, c["xn"], c["yn"], c["zn"], f43=c["f43"], f44=c["f44"], f45=c["f45"],
                    f49=c["f49"], f46=c["f46"], f47=c["f47"], ioflow=io, x45=x45, solid_forcing=c.get("sf"),
                    iowave=wave)
    out = {k: c[k] for k in ("nx", "ny", "nz", "xn", "yn", "zn", "phi", "u", "v", "w", "f43", "f44", "f45",
                              "f49", "n47", "steps", "f46", "f47")}
    for a, n in enumerate((nx, ny, nz)):
        qf, cf, isf = ref.weno_tables(a, n + 8)
        out[f"qf{a}"], out[f"cf{a}"], out[f"isf{a}"] = qf, cf, isf
        for w, name in ((a, "dxn"), (a + 3, "dxp")):
            out[f"{name}{a}"] = ref.metric(w, n + 11)
    if io is not None:
        from oracle.bindings import IOFLOW_DEFAULTS
        for k, val in dict(IOFLOW_DEFAULTS, **io).items():
            out["io_" + k] = val
    if c.get("sf") is not None:
        out["sf"] = c["sf"]
    if wave is not None:
        for k, val in wave.items():
            out["wave_" + k] = val
        out["wave_wgen"], out["wave_wbeach"] = ref.iowave_weights()
    out["psi"] = ref.psi
    out["vel_scale"] = np.array(c["vel_scale"] or "none")
    phi, u, v, w = c["phi"], c["u"], c["v"], c["w"]
    ref.set_state(phi, u, v, w)
    if x45:
        # harness field ids 8..12 = fb, fbh4, fbh5, solid, topo
        ref.set_field({1: 8, 2: 10, 3: 9, 4: 10, 5: 11, 6: 9}[x45], c["body1"])
        if x45 == 5:
            ref.set_field(12, c["body2"])
        out["x45"], out["body1"], out["body2"] = x45, c["body1"], c["body2"]
    out["weno_L"] = ref.weno_L(phi)
    out["reinidisc_L"] = ref.reinidisc_L(phi)
    out["ghost"] = ref.ghost_fill(phi)
    T = 3.0
    t = 0.0
    traj, dts, vols, ros, viscs, levels, targets, ramps = [], [], [], [], [], [], [], []
    for s in range(c["steps"]):
        if c["vel_scale"] == "vortex":
            f = math.cos(math.pi * t / T)
            ref.set_field(1, u * f)
            ref.set_field(2, v * f)
            ref.set_field(3, w * f)
        dt = ref.cfl_dt(c["n47"])
        ref.set_count(s + 1)  # lexer::count of the driver loop (read by picard_lsm)
        if wave is not None:
            # the driver's order: the wave generator's targets at the step's
            # clock (src/driver_loop_cfd.cpp:78), then the free surface
            ref.set_time(t)
            ref.wavegen_precalc()
            lsval, ramp = ref.iowave_targets()
            targets.append(lsval)
            ramps.append(ramp)
        ph = ref.step(dt)
        ros.append(ref.get_field(6))   # fluid_update_fsf inside the step (W1..W4 defaults)
        viscs.append(ref.get_field(7))
        traj.append(ph)
        levels.append(ref.io_levels())
        dts.append(dt)
        vols.append(ref.volume())
        t += dt
    out["step_phi"] = np.array(traj)
    out["step_dt"] = np.array(dts)
    out["step_volume"] = np.array(vols)
    out["step_ro"] = np.array(ros)
    out["step_visc"] = np.array(viscs)
    if io is not None:
        out["step_io_levels"] = np.array(levels)
    if wave is not None:
        out["step_wave_targets"] = np.array(targets)
        out["step_wave_ramp"] = np.array(ramps)
    np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), **out)
    return c["name"]


def main(names=()):
    ctx = mp.get_context("spawn")
    for i in range(len(CASES)):
        if names and CASES[i]()["name"] not in names:
            continue
        with ctx.Pool(1) as pool:
            print("wrote", pool.apply(run_case, (i,)))


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
