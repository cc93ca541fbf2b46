"""The REEF3D-side adapter classes (reef3d_b200/adapters/reef3d_b200_adapters.h)
compiled against the reference's own headers and run on the reference's own
lexer / fdm / ghostcell objects (oracle/_ref/libreef3d_adapter.so): in one
process, each reference object (levelset_RK3, weno_hj_df_nug, reinidisc_f /
reinidisc_fsf, reini_RK3, fluid_update_fsf) and the adapter that replaces it
start from the same REEF3D fields, and the fields they leave behind are
compared (the tank_io cases with the reference's ioflow_f inflow / outflow
boundaries, which the adapters hand to r3d_set_ioflow; the tank_wave cases
with the reference's wave generator iowave, whose relaxation zones and
per-step targets the adapter hands to r3d_set_relaxation; the stretched_df
cases with the direct-forcing convection stencils X45 4 and 5 over the
fdm's body fields).  FP64: the level
set and the operators bit-identical on every cell
(ghost layers included: the adapters finish with REEF3D's own
ghostcell::start4), volumes, density and viscosity within 1e-12 relative
(summation order, sin); with the picard correction, whose shift comes from
those sums, the level set within 1e-12 relative.  One grid per process, so each case
runs in a spawned child.  The library is built by `python -c "import
__graft_entry__ as g; g.build()"` (oracle/Makefile.ref target `adapter`)."""
import multiprocessing as mp
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _stretched(n, amp):
    from oracle.bindings import uniform_nodes
    x = uniform_nodes(n)
    return x + amp * np.sin(2 * np.pi * x) / n


def _case(name):
    sys.path.insert(0, ROOT)
    from reef3d_b200 import setups
    if name == "vortex3d":
        c = setups.vortex3d(14)
        return dict(nx=14, ny=14, nz=14, xn=c.xn, yn=c.yn, zn=c.zn, phi=c.phi, u=c.u, v=c.v, w=c.w,
                    f43=c.f43, f44=c.f44, f45=c.f45, f49=1, n47=c.n47, f46=0)
    if name == "disk2d":
        c = setups.slotted_disk(24)
        return dict(nx=24, ny=1, nz=24, xn=c.xn, yn=c.yn, zn=c.zn, phi=c.phi, u=c.u, v=c.v, w=c.w,
                    f43=c.f43, f44=c.f44, f45=c.f45, f49=1, n47=c.n47, f46=0)
    if name.startswith("tank_io"):
        # inflow / outflow faces with ioflow_f (B60 = 1): wavy free surface
        rng = np.random.default_rng(6)
        nx, ny, nz = (16, 5, 14) if name == "tank_io3d" else (20, 1, 16)
        xn, yn, zn = _stretched(nx, 0.0), _stretched(ny, 0.0), _stretched(nz, 0.0)
        c = lambda a: 0.5 * (a[2:-3] + a[3:-2])
        X, Y, Z = np.meshgrid(c(xn), c(yn), c(zn), indexing="ij")
        phi = np.ascontiguousarray(0.5 + 0.05 * np.cos(2 * np.pi * X) - Z + 0.003 * rng.standard_normal(X.shape))
        if ny == 1:
            phi[:, :3, :] = 0.0
            phi[:, 4:, :] = 0.0
        u = np.ascontiguousarray(0.3 + 0.1 * rng.standard_normal(phi.shape))
        v, w = (np.ascontiguousarray(0.05 * rng.standard_normal(phi.shape)) for _ in range(2))
        io = dict(f50=2, b77=2, f60=0.5, f62=0.52, f64=2) if ny > 1 else dict(f50=3, b77=1)
        return dict(nx=nx, ny=ny, nz=nz, xn=xn, yn=yn, zn=zn, phi=phi, u=u, v=v, w=w, f43=0.5, f44=2, f45=2.1,
                    f49=1, n47=0.25, f46=0, io=io)
    if name.startswith("tank_wave"):
        # REEF3D's wave generator (iowave) with relaxation-zone generation
        # and beach on the x faces, still water at 0.5
        rng = np.random.default_rng(7)
        nx, ny, nz = (28, 1, 16) if name == "tank_wave2d" else (20, 5, 14)
        xn, yn, zn = _stretched(nx, 0.0), _stretched(ny, 0.0), _stretched(nz, 0.0)
        c = lambda a: 0.5 * (a[2:-3] + a[3:-2])
        X, Y, Z = np.meshgrid(c(xn), c(yn), c(zn), indexing="ij")
        phi = np.ascontiguousarray(0.5 + 0.02 * np.sin(2 * np.pi * X) - Z + 0.002 * rng.standard_normal(X.shape))
        if ny == 1:
            phi[:, :3, :] = 0.0
            phi[:, 4:, :] = 0.0
        u = np.ascontiguousarray(0.2 * np.cos(2 * np.pi * X) + 0.05 * rng.standard_normal(phi.shape))
        v, w = (np.ascontiguousarray(0.05 * rng.standard_normal(phi.shape)) for _ in range(2))
        wave = dict(b92=2, amp=0.03, period=0.8, depth=0.5, b96_1=0.25, b96_2=0.25, phimean=0.5)
        if name == "tank_wave3d_ramp":
            wave.update(b101=1, b102=2.0)
        if name == "tank_wave3d_active":
            # Dirichlet wave maker and active absorbing beach: iowave sets
            # the face velocities (host side), the level set has no zones
            wave.update(b98=3, b99=3)
        return dict(nx=nx, ny=ny, nz=nz, xn=xn, yn=yn, zn=zn, phi=phi, u=u, v=v, w=w, f43=0.5, f44=2, f45=2.1,
                    f49=1, n47=0.25, f46=0, wave=wave)
    # random 3D case on a stretched grid, F49 = 0 (reinidisc_fsf) or picard
    rng = np.random.default_rng(4)
    nx, ny, nz = 11, 9, 10
    xn, yn, zn = _stretched(nx, 0.3), _stretched(ny, 0.3), _stretched(nz, 0.3)
    c = lambda a: 0.5 * (a[2:-3] + a[3:-2])
    X, Y, Z = np.meshgrid(c(xn), c(yn), c(zn), indexing="ij")
    phi = np.sqrt((X - 0.5) ** 2 + (Y - 0.45) ** 2 + (Z - 0.55) ** 2) - 0.23
    phi = np.ascontiguousarray(phi + 0.01 * rng.standard_normal(phi.shape))
    u, v, w = (np.ascontiguousarray(rng.standard_normal(phi.shape)) for _ in range(3))
    c = dict(nx=nx, ny=ny, nz=nz, xn=xn, yn=yn, zn=zn, phi=phi, u=u, v=v, w=w, f43=0.5, f44=2, f45=2.1,
             f49=0 if name == "stretched_f49_0" else 1, n47=0.125, f46=2 if name == "stretched_picard" else 0)
    if name.startswith("stretched_df"):
        # direct-forcing stencils: X45 4 over fbh5 (harness field 10), X45 5
        # over solid and topo (11, 12)
        x45 = int(name[-1])
        shape = phi.shape
        if x45 == 4:
            b = rng.uniform(0.0, 1.0, shape)
            b[rng.uniform(size=shape) < 0.3] = 1.0
            bodies = {10: b}
        else:
            bodies = {11: rng.uniform(-0.3, 1.0, shape), 12: rng.uniform(-0.3, 1.0, shape)}
        c.update(x45=x45, bodies=bodies)
    if name == "stretched_sf":
        # solid forcing after each convection stage over a random gcdf4 list
        sides = rng.choice([1, 2, 3, 4, 5, 6], 80)
        c["sf"] = np.stack([rng.integers(0, nx, 80), rng.integers(0, ny, 80), rng.integers(0, nz, 80), sides],
                           axis=1).astype(np.int32)
    return c


def _visible(nx, ny, nz):
    i = np.arange(-3, nx + 3)[:, None, None]
    j = np.arange(-3, ny + 3)[None, :, None]
    k = np.arange(-3, nz + 3)[None, None, :]
    return ((i < 0) | (i >= nx)).astype(int) + ((j < 0) | (j >= ny)) + ((k < 0) | (k >= nz)) <= 1


def _interior(a, nx, ny, nz):
    return a[3:3 + nx, 3:3 + ny, 3:3 + nz]


def _run(name, precision=0):
    sys.path.insert(0, ROOT)
    from oracle.bindings import AdapterOracle
    c = _case(name)
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    ao = AdapterOracle(nx, ny, nz, c["xn"], c["yn"], c["zn"], f43=c["f43"], f44=c["f44"], f45=c["f45"],
                       f49=c["f49"], f46=c["f46"], f47=6, precision=precision, ioflow=c.get("io"),
                       x45=c.get("x45", 0), solid_forcing=c.get("sf"), iowave=c.get("wave"))
    out = {}
    ao.set_state(c["phi"], c["u"], c["v"], c["w"])
    for fid, arr in c.get("bodies", {}).items():
        ao.set_field(fid, np.ascontiguousarray(arr))
    out["weno_L"] = bool(np.array_equal(_interior(ao.weno_L(c["phi"]), nx, ny, nz),
                                        _interior(ao.gpu_weno_L(c["phi"]), nx, ny, nz)))
    out["reinidisc_L"] = bool(np.array_equal(_interior(ao.reinidisc_L(c["phi"]), nx, ny, nz),
                                             _interior(ao.gpu_reinidisc_L(c["phi"]), nx, ny, nz)))
    phi = c["phi"]
    out["phi"], out["rel"] = [], []
    t = 0.0
    for s in range(3):
        ao.set_count(s + 1)
        ao.set_field(0, phi)
        dt = ao.cfl_dt(c["n47"])
        if c.get("wave"):
            # the driver's order: the wave generator's targets of the step,
            # then the free surface (both adapters read the same targets)
            ao.set_time(t)
            ao.wavegen_precalc()
        ref = ao.step(dt)
        ref_ro, ref_visc, ref_vol = ao.get_field(6), ao.get_field(7), ao.volume()
        ao.set_field(0, phi)
        got = ao.gpu_step(dt)
        got_ro, got_visc = ao.get_field(6), ao.get_field(7)
        got_vol = ao.gpu_update()
        scale = max(np.max(np.abs(ref)), 1e-300)
        # With picard the shift w comes from volume sums taken in another
        # order (ulps), so phi agrees within the FP64 tolerance instead of
        # bit for bit, and the reference leaves its last (pre-shift) edge and
        # corner ghosts in place: the interior and face ghosts are compared.
        m = np.ones(ref.shape, bool) if c["f46"] == 0 else _visible(nx, ny, nz)
        out["phi"].append(bool(np.array_equal(got[m], ref[m])) or c["f46"] != 0)
        out["rel"].append(max(float(np.max(np.abs(got - ref)[m]) / scale),
                              float(np.max(np.abs(got_ro - ref_ro)) / np.max(np.abs(ref_ro))),
                              float(np.max(np.abs(got_visc - ref_visc)) / np.max(np.abs(ref_visc))),
                              abs(got_vol[0] - ref_vol[0]) / abs(ref_vol[0]),
                              abs(got_vol[1] - ref_vol[1]) / abs(ref_vol[1])))
        phi = ref
        t += dt
    ao.set_count(1)
    ao.set_field(0, 1.5 * c["phi"])
    ref = ao.reini()
    ao.set_field(0, 1.5 * c["phi"])
    got = ao.gpu_reini()
    out["reini"] = bool(np.array_equal(_interior(got, nx, ny, nz), _interior(ref, nx, ny, nz)))
    ao.close()
    return out


@pytest.mark.parametrize("name", ["vortex3d", "disk2d", "stretched_f49_0", "stretched_picard", "tank_io3d",
                                  "tank_io2d", "stretched_df4", "stretched_df5", "stretched_sf", "tank_wave2d",
                                  "tank_wave3d_ramp", "tank_wave3d_active"])
def test_adapters_match_reference_objects(name):
    from oracle.bindings import AdapterOracle
    if not AdapterOracle.available():
        pytest.fail("oracle/_ref/libreef3d_adapter.so is not built (make -f oracle/Makefile.ref adapter)")
    with mp.get_context("spawn").Pool(1) as pool:
        out = pool.apply(_run, (name,))
    assert out["weno_L"] and out["reinidisc_L"] and out["reini"], out
    assert all(out["phi"]), out
    assert max(out["rel"]) <= 1e-12, out


def _run_fp32(name):
    """The free-surface adapter in the FP32 form against the reference's FP64
    levelset_RK3 for three steps (each from the reference's state)."""
    sys.path.insert(0, ROOT)
    from oracle.bindings import AdapterOracle
    c = _case(name)
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    ao = AdapterOracle(nx, ny, nz, c["xn"], c["yn"], c["zn"], f43=c["f43"], f44=c["f44"], f45=c["f45"],
                       f49=c["f49"], f46=c["f46"], f47=6, precision=1)
    ao.set_state(c["phi"], c["u"], c["v"], c["w"])
    phi, errs = c["phi"], []
    for s in range(3):
        ao.set_count(s + 1)
        ao.set_field(0, phi)
        dt = ao.cfl_dt(c["n47"])
        ref = ao.step(dt)
        ao.set_field(0, phi)
        got = ao.gpu_step(dt)
        errs.append(float(np.max(np.abs(_interior(got - ref, nx, ny, nz))) / np.max(np.abs(ref))))
        phi = ref
    ao.close()
    return errs


@pytest.mark.parametrize("name", ["vortex3d", "disk2d"])
def test_fp32_adapter_within_fp32_tolerance(name):
    """FP32 form through the same adapter: within 2e-5 relative max-norm of
    the reference per step (the FP32 tolerance of test_gpu_fp32.py)."""
    with mp.get_context("spawn").Pool(1) as pool:
        errs = pool.apply(_run_fp32, (name,))
    assert max(errs) <= 2e-5, errs


def _run_domain(name, nslabs):
    """levelset_RK3_domain (the grid over nslabs z slabs) against the
    reference's levelset_RK3 for three steps, each from the reference's state."""
    sys.path.insert(0, ROOT)
    from oracle.bindings import AdapterOracle
    c = _case(name)
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    ao = AdapterOracle(nx, ny, nz, c["xn"], c["yn"], c["zn"], f43=c["f43"], f44=c["f44"], f45=c["f45"],
                       f49=c["f49"], f46=c["f46"], f47=6, precision=0, ioflow=c.get("io"))
    ao.make_domain(nslabs)
    ao.set_state(c["phi"], c["u"], c["v"], c["w"])
    phi, same, rel = c["phi"], [], []
    for s in range(3):
        ao.set_count(s + 1)
        ao.set_field(0, phi)
        dt = ao.cfl_dt(c["n47"])
        ref = ao.step(dt)
        ref_ro, ref_vol = ao.get_field(6), ao.volume()
        ao.set_field(0, phi)
        got = ao.gpu_step_domain(dt)
        got_ro = ao.get_field(6)
        ro_rel = float(np.max(np.abs(got_ro - ref_ro)) / np.max(np.abs(ref_ro)))
        if c["f46"] == 0:
            same.append(bool(np.array_equal(got, ref)) and ro_rel <= 1e-12)
        else:  # the picard shift from volume sums in another order; faces as in _run
            m = _visible(nx, ny, nz)
            phi_rel = float(np.max(np.abs(got - ref)[m]) / np.max(np.abs(ref)))
            same.append(phi_rel <= 1e-12 and ro_rel <= 1e-12)
        phi = ref
    ao.close()
    return same


@pytest.mark.parametrize("name,nslabs", [("vortex3d", 3), ("stretched_f49_0", 3), ("disk2d", 4),
                                         ("stretched_picard", 3), ("tank_io3d", 3), ("tank_io2d", 4)])
def test_domain_adapter_matches_reference_objects(name, nslabs):
    """The free-surface adapter over z slabs (one REEF3D process spreading its
    level set over several GPUs; here the slabs share one): the level set
    bit-identical to the reference's on every cell, ghosts included, the
    density within 1e-12 relative (the device's sin), for three steps; with
    the picard correction (F46 = 2) phi (interior and faces) and density
    within 1e-12; with ioflow_f's inflow/outflow faces (tank cases) bit for
    bit as without."""
    with mp.get_context("spawn").Pool(1) as pool:
        same = pool.apply(_run_domain, (name, nslabs))
    assert all(same), same
