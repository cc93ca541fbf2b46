"""FP64 plain GPU path against the reference, through the C-ABI.

Golden vectors come from the reference's own code (tests/golden); larger
cases compare against the C restatement oracle (itself pinned bit-exact to
the reference by test_oracle_golden.py).  The bar is the FP64 tolerance of
the path: relative max-norm <= 1e-12 on phi per step; the time step, the
branch decisions (upwind side, Godunov selection, frozen interface cells)
and the index mapping are exact, which the tests check as bit-equality of
the operator outputs.
"""
import numpy as np
import pytest

import reef3d_b200 as r3d
from conftest import (GOLDEN_CASES, body_field, golden_df, golden_flags, golden_ioflow, golden_sf, golden_wave,
                      load_golden, velocity_at)
from test_oracle_golden import interior, visible_mask

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def relmax(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def make_gpu(g, precision=r3d.FP64):
    ls = r3d.LevelSet(int(g["nx"]), int(g["ny"]), int(g["nz"]), g["xn"], g["yn"], g["zn"], precision=precision,
                      **golden_flags(g))
    io = golden_ioflow(g)
    wave = golden_wave(g)
    if wave is not None:  # inflow / outflow faces of iowave with its relaxation zones
        ls.set_ioflow(waves=True, **io)
        ls.set_relaxation(wave[0], wave[1], wave[2])
    elif io is not None:  # inflow / outflow faces with ioflow_f's hooks
        ls.set_ioflow(**io)
    df = golden_df(g)
    if df is not None:  # direct-forcing convection stencils (X45)
        ls.set_direct_forcing(df[0])
        ls.upload(r3d.BODY, body_field(*df))
    if golden_sf(g) is not None:  # solid forcing after each convection stage (X48)
        ls.set_solid_forcing(golden_sf(g))
    return ls


def wave_targets(ls, g, s):
    """The wave generator's targets of step s (wave golden cases)."""
    wave = golden_wave(g)
    if wave is not None:
        ls.set_relaxation_target(wave[3][s], float(wave[4][s]))


def levels_close(got, ref):
    return all(a == b or abs(a - b) <= RTOL * abs(b) for a, b in zip(got, ref))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_operators_bit_exact_vs_reference(name):
    g = load_golden(name)
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    with make_gpu(g) as ls:
        for f, a in ((r3d.PHI, g["phi"]), (r3d.U, g["u"]), (r3d.V, g["v"]), (r3d.W, g["w"])):
            ls.upload(f, a)
        ls.convection_L(r3d.PHI)
        L = ls.download(r3d.L)
        assert np.array_equal(interior(L, nx, ny, nz), interior(g["weno_L"], nx, ny, nz))
        ls.reinidisc_L(r3d.PHI)
        R = ls.download(r3d.L)
        assert np.array_equal(interior(R, nx, ny, nz), interior(g["reinidisc_L"], nx, ny, nz))
        ls.ghost_fill(r3d.PHI)
        G = ls.download(r3d.PHI)
        m = visible_mask(nx, ny, nz)
        assert np.array_equal(G[m], g["ghost"][m])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_steps_vs_reference(name):
    g = load_golden(name)
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    m = visible_mask(nx, ny, nz)
    t = 0.0
    with make_gpu(g) as ls:
        ls.upload(r3d.PHI, g["phi"])
        for s in range(int(g["steps"])):
            u, v, w = velocity_at(g, t)
            ls.upload(r3d.U, u)
            ls.upload(r3d.V, v)
            ls.upload(r3d.W, w)
            dt = ls.cfl_dt()
            assert dt == float(g["step_dt"][s])  # exact max reduction and dt expression
            wave_targets(ls, g, s)
            ls.step()
            phi = ls.download(r3d.PHI)
            ref = g["step_phi"][s]
            assert relmax(phi[m], ref[m]) <= RTOL
            v1, v2 = ls.last_volume()
            rv1, rv2 = g["step_volume"][s]
            assert abs(v1 - rv1) <= RTOL * abs(rv1) and abs(v2 - rv2) <= RTOL * abs(rv2)
            if "step_io_levels" in g:  # water levels measured by fsfinflow
                assert levels_close(ls.io_levels(), g["step_io_levels"][s]), (s, ls.io_levels())
            t += dt


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_fluid_update_vs_reference(name):
    """ro and visc written by the step's fluid update (fluid_update_fsf with
    the reference's default W1..W4) against the reference's own fields."""
    g = load_golden(name)
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    m = visible_mask(nx, ny, nz)
    t = 0.0
    with make_gpu(g) as ls:
        ls.set_fluid()
        ls.upload(r3d.PHI, g["phi"])
        for s in range(int(g["steps"])):
            u, v, w = velocity_at(g, t)
            for f, a in ((r3d.U, u), (r3d.V, v), (r3d.W, w)):
                ls.upload(f, a)
            t += ls.cfl_dt()
            wave_targets(ls, g, s)
            ls.step()
            for fid, key in ((r3d.RO, "step_ro"), (r3d.VISC, "step_visc")):
                got, ref = ls.download(fid), g[key][s]
                assert relmax(got[m], ref[m]) <= RTOL, (key, s)
            assert relmax(ls.download(r3d.PHI)[m], g["step_phi"][s][m]) <= RTOL
            v1, v2 = ls.last_volume()
            rv1, rv2 = g["step_volume"][s]
            assert abs(v1 - rv1) <= RTOL * abs(rv1) and abs(v2 - rv2) <= RTOL * abs(rv2)
        assert ls.fluid_update() == ls.last_volume()


def random_state(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    xn = r3d.uniform_nodes(nx)
    yn = r3d.uniform_nodes(ny) if ny > 1 else r3d.uniform_nodes(1, 1.0 / nx)
    zn = r3d.uniform_nodes(nz)
    c = lambda a: 0.5 * (a[2:-3] + a[3:-2])
    X, Y, Z = np.meshgrid(c(xn), c(yn), c(zn), indexing="ij")
    if ny == 1:
        phi = np.sqrt((X - 0.45) ** 2 + (Z - 0.5) ** 2) - 0.27
    else:
        phi = np.sqrt((X - 0.45) ** 2 + (Y - 0.5) ** 2 + (Z - 0.55) ** 2) - 0.27
    phi = np.ascontiguousarray(phi + 0.002 * rng.standard_normal(phi.shape))
    if ny == 1:  # 2D: the y ghost planes hold zeros (never written on the path)
        phi[:, :3, :] = 0.0
        phi[:, 4:, :] = 0.0
    vel = [np.ascontiguousarray(0.5 + rng.standard_normal(phi.shape)) for _ in range(3)]
    return xn, yn, zn, phi, vel


@pytest.mark.parametrize("dims,f49", [((40, 33, 27), 1), ((40, 33, 27), 0), ((64, 1, 48), 1), ((37, 1, 29), 0)])
def test_multi_step_vs_oracle(port_lib, dims, f49):
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=nx + f49)
    flags = dict(f43=0.5, f44=2, f45=2.1, f49=f49, n47=0.125)
    o = port_lib(nx, ny, nz, xn, yn, zn, **flags)
    m = visible_mask(nx, ny, nz)
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=r3d.FP64, **flags) as ls:
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            ls.upload(f, a)
        ref = phi
        for s in range(4):
            dt = o.cfl_dt(u, v, w)
            assert ls.cfl_dt() == dt
            ls.step()
            ref = o.step(ref, u, v, w, dt)
            got = ls.download(r3d.PHI)
            assert relmax(got[m], ref[m]) <= RTOL, f"step {s}"
        ls.convection_L(r3d.PHI)
        assert np.array_equal(interior(ls.download(r3d.L), nx, ny, nz),
                              interior(o.weno_L(ls.download(r3d.PHI), u, v, w), nx, ny, nz))


def test_dense_layout_roundtrip():
    nx, ny, nz = 19, 11, 7
    rng = np.random.default_rng(5)
    with r3d.LevelSet(nx, ny, nz, precision=r3d.FP64) as ls:
        a = rng.standard_normal((nz, ny, nx))
        ls.upload(r3d.PHI, a, layout=r3d.LAYOUT_DENSE)
        assert np.array_equal(ls.download(r3d.PHI, layout=r3d.LAYOUT_DENSE), a)
        b = ls.download(r3d.PHI)
        assert np.array_equal(b[3:3 + nx, 3:3 + ny, 3:3 + nz], a.transpose(2, 1, 0))


@pytest.mark.parametrize("precision,extras", [(r3d.FP64, False), (r3d.FP32, False), (r3d.FP64, True),
                                              (r3d.FP32, True)])
def test_graph_replayed_run_equals_direct_steps(precision, extras):
    """r3d_ls_run(n >= 2) replays one captured step; the result equals the
    same steps launched one by one (also with picard_lsm and the fluid
    update in the step, whose counters and fields live on the device)."""
    nx, ny, nz = 36, 30, 28
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=21)
    out = []
    for graph in (True, False):
        with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=precision, f43=0.5, f44=2, n47=0.125,
                          f46=3 if extras else 0, f47=4) as ls:
            if extras:
                ls.set_fluid()
            for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
                ls.upload(f, a)
            ls.set_velocity_period(3.0)
            ls.set_time(0.0)
            if graph:
                ls.run(4, adaptive=True)
            else:
                for _ in range(4):
                    ls.run(1, adaptive=True)
            out.append((ls.download(r3d.PHI), ls.time(), ls.last_volume(),
                        ls.download(r3d.RO) if extras else None))
    assert np.array_equal(out[0][0], out[1][0])
    if extras:
        assert np.array_equal(out[0][3], out[1][3])
    assert out[0][1] == out[1][1] and out[0][2] == out[1][2]

