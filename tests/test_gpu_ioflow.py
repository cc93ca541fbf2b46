"""Inflow / outflow faces with REEF3D's ioflow_f level-set hooks on the GPU
(r3d_set_ioflow): fsfinflow's water levels and ghost values, fsfrkin /
fsfrkout on the RK buffers and the ghost labels of gcval 50+F50
(src/ioflow_waterlevel.cpp:29-177, src/gc_epol4.cpp:26-58).  The golden
io_* cases against the reference itself run in test_gpu_parity.py; here
larger cases against the C restatement (pinned bit-exact to the reference
by test_oracle_golden.py): FP64 within the path's 1e-12 relative max-norm
per step with the water levels within the same bound, FP32 within its
2e-5 tolerance of the FP64 result."""
import numpy as np
import pytest

import reef3d_b200 as r3d
from test_gpu_parity import RTOL, levels_close, relmax
from test_oracle_golden import visible_mask

pytestmark = pytest.mark.gpu

FP32_TOL = 2e-5


def tank(nx, ny, nz, seed, level=0.5, stretch=0.0):
    """Wavy free surface phi = level + waves - z and a mean flow towards the
    outflow; node coordinates for -5..n+5."""
    rng = np.random.default_rng(seed)

    def nodes(n):
        x = r3d.uniform_nodes(n)
        return x + stretch * np.sin(2 * np.pi * x) / n

    xn, yn, zn = nodes(nx), nodes(ny) if ny > 1 else r3d.uniform_nodes(1, 1.0 / nx), nodes(nz)
    c = lambda a: 0.5 * (a[2:-3] + a[3:-2])
    X, Y, Z = np.meshgrid(c(xn), c(yn), c(zn), indexing="ij")
    phi = level + 0.05 * np.cos(2 * np.pi * X) + (0.02 * np.sin(2 * np.pi * Y) if ny > 1 else 0.0) - Z
    phi = np.ascontiguousarray(phi + 0.003 * rng.standard_normal(phi.shape))
    if ny == 1:
        phi[:, :3, :] = 0.0
        phi[:, 4:, :] = 0.0
    u = np.ascontiguousarray(0.3 + 0.1 * rng.standard_normal(phi.shape))
    v = np.ascontiguousarray(0.1 * rng.standard_normal(phi.shape))
    w = np.ascontiguousarray(0.05 * np.sin(2 * np.pi * X) + 0.02 * rng.standard_normal(phi.shape))
    return xn, yn, zn, phi, (u, v, w)


IO_CASES = [
    ((48, 20, 40), dict(f50=2, b77=1), 1, 0),
    ((48, 20, 40), dict(f50=2, b77=2, f60=0.5, f62=0.52, f64=3), 0, 0),
    ((40, 16, 36), dict(f50=3, b77=2, f62=0.53, qi=0.01, qo=0.02), 1, 3),
    ((64, 1, 48), dict(f50=4), 0, 2),
    ((64, 1, 48), dict(f50=1, inflow=0, b77=2, f62=-0.1), 1, 0),
    ((40, 18, 32), dict(f50=2, outflow=0), 1, 1),
]


@pytest.mark.parametrize("dims,io,f49,f46", IO_CASES)
def test_io_steps_vs_oracle(port_lib, dims, io, f49, f46):
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = tank(nx, ny, nz, seed=nx + f46, stretch=0.2 if f46 == 3 else 0.0)
    flags = dict(f43=0.5, f44=2, f45=2.1, f49=f49, n47=0.25, f46=f46, f47=4)
    o = port_lib(nx, ny, nz, xn, yn, zn, ioflow=io, **flags)
    m = visible_mask(nx, ny, nz)
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=r3d.FP64, **flags) as ls:
        ls.set_ioflow(**io)
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
            assert levels_close(ls.io_levels(), o.io_levels()), (s, ls.io_levels(), o.io_levels())


@pytest.mark.parametrize("io", [dict(f50=2, b77=2, f62=0.52), dict(f50=3)])
def test_io_reinit_vs_oracle(port_lib, io):
    """r3d_reinit alone: fsfrkin/fsfrkout at its start, the face labels on
    every pseudo-stage (src/reini_RK3.cpp:107-137)."""
    nx, ny, nz = 36, 14, 30
    xn, yn, zn, phi, _ = tank(nx, ny, nz, seed=7)
    phi = np.ascontiguousarray(1.6 * phi)
    flags = dict(f43=0.5, f44=3, f45=2.1, f49=0, n47=0.25)
    o = port_lib(nx, ny, nz, xn, yn, zn, ioflow=io, **flags)
    m = visible_mask(nx, ny, nz)
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=r3d.FP64, **flags) as ls:
        ls.set_ioflow(**io)
        ls.upload(r3d.PHI, phi)
        ls.reinit(4)
        got = ls.download(r3d.PHI)
    assert relmax(got[m], o.reini(phi, 4)[m]) <= RTOL


def test_io_step_count_drives_outflow_ramp(port_lib):
    """The F64 ramp of the outflow level reads lexer::count: a run that
    starts at count 2 matches the oracle started there."""
    nx, ny, nz = 40, 1, 32
    io = dict(f50=2, b77=2, f60=0.45, f62=0.55, f64=6)
    xn, yn, zn, phi, (u, v, w) = tank(nx, ny, nz, seed=3)
    flags = dict(f43=0.5, f44=2, f45=2.1, f49=1, n47=0.25)
    o = port_lib(nx, ny, nz, xn, yn, zn, ioflow=io, **flags)
    o.set_count(2)
    m = visible_mask(nx, ny, nz)
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=r3d.FP64, **flags) as ls:
        ls.set_ioflow(**io)
        ls.set_step_count(2)
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            ls.upload(f, a)
        ref = phi
        for s in range(3):
            dt = o.cfl_dt(u, v, w)
            ls.cfl_dt()
            ls.step()
            ref = o.step(ref, u, v, w, dt)
            got = ls.download(r3d.PHI)
            # the outflow ghosts hold the ramped level: compared exactly
            assert np.array_equal(got[nx + 3:, 3, 3:3 + nz], ref[nx + 3:, 3, 3:3 + nz]), s
            assert relmax(got[m], ref[m]) <= RTOL


def test_io_graph_replay_equals_direct_steps():
    nx, ny, nz = 48, 12, 40
    io = dict(f50=2, b77=2, f60=0.5, f62=0.52, f64=4)
    xn, yn, zn, phi, (u, v, w) = tank(nx, ny, nz, seed=5)
    out = []
    for graph in (False, True):
        with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=r3d.FP64, f43=0.5, f44=2, f45=2.1, n47=0.25,
                          f46=3, f47=3) as ls:
            ls.set_ioflow(**io)
            for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
                ls.upload(f, a)
            if graph:
                ls.run(4, adaptive=True)
            else:
                for _ in range(4):
                    ls.cfl_dt()
                    ls.step()
            out.append((ls.download(r3d.PHI), ls.io_levels()))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]


def test_io_fp32_within_tolerance_of_fp64():
    """FP32 form with inflow/outflow faces (one-cell-per-thread kernels:
    the tiled path fills every face as a wall and is not used)."""
    nx, ny, nz = 64, 24, 48
    io = dict(f50=2, b77=2, f62=0.52)
    xn, yn, zn, phi, (u, v, w) = tank(nx, ny, nz, seed=9)
    m = visible_mask(nx, ny, nz)
    res = {}
    for prec in (r3d.FP64, r3d.FP32):
        with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=prec, f43=0.5, f44=2, f45=2.1, n47=0.25) as ls:
            if prec == r3d.FP32:
                assert ls.get_option(r3d.OPT_TILED) == 1
            ls.set_ioflow(**io)
            if prec == r3d.FP32:
                assert ls.get_option(r3d.OPT_TILED) == 0
            for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
                ls.upload(f, a)
            ls.cfl_dt()
            ls.step()
            res[prec] = (ls.download(r3d.PHI), ls.io_levels())
    assert relmax(res[r3d.FP32][0][m], res[r3d.FP64][0][m]) <= FP32_TOL
    assert all(abs(a - b) <= 1e-5 * abs(b) for a, b in zip(res[r3d.FP32][1], res[r3d.FP64][1]))


def test_io_off_restores_closed_box():
    nx, ny, nz = 32, 10, 24
    xn, yn, zn, phi, (u, v, w) = tank(nx, ny, nz, seed=2)
    out = []
    for toggle in (False, True):
        with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=r3d.FP64, f43=0.5, f44=2, f45=2.1, n47=0.25) as ls:
            if toggle:
                ls.set_ioflow(f50=3)
                ls.set_ioflow(off=True)
            for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
                ls.upload(f, a)
            ls.cfl_dt()
            ls.step()
            out.append(ls.download(r3d.PHI))
            with pytest.raises(r3d.R3DError):
                ls.io_levels()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("bad", [dict(f50=0), dict(f50=5), dict(b77=3), dict(inflow=2), dict(f64=-1)])
def test_io_rejects_bad_flags(bad):
    with r3d.LevelSet(16, 8, 16, precision=r3d.FP64) as ls:
        with pytest.raises(r3d.R3DError):
            ls.set_ioflow(**bad)


def test_io_instance_refused_by_batches():
    with r3d.LevelSet(16, 16, 16, precision=r3d.FP32) as ls:
        ls.set_ioflow()
        b = r3d.Batch()
        with pytest.raises(r3d.R3DError):
            b.add(ls)
        b.close()
