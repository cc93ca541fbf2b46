"""Slab decomposition along z (reef3d_b200.slab, r3d_set_halo /
r3d_halo_copy): a grid split into 2-4 slabs, the halo of REEF3D's MPI
exchange (src/gcx_parax.cpp) moved after every RK stage, steps the same as
the undivided grid -- the level set bit-identical (every cell computes the
same operations on the same inputs), the CFL time step identical, the
volume sums within 1e-12 relative (summed per slab, then over slabs)."""
import numpy as np
import pytest

import reef3d_b200 as r3d
from conftest import body_field
from reef3d_b200.slab import LocalSlabs, split
from test_gpu_direct_forcing import bodies
from test_gpu_parity import RTOL, random_state
from test_oracle_golden import visible_mask

pytestmark = pytest.mark.gpu


def run_whole(dims, precision, steps, flags, fluid=False, df=None):
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=nz)
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=precision, **flags) as ls:
        if fluid:
            ls.set_fluid()
        if df is not None:
            ls.set_direct_forcing(df[0])
            ls.upload(r3d.BODY, body_field(*df))
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            ls.upload(f, a)
        dts, vols = [], []
        for _ in range(steps):
            dts.append(ls.cfl_dt())
            ls.step()
            vols.append(ls.last_volume())
        out = {f: ls.download(f) for f in ((r3d.PHI, r3d.RO, r3d.VISC) if fluid else (r3d.PHI,))}
    return out, dts, vols


def run_slabs(dims, precision, steps, flags, nslabs, fluid=False, df=None):
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=nz)
    d = LocalSlabs(nx, ny, nz, xn, yn, zn, nslabs, precision=precision, fluid=fluid, **flags)
    try:
        if df is not None:
            for ls in d.slabs:
                ls.set_direct_forcing(df[0])
            d.upload(r3d.BODY, body_field(*df))
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            d.upload(f, a)
        dts, vols = [], []
        for _ in range(steps):
            dts.append(d.cfl_dt())
            vols.append(d.step())
        out = {f: d.download(f) for f in ((r3d.PHI, r3d.RO, r3d.VISC) if fluid else (r3d.PHI,))}
    finally:
        d.close()
    return out, dts, vols


FLAGS = dict(f43=0.5, f44=2, f45=2.1, f49=1, n47=0.125)


@pytest.mark.parametrize("dims,nslabs", [((40, 33, 27), 2), ((40, 33, 27), 4), ((64, 1, 48), 3), ((48, 40, 64), 3)])
@pytest.mark.parametrize("precision", [r3d.FP64, r3d.FP32])
def test_slabs_equal_undivided_grid(dims, nslabs, precision):
    flags = dict(FLAGS, f49=0 if nslabs == 3 else 1)
    whole, dts, vols = run_whole(dims, precision, 3, flags)
    parts, dts_s, vols_s = run_slabs(dims, precision, 3, flags, nslabs)
    m = visible_mask(*dims)
    assert dts == dts_s
    assert np.array_equal(whole[r3d.PHI][m], parts[r3d.PHI][m])
    for (a, b), (c, d) in zip(vols, vols_s):
        assert abs(a - c) <= RTOL * abs(a) and abs(b - d) <= RTOL * abs(b)


def test_slabs_with_fluid_update_and_direct_forcing():
    dims = (36, 20, 30)
    df = (2,) + bodies(2, (dims[0] + 6, dims[1] + 6, dims[2] + 6), 1.0 / dims[0], seed=8)
    whole, dts, _ = run_whole(dims, r3d.FP64, 2, FLAGS, fluid=True, df=df)
    parts, dts_s, _ = run_slabs(dims, r3d.FP64, 2, FLAGS, 3, fluid=True, df=df)
    m = visible_mask(*dims)
    assert dts == dts_s
    for f in (r3d.PHI, r3d.RO, r3d.VISC):
        assert np.array_equal(whole[f][m], parts[f][m]), f


def test_slab_split_and_refusals():
    assert split(10, 3) == [(0, 4), (4, 7), (7, 10)]
    with pytest.raises(ValueError):
        split(8, 3)
    with r3d.LevelSet(16, 16, 16, precision=r3d.FP64, f46=2) as ls:
        with pytest.raises(r3d.R3DError):
            ls.set_halo(1, 0)  # picard sums are global inside the step
    with r3d.LevelSet(16, 16, 16, precision=r3d.FP64) as ls:
        ls.set_halo(0, 1)
        with pytest.raises(r3d.R3DError):
            ls.set_ioflow()
        b = r3d.Batch()
        with pytest.raises(r3d.R3DError):
            b.add(ls)
        b.close()


@pytest.mark.parametrize("dims,nslabs", [((40, 33, 27), 3), ((64, 1, 48), 4), ((48, 40, 64), 2)])
@pytest.mark.parametrize("precision", [r3d.FP64, r3d.FP32])
def test_native_domain_equals_undivided_grid(dims, nslabs, precision):
    """The native slab runner (r3d_domain_*: all stages, halo copies and the
    global CFL step in one CUDA graph) steps as the undivided grid: phi
    bit-identical, the adaptive dt identical, volumes within 1e-12."""
    from reef3d_b200.slab import Domain
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=nz)
    whole, dts, vols = run_whole(dims, precision, 3, FLAGS)
    # explicit device list: the peer-copy path of the multi-GPU layout, here
    # with every slab on device 0
    with Domain(nx, ny, nz, xn, yn, zn, nslabs=nslabs, precision=precision, devices=[0] * nslabs, **FLAGS) as d:
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            d.upload(f, a)
        for s in range(3):
            d.run(1)  # adaptive
            assert d.dt() == dts[s]
            a, b = d.last_volume()
            assert abs(a - vols[s][0]) <= RTOL * abs(vols[s][0]) and abs(b - vols[s][1]) <= RTOL * abs(vols[s][1])
        got = d.download(r3d.PHI)
    m = visible_mask(*dims)
    assert np.array_equal(got[m], whole[r3d.PHI][m])


@pytest.mark.parametrize("precision", [r3d.FP64, r3d.FP32])
def test_native_domain_reconfigured_between_runs(precision):
    """Settings changed on the slabs after the domain's step graph was
    captured (new fluid densities, direct-forcing stencils switched on and
    then changed to another X45) reach the next run: the domain keeps stepping as the undivided grid given the same
    settings at the same points."""
    from reef3d_b200.slab import Domain
    dims = (36, 20, 30)
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=31)
    df2 = (2,) + bodies(2, (nx + 6, ny + 6, nz + 6), 1.0 / nx, seed=8)
    df3 = (3,) + bodies(3, (nx + 6, ny + 6, nz + 6), 1.0 / nx, seed=9)
    dens = [(998.2, 1.004e-6, 1.205, 1.41e-5), (1025.0, 1.2e-6, 1.0, 1.5e-5)]

    def script(obj, run, set_df):
        obj.set_fluid(*dens[0])
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            obj.upload(f, a)
        run(2)
        obj.set_fluid(*dens[1])
        run(1)
        set_df(df2)
        run(2)
        set_df(df3)
        run(1)
        return {f: obj.download(f) for f in (r3d.PHI, r3d.RO, r3d.VISC)}

    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=precision, **FLAGS) as ls:
        def whole_df(df):
            ls.set_direct_forcing(df[0])
            ls.upload(r3d.BODY, body_field(*df))
        whole = script(ls, lambda n: ls.run(n, adaptive=True), whole_df)
    with Domain(nx, ny, nz, xn, yn, zn, nslabs=3, precision=precision, devices=[0] * 3, **FLAGS) as d:
        def dom_df(df):
            d.set_direct_forcing(df[0])
            d.upload(r3d.BODY, body_field(*df))
        parts = script(d, lambda n: d.run(n), dom_df)
    m = visible_mask(*dims)
    for f in (r3d.PHI, r3d.RO, r3d.VISC):
        assert np.array_equal(whole[f][m], parts[f][m]), f


@pytest.mark.parametrize("f46,nslabs,precision", [(1, 3, r3d.FP64), (2, 3, r3d.FP64), (3, 4, r3d.FP64),
                                                  (2, 1, r3d.FP64), (3, 3, r3d.FP32)])
def test_native_domain_picard_equals_undivided_grid(f46, nslabs, precision):
    """The picard correction over the slabs (picard_f with F46 = 1 around the
    reinitialisation and 2 around the step, picard_lsm with 3): each
    iteration's volume summed per slab, then over the slabs, w taken from the
    grid's volume and the phi halos refreshed after the shift.  The step then
    equals the undivided grid's up to the volume sums' order (phi within
    1e-12 of its largest value in FP64, and bit-identical with one slab; a
    few single-precision roundings of the shifted values in FP32)."""
    from reef3d_b200.slab import Domain
    dims = (40, 33, 27)
    nx, ny, nz = dims
    flags = dict(FLAGS, f46=f46, f47=3)
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=nz)
    whole, dts, vols = run_whole(dims, precision, 3, flags)
    with Domain(nx, ny, nz, xn, yn, zn, nslabs=nslabs, precision=precision, devices=[0] * nslabs, **flags) as d:
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            d.upload(f, a)
        for s in range(3):
            d.run(1)
            assert d.dt() == dts[s]
            a, b = d.last_volume()
            assert abs(a - vols[s][0]) <= RTOL * abs(vols[s][0]) and abs(b - vols[s][1]) <= RTOL * abs(vols[s][1])
        got = d.download(r3d.PHI)
    m = visible_mask(*dims)
    ref = whole[r3d.PHI][m]
    if nslabs == 1:
        assert np.array_equal(got[m], ref)
    tol = (1e-12 if precision == r3d.FP64 else 1e-5) * np.abs(ref).max()
    assert np.abs(got[m] - ref).max() <= tol
    # the correction moved the level set: the run without it ends elsewhere
    plain, _, _ = run_whole(dims, precision, 3, FLAGS)
    assert np.abs(plain[r3d.PHI][m] - ref).max() > 10 * tol


@pytest.mark.parametrize("case,nslabs,precision", [(0, 3, r3d.FP64), (1, 4, r3d.FP64), (2, 3, r3d.FP64),
                                                   (3, 3, r3d.FP64), (1, 3, r3d.FP32), (5, 2, r3d.FP64)])
def test_native_domain_ioflow_equals_undivided_grid(case, nslabs, precision):
    """Inflow/outflow faces over the slabs (r3d_domain_set_ioflow): the
    crossing heights of every slab gathered into the whole grid's order and
    folded once, so the water levels and the step count are the undivided
    grid's bit for bit and so is phi (within 1e-12 of its largest value with
    the picard correction, whose volumes are summed per slab)."""
    from reef3d_b200.slab import Domain
    from test_gpu_ioflow import IO_CASES, tank
    dims, io, f49, f46 = IO_CASES[case]
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = tank(nx, ny, nz, seed=nx + f46, stretch=0.2 if f46 == 3 else 0.0)
    flags = dict(f43=0.5, f44=2, f45=2.1, f49=f49, n47=0.25, f46=f46, f47=3)
    count = 1 if f46 == 3 else 2  # picard_lsm takes its target volume at count 1
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=precision, **flags) as ls:
        ls.set_ioflow(**io)
        ls.set_step_count(count)
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            ls.upload(f, a)
        dts, levels = [], []
        for _ in range(3):
            dts.append(ls.cfl_dt())
            ls.step()
            levels.append(ls.io_levels())
        ref = ls.download(r3d.PHI)
    with Domain(nx, ny, nz, xn, yn, zn, nslabs=nslabs, precision=precision, devices=[0] * nslabs, **flags) as d:
        d.set_ioflow(**io)
        d.set_step_count(count)
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            d.upload(f, a)
        for s in range(3):
            d.run(1)
            assert d.dt() == dts[s]
            if f46 == 0:
                assert d.io_levels() == levels[s]
            else:
                assert np.allclose(d.io_levels(), levels[s], rtol=1e-12, atol=0)
        got = d.download(r3d.PHI)
    m = visible_mask(*dims)
    assert np.isfinite(ref[m]).all()
    if f46 == 0:
        assert np.array_equal(got[m], ref[m])
    else:
        assert np.abs(got[m] - ref[m]).max() <= 1e-12 * np.abs(ref[m]).max()
