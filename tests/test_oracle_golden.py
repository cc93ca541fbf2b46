"""The C restatement oracle (oracle/ls_oracle.c) against the golden vectors
the reference's own code produced (tests/golden/make_golden.py): bit-exact
on every value the path reads or writes (interior cells and the face ghost
layers; edge and corner ghosts are outside every stencil of the path)."""
import numpy as np
import pytest

from conftest import (GOLDEN_CASES, golden_df, golden_flags, golden_ioflow, golden_sf, golden_wave, load_golden,
                      velocity_at)


def visible_mask(nx, ny, nz):
    i = np.arange(-3, nx + 3)[:, None, None]
    j = np.arange(-3, ny + 3)[None, :, None]
    k = np.arange(-3, nz + 3)[None, None, :]
    out = ((i < 0) | (i >= nx)).astype(int) + ((j < 0) | (j >= ny)).astype(int) + ((k < 0) | (k >= nz)).astype(int)
    return out <= 1


def interior(a, nx, ny, nz):
    return a[3:3 + nx, 3:3 + ny, 3:3 + nz]


@pytest.fixture(params=GOLDEN_CASES)
def case(request, port_lib):
    g = load_golden(request.param)
    o = port_lib(int(g["nx"]), int(g["ny"]), int(g["nz"]), g["xn"], g["yn"], g["zn"], ioflow=golden_ioflow(g),
                 **golden_flags(g))
    df = golden_df(g)
    if df is not None:  # direct-forcing convection stencils (X45)
        o.set_direct_forcing(*df)
    if golden_sf(g) is not None:  # solid forcing after each convection stage (X48)
        o.set_solid_forcing(golden_sf(g))
    wave = golden_wave(g)
    if wave is not None:  # iowave's faces and relaxation zones
        o.set_io_waves()
        o.set_relaxation(wave[0], wave[1], wave[2])
    return g, o


def test_tables_and_metrics(case):
    g, o = case
    for a, n in enumerate((int(g["nx"]), int(g["ny"]), int(g["nz"]))):
        qf, cf, isf = o.weno_tables(a, n + 8)
        assert np.array_equal(qf, g[f"qf{a}"]) and np.array_equal(cf, g[f"cf{a}"])
        assert np.array_equal(isf, g[f"isf{a}"])
        assert np.array_equal(o.metric(a, n + 11), g[f"dxn{a}"])
        assert np.array_equal(o.metric(a + 3, n + 11), g[f"dxp{a}"])
    assert o.psi == float(g["psi"])


def test_operators(case):
    g, o = case
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    L = o.weno_L(g["phi"], g["u"], g["v"], g["w"])
    assert np.array_equal(interior(L, nx, ny, nz), interior(g["weno_L"], nx, ny, nz))
    R = o.reinidisc_L(g["phi"])
    assert np.array_equal(interior(R, nx, ny, nz), interior(g["reinidisc_L"], nx, ny, nz))
    G = o.ghost_fill(g["phi"])
    m = visible_mask(nx, ny, nz)
    assert np.array_equal(G[m], g["ghost"][m])


def test_steps_dt_volume(case):
    g, o = case
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    m = visible_mask(nx, ny, nz)
    phi = g["phi"]
    t = 0.0
    for s in range(int(g["steps"])):
        u, v, w = velocity_at(g, t)
        dt = o.cfl_dt(u, v, w)
        assert dt == g["step_dt"][s]
        wave = golden_wave(g)
        if wave is not None:  # the wave generator's targets of the step
            o.set_relaxation_target(wave[3][s], float(wave[4][s]))
        phi = o.step(phi, u, v, w, dt)
        assert np.array_equal(phi[m], g["step_phi"][s][m])
        assert o.volume(phi) == tuple(g["step_volume"][s])
        if "step_io_levels" in g:
            assert o.io_levels() == tuple(g["step_io_levels"][s])
        ro, visc = o.fluid(phi)
        assert np.array_equal(ro[m], g["step_ro"][s][m]) and np.array_equal(visc[m], g["step_visc"][s][m])
        t += dt
