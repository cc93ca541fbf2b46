"""Direct-forcing convection stencils (X45 1..6, src/weno_hj_df_nug.cpp:
398-987) on the GPU, through r3d_set_direct_forcing: the divided
differences of every WENO5 stencil masked or weighted by a body field.  The
golden df* cases against the reference itself run in test_gpu_parity.py;
here larger cases against the C restatement (pinned bit-exact to the
reference by test_oracle_golden.py): the operator bit-identical, phi within
the FP64 tolerance of 1e-12 relative max-norm per step; the FP32 form
(X45 1..5) within the FP32 tolerance of the FP64 path."""
import numpy as np
import pytest

import reef3d_b200 as r3d
from conftest import body_field
from test_gpu_parity import RTOL, random_state, relmax
from test_oracle_golden import interior, visible_mask

pytestmark = pytest.mark.gpu


def bodies(x45, shape, dxm, seed):
    """body1 = fb (X45 1), fbh5 (2, 4), fbh4 (3, 6) or solid (5); body2 = topo."""
    rng = np.random.default_rng(seed)
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
    b2 = rng.uniform(-0.3, 1.0, shape)
    return np.ascontiguousarray(b1), np.ascontiguousarray(b2)


@pytest.mark.parametrize("x45", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("dims", [(40, 33, 27), (64, 1, 48)])
def test_direct_forcing_vs_oracle(port_lib, x45, dims):
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=nx + x45)
    b1, b2 = bodies(x45, phi.shape, 1.0 / nx, seed=x45)
    flags = dict(f43=0.5, f44=2, f45=2.1, f49=1, n47=0.125)
    o = port_lib(nx, ny, nz, xn, yn, zn, **flags)
    o.set_direct_forcing(x45, b1, b2)
    m = visible_mask(nx, ny, nz)
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=r3d.FP64, **flags) as ls:
        ls.set_direct_forcing(x45)
        ls.upload(r3d.BODY, body_field(x45, b1, b2))
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            ls.upload(f, a)
        ls.convection_L(r3d.PHI)
        assert np.array_equal(interior(ls.download(r3d.L), nx, ny, nz),
                              interior(o.weno_L(phi, u, v, w), nx, ny, nz))
        ref = phi
        for s in range(2):
            dt = o.cfl_dt(u, v, w)
            assert ls.cfl_dt() == dt
            ls.step()
            ref = o.step(ref, u, v, w, dt)
            assert relmax(ls.download(r3d.PHI)[m], ref[m]) <= RTOL, f"step {s}"


def test_direct_forcing_off_restores_plain_stencils():
    nx, ny, nz = 32, 20, 24
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=4)
    b1, _ = bodies(3, phi.shape, 1.0 / nx, seed=4)
    out = []
    for toggle in (False, True):
        with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=r3d.FP64, n47=0.125) as ls:
            for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
                ls.upload(f, a)
            if toggle:
                ls.set_direct_forcing(3)
                ls.upload(r3d.BODY, b1)
                ls.convection_L(r3d.PHI)
                with_df = ls.download(r3d.L)
                ls.set_direct_forcing(0)
            ls.convection_L(r3d.PHI)
            out.append(ls.download(r3d.L))
    assert np.array_equal(out[0], out[1])
    assert not np.array_equal(interior(with_df, nx, ny, nz), interior(out[0], nx, ny, nz))


def test_direct_forcing_graph_replay_equals_direct_steps():
    nx, ny, nz = 40, 24, 32
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=6)
    b1, _ = bodies(2, phi.shape, 1.0 / nx, seed=6)
    out = []
    for graph in (False, True):
        with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=r3d.FP64, n47=0.125) as ls:
            ls.set_direct_forcing(2)
            ls.upload(r3d.BODY, b1)
            for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
                ls.upload(f, a)
            if graph:
                ls.run(3, adaptive=True)
            else:
                for _ in range(3):
                    ls.cfl_dt()
                    ls.step()
            out.append(ls.download(r3d.PHI))
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("x45", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("dims", [(40, 33, 27), (64, 1, 48)])
def test_direct_forcing_fp32_within_tolerance_of_fp64(x45, dims):
    """The FP32 form of the X45 stencils (one-cell-per-thread table kernels;
    mask decisions on the FP64 body field) within the FP32 tolerance of the
    FP64 path, 2e-5 relative max-norm per step."""
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=nx + x45)
    b1, b2 = bodies(x45, phi.shape, 1.0 / nx, seed=x45)
    m = visible_mask(nx, ny, nz)
    out = {}
    for prec in (r3d.FP64, r3d.FP32):
        with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=prec, f43=0.5, f44=2, f45=2.1, n47=0.125) as ls:
            ls.set_direct_forcing(x45)
            ls.upload(r3d.BODY, body_field(x45, b1, b2))
            # the body field stays FP64 in both forms
            assert np.array_equal(interior(ls.download(r3d.BODY), nx, ny, nz),
                                  interior(body_field(x45, b1, b2), nx, ny, nz))
            if prec == r3d.FP32:
                assert ls.get_option(r3d.OPT_TILED) == 0
            for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
                ls.upload(f, a)
            res = []
            for _ in range(2):
                ls.cfl_dt()
                ls.step()
                res.append(ls.download(r3d.PHI))
            out[prec] = res
    for a, b in zip(out[r3d.FP32], out[r3d.FP64]):
        assert relmax(a[m], b[m]) <= 2e-5


def test_direct_forcing_refusals():
    with r3d.LevelSet(16, 16, 16, precision=r3d.FP32) as ls:
        with pytest.raises(r3d.R3DError):
            ls.set_direct_forcing(6)  # 1e20 differences overflow FP32: FP64 only
    with r3d.LevelSet(16, 16, 16, precision=r3d.FP64) as ls:
        with pytest.raises(r3d.R3DError):
            ls.download(r3d.BODY)  # not enabled yet
        for bad in (-1, 7):
            with pytest.raises(r3d.R3DError):
                ls.set_direct_forcing(bad)
