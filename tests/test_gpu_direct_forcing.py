"""Direct-forcing convection stencils (X45 1..6, src/weno_hj_df_nug.cpp:
398-987) on the GPU, through r3d_set_direct_forcing: the divided
differences of every WENO5 stencil masked or weighted by a body field.  The
golden df* cases against the reference itself run in test_gpu_parity.py;
here larger cases against the C restatement (pinned bit-exact to the
reference by test_oracle_golden.py): the operator bit-identical, phi within
the FP64 tolerance of 1e-12 relative max-norm per step; the FP32 form
within the FP32 tolerance of the FP64 path (X45 6 on its own terms: its
masked differences are 1e20)."""
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


@pytest.mark.parametrize("dims", [(40, 33, 27), (64, 1, 48)])
def test_direct_forcing_6_fp32_against_fp64(dims):
    """X45 6 in the FP32 form, one step from the same state as the FP64 path
    (src/weno_hj_df_nug.cpp:868-987: a difference whose pair of cells is not
    all fluid is 1e20).  A stencil holding a masked difference has a weight
    ~1e-80 relative in FP64 and exactly 0 in FP32: cells with at least one
    stencil free of them agree within the FP32 tolerance of 2e-5 (relative
    to their largest value); cells whose three stencils all hold one get the
    reference's 1e20-scale derivative, computed in FP64 from FP32 operands:
    the same value to 1 % cell by cell (the later stages difference
    1e18-scale neighbours stored in FP32, where single-precision rounding of
    nearly equal values cancels).  One step: the reference's own 1e20-scale
    values are the masked-difference sentinel, not a level set."""
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=nx + 6)
    b1, b2 = bodies(6, phi.shape, 1.0 / nx, seed=6)
    m = visible_mask(nx, ny, nz)
    out = {}
    for prec in (r3d.FP64, r3d.FP32):
        with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=prec, f43=0.5, f44=0, f45=2.1, n47=0.125) as ls:
            ls.set_direct_forcing(6)
            ls.upload(r3d.BODY, body_field(6, b1, b2))
            for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
                ls.upload(f, a)
            ls.set_dt(0.25 / nx)
            ls.step()
            out[prec] = ls.download(r3d.PHI)[m]
    a, b = out[r3d.FP32], out[r3d.FP64]
    assert np.all(np.isfinite(a))
    huge = np.abs(b) > 1e10
    assert huge.any() and (~huge).any()
    assert relmax(a[~huge], b[~huge]) <= 2e-5
    assert np.max(np.abs(a[huge] - b[huge]) / np.abs(b[huge])) <= 1e-2


def test_direct_forcing_refusals():
    with r3d.LevelSet(16, 16, 16, precision=r3d.FP64) as ls:
        with pytest.raises(r3d.R3DError):
            ls.download(r3d.BODY)  # not enabled yet
        for bad in (-1, 7):
            with pytest.raises(r3d.R3DError):
                ls.set_direct_forcing(bad)


def sf_list(nx, ny, nz, n, seed, crowd=False):
    """Random solid-forcing entries (i, j, k, side); crowd: all on a few
    cells, so that most entries overwrite or read each other's cells."""
    rng = np.random.default_rng(seed)
    hi = (min(nx, 4), min(ny, 4), min(nz, 4)) if crowd else (nx, ny, nz)
    sides = [1, 4, 5, 6] if ny == 1 else [0, 1, 2, 3, 4, 5, 6]
    return np.stack([rng.integers(0, hi[0], n), rng.integers(0, hi[1], n), rng.integers(0, hi[2], n),
                     rng.choice(sides, n)], axis=1).astype(np.int32)


def sf_block(nx, ny, nz):
    """The list a solid block would produce (src/gcdf_update.cpp): every
    fluid cell next to a face of the block [nx/3, 2nx/3) x ... , with the
    side towards the block, so the field is carried two cells into it."""
    b = [(n // 3, 2 * n // 3) for n in (nx, ny, nz)]
    if ny == 1:
        b[1] = (0, 1)
    out = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                inb = [b[0][0] <= i < b[0][1], b[1][0] <= j < b[1][1], b[2][0] <= k < b[2][1]]
                if all(inb):
                    continue
                if inb[1] and inb[2]:
                    if i == b[0][0] - 1: out.append((i, j, k, 4))
                    if i == b[0][1]: out.append((i, j, k, 1))
                if inb[0] and inb[2] and ny > 1:
                    if j == b[1][0] - 1: out.append((i, j, k, 2))
                    if j == b[1][1]: out.append((i, j, k, 3))
                if inb[0] and inb[1]:
                    if k == b[2][0] - 1: out.append((i, j, k, 6))
                    if k == b[2][1]: out.append((i, j, k, 5))
    return np.array(out, dtype=np.int32)


@pytest.mark.parametrize("dims,kind", [((40, 33, 27), "random"), ((40, 33, 27), "crowd"), ((64, 1, 48), "crowd"),
                                       ((40, 33, 27), "block"), ((64, 1, 48), "block")])
@pytest.mark.parametrize("precision", [r3d.FP64, r3d.FP32])
def test_solid_forcing_vs_oracle(port_lib, dims, kind, precision):
    """solid_forcing_lsm after each convection stage (X48 = 1): FP64 within
    1e-12 of the restatement for every list (random and crowded ones, whose
    entries overwrite and read each other's cells, test that the list order
    survives the dependency levels); FP32 within its 2e-5 for the list of a
    solid block at 1e-3: the forcing leaves a kink two cells into the
    block, where WENO's weights turn FP32 rounding into differences of
    ~1e-4 (random lists tear the field apart further and are compared in
    FP64 only).  test_solid_forcing_copies_exactly checks the FP32 operation
    itself."""
    if precision == r3d.FP32 and kind != "block":
        pytest.skip("FP32 is compared on a physical list")
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=nx + 17)
    cells = sf_block(nx, ny, nz) if kind == "block" else sf_list(nx, ny, nz, 300, seed=nx, crowd=kind == "crowd")
    flags = dict(f43=0.5, f44=2, f45=2.1, f49=1, n47=0.125)
    o = port_lib(nx, ny, nz, xn, yn, zn, **flags)
    o.set_solid_forcing(cells)
    m = visible_mask(nx, ny, nz)
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=precision, **flags) as ls:
        ls.set_solid_forcing(cells)
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            ls.upload(f, a)
        ref = phi
        for s in range(2):
            dt = o.cfl_dt(u, v, w)
            ls.cfl_dt()
            ls.step()
            ref = o.step(ref, u, v, w, dt)
            tol = RTOL if precision == r3d.FP64 else 1e-3
            assert relmax(ls.download(r3d.PHI)[m], ref[m]) <= tol, f"step {s}"


@pytest.mark.parametrize("precision", [r3d.FP64, r3d.FP32])
def test_solid_forcing_copies_exactly(precision):
    """After a convection stage the two cells beyond each entry's side hold
    the entry cell's value, the list's last writer winning where entries
    share a target (the block's edges); block lists read only cells outside
    the block, which no entry writes."""
    nx, ny, nz = 40, 33, 27
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=23)
    cells = sf_block(nx, ny, nz)
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=precision, n47=0.125) as ls:
        ls.set_solid_forcing(cells)
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            ls.upload(f, a)
        ls.cfl_dt()
        ls.stage(r3d.STAGE_CONVECTION, 1)
        out = ls.download(r3d.WORK1)
    d = {1: (-1, 0, 0), 4: (1, 0, 0), 3: (0, -1, 0), 2: (0, 1, 0), 5: (0, 0, -1), 6: (0, 0, 1)}
    last = {}
    for i, j, k, side in cells:
        di, dj, dk = d[int(side)]
        for q in (1, 2):
            last[(i + q * di, j + q * dj, k + q * dk)] = (i, j, k)
    assert len(last) > 0
    for (ti, tj, tk), (i, j, k) in last.items():
        assert out[ti + 3, tj + 3, tk + 3] == out[i + 3, j + 3, k + 3]


def test_solid_forcing_refusals():
    with r3d.LevelSet(16, 1, 16, precision=r3d.FP64) as ls:
        with pytest.raises(r3d.R3DError):
            ls.set_solid_forcing([[3, 0, 3, 2]])  # y side of a 2D grid
        with pytest.raises(r3d.R3DError):
            ls.set_solid_forcing([[16, 0, 3, 1]])  # outside the interior
        ls.set_solid_forcing([[3, 0, 3, 1]])
        ls.set_solid_forcing([])  # off
