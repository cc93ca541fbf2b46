"""Picard mass correction (src/picard_f.cpp, src/picard_lsm.cpp) on the GPU,
through the C-ABI: f46 = 2 around each step (levelset_RK3), f46 = 1 around
each reinitialisation (reini_RK3), f46 = 3 the picard_lsm form.  FP64 against the C restatement at 1e-12
relative max-norm per step (the golden cases against the reference itself
run in test_gpu_parity.py); FP32 through the property the correction exists
for: the smoothed-Heaviside volume at the end of a step equals the one at its
start."""
import numpy as np
import pytest

import reef3d_b200 as r3d
from test_gpu_parity import RTOL, random_state, relmax
from test_oracle_golden import visible_mask

pytestmark = pytest.mark.gpu


def picard_volume(phi, nx, ny, nz, f45, dxm):
    """volcalc of src/picard_f.cpp:36-56 in numpy (a test-side check)."""
    b = phi[3:3 + nx, 3:3 + ny, 3:3 + nz]
    epsi = f45 * dxm
    H = np.where(b > epsi, 1.0, 0.0)
    band = np.abs(b) <= epsi
    H[band] = 0.5 * (1.0 + b[band] / epsi + (1.0 / 3.14159265359) * np.sin((3.14159265359 * b[band]) / epsi))
    return float(np.sum(H) * dxm ** 3)


@pytest.mark.parametrize("dims,f46", [((40, 33, 27), 2), ((40, 33, 27), 1), ((40, 33, 27), 3), ((64, 1, 48), 2),
                                      ((37, 1, 29), 1), ((37, 1, 29), 3)])
def test_picard_steps_vs_oracle(port_lib, dims, f46):
    nx, ny, nz = dims
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=nx + 7 * f46)
    flags = dict(f43=0.5, f44=2, f45=2.1, f49=1, n47=0.125, f46=f46, f47=6)
    o = port_lib(nx, ny, nz, xn, yn, zn, **flags)
    m = visible_mask(nx, ny, nz)
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=r3d.FP64, **flags) as ls:
        for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            ls.upload(f, a)
        ref = phi
        for s in range(3):
            dt = o.cfl_dt(u, v, w)
            assert ls.cfl_dt() == dt
            ls.step()
            ref = o.step(ref, u, v, w, dt)
            got = ls.download(r3d.PHI)
            assert relmax(got[m], ref[m]) <= RTOL, f"step {s}"
            v1, v2 = ls.last_volume()
            r1, r2 = o.volume(ref)
            assert abs(v1 - r1) <= RTOL * abs(r1) and abs(v2 - r2) <= RTOL * abs(r2)


def test_picard_reinit_vs_oracle(port_lib):
    """r3d_reinit with f46 = 1 wraps the pseudo-steps in volcalc/correct_ls."""
    nx, ny, nz = 33, 29, 31
    xn, yn, zn, phi, (u, v, w) = random_state(nx, ny, nz, seed=3)
    phi = np.ascontiguousarray(1.7 * phi)  # not a distance: reinitialisation moves it
    flags = dict(f43=0.5, f44=3, f45=2.1, f49=0, n47=0.125, f46=1, f47=8)
    o = port_lib(nx, ny, nz, xn, yn, zn, **flags)
    m = visible_mask(nx, ny, nz)
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=r3d.FP64, **flags) as ls:
        ls.upload(r3d.PHI, phi)
        ls.reinit(5)
        got = ls.download(r3d.PHI)
    ref = o.reini(phi, 5)
    assert relmax(got[m], ref[m]) <= RTOL


@pytest.mark.parametrize("precision", [r3d.FP64, r3d.FP32])
def test_picard_restores_step_volume(precision):
    """f46 = 2: the picard volume after the correction equals the one at the
    step start.  The positive region is a (perturbed) sphere, for which the
    equivalent-sphere radius difference r1 - r2 is the exact interface shift,
    so ten iterations reach the fixed point r(vol2) = r(vol1)."""
    n = 96
    xn, yn, zn, phi, (u, v, w) = random_state(n, n, n, seed=11)
    phi = np.ascontiguousarray(-phi)
    dxm = 1.0 / n
    out = {}
    for f46 in (0, 2):
        with r3d.LevelSet(n, n, n, xn, yn, zn, precision=precision, f43=0.5, f44=2, f45=2.1, n47=0.25,
                          f46=f46, f47=10) as ls:
            for f, a in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
                ls.upload(f, a)
            ls.cfl_dt()
            ls.step()
            out[f46] = ls.download(r3d.PHI)
    v0 = picard_volume(phi, n, n, n, 2.1, dxm)
    drift_off = abs(picard_volume(out[0], n, n, n, 2.1, dxm) - v0) / v0
    drift_on = abs(picard_volume(out[2], n, n, n, 2.1, dxm) - v0) / v0
    tol = 1e-12 if precision == r3d.FP64 else 2e-6
    assert drift_on <= tol, (drift_on, drift_off)
    assert drift_on < drift_off


def test_picard_rejected_in_batches():
    n = 16
    with r3d.LevelSet(n, n, n, precision=r3d.FP32, f46=2) as ls:
        b = r3d.Batch()
        with pytest.raises(r3d.R3DError):
            b.add(ls)
        b.close()


@pytest.mark.parametrize("what", ["fluid", "airy"])
def test_batch_refuses_per_instance_extras(what):
    """The batched step has no fluid update and no velocity generator: an
    instance that needs either is refused, not advanced without it."""
    n = 16
    with r3d.LevelSet(n, n, n, precision=r3d.FP32) as ls:
        if what == "fluid":
            ls.set_fluid()
        else:
            ls.set_velocity_airy(0.05, 2.0, 0.5)
        b = r3d.Batch()
        with pytest.raises(r3d.R3DError):
            b.add(ls)
        b.close()
