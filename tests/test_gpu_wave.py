"""Wave-tank runs: the device's Airy velocity generator against the same
closed form in numpy (reef3d_b200.setups.wave_tank), and FP64 steps with it
against the C restatement given the numpy velocity of each step's start
time (the reference holds a->u fixed through levelset_RK3::start, so the
velocity of a step is the one at its start)."""
import numpy as np
import pytest

import reef3d_b200 as r3d
from reef3d_b200 import setups
from test_gpu_parity import RTOL, relmax
from test_oracle_golden import visible_mask

pytestmark = pytest.mark.gpu

TANK = dict(nx=48, ny=5, nz=30, dx=0.05, depth=0.5, amp=0.05, wavelength=2.0)


def tank(t=0.0, velocity=True):
    return setups.wave_tank(**TANK, t=t, velocity=velocity)


@pytest.mark.parametrize("precision,tol", [(r3d.FP64, 1e-13), (r3d.FP32, 2e-7)])
def test_airy_generator_matches_closed_form(precision, tol):
    t = 0.37
    c = tank(t)
    with r3d.LevelSet(c.nx, c.ny, c.nz, c.xn, c.yn, c.zn, precision=precision, **c.flags()) as ls:
        ls.upload(r3d.V, np.ones_like(c.u))
        ls.set_time(t)
        ls.set_velocity_airy(TANK["amp"], TANK["wavelength"], TANK["depth"], 9.81)
        u, v, w = ls.download(r3d.U), ls.download(r3d.V), ls.download(r3d.W)
    m = visible_mask(c.nx, c.ny, c.nz)
    assert relmax(u[m], c.u[m]) <= tol
    assert relmax(w[m], c.w[m]) <= tol
    assert not np.any(v)


def test_wave_steps_vs_oracle(port_lib):
    c = tank(0.0)
    flags = c.flags()
    o = port_lib(c.nx, c.ny, c.nz, c.xn, c.yn, c.zn, **flags)
    m = visible_mask(c.nx, c.ny, c.nz)
    dt = 0.5 * o.cfl_dt(c.u, c.v, c.w)
    ref = c.phi
    with r3d.LevelSet(c.nx, c.ny, c.nz, c.xn, c.yn, c.zn, precision=r3d.FP64, **flags) as ls:
        ls.upload(r3d.PHI, c.phi)
        ls.set_time(0.0)
        ls.set_velocity_airy(TANK["amp"], TANK["wavelength"], TANK["depth"], 9.81)
        for s in range(4):
            cs = tank(s * dt)
            ls.step(dt)
            ref = o.step(ref, cs.u, cs.v, cs.w, dt)
            got = ls.download(r3d.PHI)
            assert relmax(got[m], ref[m]) <= RTOL, f"step {s}"
        assert abs(ls.time() - 4 * dt) <= 1e-15


def test_wave_run_adaptive_graph_equals_direct():
    """r3d_ls_run with the generator: the CFL step sees the velocity of the
    step's start time; graph replay and single launches agree."""
    c = tank(0.0, velocity=False)
    out = []
    for n_per_call in (6, 1):
        with r3d.LevelSet(c.nx, c.ny, c.nz, c.xn, c.yn, c.zn, precision=r3d.FP32, **c.flags()) as ls:
            ls.upload(r3d.PHI, c.phi)
            ls.set_time(0.0)
            ls.set_velocity_airy(TANK["amp"], TANK["wavelength"], TANK["depth"], 9.81)
            for _ in range(6 // n_per_call):
                ls.run(n_per_call, adaptive=True)
            out.append((ls.download(r3d.PHI), ls.time()))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]
    assert out[0][1] > 0.0
