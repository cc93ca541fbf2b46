"""FP64 plain GPU path against the reference at the benchmark grid sizes.

The golden vectors (tests/golden) pin every operator bit for bit on grids of
at most 24 cells a side; this file pins the same bar on the benchmark
configurations themselves.  The GPU runs the configuration's own trajectory
(adaptive CFL step, the vortex velocity following the device clock) up to a
sampled step; its level set there is handed to the reference's own code
(oracle/_ref, built from the reference sources, in a spawned child: the
reference holds one grid per process), and both advance one step from it:

* the convection operator L (weno_hj_df_nug) and the reinitialisation
  operator L (reinidisc_f) of the sampled state bit-identical on every
  interior cell -- every upwind side, Godunov selection and frozen-band
  decision is the reference's;
* the CFL time step bit-identical (ietimestep);
* phi after the step within 1e-12 relative max-norm (observed: identical),
  volume sums within 1e-12 relative (summation order).

Configurations: the 2D slotted disc 128 x 1 x 128 (rigid rotation, CFL 0.1)
at steps 0, 500 and 2000 of its revolution; the 3D single vortex 128^3 at
steps 0, 300 and 1000; the vortex at its benchmark size 256^3 at steps 0
and 1500 (one reference step there is ~20 s on one core, ~12 GB of host
memory).
"""
import multiprocessing as mp
import os
import sys

import numpy as np
import pytest

import reef3d_b200 as r3d
from reef3d_b200 import setups
from test_gpu_parity import RTOL, relmax
from test_oracle_golden import interior, visible_mask

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _case(name, n):
    return setups.slotted_disk(n) if name == "disk" else setups.vortex3d(n)


def _reference_step(name, n, phi, u, v, w, count):
    """In a spawned child: the reference's operators on phi, its CFL step on
    (u, v, w) and one levelset_RK3 step (lexer::count = count)."""
    sys.path.insert(0, ROOT)
    from oracle.bindings import RefOracle
    c = _case(name, n)
    o = RefOracle(c.nx, c.ny, c.nz, c.xn, c.yn, c.zn, f43=c.f43, f44=c.f44, f45=c.f45, f49=c.f49)
    o.set_state(phi, u, v, w)
    conv = o.weno_L(phi)
    rein = o.reinidisc_L(phi)
    dt = o.cfl_dt(c.n47)
    o.set_count(count)
    out = o.step(dt)
    vol = o.volume()
    return conv, rein, dt, out, vol


def _velocity_at(c, t):
    if c.vel_time is None:
        return c.u, c.v, c.w
    f = c.vel_time(t)
    return tuple(np.ascontiguousarray(a * f) for a in (c.u, c.v, c.w))


def check_config(name, n, samples):
    c = _case(name, n)
    nx, ny, nz = c.nx, c.ny, c.nz
    m = visible_mask(nx, ny, nz)
    ctx = mp.get_context("spawn")
    with r3d.LevelSet(nx, ny, nz, c.xn, c.yn, c.zn, precision=r3d.FP64, **c.flags()) as ls:
        for f, a in ((r3d.PHI, c.phi), (r3d.U, c.u), (r3d.V, c.v), (r3d.W, c.w)):
            ls.upload(f, a)
        ls.set_time(0.0)
        done = 0
        for s in samples:
            # the configuration's own trajectory up to step s
            if c.vel_time is not None:
                ls.set_velocity_period(c.t_end)
                ls.set_velocity_scale(1.0)
                for f, a in ((r3d.U, c.u), (r3d.V, c.v), (r3d.W, c.w)):
                    ls.upload(f, a)
            ls.run(s - done, adaptive=True)
            phi = ls.download(r3d.PHI)
            # the compared step: the velocity of the sampled time, formed on
            # the host and given to both sides
            u, v, w = _velocity_at(c, ls.time())
            ls.set_velocity_period(0.0)
            ls.set_velocity_scale(1.0)
            for f, a in ((r3d.U, u), (r3d.V, v), (r3d.W, w)):
                ls.upload(f, a)
            with ctx.Pool(1) as pool:
                conv, rein, dt, ref, (rv1, rv2) = pool.apply(_reference_step, (name, n, phi, u, v, w, s + 1))
            ls.convection_L(r3d.PHI)
            assert np.array_equal(interior(ls.download(r3d.L), nx, ny, nz), interior(conv, nx, ny, nz)), s
            ls.reinidisc_L(r3d.PHI)
            assert np.array_equal(interior(ls.download(r3d.L), nx, ny, nz), interior(rein, nx, ny, nz)), s
            assert ls.cfl_dt() == dt, s
            ls.set_step_count(s + 1)
            ls.step()
            got = ls.download(r3d.PHI)
            assert relmax(got[m], ref[m]) <= RTOL, (s, relmax(got[m], ref[m]))
            v1, v2 = ls.last_volume()
            assert abs(v1 - rv1) <= RTOL * abs(rv1) and abs(v2 - rv2) <= RTOL * abs(rv2), s
            done = s + 1


@pytest.mark.parametrize("name,n,samples", [("disk", 128, (0, 500, 2000)), ("vortex", 128, (0, 300, 1000))])
def test_config_steps_vs_reference(name, n, samples):
    check_config(name, n, samples)


def test_vortex_256_steps_vs_reference():
    check_config("vortex", 256, (0, 1500))
