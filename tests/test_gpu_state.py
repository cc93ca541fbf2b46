"""Checkpoint and resume of device-resident instances (r3d_save_state /
r3d_load_state): a run saved after some steps and resumed in a fresh
instance continues bit for bit as the uninterrupted run, in both
arithmetic forms and with the fluid update, picard_lsm (whose target volume
and step count are state) and inflow/outflow faces (whose water levels and
step count are state); loading refuses another grid or configuration."""
import numpy as np
import pytest

import reef3d_b200 as r3d
from test_gpu_ioflow import tank

pytestmark = pytest.mark.gpu


def configure(ls, extras):
    if extras:
        ls.set_fluid()
        ls.set_ioflow(f50=2, b77=2, f60=0.5, f62=0.52, f64=6)


@pytest.mark.parametrize("precision,extras", [(r3d.FP64, False), (r3d.FP32, False), (r3d.FP64, True)])
def test_resumed_run_continues_bit_for_bit(precision, extras, tmp_path):
    nx, ny, nz = 48, 16, 40
    xn, yn, zn, phi, (u, v, w) = tank(nx, ny, nz, seed=12)
    flags = dict(f43=0.5, f44=2, f45=2.1, n47=0.25, precision=precision, f46=3 if extras else 0, f47=3)
    path = str(tmp_path / "run.r3d")
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, **flags) as a:
        configure(a, extras)
        for f, arr in ((r3d.PHI, phi), (r3d.U, u), (r3d.V, v), (r3d.W, w)):
            a.upload(f, arr)
        a.run(3, adaptive=True)
        a.save_state(path)
        a.run(2, adaptive=True)
        ref = {f: a.download(f) for f in ((r3d.PHI, r3d.RO) if extras else (r3d.PHI,))}
        ref_vol, ref_t = a.last_volume(), a.time()
        ref_levels = a.io_levels() if extras else None
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, **flags) as b:
        configure(b, extras)
        b.load_state(path)
        b.run(2, adaptive=True)
        for f, arr in ref.items():
            assert np.array_equal(b.download(f), arr), f
        assert b.last_volume() == ref_vol and b.time() == ref_t
        if extras:
            assert b.io_levels() == ref_levels


def test_load_refuses_other_grid_or_configuration(tmp_path):
    path = str(tmp_path / "s.r3d")
    with r3d.LevelSet(24, 16, 20, precision=r3d.FP64) as a:
        a.save_state(path)
    with r3d.LevelSet(24, 16, 21, precision=r3d.FP64) as b:
        with pytest.raises(r3d.R3DError):
            b.load_state(path)
    with r3d.LevelSet(24, 16, 20, precision=r3d.FP32) as b:
        with pytest.raises(r3d.R3DError):
            b.load_state(path)
    with r3d.LevelSet(24, 16, 20, precision=r3d.FP64) as b:
        b.set_fluid()
        with pytest.raises(r3d.R3DError):
            b.load_state(path)
    bad = tmp_path / "bad.r3d"
    bad.write_bytes(b"not a state file at all" * 10)
    with r3d.LevelSet(24, 16, 20, precision=r3d.FP64) as b:
        with pytest.raises(r3d.R3DError):
            b.load_state(str(bad))
