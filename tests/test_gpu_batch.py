"""Batched persistent execution (many FP32 instances, 2D and 3D mixed, one
launch per RK stage, CUDA graph).  A member's result must not depend on the
batch around it: alone and in the mix it is bit-identical (same kernels,
same per-member reductions); against the FP64 oracle it meets the FP32
tolerance of test_gpu_fp32.py."""
import numpy as np
import pytest

import reef3d_b200 as r3d
from reef3d_b200 import setups
from test_gpu_parity import relmax
from test_oracle_golden import visible_mask

pytestmark = pytest.mark.gpu


def make_member(case, precision=r3d.FP32):
    ls = r3d.LevelSet(case.nx, case.ny, case.nz, case.xn, case.yn, case.zn, precision=precision, **case.flags())
    for f, a in ((r3d.PHI, case.phi), (r3d.U, case.u), (r3d.V, case.v), (r3d.W, case.w)):
        ls.upload(f, a)
    return ls


def cases(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        out.append(setups.random_instance(rng, n_edge_choices=[16, 24, 32, 40], f44=1 + q % 2))
    return out


def run_batch(cs, steps, rows=4, ctas=8, graph=True):
    ms = [make_member(c) for c in cs]
    with r3d.Batch() as b:
        for m in ms:
            b.add(m)
        b.set_config(rows, ctas)
        b.use_graph(graph)
        b.step(steps)
        b.sync()
        res = [(m.download(r3d.PHI), m.time(), m.last_volume()) for m in ms]
    for m in ms:
        m.close()
    return res


def test_member_alone_equals_member_in_mix():
    cs = cases(0, 6)
    mix = run_batch(cs, 4)
    for q in (0, 3, 5):
        alone = run_batch([cs[q]], 4)[0]
        assert np.array_equal(alone[0], mix[q][0])
        assert alone[1] == mix[q][1]
        assert alone[2] == mix[q][2]


def test_graph_and_direct_launches_agree():
    cs = cases(1, 4)
    a = run_batch(cs, 3, graph=True)
    b = run_batch(cs, 3, graph=False)
    for x, y in zip(a, b):
        assert np.array_equal(x[0], y[0]) and x[1] == y[1]


@pytest.mark.parametrize("rows,ctas", [(2, 16), (8, 4)])
def test_configs_agree_on_phi(rows, ctas):
    cs = cases(2, 4)
    a = run_batch(cs, 2, 4, 8)
    b = run_batch(cs, 2, rows, ctas)
    for x, y in zip(a, b):
        assert np.array_equal(x[0], y[0])
        assert abs(x[2][0] - y[2][0]) <= 1e-12 * abs(x[2][0])


def test_members_match_fp64_oracle(port_lib):
    cs = cases(3, 5)
    res = run_batch(cs, 1)
    for c, (phi, t, vol) in zip(cs, res):
        o = port_lib(c.nx, c.ny, c.nz, c.xn, c.yn, c.zn, **c.flags())
        dt = o.cfl_dt(c.u, c.v, c.w)
        ref = o.step(c.phi, c.u, c.v, c.w, dt)
        m = visible_mask(c.nx, c.ny, c.nz)
        assert abs(t - dt) <= 1e-6 * dt  # FP32-stored velocities
        assert relmax(phi[m], ref[m]) <= 1e-4


def test_autotune_cache(tmp_path):
    cs = cases(4, 3)
    path = str(tmp_path / "tune.txt")
    ms = [make_member(c) for c in cs]
    with r3d.Batch() as b:
        for m in ms:
            b.add(m)
        before = [m.download(r3d.PHI) for m in ms]
        cfg = b.autotune(path)
        after = [m.download(r3d.PHI) for m in ms]
        for x, y in zip(before, after):
            assert np.array_equal(x, y)  # tuning leaves the state untouched
        assert cfg in [(r, c) for r in (2, 4, 8) for c in (4, 8, 16, 32) if r * c * 32 <= 2048]
        tcfg = b.tile_config()
        assert 0 <= tcfg[0] < len(r3d.tile_configs()) and tcfg[1] in r3d.tile_chunks()
        # one line per size class (the process-wide cache may hold others):
        # key, rows, CTAs per SM, tile configuration, z chunk
        with open(path) as f:
            lines = [ln.split() for ln in f if not ln.startswith("inst-")]
        assert len(lines) == 1 and [int(x) for x in lines[0][1:]] == [cfg[0], cfg[1], tcfg[0], tcfg[1]]
        assert b.autotune(path) == cfg and b.tile_config() == tcfg
        b.step(2)
        b.sync()
    for m in ms:
        m.close()


def test_remove_and_readd():
    cs = cases(5, 3)
    ms = [make_member(c) for c in cs]
    with r3d.Batch() as b:
        for m in ms:
            b.add(m)
        b.step(1)
        b.remove(ms[1])
        t1 = ms[1].time()
        b.step(2)
        assert ms[1].time() == t1  # removed members do not advance
        assert b.size() == 2
        b.add(ms[1])
        b.step(1)
        b.sync()
        assert ms[1].time() > t1
    for m in ms:
        m.close()


@pytest.mark.parametrize("seed", [7, 8])
def test_device_init_matches_host_setup(seed):
    rng = np.random.default_rng(seed)
    c = setups.random_instance(rng, n_edge_choices=[20, 24, 28])
    with r3d.LevelSet(c.nx, c.ny, c.nz, c.xn, c.yn, c.zn, precision=r3d.FP64, **c.flags()) as ls:
        ls.init_spheres_tg(c.spheres, c.modes)
        m = visible_mask(c.nx, c.ny, c.nz)
        if c.ny == 1:
            m[:, :3, :] = False
            m[:, 4:, :] = False
        for f, a in ((r3d.PHI, c.phi), (r3d.U, c.u), (r3d.V, c.v), (r3d.W, c.w)):
            got = ls.download(f)
            assert np.max(np.abs(got[m] - a[m])) <= 1e-12


def test_batched_tiled_member_equals_single_instance_run():
    """A 3D uniform member runs the same tiled item code in a batch as a
    single instance does on its own: identical level set and clock."""
    rng = np.random.default_rng(9)
    c = setups.random_instance(rng, two_d=False, edge=(70, 33, 41))
    single = make_member(c)
    assert single.get_option(r3d.OPT_TILED) == 1
    single.set_time(0.0)
    single.run(3, adaptive=True)
    ref = single.download(r3d.PHI)
    t_ref = single.time()
    single.close()
    res = run_batch([c] + cases(10, 3), 3)
    assert np.array_equal(res[0][0], ref)
    assert res[0][1] == t_ref
