"""The reference's restart state file (cfd_state, src/cfd_state_write.cpp:
34-146 and src/cfd_state_read.cpp:44-195).

The reference's own writer and reader (oracle/_ref, built from the reference
sources, run in a spawned child) pin the layout: its file for a known state
is decoded here block by block (CPU).  On the GPU, r3d_write_reef3d_state
writes the same bytes for the same state, and r3d_read_reef3d_state loads the
reference's file: the level set and the velocities (rounded to single
precision, as the file holds them) and the other fields."""
import multiprocessing as mp
import os
import struct
import sys

import numpy as np
import pytest

import reef3d_b200 as r3d

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle.bindings import REF_LIB  # noqa: E402

CASES = {"box3d": (12, 10, 8), "disk2d": (20, 1, 16)}
HEADER = struct.Struct("=ii6d")
# harness field ids (oracle/ref_harness.cpp): phi, u, v, w, topo, press, eddyv, conc
FID = {"phi": 0, "u": 1, "v": 2, "w": 3, "topo": 12, "press": 13, "eddyv": 14, "conc": 15}

needs_ref = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built")


def grid(name):
    nx, ny, nz = CASES[name]
    xn = r3d.uniform_nodes(nx)
    yn = r3d.uniform_nodes(ny) if ny > 1 else r3d.uniform_nodes(1, 1.0 / nx)
    zn = r3d.uniform_nodes(nz)
    return nx, ny, nz, xn, yn, zn


def padded(nx, ny, nz):
    return (nx + 6, ny + 6, nz + 6)


def state_fields(name, seed=3):
    """Random padded fields (the reference's layout) of every field the
    file holds that the harness can set."""
    nx, ny, nz = CASES[name]
    rng = np.random.default_rng(seed)
    return {k: rng.uniform(-1.0, 1.0, padded(nx, ny, nz)) for k in FID}


def interior(a, nx, ny, nz):
    return a[3:3 + nx, 3:3 + ny, 3:3 + nz]


def blocks(nx, ny, nz):
    """(name, count) of the file's float blocks: ulast = vlast = wlast = 1."""
    c = nx * ny * nz
    return [("topo", c), ("u", (nx - 1) * ny * nz), ("v", nx * (ny - 1) * nz), ("w", nx * ny * (nz - 1)),
            ("press", c), ("phi", c), ("kin", c), ("eps", c), ("eddyv", c), ("qbe", nx * ny), ("conc", c)]


def loop_order(a, nx, ny, nz, ex=(0, 0, 0)):
    """Interior values of a padded field in the reference's loop order (i
    outermost, k innermost), the far face dropped along the axis ex marks."""
    return interior(a, nx, ny, nz)[:nx - ex[0], :ny - ex[1], :nz - ex[2]].reshape(-1)


def _ref_write_read(name, directory):
    sys.path.insert(0, ROOT)
    from oracle.bindings import RefOracle
    nx, ny, nz, xn, yn, zn = grid(name)
    o = RefOracle(nx, ny, nz, xn, yn, zn)
    f = state_fields(name)
    for k, fid in FID.items():
        o.set_field(fid, f[k])
    path = o.write_state(directory, 17, 4, 0.625)
    for fid in FID.values():
        o.set_field(fid, np.zeros(padded(nx, ny, nz)))
    count, simtime = o.read_state(directory, 0)
    back = {k: o.get_field(fid) for k, fid in FID.items()}
    return path, count, simtime, back


def reference_state(name, directory):
    os.makedirs(directory, exist_ok=True)
    with mp.get_context("spawn").Pool(1) as pool:
        return pool.apply(_ref_write_read, (name, str(directory)))


@needs_ref
@pytest.mark.parametrize("name", list(CASES))
def test_reference_state_layout(name, tmp_path):
    """The reference's file for a known state, decoded with the layout the
    library writes: header, then each block in loop order."""
    nx, ny, nz = CASES[name]
    path, count, simtime, back = reference_state(name, tmp_path)
    raw = open(path, "rb").read()
    hdr = HEADER.unpack_from(raw)
    assert hdr[:3] == (17, 4, 0.625)
    data = np.frombuffer(raw[HEADER.size:], dtype=np.float32)
    assert data.size == sum(n for _, n in blocks(nx, ny, nz))
    f = state_fields(name)
    pos = 0
    for blk, n in blocks(nx, ny, nz):
        got = data[pos:pos + n]
        pos += n
        if blk in ("kin", "eps", "qbe"):  # the void turbulence and sediment models
            assert not got.any(), blk
            continue
        ex = {"u": (1, 0, 0), "v": (0, 1, 0), "w": (0, 0, 1)}.get(blk, (0, 0, 0))
        assert np.array_equal(got, loop_order(f[blk], nx, ny, nz, ex).astype(np.float32)), blk
    # and read back by the reference: the file's values on the interior
    assert (count, simtime) == (17, 0.625)
    for k in ("phi", "press", "topo", "eddyv", "conc"):
        assert np.array_equal(interior(back[k], nx, ny, nz), interior(f[k], nx, ny, nz).astype(np.float32)), k


def dense(a, nx, ny, nz):
    """Padded reference-layout field -> dense x-contiguous (nz, ny, nx)."""
    return np.ascontiguousarray(interior(a, nx, ny, nz).transpose(2, 1, 0))


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("precision", [r3d.FP64, r3d.FP32])
@pytest.mark.parametrize("name", list(CASES))
def test_library_state_file_equals_reference(name, precision, tmp_path):
    nx, ny, nz, xn, yn, zn = grid(name)
    path, _, _, _ = reference_state(name, tmp_path / "ref")
    f = state_fields(name)
    extra = {k: dense(f[k], nx, ny, nz) for k in ("topo", "press", "eddyv", "conc")}
    ours = str(tmp_path / r3d.reef3d_state_name(0))
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=precision) as ls:
        for fid, k in ((r3d.PHI, "phi"), (r3d.U, "u"), (r3d.V, "v"), (r3d.W, "w")):
            ls.upload(fid, f[k])
        ls.write_reef3d_state(ours, count=17, printcount=4, simtime=0.625, extra=extra)
        # (an FP32 instance holds the float-rounded fields: the same bytes)
        assert open(ours, "rb").read() == open(path, "rb").read()
    # the reference's file into a fresh instance
    with r3d.LevelSet(nx, ny, nz, xn, yn, zn, precision=precision) as ls:
        for fid, k in ((r3d.PHI, "phi"), (r3d.U, "u"), (r3d.V, "v"), (r3d.W, "w")):
            ls.upload(fid, np.zeros_like(f[k]))
        info = ls.read_reef3d_state(path, extra=True)
        assert (info["count"], info["printcount"], info["simtime"]) == (17, 4, 0.625)
        got = ls.download(r3d.PHI)
        assert np.array_equal(interior(got, nx, ny, nz), interior(f["phi"], nx, ny, nz).astype(np.float32))
        for fid, k, ex in ((r3d.U, "u", (1, 0, 0)), (r3d.V, "v", (0, 1, 0)), (r3d.W, "w", (0, 0, 1))):
            a = interior(ls.download(fid), nx, ny, nz)[:nx - ex[0], :ny - ex[1], :nz - ex[2]]
            b = interior(f[k], nx, ny, nz)[:nx - ex[0], :ny - ex[1], :nz - ex[2]].astype(np.float32)
            assert np.array_equal(a, b), k
        for k in ("topo", "press", "eddyv", "conc"):
            assert np.array_equal(info["extra"][k], extra[k].astype(np.float32)), k
        assert not info["extra"]["kin"].any() and not info["extra"]["qbe"].any()


def test_state_file_name():
    assert r3d.reef3d_state_name(12) == "REEF3D-CFD-State-00000012-000001.r3d"
