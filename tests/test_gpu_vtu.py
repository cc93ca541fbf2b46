"""VTU output of device-resident fields (r3d_write_vtu) against the
reference's own printer interpolations (ipol4phi, ipol4_a, ipol4 over the
TPLOOP nodes, src/printer_CFD.cpp:678-727), run on the same step in a
spawned child through oracle/_ref: the Float32 point data bit-identical on
every node except the corner nodes, which read the triple-corner ghost
cells the reference never writes; the file's mesh is the reference printer's
(node coordinates, hexahedra in k, j, i order)."""
import multiprocessing as mp
import os
import re
import sys

import numpy as np
import pytest

import reef3d_b200 as r3d

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def read_vtu(path):
    """Arrays of a VTU file with appended raw data and 32-bit block sizes."""
    data = open(path, "rb").read()
    head, raw = data.split(b'<AppendedData encoding="raw">\n_', 1)
    text = head.decode()
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)"(?: Name="(\w+)")?(?: NumberOfComponents="(\d)")? '
                         r'format="appended" offset="(\d+)"/>', text):
        kind, name, _, off = m.group(1), m.group(2) or "points", m.group(3), int(m.group(4))
        n = int(np.frombuffer(raw[off:off + 4], dtype=np.uint32)[0])
        out[name] = np.frombuffer(raw[off + 4:off + 4 + n], dtype=np.float32 if kind == "Float32" else np.int32)
    return out


def _case(name):
    sys.path.insert(0, ROOT)
    from reef3d_b200 import setups
    c = setups.vortex3d(12) if name == "vortex3d" else setups.slotted_disk(20)
    return c


def _ref(name):
    sys.path.insert(0, ROOT)
    from oracle.bindings import RefOracle
    c = _case(name)
    o = RefOracle(c.nx, c.ny, c.nz, c.xn, c.yn, c.zn, f43=c.f43, f44=c.f44, f45=c.f45, f49=c.f49)
    o.set_state(c.phi, c.u, c.v, c.w)
    dt = o.cfl_dt(c.n47)
    o.set_count(1)
    o.step(dt)
    return dt, o.vtu_point_data()


def corner_nodes(nx, ny, nz):
    nyp = ny + 1 if ny > 1 else 2
    k, j, i = np.meshgrid(np.arange(-1, nz), np.arange(-1, nyp - 1), np.arange(-1, nx), indexing="ij")
    ci = (i == -1) | (i == nx - 1)
    ck = (k == -1) | (k == nz - 1)
    cj = (j == -1) | (j == ny - 1) if ny > 1 else np.ones_like(ci)
    return (ci & cj & ck).ravel()


@pytest.mark.parametrize("name", ["vortex3d", "disk2d"])
def test_vtu_point_data_matches_reference_printer(name, tmp_path):
    with mp.get_context("spawn").Pool(1) as pool:
        dt, (rphi, rro, rvisc) = pool.apply(_ref, (name,))
    c = _case(name)
    with r3d.LevelSet(c.nx, c.ny, c.nz, c.xn, c.yn, c.zn, f43=c.f43, f44=c.f44, f45=c.f45, f49=c.f49, n47=c.n47,
                      precision=r3d.FP64) as ls:
        ls.set_fluid()
        for f, a in ((r3d.PHI, c.phi), (r3d.U, c.u), (r3d.V, c.v), (r3d.W, c.w)):
            ls.upload(f, a)
        assert ls.cfl_dt() == dt
        ls.step()
        path = str(tmp_path / "out.vtu")
        ls.write_vtu(path)
    v = read_vtu(path)
    nyp = c.ny + 1 if c.ny > 1 else 2
    npts, ncell = (c.nx + 1) * nyp * (c.nz + 1), c.nx * c.ny * c.nz
    keep = ~corner_nodes(c.nx, c.ny, c.nz)
    assert v["phi"].size == npts and np.array_equal(v["phi"][keep], rphi[keep])
    assert np.array_equal(v["rho"][keep], rro[keep]) and np.array_equal(v["viscosity"], rvisc)
    # mesh: node coordinates of the reference's grid, hexahedra over the interior
    pts = v["points"].reshape(-1, 3)
    assert pts.shape[0] == npts
    assert np.array_equal(pts[:c.nx + 1, 0], c.xn[5:6 + c.nx].astype(np.float32))
    con = v["connectivity"].reshape(-1, 8)
    assert con.shape[0] == ncell and con.min() == 0 and con.max() == npts - 1
    assert np.array_equal(v["types"], np.full(ncell, 12, np.int32))
    assert np.array_equal(v["offsets"], 8 * np.arange(1, ncell + 1, dtype=np.int32))
