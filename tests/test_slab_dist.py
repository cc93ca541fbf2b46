"""Host side of the slab decomposition over torch.distributed
(reef3d_b200.slab.DistSlab) on the gloo backend, world sizes 2 and 3: the
exchange schedule (which planes go to which neighbour after every stage),
the halo-face marking and the reductions of the CFL step and the volume.
The GPU instance is replaced by a host stand-in with the same interface
whose stages are a nonlinear stencil reaching three cells in z (basic
arithmetic only, which rounds the same in every array position), so a wrong
or missing halo plane changes the result; a split run must then reproduce
the one-rank run bit for bit."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

PHI, WORK1, WORK2, RO, VISC = 0, 5, 6, 7, 8


class HostSlab:
    """Host stand-in of reef3d_b200.LevelSet for the slab driver: fields in
    the reference's padded layout (k fastest), wall copies on every face
    except the halo faces."""

    def __init__(self, nx, ny, nz, xn, yn, zn, n47=0.25, f44=2, **_):
        self.n = (nx, ny, nz)
        self.shape = (nx + 6, ny + 6, nz + 6)
        self.f = {k: np.zeros(self.shape) for k in (PHI, WORK1, WORK2, RO, VISC, 1, 2, 3)}
        self.zc = 0.5 * (np.asarray(zn)[2:-3] + np.asarray(zn)[3:-2])  # centres of k = -3..nz+2
        self.dz = float(np.min(np.diff(np.asarray(zn)[5:5 + nz + 1])))
        self.n47, self.halo, self.dt, self.t = n47, (0, 0), 0.0, 0.0

    def set_halo(self, lo, hi):
        self.halo = (int(bool(lo)), int(bool(hi)))

    def set_fluid(self):
        pass

    def set_grid_spacing(self, dxm, dym, dzm):
        pass

    def upload(self, field, a):
        self.f[field][...] = a

    def download(self, field):
        return self.f[field].copy()

    def halo_bytes(self):
        return 3 * self.shape[0] * self.shape[1] * 8

    def halo_copy(self, field, side, direction, ptr):
        nz = self.n[2]
        buf = np.ctypeslib.as_array((ctypes.c_double * (self.halo_bytes() // 8)).from_address(ptr))
        buf = buf.reshape(self.shape[0], self.shape[1], 3)
        if direction == 0:
            k0 = 3 if side == 0 else nz
            buf[...] = self.f[field][:, :, k0:k0 + 3]
        else:
            k0 = 0 if side == 0 else nz + 3
            self.f[field][:, :, k0:k0 + 3] = buf

    def sync(self):
        pass

    def cfl_max(self):
        nx, ny, nz = self.n
        kw = nz if self.halo[1] else nz - 1  # w faces 0..nz-2, and nz-1 with a neighbour above
        u = np.abs(self.f[1][3:3 + nx - 1, 3:3 + ny, 3:3 + nz]).max()
        w = np.abs(self.f[3][3:3 + nx, 3:3 + ny, 3:3 + kw]).max()
        return (float(u), 0.0, float(w))

    def cfl_dt_from_max(self, vm):
        return self.n47 * 2.0 / (np.sqrt(vm[0] ** 2 + vm[1] ** 2 + vm[2] ** 2) / self.dz)

    def set_dt(self, dt):
        self.dt = dt

    def set_time(self, t):
        self.t = t

    def _walls(self, a):
        nx, ny, nz = self.n
        for q in range(1, 4):
            a[3 - q, :, :] = a[3, :, :]
            a[2 + nx + q, :, :] = a[2 + nx, :, :]
            a[:, 3 - q, :] = a[:, 3, :]
            a[:, 2 + ny + q, :] = a[:, 2 + ny, :]
            if not self.halo[0]:
                a[:, :, 3 - q] = a[:, :, 3]
            if not self.halo[1]:
                a[:, :, 2 + nz + q] = a[:, :, 2 + nz]

    def stage(self, kind, st):
        nx, ny, nz = self.n
        src = {1: PHI, 2: WORK1, 3: WORK2}[st]
        out = {1: WORK1, 2: WORK2, 3: PHI}[st]
        f, fn = self.f[src], self.f[PHI]
        I = (slice(3, 3 + nx), slice(3, 3 + ny), slice(3, 3 + nz))
        zs = lambda d: f[3:3 + nx, 3:3 + ny, 3 + d:3 + nz + d]
        xs = lambda d: f[3 + d:3 + nx + d, 3:3 + ny, 3:3 + nz]
        w = self.f[3][I]
        L = -w * (zs(3) - zs(-3) + 2.0 * (zs(1) - zs(-1))) + 0.1 * zs(2) * zs(-2) / (1.0 + zs(2) * zs(2)) \
            + 0.05 * (xs(1) - xs(-1))
        if kind == 1:
            L = L - 0.3 * zs(0) / (1.0 + zs(0) * zs(0))
        dt = self.dt if kind == 0 else 0.01  # a pseudo time step the same for every cell
        if st == 1:
            val = fn[I] + dt * L
        elif st == 2:
            val = 0.75 * fn[I] + 0.25 * f[I] + 0.25 * dt * L
        else:
            val = (1.0 / 3.0) * fn[I] + (2.0 / 3.0) * f[I] + (2.0 / 3.0) * dt * L
        self.f[out][I] = val
        self._walls(self.f[out])

    def volume(self):
        nx, ny, nz = self.n
        p = self.f[PHI][3:3 + nx, 3:3 + ny, 3:3 + nz]
        return float(np.sum(p > 0.0)), float(np.sum(p <= 0.0))

    def fluid_update(self):
        return self.volume()

    def close(self):
        pass


def _case():
    nx, ny, nz = 8, 6, 20
    xn = np.linspace(-5, nx + 5, nx + 11) / nx
    yn = np.linspace(-5, ny + 5, ny + 11) / ny
    zn = np.linspace(-5, nz + 5, nz + 11) / nz
    rng = np.random.default_rng(3)
    shape = (nx + 6, ny + 6, nz + 6)
    phi = rng.standard_normal(shape)
    u, v, w = (rng.standard_normal(shape) for _ in range(3))
    return (nx, ny, nz), xn, yn, zn, phi, u, v, w


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    import torch.distributed as dist
    from reef3d_b200.slab import DistSlab, slab_of
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        (nx, ny, nz), xn, yn, zn, phi, u, v, w = _case()
        d = DistSlab(nx, ny, nz, xn, yn, zn, device="cpu", factory=HostSlab, n47=0.25, f44=2)
        for fid, a in ((PHI, phi), (1, u), (2, v), (3, w)):
            d.ls.upload(fid, slab_of(a, d.k0, d.k1))
        dts, vols = [], []
        for _ in range(3):
            dts.append(d.cfl_dt())
            vols.append(d.step())
        q.put((rank, d.k0, d.k1, d.ls.download(PHI), dts, vols))
    finally:
        dist.destroy_process_group()


def _run(world):
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = sorted((q.get(timeout=180) for _ in ps), key=lambda r: r[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


@pytest.mark.parametrize("world", [2, 3])
def test_split_run_equals_one_rank_run(world):
    one = _run(1)[0]
    parts = _run(world)
    whole = one[3]
    for rank, k0, k1, phi, dts, vols in parts:
        assert dts == one[4]
        # interior planes of the slab equal the undivided run's
        assert np.array_equal(phi[3:-3, 3:-3, 3:-3], whole[3:-3, 3:-3, 3 + k0:3 + k1]), rank
        for (a, b), (c, e) in zip(vols, one[5]):
            assert a == c and b == e  # counts: exact under any summation order
