"""Subdomain (slab) runs of one grid: the grid is split along z into slabs
of consecutive cells, one instance per slab, and the halo exchange of
REEF3D's MPI decomposition (ghostcell::gcparax, src/gcx_parax.cpp: three
ghost layers from the neighbour after every RK stage) runs between the
stages, with the CFL maxima and the volume sums reduced over slabs
(pgc->globalmax / globalsum, src/gcx_global.cpp:27-49).

Two ways to hold the slabs:

* ``LocalSlabs``: every slab in this process (on one GPU or several); halos
  move device to device through the library's pack/unpack calls.
* ``DistSlab``: one slab per rank of ``torch.distributed`` (one process per
  GPU, NCCL over NVLink); halos move by point-to-point send/recv, maxima,
  minima and sums by all-reduce.
* ``Domain``: the native runner (r3d_domain_*): slabs on one GPU or on
  several, each on its own stream, the whole decomposed step -- stages, halo
  peer copies, the global CFL step -- captured in one CUDA graph.

A step is the step of ``r3d_ls_step`` taken stage by stage (three
convection stages, f44 reinitialisation pseudo-steps of three stages, the
volume sums or the fluid update), each stage followed by the exchange of
the field it wrote.  Host-driven slabs (LocalSlabs, DistSlab) run without
the picard correction and without inflow/outflow faces, whose sums the
reference takes globally in the middle of a step; the native Domain runs the
picard correction over the whole grid (per-slab volume sums added on the
device between the slabs' passes).
"""
import numpy as np

import ctypes

from . import (FP64, PHI, R3D_OK, R3DError, RO, VISC, WORK1, WORK2, LevelSet, STAGE_CONVECTION, STAGE_REINIT,
               grid_spacing, load_library, make_desc, uniform_nodes)

# stage s writes phi -> WORK1 -> WORK2 -> phi (convection and reinitialisation)
STAGE_OUT = {1: WORK1, 2: WORK2, 3: PHI}


def split(nz, nslabs):
    """(k0, k1) of each slab: near-equal runs of consecutive z cells, every
    slab at least 3 cells (the halo depth)."""
    if nslabs < 1 or nz < 3 * nslabs:
        raise ValueError(f"{nz} z cells cannot make {nslabs} slabs of >= 3 cells")
    base, extra = divmod(nz, nslabs)
    out, k = [], 0
    for r in range(nslabs):
        n = base + (1 if r < extra else 0)
        out.append((k, k + n))
        k += n
    return out


def slab_nodes(zn, k0, k1):
    """Node coordinates of slab [k0, k1) for node indices -5..(k1-k0)+5,
    taken from the grid's (which covers -5..nz+5)."""
    zn = np.asarray(zn, dtype=np.float64)
    return np.ascontiguousarray(zn[k0:k1 + 11])


def slab_of(a, k0, k1):
    """Slab [k0, k1) of a field in the reference's padded layout, with its
    three ghost planes on either side."""
    return np.ascontiguousarray(a[:, :, k0:k1 + 6])


class _Stepper:
    """The stage sequence shared by both slab holders.  Subclasses provide
    ``_slabs`` (the instances), ``_exchange(field)``, ``_max3``, ``_min``
    and ``_sum2`` (reductions over slabs)."""

    f44 = 2
    fluid = False
    t = 0.0

    def cfl_dt(self):
        """Time step of the undivided grid: maxima over slabs, then the
        minimum of the slabs' steps (their smallest cells differ)."""
        vmax = self._max3([s.cfl_max() for s in self._slabs])
        dt = self._min([s.cfl_dt_from_max(vmax) for s in self._slabs])
        for s in self._slabs:
            s.set_dt(dt)
        self.dt = dt
        return dt

    def step(self):
        for st in (1, 2, 3):
            for s in self._slabs:
                s.stage(STAGE_CONVECTION, st)
            self._exchange(STAGE_OUT[st])
        for _ in range(self.f44):
            for st in (1, 2, 3):
                for s in self._slabs:
                    s.stage(STAGE_REINIT, st)
                self._exchange(STAGE_OUT[st])
        if self.fluid:
            vols = [s.fluid_update() for s in self._slabs]
            self._exchange(RO)
            self._exchange(VISC)
        else:
            vols = [s.volume() for s in self._slabs]
        self.last_volume = self._sum2(vols)
        self.t += self.dt
        for s in self._slabs:
            s.set_time(self.t)
        return self.last_volume

    def run(self, nsteps):
        for _ in range(nsteps):
            self.cfl_dt()
            self.step()


def _make_slab(factory, nx, ny, k0, k1, xn, yn, zn, nz, flags):
    """Slab [k0, k1) as an instance of its own: the slab's node coordinates,
    halo faces towards its neighbours, and the whole grid's spacing
    constants (DXM is a mean over the whole grid, src/grid.cpp:102-148)."""
    ls = factory(nx, ny, k1 - k0, xn, yn, slab_nodes(zn, k0, k1), **flags)
    ls.set_halo(k0 > 0, k1 < nz)
    dxm, dym, dzm, _ = grid_spacing(nx, ny, nz, xn, yn, zn, flags.get("f45", 2.1))
    ls.set_grid_spacing(dxm, dym, dzm)
    return ls


class LocalSlabs(_Stepper):
    """All slabs of one grid in this process.  devices: CUDA device index
    of each slab (default: the current device for all)."""

    def __init__(self, nx, ny, nz, xn, yn, zn, nslabs, devices=None, fluid=False, factory=LevelSet, **flags):
        import torch
        if flags.get("f46", 0):
            raise R3DError(1, "slab runs have no picard correction")
        self.nz, self.bounds = nz, split(nz, nslabs)
        self.f44 = flags.get("f44", 2)
        self.fluid = fluid
        self.dt = 0.0
        devs = devices or [torch.cuda.current_device()] * nslabs
        self._slabs = []
        for (k0, k1), d in zip(self.bounds, devs):
            with torch.cuda.device(d):
                ls = _make_slab(factory, nx, ny, k0, k1, xn, yn, zn, nz, flags)
                if fluid:
                    ls.set_fluid()
            self._slabs.append(ls)
        # one buffer per direction of each interface, on the receiving slab's device
        nb = self._slabs[0].halo_bytes()
        self._up = [torch.empty(nb, dtype=torch.uint8, device=f"cuda:{devs[r + 1]}") for r in range(nslabs - 1)]
        self._dn = [torch.empty(nb, dtype=torch.uint8, device=f"cuda:{devs[r]}") for r in range(nslabs - 1)]

    @property
    def slabs(self):
        return self._slabs

    def upload(self, field, a):
        """A field of the whole grid (reference layout, nz+6 z planes)."""
        for ls, (k0, k1) in zip(self._slabs, self.bounds):
            ls.upload(field, slab_of(a, k0, k1))

    def download(self, field):
        parts = [ls.download(field) for ls in self._slabs]
        out = np.concatenate([parts[0][:, :, :3]] + [p[:, :, 3:-3] for p in parts] + [parts[-1][:, :, -3:]], axis=2)
        return out

    def _exchange(self, field):
        s = self._slabs
        for r in range(len(s) - 1):
            s[r].halo_copy(field, 1, 0, self._up[r].data_ptr())      # top interior planes of slab r
            s[r + 1].halo_copy(field, 0, 0, self._dn[r].data_ptr())  # bottom interior planes of slab r+1
        for ls in s:
            ls.sync()
        for r in range(len(s) - 1):
            s[r + 1].halo_copy(field, 0, 1, self._up[r].data_ptr())  # into slab r+1's bottom ghosts
            s[r].halo_copy(field, 1, 1, self._dn[r].data_ptr())      # into slab r's top ghosts

    def _max3(self, vals):
        return tuple(max(v[a] for v in vals) for a in range(3))

    def _min(self, vals):
        return min(vals)

    def _sum2(self, vals):
        v1 = 0.0
        v2 = 0.0
        for a, b in vals:
            v1 += a
            v2 += b
        return v1, v2

    def close(self):
        for ls in self._slabs:
            ls.close()
        self._slabs = []


class DistSlab(_Stepper):
    """This rank's slab of one grid split over the ranks of a
    torch.distributed process group (rank r holds the r-th slab from the
    bottom).  device: the torch device the halo buffers live on ("cuda:N"
    with NCCL; "cpu" with gloo for host-side tests, where `factory` makes a
    host stand-in of LevelSet)."""

    def __init__(self, nx, ny, nz, xn, yn, zn, group=None, device=None, fluid=False, factory=LevelSet, **flags):
        import torch
        import torch.distributed as dist
        if flags.get("f46", 0):
            raise R3DError(1, "slab runs have no picard correction")
        self.dist, self.torch, self.group = dist, torch, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.nz, self.bounds = nz, split(nz, self.world)
        self.k0, self.k1 = self.bounds[self.rank]
        self.f44 = flags.get("f44", 2)
        self.fluid = fluid
        self.dt = 0.0
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.ls = _make_slab(factory, nx, ny, self.k0, self.k1, xn, yn, zn, nz, flags)
        if fluid:
            self.ls.set_fluid()
        self._slabs = [self.ls]
        nb = self.ls.halo_bytes()
        self._buf = {key: torch.empty(nb, dtype=torch.uint8, device=self.device)
                     for key in ("send_lo", "send_hi", "recv_lo", "recv_hi")}

    def _peer(self, r):
        return self.dist.get_global_rank(self.group, r) if self.group is not None else r

    def _exchange(self, field):
        dist, b = self.dist, self._buf
        lo, hi = self.rank > 0, self.rank < self.world - 1
        if lo:
            self.ls.halo_copy(field, 0, 0, b["send_lo"].data_ptr())
        if hi:
            self.ls.halo_copy(field, 1, 0, b["send_hi"].data_ptr())
        self.ls.sync()  # the packs are complete before the transport reads the buffers
        ops = []
        if lo:
            ops += [dist.P2POp(dist.isend, b["send_lo"], self._peer(self.rank - 1), self.group),
                    dist.P2POp(dist.irecv, b["recv_lo"], self._peer(self.rank - 1), self.group)]
        if hi:
            ops += [dist.P2POp(dist.isend, b["send_hi"], self._peer(self.rank + 1), self.group),
                    dist.P2POp(dist.irecv, b["recv_hi"], self._peer(self.rank + 1), self.group)]
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if self.device.type == "cuda":
            self.torch.cuda.current_stream(self.device).synchronize()
        if lo:
            self.ls.halo_copy(field, 0, 1, b["recv_lo"].data_ptr())
        if hi:
            self.ls.halo_copy(field, 1, 1, b["recv_hi"].data_ptr())

    def _reduce(self, vals, op):
        t = self.torch.tensor(vals, dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op, group=self.group)
        return [float(x) for x in t.cpu()]

    def _max3(self, vals):
        return tuple(self._reduce(list(vals[0]), self.dist.ReduceOp.MAX))

    def _min(self, vals):
        return self._reduce([vals[0]], self.dist.ReduceOp.MIN)[0]

    def _sum2(self, vals):
        return tuple(self._reduce(list(vals[0]), self.dist.ReduceOp.SUM))

    def close(self):
        self.ls.close()


class Domain:
    """One grid split along z into `nslabs` slabs (on the current GPU, or
    slab r on devices[r]) and stepped as one by the native runner
    (r3d_domain_*): fields in the reference's layout of the whole grid.
    f46/f47: the picard correction of the whole grid (as LevelSet's)."""

    def __init__(self, nx, ny, nz, xn=None, yn=None, zn=None, nslabs=2, f43=0.55, f44=3, f45=2.1, f49=1,
                 n47=0.3, precision=FP64, devices=None, f46=0, f47=10):
        self._lib = load_library()
        xn = uniform_nodes(nx) if xn is None else xn
        yn = uniform_nodes(ny) if yn is None else yn
        zn = uniform_nodes(nz) if zn is None else zn
        self.nx, self.ny, self.nz, self.nslabs = nx, ny, nz, nslabs
        self.desc = make_desc(nx, ny, nz, xn, yn, zn, f43, f44, f45, f49, n47, precision, f46, f47)
        d = ctypes.c_void_p()
        devs = None
        if devices is not None:
            devs = (ctypes.c_int * nslabs)(*devices)
        rc = self._lib.r3d_domain_create(ctypes.byref(self.desc), nslabs, devs, ctypes.byref(d))
        if rc != R3D_OK:
            msg = self._lib.r3d_last_error(None)
            raise R3DError(rc, msg.decode() if msg else "")
        self.d = d

    def _check(self, rc):
        if rc != R3D_OK:
            msg = self._lib.r3d_domain_last_error(self.d)
            raise R3DError(rc, msg.decode() if msg else "")

    def upload(self, field, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self._check(self._lib.r3d_domain_upload(self.d, field, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def download(self, field):
        a = np.zeros((self.nx + 6, self.ny + 6, self.nz + 6))
        self._check(self._lib.r3d_domain_download(self.d, field, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return a

    def run(self, nsteps, dt=0.0):
        """nsteps steps; dt <= 0: adaptive (CFL over all slabs)."""
        self._check(self._lib.r3d_domain_run(self.d, nsteps, dt))

    def last_volume(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.r3d_domain_last_volume(self.d, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_fluid(self, ro_water=998.2, visc_water=1.004e-6, ro_air=1.205, visc_air=1.41e-5):
        """Density/viscosity update on every slab (r3d_domain_set_fluid)."""
        self._check(self._lib.r3d_domain_set_fluid(self.d, ro_water, visc_water, ro_air, visc_air))

    def dt(self):
        v = ctypes.c_double()
        self._check(self._lib.r3d_domain_get_dt(self.d, ctypes.byref(v)))
        return v.value

    def _slab(self, s):
        h = ctypes.c_void_p()
        self._check(self._lib.r3d_domain_slab(self.d, s, ctypes.byref(h), None, None))
        return h

    def set_ioflow(self, **flags):
        """Inflow / outflow faces on every slab (r3d_domain_set_ioflow), the
        keys of LevelSet.set_ioflow; off=True closes them."""
        from . import IOFLOW_DEFAULTS, IoflowDesc
        if flags.pop("off", False):
            self._check(self._lib.r3d_domain_set_ioflow(self.d, None))
            return
        unknown = set(flags) - set(IOFLOW_DEFAULTS)
        if unknown:
            raise TypeError(f"unknown ioflow flags {sorted(unknown)}")
        desc = IoflowDesc(**dict(IOFLOW_DEFAULTS, **flags))
        self._check(self._lib.r3d_domain_set_ioflow(self.d, ctypes.byref(desc)))

    def io_levels(self):
        """(phimean, phiout) of the grid, measured by the last step."""
        a, b = ctypes.c_double(), ctypes.c_double()
        h = self._slab(0)
        if self._lib.r3d_io_levels(h, ctypes.byref(a), ctypes.byref(b)) != R3D_OK:
            raise R3DError(1, self._lib.r3d_last_error(h).decode())
        return a.value, b.value

    def set_direct_forcing(self, x45):
        """X45 direct-forcing convection stencils on every slab (each slab's
        r3d_set_direct_forcing); the BODY field goes up by upload()."""
        for s in range(self.nslabs):
            h = self._slab(s)
            if self._lib.r3d_set_direct_forcing(h, x45) != R3D_OK:
                raise R3DError(1, self._lib.r3d_last_error(h).decode())

    def set_step_count(self, count):
        """lexer::count of the next step (every slab's)."""
        for s in range(self.nslabs):
            h = self._slab(s)
            if self._lib.r3d_set_step_count(h, count) != R3D_OK:
                raise R3DError(1, self._lib.r3d_last_error(h).decode())

    def close(self):
        if getattr(self, "d", None) is not None and self.d.value:
            self._lib.r3d_domain_destroy(self.d)
            self.d = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
