"""ctypes bindings for the two CPU oracles (test infrastructure only).

* ``PortOracle`` wraps ``oracle/liboracle.so``: the project's C restatement of
  the reference's level-set path (``oracle/ls_oracle.c``).  Re-entrant.
* ``RefOracle`` wraps ``oracle/_ref/libreef3d_ref.so``: the reference's own
  sources compiled with ``oracle/Makefile.ref`` and driven through
  ``oracle/ref_harness.cpp``.  One grid per process (the reference keeps loop
  indices and WENO tables in static members), so callers run it in a fresh
  process per grid.

Both work on the reference's padded field layout (margin 3 on every side, k
contiguous): arrays of shape ``(nx+6, ny+6, nz+6)`` in C order.
Only tests, the smoke check and the CPU-baseline leg of the benchmark use
this module.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libreef3d_ref.so")
REF_LIB_FAST = os.path.join(HERE, "_ref", "fast", "libreef3d_ref.so")
ADAPTER_LIB = os.path.join(HERE, "_ref", "libreef3d_adapter.so")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.c_int


def _dp(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


# ioflow_f flags in refls_set_ioflow's argument order, with the reference's
# defaults (src/ini.cpp:208-441; F50 = 2 the level-set default).
IOFLOW_KEYS = ("inflow", "outflow", "f50", "b77", "f56", "f60", "f61", "f62", "f64", "qi", "qo")
IOFLOW_DEFAULTS = dict(inflow=1, outflow=1, f50=2, b77=1, f56=1.0e20, f60=-1.0e20, f61=-1.0e20, f62=-1.0e20,
                       f64=0, qi=0.0, qo=0.0)
# iowave flags in refls_set_iowave's argument order: wave theory B92, wave
# amplitude and period (B93_1, B93_2), depth B94_wdt, generation / beach zone
# lengths B96_1 / B96_2, still water level F56, ramp B101 / B102, wave maker
# B98 (2 relaxation zone, 3 Dirichlet, 4 active) and beach B99 (2 relaxation
# zone, 3-5 active)
IOWAVE_KEYS = ("b92", "amp", "period", "depth", "b96_1", "b96_2", "phimean", "b101", "b102", "b98", "b99")
IOWAVE_DEFAULTS = dict(b92=2, amp=0.05, period=1.0, depth=0.5, b96_1=0.5, b96_2=0.5, phimean=0.5, b101=0,
                       b102=1.0, b98=2, b99=2)


def padded_shape(nx, ny, nz):
    return (nx + 6, ny + 6, nz + 6)


def uniform_nodes(n, length=1.0, origin=0.0):
    """Node coordinates for indices -5..n+5 of a uniform axis (n+11 values),
    x_i = origin + i*(length/n)."""
    h = length / n
    return np.array([origin + i * h for i in range(-5, n + 6)], dtype=np.float64)


class PortOracle:
    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = ctypes.CDLL(PORT_LIB)
            lib.lso_new.restype = ctypes.c_void_p
            lib.lso_new.argtypes = [_I, _I, _I, _D, _D, _D, ctypes.c_double, _I, ctypes.c_double, _I,
                                    ctypes.c_double]
            lib.lso_delete.argtypes = [ctypes.c_void_p]
            lib.lso_ncell.restype = ctypes.c_long
            lib.lso_ncell.argtypes = [ctypes.c_void_p]
            for fn in ("lso_psi", "lso_dxm"):
                getattr(lib, fn).restype = ctypes.c_double
                getattr(lib, fn).argtypes = [ctypes.c_void_p]
            lib.lso_get_metric.argtypes = [ctypes.c_void_p, _I, _D, _I]
            lib.lso_get_weno_tables.argtypes = [ctypes.c_void_p, _I, _D, _D, _D, _I]
            lib.lso_weno_L.argtypes = [ctypes.c_void_p, _D, _D, _D, _D, _D]
            lib.lso_reinidisc_L.argtypes = [ctypes.c_void_p, _D, _D]
            lib.lso_ghost_fill.argtypes = [ctypes.c_void_p, _D]
            lib.lso_reini.argtypes = [ctypes.c_void_p, _D, _D, _D, _D, _I]
            lib.lso_ls_step.argtypes = [ctypes.c_void_p, _D, _D, _D, _D, ctypes.c_double, _D, _D, _D]
            lib.lso_volume.argtypes = [ctypes.c_void_p, _D, _D, _D]
            lib.lso_cfl_dt.restype = ctypes.c_double
            lib.lso_cfl_dt.argtypes = [ctypes.c_void_p, _D, _D, _D]
            lib.lso_set_picard.argtypes = [ctypes.c_void_p, _I, _I]
            lib.lso_fluid.argtypes = [ctypes.c_void_p, _D, _D, _D] + [ctypes.c_double] * 4
            lib.lso_set_ioflow.argtypes = ([ctypes.c_void_p, _I, _I, _I, _I] + [ctypes.c_double] * 4 + [_I]
                                           + [ctypes.c_double] * 2)
            lib.lso_io_levels.argtypes = [ctypes.c_void_p, _D]
            lib.lso_set_count.argtypes = [ctypes.c_void_p, _I]
            lib.lso_set_direct_forcing.argtypes = [ctypes.c_void_p, _I, _D, _D]
            lib.lso_set_solid_forcing.argtypes = [ctypes.c_void_p, _I, ctypes.POINTER(ctypes.c_int)]
            cls._lib = lib
        return cls._lib

    def __init__(self, nx, ny, nz, xn, yn, zn, f43=0.55, f44=3, f45=2.1, f49=1, n47=0.3, f46=0, f47=10,
                 ioflow=None):
        self.lib()
        self.nx, self.ny, self.nz = nx, ny, nz
        self.shape = padded_shape(nx, ny, nz)
        self.f44 = f44
        self._xn = np.ascontiguousarray(xn, dtype=np.float64)
        self._yn = np.ascontiguousarray(yn, dtype=np.float64)
        self._zn = np.ascontiguousarray(zn, dtype=np.float64)
        self.h = self._lib.lso_new(nx, ny, nz, _dp(self._xn), _dp(self._yn), _dp(self._zn),
                                   f43, f44, f45, f49, n47)
        if not self.h:
            raise ValueError("lso_new failed")
        self._lib.lso_set_picard(self.h, f46, f47)
        if ioflow is not None:
            io = dict(IOFLOW_DEFAULTS, **ioflow)
            self._lib.lso_set_ioflow(self.h, *(io[k] for k in IOFLOW_KEYS))

    def set_solid_forcing(self, cells):
        """solid_forcing_lsm entries (i, j, k, side) after each convection stage."""
        self._sf = np.ascontiguousarray(cells, dtype=np.int32).reshape(-1)
        self._lib.lso_set_solid_forcing(self.h, self._sf.size // 4, self._sf.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))

    def set_direct_forcing(self, x45, body1, body2=None):
        """X45 stencils reading body1 (fb, fbh5, fbh4 or solid) and body2
        (topo, X45 = 5), padded fields."""
        self._body = [np.ascontiguousarray(body1, dtype=np.float64),
                      np.ascontiguousarray(body2 if body2 is not None else body1, dtype=np.float64)]
        self._lib.lso_set_direct_forcing(self.h, x45, _dp(self._body[0]), _dp(self._body[1]))

    def set_io_waves(self, on=True):
        """The inflow / outflow faces belong to iowave (no fsfinflow)."""
        self._lib.lso_set_io_waves.argtypes = [ctypes.c_void_p, _I]
        self._lib.lso_set_io_waves(self.h, 1 if on else 0)

    def set_relaxation(self, wg, wb, phimean):
        """iowave::phi_relax after each convection stage: weights per column
        (nx, ny), negative outside the zone."""
        self._rz = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (wg, wb)]
        self._lib.lso_set_relaxation.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_double]
        self._lib.lso_set_relaxation(self.h, *(None if a is None else _dp(a) for a in self._rz), phimean)

    def set_relaxation_target(self, lsval, ramp):
        self._rz_ls = np.ascontiguousarray(lsval, dtype=np.float64)
        self._lib.lso_set_relaxation_target.argtypes = [ctypes.c_void_p, _D, ctypes.c_double]
        self._lib.lso_set_relaxation_target(self.h, _dp(self._rz_ls), ramp)

    def io_levels(self):
        """(phimean, phiout) after the last step's fsfinflow."""
        out = np.zeros(2)
        self._lib.lso_io_levels(self.h, _dp(out))
        return float(out[0]), float(out[1])

    def set_count(self, count):
        """lexer::count the next step runs as."""
        self._lib.lso_set_count(self.h, count)

    def __del__(self):
        if getattr(self, "h", None) and self._lib is not None:
            self._lib.lso_delete(self.h)
            self.h = None

    def zeros(self):
        return np.zeros(self.shape, dtype=np.float64)

    @property
    def psi(self):
        return self._lib.lso_psi(self.h)

    @property
    def dxm(self):
        return self._lib.lso_dxm(self.h)

    def metric(self, which, n):
        out = np.zeros(n)
        self._lib.lso_get_metric(self.h, which, _dp(out), n)
        return out

    def weno_tables(self, axis, n):
        qf, cf, isf = np.zeros(n * 12), np.zeros(n * 6), np.zeros(n * 18)
        self._lib.lso_get_weno_tables(self.h, axis, _dp(qf), _dp(cf), _dp(isf), n)
        return qf, cf, isf

    def weno_L(self, phi, u, v, w):
        L = self.zeros()
        self._lib.lso_weno_L(self.h, _dp(phi), _dp(u), _dp(v), _dp(w), _dp(L))
        return L

    def reinidisc_L(self, f):
        L = self.zeros()
        self._lib.lso_reinidisc_L(self.h, _dp(f), _dp(L))
        return L

    def ghost_fill(self, f):
        f = np.array(f, dtype=np.float64, order="C", copy=True)
        self._lib.lso_ghost_fill(self.h, _dp(f))
        return f

    def reini(self, f, iters):
        f = np.array(f, dtype=np.float64, order="C", copy=True)
        a1, a2, L = self.zeros(), self.zeros(), self.zeros()
        self._lib.lso_reini(self.h, _dp(f), _dp(a1), _dp(a2), _dp(L), iters)
        return f

    def step(self, phi, u, v, w, dt):
        phi = np.array(phi, dtype=np.float64, order="C", copy=True)
        a1, a2, L = self.zeros(), self.zeros(), self.zeros()
        self._lib.lso_ls_step(self.h, _dp(phi), _dp(u), _dp(v), _dp(w), dt, _dp(a1), _dp(a2), _dp(L))
        return phi

    def volume(self, phi):
        v1, v2 = ctypes.c_double(), ctypes.c_double()
        self._lib.lso_volume(self.h, _dp(np.ascontiguousarray(phi)), ctypes.byref(v1), ctypes.byref(v2))
        return v1.value, v2.value

    def cfl_dt(self, u, v, w):
        return self._lib.lso_cfl_dt(self.h, _dp(u), _dp(v), _dp(w))

    def fluid(self, phi, w1=998.2, w2=1.004e-6, w3=1.205, w4=1.41e-5):
        """(ro, visc) of fluid_update_fsf (defaults: the reference's W1..W4)."""
        ro, visc = self.zeros(), self.zeros()
        self._lib.lso_fluid(self.h, _dp(np.ascontiguousarray(phi)), _dp(ro), _dp(visc), w1, w2, w3, w4)
        return ro, visc


class RefOracle:
    """The reference's own objects; at most one per process."""

    _lib = None

    @classmethod
    def available(cls):
        return os.path.exists(REF_LIB)

    _loaded = set()

    def __init__(self, nx, ny, nz, xn, yn, zn, f43=0.55, f44=3, f45=2.1, f49=1, fast=False, f46=0, f47=10,
                 path=None, ioflow=None, x45=0, solid_forcing=None, iowave=None):
        """ioflow: None for the closed box, else a dict of IOFLOW_DEFAULTS'
        keys: inflow (x-min) / outflow (x-max) faces and ioflow_f's flags.
        iowave: None, else a dict of IOWAVE_KEYS (REEF3D's wave generator with
        relaxation zones on the x faces; replaces ioflow)."""
        path = path or (REF_LIB_FAST if fast else REF_LIB)
        if path in RefOracle._loaded:
            raise RuntimeError("the reference oracle holds one grid per process")
        RefOracle._loaded.add(path)
        lib = ctypes.CDLL(path)
        lib.refls_set_picard.argtypes = [_I, _I]
        lib.refls_set_picard(f46, f47)
        lib.refls_set_x45.argtypes = [_I]
        lib.refls_set_x45(x45)
        if solid_forcing is not None:
            cells = np.ascontiguousarray(solid_forcing, dtype=np.int32).reshape(-1)
            lib.refls_set_solid_forcing.argtypes = [_I, ctypes.POINTER(ctypes.c_int)]
            lib.refls_set_solid_forcing(cells.size // 4, cells.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        if iowave is not None:
            lib.refls_set_iowave.argtypes = [_I] + [ctypes.c_double] * 6 + [_I, ctypes.c_double, _I, _I]
            w = dict(IOWAVE_DEFAULTS, **iowave)
            lib.refls_set_iowave(*(w[k] for k in IOWAVE_KEYS))
        if ioflow is not None:
            io = dict(IOFLOW_DEFAULTS, **ioflow)
            lib.refls_set_ioflow.argtypes = [_I, _I, _I, _I] + [ctypes.c_double] * 4 + [_I] + [ctypes.c_double] * 2
            lib.refls_set_ioflow(*(io[k] for k in IOFLOW_KEYS))
        lib.refls_io_levels.argtypes = [_D]
        lib.refls_init.argtypes = [_I, _I, _I, _D, _D, _D, _I, ctypes.c_double, ctypes.c_double, _I]
        lib.refls_padded_size.restype = ctypes.c_long
        lib.refls_set_field.argtypes = [_I, _D]
        lib.refls_get_field.argtypes = [_I, _D]
        lib.refls_set_dt.argtypes = [ctypes.c_double]
        lib.refls_set_count.argtypes = [_I]
        for fn in ("refls_psi", "refls_dxm", "refls_volume1", "refls_volume2"):
            getattr(lib, fn).restype = ctypes.c_double
        lib.refls_get_metric.argtypes = [_I, _D, _I]
        lib.refls_get_weno_tables.argtypes = [_I, _D, _D, _D, _I]
        lib.refls_weno_L.argtypes = [_D, _D]
        lib.refls_reinidisc_L.argtypes = [_D, _D]
        lib.refls_ghost_fill.argtypes = [_D]
        lib.refls_cfl_dt.restype = ctypes.c_double
        lib.refls_cfl_dt.argtypes = [ctypes.c_double]
        self._lib = lib
        self.nx, self.ny, self.nz = nx, ny, nz
        self.shape = padded_shape(nx, ny, nz)
        xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (xn, yn, zn)]
        rc = lib.refls_init(nx, ny, nz, _dp(xs[0]), _dp(xs[1]), _dp(xs[2]), f44, f43, f45, f49)
        if rc != 0:
            raise RuntimeError("refls_init failed")
        assert lib.refls_padded_size() == int(np.prod(self.shape))

    def zeros(self):
        return np.zeros(self.shape, dtype=np.float64)

    def set_field(self, fid, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self._lib.refls_set_field(fid, _dp(a))

    def get_field(self, fid):
        a = self.zeros()
        self._lib.refls_get_field(fid, _dp(a))
        return a

    def write_state(self, directory, count, printcount, simtime):
        """The reference's restart state file (cfd_state::write) of the
        current fields under directory/REEF3D_CFD_STATE/; returns its path."""
        lib = self._lib
        lib.refls_write_state.argtypes = [ctypes.c_char_p, _I, _I, ctypes.c_double]
        if lib.refls_write_state(os.fsencode(directory), count, printcount, simtime) != 0:
            raise RuntimeError("refls_write_state failed")
        return os.path.join(directory, "REEF3D_CFD_STATE", "REEF3D-CFD-State-%08i-%06i.r3d" % (0, 1))

    def read_state(self, directory, num=0):
        """cfd_state::read of state `num` from directory/REEF3D_CFD_STATE/;
        returns (count, simtime)."""
        lib = self._lib
        lib.refls_read_state.argtypes = [ctypes.c_char_p, _I, ctypes.POINTER(ctypes.c_int), _D]
        c, t = ctypes.c_int(), ctypes.c_double()
        if lib.refls_read_state(os.fsencode(directory), num, ctypes.byref(c), ctypes.byref(t)) != 0:
            raise RuntimeError("refls_read_state failed")
        return c.value, t.value

    def set_state(self, phi, u, v, w):
        for fid, arr in ((0, phi), (1, u), (2, v), (3, w)):
            self.set_field(fid, arr)

    @property
    def psi(self):
        return self._lib.refls_psi()

    @property
    def dxm(self):
        return self._lib.refls_dxm()

    def metric(self, which, n):
        out = np.zeros(n)
        self._lib.refls_get_metric(which, _dp(out), n)
        return out

    def weno_tables(self, axis, n):
        qf, cf, isf = np.zeros(n * 12), np.zeros(n * 6), np.zeros(n * 18)
        self._lib.refls_get_weno_tables(axis, _dp(qf), _dp(cf), _dp(isf), n)
        return qf, cf, isf

    def weno_L(self, phi):
        L = self.zeros()
        self._lib.refls_weno_L(_dp(np.ascontiguousarray(phi)), _dp(L))
        return L

    def reinidisc_L(self, f):
        L = self.zeros()
        self._lib.refls_reinidisc_L(_dp(np.ascontiguousarray(f)), _dp(L))
        return L

    def ghost_fill(self, f):
        f = np.array(f, dtype=np.float64, order="C", copy=True)
        self._lib.refls_ghost_fill(_dp(f))
        return f

    def reini(self):
        self._lib.refls_reini()
        return self.get_field(0)

    def set_count(self, count):
        """lexer::count, the time step counter (1 for the first step)."""
        self._lib.refls_set_count(count)

    def step(self, dt):
        self._lib.refls_set_dt(dt)
        self._lib.refls_step()
        return self.get_field(0)

    def cfl_dt(self, n47):
        return self._lib.refls_cfl_dt(n47)

    def volume(self):
        self._lib.refls_update()
        return self._lib.refls_volume1(), self._lib.refls_volume2()

    def vtu_point_data(self):
        """The reference printer's phi, rho, viscosity at the grid nodes."""
        ny = self.ny + 1 if self.ny > 1 else 2
        n = (self.nx + 1) * ny * (self.nz + 1)
        out = [np.zeros(n, dtype=np.float32) for _ in range(3)]
        fp = ctypes.POINTER(ctypes.c_float)
        self._lib.refls_vtu_point_data(*(a.ctypes.data_as(fp) for a in out))
        return out

    def set_time(self, t):
        """lexer::simtime (the wave generator's clock)."""
        self._lib.refls_set_time.argtypes = [ctypes.c_double]
        self._lib.refls_set_time(t)

    def wavegen_precalc(self):
        """iowave::wavegen_precalc: the generation zone's targets at the clock."""
        if self._lib.refls_wavegen_precalc() != 0:
            raise RuntimeError("no wave generator")

    def iowave_weights(self):
        """(relax4_wg, relax4_nb) per interior column as (nx, ny) arrays, -1
        outside the zones."""
        wg, wb = np.zeros(self.nx * self.ny), np.zeros(self.nx * self.ny)
        self._lib.refls_iowave_weights.argtypes = [_D, _D]
        if self._lib.refls_iowave_weights(_dp(wg), _dp(wb)) != 0:
            raise RuntimeError("no wave generator")
        return wg.reshape(self.nx, self.ny), wb.reshape(self.nx, self.ny)

    def iowave_targets(self):
        """(lsval, ramp) of the generation zone at the last wavegen_precalc."""
        n = self.nx * self.ny * self.nz
        ls, ramp = np.zeros(n), np.zeros(1)
        self._lib.refls_iowave_targets.argtypes = [_D, ctypes.c_long, _D]
        self._lib.refls_iowave_targets.restype = ctypes.c_long
        m = self._lib.refls_iowave_targets(_dp(ls), n, _dp(ramp))
        if m < 0:
            raise RuntimeError("no wave generator")
        return ls[:m].copy(), float(ramp[0])

    def set_time(self, t):
        """lexer::simtime (the wave generator's clock)."""
        self._lib.refls_set_time.argtypes = [ctypes.c_double]
        self._lib.refls_set_time(t)

    def wavegen_precalc(self):
        """iowave::wavegen_precalc: the generation zone's targets at the clock."""
        if self._lib.refls_wavegen_precalc() != 0:
            raise RuntimeError("no wave generator")

    def iowave_weights(self):
        """(relax4_wg, relax4_nb) per interior column as (nx, ny) arrays, -1
        outside the zones."""
        wg, wb = np.zeros(self.nx * self.ny), np.zeros(self.nx * self.ny)
        self._lib.refls_iowave_weights.argtypes = [_D, _D]
        if self._lib.refls_iowave_weights(_dp(wg), _dp(wb)) != 0:
            raise RuntimeError("no wave generator")
        return wg.reshape(self.nx, self.ny), wb.reshape(self.nx, self.ny)

    def iowave_targets(self):
        """(lsval, ramp) of the generation zone at the last wavegen_precalc."""
        n = self.nx * self.ny * self.nz
        ls, ramp = np.zeros(n), np.zeros(1)
        self._lib.refls_iowave_targets.argtypes = [_D, ctypes.c_long, _D]
        self._lib.refls_iowave_targets.restype = ctypes.c_long
        m = self._lib.refls_iowave_targets(_dp(ls), n, _dp(ramp))
        if m < 0:
            raise RuntimeError("no wave generator")
        return ls[:m].copy(), float(ramp[0])

    def io_levels(self):
        """(phimean, phiout) after the last step's fsfinflow."""
        out = np.zeros(4)
        self._lib.refls_io_levels(_dp(out))
        return float(out[0]), float(out[1])


class AdapterOracle(RefOracle):
    """The reference's own objects plus the REEF3D-side adapter classes
    (``reef3d_b200/adapters/reef3d_b200_adapters.h``) compiled into
    ``oracle/_ref/libreef3d_adapter.so`` against the reference's headers.
    The ``refls_*`` calls run the reference on the CPU, the ``gpu_*`` calls
    run the adapters (and through them libreef3d_b200.so) on the same REEF3D
    lexer/fdm/ghostcell objects.  One grid per process; needs a GPU."""

    @classmethod
    def available(cls):
        return os.path.exists(ADAPTER_LIB)

    def __init__(self, *args, precision=0, resident=False, **kw):
        super().__init__(*args, path=ADAPTER_LIB, **kw)
        lib = self._lib
        lib.refad_weno_L.argtypes = [_D, _D]
        lib.refad_reinidisc_L.argtypes = [_D, _D]
        lib.refad_create.argtypes = [_I, _I]
        self._precision = precision
        if lib.refad_create(precision, 1 if resident else 0) != 0:
            raise RuntimeError("refad_create failed")

    def make_domain(self, nslabs):
        """Also build the slab-domain free-surface adapter (levelset_RK3_domain)."""
        self._lib.refad_create_domain.argtypes = [_I, _I]
        if self._lib.refad_create_domain(self._precision, nslabs) != 0:
            raise RuntimeError("refad_create_domain failed")

    def gpu_step_domain(self, dt):
        """freesurface::start of levelset_RK3_domain on a->phi."""
        self._lib.refls_set_dt(dt)
        self._lib.refad_step_domain()
        return self.get_field(0)

    def gpu_step(self, dt):
        """freesurface::start of levelset_RK3_gpu on a->phi."""
        self._lib.refls_set_dt(dt)
        self._lib.refad_step()
        return self.get_field(0)

    def gpu_update(self):
        self._lib.refad_update()
        return self._lib.refls_volume1(), self._lib.refls_volume2()

    def gpu_weno_L(self, phi):
        L = self.zeros()
        self._lib.refad_weno_L(_dp(np.ascontiguousarray(phi)), _dp(L))
        return L

    def gpu_reinidisc_L(self, phi):
        L = self.zeros()
        self._lib.refad_reinidisc_L(_dp(np.ascontiguousarray(phi)), _dp(L))
        return L

    def gpu_reini(self):
        self._lib.refad_reini()
        return self.get_field(0)

    def close(self):
        self._lib.refad_destroy()
