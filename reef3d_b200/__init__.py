"""reef3d_b200: B200-native level-set transport for REEF3D.

Python host layer over the C-ABI of ``libreef3d_b200.so``
(``include/reef3d_b200.h``).  The library is built in-tree by
``reef3d_b200/build.py``; importing this package loads it and raises if it
is missing (there is no CPU fallback).

``LevelSet`` owns one device-resident instance.  ``reef3d_b200.compat``
mirrors the reference's class interfaces (levelset_RK3, weno_hj_df_nug,
reini_RK3, reinidisc_f/fsf, ghostcell::start4) on host arrays in the
reference's field layout.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libreef3d_b200.so")

R3D_OK, R3D_EINVAL, R3D_ENOMEM, R3D_EDEVICE, R3D_ETIMEOUT, R3D_ESTATE = 0, 1, 2, 3, 4, 5
FP64, FP32 = 0, 1
PHI, U, V, W, L, WORK1, WORK2, RO, VISC, BODY = range(10)
LAYOUT_REEF3D, LAYOUT_DENSE = 0, 1
STAGE_CONVECTION, STAGE_REINIT = 0, 1
OPT_TILED, OPT_CHUNK, OPT_BAND64, OPT_WAIT_TEST, OPT_TILE_CFG = 0, 1, 2, 3, 4
OPT_TILE_CFG_REINIT, OPT_CHUNK_REINIT = 6, 7

_ERRNAMES = {1: "EINVAL", 2: "ENOMEM", 3: "EDEVICE", 4: "ETIMEOUT", 5: "ESTATE"}


class R3DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"r3d error {_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


class GridDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("xn", ctypes.POINTER(ctypes.c_double)), ("yn", ctypes.POINTER(ctypes.c_double)),
        ("zn", ctypes.POINTER(ctypes.c_double)),
        ("f43", ctypes.c_double), ("f44", ctypes.c_int), ("f45", ctypes.c_double), ("f49", ctypes.c_int),
        ("n47", ctypes.c_double), ("precision", ctypes.c_int),
        ("f46", ctypes.c_int), ("f47", ctypes.c_int),
    ]


class StateInfo(ctypes.Structure):
    """r3d_state_info: the header of the reference's restart state file."""
    _fields_ = [("count", ctypes.c_int), ("printcount", ctypes.c_int)] + [
        (n, ctypes.c_double) for n in ("simtime", "printtime", "sedprinttime", "fsfprinttime", "probeprinttime",
                                       "stateprinttime")]


# the fields of the reference's state file the library does not hold, in the
# order of r3d_write_reef3d_state's `extra`
STATE_EXTRA = ("topo", "press", "kin", "eps", "eddyv", "qbe", "conc")


def reef3d_state_name(num, rank=0):
    """The reference's state file name (src/cfd_state_filename.cpp:27)."""
    return "REEF3D-CFD-State-%08i-%06i.r3d" % (num, rank + 1)


class IoflowDesc(ctypes.Structure):
    """r3d_ioflow_desc: inflow (x-min) / outflow (x-max) faces and ioflow_f's flags."""
    _fields_ = [
        ("inflow", ctypes.c_int), ("outflow", ctypes.c_int), ("f50", ctypes.c_int), ("b77", ctypes.c_int),
        ("f56", ctypes.c_double), ("f60", ctypes.c_double), ("f61", ctypes.c_double), ("f62", ctypes.c_double),
        ("f64", ctypes.c_int), ("qi", ctypes.c_double), ("qo", ctypes.c_double),
    ]


class JobDesc(ctypes.Structure):
    """r3d_job_desc: one transport job of the serving runtime."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("steps", ctypes.c_int),
        ("f44", ctypes.c_int), ("n47", ctypes.c_double),
        ("nspheres", ctypes.c_int), ("spheres", ctypes.POINTER(ctypes.c_double)),
        ("nmodes", ctypes.c_int), ("modes", ctypes.POINTER(ctypes.c_double)),
    ]


class JobResult(ctypes.Structure):
    """r3d_job_result."""
    _fields_ = [
        ("state", ctypes.c_int), ("steps_done", ctypes.c_int), ("volume1", ctypes.c_double),
        ("volume2", ctypes.c_double), ("sim_time", ctypes.c_double), ("t_submit", ctypes.c_double),
        ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double), ("instance", ctypes.c_void_p),
    ]


# the reference's defaults of those flags (src/ini.cpp:208-441; F50 = 2)
IOFLOW_DEFAULTS = dict(inflow=1, outflow=1, f50=2, b77=1, f56=1.0e20, f60=-1.0e20, f61=-1.0e20, f62=-1.0e20,
                       f64=0, qi=0.0, qo=0.0)

_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_H = ctypes.c_void_p

# every symbol the C-ABI exports (include/reef3d_b200.h)
EXPORTS = {
    "r3d_create": ([ctypes.POINTER(GridDesc), ctypes.POINTER(_H)], ctypes.c_int),
    "r3d_destroy": ([_H], ctypes.c_int),
    "r3d_last_error": ([_H], ctypes.c_char_p),
    "r3d_footprint": ([ctypes.POINTER(GridDesc), ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "r3d_upload": ([_H, ctypes.c_int, _D, ctypes.c_int], ctypes.c_int),
    "r3d_download": ([_H, ctypes.c_int, _D, ctypes.c_int], ctypes.c_int),
    "r3d_set_dt": ([_H, ctypes.c_double], ctypes.c_int),
    "r3d_cfl_dt": ([_H, _D], ctypes.c_int),
    "r3d_ls_step": ([_H, ctypes.c_double], ctypes.c_int),
    "r3d_ls_run": ([_H, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "r3d_reinit": ([_H, ctypes.c_int], ctypes.c_int),
    "r3d_convection_L": ([_H, ctypes.c_int], ctypes.c_int),
    "r3d_reinidisc_L": ([_H, ctypes.c_int], ctypes.c_int),
    "r3d_ghost_fill": ([_H, ctypes.c_int], ctypes.c_int),
    "r3d_volume": ([_H, _D, _D], ctypes.c_int),
    "r3d_last_volume": ([_H, _D, _D], ctypes.c_int),
    "r3d_set_velocity_airy": ([_H] + [ctypes.c_double] * 4, ctypes.c_int),
    "r3d_set_fluid": ([_H, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double], ctypes.c_int),
    "r3d_fluid_update": ([_H, _D, _D], ctypes.c_int),
    "r3d_set_ioflow": ([_H, ctypes.POINTER(IoflowDesc)], ctypes.c_int),
    "r3d_set_ioflow_waves": ([_H, ctypes.POINTER(IoflowDesc)], ctypes.c_int),
    "r3d_set_direct_forcing": ([_H, ctypes.c_int], ctypes.c_int),
    "r3d_set_relaxation": ([_H, _D, _D, ctypes.c_double], ctypes.c_int),
    "r3d_set_relaxation_target": ([_H, _D, ctypes.c_longlong, ctypes.c_double], ctypes.c_int),
    "r3d_set_solid_forcing": ([_H, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "r3d_set_halo": ([_H, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "r3d_write_vtu": ([_H, ctypes.c_char_p], ctypes.c_int),
    "r3d_save_state": ([_H, ctypes.c_char_p], ctypes.c_int),
    "r3d_load_state": ([_H, ctypes.c_char_p], ctypes.c_int),
    "r3d_write_reef3d_state": ([_H, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "r3d_read_reef3d_state": ([_H, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "r3d_grid_spacing": ([ctypes.POINTER(GridDesc), _D], ctypes.c_int),
    "r3d_set_grid_spacing": ([_H, ctypes.c_double, ctypes.c_double, ctypes.c_double], ctypes.c_int),
    "r3d_halo_bytes": ([_H, ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "r3d_halo_copy": ([_H, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "r3d_cfl_max": ([_H, _D], ctypes.c_int),
    "r3d_cfl_dt_from_max": ([_H, _D, _D], ctypes.c_int),
    "r3d_io_levels": ([_H, _D, _D], ctypes.c_int),
    "r3d_set_step_count": ([_H, ctypes.c_longlong], ctypes.c_int),
    "r3d_set_velocity_scale": ([_H, ctypes.c_double], ctypes.c_int),
    "r3d_set_velocity_period": ([_H, ctypes.c_double], ctypes.c_int),
    "r3d_set_time": ([_H, ctypes.c_double], ctypes.c_int),
    "r3d_get_time": ([_H, _D], ctypes.c_int),
    "r3d_stage": ([_H, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "r3d_init_spheres_tg": ([_H, ctypes.c_int, _D, ctypes.c_int, _D], ctypes.c_int),
    "r3d_set_option": ([_H, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "r3d_get_option": ([_H, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "r3d_tile_config_count": ([], ctypes.c_int),
    "r3d_tile_chunk_candidates": ([ctypes.POINTER(ctypes.c_int), ctypes.c_int], ctypes.c_int),
    "r3d_tile_config_describe": ([ctypes.c_int] + [ctypes.POINTER(ctypes.c_int)] * 5, ctypes.c_int),
    "r3d_autotune": ([_H, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "r3d_sync": ([_H], ctypes.c_int),
    "r3d_stream": ([_H, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "r3d_launch_count": ([_H, ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "r3d_volume_dense_noalloc": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                  ctypes.c_void_p], ctypes.c_int),
    "r3d_batch_create": ([ctypes.POINTER(_H)], ctypes.c_int),
    "r3d_batch_destroy": ([_H], ctypes.c_int),
    "r3d_batch_last_error": ([_H], ctypes.c_char_p),
    "r3d_batch_add": ([_H, _H], ctypes.c_int),
    "r3d_batch_remove": ([_H, _H], ctypes.c_int),
    "r3d_batch_size": ([_H, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "r3d_batch_set_config": ([_H, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "r3d_batch_get_config": ([_H, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "r3d_batch_autotune": ([_H, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
                           ctypes.c_int),
    "r3d_batch_set_tile_config": ([_H, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "r3d_batch_get_tile_config": ([_H, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "r3d_batch_use_graph": ([_H, ctypes.c_int], ctypes.c_int),
    "r3d_batch_step": ([_H, ctypes.c_int], ctypes.c_int),
    "r3d_batch_sync": ([_H], ctypes.c_int),
    "r3d_batch_stream": ([_H, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "r3d_batch_launch_count": ([_H, ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "r3d_domain_create": ([ctypes.POINTER(GridDesc), ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_H)],
                          ctypes.c_int),
    "r3d_domain_destroy": ([_H], ctypes.c_int),
    "r3d_domain_last_error": ([_H], ctypes.c_char_p),
    "r3d_domain_slab": ([_H, ctypes.c_int, ctypes.POINTER(_H), ctypes.POINTER(ctypes.c_int),
                         ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "r3d_domain_upload": ([_H, ctypes.c_int, _D], ctypes.c_int),
    "r3d_domain_download": ([_H, ctypes.c_int, _D], ctypes.c_int),
    "r3d_domain_run": ([_H, ctypes.c_int, ctypes.c_double], ctypes.c_int),
    "r3d_domain_last_volume": ([_H, _D, _D], ctypes.c_int),
    "r3d_domain_get_dt": ([_H, _D], ctypes.c_int),
    "r3d_domain_set_fluid": ([_H] + [ctypes.c_double] * 4, ctypes.c_int),
    "r3d_domain_set_ioflow": ([_H, ctypes.POINTER(IoflowDesc)], ctypes.c_int),
    "r3d_domain_fluid_update": ([_H, _D, _D], ctypes.c_int),
    "r3d_serve_create": ([ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_H)], ctypes.c_int),
    "r3d_serve_destroy": ([_H], ctypes.c_int),
    "r3d_serve_last_error": ([_H], ctypes.c_char_p),
    "r3d_serve_submit": ([_H, ctypes.POINTER(JobDesc), ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "r3d_serve_poll": ([_H, ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "r3d_serve_status": ([_H, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), _D, _D,
                          ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "r3d_serve_result": ([_H, ctypes.c_longlong, ctypes.POINTER(JobResult)], ctypes.c_int),
    "r3d_serve_release": ([_H, ctypes.c_longlong], ctypes.c_int),
    "r3d_serve_batch": ([_H, ctypes.POINTER(_H)], ctypes.c_int),
}


def tile_chunks():
    """The z chunks the autotuners try (r3d_tile_chunk_candidates)."""
    lib = load_library()
    n = lib.r3d_tile_chunk_candidates(None, 0)
    buf = (ctypes.c_int * n)()
    lib.r3d_tile_chunk_candidates(buf, n)
    return list(buf)


def tile_configs():
    """[(tx, ty, rows_per_thread, ring, threads)] of the tiled kernels'
    configurations, by id."""
    lib = load_library()
    out = []
    for c in range(lib.r3d_tile_config_count()):
        v = [ctypes.c_int() for _ in range(5)]
        if lib.r3d_tile_config_describe(c, *(ctypes.byref(x) for x in v)) != R3D_OK:
            raise R3DError(R3D_EINVAL, f"tile configuration {c}")
        out.append(tuple(x.value for x in v))
    return out


def load_library(path=LIB_PATH):
    """Load libreef3d_b200.so (fails loudly if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: run `python reef3d_b200/build.py` (no CPU fallback exists)")
    lib = ctypes.CDLL(path)
    for name, (args, res) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _check(rc, h=None):
    if rc != R3D_OK:
        msg = _lib.r3d_last_error(h)
        raise R3DError(rc, msg.decode() if msg else "")


def _extra_arrays(extra, dims, fill):
    """The 7 `extra` pointers of the state-file calls: dense arrays (shape
    (nz, ny, nx), qbe (ny, nx)) given (fill) or allocated to receive."""
    if extra is None:
        return None, None
    nx, ny, nz = dims
    keep, ptrs = [], (_D * len(STATE_EXTRA))()
    for q, name in enumerate(STATE_EXTRA):
        shape = (ny, nx) if name == "qbe" else (nz, ny, nx)
        a = extra.get(name)
        if a is None and fill:
            keep.append(None)
            continue
        a = np.zeros(shape) if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(shape)
        keep.append(a)
        ptrs[q] = _dp(a)
    return keep, ptrs


def _dp(a):
    return a.ctypes.data_as(_D)


def uniform_nodes(n, length=1.0, origin=0.0):
    """Node coordinates for node indices -5..n+5 of a uniform axis (n+11
    values), x_i = origin + i*(length/n), as a DIVEMesh grid stores them."""
    h = length / n
    return np.array([origin + i * h for i in range(-5, n + 6)], dtype=np.float64)


def make_desc(nx, ny, nz, xn, yn, zn, f43=0.55, f44=3, f45=2.1, f49=1, n47=0.3, precision=FP64, f46=0, f47=10):
    xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (xn, yn, zn)]
    for a, n in zip(xs, (nx, ny, nz)):
        if a.shape != (n + 11,):
            raise ValueError(f"node array of an axis with {n} cells needs {n + 11} values, got {a.shape}")
    d = GridDesc(nx, ny, nz, _dp(xs[0]), _dp(xs[1]), _dp(xs[2]), f43, f44, f45, f49, n47, precision, f46, f47)
    d._keep = xs
    return d


def footprint(nx, ny, nz, precision=FP32):
    """Device bytes of one instance (fields, tables, scratch)."""
    load_library()
    d = make_desc(nx, ny, nz, uniform_nodes(nx), uniform_nodes(ny), uniform_nodes(nz), precision=precision)
    out = ctypes.c_size_t()
    _check(_lib.r3d_footprint(ctypes.byref(d), ctypes.byref(out)))
    return out.value


def grid_spacing(nx, ny, nz, xn=None, yn=None, zn=None, f45=2.1):
    """(DXM, DYM, DZM, psi) of a grid (r3d_grid_spacing; host only)."""
    load_library()
    xn = uniform_nodes(nx) if xn is None else xn
    yn = uniform_nodes(ny) if yn is None else yn
    zn = uniform_nodes(nz) if zn is None else zn
    d = make_desc(nx, ny, nz, xn, yn, zn, 0.5, 2, f45, 1, 0.3, FP64, 0, 10)
    out = (ctypes.c_double * 4)()
    _check(_lib.r3d_grid_spacing(ctypes.byref(d), out))
    return tuple(out)


class LevelSet:
    """One device-resident level-set instance (the state levelset_RK3,
    weno_hj_df_nug and reini_RK3 act on in the reference)."""

    def __init__(self, nx, ny, nz, xn=None, yn=None, zn=None, f43=0.55, f44=3, f45=2.1, f49=1, n47=0.3,
                 precision=FP64, f46=0, f47=10):
        load_library()
        xn = uniform_nodes(nx) if xn is None else xn
        yn = uniform_nodes(ny) if yn is None else yn
        zn = uniform_nodes(nz) if zn is None else zn
        self.nx, self.ny, self.nz = nx, ny, nz
        self.f44, self.precision = f44, precision
        self.desc = make_desc(nx, ny, nz, xn, yn, zn, f43, f44, f45, f49, n47, precision, f46, f47)
        h = _H()
        _check(_lib.r3d_create(ctypes.byref(self.desc), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.r3d_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- shapes
    @property
    def reef3d_shape(self):
        return (self.nx + 6, self.ny + 6, self.nz + 6)

    @property
    def dense_shape(self):
        return (self.nz, self.ny, self.nx)

    def _shape(self, layout):
        return self.reef3d_shape if layout == LAYOUT_REEF3D else self.dense_shape

    # -- host copies
    def upload(self, field, arr, layout=LAYOUT_REEF3D):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != self._shape(layout):
            raise ValueError(f"expected shape {self._shape(layout)}, got {a.shape}")
        _check(_lib.r3d_upload(self.h, field, _dp(a), layout), self.h)

    def download(self, field, layout=LAYOUT_REEF3D, out=None):
        a = np.zeros(self._shape(layout), dtype=np.float64) if out is None else out
        _check(_lib.r3d_download(self.h, field, _dp(a), layout), self.h)
        return a

    def upload_ptr(self, field, ptr, layout=LAYOUT_REEF3D):
        """Upload from a raw host pointer (e.g. pinned memory)."""
        _check(_lib.r3d_upload(self.h, field, ctypes.cast(ptr, _D), layout), self.h)

    def download_ptr(self, field, ptr, layout=LAYOUT_REEF3D):
        _check(_lib.r3d_download(self.h, field, ctypes.cast(ptr, _D), layout), self.h)

    # -- path
    def set_dt(self, dt):
        _check(_lib.r3d_set_dt(self.h, dt), self.h)

    def cfl_dt(self):
        v = ctypes.c_double()
        _check(_lib.r3d_cfl_dt(self.h, ctypes.byref(v)), self.h)
        return v.value

    def step(self, dt=0.0):
        _check(_lib.r3d_ls_step(self.h, dt), self.h)

    def run(self, nsteps, adaptive=True):
        _check(_lib.r3d_ls_run(self.h, nsteps, 1 if adaptive else 0), self.h)

    def reinit(self, iters=0):
        _check(_lib.r3d_reinit(self.h, iters), self.h)

    def convection_L(self, field=PHI):
        _check(_lib.r3d_convection_L(self.h, field), self.h)

    def reinidisc_L(self, field=PHI):
        _check(_lib.r3d_reinidisc_L(self.h, field), self.h)

    def ghost_fill(self, field=PHI):
        _check(_lib.r3d_ghost_fill(self.h, field), self.h)

    def volume(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(_lib.r3d_volume(self.h, ctypes.byref(a), ctypes.byref(b)), self.h)
        return a.value, b.value

    def last_volume(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(_lib.r3d_last_volume(self.h, ctypes.byref(a), ctypes.byref(b)), self.h)
        return a.value, b.value

    def set_fluid(self, ro_water=998.2, visc_water=1.004e-6, ro_air=1.205, visc_air=1.41e-5):
        """Turn on the density/viscosity update of every step (fluid_update_fsf;
        defaults are the reference's W1..W4)."""
        _check(_lib.r3d_set_fluid(self.h, ro_water, visc_water, ro_air, visc_air), self.h)

    def fluid_update(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(_lib.r3d_fluid_update(self.h, ctypes.byref(a), ctypes.byref(b)), self.h)
        return a.value, b.value

    def set_velocity_scale(self, scale):
        _check(_lib.r3d_set_velocity_scale(self.h, scale), self.h)

    def set_solid_forcing(self, cells):
        """solid_forcing_lsm after each convection stage: cells = (n, 4)
        entries (i, j, k, side) of the direct-forcing boundary list; empty
        turns it off (r3d_set_solid_forcing)."""
        c = np.ascontiguousarray(np.asarray(cells, dtype=np.int32).reshape(-1))
        _check(_lib.r3d_set_solid_forcing(self.h, c.size // 4, c.ctypes.data_as(ctypes.POINTER(ctypes.c_int))),
               self.h)

    def set_direct_forcing(self, x45):
        """X45 direct-forcing convection stencils reading the BODY field
        (r3d_set_direct_forcing); 0 turns them off."""
        _check(_lib.r3d_set_direct_forcing(self.h, x45), self.h)

    def set_relaxation(self, w_gen=None, w_beach=None, phimean=0.0):
        """Wave-generation / numerical-beach relaxation zones after every
        convection stage (r3d_set_relaxation): weights per column as arrays
        of shape (nx, ny), negative outside the zone; None: no such zone."""
        def arr(a):
            if a is None:
                return None, None
            a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
            return a, a.ctypes.data_as(_D)
        g, gp = arr(w_gen)
        b, bp = arr(w_beach)
        _check(_lib.r3d_set_relaxation(self.h, gp, bp, phimean), self.h)

    def set_relaxation_target(self, lsval, ramp):
        """The generation zone's targets of the coming step and the ramp."""
        a = np.ascontiguousarray(lsval, dtype=np.float64).reshape(-1)
        _check(_lib.r3d_set_relaxation_target(self.h, a.ctypes.data_as(_D), a.size, ramp), self.h)

    def write_vtu(self, path):
        """The level set (and rho, viscosity) as a VTU file like the
        reference's printer (r3d_write_vtu)."""
        _check(_lib.r3d_write_vtu(self.h, os.fsencode(path)), self.h)

    def save_state(self, path):
        """Checkpoint every device field and step scalar (r3d_save_state)."""
        _check(_lib.r3d_save_state(self.h, os.fsencode(path)), self.h)

    def load_state(self, path):
        """Resume from a checkpoint of the same grid and configuration."""
        _check(_lib.r3d_load_state(self.h, os.fsencode(path)), self.h)

    def write_reef3d_state(self, path, count=0, printcount=0, simtime=0.0, times=None, extra=None):
        """The reference's restart state file of this instance
        (r3d_write_reef3d_state): level set and velocities from the device;
        `extra` maps names of STATE_EXTRA to dense arrays (x contiguous,
        `qbe` nx*ny), the others are written as zeros; `times` maps the
        header's other times (printtime, ...) to values."""
        info = StateInfo(count=count, printcount=printcount, simtime=simtime, **(times or {}))
        keep, ptrs = _extra_arrays(extra, (self.nx, self.ny, self.nz), fill=True)
        _check(_lib.r3d_write_reef3d_state(self.h, os.fsencode(path), ctypes.byref(info), ptrs), self.h)
        del keep

    def read_reef3d_state(self, path, extra=False):
        """Load the level set and velocities of a reference state file
        (r3d_read_reef3d_state); returns the header as a dict, with the
        file's other fields under "extra" (dense arrays) when `extra`."""
        info = StateInfo()
        want = {n: None for n in STATE_EXTRA} if extra else None
        keep, ptrs = _extra_arrays(want, (self.nx, self.ny, self.nz), fill=False)
        _check(_lib.r3d_read_reef3d_state(self.h, os.fsencode(path), ctypes.byref(info), ptrs), self.h)
        out = {n: getattr(info, n) for n, _ in StateInfo._fields_}
        if extra:
            out["extra"] = dict(zip(STATE_EXTRA, keep))
        return out

    def set_halo(self, zlo, zhi):
        """Mark the z-min / z-max faces as subdomain boundaries (r3d_set_halo)."""
        _check(_lib.r3d_set_halo(self.h, int(bool(zlo)), int(bool(zhi))), self.h)

    def set_grid_spacing(self, dxm, dym, dzm):
        """The whole grid's DXM, DYM, DZM for a subdomain instance."""
        _check(_lib.r3d_set_grid_spacing(self.h, dxm, dym, dzm), self.h)

    def halo_bytes(self):
        n = ctypes.c_size_t()
        _check(_lib.r3d_halo_bytes(self.h, ctypes.byref(n)), self.h)
        return n.value

    def halo_copy(self, field, side, dir, ptr):
        """dir 0: pack the 3 interior z planes next to side (0 z-min, 1
        z-max) into the device buffer at ptr; dir 1: unpack ptr into the 3
        ghost planes.  Asynchronous on the instance's stream."""
        _check(_lib.r3d_halo_copy(self.h, field, side, dir, ctypes.c_void_p(ptr)), self.h)

    def cfl_max(self):
        """(|u|max, |v|max, |w|max) over this instance's CFL faces."""
        out = (ctypes.c_double * 3)()
        _check(_lib.r3d_cfl_max(self.h, out), self.h)
        return tuple(out)

    def cfl_dt_from_max(self, vmax):
        """Time step from given maxima with this instance's smallest cell."""
        vm = (ctypes.c_double * 3)(*vmax)
        dt = ctypes.c_double()
        _check(_lib.r3d_cfl_dt_from_max(self.h, vm, ctypes.byref(dt)), self.h)
        return dt.value

    def set_ioflow(self, **flags):
        """Inflow / outflow faces with ioflow_f's hooks (r3d_set_ioflow):
        keys of IOFLOW_DEFAULTS, unspecified ones at the reference's
        defaults.  set_ioflow(off=True) restores the closed box;
        waves=True hands the faces to the wave generator's hooks instead
        (r3d_set_ioflow_waves)."""
        if flags.pop("off", False):
            _check(_lib.r3d_set_ioflow(self.h, None), self.h)
            return
        waves = flags.pop("waves", False)
        unknown = set(flags) - set(IOFLOW_DEFAULTS)
        if unknown:
            raise TypeError(f"unknown ioflow flags {sorted(unknown)}")
        d = IoflowDesc(**dict(IOFLOW_DEFAULTS, **flags))
        fn = _lib.r3d_set_ioflow_waves if waves else _lib.r3d_set_ioflow
        _check(fn(self.h, ctypes.byref(d)), self.h)

    def io_levels(self):
        """(phimean, phiout) measured by the last step's fsfinflow."""
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(_lib.r3d_io_levels(self.h, ctypes.byref(a), ctypes.byref(b)), self.h)
        return a.value, b.value

    def set_step_count(self, count):
        """lexer::count of the next step."""
        _check(_lib.r3d_set_step_count(self.h, count), self.h)

    def set_velocity_airy(self, amplitude, wavelength, depth, gravity=9.81):
        """Regenerate u, w from the Airy wave at the device clock before every step."""
        _check(_lib.r3d_set_velocity_airy(self.h, amplitude, wavelength, depth, gravity), self.h)

    def set_velocity_period(self, period):
        _check(_lib.r3d_set_velocity_period(self.h, period), self.h)

    def set_time(self, t):
        _check(_lib.r3d_set_time(self.h, t), self.h)

    def time(self):
        v = ctypes.c_double()
        _check(_lib.r3d_get_time(self.h, ctypes.byref(v)), self.h)
        return v.value

    def stage(self, kind, stage):
        _check(_lib.r3d_stage(self.h, kind, stage), self.h)

    def init_spheres_tg(self, spheres, modes):
        """Device-side initial fields: spheres = [(cx, cy, cz, r), ...],
        modes = [(k, A), ...] (see r3d_init_spheres_tg)."""
        sp = np.ascontiguousarray(np.asarray(spheres, dtype=np.float64).reshape(-1, 4))
        mo = np.ascontiguousarray(np.asarray(modes, dtype=np.float64).reshape(-1, 2))
        _check(_lib.r3d_init_spheres_tg(self.h, sp.shape[0], _dp(sp), mo.shape[0], _dp(mo)), self.h)

    def set_option(self, option, value):
        _check(_lib.r3d_set_option(self.h, option, int(value)), self.h)

    def autotune(self, cache_path=None):
        """Tile configuration and z chunk picked by timing (r3d_autotune);
        returns (cfg, chunk)."""
        c, k = ctypes.c_int(), ctypes.c_int()
        p = os.fsencode(cache_path) if cache_path else None
        _check(_lib.r3d_autotune(self.h, p, ctypes.byref(c), ctypes.byref(k)), self.h)
        return c.value, k.value

    def get_option(self, option):
        v = ctypes.c_int()
        _check(_lib.r3d_get_option(self.h, option, ctypes.byref(v)), self.h)
        return v.value

    def sync(self):
        _check(_lib.r3d_sync(self.h), self.h)

    def stream(self):
        s = ctypes.c_void_p()
        _check(_lib.r3d_stream(self.h, ctypes.byref(s)), self.h)
        return s.value

    def launch_count(self):
        c = ctypes.c_longlong()
        _check(_lib.r3d_launch_count(self.h, ctypes.byref(c)), self.h)
        return c.value


def _bcheck(rc, b=None):
    if rc != R3D_OK:
        msg = _lib.r3d_batch_last_error(b)
        raise R3DError(rc, msg.decode() if msg else "")


class Batch:
    """Many FP32 instances advanced together (one persistent launch per RK
    stage over all members, the step replayed from a CUDA graph)."""

    def __init__(self):
        load_library()
        b = _H()
        _bcheck(_lib.r3d_batch_create(ctypes.byref(b)))
        self.b = b
        self.members = []

    def close(self):
        if getattr(self, "b", None) is not None and _lib is not None:
            _lib.r3d_batch_destroy(self.b)
            self.b = None
            self.members = []

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add(self, ls):
        _bcheck(_lib.r3d_batch_add(self.b, ls.h), self.b)
        self.members.append(ls)

    def remove(self, ls):
        _bcheck(_lib.r3d_batch_remove(self.b, ls.h), self.b)
        self.members.remove(ls)

    def size(self):
        n = ctypes.c_int()
        _bcheck(_lib.r3d_batch_size(self.b, ctypes.byref(n)), self.b)
        return n.value

    def set_config(self, rows, ctas_per_sm):
        _bcheck(_lib.r3d_batch_set_config(self.b, rows, ctas_per_sm), self.b)

    def config(self):
        r, c = ctypes.c_int(), ctypes.c_int()
        _bcheck(_lib.r3d_batch_get_config(self.b, ctypes.byref(r), ctypes.byref(c)), self.b)
        return r.value, c.value

    def autotune(self, cache_path=None):
        """(rows, ctas_per_sm) of the cell members; the tiled members' choice
        is tile_config()."""
        r, c = ctypes.c_int(), ctypes.c_int()
        p = cache_path.encode() if cache_path else None
        _bcheck(_lib.r3d_batch_autotune(self.b, p, ctypes.byref(r), ctypes.byref(c)), self.b)
        return r.value, c.value

    def set_tile_config(self, cfg, chunk):
        _bcheck(_lib.r3d_batch_set_tile_config(self.b, cfg, chunk), self.b)

    def tile_config(self):
        """(tile configuration id, z chunk) of the tiled members' launches."""
        c, k = ctypes.c_int(), ctypes.c_int()
        _bcheck(_lib.r3d_batch_get_tile_config(self.b, ctypes.byref(c), ctypes.byref(k)), self.b)
        return c.value, k.value

    def use_graph(self, on):
        _bcheck(_lib.r3d_batch_use_graph(self.b, 1 if on else 0), self.b)

    def step(self, nsteps=1):
        _bcheck(_lib.r3d_batch_step(self.b, nsteps), self.b)

    def sync(self):
        _bcheck(_lib.r3d_batch_sync(self.b), self.b)

    def stream(self):
        s = ctypes.c_void_p()
        _bcheck(_lib.r3d_batch_stream(self.b, ctypes.byref(s)), self.b)
        return s.value

    def launch_count(self):
        c = ctypes.c_longlong()
        _bcheck(_lib.r3d_batch_launch_count(self.b, ctypes.byref(c)), self.b)
        return c.value
