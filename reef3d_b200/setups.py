"""Initial level sets and prescribed velocities of the benchmark workloads
(the role of the reference's analytic benchmark setups, src/benchmark_*.cpp,
for the shapes this project measures).

Every array is returned in the reference's padded field layout
(nx+6, ny+6, nz+6), k contiguous, so it can be handed to the reference's
objects and to ``LevelSet.upload`` alike.  Velocities are staggered like the
reference's: u(i,j,k) sits on the x face i+1/2, v on the y face j+1/2, w on
the z face k+1/2 (src/flux_HJ_CDS2.cpp:59-127).  The level set is negative
inside the body.
"""
import math

import numpy as np

from . import uniform_nodes


def centres(xn):
    """Cell centres for padded indices -3..n+2 from nodes -5..n+5."""
    return 0.5 * (xn[2:-3] + xn[3:-2])


def faces(xn):
    """Face (i+1/2) positions for padded indices -3..n+2: node i+1."""
    return xn[3:-2]


def _mesh(a, b, c):
    return np.meshgrid(a, b, c, indexing="ij")


def _zero_y_ghosts(a):
    """2D (ny == 1): the y ghost planes of the reference's padded field hold
    zeros (nothing on the path writes them; the F49=0 reinitialisation test
    reads them, src/reinidisc_fsf.cpp:70-72)."""
    a[:, :3, :] = 0.0
    a[:, 4:, :] = 0.0
    return a


class Case:
    """Grid, control flags and fields of one instance."""

    def __init__(self, name, nx, ny, nz, xn, yn, zn, phi, u, v, w, f43=0.5, f44=2, f45=2.1, f49=1, n47=0.125,
                 t_end=None, vel_time=None):
        self.name = name
        self.nx, self.ny, self.nz = nx, ny, nz
        self.xn, self.yn, self.zn = xn, yn, zn
        self.phi, self.u, self.v, self.w = phi, u, v, w
        self.f43, self.f44, self.f45, self.f49, self.n47 = f43, f44, f45, f49, n47
        self.t_end = t_end
        self.vel_time = vel_time  # callable t -> scale of the stored velocity, or None

    @property
    def cells(self):
        return self.nx * self.ny * self.nz

    def flags(self):
        return dict(f43=self.f43, f44=self.f44, f45=self.f45, f49=self.f49, n47=self.n47)


def slotted_disk_sdf(X, Z, cx=0.5, cz=0.75, r=0.15, slot_w=0.05, slot_depth=0.25):
    """Exact signed distance to a disc of radius r at (cx,cz) with a
    vertical slot of width slot_w and depth slot_depth cut from the bottom.
    Negative inside the slotted disc."""
    hw = 0.5 * slot_w
    zb = cz - math.sqrt(r * r - hw * hw)  # where the slot walls meet the circle
    zt = cz - r + slot_depth              # slot top
    dx, dz = X - cx, Z - cz
    rho = np.sqrt(dx * dx + dz * dz)
    # distance to the circle arc outside the slot opening
    with np.errstate(invalid="ignore", divide="ignore"):
        px = cx + r * dx / np.where(rho > 0, rho, 1.0)
        pz = cz + r * dz / np.where(rho > 0, rho, 1.0)
    on_gap = (np.abs(px - cx) < hw) & (pz < cz)
    d_arc = np.abs(rho - r)
    e1 = np.hypot(X - (cx - hw), Z - zb)
    e2 = np.hypot(X - (cx + hw), Z - zb)
    d_arc = np.where(on_gap, np.minimum(e1, e2), d_arc)

    def seg_v(x0, z0, z1):
        zc = np.clip(Z, z0, z1)
        return np.hypot(X - x0, Z - zc)

    def seg_h(z0, x0, x1):
        xc = np.clip(X, x0, x1)
        return np.hypot(X - xc, Z - z0)

    d = np.minimum(d_arc, seg_v(cx - hw, zb, zt))
    d = np.minimum(d, seg_v(cx + hw, zb, zt))
    d = np.minimum(d, seg_h(zt, cx - hw, cx + hw))
    inside = (rho < r) & ~((np.abs(X - cx) < hw) & (Z < zt))
    return np.where(inside, -d, d)


def slotted_disk(n=128, cfl=0.1):
    """2D slotted-disc rigid rotation on [0,1]^2 (x-z plane, one cell thick
    in y): u = 2pi(0.5-z), w = 2pi(x-0.5), period 1."""
    xn, zn = uniform_nodes(n), uniform_nodes(n)
    yn = uniform_nodes(1, length=1.0 / n)
    xc, yc, zc = centres(xn), centres(yn), centres(zn)
    X, Y, Z = _mesh(xc, yc, zc)
    phi = slotted_disk_sdf(X, Z)
    _zero_y_ghosts(phi)
    _, _, Zu = _mesh(faces(xn), yc, zc)
    u = 2.0 * math.pi * (0.5 - Zu)
    Xw, _, _ = _mesh(xc, yc, faces(zn))
    w = 2.0 * math.pi * (Xw - 0.5)
    v = np.zeros_like(u)
    return Case("slotted_disk_2d", n, 1, n, xn, yn, zn, *(np.ascontiguousarray(a) for a in (phi, u, v, w)),
                f43=0.5, f44=2, n47=cfl / 2.0, t_end=1.0)


def vortex3d(n=256, cfl=0.25, T=3.0):
    """3D single-vortex deformation of a sphere (r=0.15 at (0.35,0.35,0.35))
    on the unit cube; the stored velocity is the spatial part and
    ``vel_time(t) = cos(pi t/T)`` scales it."""
    xn = uniform_nodes(n)
    xc, xf = centres(xn), faces(xn)
    X, Y, Z = _mesh(xc, xc, xc)
    phi = np.sqrt((X - 0.35) ** 2 + (Y - 0.35) ** 2 + (Z - 0.35) ** 2) - 0.15
    s = np.sin
    pi = math.pi
    sx, sy, sz = s(pi * xc), s(pi * xc), s(pi * xc)
    s2x, s2y, s2z = s(2 * pi * xc), s(2 * pi * xc), s(2 * pi * xc)
    fx, f2x = s(pi * xf), s(2 * pi * xf)
    u = 2.0 * (fx ** 2)[:, None, None] * s2y[None, :, None] * s2z[None, None, :]
    v = -s2x[:, None, None] * (fx ** 2)[None, :, None] * s2z[None, None, :]
    w = -s2x[:, None, None] * s2y[None, :, None] * (fx ** 2)[None, None, :]
    del sx, sy, sz, f2x
    return Case("vortex3d", n, n, n, xn, xn, xn, *(np.ascontiguousarray(a) for a in (phi, u, v, w)),
                f43=0.5, f44=2, n47=cfl / 2.0, t_end=T, vel_time=lambda t: math.cos(math.pi * t / T))


def wave_tank(nx=1024, ny=128, nz=256, dx=0.01, depth=0.5, amp=0.05, wavelength=2.0, t=0.0, cfl=0.2, g=9.81,
              velocity=True):
    """Wave-tank-shaped free surface: phi = z - (depth + amp cos(kx)) with the
    linear (Airy) orbital velocity of that wave at time t, bed at z=0, carried
    upward unchanged above the still-water level.
    velocity=False leaves u, v, w as None (for instances whose velocity the
    device's Airy generator writes)."""
    xn = uniform_nodes(nx, nx * dx)
    yn = uniform_nodes(ny, ny * dx)
    zn = uniform_nodes(nz, nz * dx)
    xc, yc, zc = centres(xn), centres(yn), centres(zn)
    k = 2.0 * math.pi / wavelength
    om = math.sqrt(g * k * math.tanh(k * depth))
    phi = (zc[None, None, :] - (depth + amp * np.cos(k * xc))[:, None, None]) * np.ones((1, len(yc), 1))
    if not velocity:
        return Case("wave_tank", nx, ny, nz, xn, yn, zn, np.ascontiguousarray(phi), None, None, None,
                    f43=0.5, f44=1, n47=cfl / 2.0)
    a = amp * om / math.sinh(k * depth)
    # above the still-water level the surface value (see r3d_set_velocity_airy)
    uf = a * np.cosh(k * np.minimum(zc, depth))[None, :] * np.cos(k * faces(xn) - om * t)[:, None]
    wf = a * np.sinh(k * np.minimum(faces(zn), depth))[None, :] * np.sin(k * xc - om * t)[:, None]
    u = np.broadcast_to(uf[:, None, :], phi.shape)
    w = np.broadcast_to(wf[:, None, :], phi.shape)
    v = np.zeros(phi.shape)
    return Case("wave_tank", nx, ny, nz, xn, yn, zn, *(np.ascontiguousarray(x) for x in (phi, u, v, w)),
                f43=0.5, f44=1, n47=cfl / 2.0)


def sphere_union_sdf(X, Y, Z, centres_, radii, two_d=False):
    d = None
    for c, r in zip(centres_, radii):
        if two_d:
            e = np.sqrt((X - c[0]) ** 2 + (Z - c[2]) ** 2) - r
        else:
            e = np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - r
        d = e if d is None else np.minimum(d, e)
    return d


def taylor_green(X, Y, Z, modes, comp, two_d=False):
    """Sum of Taylor-Green modes (k, amplitude); divergence-free in 3D for
    each mode: u = A sin(kx)cos(ky)cos(kz), v = -A cos(kx)sin(ky)cos(kz), w=0
    (2D: u = A sin(kx)cos(kz), w = -A cos(kx)sin(kz))."""
    out = np.zeros(np.broadcast(X, Y, Z).shape)
    for k, A in modes:
        kx = k * math.pi
        if two_d:
            if comp == 0:
                out += A * np.sin(kx * X) * np.cos(kx * Z)
            elif comp == 2:
                out += -A * np.cos(kx * X) * np.sin(kx * Z)
        else:
            if comp == 0:
                out += A * np.sin(kx * X) * np.cos(kx * Y) * np.cos(kx * Z)
            elif comp == 1:
                out += -A * np.cos(kx * X) * np.sin(kx * Y) * np.cos(kx * Z)
    return out


def random_instance(rng, n_edge_choices=None, two_d=None, name="ensemble", f44=2, cfl=0.25, edge=None):
    """One ensemble/serving instance: union of 1-8 spheres (centres U[0.2,0.8],
    radii U[0.05,0.2]) advected by 4 Taylor-Green modes (wavenumbers in
    {1,2,3}, amplitudes N(0,0.5)).  Draw order: 2D flag, edges, sphere
    count, centres, radii, modes."""
    if two_d is None:
        two_d = bool(rng.integers(0, 2))
    if edge is None:
        choices = n_edge_choices if n_edge_choices is not None else list(range(64, 257, 32))
        nx = int(rng.choice(choices))
        nz = int(rng.choice(choices))
        ny = 1 if two_d else int(rng.choice(choices))
    else:
        nx, ny, nz = edge
    ns = int(rng.integers(1, 9))
    cs = rng.uniform(0.2, 0.8, size=(ns, 3))
    rs = rng.uniform(0.05, 0.2, size=ns)
    modes = [(int(rng.integers(1, 4)), float(rng.normal(0.0, 0.5))) for _ in range(4)]
    xn = uniform_nodes(nx)
    yn = uniform_nodes(ny) if not two_d else uniform_nodes(1, length=1.0 / nx)
    zn = uniform_nodes(nz)
    xc, yc, zc = centres(xn), centres(yn), centres(zn)
    X, Y, Z = _mesh(xc, yc, zc)
    phi = sphere_union_sdf(X, Y, Z, cs, rs, two_d)
    if two_d:
        _zero_y_ghosts(phi)
    Xu, Yu, Zu = _mesh(faces(xn), yc, zc)
    u = taylor_green(Xu, Yu, Zu, modes, 0, two_d)
    if two_d:
        v = np.zeros_like(u)
    else:
        Xv, Yv, Zv = _mesh(xc, faces(yn), zc)
        v = taylor_green(Xv, Yv, Zv, modes, 1, two_d)
    Xw, Yw, Zw = _mesh(xc, yc, faces(zn))
    w = taylor_green(Xw, Yw, Zw, modes, 2, two_d)
    case = Case(name, nx, ny, nz, xn, yn, zn, *(np.ascontiguousarray(a) for a in (phi, u, v, w)),
                f43=0.5, f44=f44, n47=cfl / 2.0)
    case.spheres = [(float(c[0]), float(c[1]), float(c[2]), float(r)) for c, r in zip(cs, rs)]
    case.modes = modes
    return case
