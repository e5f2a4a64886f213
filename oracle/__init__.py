"""ORACLE — test infrastructure only, never part of the product path.

ctypes wrapper over ``liboracle.so``, the C++17 restatement of the reference's FP64 CPU solver
(vortexlab ``src/lattice.rs``, ``src/sim.rs``, ``src/geometry.rs``, ``src/cases/*.rs``,
``src/signal.rs``). Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module. The class and method names follow the reference's Rust API
(``Builder``, ``Sim``, ``Channel``) so parity tests read like the reference's own tests.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

BGK, TRT = 0, 1
PARABOLIC, UNIFORM, UNIFORM_OPEN = 0, 1, 2
VEL_NONE, VEL_CONST, VEL_PARABOLIC, VEL_ROTATION = 0, 1, 2, 3
SHARP, CHAMFERED, ROUNDED, RECESSED, DOUBLE_RECESSED = 0, 1, 2, 3, 4

_lib = None


def build():
    """Compile liboracle.so with the committed Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    d, i, u64, sz, vp = C.c_double, C.c_int, C.c_uint64, C.c_size_t, C.c_void_p
    P = C.POINTER
    sig = {
        "vlo_last_error": (C.c_char_p, []),
        "vlo_equilibrium": (None, [d, d, d, P(d)]),
        "vlo_moments": (None, [P(d), P(d)]),
        "vlo_collide_bgk": (None, [P(d), d, P(d)]),
        "vlo_collide_trt": (None, [P(d), d, d, P(d)]),
        "vlo_collide_forced": (None, [P(d), d, d, d, d, P(d)]),
        "vlo_omegas": (None, [i, d, d, P(d)]),
        "vlo_tau_for": (d, [d]),
        "vlo_shape_circle": (vp, [d, d, d]),
        "vlo_shape_polygon": (vp, [P(d), i]),
        "vlo_shape_rounded_square": (vp, [d, d, d, d]),
        "vlo_shape_rotated": (vp, [vp, d, d, d]),
        "vlo_shape_translated": (vp, [vp, d, d]),
        "vlo_shape_outside_band": (vp, [d, d]),
        "vlo_shape_star": (vp, [d, d, P(d), i, d]),
        "vlo_shape_ellipse": (vp, [d, d, d, d]),
        "vlo_shape_section": (vp, [i, d, d, d, d, d]),
        "vlo_shape_bitmap": (vp, [sz, sz, P(C.c_float), d, d, d]),
        "vlo_shape_disks": (vp, [P(d), sz]),
        "vlo_shape_free": (None, [vp]),
        "vlo_shape_inside": (i, [vp, d, d]),
        "vlo_cut_fraction": (d, [vp, d, d, d, d]),
        "vlo_bounding_box": (i, [vp, d, d, P(d)]),
        "vlo_builder_new": (vp, [sz, sz]),
        "vlo_builder_free": (None, [vp]),
        "vlo_builder_config": (None, [vp, i, i, d, i, d, d, d]),
        "vlo_builder_add_wall": (i, [vp, i, P(d), i, C.c_long, vp]),
        "vlo_builder_add_pressure": (i, [vp, d]),
        "vlo_builder_add_radiating": (i, [vp, d]),
        "vlo_builder_fill_rect": (None, [vp, sz, sz, sz, sz, i]),
        "vlo_builder_fill_shape": (i, [vp, i]),
        "vlo_sim_build": (vp, [vp, sz]),
        "vlo_sim_free": (None, [vp]),
        "vlo_sim_nx": (sz, [vp]),
        "vlo_sim_ny": (sz, [vp]),
        "vlo_sim_fluid_nodes": (sz, [vp]),
        "vlo_sim_link_count": (sz, [vp]),
        "vlo_sim_bnode_count": (sz, [vp]),
        "vlo_sim_pnode_count": (sz, [vp]),
        "vlo_sim_threads": (sz, [vp]),
        "vlo_sim_set_threads": (None, [vp, sz]),
        "vlo_sim_ngroups": (i, [vp]),
        "vlo_sim_t": (u64, [vp]),
        "vlo_sim_flags": (None, [vp, P(C.c_uint8)]),
        "vlo_sim_init_arrays": (None, [vp, P(d), P(d), P(d)]),
        "vlo_sim_link_table": (None, [vp, P(C.c_int32), P(C.c_int32), P(d), P(C.c_int32)]),
        "vlo_sim_step": (None, [vp, u64]),
        "vlo_sim_set_vscale": (None, [vp, i, d]),
        "vlo_sim_get_vscale": (d, [vp, i]),
        "vlo_sim_set_outflow_target": (None, [vp, i, d]),
        "vlo_sim_outlet_density_offset": (d, [vp]),
        "vlo_sim_force": (None, [vp, P(d)]),
        "vlo_sim_get_f": (None, [vp, P(d)]),
        "vlo_sim_set_f": (None, [vp, P(d)]),
        "vlo_sim_macros": (None, [vp, sz, sz, P(d)]),
        "vlo_sim_total_mass": (d, [vp]),
        "vlo_sim_total_momentum": (None, [vp, P(d)]),
        "vlo_sim_max_speed": (d, [vp]),
        "vlo_sim_vorticity": (None, [vp, P(C.c_float)]),
        "vlo_sim_probe_density": (d, [vp, d, d]),
        "vlo_sim_probe_density_at_wall": (d, [vp, d, d, d, d]),
        "vlo_sim_state_hash": (u64, [vp]),
        "vlo_ramp": (d, [u64, u64]),
        "vlo_channel_new": (vp, [sz, sz, i, d, d, i, d, vp, u64, P(d), sz]),
        "vlo_channel_free": (None, [vp]),
        "vlo_channel_sim": (vp, [vp]),
        "vlo_channel_set_absorbing": (None, [vp, i]),
        "vlo_channel_u_ref": (d, [vp]),
        "vlo_channel_run": (None, [vp, u64, P(d), P(d), d, d, d]),
        "vlo_fft": (None, [P(d), P(d), sz]),
        "vlo_mean": (d, [P(d), sz]),
        "vlo_rms": (d, [P(d), sz]),
        "vlo_dominant_frequency": (None, [P(d), sz, d, P(d)]),
        "vlo_peaks": (sz, [P(d), sz, P(d), P(d), sz]),
        "vlo_crossing_frequency": (i, [P(d), sz, d, P(d)]),
        "vlo_sample_at": (d, [P(d), sz, d]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _arr(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


class OracleError(RuntimeError):
    pass


def _err():
    return OracleError(lib().vlo_last_error().decode())


# ------------------------------------------------------------------ lattice
def equilibrium(rho, ux, uy):
    out = np.zeros(9)
    lib().vlo_equilibrium(rho, ux, uy, _dp(out))
    return out


def moments(f):
    f = _arr(f)
    out = np.zeros(3)
    lib().vlo_moments(_dp(f), _dp(out))
    return tuple(out)


def collide_bgk(f, omega):
    f = _arr(f)
    out = np.zeros(9)
    lib().vlo_collide_bgk(_dp(f), omega, _dp(out))
    return out


def collide_trt(f, op, om):
    f = _arr(f)
    out = np.zeros(9)
    lib().vlo_collide_trt(_dp(f), op, om, _dp(out))
    return out


def collide_forced(f, op, om, gx, gy):
    f = _arr(f)
    out = np.zeros(9)
    lib().vlo_collide_forced(_dp(f), op, om, gx, gy, _dp(out))
    return out


def omegas(collision, magic, tau):
    out = np.zeros(2)
    lib().vlo_omegas(collision, magic, tau, _dp(out))
    return tuple(out)


def tau_for(nu):
    return lib().vlo_tau_for(nu)


def ramp(t, steps):
    return lib().vlo_ramp(t, steps)


# ------------------------------------------------------------------ shapes
class Shape:
    """Owning handle to an oracle shape; wrapping shapes take ownership of the inner one."""

    def __init__(self, ptr):
        if not ptr:
            raise _err()
        self.ptr = ptr

    def take(self):
        p, self.ptr = self.ptr, None
        return p

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().vlo_shape_free(self.ptr)

    def inside(self, x, y):
        return bool(lib().vlo_shape_inside(self.ptr, x, y))

    def cut_fraction(self, x, y, dx, dy):
        return lib().vlo_cut_fraction(self.ptr, x, y, dx, dy)

    def bounding_box(self, reach, step):
        out = np.zeros(4)
        return tuple(out) if lib().vlo_bounding_box(self.ptr, reach, step, _dp(out)) else None

    @staticmethod
    def circle(cx, cy, r):
        return Shape(lib().vlo_shape_circle(cx, cy, r))

    @staticmethod
    def polygon(pts):
        xy = _arr(pts).reshape(-1)
        return Shape(lib().vlo_shape_polygon(_dp(xy), len(xy) // 2))

    @staticmethod
    def rounded_square(cx, cy, half, r):
        return Shape(lib().vlo_shape_rounded_square(cx, cy, half, r))

    @staticmethod
    def rotated(inner, cx, cy, angle):
        return Shape(lib().vlo_shape_rotated(inner.take(), cx, cy, angle))

    @staticmethod
    def translated(inner, dx, dy):
        return Shape(lib().vlo_shape_translated(inner.take(), dx, dy))

    @staticmethod
    def outside_band(y0, y1):
        return Shape(lib().vlo_shape_outside_band(y0, y1))

    @staticmethod
    def star(cx, cy, radii, phase):
        r = _arr(radii)
        return Shape(lib().vlo_shape_star(cx, cy, _dp(r), len(r), phase))

    @staticmethod
    def ellipse(cx, cy, a, b):
        return Shape(lib().vlo_shape_ellipse(cx, cy, a, b))

    @staticmethod
    def disks(cxcyr):
        a = _arr(cxcyr).reshape(-1)
        return Shape(lib().vlo_shape_disks(_dp(a), len(a) // 3))

    @staticmethod
    def section(corner, b, cx, cy, d, angle=0.0):
        return Shape(lib().vlo_shape_section(corner, b, cx, cy, d, angle))

    @staticmethod
    def bitmap(level, x0, y0, scale):
        lv = np.ascontiguousarray(level, dtype=np.float32)
        h, w = lv.shape
        return Shape(lib().vlo_shape_bitmap(w, h, lv.ctypes.data_as(C.POINTER(C.c_float)), x0, y0, scale))


# ------------------------------------------------------------------ builder / sim
class Builder:
    """src/sim.rs:70-137. Attributes mirror the reference's pub fields."""

    def __init__(self, nx, ny):
        self.ptr = lib().vlo_builder_new(nx, ny)
        if not self.ptr:
            raise _err()
        self.nx, self.ny = nx, ny
        self.periodic_x = False
        self.periodic_y = False
        self.tau = 1.0
        self.collision = TRT
        self.magic = 3.0 / 16.0
        self.accel = (0.0, 0.0)

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().vlo_builder_free(self.ptr)

    def add_wall(self, velocity=None, vgroup=0, fgroup=None, shape=None):
        """velocity: None | ("const", ux, uy) | ("parabolic", u_mean, h) | ("rotation", cx, cy)."""
        kind, params = _velocity(velocity)
        p = _arr(params)
        k = lib().vlo_builder_add_wall(self.ptr, kind, _dp(p), vgroup, -1 if fgroup is None else fgroup,
                                       shape.take() if shape is not None else None)
        if k < 0:
            raise _err()
        return k

    def add_static_wall(self):
        return self.add_wall()

    def add_pressure(self, rho):
        return lib().vlo_builder_add_pressure(self.ptr, rho)

    def add_radiating(self, rho):
        return lib().vlo_builder_add_radiating(self.ptr, rho)

    def fill_rect(self, x0, x1, y0, y1, kind):
        lib().vlo_builder_fill_rect(self.ptr, x0, x1, y0, y1, kind)

    def fill_shape(self, kind):
        if lib().vlo_builder_fill_shape(self.ptr, kind) != 0:
            raise _err()

    def build(self, threads=1):
        lib().vlo_builder_config(self.ptr, int(self.periodic_x), int(self.periodic_y), self.tau,
                                 self.collision, self.magic, self.accel[0], self.accel[1])
        p, self.ptr = self.ptr, None
        s = lib().vlo_sim_build(p, threads)
        if not s:
            raise _err()
        return Sim(s, owned=True)


def _velocity(v):
    if v is None:
        return VEL_NONE, [0, 0, 0, 0]
    tag = v[0]
    vals = list(v[1:]) + [0.0] * (4 - len(v[1:]))
    return {"const": VEL_CONST, "parabolic": VEL_PARABOLIC, "rotation": VEL_ROTATION}[tag], vals


class _VScale:
    def __init__(self, sim):
        self.sim = sim

    def __getitem__(self, g):
        return lib().vlo_sim_get_vscale(self.sim.ptr, g)

    def __setitem__(self, g, v):
        lib().vlo_sim_set_vscale(self.sim.ptr, g, v)


class Sim:
    """src/sim.rs:180-673."""

    def __init__(self, ptr, owned):
        self.ptr = ptr
        self.owned = owned
        L = lib()
        self.nx, self.ny = L.vlo_sim_nx(ptr), L.vlo_sim_ny(ptr)
        self.n = self.nx * self.ny

    def __del__(self):
        if getattr(self, "owned", False) and self.ptr:
            lib().vlo_sim_free(self.ptr)

    @property
    def vscale(self):
        return _VScale(self)

    @property
    def t(self):
        return lib().vlo_sim_t(self.ptr)

    @property
    def outflow_target(self):
        raise AttributeError("write-only in the oracle wrapper")

    @outflow_target.setter
    def outflow_target(self, v):
        lib().vlo_sim_set_outflow_target(self.ptr, 0 if v is None else 1, 0.0 if v is None else v)

    @property
    def outlet_density_offset(self):
        return lib().vlo_sim_outlet_density_offset(self.ptr)

    @property
    def force(self):
        g = lib().vlo_sim_ngroups(self.ptr)
        out = np.zeros(2 * g)
        if g:
            lib().vlo_sim_force(self.ptr, _dp(out))
        return out.reshape(g, 2)

    def fluid_nodes(self):
        return lib().vlo_sim_fluid_nodes(self.ptr)

    def link_count(self):
        return lib().vlo_sim_link_count(self.ptr)

    def bnode_count(self):
        return lib().vlo_sim_bnode_count(self.ptr)

    def pnode_count(self):
        return lib().vlo_sim_pnode_count(self.ptr)

    def threads(self):
        return lib().vlo_sim_threads(self.ptr)

    def set_threads(self, threads):
        """Runs later steps on a pool of ``threads`` workers (results do not depend on it)."""
        lib().vlo_sim_set_threads(self.ptr, threads)

    def flags(self):
        out = np.zeros(self.n, dtype=np.uint8)
        lib().vlo_sim_flags(self.ptr, out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out.reshape(self.ny, self.nx)

    def init(self, field):
        """field: callable (x, y) -> (rho, ux, uy), or a tuple of three (ny, nx) arrays."""
        if callable(field):
            rho = np.empty((self.ny, self.nx)); ux = np.empty_like(rho); uy = np.empty_like(rho)
            for y in range(self.ny):
                for x in range(self.nx):
                    rho[y, x], ux[y, x], uy[y, x] = field(x, y)
        else:
            rho, ux, uy = (np.broadcast_to(np.asarray(a, dtype=np.float64), (self.ny, self.nx)) for a in field)
        rho, ux, uy = _arr(rho).reshape(-1), _arr(ux).reshape(-1), _arr(uy).reshape(-1)
        lib().vlo_sim_init_arrays(self.ptr, _dp(rho), _dp(ux), _dp(uy))

    def step(self, n=1):
        lib().vlo_sim_step(self.ptr, n)

    def populations(self):
        out = np.zeros(9 * self.n)
        lib().vlo_sim_get_f(self.ptr, _dp(out))
        return out.reshape(9, self.ny, self.nx)

    def set_populations(self, f):
        f = _arr(f).reshape(-1)
        assert f.size == 9 * self.n
        lib().vlo_sim_set_f(self.ptr, _dp(f))

    def macros(self, x, y):
        out = np.zeros(3)
        lib().vlo_sim_macros(self.ptr, x, y, _dp(out))
        return tuple(out)

    def total_mass(self):
        return lib().vlo_sim_total_mass(self.ptr)

    def total_momentum(self):
        out = np.zeros(2)
        lib().vlo_sim_total_momentum(self.ptr, _dp(out))
        return tuple(out)

    def max_speed(self):
        return lib().vlo_sim_max_speed(self.ptr)

    def vorticity(self):
        out = np.zeros(self.n, dtype=np.float32)
        lib().vlo_sim_vorticity(self.ptr, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out.reshape(self.ny, self.nx)

    def probe_density(self, x, y):
        return lib().vlo_sim_probe_density(self.ptr, x, y)

    def probe_density_at_wall(self, x, y, nx, ny):
        return lib().vlo_sim_probe_density_at_wall(self.ptr, x, y, nx, ny)

    def state_hash(self):
        return lib().vlo_sim_state_hash(self.ptr)

    def link_table(self):
        nb, nl = self.bnode_count(), self.link_count()
        bidx = np.zeros(nb, dtype=np.int32)
        bfirst = np.zeros(nb + 1, dtype=np.int32)
        lf = np.zeros(5 * max(nl, 1))
        li = np.zeros(7 * max(nl, 1), dtype=np.int32)
        P32 = C.POINTER(C.c_int32)
        lib().vlo_sim_link_table(self.ptr, bidx.ctypes.data_as(P32), bfirst.ctypes.data_as(P32), _dp(lf),
                                 li.ctypes.data_as(P32))
        return dict(flags=self.flags(), bnode_idx=bidx, bnode_first=bfirst, link_f64=lf[:5 * nl].reshape(-1, 5),
                    link_i32=li[:7 * nl].reshape(-1, 7), npnodes=self.pnode_count())


# ------------------------------------------------------------------ cases
class Channel:
    """src/cases/channel.rs:60-137. `body` is a Shape (ownership taken)."""

    def __init__(self, nx, ny, inflow, u, nu, collision, body, ramp_steps, kick=None, threads=1, magic=3.0 / 16.0):
        k = None
        if kick is not None:
            k = _arr(kick)
        self.ptr = lib().vlo_channel_new(nx, ny, inflow, u, nu, collision, magic, body.take(), ramp_steps,
                                         _dp(k) if k is not None else None, threads)
        if not self.ptr:
            raise _err()
        self.sim = Sim(lib().vlo_channel_sim(self.ptr), owned=False)
        self.u_ref = lib().vlo_channel_u_ref(self.ptr)

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().vlo_channel_free(self.ptr)

    def set_absorbing_outlet(self, on):
        lib().vlo_channel_set_absorbing(self.ptr, int(on))

    def run(self, steps, record_force=True, dp_probe=None):
        """Runs `steps` Channel::step calls. Returns (force history (steps, 2) | None, dp | None).

        dp_probe = (xc, yc, r) records the cylinder pressure drop (src/cases/cylinder.rs:54-59).
        """
        fh = np.zeros((steps, 2)) if record_force else None
        dp = np.zeros(steps) if dp_probe is not None else None
        xc, yc, r = dp_probe if dp_probe is not None else (0.0, 0.0, 0.0)
        lib().vlo_channel_run(self.ptr, steps, _dp(fh) if fh is not None else None,
                              _dp(dp) if dp is not None else None, xc, yc, r)
        return fh, dp

    def step(self):
        self.run(1, record_force=False)

    def coefficients(self, d):
        k = 2.0 / (self.u_ref * self.u_ref * d)
        f = self.sim.force
        return k * f[0, 0], k * f[0, 1]


def cylinder_rig(n, u_mean=0.05, re=100.0, collision=TRT, ramp_units=8.0, threads=1):
    """src/cases/cylinder.rs:35-50. Returns (channel, n, xc, yc)."""
    nf = float(n)
    xc = yc = 0.5 + 2.0 * nf
    nu = u_mean * nf / re
    ch = Channel(22 * n + 2, 41 * n // 10 + 2, PARABOLIC, u_mean, nu, collision, Shape.circle(xc, yc, 0.5 * nf),
                 int(ramp_units * nf / u_mean), None, threads)
    return ch, nf, xc, yc


# ------------------------------------------------------------------ signal
def fft(re, im):
    re, im = _arr(re).copy(), _arr(im).copy()
    lib().vlo_fft(_dp(re), _dp(im), len(re))
    return re, im


def mean(x):
    x = _arr(x)
    return lib().vlo_mean(_dp(x), len(x))


def rms(x):
    x = _arr(x)
    return lib().vlo_rms(_dp(x), len(x))


def dominant_frequency(x, dt):
    x = _arr(x)
    out = np.zeros(2)
    lib().vlo_dominant_frequency(_dp(x), len(x), dt, _dp(out))
    return tuple(out)


def peaks(x):
    x = _arr(x)
    cap = len(x)
    pos, val = np.zeros(max(cap, 1)), np.zeros(max(cap, 1))
    k = lib().vlo_peaks(_dp(x), len(x), _dp(pos), _dp(val), cap)
    return list(zip(pos[:k], val[:k]))


def crossing_frequency(x, dt):
    x = _arr(x)
    out = np.zeros(1)
    return out[0] if lib().vlo_crossing_frequency(_dp(x), len(x), dt, _dp(out)) else None


def sample_at(x, pos):
    x = _arr(x)
    return lib().vlo_sample_at(_dp(x), len(x), pos)
