"""vortexlab-b200: the vortexlab D2Q9 lattice-Boltzmann time step on one B200.

The Python surface mirrors the reference's Rust API so that code written against it ports line by
line: ``Builder`` (src/sim.rs:70-137), ``Sim`` (src/sim.rs:180-673), ``Kind`` / ``Wall``
(src/sim.rs:38-63), ``Collision`` (src/lattice.rs:28-45), the shapes of src/geometry.rs,
``Channel`` / ``Spec`` / ``Inflow`` / ``Kick`` (src/cases/channel.rs), ``cylinder`` and ``Tunnel``
(src/cases/cylinder.rs, src/cases/tunnel.rs) and the signal analysis of src/signal.rs.

Everything here is a thin ctypes layer over the C ABI in include/vortexlab.h; the time step runs
in hand-written sm_100a CUDA kernels on the device that is current when a sim is built. There is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import VortexError, check, lib, nonnull

__all__ = [
    "VortexError", "Collision", "Velocity", "Wall", "Kind", "FLUID", "Builder", "Sim",
    "Circle", "Polygon", "RoundedSquare", "Rotated", "Translated", "Bitmap", "OutsideBand", "Ellipse",
    "Star", "Disks", "Corner", "section", "cut_fraction", "Inflow", "Kick", "Spec", "Channel",
    "Series", "Stats", "cylinder", "Tunnel", "signal", "ramp", "tau_for", "viscosity", "PRECISIONS",
    "device_count",
]

FLUID = 0
PRECISIONS = {"f64": 0, "f32": 1, "f16s": 2, "f16c": 3, "f16x": 4}
CS2 = 1.0 / 3.0


def device_count() -> int:
    return lib.vl_device_count()


def set_device(device: int):
    """Makes ``device`` current for sims built afterwards on this thread."""
    check(lib.vl_set_device(device))


class PinnedArray:
    """A float64 numpy array in page-locked host memory (freed with the object)."""

    def __init__(self, n: int):
        self._p = nonnull(lib.vl_pinned_alloc(8 * max(n, 1)))
        buf = (C.c_double * max(n, 1)).from_address(self._p)
        self.array = np.frombuffer(buf, dtype=np.float64, count=n)

    def __del__(self):
        if getattr(self, "_p", None):
            self.array = None
            lib.vl_pinned_free(self._p)
            self._p = None


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _arr(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def _prec(p):
    if isinstance(p, int):
        return p
    try:
        return PRECISIONS[p]
    except KeyError:
        raise ValueError(f"precision must be one of {list(PRECISIONS)}") from None


# ====================================================================== lattice
class Collision:
    """src/lattice.rs:28-45: ``Collision.Bgk`` or ``Collision.Trt(magic)``."""

    def __init__(self, kind: int, magic: float = 3.0 / 16.0):
        self.kind = kind
        self.magic = magic

    @staticmethod
    def Trt(magic: float = 3.0 / 16.0) -> "Collision":
        return Collision(1, magic)

    def omegas(self, tau: float):
        if self.kind == 0:
            return 1.0 / tau, 1.0 / tau
        return 1.0 / tau, 1.0 / (0.5 + self.magic / (tau - 0.5))

    def __eq__(self, other):
        return isinstance(other, Collision) and other.kind == self.kind and (self.kind == 0 or other.magic == self.magic)

    def __repr__(self):
        return "Bgk" if self.kind == 0 else f"Trt {{ magic: {self.magic} }}"


Collision.Bgk = Collision(0)
TRT = Collision.Trt(3.0 / 16.0)


def tau_for(nu: float) -> float:
    """src/lattice.rs:53-55."""
    return lib.vl_tau_for(nu)


def viscosity(tau: float) -> float:
    """src/lattice.rs:48-50."""
    return (tau - 0.5) * CS2


def ramp(t: int, steps: int) -> float:
    """src/cases/mod.rs:11-18."""
    return lib.vl_ramp(t, steps)


# ====================================================================== shapes
class Shape:
    """A shape description; ``_make()`` builds a fresh native handle (ownership passes on use)."""

    def _make(self):
        raise NotImplementedError

    def inside(self, x: float, y: float) -> bool:
        h = self._make()
        try:
            return bool(lib.vl_shape_inside(h, x, y))
        finally:
            lib.vl_shape_free(h)


@dataclass
class Circle(Shape):
    cx: float
    cy: float
    r: float

    def _make(self):
        return nonnull(lib.vl_shape_circle(self.cx, self.cy, self.r))


@dataclass
class Polygon(Shape):
    pts: Sequence[Sequence[float]]

    def _make(self):
        xy = _arr(self.pts).reshape(-1)
        return nonnull(lib.vl_shape_polygon(_dp(xy), len(xy) // 2))


@dataclass
class RoundedSquare(Shape):
    cx: float
    cy: float
    half: float
    r: float

    def _make(self):
        return nonnull(lib.vl_shape_rounded_square(self.cx, self.cy, self.half, self.r))


@dataclass
class Rotated(Shape):
    inner: Shape
    cx: float
    cy: float
    angle: float

    def _make(self):
        return nonnull(lib.vl_shape_rotated(self.inner._make(), self.cx, self.cy, self.angle))


@dataclass
class Translated(Shape):
    inner: Shape
    dx: float
    dy: float

    def _make(self):
        return nonnull(lib.vl_shape_translated(self.inner._make(), self.dx, self.dy))


@dataclass
class OutsideBand(Shape):
    y0: float
    y1: float

    def _make(self):
        return nonnull(lib.vl_shape_outside_band(self.y0, self.y1))


@dataclass
class Ellipse(Shape):
    cx: float
    cy: float
    a: float
    b: float

    def _make(self):
        return nonnull(lib.vl_shape_ellipse(self.cx, self.cy, self.a, self.b))


@dataclass
class Star(Shape):
    cx: float
    cy: float
    radii: Sequence[float]
    phase: float = 0.0

    def _make(self):
        r = _arr(self.radii)
        return nonnull(lib.vl_shape_star(self.cx, self.cy, _dp(r), len(r), self.phase))


@dataclass
class Disks(Shape):
    """Union of disks; ``disks`` is an (n, 3) array of (cx, cy, r)."""

    disks: np.ndarray

    def _make(self):
        d = _arr(self.disks).reshape(-1)
        return nonnull(lib.vl_shape_disks(_dp(d), len(d) // 3))


@dataclass
class Bitmap(Shape):
    level: np.ndarray  # (h, w), row 0 at the top
    x0: float
    y0: float
    scale: float

    def _make(self):
        lv = np.ascontiguousarray(self.level, dtype=np.float32)
        h, w = lv.shape
        return nonnull(lib.vl_shape_bitmap(w, h, lv.ctypes.data_as(C.POINTER(C.c_float)), self.x0, self.y0, self.scale))


class Corner:
    """src/geometry.rs:188-201 (``Corner::Chamfered(b)`` etc. as ``(kind, b)`` tuples)."""

    Sharp = (0, 0.0)

    @staticmethod
    def Chamfered(b):
        return (1, b)

    @staticmethod
    def Rounded(b):
        return (2, b)

    @staticmethod
    def Recessed(b):
        return (3, b)

    @staticmethod
    def DoubleRecessed(b):
        return (4, b)


@dataclass
class _Section(Shape):
    corner: tuple
    cx: float
    cy: float
    d: float
    angle: float

    def _make(self):
        return nonnull(lib.vl_shape_section(self.corner[0], self.corner[1], self.cx, self.cy, self.d, self.angle))


def section(corner, cx, cy, d, angle=0.0) -> Shape:
    """src/geometry.rs:251-261."""
    return _Section(corner, cx, cy, d, angle)


def cut_fraction(shape: Shape, x, y, dx, dy) -> float:
    """src/geometry.rs:268-279."""
    h = shape._make()
    try:
        return lib.vl_cut_fraction(h, x, y, dx, dy)
    finally:
        lib.vl_shape_free(h)


def bounding_box(shape: Shape, reach, step):
    """src/geometry.rs:99-115."""
    h = shape._make()
    out = np.zeros(4)
    try:
        return tuple(out) if check(lib.vl_bounding_box(h, reach, step, _dp(out))) else None
    finally:
        lib.vl_shape_free(h)


# ====================================================================== kinds / builder
class Velocity:
    """Wall velocity as tagged data (replaces the closure of src/sim.rs:34)."""

    @staticmethod
    def const(ux, uy):
        return (1, (ux, uy, 0.0, 0.0))

    @staticmethod
    def parabolic(u_mean, h):
        return (2, (u_mean, h, 0.0, 0.0))

    @staticmethod
    def rotation(cx, cy):
        return (3, (cx, cy, 0.0, 0.0))


@dataclass
class Wall:
    """src/sim.rs:38-49."""

    velocity: Optional[tuple] = None
    vgroup: int = 0
    fgroup: Optional[int] = None
    shape: Optional[Shape] = None


class Kind:
    """src/sim.rs:52-63."""

    def __init__(self, tag, payload=None):
        self.tag = tag
        self.payload = payload

    @staticmethod
    def Wall(w: Wall):
        return Kind("wall", w)

    @staticmethod
    def Pressure(rho: float):
        return Kind("pressure", rho)

    @staticmethod
    def Radiating(rho: float):
        return Kind("radiating", rho)


class Builder:
    """src/sim.rs:70-137. Scalar attributes are applied when ``build`` is called."""

    def __init__(self, nx: int, ny: int):
        self._h = nonnull(lib.vl_builder_new(nx, ny))
        self.nx, self.ny = nx, ny
        self.periodic_x = False
        self.periodic_y = False
        self.tau = 1.0
        self.collision = TRT
        self.accel = (0.0, 0.0)

    def __del__(self):
        if getattr(self, "_h", None):
            lib.vl_builder_free(self._h)

    def add(self, kind: Kind) -> int:
        if kind.tag == "wall":
            w: Wall = kind.payload
            s = _lib.vl_wall()
            if w.velocity is not None:
                s.velocity.kind = w.velocity[0]
                for i, v in enumerate(w.velocity[1]):
                    s.velocity.p[i] = v
            s.vgroup = w.vgroup
            s.fgroup = -1 if w.fgroup is None else w.fgroup
            s.shape = w.shape._make() if w.shape is not None else None
            return check(lib.vl_builder_add_wall(self._h, C.byref(s)))
        if kind.tag == "pressure":
            return check(lib.vl_builder_add_pressure(self._h, kind.payload))
        if kind.tag == "radiating":
            return check(lib.vl_builder_add_radiating(self._h, kind.payload))
        raise ValueError("unknown kind")

    def add_static_wall(self) -> int:
        return check(lib.vl_builder_add_static_wall(self._h))

    def fill_rect(self, x0, x1, y0, y1, kind):
        check(lib.vl_builder_fill_rect(self._h, x0, x1, y0, y1, kind))

    def fill_shape(self, kind):
        check(lib.vl_builder_fill_shape(self._h, kind))

    def _apply(self):
        check(lib.vl_builder_set_periodic(self._h, int(self.periodic_x), int(self.periodic_y)))
        check(lib.vl_builder_set_tau(self._h, self.tau))
        check(lib.vl_builder_set_collision(self._h, self.collision.kind, self.collision.magic))
        check(lib.vl_builder_set_accel(self._h, self.accel[0], self.accel[1]))

    def link_table(self):
        """Host-side link tables (no GPU needed): dict of numpy arrays."""
        self._apply()
        nl, nb, npn = C.c_size_t(), C.c_size_t(), C.c_size_t()
        check(lib.vl_builder_link_table(self._h, C.byref(nl), C.byref(nb), C.byref(npn), None, None, None, None, None))
        flags = np.zeros(self.nx * self.ny, dtype=np.uint8)
        bidx = np.zeros(nb.value, dtype=np.int32)
        bfirst = np.zeros(nb.value + 1, dtype=np.int32)
        lf = np.zeros(5 * nl.value)
        li = np.zeros(7 * nl.value, dtype=np.int32)
        P8, P32 = C.POINTER(C.c_uint8), C.POINTER(C.c_int32)
        check(lib.vl_builder_link_table(self._h, C.byref(nl), C.byref(nb), C.byref(npn), flags.ctypes.data_as(P8),
                                        bidx.ctypes.data_as(P32), bfirst.ctypes.data_as(P32), _dp(lf),
                                        li.ctypes.data_as(P32)))
        return dict(flags=flags.reshape(self.ny, self.nx), bnode_idx=bidx, bnode_first=bfirst,
                    link_f64=lf.reshape(-1, 5), link_i32=li.reshape(-1, 7), npnodes=npn.value)

    def stage_split(self):
        """How the staged step splits its work on these tables (host only): dict with
        links_per_block, link_blocks, split_blocks (0: not split) and split_rows."""
        self._apply()
        v = [C.c_int() for _ in range(4)]
        check(lib.vl_builder_stage_split(self._h, *(C.byref(x) for x in v)))
        return dict(zip(("links_per_block", "link_blocks", "split_blocks", "split_rows"), (x.value for x in v)))

    def build(self, threads: Optional[int] = None, precision="f64") -> "Sim":
        """Builder::build (src/sim.rs:134-136). ``threads`` is accepted for API compatibility: the
        reference's thread pool (src/pool.rs) is replaced by one CUDA stream."""
        self._apply()
        h, self._h = self._h, None
        return Sim(nonnull(lib.vl_builder_build(h, _prec(precision))), owned=True)


# ====================================================================== sim
class _VScale:
    def __init__(self, sim):
        self._sim = sim

    def __getitem__(self, g):
        out = np.zeros(4)
        check(lib.vl_sim_get_vscale(self._sim._h, _dp(out)))
        return out[g]

    def __setitem__(self, g, v):
        check(lib.vl_sim_set_vscale(self._sim._h, g, float(v)))

    def __iter__(self):
        out = np.zeros(4)
        check(lib.vl_sim_get_vscale(self._sim._h, _dp(out)))
        return iter(out.tolist())


class Sim:
    """src/sim.rs:180-673, device resident."""

    def __init__(self, handle, owned=True):
        self._h = handle
        self._owned = owned
        nx, ny, fl, nl, nb = (C.c_size_t() for _ in range(5))
        ng, pr = C.c_int(), C.c_int()
        check(lib.vl_sim_info(handle, C.byref(nx), C.byref(ny), C.byref(fl), C.byref(nl), C.byref(nb), C.byref(ng),
                              C.byref(pr)))
        self.nx, self.ny = nx.value, ny.value
        self.n = self.nx * self.ny
        self._fluid, self._links, self._bnodes = fl.value, nl.value, nb.value
        self.ngroups = ng.value
        self.precision = pr.value
        self._target = None
        self._flags = None

    def __del__(self):
        if getattr(self, "_owned", False) and self._h:
            lib.vl_sim_free(self._h)
            self._h = None

    def close(self):
        self.__del__()

    # ---- pub fields
    @property
    def vscale(self):
        return _VScale(self)

    @property
    def force(self) -> np.ndarray:
        out = np.zeros(2 * max(self.ngroups, 1))
        check(lib.vl_sim_force(self._h, _dp(out)))
        return out[: 2 * self.ngroups].reshape(self.ngroups, 2)

    @property
    def outflow_target(self):
        return self._target

    @outflow_target.setter
    def outflow_target(self, v):
        self._target = v
        check(lib.vl_sim_set_outflow_target(self._h, 0 if v is None else 1, 0.0 if v is None else float(v)))

    @property
    def outlet_density_offset(self) -> float:
        out = C.c_double()
        check(lib.vl_sim_outlet_density_offset(self._h, C.byref(out)))
        return out.value

    @property
    def t(self) -> int:
        out = C.c_uint64()
        check(lib.vl_sim_t(self._h, C.byref(out)))
        return out.value

    # ---- accessors
    def fluid_nodes(self) -> int:
        return self._fluid

    def link_count(self) -> int:
        return self._links

    def bnode_count(self) -> int:
        return self._bnodes

    def flags(self) -> np.ndarray:
        if self._flags is None:
            f = np.zeros(self.n, dtype=np.uint8)
            check(lib.vl_sim_flags(self._h, f.ctypes.data_as(C.POINTER(C.c_uint8))))
            self._flags = f.reshape(self.ny, self.nx)
        return self._flags

    def is_fluid(self, x, y) -> bool:
        return bool(self.flags()[y, x] != 2)

    # ---- state
    def init(self, field):
        """Sim::init (src/sim.rs:357-371). ``field``: callable (x, y) -> (rho, ux, uy), a tuple of
        three (ny, nx) arrays, or a tuple of three scalars (uniform)."""
        if callable(field):
            rho = np.empty((self.ny, self.nx)); ux = np.empty_like(rho); uy = np.empty_like(rho)
            for y in range(self.ny):
                for x in range(self.nx):
                    rho[y, x], ux[y, x], uy[y, x] = field(x, y)
            field = (rho, ux, uy)
        if all(np.ndim(a) == 0 for a in field):
            check(lib.vl_sim_init(self._h, None, None, None, float(field[0]), float(field[1]), float(field[2])))
            return
        rho, ux, uy = (_arr(np.broadcast_to(np.asarray(a, dtype=np.float64), (self.ny, self.nx))).reshape(-1)
                       for a in field)
        check(lib.vl_sim_init(self._h, _dp(rho), _dp(ux), _dp(uy), 1.0, 0.0, 0.0))

    def step(self, n: int = 1):
        """Sim::step (src/sim.rs:391-420), ``n`` times, queued on the sim's stream."""
        check(lib.vl_sim_step(self._h, n))

    def synchronize(self):
        check(lib.vl_sim_synchronize(self._h))

    def populations(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """All populations as FP64 in the reference layout, shape (9, ny, nx). ``out`` may be a
        preallocated contiguous float64 buffer of 9 * nx * ny values (for example pinned memory)."""
        if out is None:
            out = np.zeros(9 * self.n)
        elif out.dtype != np.float64 or out.size != 9 * self.n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of 9 * nx * ny values")
        check(lib.vl_sim_download(self._h, _dp(out)))
        return out.reshape(9, self.ny, self.nx)

    def set_populations(self, f):
        f = _arr(f).reshape(-1)
        if f.size != 9 * self.n:
            raise ValueError("need 9 * nx * ny populations")
        check(lib.vl_sim_upload(self._h, _dp(f)))

    def macros(self, x, y):
        out = np.zeros(3)
        check(lib.vl_sim_macros(self._h, x, y, _dp(out)))
        return tuple(out)

    def macros_field(self):
        rho, ux, uy = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        check(lib.vl_sim_macros_field(self._h, _dp(rho), _dp(ux), _dp(uy)))
        return rho.reshape(self.ny, self.nx), ux.reshape(self.ny, self.nx), uy.reshape(self.ny, self.nx)

    def total_mass(self) -> float:
        out = C.c_double()
        check(lib.vl_sim_total_mass(self._h, C.byref(out)))
        return out.value

    def total_momentum(self):
        out = np.zeros(2)
        check(lib.vl_sim_total_momentum(self._h, _dp(out)))
        return tuple(out)

    def max_speed(self) -> float:
        out = C.c_double()
        check(lib.vl_sim_max_speed(self._h, C.byref(out)))
        return out.value

    def vorticity(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.float32)
        check(lib.vl_sim_vorticity(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out.reshape(self.ny, self.nx)

    def probe_density(self, x, y) -> float:
        out = C.c_double()
        check(lib.vl_sim_probe_density(self._h, x, y, C.byref(out)))
        return out.value

    def probe_density_at_wall(self, x, y, nx, ny) -> float:
        out = C.c_double()
        check(lib.vl_sim_probe_density_at_wall(self._h, x, y, nx, ny, C.byref(out)))
        return out.value

    def state_hash(self) -> int:
        out = C.c_uint64()
        check(lib.vl_sim_state_hash(self._h, C.byref(out)))
        return out.value

    def status(self):
        nf, t = C.c_int(), C.c_uint64()
        check(lib.vl_sim_status(self._h, C.byref(nf), C.byref(t)))
        return bool(nf.value), t.value

    # ---- recording / timing
    def record(self, capacity: int):
        check(lib.vl_sim_record(self._h, capacity))

    def history(self) -> np.ndarray:
        cnt = C.c_uint64()
        check(lib.vl_sim_history(self._h, None, C.byref(cnt)))
        out = np.zeros(max(cnt.value, 1) * _lib.VL_REC)
        check(lib.vl_sim_history(self._h, _dp(out), C.byref(cnt)))
        return out[: cnt.value * _lib.VL_REC].reshape(cnt.value, _lib.VL_REC)

    def set_dp_probe(self, xc, yc, r, u_ref):
        check(lib.vl_sim_set_dp_probe(self._h, xc, yc, r, u_ref))

    def last_step_ms(self) -> float:
        out = C.c_float()
        check(lib.vl_sim_last_step_ms(self._h, C.byref(out)))
        return out.value

    def step_profiled(self, n: int):
        """Runs ``n`` steps with CUDA events around each kernel: (link_ms, bulk_ms, total_ms)."""
        lk, bk, tot = C.c_double(), C.c_double(), C.c_double()
        check(lib.vl_sim_step_profiled(self._h, n, C.byref(lk), C.byref(bk), C.byref(tot)))
        return lk.value, bk.value, tot.value

    SCHEDULES = {"concurrent": 0, "links-first": 1, "bulk-first": 2, "staged": 3}

    @property
    def schedule(self) -> str:
        inv = {v: k for k, v in self.SCHEDULES.items()}
        return inv[check(lib.vl_sim_get_schedule(self._h))]

    @schedule.setter
    def schedule(self, name: str):
        check(lib.vl_sim_set_schedule(self._h, self.SCHEDULES[name]))

    def set_cells_per_thread(self, cells: int):
        """FP32 / 16-bit storage: the most bulk cells per thread (1, 2 or 4; default 2 for FP32, 4
        for the 16-bit formats)."""
        check(lib.vl_sim_set_cells_per_thread(self._h, cells))

    def set_prefetch_rows(self, rows: int):
        """Bulk-kernel blocks ask the L2 for the rows their tile reads `rows` rows later (0: off)."""
        check(lib.vl_sim_set_prefetch_rows(self._h, rows))

    def set_bulk_copies(self, on: bool):
        """FP32 / 16-bit storage: stream the bulk kernel's loads through shared memory (default)."""
        check(lib.vl_sim_set_bulk_copies(self._h, int(bool(on))))

    def autotune(self, steps_each: int = 8):
        """Times the four kernel schedules without advancing the state; keeps the fastest.
        Returns {schedule: ms per step}."""
        out = np.zeros(len(self.SCHEDULES))
        check(lib.vl_sim_autotune(self._h, steps_each, _dp(out)))
        return dict(zip(self.SCHEDULES, out.tolist()))

    def launch_count(self) -> int:
        out = C.c_uint64()
        check(lib.vl_sim_launch_count(self._h, C.byref(out)))
        return out.value


# ====================================================================== channel
class Inflow:
    """src/cases/channel.rs:22-33 as (kind, u) tuples."""

    @staticmethod
    def Parabolic(u_mean):
        return (0, u_mean)

    @staticmethod
    def Uniform(u):
        return (1, u)

    @staticmethod
    def UniformOpen(u):
        return (2, u)


@dataclass
class Kick:
    """src/cases/channel.rs:37-45."""

    cx: float
    cy: float
    omega: float
    start: int
    duration: int


@dataclass
class Spec:
    """src/cases/channel.rs:47-58."""

    nx: int
    ny: int
    inflow: tuple
    nu: float
    collision: Collision
    body: Shape
    ramp_steps: int
    kick: Optional[Kick] = None


class Channel:
    """src/cases/channel.rs:60-137 on the device; per-step controls come from an uploaded schedule."""

    def __init__(self, spec: Spec, threads: Optional[int] = None, precision="f64"):
        s = _lib.vl_channel_spec()
        s.nx, s.ny = spec.nx, spec.ny
        s.inflow, s.u = spec.inflow
        s.nu = spec.nu
        s.collision, s.magic = spec.collision.kind, spec.collision.magic
        s.body = spec.body._make()
        s.ramp_steps = spec.ramp_steps
        if spec.kick is not None:
            k = spec.kick
            s.has_kick = 1
            s.kick_cx, s.kick_cy, s.kick_omega, s.kick_start, s.kick_duration = k.cx, k.cy, k.omega, k.start, k.duration
        self._h = nonnull(lib.vl_channel_new(C.byref(s), _prec(precision)))
        self.sim = Sim(lib.vl_channel_sim(self._h), owned=False)
        self.u_ref = lib.vl_channel_u_ref(self._h)
        self._absorbing = True

    def __del__(self):
        if getattr(self, "_h", None):
            self.sim._h = None
            lib.vl_channel_free(self._h)
            self._h = None

    def close(self):
        self.__del__()

    @property
    def absorbing_outlet(self):
        return self._absorbing

    @absorbing_outlet.setter
    def absorbing_outlet(self, on):
        self._absorbing = bool(on)
        check(lib.vl_channel_set_absorbing(self._h, int(on)))

    def step(self, n: int = 1):
        check(lib.vl_channel_step(self._h, n))

    def coefficients(self, d: float):
        cd, cl = C.c_double(), C.c_double()
        check(lib.vl_channel_coefficients(self._h, d, C.byref(cd), C.byref(cl)))
        return cd.value, cl.value


@dataclass
class Series:
    """src/cases/channel.rs:140-146."""

    dt: float
    cd: np.ndarray
    cl: np.ndarray

    def stats(self, frm: float) -> "Stats":
        """src/cases/channel.rs:164-189."""
        i0 = min(int(frm / self.dt) if frm / self.dt > 0 else 0, max(len(self.cd) - 2, 0))
        cd, cl = self.cd[i0:], self.cl[i0:]
        cl_rms = signal.rms(cl)
        st, st_cross, periodic = 0.0, 0.0, False
        if cl_rms > 1e-6:
            f = signal.dominant_frequency(cl, self.dt)[0]
            st_cross = signal.crossing_frequency(cl, self.dt) or 0.0
            periodic = f * len(cl) * self.dt >= 3.0 and abs(st_cross / f - 1.0) < 0.05
            if periodic:
                st = f
        return Stats(signal.mean(cd), signal.rms(cd), signal.mean(cl), cl_rms, st, st_cross, periodic)


@dataclass
class Stats:
    """src/cases/channel.rs:149-162."""

    cd_mean: float
    cd_rms: float
    cl_mean: float
    cl_rms: float
    st: float
    st_crossings: float
    periodic: bool


from . import cylinder, signal  # noqa: E402
from .tunnel import Tunnel  # noqa: E402
