"""Many tunnels at once (include/vortexlab.h, vl_batch_*), and the seeded population of tunnels
used to exercise it.

``Batch`` packs channels of uneven sizes, shapes and Reynolds numbers into one device arena and
advances them together, each for its own number of steps; every tunnel follows Channel::step
(src/cases/channel.rs:118-130) exactly, so a tunnel in a batch is bit-identical to the same tunnel
run alone (FP64: the reference's operation order; the narrow formats: the explicitly rounded FP32
collision that every narrow kernel shares).
``seeded_tunnels`` draws the bodies and flow parameters of the batched workload.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import PRECISIONS, Ellipse, Polygon, Rotated, Spec, Star, _lib
from ._lib import check, lib, nonnull
from .tunnel import Tunnel
from .workloads import XorShift64Star


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Batch:
    SCHEDULES = {"concurrent": 0, "links-first": 1, "bulk-first": 2, "staged": 3}
    TILES = {(8, 1): "256x1", (7, 2): "128x2", (6, 4): "64x4", (5, 8): "32x8", (5, 0): "packed"}

    def __init__(self, precision="f32"):
        self.precision = precision
        self._h = nonnull(lib.vl_batch_new(PRECISIONS[precision] if isinstance(precision, str) else precision))
        self.count = 0
        self.built = False

    def __del__(self):
        if getattr(self, "_h", None):
            lib.vl_batch_free(self._h)
            self._h = None

    def close(self):
        self.__del__()

    def add(self, spec: Spec, steps: int) -> int:
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
        k = check(lib.vl_batch_add_channel(self._h, C.byref(s), steps))
        self.count += 1
        return k

    def build(self):
        check(lib.vl_batch_build(self._h))
        self.built = True

    def info(self, k):
        nx, ny, fl, st = C.c_size_t(), C.c_size_t(), C.c_size_t(), C.c_uint64()
        check(lib.vl_batch_tunnel_info(self._h, k, C.byref(nx), C.byref(ny), C.byref(fl), C.byref(st)))
        return dict(nx=nx.value, ny=ny.value, fluid_nodes=fl.value, steps=st.value)

    @property
    def tile(self) -> str:
        a, b = C.c_int(), C.c_int()
        check(lib.vl_batch_get_tile(self._h, C.byref(a), C.byref(b)))
        return self.TILES[(a.value, b.value)]

    @tile.setter
    def tile(self, name: str):
        inv = {v: k for k, v in self.TILES.items()}
        check(lib.vl_batch_set_tile(self._h, *inv[name]))

    @property
    def schedule(self):
        raise AttributeError("write-only")

    @schedule.setter
    def schedule(self, name):
        check(lib.vl_batch_set_schedule(self._h, self.SCHEDULES[name]))

    def set_cells_per_thread(self, cells: int):
        """FP32 / 16-bit storage: 2 (default where every row length is even) bulk cells per thread, or 1."""
        check(lib.vl_batch_set_cells_per_thread(self._h, cells))

    def set_prefetch_tiles(self, tiles: int):
        """Bulk blocks prefetch into the L2 the tile `tiles` places ahead in the list (0: off)."""
        check(lib.vl_batch_set_prefetch_tiles(self._h, tiles))

    def autotune(self, steps_each=4):
        """Times the four row tile shapes and the packed layout without advancing the tunnels;
        keeps the fastest."""
        out = np.zeros(len(self.TILES))
        check(lib.vl_batch_autotune_layouts(self._h, steps_each, _dp(out), len(out)))
        return dict(zip(self.TILES.values(), out.tolist()))

    def run(self, max_steps: int = 0):
        check(lib.vl_batch_run(self._h, max_steps))

    def run_async(self, max_steps: int = 0):
        """Enqueues the steps of `run` without waiting for them (`wait` does)."""
        check(lib.vl_batch_run_async(self._h, max_steps))

    def wait(self):
        check(lib.vl_batch_wait(self._h))

    def hold(self, k):
        """Keeps tunnel k at its start state, taking no steps, until `start(k)` (before the first step)."""
        check(lib.vl_batch_hold(self._h, k))

    def start(self, k) -> int:
        """Starts held tunnel k at the next global step after the enqueued ones; returns that step."""
        out = C.c_uint64()
        check(lib.vl_batch_start(self._h, k, C.byref(out)))
        return out.value

    def history_copy(self, ranges):
        """Force records of several tunnels at once: `ranges` is a list of (k, first, count) with
        every step complete at the last `wait`; returns one (count, 2) array per range. Does not
        wait for a run in flight."""
        n = len(ranges)
        ks = (C.c_int * max(n, 1))(*[r[0] for r in ranges])
        firsts = (C.c_uint64 * max(n, 1))(*[r[1] for r in ranges])
        counts = (C.c_uint64 * max(n, 1))(*[r[2] for r in ranges])
        out = np.empty((max(sum(r[2] for r in ranges), 1), 2))
        check(lib.vl_batch_history_copy(self._h, n, ks, firsts, counts, _dp(out)))
        res, at = [], 0
        for r in ranges:
            res.append(out[at:at + r[2]])
            at += r[2]
        return res

    def last_run_ms(self) -> float:
        out = C.c_float()
        check(lib.vl_batch_last_run_ms(self._h, C.byref(out)))
        return out.value

    def global_step(self) -> int:
        out = C.c_uint64()
        check(lib.vl_batch_global_step(self._h, C.byref(out)))
        return out.value

    def launch_count(self) -> int:
        out = C.c_uint64()
        check(lib.vl_batch_launch_count(self._h, C.byref(out)))
        return out.value

    def status(self, k):
        t, nf, f = C.c_uint64(), C.c_int(), np.zeros(2)
        check(lib.vl_batch_status(self._h, k, C.byref(t), C.byref(nf), _dp(f)))
        return t.value, bool(nf.value), f

    def force_history(self, k) -> np.ndarray:
        cnt = C.c_uint64()
        check(lib.vl_batch_force_history(self._h, k, None, C.byref(cnt)))
        out = np.zeros(2 * max(cnt.value, 1))
        check(lib.vl_batch_force_history(self._h, k, _dp(out), C.byref(cnt)))
        return out[: 2 * cnt.value].reshape(cnt.value, 2)

    def force_history_range(self, k, first: int, max_count: int) -> np.ndarray:
        """Force records of steps [first, first + max_count) that tunnel k has run so far."""
        cnt = C.c_uint64()
        out = np.zeros(2 * max(int(max_count), 1))
        check(lib.vl_batch_force_history_range(self._h, k, int(first), int(max_count), _dp(out), C.byref(cnt)))
        return out[: 2 * cnt.value].reshape(cnt.value, 2)

    def populations(self, k) -> np.ndarray:
        i = self.info(k)
        out = np.zeros(9 * i["nx"] * i["ny"])
        check(lib.vl_batch_download(self._h, k, _dp(out)))
        return out.reshape(9, i["ny"], i["nx"])

    def set_steps(self, k, steps: int):
        """Ends tunnel k after `steps` steps (at most the count it was added with, not before the
        current global step)."""
        check(lib.vl_batch_set_steps(self._h, k, int(steps)))

    def macros_field(self, k):
        """(rho, ux, uy), each (ny, nx), of tunnel k at its current step."""
        i = self.info(k)
        n = i["nx"] * i["ny"]
        rho, ux, uy = np.zeros(n), np.zeros(n), np.zeros(n)
        check(lib.vl_batch_macros_field(self._h, k, _dp(rho), _dp(ux), _dp(uy)))
        return tuple(a.reshape(i["ny"], i["nx"]) for a in (rho, ux, uy))

    def init(self, k, rho, ux, uy):
        """Sim::init of tunnel k from (ny, nx) fields, before the batch's first step."""
        i = self.info(k)
        shape = (i["ny"], i["nx"])
        arrs = [np.ascontiguousarray(np.broadcast_to(np.asarray(a, np.float64), shape)).reshape(-1)
                for a in (rho, ux, uy)]
        check(lib.vl_batch_init(self._h, k, *(_dp(a) for a in arrs)))

    def flags(self, k) -> np.ndarray:
        i = self.info(k)
        out = np.zeros(i["nx"] * i["ny"], dtype=np.uint8)
        check(lib.vl_batch_flags(self._h, k, out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out.reshape(i["ny"], i["nx"])

    def state_hash(self, k) -> int:
        out = C.c_uint64()
        check(lib.vl_batch_state_hash(self._h, k, C.byref(out)))
        return out.value


# ---------------------------------------------------------------------------- seeded tunnels
@dataclass
class TunnelCase:
    tunnel: Tunnel
    body: object
    kind: str
    params: dict

    @property
    def steps(self) -> int:
        return int(self.units * self.tunnel.steps_per_unit())

    units: float = 40.0


def _notched_square(cx, cy, d, notches, depth):
    """Square of side d centred at (cx, cy), counter-clockwise from the top-right corner, with a
    square notch of side depth * d cut from each of the first `notches` corners. At a notched
    corner the outline steps back along the edge it arrives on, in by the notch depth, and out
    along the edge it leaves on."""
    h, b = 0.5 * d, depth * d
    pts = []
    for k, (x, y) in enumerate([(h, h), (-h, h), (-h, -h), (h, -h)]):
        if k >= notches:
            pts.append((x, y))
            continue
        sx, sy = math.copysign(b, x), math.copysign(b, y)
        inner = (x - sx, y - sy)
        if k % 2 == 0:  # arriving on a vertical edge, leaving on a horizontal one
            pts += [(x, y - sy), inner, (x - sx, y)]
        else:           # arriving on a horizontal edge, leaving on a vertical one
            pts += [(x - sx, y), inner, (x, y - sy)]
    return [(cx + x, cy + y) for x, y in pts]


def seeded_tunnels(seed=0x5EED0004, count=256, dmin=15, dmax=60, re=(50.0, 200.0), u=0.05, units=40.0,
                   precision="f32"):
    """Tunnels 20 D long (5 D upstream, 15 D downstream of the body centre) and 10 D high with
    sound-absorbing sides; bodies uniform over three classes: ellipses of aspect 1-4, squares with
    0-2 notched corners (notch depth 5-15 % of the side), star-convex polygons of 6-12 vertices;
    all rotated by 0-30 degrees; D uniform in [dmin, dmax], Re uniform in `re`."""
    rng = XorShift64Star(seed)
    out = []
    for _ in range(count):
        d = int(round(dmin + (dmax - dmin) * rng.next()))
        r = re[0] + (re[1] - re[0]) * rng.next()
        angle = math.radians(30.0 * rng.next())
        cls = min(int(3 * rng.next()), 2)
        tn = Tunnel(d=d, re=r, u=u, upstream=5.0, downstream=15.0, height=10.0, precision=precision)
        cx, cy = tn.centre()
        if cls == 0:
            aspect = 1.0 + 3.0 * rng.next()
            body = Ellipse(cx, cy, 0.5 * d * aspect, 0.5 * d)
            params = dict(aspect=aspect)
            kind = "ellipse"
        elif cls == 1:
            notches = min(int(3 * rng.next()), 2)
            depth = 0.05 + 0.10 * rng.next()
            body = Polygon(_notched_square(cx, cy, float(d), notches, depth))
            params = dict(notches=notches, depth=depth)
            kind = "square"
        else:
            m = 6 + min(int(7 * rng.next()), 6)
            radii = [0.5 * d * (0.6 + 0.4 * rng.next()) for _ in range(m)]
            body = Star(cx, cy, radii, 2.0 * math.pi * rng.next())
            params = dict(vertices=m)
            kind = "star"
        if angle != 0.0:
            body = Rotated(body, cx, cy, angle)
        params.update(d=d, re=r, angle_deg=math.degrees(angle))
        out.append(TunnelCase(tn, body, kind, params, units))
    return out
