"""Domain descriptions that build the same sim on the device (vortexlab_b200) and on the oracle.

A description is a plain dict:
  nx, ny, periodic=(px, py), tau, collision ("bgk" | ("trt", magic)), accel=(gx, gy),
  kinds: list of ("wall", velocity, vgroup, fgroup, shape) | ("pressure", rho) | ("radiating", rho)
         velocity: None | ("const", ux, uy) | ("parabolic", u_mean, h) | ("rotation", cx, cy)
         shape: None | ("circle", cx, cy, r) | ("section", corner, b, cx, cy, d, angle)
                | ("disks", array) | ("band", y0, y1) | ("polygon", pts) | ("ellipse", cx, cy, a, b)
  paint: list of ("rect", x0, x1, y0, y1, kind) | ("shape", kind)
Kind ids count from 1 in list order; 0 is fluid.
"""
from __future__ import annotations

import numpy as np

import oracle as O
import vortexlab_b200 as V


def _v_shape(s):
    t = s[0]
    if t == "circle":
        return V.Circle(*s[1:])
    if t == "section":
        corner, b, cx, cy, d, angle = s[1:]
        return V.section((corner, b), cx, cy, d, angle)
    if t == "disks":
        return V.Disks(s[1])
    if t == "band":
        return V.OutsideBand(*s[1:])
    if t == "polygon":
        return V.Polygon(s[1])
    if t == "ellipse":
        return V.Ellipse(*s[1:])
    raise ValueError(t)


def _o_shape(s):
    t = s[0]
    if t == "circle":
        return O.Shape.circle(*s[1:])
    if t == "section":
        corner, b, cx, cy, d, angle = s[1:]
        return O.Shape.section(corner, b, cx, cy, d, angle)
    if t == "disks":
        return O.Shape.disks(s[1])
    if t == "band":
        return O.Shape.outside_band(*s[1:])
    if t == "polygon":
        return O.Shape.polygon(s[1])
    if t == "ellipse":
        return O.Shape.ellipse(*s[1:])
    raise ValueError(t)


def _v_vel(v):
    if v is None:
        return None
    return {"const": V.Velocity.const, "parabolic": V.Velocity.parabolic, "rotation": V.Velocity.rotation}[v[0]](*v[1:])


def _coll(desc):
    c = desc.get("collision", ("trt", 3.0 / 16.0))
    return ("bgk", 0.0) if c == "bgk" else c


def product_builder(desc):
    b = V.Builder(desc["nx"], desc["ny"])
    b.periodic_x, b.periodic_y = desc.get("periodic", (False, False))
    b.tau = desc.get("tau", 1.0)
    c = _coll(desc)
    b.collision = V.Collision.Bgk if c[0] == "bgk" else V.Collision.Trt(c[1])
    b.accel = desc.get("accel", (0.0, 0.0))
    for k in desc.get("kinds", []):
        if k[0] == "wall":
            _, vel, vg, fg, shape = k
            b.add(V.Kind.Wall(V.Wall(velocity=_v_vel(vel), vgroup=vg, fgroup=fg,
                                     shape=_v_shape(shape) if shape is not None else None)))
        elif k[0] == "pressure":
            b.add(V.Kind.Pressure(k[1]))
        else:
            b.add(V.Kind.Radiating(k[1]))
    for p in desc.get("paint", []):
        if p[0] == "rect":
            b.fill_rect(*p[1:])
        else:
            b.fill_shape(p[1])
    return b


def product_sim(desc, precision="f64"):
    return product_builder(desc).build(precision=precision)


def oracle_sim(desc, threads=1):
    b = O.Builder(desc["nx"], desc["ny"])
    b.periodic_x, b.periodic_y = desc.get("periodic", (False, False))
    b.tau = desc.get("tau", 1.0)
    c = _coll(desc)
    b.collision = O.BGK if c[0] == "bgk" else O.TRT
    b.magic = c[1] if c[0] != "bgk" else 3.0 / 16.0
    b.accel = desc.get("accel", (0.0, 0.0))
    for k in desc.get("kinds", []):
        if k[0] == "wall":
            _, vel, vg, fg, shape = k
            b.add_wall(velocity=vel, vgroup=vg, fgroup=fg, shape=_o_shape(shape) if shape is not None else None)
        elif k[0] == "pressure":
            b.add_pressure(k[1])
        else:
            b.add_radiating(k[1])
    for p in desc.get("paint", []):
        if p[0] == "rect":
            b.fill_rect(*p[1:])
        else:
            b.fill_shape(p[1])
    return b.build(threads)


# ---------------------------------------------------------------- named domains
def swirl(nx, ny):
    """tests/solver.rs:14-19 as arrays."""
    x = np.arange(nx)[None, :].astype(np.float64)
    y = np.arange(ny)[:, None].astype(np.float64)
    a = 2.0 * np.pi * x / nx
    b = 2.0 * np.pi * y / ny
    rho = 1.0 + 0.02 * np.sin(a + 2.0 * b)
    ux = 0.05 * np.sin(b) + 0.01 + 0.0 * a
    uy = -0.04 * np.cos(a) + 0.02 * np.sin(a - b)
    return (np.broadcast_to(rho, (ny, nx)).copy(), np.broadcast_to(ux, (ny, nx)).copy(),
            np.broadcast_to(uy, (ny, nx)).copy())


def periodic_box(nx=48, ny=36, tau=0.62, collision=("trt", 3.0 / 16.0), accel=(0.0, 0.0)):
    return dict(nx=nx, ny=ny, periodic=(True, True), tau=tau, collision=collision, accel=accel)


def disk_box(nx, ny, disks, tau=0.55):
    return dict(nx=nx, ny=ny, periodic=(True, True), tau=tau, collision="bgk",
                kinds=[("wall", None, 0, 0, ("disks", disks))], paint=[("shape", 1)])


def tunnel_like(nx=122, ny=42, d=10, u=0.05, nu=0.01, radiating=True, angle=0.3):
    """A small towing tank: uniform inlet, pressure outlet, radiating or moving side walls, and a
    rotated notched square body with rotation velocity (the kick) and force group 0."""
    cx, cy = 30.5, 0.5 + 0.5 * (ny - 2)
    tau = nu / (1.0 / 3.0) + 0.5
    walls = ("radiating", 1.0) if radiating else ("wall", ("const", u, 0.0), 1, None, None)
    kinds = [("wall", ("const", u, 0.0), 1, None, None), ("pressure", 1.0), walls,
             ("wall", ("rotation", cx, cy), 2, 0, ("section", 4, 0.1, cx, cy, float(d), angle))]
    paint = [("rect", 0, 0, 0, ny - 1, 1), ("rect", nx - 1, nx - 1, 0, ny - 1, 2),
             ("rect", 1, nx - 2, 0, 0, 3), ("rect", 1, nx - 2, ny - 1, ny - 1, 3)]
    if not radiating:
        paint += [("rect", 0, nx - 1, 0, 0, 3), ("rect", 0, nx - 1, ny - 1, ny - 1, 3)]
    paint.append(("shape", 4))
    return dict(nx=nx, ny=ny, tau=tau, collision=("trt", 3.0 / 16.0), kinds=kinds, paint=paint)


def couette(frame=0.03, shear=0.04, collision="bgk", nx=6, rows=20):
    """tests/solver.rs:86-102."""
    return dict(nx=nx, ny=rows + 2, periodic=(True, False), tau=0.9, collision=collision,
                kinds=[("wall", ("const", frame, 0.0), 0, 0, None),
                       ("wall", ("const", frame + shear, 0.0), 0, 1, None)],
                paint=[("rect", 0, nx - 1, 0, 0, 1), ("rect", 0, nx - 1, rows + 1, rows + 1, 2)])


def poiseuille(rows=16, tau=0.8, q=0.8, collision=("trt", 3.0 / 16.0)):
    """src/cases/poiseuille.rs:41-60 (body-force driven periodic channel)."""
    nx, ny = 4, rows + 2
    y0, y1 = 1.0 - q, rows + q
    width = y1 - y0
    nu = (tau - 0.5) / 3.0
    umax = 0.1 * 16.0 / rows
    g = 8.0 * nu * umax / (width * width)
    shape = None if q == 0.5 else ("band", y0, y1)
    return dict(nx=nx, ny=ny, periodic=(True, False), tau=tau, collision=collision, accel=(g, 0.0),
                kinds=[("wall", None, 0, 0, shape)],
                paint=[("rect", 0, nx - 1, 0, 0, 1), ("rect", 0, nx - 1, ny - 1, ny - 1, 1)])


def oracle_shape(body):
    """The oracle's copy of a product shape description (the batched-tunnel bodies)."""
    import vortexlab_b200 as V
    if isinstance(body, V.Rotated):
        return O.Shape.rotated(oracle_shape(body.inner), body.cx, body.cy, body.angle)
    if isinstance(body, V.Translated):
        return O.Shape.translated(oracle_shape(body.inner), body.dx, body.dy)
    if isinstance(body, V.Ellipse):
        return O.Shape.ellipse(body.cx, body.cy, body.a, body.b)
    if isinstance(body, V.Star):
        return O.Shape.star(body.cx, body.cy, list(body.radii), body.phase)
    if isinstance(body, V.Polygon):
        return O.Shape.polygon(body.pts)
    if isinstance(body, V.Circle):
        return O.Shape.circle(body.cx, body.cy, body.r)
    raise TypeError(f"no oracle shape for {type(body).__name__}")


def oracle_channel(spec, threads=1):
    """The oracle's Channel (src/cases/channel.rs:71-116) for a product Spec."""
    kick = None
    if spec.kick is not None:
        k = spec.kick
        kick = (k.cx, k.cy, k.omega, float(k.start), float(k.duration))
    coll = O.BGK if spec.collision.kind == 0 else O.TRT
    return O.Channel(spec.nx, spec.ny, spec.inflow[0], spec.inflow[1], spec.nu, coll, oracle_shape(spec.body),
                     spec.ramp_steps, kick, threads, spec.collision.magic)
