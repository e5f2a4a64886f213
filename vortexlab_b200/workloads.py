"""Seeded synthetic workloads.

``disk_field`` places solid disks in a periodic box with the xorshift64* generator the reference's
tests use (src/lattice.rs:162-171): radii uniform in [rmin, rmax], centres uniform with every disk
at least one cell clear of the box edge, added until the painted solid fraction (cells whose
centre is strictly inside a disk) reaches ``fraction``. The throughput workload is the
8192 x 4096 box, seed 0x5EED0001, 5 % solid, BGK tau = 0.55, uniform start (1, 0.05, 0).
"""
from __future__ import annotations

import numpy as np

M64 = (1 << 64) - 1


class XorShift64Star:
    """src/lattice.rs:162-171: next() in [0, 1) with 53 random bits."""

    def __init__(self, seed: int):
        self.s = seed & M64

    def next(self) -> float:
        s = self.s
        s ^= s >> 12
        s ^= (s << 25) & M64
        s ^= s >> 27
        self.s = s
        return (((s * 0x2545F4914F6CDD1D) & M64) >> 11) / float(1 << 53)


def disk_field(nx: int, ny: int, seed: int = 0x5EED0001, fraction: float = 0.05, rmin: float = 4.0,
               rmax: float = 16.0) -> np.ndarray:
    """(n, 3) array of (cx, cy, r); the painted solid fraction is the first value >= ``fraction``."""
    rng = XorShift64Star(seed)
    solid = np.zeros((ny, nx), dtype=bool)
    need = fraction * nx * ny
    count = 0
    disks = []
    while count < need:
        r = rmin + (rmax - rmin) * rng.next()
        cx = r + 1.0 + (nx - 2.0 * r - 2.0) * rng.next()
        cy = r + 1.0 + (ny - 2.0 * r - 2.0) * rng.next()
        x0, x1 = int(np.floor(cx - r)), int(np.ceil(cx + r))
        y0, y1 = int(np.floor(cy - r)), int(np.ceil(cy + r))
        xs = np.arange(x0, x1 + 1, dtype=np.float64)
        ys = np.arange(y0, y1 + 1, dtype=np.float64)
        dx = xs[None, :] - cx
        dy = ys[:, None] - cy
        inside = dx * dx + dy * dy < r * r
        sub = solid[y0:y1 + 1, x0:x1 + 1]
        count += int(np.count_nonzero(inside & ~sub))
        sub |= inside
        disks.append((cx, cy, r))
    return np.array(disks, dtype=np.float64)


THROUGHPUT_BOX = dict(nx=8192, ny=4096, seed=0x5EED0001, fraction=0.05, tau=0.55, u=0.05)


def build_disk_box(V, nx, ny, disks, tau=0.55, precision="f64"):
    """Builds the periodic BGK box on the device with the package ``V`` (vortexlab_b200)."""
    b = V.Builder(nx, ny)
    b.periodic_x = b.periodic_y = True
    b.tau = tau
    b.collision = V.Collision.Bgk
    k = b.add(V.Kind.Wall(V.Wall(fgroup=0, shape=V.Disks(disks))))
    b.fill_shape(k)
    return b.build(precision=precision)
