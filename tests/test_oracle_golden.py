"""The oracle, pinned: the reference's published state hashes and its own unit tests.

The hashes are FNV-1a over every population bit after `vortexlab bench` (docs/report/index.html:59,
Makefile:42-43); matching them shows the restatement performs the reference's floating-point
operations in the same order. The unit tests are src/lattice.rs:184-288, src/geometry.rs:298-357,
src/signal.rs:351-405 and src/cases/channel.rs:195-217, with the reference's tolerances.
"""
import math

import numpy as np
import pytest

import oracle as O


@pytest.mark.parametrize("grid", ["882x166", "1762x330"])
def test_oracle_reproduces_published_hash(O, published, grid):
    case = published["bench_state_hashes"][grid]
    ch, n, xc, yc = O.cylinder_rig(case["n"], threads=8)
    assert (f"{ch.sim.nx}x{ch.sim.ny}", ch.sim.fluid_nodes()) == (grid, case["fluid_nodes"])
    ch.run(case["steps"], record_force=False)
    assert {f"{ch.sim.state_hash():016x}"} == set(case["hashes"].values())


def test_result_does_not_depend_on_thread_count(O):
    """tests/solver.rs:255-291 (222 x 43 cylinder channel, 400 steps)."""
    ref = None
    for threads in [1, 2, 3, 4, 7]:
        ch = O.Channel(222, 43, O.PARABOLIC, 0.05, 0.05 * 10.0 / 100.0, O.TRT, O.Shape.circle(20.5, 20.5, 5.0), 100,
                       threads=threads)
        assert ch.sim.threads() == threads
        fh, _ = ch.run(400)
        got = (ch.sim.state_hash(), fh[-1].tobytes())
        ref = ref or got
        assert got == ref
    assert ch.coefficients(10.0)[0] > 1.0


class Rng:
    """src/lattice.rs:162-171."""

    def __init__(self, s):
        self.s = s

    def next(self):
        M = (1 << 64) - 1
        s = self.s
        s ^= s >> 12
        s ^= (s << 25) & M
        s ^= s >> 27
        self.s = s
        return (((s * 0x2545F4914F6CDD1D) & M) >> 11) / float(1 << 53)


W = [4 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 36, 1 / 36, 1 / 36, 1 / 36]


def random_state(rng):
    rho = 0.8 + 0.4 * rng.next()
    ux = 0.2 * (rng.next() - 0.5)
    uy = 0.2 * (rng.next() - 0.5)
    f = O.equilibrium(rho, ux, uy)
    for i in range(9):
        f[i] += 0.02 * W[i] * (rng.next() - 0.5)
    return f


def test_equilibrium_moments(O):
    rng = Rng(0x123456789ABCDEF1)
    cx = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1.0])
    cy = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1.0])
    for _ in range(200):
        rho = 0.5 + rng.next()
        ux = 0.3 * (rng.next() - 0.5)
        uy = 0.3 * (rng.next() - 0.5)
        f = O.equilibrium(rho, ux, uy)
        r, jx, jy = O.moments(f)
        assert abs(r - rho) < 1e-14 and abs(jx - rho * ux) < 1e-14 and abs(jy - rho * uy) < 1e-14
        assert abs(np.dot(f, cx * cx) - rho * (1 / 3 + ux * ux)) < 1e-14
        assert abs(np.dot(f, cy * cy) - rho * (1 / 3 + uy * uy)) < 1e-14
        assert abs(np.dot(f, cx * cy) - rho * ux * uy) < 1e-14


def test_collisions_conserve_mass_and_momentum(O):
    rng = Rng(42)
    for _ in range(300):
        f = random_state(rng)
        tau = 0.51 + 1.5 * rng.next()
        op, om = O.omegas(O.TRT, 0.25, tau)
        r0, x0, y0 = O.moments(f)
        for out in (O.collide_bgk(f, op), O.collide_trt(f, op, om)):
            r, x, y = O.moments(out)
            assert abs(r - r0) < 1e-14 and abs(x - x0) < 1e-14 and abs(y - y0) < 1e-14


def test_equilibrium_is_a_fixed_point_and_trt_equal_rates_is_bgk(O):
    f = O.equilibrium(1.1, 0.07, -0.03)
    for out in (O.collide_bgk(f, 1.7), O.collide_trt(f, 1.7, 0.9)):
        assert np.max(np.abs(out - f)) < 1e-15
    rng = Rng(7)
    for _ in range(200):
        f = random_state(rng)
        om = 0.6 + 1.3 * rng.next()
        assert np.max(np.abs(O.collide_bgk(f, om) - O.collide_trt(f, om, om))) < 1e-15


def test_forced_collision_adds_exactly_the_force(O):
    rng = Rng(99)
    for _ in range(200):
        f = random_state(rng)
        gx, gy = 1e-3 * (rng.next() - 0.5), 1e-3 * (rng.next() - 0.5)
        op, om = O.omegas(O.TRT, 3.0 / 16.0, 0.5 + rng.next())
        out = O.collide_forced(f, op, om, gx, gy)
        r0, x0, y0 = O.moments(f)
        r, x, y = O.moments(out)
        assert abs(r - r0) < 1e-14 and abs(x - x0 - r0 * gx) < 1e-14 and abs(y - y0 - r0 * gy) < 1e-14
        assert np.max(np.abs(O.collide_forced(f, op, om, 0.0, 0.0) - O.collide_trt(f, op, om))) < 1e-15


def test_viscosity_round_trip(O):
    op, om = O.omegas(O.TRT, 0.1875, 0.8)
    assert abs((1 / op - 0.5) * (1 / om - 0.5) - 0.1875) < 1e-15


def test_cut_fraction_on_a_circle(O):
    c = O.Shape.circle(0.0, 0.0, 10.3)
    assert abs(c.cut_fraction(-11.0, 0.0, 1.0, 0.0) - 0.7) < 1e-9
    assert abs(c.cut_fraction(8.0, 8.0, -1.0, -1.0) - (8.0 - 10.3 / math.sqrt(2))) < 1e-9


def _area(s, x0, x1, n):
    h = (x1 - x0) / n
    cnt = 0
    for j in range(n):
        for i in range(n):
            cnt += s.inside(x0 + (i + 0.5) * h, x0 + (j + 0.5) * h)
    return cnt * h * h


def test_section_areas_match_geometry(O):
    cases = [(O.SHARP, 0.0, 1.0), (O.CHAMFERED, 0.1, 1 - 4 * 0.005), (O.ROUNDED, 0.1, 1 - (4 - math.pi) * 0.01),
             (O.RECESSED, 0.1, 1 - 4 * 0.01), (O.DOUBLE_RECESSED, 0.05, 1 - 4 * 3 * 0.0025)]
    for corner, b, expect in cases:
        s = O.Shape.section(corner, b, 0.0, 0.0, 1.0, 0.0)
        assert abs(_area(s, -0.6, 0.6, 300) - expect) < 8e-3
        assert s.inside(0.499, 0.0) and s.inside(0.0, 0.499) and not s.inside(0.501, 0.0)


def test_rotation_translation_bitmap(O):
    s = O.Shape.section(O.SHARP, 0.0, 0.0, 0.0, 1.0, math.pi / 4)
    assert s.inside(0.69, 0.0) and not s.inside(0.72, 0.0) and not s.inside(0.45, 0.45)
    t = O.Shape.translated(O.Shape.section(O.SHARP, 0.0, 0.0, 0.0, 4.0, 0.0), 1.0, -0.5)
    assert t.inside(2.9, 1.4) and not t.inside(3.1, 0.0) and not t.inside(0.0, 1.6)
    x0, x1, y0, y1 = t.bounding_box(6.0, 0.05)
    assert abs(x0 + 1) < 0.06 and abs(x1 - 3) < 0.06 and abs(y0 + 2.5) < 0.06 and abs(y1 - 1.5) < 0.06
    assert O.Shape.circle(50.0, 0.0, 1.0).bounding_box(6.0, 0.1) is None
    level = np.zeros((4, 4), dtype=np.float32)
    level[:, 2:] = 1.0
    b = O.Shape.bitmap(level, 10.0, 20.0, 2.0)
    assert not b.inside(13.9, 24.0) and b.inside(14.1, 24.0)
    assert abs(b.cut_fraction(13.0, 24.0, 2.0, 0.0) - 0.5) < 1e-6


def _lcg(seed):
    seed[0] = (seed[0] * 6364136223846793005 + 1442695040888963407) & ((1 << 64) - 1)
    return (seed[0] >> 11) / float(1 << 53) - 0.5


def test_fft_matches_naive_dft(O):
    seed = [2024]
    for n in [1, 2, 4, 8, 64, 256]:
        re = np.array([_lcg(seed) for _ in range(n)])
        im = np.array([_lcg(seed) for _ in range(n)])
        fr, fi = O.fft(re, im)
        ref = np.fft.fft(re + 1j * im)
        assert np.max(np.abs(fr - ref.real)) < 1e-10 and np.max(np.abs(fi - ref.imag)) < 1e-10


def test_dominant_frequency_between_bins(O):
    n, dt = 3000, 0.01
    f0 = 13.37 / (n * dt)
    x = 2.5 + 0.8 * np.sin(2 * np.pi * f0 * np.arange(n) * dt + 0.4)
    f, amp = O.dominant_frequency(x, dt)
    assert abs(f / f0 - 1) < 2e-4 and abs(amp - 0.8) < 0.01
    assert abs(O.crossing_frequency(x, dt) / f0 - 1) < 1e-3


def test_peaks_and_statistics(O):
    x = 1.0 + 0.5 * np.sin(2 * np.pi * np.arange(2000) / 400.0)
    p = O.peaks(x)
    assert len(p) == 5
    for k, (pos, val) in enumerate(p):
        assert abs(pos - (100 + 400 * k)) < 1e-6 and abs(val - 1.5) < 1e-9
    assert abs(O.mean(x) - 1.0) < 1e-12 and abs(O.rms(x) - 0.5 / math.sqrt(2)) < 1e-12
    assert abs(O.sample_at(x, 100.5) - 0.5 * (x[100] + x[101])) < 1e-15


def test_ramp(O):
    assert O.ramp(0, 0) == 1.0 and O.ramp(10, 10) == 1.0 and O.ramp(5, 10) == 0.5
