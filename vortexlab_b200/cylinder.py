"""Schafer-Turek "flow around a cylinder" rig on the device (src/cases/cylinder.rs).

Channel 22n x 4.1n cells (n cells per diameter), cylinder of diameter n at (2n + 1/2, 2n + 1/2),
parabolic inflow with mean velocity ``u_mean``, TRT by default. Forces and the pressure drop are
recorded on the device every step and downloaded once (the reference reads them on the host after
every step, src/cases/cylinder.rs:176-190).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import TRT, Channel, Circle, Collision, Inflow, Series, Spec, VortexError, signal, tau_for


@dataclass
class Setup:
    """src/cases/cylinder.rs:18-26."""

    n: int
    u_mean: float = 0.05
    collision: Collision = field(default_factory=lambda: TRT)
    threads: Optional[int] = None
    precision: str = "f64"


@dataclass
class Rig:
    ch: Channel
    n: float
    xc: float
    yc: float

    def pressure_drop(self) -> float:
        """src/cases/cylinder.rs:54-59, from the current state."""
        r = 0.5 * self.n
        front = self.ch.sim.probe_density_at_wall(self.xc - r, self.yc, -1.0, 0.0)
        back = self.ch.sim.probe_density_at_wall(self.xc + r, self.yc, 1.0, 0.0)
        return (1.0 / 3.0) * (front - back) / (self.ch.u_ref * self.ch.u_ref)


def rig(s: Setup, re: float, ramp_units: float) -> Rig:
    """src/cases/cylinder.rs:35-50."""
    if s.n < 10 or s.n % 10 != 0:
        raise ValueError("cells per diameter must be a multiple of 10")
    n = float(s.n)
    xc = yc = 0.5 + 2.0 * n
    spec = Spec(nx=22 * s.n + 2, ny=41 * s.n // 10 + 2, inflow=Inflow.Parabolic(s.u_mean), nu=s.u_mean * n / re,
                collision=s.collision, body=Circle(xc, yc, 0.5 * n), ramp_steps=int(ramp_units * n / s.u_mean))
    return Rig(Channel(spec, precision=s.precision), n, xc, yc)


@dataclass
class Unsteady:
    """src/cases/cylinder.rs:142-165."""

    n: int
    cd_max: float
    cd_min: float
    cl_max: float
    cl_min: float
    st: float
    st_crossings: float
    dp: float
    peak_spread: float
    periods: int
    steps: int
    seconds: float
    series: Series
    dp_series: np.ndarray
    window_start: int


def run_record(r: Rig, steps: int, chunk: int = 1 << 16):
    """Runs ``steps`` channel steps recording (cd, cl, dp) every step on the device."""
    sim = r.ch.sim
    sim.set_dp_probe(r.xc, r.yc, 0.5 * r.n, r.ch.u_ref)
    k = 2.0 / (r.ch.u_ref * r.ch.u_ref * r.n)
    cd, cl, dp = np.zeros(steps), np.zeros(steps), np.zeros(steps)
    done = 0
    while done < steps:
        m = min(chunk, steps - done)
        sim.record(m)
        r.ch.step(m)
        h = sim.history()
        cd[done:done + m] = k * h[:, 0]
        cl[done:done + m] = k * h[:, 1]
        dp[done:done + m] = h[:, 9]
        done += m
    return cd, cl, dp


def run_2d2(s: Setup, total_units: float, window_units: float) -> Unsteady:
    """Case 2D-2 (Re = 100), src/cases/cylinder.rs:169-220. Raises VortexError on divergence."""
    start = time.time()
    r = rig(s, 100.0, 8.0)
    unit = r.n / s.u_mean
    steps = int(total_units * unit)
    cd, cl, dp = run_record(r, steps)
    bad = np.nonzero(~np.isfinite(cd))[0]
    if len(bad):
        raise VortexError(-3, f"diverged after {int(bad[0]) + 1} steps (tau = {tau_for(s.u_mean * r.n / 100.0):.4f}): "
                              f"under-resolved at {s.n} cells per diameter")
    series = Series(1.0 / unit, cd, cl)
    i0 = steps - min(int(window_units * unit), steps)
    cdw, clw, dpw = cd[i0:], cl[i0:], dp[i0:]
    f, _ = signal.dominant_frequency(clw, series.dt)
    period = 1.0 / (f * series.dt)
    pk = signal.peaks(clw)
    tops = [p[1] for p in pk]
    cl_max = max(tops) if tops else float("-inf")
    spread = (cl_max - min(tops)) / signal.mean(tops) if tops else float("nan")
    half = [signal.sample_at(dpw, p[0] + 0.5 * period) for p in pk if p[0] + 0.5 * period < len(dpw) - 1]
    return Unsteady(n=s.n, cd_max=float(np.max(cdw)), cd_min=float(np.min(cdw)), cl_max=cl_max,
                    cl_min=float(np.min(clw)), st=f,
                    st_crossings=signal.crossing_frequency(clw, series.dt) or float("nan"),
                    dp=signal.mean(half) if half else float("nan"), peak_spread=spread, periods=len(tops),
                    steps=steps, seconds=time.time() - start, series=series, dp_series=dp, window_start=i0)


def bench(s: Setup, steps: int):
    """src/cases/cylinder.rs:224-232: times ``steps`` steps (forces every step). Returns
    (channel, seconds) with the device time of the batch."""
    r = rig(s, 100.0, 8.0)
    r.ch.step(steps)
    r.ch.sim.synchronize()
    return r.ch, r.ch.sim.last_step_ms() * 1e-3
