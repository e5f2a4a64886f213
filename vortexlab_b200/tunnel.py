"""The towing tank (src/cases/tunnel.rs:11-93) on the device."""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import TRT, Channel, Collision, Inflow, Kick, Series, Spec, VortexError, tau_for


@dataclass
class Tunnel:
    d: int
    re: float
    u: float
    upstream: float
    downstream: float
    height: float
    length: float = 1.0
    collision: Collision = field(default_factory=lambda: TRT)
    threads: int = 1
    open_sides: bool = True
    precision: str = "f64"

    def grid(self):
        """src/cases/tunnel.rs:35-38."""
        d = float(self.d)
        return int(round_half_away((self.upstream + self.downstream) * d)) + 2, int(round_half_away(self.height * d)) + 2

    def centre(self):
        """src/cases/tunnel.rs:41-44."""
        d = float(self.d)
        return 0.5 + round_half_away(self.upstream * d), 0.5 + 0.5 * round_half_away(self.height * d)

    def steps_per_unit(self) -> float:
        return float(self.d) / self.u

    def spec(self, body) -> Spec:
        """The channel of src/cases/tunnel.rs:52-67: 5-unit inflow ramp, then a 2-unit twist of the
        body."""
        nx, ny = self.grid()
        cx, cy = self.centre()
        unit = self.steps_per_unit()
        return Spec(nx=nx, ny=ny, inflow=Inflow.UniformOpen(self.u) if self.open_sides else Inflow.Uniform(self.u),
                    nu=self.u * self.d / self.re, collision=self.collision, body=body, ramp_steps=int(5.0 * unit),
                    kick=Kick(cx, cy, 0.4 * self.u / self.d, int(5.0 * unit), int(2.0 * unit)))

    def spec_warm(self, body) -> Spec:
        """The same channel for a run that starts from a developed field: no inflow ramp and no
        twist of the body (the start field already carries the wake)."""
        s = self.spec(body)
        s.ramp_steps = 0
        s.kick = None
        return s

    def build(self, body) -> Channel:
        """src/cases/tunnel.rs:52-67."""
        return Channel(self.spec(body), precision=self.precision)

    def run(self, ch: Channel, units: float) -> Series:
        """src/cases/tunnel.rs:71-92 (force coefficients every step, recorded on the device)."""
        unit = self.steps_per_unit()
        steps = int(units * unit)
        sim = ch.sim
        sim.record(steps)
        ch.step(steps)
        h = sim.history()
        k = 2.0 / (ch.u_ref * ch.u_ref * float(self.d))
        cd, cl = k * h[:, 0], k * h[:, 1]
        bad = np.nonzero(~np.isfinite(cd))[0]
        if len(bad):
            raise VortexError(-3, f"the simulation became unstable after {int(bad[0])} steps "
                                  f"(tau = {tau_for(self.u * self.d / self.re):.4f})")
        return Series(1.0 / unit, cd, cl)


def round_half_away(v: float) -> float:
    """Rust's f64::round (half away from zero)."""
    import math
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)
