"""The on-line stopping rule on synthetic force histories (host only)."""
import numpy as np

from vortexlab_b200.online import StopRule, reference, settled


def _history(units=60.0, dt=1.0 / 600.0, st=0.2, settle=15.0, cd=1.4, amp=0.5):
    """c_D relaxing to `cd` and a lift oscillation growing to `amp` at frequency `st`, both with a
    time constant of settle / 5 convective units."""
    t = np.arange(int(units / dt)) * dt
    env = 1.0 - np.exp(-t / (settle / 5.0))
    cdh = cd * (1.0 + 0.2 * np.exp(-t / (settle / 5.0)))
    clh = amp * env * np.sin(2.0 * np.pi * st * t)
    return cdh, clh, dt


def _first_stop(cd, cl, dt, rule, check=2.0):
    every = int(check / dt)
    for end in range(every, len(cd) + 1, every):
        r = settled(cd[:end], cl[:end], dt, rule)
        if r is not None:
            return end * dt, r
    return None, None


def test_rule_waits_for_the_transient_and_reports_the_settled_values():
    cd, cl, dt = _history()
    rule = StopRule()
    t_stop, r = _first_stop(cd, cl, dt, rule)
    assert t_stop is not None and 10.0 <= t_stop <= 40.0
    c, st, steady = r
    assert not steady
    assert abs(c - 1.4) <= 0.005 * 1.4
    assert abs(st - 0.2) <= 0.005 * 0.2
    # before the transient has decayed, the windows disagree
    assert settled(cd[: int(8.0 / dt)], cl[: int(8.0 / dt)], dt, rule) is None


def test_rule_never_stops_a_drifting_run():
    cd, cl, dt = _history()
    drift = cd * (1.0 + 0.002 * np.arange(len(cd)) * dt)       # 0.2 % per convective unit
    t_stop, _ = _first_stop(drift, cl, dt, StopRule())
    assert t_stop is None


def test_steady_wake_stops_on_drag_alone():
    cd, cl, dt = _history(amp=0.0)
    t_stop, r = _first_stop(cd, cl, dt, StopRule())
    assert t_stop is not None and r[2] and r[1] == 0.0
    c, st, steady = reference(cd, cl, dt, StopRule())
    assert steady and abs(c - 1.4) <= 1e-3


def test_non_finite_history_never_stops():
    cd, cl, dt = _history()
    cd[-10:] = np.nan
    assert settled(cd, cl, dt, StopRule()) is None


def test_cached_window_stops_like_the_full_rule():
    """Reusing the spectral window length between checks (as the on-line batch driver does) stops
    within one check of the rule evaluated from scratch, with the same settled values to 0.1 %."""
    cd, cl, dt = _history(units=80.0, settle=25.0)
    rule = StopRule()
    t_full, r_full = _first_stop(cd, cl, dt, rule)
    every = int(2.0 / dt)
    cache = {}
    t_cached = r_cached = None
    for end in range(every, len(cd) + 1, every):
        r = settled(cd[:end], cl[:end], dt, rule, cache)
        if r is not None:
            t_cached, r_cached = end * dt, r
            break
    assert t_full is not None and t_cached is not None
    assert abs(t_cached - t_full) <= 2.0 + 1e-9
    assert abs(r_cached[0] - r_full[0]) <= 1e-3 * abs(r_full[0])
    assert abs(r_cached[1] - r_full[1]) <= 1e-3 * r_full[1]


class _FakeBatch:
    """Host stand-in for a batch of tunnels with the asynchronous run semantics of the library:
    run_async advances the global step at once, records become readable after wait, a tunnel can
    be ended only at or after the step the enqueued run ends at, and a held tunnel takes its step 0
    at the global step after the enqueued ones when it is started."""

    def __init__(self, histories, steps, held=()):
        self.h = histories          # per tunnel (n, 2) force records of its own steps
        self.steps = list(steps)
        self.start_at = [None if k in held else 0 for k in range(len(steps))]
        self.s = 0
        self.s_done = 0
        self.run_steps = 0

    def own(self, k, g):
        st = self.start_at[k]
        return 0 if st is None else max(0, min(g - st, self.steps[k]))

    def info(self, k):
        return {"steps": self.steps[k]}

    def run_async(self, n):
        ends = [st + e for st, e in zip(self.start_at, self.steps) if st is not None]
        end = min(max(ends), self.s + n)
        self.run_steps += sum(self.own(k, max(end, self.s)) - self.own(k, self.s) for k in range(len(self.steps)))
        self.s = max(self.s, end)

    def wait(self):
        self.s_done = self.s

    def global_step(self):
        return self.s

    def history_copy(self, ranges):
        out = []
        for k, first, count in ranges:
            assert first + count <= self.own(k, self.s_done), (k, first, count, self.s_done)
            out.append(self.h[k][first:first + count])
        return out

    def set_steps(self, k, steps):
        assert steps >= self.own(k, self.s) and steps <= self.steps[k]
        self.steps[k] = steps

    def start(self, k):
        assert self.start_at[k] is None
        self.start_at[k] = self.s
        return self.s

    def status(self, k):
        return self.own(k, self.s), False, None


class _Tun:
    def __init__(self, spu, u=0.05, d=20.0):
        self.spu, self.u, self.d = spu, u, d

    def steps_per_unit(self):
        return self.spu


class _Case:
    def __init__(self, spu):
        self.tunnel = _Tun(spu)


def test_overlapped_batch_checks_stop_each_tunnel_within_a_chunk():
    """batch_online with a chunk in flight during the checks: each tunnel stops where the rule
    first holds on its own records (checked every 2 convective units), is ended at the end of the
    chunk enqueued at that moment, never reads a record that is not complete, and every step it ran
    is counted."""
    from vortexlab_b200.online import batch_online
    rule = StopRule()
    spus, settles = [300, 600, 450], [10.0, 25.0, 400.0]     # the last never settles in 60 units
    hist, cases = [], []
    k_force = 2.0 / (0.05 * 0.05 * 20.0)
    for spu, st in zip(spus, settles):
        cd, cl, dt = _history(units=60.0, dt=1.0 / spu, settle=st)
        hist.append(np.stack([cd / k_force, cl / k_force], axis=1))
        cases.append(_Case(spu))
    b = _FakeBatch(hist, [len(h) for h in hist])
    res, _ = batch_online(b, cases, rule, max_units=60.0, check_units=2.0)
    chunk = 600
    for k, (spu, r) in enumerate(zip(spus, res)):
        cd, cl = hist[k][:, 0] * k_force, hist[k][:, 1] * k_force
        every = 2 * spu
        want = None
        for end in range(every, len(cd) + 1, every):
            if settled(cd[:end], cl[:end], 1.0 / spu, rule) is not None:
                want = end
                break
        if want is None:
            assert r["stop"] is None and r["steps"] == len(cd), k
        else:
            assert r["stop"]["steps"] == want, (k, r["stop"], want)
            assert want <= r["steps"] <= want + chunk, (k, r["steps"], want)
    assert b.run_steps == sum(r["steps"] for r in res)


def test_overlapped_checks_start_a_held_twin_when_a_tunnel_fails():
    """A tunnel that reaches its end unsettled starts its held twin at once; the twin is checked
    from its own step 0 and stops where the rule first holds on its own records; a twin of a
    settled tunnel is never started."""
    from vortexlab_b200.online import batch_online
    rule = StopRule()
    k_force = 2.0 / (0.05 * 0.05 * 20.0)
    spu = 300
    hist = []
    for st in (400.0, 10.0, 10.0, 400.0):         # 0 never settles, 2 is its twin and settles; 1 settles, 3 its twin
        cd, cl, dt = _history(units=60.0, dt=1.0 / spu, settle=st)
        hist.append(np.stack([cd / k_force, cl / k_force], axis=1))
    cases = [_Case(spu) for _ in hist]
    b = _FakeBatch(hist, [len(h) for h in hist], held=(2, 3))
    res, _ = batch_online(b, cases, rule, max_units=60.0, check_units=2.0, twins={0: 2, 1: 3})
    assert res[0]["stop"] is None and res[0]["steps"] == len(hist[0])
    assert res[2]["start"] is not None and res[2]["start"] >= len(hist[0])
    assert res[2]["stop"] is not None
    assert res[1]["stop"] is not None and res[3]["start"] is None and res[3]["steps"] == 0
    cd, cl = hist[2][:, 0] * k_force, hist[2][:, 1] * k_force
    want = next(e for e in range(2 * spu, len(cd) + 1, 2 * spu) if settled(cd[:e], cl[:e], 1.0 / spu, rule) is not None)
    assert abs(res[2]["stop"]["steps"] - want) <= 2 * spu      # its checks fall between the 2-unit marks
    assert b.run_steps == sum(r["steps"] for r in res)
