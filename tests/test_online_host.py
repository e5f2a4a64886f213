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
