"""On-line stopping of tunnel runs from their own force history, and the time-to-converged study
built on it.

A run stops when its statistics have settled: the mean c_D and the Strouhal number of its last
`windows` trailing windows of three shedding periods (each window ending half a window after the
previous one) agree within `tol` (src/cases/channel.rs:166-188, `Series::stats`, computes the same
window statistics once at the end of a run; here they are evaluated while the run goes on, and
nothing but the run's own history decides). A wake whose lift does not oscillate is steady: its
windows are five convective units and only c_D is compared.

The time-to-converged study (`comparison`) runs three arms on the same tunnels:

* plain: FP64, one tunnel at a time, uniform start (inlet ramp, body twist), run to `max_units`
  in chunks of `check_units` with the wall clock read after each chunk. The stopping rule is then
  applied at those chunk ends: the plain run's time to converged is the measured elapsed time at
  the first chunk end where it holds (the rule's own host time is not charged to this arm). The
  statistics of its last window at `max_units` are the reference values.
* cold: FP32, all tunnels in one batch, uniform start, stopped on-line.
* warm: FP32, all tunnels in one batch in their warm form (no ramp, no twist), started from the
  network's prediction, stopped on-line; each tunnel's uniform-start twin waits held in the same
  batch and is started the moment the tunnel diverges or reaches `max_units` unsettled (the
  fallback), its steps and time counted with the rest.

Every tunnel is counted. The aggregate speed-up is measured: the plain arm's summed elapsed times
to converged against the fast arm's whole wall time (inference, runs, on-line checks, fallback).
The per-tunnel speed-up divides a tunnel's plain time by its share of the batch time (the batch's
seconds per lattice update times the tunnel's cells and steps): an apportioned figure, labelled so.
Accuracy: the fast arm's statistics at its stop against the plain reference (0.5 % on c_D and St).
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import signal


# Global steps per chunk of a batch run = the most frequent tunnel's check interval / CHUNK_DIV:
# a tunnel found settled runs on to the end of the chunk already enqueued.
CHUNK_DIV = 2


@dataclass
class StopRule:
    tol: float = 0.002          # agreement of the trailing windows (relative, c_D mean and St)
    windows: int = 3            # trailing windows that must agree
    periods: float = 3.0        # window length in shedding periods
    min_units: float = 10.0     # no stop before (start transient)
    spectrum_units: float = 10.0
    steady_units: float = 5.0   # window of a steady wake
    steady_lift: float = 1e-3   # lift rms below this (times |c_D|): steady


def _window(cd, cl, dt, rule):
    """(window in steps, steady?) from the lift spectrum of the last `spectrum_units`. The spectrum
    is taken of every m-th record (about 64 per convective unit; a shedding period is several
    units, so the line is far below the decimated Nyquist frequency): the window only needs the
    period to a fraction of a percent, and the full-rate spectrum costs milliseconds per check."""
    n = min(len(cl), int(rule.spectrum_units / dt))
    if n < 8 or not (np.all(np.isfinite(cl[-n:])) and np.all(np.isfinite(cd[-n:]))):
        return None, False
    seg = cl[-n:]
    if np.std(seg) <= rule.steady_lift * max(abs(float(np.mean(cd[-n:]))), 1e-12):
        return int(rule.steady_units / dt), True
    m = max(1, int(1.0 / (64.0 * dt)))
    f = signal.dominant_frequency(seg[len(seg) % m::m], dt * m)[0]
    if not (f > 0 and np.isfinite(f)):
        return int(rule.steady_units / dt), True
    return max(8, int(rule.periods / f / dt)), False


def window_values(cd, cl, dt, end, win, steady):
    """(mean c_D, St) of the window of `win` steps ending at `end`; St = 0 for a steady wake."""
    cdw, clw = cd[end - win:end], cl[end - win:end]
    if steady:
        return float(np.mean(cdw)), 0.0
    return float(np.mean(cdw)), float(signal.crossing_frequency(clw, dt) or 0.0)


def settled(cd, cl, dt, rule: StopRule, cache=None):
    """Whether the run whose history is (cd, cl) has settled; with the statistics of its last
    window (c_D, St, steady) when it has, else None. `cache` (a dict kept per run) reuses the
    window length from the lift spectrum for `spectrum_units / 2` convective units."""
    n = len(cd)
    if n * dt < rule.min_units:
        return None
    if cache is not None and "win" in cache and (n - cache["at"]) * dt < 0.5 * rule.spectrum_units:
        win, steady = cache["win"], cache["steady"]
        if not (np.isfinite(cd[-1]) and np.isfinite(cl[-1])):
            return None
    else:
        win, steady = _window(cd, cl, dt, rule)
        if cache is not None:
            cache.update(win=win, steady=steady, at=n)
    if win is None:
        return None
    hop = max(1, win // 2)
    first_end = n - (rule.windows - 1) * hop
    if first_end - win < 0:
        return None
    vals = [window_values(cd, cl, dt, n - j * hop, win, steady) for j in range(rule.windows)]
    c0, s0 = vals[0]
    for c, s in vals[1:]:
        if abs(c - c0) > rule.tol * abs(c0):
            return None
        if not steady and (s0 <= 0 or abs(s - s0) > rule.tol * s0):
            return None
    return c0, s0, steady


def reference(cd, cl, dt, rule: StopRule):
    """The statistics of the last window of a long run (c_D, St, steady)."""
    win, steady = _window(cd, cl, dt, rule)
    if win is None or win > len(cd):
        return float("nan"), float("nan"), False
    c, s = window_values(cd, cl, dt, len(cd), win, steady)
    return c, s, steady


def _coeff(h, u, d):
    k = 2.0 / (u * u * d)
    return k * h[:, 0], k * h[:, 1]


def plain_arm(cases, rule: StopRule, max_units=100.0, check_units=2.0, log=None):
    """FP64 single runs to `max_units` (section "plain" of the module text). Per case: reference
    values, the stop (units, elapsed seconds, statistics) and the whole run's wall time."""
    out = []
    for i, c in enumerate(cases):
        tn = c.tunnel
        tn.precision = "f64"
        ch = tn.build(c.body)
        ch.sim.autotune(4)
        spu = tn.steps_per_unit()
        steps = int(max_units * spu)
        chunk = max(1, int(check_units * spu))
        ch.sim.record(steps)
        marks = []
        ch.sim.synchronize()
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            n = min(chunk, steps - done)
            ch.step(n)
            ch.sim.synchronize()
            done += n
            marks.append((done, time.perf_counter() - t0))
        h = ch.sim.history()
        schedule = ch.sim.schedule
        ch.close()
        cd, cl = _coeff(h, tn.u, tn.d)
        dt = 1.0 / spu
        ref = reference(cd, cl, dt, rule)
        stop = None
        if np.all(np.isfinite(cd)):
            cache = {}
            for end, secs in marks:
                r = settled(cd[:end], cl[:end], dt, rule, cache)
                if r is not None:
                    stop = dict(steps=end, units=end * dt, seconds=secs, cd=r[0], st=r[1], steady=r[2])
                    break
        out.append(dict(ref_cd=ref[0], ref_st=ref[1], ref_steady=ref[2], stop=stop, run_s=marks[-1][1],
                        steps=steps, schedule=schedule, finite=bool(np.all(np.isfinite(cd)))))
        if log and (i + 1) % 20 == 0:
            log(f"plain {i + 1}/{len(cases)}")
    return out


def batch_online(b, cases, rule: StopRule, max_units=100.0, check_units=2.0, chunk_global=None, twins=None):
    """Runs a built batch (`cases[i]` describes its tunnel i, added with max_units of steps) and
    stops each tunnel when the rule holds on its own history. The device runs the next chunk of
    global steps while the host reads the records of the chunk just finished (one copy for every
    tunnel due a check) and applies the rule, so a tunnel found settled at its step t is ended at
    the end of the chunk already enqueued: it runs at most one chunk past its stop, and those steps
    count in the wall time and in the lattice updates like any other. A non-finite force record
    marks a tunnel diverged (and ends it). `twins` maps a tunnel to a held tunnel of the same batch
    (vl_batch_hold): when the tunnel diverges or reaches its end unsettled, its twin is started at
    once (vl_batch_start), beside the tunnels still running, and checked like any other from its
    own step 0. Returns per-tunnel dicts (stop or None, steps run, finite, start: the global step of
    its step 0 or None if never started) and the host seconds spent in the checks (overlapped with
    the device)."""
    nt = len(cases)
    twins = dict(twins or {})
    held = set(twins.values())
    spu = np.array([c.tunnel.steps_per_unit() for c in cases])
    dt = 1.0 / spu
    every = np.maximum(1, (check_units * spu).astype(np.int64))   # steps between a tunnel's checks
    if chunk_global is None:
        chunk_global = max(1, int(every.min()) // CHUNK_DIV)
    ends = [int(b.info(k)["steps"]) for k in range(nt)]            # in the tunnel's own steps
    # c_D and c_L of each tunnel, filled in place as the records arrive
    cds = [np.empty(e) for e in ends]
    cls = [np.empty(e) for e in ends]
    have = [0] * nt
    caches = [dict() for _ in range(nt)]
    next_check = every.copy()
    start = [None if k in held else 0 for k in range(nt)]
    active = set(k for k in range(nt) if k not in held)
    result = [dict(stop=None, steps=0, finite=True, start=start[k]) for k in range(nt)]
    host_s = 0.0
    parts = dict(wait_s=0.0, copy_s=0.0, end_s=0.0)

    def own(k, g):           # steps tunnel k has done by global step g
        return 0 if start[k] is None else max(0, min(g - start[k], ends[k]))

    def end_at(k, g_next):
        e = g_next - start[k]
        if e < ends[k]:
            t1 = time.perf_counter()
            b.set_steps(k, e)
            parts["end_s"] += time.perf_counter() - t1
            ends[k] = e

    def fail_over(k):
        j = twins.get(k)
        if j is not None and start[j] is None:
            start[j] = b.start(j)
            result[j]["start"] = start[j]
            active.add(j)

    def pending(g):
        return any(start[k] + ends[k] > g for k in active)

    b.run_async(int(chunk_global))
    while True:
        t1 = time.perf_counter()
        b.wait()
        parts["wait_s"] += time.perf_counter() - t1
        s_done = b.global_step()
        more = pending(s_done)
        if more:
            b.run_async(int(chunk_global))
        s_next = b.global_step()
        t0 = time.perf_counter()
        due = []
        for k in sorted(active):
            t = own(k, s_done)
            if t < next_check[k] and t < ends[k]:
                continue
            due.append((k, have[k], t - have[k]))
        t1 = time.perf_counter()
        got = b.history_copy(due) if due else []
        parts["copy_s"] += time.perf_counter() - t1
        for (k, first, count), new in zip(due, got):
            t = first + count
            tn = cases[k].tunnel
            ncd, ncl = _coeff(new, tn.u, tn.d)
            cds[k][first:t] = ncd
            cls[k][first:t] = ncl
            have[k] = t
            next_check[k] = t + every[k]
            result[k]["steps"] = t
            if not (np.all(np.isfinite(ncd)) and np.all(np.isfinite(ncl))):
                result[k]["finite"] = False
                active.discard(k)
                end_at(k, s_next)
                fail_over(k)
                continue
            r = settled(cds[k][:t], cls[k][:t], dt[k], rule, caches[k])
            if r is not None:
                result[k].update(stop=dict(steps=t, units=float(t * dt[k]), cd=r[0], st=r[1], steady=r[2]))
                active.discard(k)
                end_at(k, s_next)
            elif t >= ends[k]:
                active.discard(k)
                fail_over(k)
        host_s += time.perf_counter() - t0
        if not more:
            if not pending(s_done):
                break
            b.run_async(int(chunk_global))      # twins started just now
    b.wait()
    for k in range(nt):
        t, nonfinite, _ = b.status(k)
        result[k]["steps"] = int(t)
        if nonfinite:
            result[k]["finite"] = False
    batch_online.last_parts = parts
    return result, host_s


def _lattice_cells(case):
    nx, ny = case.tunnel.grid()
    return nx * ny


def fast_arm(cases, rule: StopRule, net=None, precision="f32", max_units=100.0, check_units=2.0):
    """All cases in one FP32 batch, uniform start (net None) or warm start from the network,
    stopped on-line. With the network, each case's uniform-start twin (inlet ramp and twist) waits
    held in the same batch and is started the moment the warm-started tunnel diverges or reaches
    max_units unsettled: the fallback runs beside the tunnels still running and its steps are
    counted. Returns (per-case dicts, measured wall seconds, info). The wall time is what the plain
    arm's is: the runs themselves (here the network's encoding, inference and initialisation and
    the batch run with its on-line checks and fallbacks), not the building of the domains or the
    autotuning, which the plain arm does untimed too."""
    from .batch import Batch
    for c in cases:
        c.units = max_units
    n = len(cases)
    t_init = 0.0
    twins = None
    if net is not None:
        from .warmstart import warm_batch
        b, t_init = warm_batch(net, cases, precision, twins=True)
        listed = list(cases) + list(cases)
        twins = {k: n + k for k in range(n)}
    else:
        b = Batch(precision)
        for c in cases:
            b.add(c.tunnel.spec(c.body), c.steps)
        b.build()
        listed = list(cases)
    tune = b.autotune(3)
    t_run = time.perf_counter()
    res_all, host_s = batch_online(b, listed, rule, max_units, check_units, twins=twins)
    run_s = time.perf_counter() - t_run
    lu = sum(_lattice_cells(c) * r["steps"] for c, r in zip(listed, res_all))
    info = dict(tile=b.tile, autotune_ms_per_step=tune, init_s=t_init, run_s=run_s, check_host_s=host_s,
                check_parts={k: round(v, 3) for k, v in batch_online.last_parts.items()},
                device_ms=b.last_run_ms(), lattice_updates=lu)
    b.close()
    res = []
    for k in range(n):
        r = res_all[k]
        r["fallback"] = False
        if twins is not None and res_all[n + k]["start"] is not None:
            rf = res_all[n + k]
            rf["fallback"] = True
            rf["first_steps"] = r["steps"]
            r = rf
        res.append(r)
    info["fallback_tunnels"] = sum(r["fallback"] for r in res)
    wall = t_init + run_s
    info["wall_s"] = wall
    return res, wall, info


def comparison(cases, net=None, rule: StopRule = None, max_units=100.0, check_units=2.0, tol=0.005, log=None):
    """The three arms of the module text on `cases`. Returns dict(summary, rows)."""
    rule = rule or StopRule()
    plain = plain_arm(cases, rule, max_units, check_units, log=log)
    arms = {"cold": fast_arm(cases, rule, None, max_units=max_units, check_units=check_units)}
    if net is not None:
        arms["warm"] = fast_arm(cases, rule, net, max_units=max_units, check_units=check_units)
    rows = []
    for k, (c, p) in enumerate(zip(cases, plain)):
        row = dict(kind=c.kind, d=c.params["d"], re=round(c.params["re"], 1), ref_cd=p["ref_cd"], ref_st=p["ref_st"],
                   ref_steady=p["ref_steady"], plain_stop_units=p["stop"]["units"] if p["stop"] else None,
                   plain_s=p["stop"]["seconds"] if p["stop"] else p["run_s"], plain_settled=p["stop"] is not None)
        cells = _lattice_cells(c)
        for name, (res, wall, info) in arms.items():
            r = res[k]
            s_per_lu = wall / max(info["lattice_updates"], 1)
            steps = r["steps"] + r.get("first_steps", 0)
            row[f"{name}_settled"] = r["stop"] is not None
            row[f"{name}_fallback"] = r.get("fallback", False)
            row[f"{name}_stop_units"] = r["stop"]["units"] if r["stop"] else None
            row[f"{name}_s_apportioned"] = s_per_lu * cells * steps
            if r["stop"] and np.isfinite(p["ref_cd"]):
                cd_err = (r["stop"]["cd"] - p["ref_cd"]) / abs(p["ref_cd"])
                st_err = 0.0 if p["ref_steady"] else ((r["stop"]["st"] - p["ref_st"]) / p["ref_st"]
                                                      if p["ref_st"] > 0 else float("nan"))
            else:
                cd_err = st_err = float("nan")
            row[f"{name}_cd_err"] = cd_err
            row[f"{name}_st_err"] = st_err
            row[f"{name}_within_tol"] = bool(abs(cd_err) <= tol and abs(st_err) <= tol)
        rows.append(row)
    plain_total = sum(r["plain_s"] for r in rows)

    def agg(name):
        res, wall, info = arms[name]
        sp = [r["plain_s"] / r[f"{name}_s_apportioned"] for r in rows]
        return dict(tunnels=len(rows), settled=sum(r[f"{name}_settled"] for r in rows),
                    within_tol=sum(r[f"{name}_within_tol"] for r in rows),
                    fallback=sum(r[f"{name}_fallback"] for r in rows),
                    wall_s=wall, aggregate_speedup_measured=plain_total / wall,
                    median_speedup_apportioned=float(np.median(sp)),
                    median_stop_units=float(np.median([r[f"{name}_stop_units"] or max_units for r in rows])),
                    max_abs_cd_err=float(np.nanmax([abs(r[f"{name}_cd_err"]) for r in rows])),
                    max_abs_st_err=float(np.nanmax([abs(r[f"{name}_st_err"]) for r in rows])),
                    info=info)

    summary = dict(tunnels=len(rows), plain_settled=sum(r["plain_settled"] for r in rows), plain_total_s=plain_total,
                   plain_median_stop_units=float(np.median([r["plain_stop_units"] or max_units for r in rows])),
                   rule=rule.__dict__, max_units=max_units, check_units=check_units, tol=tol,
                   **{name: agg(name) for name in arms})
    return dict(summary=summary, rows=rows)
