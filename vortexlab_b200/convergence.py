"""Time to a converged drag coefficient and Strouhal number: a tunnel run the plain way (FP64,
one tunnel at a time, uniform start) against the fast form (FP32 storage, all tunnels in one
batch, optionally a learned warm start).

Statistics of a trailing window of three shedding periods (the period from the lift spectrum of
the FP64 run's last 10 convective units, src/signal.rs:92-107): the window's mean c_D and its
Strouhal number from lift mean-crossings (src/signal.rs:127-140). Reference values: those
statistics over the last window of the FP64 run. A run has converged at step t when every window
ending at t or later (checked every half period) is within `tol` (0.5 %) of the reference on both.
"""
from __future__ import annotations

import time
import numpy as np

from . import signal


def window_steps(cl, dt, units=10.0, periods=3.0):
    """Window length in steps: `periods` shedding periods from the lift spectrum of the last
    `units` convective units; None if the lift does not oscillate."""
    n = min(len(cl), int(units / dt))
    if n < 4 or not np.all(np.isfinite(cl[-n:])):
        return None
    f = signal.dominant_frequency(cl[-n:], dt)[0]
    if not (f > 0 and np.isfinite(f)):
        return None
    return min(len(cl), int(periods / f / dt))


def window_stats(cd, cl, dt, end, win):
    cdw, clw = cd[end - win:end], cl[end - win:end]
    return float(np.mean(cdw)), float(signal.crossing_frequency(clw, dt) or 0.0)


def reference_values(cd, cl, dt):
    """(c_D, St, window) over the last window of a run."""
    win = window_steps(cl, dt)
    if win is None:
        return float("nan"), float("nan"), None
    cd_ref, st_ref = window_stats(cd, cl, dt, len(cd), win)
    return cd_ref, st_ref, win


def convergence_step(cd, cl, dt, cd_ref, st_ref, win, tol=0.005):
    """Earliest step from which every trailing window (ending there or later, every half
    period) is within `tol` of the reference on both c_D and St; -1 if never."""
    if win is None or not (st_ref > 0 and np.isfinite(st_ref) and np.isfinite(cd_ref)):
        return -1
    hop = max(1, win // 6)
    ends = list(range(win, len(cd) + 1, hop))
    if ends[-1] != len(cd):
        ends.append(len(cd))
    ok = []
    for e in ends:
        c, st = window_stats(cd, cl, dt, e, win)
        ok.append(abs(c - cd_ref) <= tol * abs(cd_ref) and abs(st - st_ref) <= tol * st_ref)
    bad = [i for i, v in enumerate(ok) if not v]
    if not bad:
        return ends[0]
    if bad[-1] == len(ok) - 1:
        return -1
    return ends[bad[-1] + 1]


def plain_runs(cases, tol=0.005):
    """FP64 single-tunnel runs (uniform start), one after the other, each with the fastest of the
    step schedules for its grid (timed on its start state before the timed run; every schedule
    gives the same populations). Returns per-case dicts with the reference values, steps to
    convergence, the wall time of the run and the schedule used."""
    out = []
    for c in cases:
        tn = c.tunnel
        tn.precision = "f64"
        ch = tn.build(c.body)
        ch.sim.autotune(4)
        ch.sim.record(c.steps)
        t0 = time.perf_counter()
        ch.step(c.steps)
        h = ch.sim.history()
        wall = time.perf_counter() - t0
        k = 2.0 / (ch.u_ref * ch.u_ref * tn.d)
        cd, cl = k * h[:, 0], k * h[:, 1]
        dt = 1.0 / tn.steps_per_unit()
        cd_ref, st_ref, win = reference_values(cd, cl, dt)
        conv = convergence_step(cd, cl, dt, cd_ref, st_ref, win, tol)
        out.append(dict(cd_ref=cd_ref, st_ref=st_ref, win=win, conv_steps=conv, steps=c.steps, wall_s=wall,
                        ms_per_step=1e3 * wall / c.steps, dt=dt, d=tn.d, schedule=ch.sim.schedule))
        ch.close()
    return out


def batched_run(cases, refs, precision="f32", tol=0.005, warm=None, autotune=True):
    """All cases in one batch. With `warm` (a trained warmstart.UNet) every tunnel runs in its warm
    form (no ramp, no twist) from the network's prediction; the inference and upload time is
    counted in the wall time. Returns (per-case dicts, total wall seconds, batch info)."""
    from .batch import Batch
    t_init = 0.0
    if warm is not None:
        from .warmstart import warm_batch
        b, t_init = warm_batch(warm, cases, precision)
    else:
        b = Batch(precision)
        for c in cases:
            b.add(c.tunnel.spec(c.body), c.steps)
        b.build()
    tune = b.autotune(3) if autotune else None
    t0 = time.perf_counter()
    b.run()
    wall = time.perf_counter() - t0 + t_init
    out = []
    total_lu = 0
    for k, c in enumerate(cases):
        h = b.force_history(k)
        tn = c.tunnel
        kk = 2.0 / (tn.u * tn.u * tn.d)
        cd, cl = kk * h[:, 0], kk * h[:, 1]
        dt = 1.0 / tn.steps_per_unit()
        r = refs[k]
        conv = convergence_step(cd, cl, dt, r["cd_ref"], r["st_ref"], r["win"], tol)
        cd_f, st_f = window_stats(cd, cl, dt, len(cd), r["win"]) if r["win"] else (float("nan"), float("nan"))
        info = b.info(k)
        total_lu += info["fluid_nodes"] * c.steps
        out.append(dict(conv_steps=conv, cd_final=cd_f, st_final=st_f,
                        cd_err=(cd_f - r["cd_ref"]) / abs(r["cd_ref"]),
                        st_err=(st_f - r["st_ref"]) / r["st_ref"] if r["st_ref"] else float("nan")))
    binfo = dict(tile=b.tile, autotune_ms_per_step=tune, device_ms=b.last_run_ms(), launches=b.launch_count(),
                 mlups=total_lu / (b.last_run_ms() * 1e-3) / 1e6, init_s=t_init)
    b.close()
    return out, wall, binfo


def study(subset=32, seed=0x5EED0004, count=256, precision="f32", tol=0.005):
    """Plain FP64 runs of a subset of the seeded tunnels against the same tunnels in one batch.
    Wall time to convergence: steps to convergence x the run's cost per lattice update (the plain
    run's own, or the batch's total wall time divided by its total lattice updates)."""
    from .batch import seeded_tunnels
    cases = seeded_tunnels(seed=seed, count=count)
    pick = cases[:: max(1, count // subset)][:subset]
    refs = plain_runs(pick, tol=tol)
    fast, wall, binfo = batched_run(pick, refs, precision=precision, tol=tol)
    rows = []
    for c, r, f in zip(pick, refs, fast):
        lu_cost_plain = r["wall_s"] / r["steps"]            # seconds per step of this tunnel alone
        row = dict(kind=c.kind, d=c.params["d"], re=round(c.params["re"], 1), steps=c.steps,
                   cd_ref=r["cd_ref"], st_ref=r["st_ref"], plain_conv_steps=r["conv_steps"],
                   fast_conv_steps=f["conv_steps"], cd_err=f["cd_err"], st_err=f["st_err"],
                   plain_s_to_conv=lu_cost_plain * r["conv_steps"] if r["conv_steps"] >= 0 else None)
        rows.append(row)
    # batch cost per lattice update
    total_lu = sum(c.tunnel.grid()[0] * c.tunnel.grid()[1] * c.steps for c in pick)
    s_per_lu = wall / total_lu
    for c, row in zip(pick, rows):
        nx, ny = c.tunnel.grid()
        row["fast_s_to_conv"] = s_per_lu * nx * ny * row["fast_conv_steps"] if row["fast_conv_steps"] >= 0 else None
        if row["plain_s_to_conv"] and row["fast_s_to_conv"]:
            row["speedup"] = row["plain_s_to_conv"] / row["fast_s_to_conv"]
    ok = [r for r in rows if r.get("speedup")]
    summary = dict(tunnels=len(rows), converged_both=len(ok),
                   median_speedup=float(np.median([r["speedup"] for r in ok])) if ok else None,
                   aggregate_speedup=(sum(r["plain_s_to_conv"] for r in ok) / sum(r["fast_s_to_conv"] for r in ok))
                   if ok else None,
                   max_abs_cd_err=float(max(abs(r["cd_err"]) for r in rows)),
                   max_abs_st_err=float(max(abs(r["st_err"]) for r in rows)),
                   plain_total_s=sum(r["wall_s"] for r in refs), batch_wall_s=wall, batch=binfo)
    return dict(summary=summary, rows=rows)


def warm_comparison(net, cases, refs=None, precision="f32", tol=0.005):
    """Time to converged c_D and St for the plain form (FP64, one tunnel at a time, uniform start),
    the batched form from a uniform start and the batched form from the network's warm start.
    Wall time of a batched tunnel: its steps to convergence x its cells x the batch's seconds per
    cell update (inference and upload included for the warm form)."""
    refs = refs if refs is not None else plain_runs(cases, tol=tol)
    arms = {}
    for name, w in (("cold", None), ("warm", net)):
        res, wall, binfo = batched_run(cases, refs, precision=precision, tol=tol, warm=w)
        total = sum(c.tunnel.grid()[0] * c.tunnel.grid()[1] * c.steps for c in cases)
        arms[name] = (res, wall / total, binfo)
    rows = []
    for k, (c, r) in enumerate(zip(cases, refs)):
        nx, ny = c.tunnel.grid()
        row = dict(kind=c.kind, d=c.params["d"], re=round(c.params["re"], 1), steps=c.steps, cd_ref=r["cd_ref"],
                   st_ref=r["st_ref"], plain_conv_steps=r["conv_steps"], plain_schedule=r["schedule"],
                   plain_s=r["wall_s"] / r["steps"] * r["conv_steps"] if r["conv_steps"] >= 0 else None)
        for name, (res, s_lu, _) in arms.items():
            f = res[k]
            row[f"{name}_conv_steps"] = f["conv_steps"]
            row[f"{name}_cd_err"] = f["cd_err"]
            row[f"{name}_st_err"] = f["st_err"]
            row[f"{name}_s"] = s_lu * nx * ny * f["conv_steps"] if f["conv_steps"] >= 0 else None
        rows.append(row)

    def agg(name):
        ok = [r for r in rows if r["plain_s"] and r[f"{name}_s"]]
        if not ok:
            return dict(converged=0)
        sp = [r["plain_s"] / r[f"{name}_s"] for r in ok]
        steps = [r[f"{name}_conv_steps"] / r["plain_conv_steps"] for r in ok]
        return dict(converged=len(ok), median_speedup=float(np.median(sp)),
                    aggregate_speedup=sum(r["plain_s"] for r in ok) / sum(r[f"{name}_s"] for r in ok),
                    median_step_ratio=float(np.median(steps)),
                    max_abs_cd_err=float(max(abs(r[f"{name}_cd_err"]) for r in ok)),
                    max_abs_st_err=float(max(abs(r[f"{name}_st_err"]) for r in ok)))

    schedules = {}
    for r in rows:
        schedules[r["plain_schedule"]] = schedules.get(r["plain_schedule"], 0) + 1
    summary = dict(tunnels=len(rows), plain_converged=sum(1 for r in rows if r["plain_s"]),
                   plain_schedules=schedules, cold=agg("cold"), warm=agg("warm"),
                   batch={n: a[2] for n, a in arms.items()})
    return dict(summary=summary, rows=rows)


def throughput(seed=0x5EED0004, count=256, precision="f32", max_steps=0, schedule="concurrent", cells=2,
               prefetch=-1):
    """The full seeded batch: MLUPS of the whole run (or of its first `max_steps` global steps).
    `cells`: bulk cells per thread (2: the two-cell kernel where every row length is even);
    `prefetch`: L2 prefetch distance in tiles (-1: the library default)."""
    from .batch import Batch, seeded_tunnels
    cases = seeded_tunnels(seed=seed, count=count, precision=precision)
    b = Batch(precision)
    t0 = time.perf_counter()
    for c in cases:
        b.add(c.tunnel.spec(c.body), c.steps)
    b.build()
    setup = time.perf_counter() - t0
    b.schedule = schedule
    b.set_cells_per_thread(cells)
    if prefetch >= 0:
        b.set_prefetch_tiles(prefetch)
    tune = b.autotune(3)
    b.run(max_steps)
    ms = b.last_run_ms()
    lu = 0
    for k, c in enumerate(cases):
        t, nonfinite, _ = b.status(k)
        lu += b.info(k)["fluid_nodes"] * t
    out = dict(tunnels=count, precision=precision, global_steps=b.global_step(), lattice_updates=lu,
               seconds=ms * 1e-3, mlups=lu / (ms * 1e-3) / 1e6, tile=b.tile, schedule=schedule, cells_per_thread=cells,
               prefetch_tiles=prefetch, autotune_ms_per_step=tune,
               setup_s=setup, launches=b.launch_count(),
               diverged=[k for k in range(count) if b.status(k)[1]])
    b.close()
    return out


if __name__ == "__main__":
    import json
    import sys
    what = sys.argv[1] if len(sys.argv) > 1 else "study"
    # python -m vortexlab_b200.convergence throughput [max_steps schedule precision cells prefetch count]
    if what == "throughput":
        print(json.dumps(throughput(max_steps=int(sys.argv[2]) if len(sys.argv) > 2 else 0,
                                    schedule=sys.argv[3] if len(sys.argv) > 3 else "concurrent",
                                    precision=sys.argv[4] if len(sys.argv) > 4 else "f32",
                                    cells=int(sys.argv[5]) if len(sys.argv) > 5 else 2,
                                    prefetch=int(sys.argv[6]) if len(sys.argv) > 6 else -1,
                                    count=int(sys.argv[7]) if len(sys.argv) > 7 else 256), default=float))
    else:
        print(json.dumps(study(subset=int(sys.argv[2]) if len(sys.argv) > 2 else 32), default=float, indent=1))
