"""Precision study: the same runs with populations stored in FP64, FP32 and FP16 (shifted form
f_i - w_i), reporting the error of the force coefficients, the Strouhal number and the pressure
drop against the FP64 run.

The FP64 device path is bit-identical to the reference's CPU solver (the published state hashes
are reproduced), so the FP64 column is the reference's own result for these cases.

Cases:
  * Schafer-Turek 2D-2 (src/cases/cylinder.rs:169-220): cylinder at n cells per diameter,
    Re = 100, u_mean = 0.05, TRT 3/16, `units` convective units, statistics over the last
    `window` units (c_D max/min, c_L max/min, St, St from crossings, dP).
  * Square cylinder in the towing tank (src/cases/tunnel.rs:52-92): side d cells, Re = 150,
    u = 0.05, upstream 10 d, downstream 20 d, height 15 d, sound-absorbing sides; statistics of
    the force history after `discard` units (c_D mean/max, c_L max/rms, St).
"""
from __future__ import annotations

import time

import numpy as np

from . import cylinder, section, signal
from .tunnel import Tunnel

PRECISIONS = ("f64", "f32", "f16s", "f16c", "f16x")


def cylinder_2d2(n=80, units=100.0, window=20.0, precisions=PRECISIONS):
    out = {}
    for p in precisions:
        t0 = time.perf_counter()
        u = cylinder.run_2d2(cylinder.Setup(n=n, precision=p), units, window)
        out[p] = dict(cd_max=u.cd_max, cd_min=u.cd_min, cl_max=u.cl_max, cl_min=u.cl_min, st=u.st,
                      st_crossings=u.st_crossings, dp=u.dp, periods=u.periods, steps=u.steps,
                      seconds=time.perf_counter() - t0)
    return out


def square_tunnel(d=60, re=150.0, u=0.05, units=70.0, discard=40.0, precisions=PRECISIONS):
    out = {}
    for p in precisions:
        t0 = time.perf_counter()
        tn = Tunnel(d=d, re=re, u=u, upstream=10.0, downstream=20.0, height=15.0, precision=p)
        cx, cy = tn.centre()
        ch = tn.build(section((0, 0.0), cx, cy, float(d), 0.0))
        series = tn.run(ch, units)
        st = series.stats(discard)
        i0 = int(discard / series.dt)
        out[p] = dict(cd_mean=st.cd_mean, cd_max=float(np.max(series.cd[i0:])), cl_max=float(np.max(series.cl[i0:])),
                      cl_rms=st.cl_rms, st=st.st, st_crossings=st.st_crossings,
                      st_spectrum=float(signal.dominant_frequency(series.cl[i0:], series.dt)[0]),
                      periodic=st.periodic,
                      steps=len(series.cd), grid=tn.grid(), seconds=time.perf_counter() - t0)
        ch.close()
    return out


def relative_errors(table, ref="f64", keys=None):
    """{precision: {quantity: (value - ref) / |ref|}} for every non-reference precision."""
    base = table[ref]
    keys = keys or [k for k, v in base.items() if isinstance(v, float) and k != "seconds"]
    return {p: {k: (row[k] - base[k]) / abs(base[k]) if base[k] else float("nan") for k in keys}
            for p, row in table.items() if p != ref}


if __name__ == "__main__":
    import json
    import sys
    # python -m vortexlab_b200.precision [both|cylinder|square] [f64,f32,...]   (f64 always included)
    which = sys.argv[1] if len(sys.argv) > 1 else "both"
    precs = PRECISIONS
    if len(sys.argv) > 2:
        precs = tuple(["f64"] + [p for p in sys.argv[2].split(",") if p != "f64"])
    res = {}
    if which in ("both", "cylinder"):
        t = cylinder_2d2(precisions=precs)
        res["cylinder_2d2_n80"] = {"values": t, "rel_error_vs_f64": relative_errors(t)}
    if which in ("both", "square"):
        t = square_tunnel(precisions=precs)
        res["square_d60_re150"] = {"values": t, "rel_error_vs_f64": relative_errors(t)}
    print(json.dumps(res, indent=1, default=float))
