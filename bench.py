#!/usr/bin/env python
"""Throughput of the vortexlab D2Q9 time step on B200: MLUPS and fraction of the HBM roofline.

Workload (one step = one time step of the whole box, FP64 populations): the periodic 8192 x 4096
box with seeded solid disks filling 5 % of the cells (radii 4-16, seed 0x5EED0001), BGK
tau = 0.55, uniform start (rho, ux, uy) = (1, 0.05, 0); the force on the disks is summed every
step. 4.8 GB of populations per buffer pair, far larger than the 126 MB L2, so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vortexlab|reference]

Prints one JSON line. Under torchrun (N > 1) every rank runs its own replica of the box (the step
has no data exchange between replicas); the time is the max over ranks and `value` the job total.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BOX = dict(nx=8192, ny=4096, seed=0x5EED0001, fraction=0.05, tau=0.55, u=0.05)
BYTES_PER_LU = {"f64": 144, "f32": 72, "f16s": 36, "f16c": 36, "f16x": 36}
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes per node update of the bulk kernel from ncu, per (precision, staged):
# dram__bytes_read.sum + dram__bytes_write.sum of both launches of one staged step of the
# 4096 x 2048 box (7,968,653 fluid nodes; 624.1 MB read + 486.2 MB written, 1,110.3 MB), and of one
# launch of the two-kernel step on the 2048 x 2048 box (interior nodes), divided by the nodes the
# kernel updates; scaled to the headline box by nodes. Writes still dirty in L2 when a launch ends
# are not counted (up to the 126 MB L2, about 3 % of a 4096 x 2048 step). See
# profiles/k_bulk_dram_traffic_f64.md.
NCU_DRAM_BYTES_PER_LU = {("f64", False): 139.3, ("f64", True): 139.33}
NCU_TRAFFIC_SOURCE = {
    True: "ncu dram__bytes_read.sum + dram__bytes_write.sum of one staged step (both launches) of the 4096x2048 "
          "box, per fluid node, scaled by nodes",
    False: "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch on the 2048x2048 box, per interior "
           "node, scaled by nodes"}
# steps of the full-size parity check against the oracle (about 3 s of oracle time on 16 threads)
PARITY_STEPS = 20


def workload_name(prec):
    return (f"periodic box {BOX['nx']}x{BOX['ny']}, seeded disks {int(BOX['fraction'] * 100)}% solid "
            f"(r 4-16, seed 0x{BOX['seed']:X}), BGK tau={BOX['tau']}, u={BOX['u']}, {prec} populations")


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    INTERVAL_MS = 20

    def __init__(self, gpu_index):
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="vl_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.INTERVAL_MS)],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # wait (at most 5 s) for the first sample, so that the sampling covers what follows
        t0 = time.perf_counter()
        while self.proc is not None and time.perf_counter() - t0 < 5.0:
            self.f.flush()
            if os.path.getsize(self.path) > 0 or self.proc.poll() is not None:
                break
            time.sleep(0.01)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as fh:
            lines = fh.readlines()
        os.unlink(self.path)
        for line in lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 8:
                continue
            try:
                rows.append((float(p[0]), float(p[1]), p[4:8]))
            except ValueError:
                continue
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, _, r in rows for k in range(4) if r[k].lower() == "active"})
        loaded = [r[0] for r in rows if r[0] > 0.5 * r[1]] or [r[0] for r in rows]
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows), "interval_ms": self.INTERVAL_MS}


def dist_setup(world):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return dist


def dist_max(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_sum(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def _workloads():
    """The seeded workload generators (vortexlab_b200/workloads.py, numpy only), loaded from their
    file so that the CPU legs import nothing of the CUDA library."""
    import importlib.util
    name = "_vl_workloads_standalone"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "vortexlab_b200", "workloads.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules[name] = mod
    return sys.modules[name]


def box_config(prec, fluid, interior, links, bnodes, world):
    """The workload's description, identical in both arms."""
    return {"workload": workload_name(prec), "grid": [BOX["nx"], BOX["ny"]], "fluid_nodes": int(fluid),
            "interior_nodes": int(interior), "links": int(links), "boundary_nodes": int(bnodes),
            "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (populations 2 x 9 x 33.5M values), no flush needed"}


def oracle_box(threads):
    """The box on the oracle (the reference's FP64 CPU algorithm restated), at the uniform start."""
    import numpy as np

    import oracle as O
    nx, ny = BOX["nx"], BOX["ny"]
    disks = _workloads().disk_field(nx, ny, BOX["seed"], BOX["fraction"])
    b = O.Builder(nx, ny)
    b.periodic_x = b.periodic_y = True
    b.tau = BOX["tau"]
    b.collision = O.BGK
    k = b.add_wall(fgroup=0, shape=O.Shape.disks(disks))
    b.fill_shape(k)
    sim = b.build(threads)
    sim.init((np.ones((ny, nx)), np.full((ny, nx), BOX["u"]), np.zeros((ny, nx))))
    return sim


def time_oracle(sim, threads, max_steps, budget_s):
    """Times the oracle on `threads` host threads (row-split pool, serial link pass, as the
    reference's pool): one untimed step, then as many full steps as fit the budget (at most
    max_steps)."""
    sim.set_threads(threads)
    t0 = time.perf_counter()
    sim.step(1)
    one = time.perf_counter() - t0
    steps = int(max(1, min(max_steps, budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    sim.step(steps)
    secs = time.perf_counter() - t0
    return sim.fluid_nodes() * steps / secs / 1e6, steps, secs


def box_parity(sim, pops, hist, steps, osim):
    """The full box after `steps` steps from the uniform start on the device (populations `pops`,
    per-step force `hist`) against the oracle run from the same start: state hash (FNV-1a over
    every fluid population, src/sim.rs:654-668), largest population difference, and the force of
    every step relative to the largest oracle force."""
    import numpy as np
    t0 = time.perf_counter()
    fo = np.zeros((steps, 2))
    for k in range(steps):
        osim.step(1)
        fo[k] = osim.force[0]
    ref = osim.populations().reshape(-1)
    max_abs = 0.0
    chunk = 1 << 24
    for i in range(0, ref.size, chunk):
        max_abs = max(max_abs, float(np.max(np.abs(ref[i:i + chunk] - pops[i:i + chunk]))))
    del ref
    hg, ho = sim.state_hash(), osim.state_hash()
    fg = hist[:steps, :2]
    force_rel = float(np.max(np.abs(fg - fo)) / max(np.max(np.abs(fo)), 1e-300))
    return {"steps": steps, "state_hash_gpu": f"{hg:016x}", "state_hash_oracle": f"{ho:016x}",
            "hash_equal": hg == ho, "max_abs_pop": max_abs, "force_rel": force_rel,
            "bars": "populations 1e-10 absolute (bit-identical expected), force 1e-9 relative",
            "ok": bool(max_abs <= 1e-10 and force_rel <= 1e-9),
            "seconds": round(time.perf_counter() - t0, 1)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import numpy as np
    threads = os.cpu_count() or 1
    sim = oracle_box(threads)
    flags = sim.flags()
    interior = int(np.count_nonzero(flags == 0))
    warm = max(args.warmup, 0)
    t0 = time.perf_counter()
    sim.step(max(warm, 1))
    one = (time.perf_counter() - t0) / max(warm, 1)
    # every timed step is a full step of the box; at most about two minutes of them
    steps = int(max(1, min(args.steps, 120.0 / max(one, 1e-6))))
    t0 = time.perf_counter()
    sim.step(steps)
    secs = time.perf_counter() - t0
    mlups = sim.fluid_nodes() * steps / secs / 1e6
    sample = f"{steps} full steps of the {BOX['nx']}x{BOX['ny']} box after {max(warm, 1)} untimed ({secs:.1f} s)"
    line = {
        "impl": "reference", "metric": "MLUPS", "value": round(mlups, 2), "unit": "MLUPS", "n_gpus": args.gpus,
        "steps": steps, "warmup": max(warm, 1), "ms_per_step": round(1e3 * secs / steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": box_config("f64", sim.fluid_nodes(), interior, sim.link_count(), sim.bnode_count(), args.gpus),
        "run": {"threads": threads, "code": "oracle/liboracle.so: the reference's FP64 CPU step restated in C++ "
                                            "(row-split thread pool, serial link pass)"},
        "cpu_baseline": {"value": round(mlups, 2), "unit": "MLUPS", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(mlups, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def channel_n80(V):
    """The reference's own benchmark (`vortexlab bench --n 80 --steps 1000`): MLUPS and state hash,
    checked against the hash it publishes (tests/golden/published.json)."""
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "published.json")) as f:
        want = set(json.load(f)["bench_state_hashes"]["1762x330"]["hashes"].values())
    ch, secs = V.cylinder.bench(V.cylinder.Setup(n=80), 1000)
    h = ch.sim.state_hash()
    out = {"grid": f"{ch.sim.nx}x{ch.sim.ny}", "fluid_nodes": ch.sim.fluid_nodes(), "steps": 1000,
           "mlups": round(ch.sim.fluid_nodes() * 1000 / secs / 1e6, 1), "ms_per_step": round(secs * 1e3 / 1000, 5),
           "state_hash": f"{h:016x}", "published_hash_match": {f"{h:016x}"} == want}
    ch.close()
    return out


def batched_256(global_steps=1000):
    """The batched configuration: 256 seeded tunnels (seed 0x5EED0004: ellipses, notched squares,
    star-convex polygons, D 15-60, Re 50-200, 20 D x 10 D, TRT), FP32 storage, one batch; the
    first `global_steps` global steps after the tile autotuner, device-timed (CUDA events around
    the run on its stream). Roofline of the whole step (bulk and link kernels) at 72 B per fluid
    node update."""
    from vortexlab_b200.convergence import throughput
    r = throughput(max_steps=global_steps)
    peak, peak_kind = hbm_peak()
    achieved = r["mlups"] * 1e6 * BYTES_PER_LU["f32"] / 1e9
    return {"workload": "256 seeded tunnels (seed 0x5EED0004), D 15-60, Re 50-200, TRT, f32 populations, "
                        f"first {r['global_steps']} global steps",
            "mlups": round(r["mlups"], 1), "seconds": round(r["seconds"], 4),
            "lattice_updates": int(r["lattice_updates"]), "tile": r["tile"], "schedule": r["schedule"],
            "cells_per_thread": r["cells_per_thread"], "launches": int(r["launches"]),
            "diverged": r["diverged"],
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                         "kernel": "whole batched step (bulk and link kernels)", "bytes_per_node_update": 72}}


def time_to_converged():
    """The second half of the headline metric on a bounded sample: time to converged c_D and St of
    the fast form (FP32, batched, learned warm start with the shipped network, uniform-start
    fallback) and of the batched form from a uniform start, against the plain FP64 GPU path (one
    tunnel at a time), on 8 held-out tunnels (D <= 22, Re >= 100). Every run stops on-line when its
    own trailing windows have settled (vortexlab_b200/online.py); every tunnel is counted."""
    import numpy as np

    from vortexlab_b200 import online as OL
    from vortexlab_b200 import warmstart as WS
    from vortexlab_b200.batch import seeded_tunnels
    cases = [c for c in seeded_tunnels(seed=WS.TEST_SEED, count=256, units=100.0)
             if c.params["d"] <= 22 and c.params["re"] >= 100.0][:8]
    net = WS.load_pretrained()          # resident network: buffers allocated, kernels loaded
    WS.predict(net, np.zeros((1, WS.H, WS.W, WS.CIN), np.float32))
    t0 = time.perf_counter()
    out = OL.comparison(cases, net)
    s = out["summary"]

    def arm(a):
        keep = ("settled", "within_tol", "fallback", "wall_s", "aggregate_speedup_measured",
                "median_speedup_apportioned", "median_stop_units", "max_abs_cd_err", "max_abs_st_err")
        return {k: (float(f"{a[k]:.4g}") if isinstance(a[k], float) else a[k]) for k in keep}
    return {"sample": "8 held-out tunnels of seed 0x5EED0004 with D <= 22 and Re >= 100, at most 100 convective units",
            "stopping": "on-line, from each run's own history: 3 trailing windows of 3 shedding periods agree "
                        "within 0.2 % on mean c_D and St",
            "accuracy": "fast-arm statistics at its stop within 0.5 % of the plain FP64 run's last window",
            "plain_settled": s["plain_settled"], "plain_total_s": round(s["plain_total_s"], 3),
            "fast_form": arm(s["warm"]), "uniform_start_batched": arm(s["cold"]),
            "seconds": round(time.perf_counter() - t0, 1)}


def bulk_roofline(prec, staged, fluid, interior, steps, link_ms, bulk_ms, total_ms):
    """Roofline of the dominant kernel, the bulk kernel: pull + collide of the interior nodes, or of
    every fluid node in the staged step (whose first kernel only evaluates the link rules)."""
    peak, peak_kind = hbm_peak()
    bpl = BYTES_PER_LU[prec]
    bulk_nodes = fluid if staged else interior
    achieved = bulk_nodes * bpl / (bulk_ms * 1e-3 / steps) / 1e9
    traffic = NCU_DRAM_BYTES_PER_LU.get((prec, staged))
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
            "traffic": None if traffic is None else round(traffic * bulk_nodes),
            "traffic_source": None if traffic is None else NCU_TRAFFIC_SOURCE[staged],
            "kernel": ("k_bulk (staged: all fluid nodes; both launches of a step, with the second link "
                       "part beside them)") if staged else "k_bulk (interior nodes)",
            "bytes_per_node_update": bpl,
            "algorithmic_bytes_per_launch": bulk_nodes * bpl,
            "kernel_ms_per_launch": round(bulk_ms / steps, 4),
            "link_kernel_ms_per_launch": round(link_ms / steps, 4),
            "bulk_share": round(bulk_ms / max(bulk_ms + link_ms, 1e-12), 4),
            "step_frac_of_peak": round(fluid * bpl / (total_ms * 1e-3 / steps) / 1e9 / peak, 4)}


def box_variant(V, prec, steps, warmup):
    """The same box with populations stored in `prec` (the narrower storage of the fast form):
    MLUPS and the bulk kernel's roofline, device-timed like the headline."""
    import numpy as np

    from vortexlab_b200.workloads import build_disk_box, disk_field
    disks = disk_field(BOX["nx"], BOX["ny"], BOX["seed"], BOX["fraction"])
    sim = build_disk_box(V, BOX["nx"], BOX["ny"], disks, tau=BOX["tau"], precision=prec)
    interior = int(np.count_nonzero(sim.flags() == 0))
    fluid = sim.fluid_nodes()
    sim.init((1.0, BOX["u"], 0.0))
    tune = sim.autotune(8)
    sim.step(max(warmup, 3))
    sim.synchronize()
    link_ms, bulk_ms, total_ms = sim.step_profiled(steps)
    out = {"workload": workload_name(prec), "steps": steps, "schedule": sim.schedule,
           "autotune_ms_per_step": tune, "mlups": round(fluid * steps / (total_ms * 1e-3) / 1e6, 1),
           "ms_per_step": round(total_ms / steps, 4),
           "roofline": bulk_roofline(prec, sim.schedule == "staged", fluid, interior, steps, link_ms, bulk_ms,
                                     total_ms),
           "finite": bool(np.isfinite(sim.force).all())}
    sim.close()
    return out


def run_vortexlab(args):
    import numpy as np

    import vortexlab_b200 as V
    from vortexlab_b200.workloads import build_disk_box, disk_field
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = dist_setup(world)
    V.set_device(local)
    prec = args.precision
    nx, ny = BOX["nx"], BOX["ny"]
    t0 = time.perf_counter()
    disks = disk_field(nx, ny, BOX["seed"], BOX["fraction"])
    sim = build_disk_box(V, nx, ny, disks, tau=BOX["tau"], precision=prec)
    setup_s = time.perf_counter() - t0
    flags = sim.flags()
    interior = int(np.count_nonzero(flags == 0))
    fluid = sim.fluid_nodes()
    sim.init((1.0, BOX["u"], 0.0))
    if prec != "f64" and args.cells:
        sim.set_cells_per_thread(args.cells)
    if prec != "f64" and args.bulk_copies:
        sim.set_bulk_copies(True)
    if args.prefetch >= 0:
        sim.set_prefetch_rows(args.prefetch)
    tune = sim.autotune(8) if args.schedule == "auto" else None
    if args.schedule != "auto":
        sim.schedule = args.schedule
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    gpu_index = vis.split(",")[local] if vis and len(vis.split(",")) > local else local
    n = nx * ny
    rho_h, ux_h, uy_h, pops_h = (V.PinnedArray(n), V.PinnedArray(n), V.PinnedArray(n), V.PinnedArray(9 * n))
    rho_h.array[:] = 1.0
    ux_h.array[:] = BOX["u"]
    uy_h.array[:] = 0.0
    sim.synchronize()
    # clocks are sampled from the warm-up through the timed region and the end-to-end run
    sampler = ClockSampler(gpu_index)
    sim.step(max(args.warmup, 3))
    sim.synchronize()
    if dist:
        dist.barrier()
    sim.synchronize()
    launches0 = sim.launch_count()
    link_ms, bulk_ms, total_ms = sim.step_profiled(args.steps)
    launches = sim.launch_count() - launches0
    sim.synchronize()
    if dist:
        dist.barrier()
    total_ms_max = dist_max(dist, total_ms)
    secs = total_ms_max * 1e-3
    value = world * fluid * args.steps / secs / 1e6
    staged = sim.schedule == "staged"
    roofline = bulk_roofline(prec, staged, fluid, interior, args.steps, link_ms, bulk_ms, total_ms)

    # end to end through the public API with host buffers: upload the start field from pinned host
    # memory, run the steps with the per-step force recorded on the device, download the force
    # history and the final populations.
    sim.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    sim.init((rho_h.array.reshape(ny, nx), ux_h.array.reshape(ny, nx), uy_h.array.reshape(ny, nx)))
    sim.record(args.steps)
    sim.step(args.steps)
    hist = sim.history()
    sim.populations(out=pops_h.array)
    e2e_s = time.perf_counter() - t0
    clocks = sampler.stop()
    e2e_s = dist_max(dist, e2e_s)
    e2e_value = world * fluid * args.steps / e2e_s / 1e6
    h2d = 3 * n * 8
    d2h = hist.nbytes + 9 * n * 8
    finite = bool(np.isfinite(hist[:, :2]).all())
    if clocks is not None:
        clocks["window"] = "warm-up, timed region and end-to-end run"

    line = {
        "metric": "MLUPS", "value": round(value, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(total_ms_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": prec, "data": "synthetic",
        "config": box_config(prec, fluid, interior, sim.link_count(), sim.bnode_count(), world),
        "run": {"timing": "CUDA events around every kernel on the stream it runs on, max over ranks",
                "schedule": sim.schedule, "autotune_ms_per_step": tune, "setup_s": round(setup_s, 2),
                "cells_per_thread": (args.cells or "default") if prec != "f64" else 1,
                "bulk_copies": prec != "f64" and args.bulk_copies, "prefetch_rows": args.prefetch if args.prefetch >= 0 else "default"},
        "roofline": roofline,
        "e2e": {"value": round(e2e_value, 1), "unit": "MLUPS", "h2d_bytes_per_step": round(h2d / args.steps),
                "d2h_bytes_per_step": round(d2h / args.steps), "seconds": round(e2e_s, 4),
                "path": "Sim.init(host field) + Sim.record + Sim.step + Sim.history + Sim.populations",
                "force_finite": finite},
        "gpu_launches": int(dist_sum(dist, launches)),
        "clocks": clocks,
    }
    osim = None
    threads = os.cpu_count() or 1
    if rank == 0 and world == 1 and not args.no_parity and prec == "f64":
        # the full box against the oracle: PARITY_STEPS steps from the uniform start on both
        osim = oracle_box(threads)
        ps = PARITY_STEPS
        sim.init((1.0, BOX["u"], 0.0))
        sim.record(ps)
        sim.step(ps)
        ph = sim.history()
        sim.populations(out=pops_h.array)
        line["parity"] = box_parity(sim, pops_h.array, ph, ps, osim)
        line["parity"]["schedule"] = sim.schedule
    del rho_h, ux_h, uy_h, pops_h
    sim.close()
    if rank == 0 and world == 1 and not args.no_extras:
        line["precision_f32"] = box_variant(V, "f32", args.steps, args.warmup)
        line["precision_f16s"] = box_variant(V, "f16s", args.steps, args.warmup)
        line["batched_256"] = batched_256()
        line["channel_n80"] = channel_n80(V)
        line["time_to_converged"] = time_to_converged()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if osim is None:
            osim = oracle_box(threads)
        mlups, steps, secs = time_oracle(osim, threads, 50, budget_s=15.0)
        m1, s1, t1 = time_oracle(osim, 1, 20, budget_s=8.0)
        line["cpu_baseline"] = {"value": round(mlups, 2), "unit": "MLUPS", "cores": threads, "kind": "port",
                                "sample": f"{steps} full steps of the same box after 1 untimed step ({secs:.1f} s)",
                                "single_thread": {"value": round(m1, 2), "cores": 1,
                                                  "sample": f"{s1} full steps after 1 untimed step ({t1:.1f} s)"}}
    del osim
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["vortexlab", "reference"], default="vortexlab")
    ap.add_argument("--precision", choices=["f64", "f32", "f16s", "f16c", "f16x"], default="f64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--schedule", default="auto", choices=["auto", "concurrent", "links-first", "bulk-first", "staged"])
    ap.add_argument("--box", default=None, help="NXxNY: a smaller box of the same kind (profiling cases)")
    ap.add_argument("--bulk-copies", action="store_true",
                    help="narrow storage: stream the bulk kernel's loads through shared memory (Sim.set_bulk_copies)")
    ap.add_argument("--prefetch", type=int, default=-1,
                    help="rows ahead the bulk kernel's blocks prefetch into the L2 (Sim.set_prefetch_rows; "
                         "-1: the library's default)")
    ap.add_argument("--cells", type=int, default=0, choices=[0, 1, 2, 4],
                    help="narrow storage: the most bulk cells per thread (Sim.set_cells_per_thread; 0: the "
                         "library's default)")
    args = ap.parse_args()
    if args.box:
        nx, ny = (int(v) for v in args.box.lower().split("x"))
        BOX.update(nx=nx, ny=ny)
    if args.impl == "reference":
        return run_reference(args)
    return run_vortexlab(args)


if __name__ == "__main__":
    sys.exit(main())
