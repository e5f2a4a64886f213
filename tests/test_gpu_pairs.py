"""The multi-cell bulk kernels of the narrow storage formats (FP32, 16-bit) against the one-cell kernel.

With FP32 or 16-bit storage the bulk kernel updates 4 or 2 neighbouring cells per thread where the
row length allows: vector loads and stores of each population plane, the x-shifted planes
completed by a warp shuffle (and a memory read at the warp's edges and the periodic wrap), the
collision on packed FP32 pairs; where rows are whole 16-byte units it reads the planes from
shared-memory copies that asynchronous bulk copies fill (the bulk-copy-fed kernel). Every lane performs the one-cell kernel's operations, so all forms
must give bit-identical populations, on every link rule and on grids whose rows end inside a warp,
in the two-kernel and the staged step. The link kernel collides boundary nodes with the same
operators, so the schedules agree with each other bit for bit as well.
"""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


def _domains():
    from vortexlab_b200.workloads import disk_field
    return {
        # 640 cells per row: with 2 cells per thread one full 512-cell tile and one whose last four
        # warps are past the row end; with 4, one 1024-cell tile of which three warps are
        "disk_box_640x200": S.disk_box(640, 200, disk_field(640, 200, seed=11)),
        # 1000 cells per row: the last warp of 4-cell groups ends inside the row
        "disk_box_1000x96": S.disk_box(1000, 96, disk_field(1000, 96, seed=12)),
        # 122 cells per row (a row ends inside a warp), TRT, inlet, absorbing outlet, moving body
        "tunnel_like": S.tunnel_like(radiating=True),
        "tunnel_walls": S.tunnel_like(radiating=False),
        # 128 cells per row: whole 16-byte units in every format, so the bulk-copy-fed kernel runs
        # on every link rule
        "tunnel_128": S.tunnel_like(nx=128, radiating=True),
    }


def _aligned(d, prec):
    elem = {"f64": 8, "f32": 4, "f16s": 2, "f16c": 2, "f16x": 2}[prec]
    return d["nx"] * elem % 16 == 0


def _run(d, prec, schedule, cells, steps, copies=True, prefetch=0):
    sim = S.product_sim(d, precision=prec)
    if prec != "f64":
        sim.set_cells_per_thread(cells)
        sim.set_bulk_copies(copies)
    if prefetch:
        sim.set_prefetch_rows(prefetch)
    sim.schedule = schedule
    nx, ny = d["nx"], d["ny"]
    sim.record(steps)
    if d.get("periodic", (False, False)) == (True, True):
        sim.init(S.swirl(nx, ny))
        sim.step(steps)
    else:
        # the inlet ramp, a small oscillating body rotation and the absorbing outlet target, set
        # between chunks of 25 steps as the oracle parity test of this domain does
        sim.init((1.0, 0.05, 0.0))
        for k in range(steps // 25):
            v1 = 0.5 + 0.0125 * k
            sim.vscale[1] = v1
            sim.vscale[2] = 0.002 * np.sin(0.3 * k)
            sim.outflow_target = 0.05 * v1
            sim.step(25)
    return sim.populations(), sim.history()


@pytest.mark.parametrize("prec", ["f32", "f16s", "f16c", "f16x"])
@pytest.mark.parametrize("name", list(_domains().keys()))
def test_two_cell_kernel_matches_one_cell_kernel(gpu, prec, name):
    d = _domains()[name]
    steps = 150
    out = {}
    for schedule in ("concurrent", "staged"):
        for cells, copies in ((4, True), (4, False), (2, True), (2, False), (1, False)):
            out[(schedule, cells, copies)] = _run(d, prec, schedule, cells, steps, copies)
        if _aligned(d, prec):
            out[(schedule, 4, "prefetch")] = _run(d, prec, schedule, 4, steps, False, prefetch=7)
    ref_f, ref_h = out[("concurrent", 1, False)]
    assert np.isfinite(ref_f).all()
    bad = []
    for key, (f, h) in out.items():
        if not np.array_equal(f, ref_f):
            diff = np.nonzero(f != ref_f)
            bad.append(f"{key}: {len(diff[0])} populations differ (max {np.max(np.abs(f - ref_f)):.3g}; first at "
                       f"plane {diff[0][0]}, y {diff[1][0]}, x {diff[2][0]})")
        # the force of the staged step is summed per block of links (equal to rounding)
        if key[0] == "concurrent":
            if not np.array_equal(h[:, :2], ref_h[:, :2]):
                bad.append(f"{key}: force history differs")
        elif np.max(np.abs(h[:, :2] - ref_h[:, :2])) > 1e-12 * np.max(np.abs(ref_h[:, :2])):
            bad.append(f"{key}: force history beyond 1e-12")
    assert not bad, "; ".join(bad)


def test_odd_row_length_uses_the_one_cell_kernel(gpu):
    """A row of odd length cannot hold aligned pairs: the bulk kernel falls back to one cell per
    thread, and the two settings give the same result."""
    d = S.tunnel_like(nx=121, radiating=False)
    a, _ = _run(d, "f32", "staged", 2, 100)
    b, _ = _run(d, "f32", "staged", 1, 100)
    assert np.array_equal(a, b) and np.isfinite(a).all()


@pytest.mark.parametrize("name", ["disk_box_640x200", "tunnel_128"])
def test_prefetch_changes_nothing(gpu, name):
    """The L2 prefetch of later rows' tiles is a hint only: FP64 populations and forces are the same
    with and without it, in the two-kernel and the staged step."""
    d = _domains()[name]
    for schedule in ("concurrent", "staged"):
        a, ha = _run(d, "f64", schedule, 1, 100)
        b, hb = _run(d, "f64", schedule, 1, 100, prefetch=5)
        assert np.array_equal(a, b) and np.array_equal(ha, hb), schedule
