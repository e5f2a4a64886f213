"""Host-side logic of the product, checked without a GPU: the shared library loads and exports every
entry point of include/vortexlab.h; the host domain compiler produces link tables identical to the
oracle's (which reproduces the reference's published hashes); shapes and signal analysis agree with
the oracle bit for bit; contract violations are reported as errors; with no CUDA device every sim
constructor fails loudly (no CPU fallback)."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

import scenarios as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    out = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if name.endswith(".h"):
            text = open(os.path.join(ROOT, "include", name)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            out |= set(re.findall(r"\b(vl_[a-z0-9_]+)\s*\(", text))
    return out


def test_library_exports_every_declared_symbol(V):
    from vortexlab_b200 import _lib
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [s for s in sorted(declared_symbols()) if not hasattr(lib, s)]
    assert not missing, missing
    assert set(_lib.DECLARED) <= declared_symbols()
    assert V.lib.vl_abi_version() == 2


def test_no_cpu_fallback_without_a_device(V):
    if V.device_count() > 0:
        pytest.skip("a CUDA device is present")
    b = V.Builder(8, 8)
    b.periodic_x = b.periodic_y = True
    with pytest.raises(V.VortexError) as e:
        b.build()
    assert e.value.code == -2


def _domains():
    from vortexlab_b200.workloads import disk_field
    return {
        "disk_box": S.disk_box(256, 128, disk_field(256, 128, seed=3)),
        "tunnel_radiating": S.tunnel_like(radiating=True),
        "tunnel_walls": S.tunnel_like(radiating=False),
        "couette": S.couette(),
        "poiseuille_q08": S.poiseuille(16, q=0.8),
    }


@pytest.mark.parametrize("name", list(_domains().keys()))
def test_link_tables_match_oracle(V, O, name):
    d = _domains()[name]
    mine = S.product_builder(d).link_table()
    ref = S.oracle_sim(d).link_table()
    assert np.array_equal(mine["flags"], ref["flags"])
    assert np.array_equal(mine["bnode_idx"], ref["bnode_idx"])
    assert np.array_equal(mine["bnode_first"], ref["bnode_first"])
    assert np.array_equal(mine["link_i32"], ref["link_i32"])
    assert np.array_equal(mine["link_f64"], ref["link_f64"])  # q, cu6, u_w, rho bit for bit
    assert mine["npnodes"] == ref["npnodes"]


def test_channel_link_tables_match_oracle(V, O):
    """The Schafer-Turek rig at n = 20 (parabolic inlet, pressure outlet, curved body)."""
    n = 20
    nx, ny, h = 22 * n + 2, 41 * n // 10 + 2, float(41 * n // 10)
    xc = yc = 0.5 + 2.0 * n
    d = dict(nx=nx, ny=ny, tau=V.tau_for(0.05 * n / 100.0), collision=("trt", 3.0 / 16.0),
             kinds=[("wall", ("parabolic", 0.05, h), 1, None, None), ("pressure", 1.0), ("wall", None, 0, None, None),
                    ("wall", None, 2, 0, ("circle", xc, yc, 0.5 * n))],
             paint=[("rect", 0, 0, 0, ny - 1, 1), ("rect", nx - 1, nx - 1, 0, ny - 1, 2), ("rect", 1, nx - 2, 0, 0, 3),
                    ("rect", 1, nx - 2, ny - 1, ny - 1, 3), ("rect", 0, nx - 1, 0, 0, 3),
                    ("rect", 0, nx - 1, ny - 1, ny - 1, 3), ("shape", 4)])
    mine = S.product_builder(d).link_table()
    och, _, _, _ = O.cylinder_rig(n)
    ref = och.sim.link_table()
    for k in ("flags", "bnode_idx", "bnode_first", "link_i32", "link_f64"):
        assert np.array_equal(mine[k], ref[k]), k
    assert mine["npnodes"] == ref["npnodes"] == ny - 2


def test_shapes_match_oracle(V, O):
    rng = np.random.default_rng(5)
    pairs = [
        (V.Circle(0.3, -0.2, 7.1), O.Shape.circle(0.3, -0.2, 7.1)),
        (V.section(V.Corner.DoubleRecessed(0.1), 1.5, 0.5, 12.0, 0.3), O.Shape.section(4, 0.1, 1.5, 0.5, 12.0, 0.3)),
        (V.section(V.Corner.Rounded(0.2), 0.0, 0.0, 10.0, 0.0), O.Shape.section(2, 0.2, 0.0, 0.0, 10.0, 0.0)),
        (V.section(V.Corner.Chamfered(0.15), 0.0, 0.0, 10.0, 0.2), O.Shape.section(1, 0.15, 0.0, 0.0, 10.0, 0.2)),
        (V.Ellipse(0.0, 1.0, 8.0, 3.0), O.Shape.ellipse(0.0, 1.0, 8.0, 3.0)),
        (V.Translated(V.Circle(0, 0, 5.0), 1.0, 2.0), O.Shape.translated(O.Shape.circle(0, 0, 5.0), 1.0, 2.0)),
    ]
    for v, o in pairs:
        for _ in range(300):
            x, y = rng.uniform(-12, 12, 2)
            assert v.inside(x, y) == o.inside(x, y)
            dx, dy = rng.integers(-1, 2, 2)
            if (dx, dy) != (0, 0) and not v.inside(x, y) and v.inside(x + dx, y + dy):
                assert V.cut_fraction(v, x, y, float(dx), float(dy)) == o.cut_fraction(x, y, float(dx), float(dy))


def test_signal_matches_oracle(V, O):
    rng = np.random.default_rng(11)
    x = 0.3 + np.sin(0.05 * np.arange(5000)) + 0.01 * rng.standard_normal(5000)
    assert V.signal.dominant_frequency(x, 0.01) == O.dominant_frequency(x, 0.01)
    assert V.signal.peaks(x) == O.peaks(x)
    assert V.signal.crossing_frequency(x, 0.01) == O.crossing_frequency(x, 0.01)
    assert V.signal.mean(x) == O.mean(x) and V.signal.rms(x) == O.rms(x)
    assert V.signal.sample_at(x, 17.25) == O.sample_at(x, 17.25)
    re_, im_ = rng.standard_normal(64), rng.standard_normal(64)
    a, b = V.signal.fft(re_, im_), O.fft(re_, im_)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_series_stats_reports_strouhal_only_for_regular_oscillation(V):
    """src/cases/channel.rs:195-217."""
    dt = 0.01

    def wave(f, n):
        cl = 0.4 * np.sin(2 * np.pi * f * np.arange(n) * dt)
        return V.Series(dt, np.full(n, 1.5), cl)

    s = wave(0.16, 10000).stats(50.0)
    assert s.periodic and abs(s.st - 0.16) < 1e-3 and abs(s.st_crossings - 0.16) < 2e-3
    assert abs(s.cl_rms - 0.4 / math.sqrt(2)) < 5e-3 and abs(s.cd_mean - 1.5) < 1e-12
    s = wave(0.03, 10000).stats(50.0)
    assert not s.periodic and s.st == 0.0
    n = 5000
    drift = V.Series(dt, np.ones(n), (np.arange(n) / n) ** 2)
    assert not drift.stats(10.0).periodic
    s = V.Series(dt, np.ones(n), np.zeros(n)).stats(10.0)
    assert not s.periodic and s.st == 0.0 and s.cl_rms == 0.0


def test_contract_violations_are_errors(V):
    with pytest.raises(V.VortexError):
        V.Builder(2, 5)
    b = V.Builder(10, 10)
    b.tau = 0.5
    with pytest.raises(V.VortexError, match="tau"):
        b.link_table()
    b = V.Builder(10, 10)  # not periodic, no walls: fluid touches the edge
    with pytest.raises(V.VortexError, match="non-periodic edge"):
        b.link_table()
    b = V.Builder(10, 10)
    with pytest.raises(V.VortexError, match="vgroup"):
        b.add(V.Kind.Wall(V.Wall(vgroup=4)))
    with pytest.raises(V.VortexError, match="outline"):
        b.fill_shape(b.add_static_wall())


def test_disk_field_is_seeded_and_reaches_the_fraction():
    from vortexlab_b200.workloads import disk_field
    a = disk_field(1024, 512, seed=0x5EED0001)
    b = disk_field(1024, 512, seed=0x5EED0001)
    assert np.array_equal(a, b)
    x = np.arange(1024)[None, :]
    y = np.arange(512)[:, None]
    solid = np.zeros((512, 1024), dtype=bool)
    for cx, cy, r in a:
        solid |= (x - cx) ** 2 + (y - cy) ** 2 < r * r
    frac = solid.mean()
    assert 0.05 <= frac < 0.052
    assert np.all(a[:, 2] >= 4.0) and np.all(a[:, 2] <= 16.0)


@pytest.mark.parametrize("name", list(_domains().keys()))
def test_staged_step_lookup(V, name):
    """The staged bulk kernel finds a boundary cell's node and links from the row tile alone: the
    node's CSR rank is the warp slot's first rank plus the boundary cells before the lane, and the
    link of direction j is first + popc(mask below j). Replayed here on the host tables, for every
    boundary cell, with the kernel's tiling (256-cell row tiles, 32-cell warp slots)."""
    t = S.product_builder(_domains()[name]).link_table()
    flags, bidx, bfirst, dirs = t["flags"], t["bnode_idx"], t["bnode_first"], t["link_i32"][:, 0]
    ny, nx = flags.shape
    nb = len(bidx)
    mask = np.zeros(nb, dtype=np.int64)
    for k in range(nb):
        d = dirs[bfirst[k]:bfirst[k + 1]]
        assert np.all(np.diff(d) > 0) and d.min() >= 1 and d.max() <= 8
        mask[k] = np.bitwise_or.reduce(1 << d.astype(np.int64))
    flat = flags.reshape(-1)
    before = np.concatenate([[0], np.cumsum(flat == 1)])  # boundary cells before each cell
    tiles = (nx + 255) // 256
    seen = 0
    for y in range(ny):
        for w in range(tiles * 8):
            x0 = w * 32
            lanes = np.arange(x0, min(x0 + 32, nx))
            if len(lanes) == 0:
                continue
            first = before[y * nx + x0]
            row = flat[y * nx + lanes]
            for r, x in enumerate(lanes[row == 1]):
                k = first + r
                assert k < nb and bidx[k] == y * nx + x
                for j in range(1, 9):
                    if mask[k] >> j & 1:
                        l = bfirst[k] + bin(int(mask[k]) & ((1 << j) - 1)).count("1")
                        assert bfirst[k] <= l < bfirst[k + 1] and dirs[l] == j
                seen += 1
    assert seen == nb


@pytest.mark.parametrize("name", list(_domains().keys()))
def test_staged_split_point(V, name):
    """The staged step runs a part of its link blocks first, then the bulk tiles of the rows before
    the row of the node of the first link left to the second part, while that part runs. The split
    the library computes (vl_builder_stage_split, the same function the device sim uses) is checked
    on the host tables: every boundary node of those rows has all its links in the first part, and
    the rows after the split hold every node with a link in the second."""
    bld = S.product_builder(_domains()[name])
    sp = bld.stage_split()
    t = bld.link_table()
    flags, bidx, bfirst = t["flags"], t["bnode_idx"], t["bnode_first"]
    ny, nx = flags.shape
    nlinks = int(bfirst[-1])
    per = sp["links_per_block"]
    assert sp["link_blocks"] == max(1, (nlinks + per - 1) // per)
    if sp["split_blocks"] == 0:
        pytest.skip("the step is not split on this domain")
    assert 0 < sp["split_blocks"] < sp["link_blocks"] and 0 < sp["split_rows"] < ny
    lnode = np.repeat(np.arange(len(bidx)), np.diff(bfirst))
    first_b = sp["split_blocks"] * per
    row = sp["split_rows"]
    assert int(bidx[lnode[first_b]]) // nx == row
    rows = bidx // nx
    assert np.all(bfirst[1:][rows < row] <= first_b)
    assert np.all(rows[lnode[first_b:]] >= row)
