"""Batched tunnels: a tunnel advanced in a batch with others of other sizes, shapes and Reynolds
numbers matches the same tunnel run alone (state and per-step force) bit for bit, in every tile
shape, kernel schedule and storage format; autotuning does not perturb the run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases(V):
    from vortexlab_b200.batch import seeded_tunnels
    cases = seeded_tunnels(seed=99, count=4, dmin=8, dmax=14, units=3.0)
    return cases


@pytest.mark.parametrize("prec", ["f64", "f32", "f16s", "f16x"])
def test_batched_tunnels_match_single_runs(gpu, prec):
    """Every tile shape and schedule, and for the narrow formats both bulk forms (two cells per
    thread, one): the batched tunnel's populations and force history are bit-identical to the
    tunnel run alone (FP64: the reference's operation order; FP32 / 16-bit: the explicit FP32
    operators that every narrow kernel shares)."""
    V = gpu
    from vortexlab_b200.batch import Batch
    cases = _cases(V)
    single = []
    for c in cases:
        c.tunnel.precision = prec
        ch = c.tunnel.build(c.body)
        ch.sim.record(c.steps)
        ch.step(c.steps)
        single.append((ch.sim.state_hash(), ch.sim.history()[:, :2].copy(), ch.sim.populations().copy()))
        ch.close()
    runs = [("256x1", "concurrent", 2), ("64x4", "links-first", 2), ("32x8", "bulk-first", 2),
            ("128x2", "staged", 2), ("32x8", "staged", 2), ("packed", "concurrent", 2), ("packed", "staged", 2)]
    if prec != "f64":
        runs += [("256x1", "concurrent", 1), ("128x2", "staged", 1), ("packed", "concurrent", 1),
                 ("packed", "staged", 1)]
    for tile, sched, cells in runs:
        b = Batch(prec)
        for c in cases:
            b.add(c.tunnel.spec(c.body), c.steps)
        b.build()
        b.tile = tile
        b.schedule = sched
        b.set_cells_per_thread(cells)
        b.run()
        for k, c in enumerate(cases):
            t, nonfinite, _ = b.status(k)
            assert t == c.steps and not nonfinite
            assert b.state_hash(k) == single[k][0], (tile, sched, cells, k)
            assert np.array_equal(b.populations(k), single[k][2]), (tile, sched, cells, k)
            assert np.array_equal(b.force_history(k), single[k][1]), (tile, sched, cells, k)
        b.close()


def test_batch_autotune_and_partial_runs_do_not_change_results(gpu):
    V = gpu
    from vortexlab_b200.batch import Batch
    cases = _cases(V)
    out = []
    for mode in ("plain", "tuned", "staged plain", "staged tuned"):
        b = Batch("f32")
        for c in cases:
            b.add(c.tunnel.spec(c.body), c.steps)
        b.build()
        if mode.startswith("staged"):
            b.schedule = "staged"
        if mode.endswith("tuned"):
            ms = b.autotune(2)
            assert set(ms) == {"256x1", "128x2", "64x4", "32x8", "packed"}
            b.run(37)      # stop in the middle of a segment, then continue
            b.run()
        else:
            b.run()
        out.append([b.state_hash(k) for k in range(len(cases))])
        assert b.launch_count() >= 2 * max(c.steps for c in cases)
        b.close()
    assert out[0] == out[1] and out[2] == out[3]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_batch_init_and_macros_match_single_runs(gpu, prec):
    """A tunnel of the warm form (no ramp, no twist) initialised in a batch from given fields
    matches the same channel initialised alone with Sim::init: bit-identical in FP64; in FP32 the
    comparison allows rounding (the bit-identity of batched and single FP32 runs is the first test
    of this file)."""
    V = gpu
    from vortexlab_b200 import Channel
    from vortexlab_b200.batch import Batch
    cases = _cases(V)
    fields = []

    def nsteps(c):        # FP32: few steps, before rounding differences can grow through the flow
        return c.steps if prec == "f64" else 20

    for k, c in enumerate(cases):
        nx, ny = c.tunnel.grid()
        X, Y = np.meshgrid(np.arange(nx), np.arange(ny))
        u = c.tunnel.u
        fields.append((1.0 + 1e-4 * np.sin(X / 7.0 + k), u * (1.0 + 0.02 * np.cos(Y / 9.0)), 0.01 * u * np.sin(X / 11.0)))
    single = []
    for c, f in zip(cases, fields):
        ch = Channel(c.tunnel.spec_warm(c.body), precision=prec)
        ch.sim.init(f)
        ch.sim.record(nsteps(c))
        ch.step(nsteps(c))
        single.append((ch.sim.state_hash(), ch.sim.history()[:, :2].copy(), ch.sim.macros_field()))
        ch.close()
    b = Batch(prec)
    for c in cases:
        b.add(c.tunnel.spec_warm(c.body), nsteps(c))
    b.build()
    for k, f in enumerate(fields):
        b.init(k, *f)
    b.run()
    with pytest.raises(V.VortexError):
        b.init(0, *fields[0])
    for k in range(len(cases)):
        assert not b.status(k)[1] and np.all(np.isfinite(single[k][1])), k
        if prec == "f64":
            assert b.state_hash(k) == single[k][0], k
            assert np.array_equal(b.force_history(k), single[k][1]), k
            for a, s in zip(b.macros_field(k), single[k][2]):
                assert np.array_equal(a, s), k
        else:
            h = b.force_history(k)
            assert np.max(np.abs(h - single[k][1])) <= 1e-4 * np.max(np.abs(single[k][1])), k
            for a, s in zip(b.macros_field(k), single[k][2]):
                assert np.max(np.abs(a - s)) <= 1e-5, k
    b.close()


def test_batch_set_steps_matches_a_shorter_run(gpu):
    """Ending a running tunnel early (vl_batch_set_steps) gives the state and history of a tunnel
    added with that many steps; the others are untouched; a tunnel cannot be ended in its past."""
    V = gpu
    from vortexlab_b200.batch import Batch
    cases = _cases(V)
    ref = Batch("f32")
    for k, c in enumerate(cases):
        ref.add(c.tunnel.spec(c.body), 40 if k == 0 else c.steps)
    ref.build()
    ref.run()
    b = Batch("f32")
    for c in cases:
        b.add(c.tunnel.spec(c.body), c.steps)
    b.build()
    b.run(25)
    b.set_steps(0, 40)
    with pytest.raises(V.VortexError):
        b.set_steps(1, 10)
    with pytest.raises(V.VortexError):
        b.set_steps(2, cases[2].steps + 1)
    b.run()
    assert b.info(0)["steps"] == 40 and b.status(0)[0] == 40
    for k in range(len(cases)):
        assert b.state_hash(k) == ref.state_hash(k), k
        assert np.array_equal(b.force_history(k), ref.force_history(k)), k


def test_async_runs_and_history_copy(gpu):
    """Chunks enqueued with run_async, tunnels ended while a chunk is in flight and histories read
    beside it (vl_batch_history_copy) give the states and records of synchronous runs with the same
    ends; a range past the steps complete at the last wait is refused."""
    V = gpu
    from vortexlab_b200.batch import Batch
    cases = _cases(V)
    ref = Batch("f32")
    for k, c in enumerate(cases):
        ref.add(c.tunnel.spec(c.body), 30 if k == 1 else c.steps)
    ref.build()
    ref.run()
    b = Batch("f32")
    for c in cases:
        b.add(c.tunnel.spec(c.body), c.steps)
    b.build()
    b.run_async(10)
    b.wait()
    b.run_async(20)                       # steps 10..30 in flight
    got = b.history_copy([(0, 0, 10), (2, 3, 7), (1, 0, 0)])
    with pytest.raises(V.VortexError):
        b.history_copy([(0, 5, 6)])       # step 10 is not complete at the last wait
    b.set_steps(1, 30)                    # the end of the chunk in flight
    with pytest.raises(V.VortexError):
        b.set_steps(3, 29)                # inside the chunk in flight
    b.run_async()
    b.wait()
    assert got[0].shape == (10, 2) and got[2].shape == (0, 2)
    assert np.array_equal(got[0], ref.force_history(0)[:10])
    assert np.array_equal(got[1], ref.force_history(2)[3:10])
    assert b.status(1)[0] == 30
    for k in range(len(cases)):
        assert b.state_hash(k) == ref.state_hash(k), k
        assert np.array_equal(b.force_history(k), ref.force_history(k)), k
    whole = b.history_copy([(k, 0, cases[k].steps if k != 1 else 30) for k in range(len(cases))])
    for k in range(len(cases)):
        assert np.array_equal(whole[k], ref.force_history(k)), k
    b.close()
    ref.close()


def test_held_tunnel_started_later_runs_as_from_step_zero(gpu):
    """A tunnel held at its start state and started mid-run (vl_batch_hold / vl_batch_start) takes
    the same steps as from global step 0: state and force history bit-identical; its steps, ends
    and history ranges count from its own step 0; the other tunnels are untouched."""
    V = gpu
    from vortexlab_b200.batch import Batch
    cases = _cases(V)
    ref = Batch("f32")
    for k, c in enumerate(cases):
        ref.add(c.tunnel.spec(c.body), 50 if k == 1 else c.steps)
    ref.build()
    ref.run()
    b = Batch("f32")
    for c in cases:
        b.add(c.tunnel.spec(c.body), c.steps)
    b.build()
    b.hold(1)
    b.run_async(37)
    b.wait()
    assert b.status(1)[0] == 0
    with pytest.raises(V.VortexError):
        b.hold(2)                       # only before the batch's first step
    b.run_async(10)                     # global steps 37..47 in flight
    assert b.start(1) == 47             # its step 0 follows them (an odd global step: the other buffer)
    b.set_steps(1, 50)                  # 50 of its own steps
    with pytest.raises(V.VortexError):
        b.start(1)                      # not held any more
    with pytest.raises(V.VortexError):
        b.history_copy([(1, 0, 1)])     # none of its steps is complete yet
    b.run_async(30)
    b.wait()
    got = b.history_copy([(1, 0, 30)])[0]
    b.run()
    assert b.status(1)[0] == 50
    assert np.array_equal(got, ref.force_history(1)[:30])
    for k in range(len(cases)):
        assert b.state_hash(k) == ref.state_hash(k), k
        assert np.array_equal(b.force_history(k), ref.force_history(k)), k
    b.close()
    ref.close()


def test_batch_init_from_a_grid_matches_the_host_decode(gpu):
    """vl_batch_init_grid (bilinear sampling and decoding of a coarse grid of normalised fields on
    the device) gives the fields of the host decode followed by vl_batch_init."""
    V = gpu
    import torch
    from vortexlab_b200 import warmstart as WS
    from vortexlab_b200.batch import Batch
    cases = _cases(V)
    rng = np.random.default_rng(4)
    grids = [(0.2 * rng.standard_normal((WS.H, WS.W, 8))).astype(np.float32) for _ in cases]
    out = []
    for device in (False, True):
        b = Batch("f64")
        for c in cases:
            b.add(c.tunnel.spec_warm(c.body), 5)
        b.build()
        for k, (c, g) in enumerate(zip(cases, grids)):
            tn = c.tunnel
            i = b.info(k)
            if device:
                gt = torch.from_numpy(g).cuda()
                rc = V.lib.vl_batch_init_grid(b._h, k, V._lib.C.c_void_p(gt.data_ptr()), WS.H, WS.W, 8, 0.5,
                                              20.0 * tn.d / WS.W, 0.5, 10.0 * tn.d / WS.H, tn.u)
                assert rc == 0, V._lib.last_error()
            else:
                b.init(k, *WS.decode_to_lattice(g, i["nx"], i["ny"], tn.d, tn.u))
        out.append([b.macros_field(k) for k in range(len(cases))])
        b.close()
    for host, dev in zip(*out):
        for a, d in zip(host, dev):
            assert np.max(np.abs(a - d)) <= 1e-12
