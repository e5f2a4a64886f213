"""Batched tunnels: a tunnel advanced in a batch with others of other sizes, shapes and Reynolds
numbers is bit-identical to the same tunnel run alone (state and per-step force), in every tile
shape and kernel schedule; autotuning does not perturb the run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases(V):
    from vortexlab_b200.batch import seeded_tunnels
    cases = seeded_tunnels(seed=99, count=4, dmin=8, dmax=14, units=3.0)
    return cases


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_batched_tunnels_match_single_runs(gpu, prec):
    V = gpu
    from vortexlab_b200.batch import Batch
    cases = _cases(V)
    single = []
    for c in cases:
        c.tunnel.precision = prec
        ch = c.tunnel.build(c.body)
        ch.sim.record(c.steps)
        ch.step(c.steps)
        single.append((ch.sim.state_hash(), ch.sim.history()[:, :2].copy()))
        ch.close()
    for tile, sched in [("256x1", "concurrent"), ("64x4", "links-first"), ("32x8", "bulk-first")]:
        b = Batch(prec)
        for c in cases:
            b.add(c.tunnel.spec(c.body), c.steps)
        b.build()
        b.tile = tile
        b.schedule = sched
        b.run()
        for k, c in enumerate(cases):
            t, nonfinite, _ = b.status(k)
            assert t == c.steps and not nonfinite
            assert b.state_hash(k) == single[k][0], (tile, sched, k)
            assert np.array_equal(b.force_history(k), single[k][1]), (tile, sched, k)
        b.close()


def test_batch_autotune_and_partial_runs_do_not_change_results(gpu):
    V = gpu
    from vortexlab_b200.batch import Batch
    cases = _cases(V)
    out = []
    for mode in ("plain", "tuned"):
        b = Batch("f32")
        for c in cases:
            b.add(c.tunnel.spec(c.body), c.steps)
        b.build()
        if mode == "tuned":
            ms = b.autotune(2)
            assert set(ms) == {"256x1", "128x2", "64x4", "32x8"}
            b.run(37)      # stop in the middle of a segment, then continue
            b.run()
        else:
            b.run()
        out.append([b.state_hash(k) for k in range(len(cases))])
        assert b.launch_count() >= 2 * max(c.steps for c in cases)
        b.close()
    assert out[0] == out[1]
