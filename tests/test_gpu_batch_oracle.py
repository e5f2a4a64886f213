"""Batched configuration-4 tunnels against the oracle directly (not through a single GPU run).

Small seeded tunnels of the batched-tunnel population (an ellipse, a notched square and a
star-convex polygon, rotated; D 10-14 and Re 50-90, which these small grids resolve; 20 D x 10 D with sound-absorbing sides, uniform inflow ramped over 5
convective units, the body twisted by the kick from unit 5 to 7), run for 7.5 convective units in
one batch and each on the oracle's Channel (src/cases/channel.rs:71-130, src/cases/tunnel.rs:52-67):

* FP64: every tunnel's state hash equals the oracle's (populations bit-identical; the bar is 1e-10
  absolute) and its per-step force agrees within 1e-9 relative;
* FP32 storage (collision in FP32, force in FP64): populations within 2e-5 absolute and the per-step
  force within 2e-3 of the largest force magnitude of the oracle run.
"""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu

UNITS = 7.5
POP_ABS_F64, FORCE_REL_F64 = 1e-10, 1e-9
POP_ABS_F32, FORCE_REL_F32 = 2e-5, 2e-3


def _cases():
    from vortexlab_b200.batch import seeded_tunnels
    pool = seeded_tunnels(seed=0x5EED0042, count=24, dmin=10, dmax=14, re=(50.0, 90.0), units=UNITS)
    out = {}
    for c in pool:
        if c.kind not in out and c.params["angle_deg"] > 3.0 and (c.kind != "square" or c.params["notches"] > 0):
            out[c.kind] = c
    assert set(out) == {"ellipse", "square", "star"}, sorted(out)
    return [out[k] for k in ("ellipse", "square", "star")]


@pytest.fixture(scope="module")
def oracle_runs(O):
    runs = []
    for c in _cases():
        ch = S.oracle_channel(c.tunnel.spec(c.body), threads=4)
        fh, _ = ch.run(c.steps)
        runs.append((ch.sim.state_hash(), fh, ch.sim.populations()))
    return runs


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_batched_tunnels_against_the_oracle(gpu, oracle_runs, prec):
    from vortexlab_b200.batch import Batch
    cases = _cases()
    b = Batch(prec)
    for c in cases:
        b.add(c.tunnel.spec(c.body), c.steps)
    b.build()
    b.run()
    try:
        for k, (c, (ohash, ofh, opop)) in enumerate(zip(cases, oracle_runs)):
            t, nonfinite, _ = b.status(k)
            assert t == c.steps and not nonfinite, c.kind
            h = b.force_history(k)
            scale = np.max(np.abs(ofh))
            pop = b.populations(k)
            if prec == "f64":
                assert np.max(np.abs(pop - opop)) <= POP_ABS_F64, c.kind
                assert b.state_hash(k) == ohash, c.kind
                assert np.max(np.abs(h - ofh)) <= FORCE_REL_F64 * scale, c.kind
            else:
                assert np.max(np.abs(pop - opop)) <= POP_ABS_F32, (c.kind, np.max(np.abs(pop - opop)))
                assert np.max(np.abs(h - ofh)) <= FORCE_REL_F32 * scale, (c.kind, np.max(np.abs(h - ofh)) / scale)
    finally:
        b.close()
