"""What the trained warm start gains over the method without it, on held-out tunnels: the network
shipped with the library (trained on 2000 tunnels of another seed) against the uniform start, both
in the batched FP32 form, judged against plain FP64 single-tunnel runs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _held_out(count=8):
    """The first `count` tunnels of the held-out population with D <= 22 and Re >= 100 (shedding
    wakes small enough for a test), run for 100 convective units."""
    from vortexlab_b200 import warmstart as WS
    from vortexlab_b200.batch import seeded_tunnels
    cases = seeded_tunnels(seed=WS.TEST_SEED, count=256, units=100.0)
    return [c for c in cases if c.params["d"] <= 22 and c.params["re"] >= 100.0][:count]


def test_warm_start_converges_in_fewer_steps(gpu):
    from vortexlab_b200 import convergence as CV
    from vortexlab_b200 import warmstart as WS
    cases = _held_out()
    net = WS.load_pretrained()
    out = CV.warm_comparison(net, cases)
    rows = out["rows"]
    both = [r for r in rows if r["plain_conv_steps"] > 0 and r["cold_conv_steps"] > 0 and r["warm_conv_steps"] > 0]
    assert len(both) >= 6, rows
    ratio = np.median([r["warm_conv_steps"] / r["cold_conv_steps"] for r in both])
    assert ratio < 0.8, ratio                         # the warm start removes at least 20 % of the steps
    for r in both:                                    # and ends on the plain run's statistics
        assert abs(r["warm_cd_err"]) <= 0.005 and abs(r["warm_st_err"]) <= 0.005, r
    warm = out["summary"]["warm"]
    cold = out["summary"]["cold"]
    assert warm["median_speedup"] > cold["median_speedup"], out["summary"]
