"""The throughput workload at its full size against the oracle.

The 8192 x 4096 periodic BGK box with seeded disks filling 5 % of the cells (31.9 M fluid nodes,
891,696 links, 386,109 boundary nodes) exercises what the smaller parity cases cannot: the staged
step's split of its link blocks and row tiles, the per-warp rank table over 1 M warp slots, the
fixed tree over thousands of force partials, and plane offsets near 3e8 elements. Both the
staged step and the two-kernel concurrent step run 12 steps from the uniform start; populations
must be bit-identical to the oracle's (the bar is 1e-10 absolute) and every step's force within
1e-9 relative (src/sim.rs:391-508, state hash src/sim.rs:654-668).
"""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

NX, NY, SEED, FRACTION, TAU, U = 8192, 4096, 0x5EED0001, 0.05, 0.55, 0.05
STEPS = 12
POP_ABS = 1e-10
FORCE_REL = 1e-9


@pytest.fixture(scope="module")
def oracle_run(O):
    import os

    from vortexlab_b200.workloads import disk_field
    disks = disk_field(NX, NY, SEED, FRACTION)
    b = O.Builder(NX, NY)
    b.periodic_x = b.periodic_y = True
    b.tau = TAU
    b.collision = O.BGK
    b.fill_shape(b.add_wall(fgroup=0, shape=O.Shape.disks(disks)))
    osim = b.build(os.cpu_count() or 1)
    osim.init((np.ones((NY, NX)), np.full((NY, NX), U), np.zeros((NY, NX))))
    force = np.zeros((STEPS, 2))
    for k in range(STEPS):
        osim.step(1)
        force[k] = osim.force[0]
    return disks, osim, force


@pytest.mark.parametrize("schedule", ["staged", "concurrent"])
def test_full_box_against_oracle(gpu, oracle_run, schedule):
    V = gpu
    from vortexlab_b200.workloads import build_disk_box
    disks, osim, oforce = oracle_run
    sim = build_disk_box(V, NX, NY, disks, tau=TAU)
    try:
        assert sim.fluid_nodes() == osim.fluid_nodes()
        assert sim.link_count() == osim.link_count()
        sim.schedule = schedule
        sim.init((1.0, U, 0.0))
        sim.record(STEPS)
        sim.step(STEPS)
        hist = sim.history()
        f = sim.populations().reshape(9, -1)
        fo = osim.populations().reshape(9, -1)
        for i in range(9):
            d = float(np.max(np.abs(f[i] - fo[i])))
            assert d <= POP_ABS, f"plane {i}: {d}"
            assert np.array_equal(f[i], fo[i]), f"plane {i} is not bit-identical"
        del f, fo
        assert sim.state_hash() == osim.state_hash()
        scale = np.max(np.abs(oforce))
        assert np.max(np.abs(hist[:, :2] - oforce)) <= FORCE_REL * scale
        assert sim.t == STEPS
    finally:
        sim.close()
