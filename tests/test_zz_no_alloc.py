"""vl_reduce_f64_static: the allocation-free reduction for callers that cannot allocate device memory
(a host framework or plugin that owns every device buffer). The caller hands in its own device
buffers — here allocated by torch, standing in for such a host — and the call itself allocates
nothing; its results must match the sim's own reductions (vl_sim_total_mass, vl_sim_total_momentum,
vl_sim_max_speed) within the tolerances of the other reduction tests, on two calls in a row, on a
grid of several chunks with a partial last one, with a plane stride above the cell count (padding
filled with NaN that must never be read), and on a one-chunk grid right after a four-chunk one (the
second call must not combine the first call's leftover partials). Free device memory must not
change across a call. Collected last so that a run stopping at the first failure has run every other test first."""
import ctypes as C

import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


def _call(V, f, ns, flag, n, out, gx=0.0, gy=0.0):
    return V.lib.vl_reduce_f64_static(C.c_void_p(f), ns, C.c_void_p(flag), n, gx, gy, C.c_void_p(out), None)


def test_static_scratch_reduction_matches_the_sim_reductions(gpu):
    V = gpu
    import torch

    d = S.periodic_box(48, 36, collision="bgk")
    d["kinds"] = [("wall", ("const", 0.01, -0.02), 0, 0, ("circle", 20.3, 15.7, 6.4))]
    d["paint"] = [("shape", 1)]
    sim = S.product_sim(d)
    sim.init(S.swirl(48, 36))
    n = sim.n
    dev = torch.device("cuda", 0)
    flag = torch.from_numpy(sim.flags().reshape(-1).copy()).to(dev)
    out = torch.full((4,), float("nan"), dtype=torch.float64, device=dev)
    for call in range(2):
        sim.step(37)
        pops = torch.from_numpy(sim.populations().reshape(-1).copy()).to(dev)
        torch.cuda.synchronize()
        rc = _call(V, pops.data_ptr(), n, flag.data_ptr(), n, out.data_ptr())
        assert rc == 0, V._lib.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        mass, mom, vmax = sim.total_mass(), sim.total_momentum(), sim.max_speed()
        assert abs(got[0] - mass) <= 1e-13 * abs(mass), (call, got[0], mass)
        assert abs(got[1] - mom[0]) <= 1e-14 and abs(got[2] - mom[1]) <= 1e-14, (call, got[1:3], mom)
        assert got[3] == vmax, (call, got[3], vmax)


def test_static_scratch_reduction_rejects_more_cells_than_its_scratch_holds(gpu):
    V = gpu
    import torch

    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    limit = 33554432  # VL_REDUCE_STATIC_MAX_CELLS
    rc = _call(V, buf.data_ptr(), limit + 1, buf.data_ptr(), limit + 1, buf.data_ptr())
    assert rc == -1 and "VL_REDUCE_STATIC_MAX_CELLS" in V._lib.last_error()


def _sim_with_body(nx, ny):
    d = S.periodic_box(nx, ny, collision="bgk")
    d["kinds"] = [("wall", ("const", 0.01, -0.02), 0, 0, ("circle", 0.42 * nx, 0.44 * ny, 0.13 * min(nx, ny)))]
    d["paint"] = [("shape", 1)]
    sim = S.product_sim(d)
    sim.init(S.swirl(nx, ny))
    sim.step(23)
    return sim


def _check(sim, got, what):
    mass, mom, vmax = sim.total_mass(), sim.total_momentum(), sim.max_speed()
    assert abs(got[0] - mass) <= 1e-13 * abs(mass), (what, got[0], mass)
    assert abs(got[1] - mom[0]) <= 1e-14 and abs(got[2] - mom[1]) <= 1e-14, (what, got[1:3], mom)
    assert got[3] == vmax, (what, got[3], vmax)


def test_static_scratch_reduction_over_chunks_padding_and_a_smaller_second_call(gpu):
    V = gpu
    import torch

    dev = torch.device("cuda", 0)
    big = _sim_with_body(250, 240)      # 60,000 cells: 3 full chunks of 16,384 and a partial fourth
    small = _sim_with_body(48, 36)      # 1,728 cells: one chunk
    n_big, n_small = big.n, small.n
    assert n_big == 60000 and n_big % 16384 != 0 and n_big // 16384 == 3
    ns = n_big + 1000                   # plane stride above n; the padding is NaN
    padded = np.full((9, ns), np.nan)
    padded[:, :n_big] = big.populations().reshape(9, n_big)
    pops_big = torch.from_numpy(padded.reshape(-1)).to(dev)
    flag_big = torch.from_numpy(big.flags().reshape(-1).copy()).to(dev)
    pops_small = torch.from_numpy(small.populations().reshape(-1).copy()).to(dev)
    flag_small = torch.from_numpy(small.flags().reshape(-1).copy()).to(dev)
    out = torch.full((4,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    assert _call(V, pops_big.data_ptr(), ns, flag_big.data_ptr(), n_big, out.data_ptr()) == 0, V._lib.last_error()
    torch.cuda.synchronize()
    _check(big, out.cpu().numpy(), "four chunks, padded planes")

    free0 = torch.cuda.mem_get_info(dev)[0]
    assert _call(V, pops_small.data_ptr(), n_small, flag_small.data_ptr(), n_small, out.data_ptr()) == 0, \
        V._lib.last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free0, "the call changed the free device memory"
    _check(small, out.cpu().numpy(), "one chunk after four")

    assert _call(V, pops_big.data_ptr(), ns, flag_big.data_ptr(), n_big, out.data_ptr()) == 0, V._lib.last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free0
    _check(big, out.cpu().numpy(), "four chunks again")
