"""Reduced-precision storage (FP32; FP16 of f_i - w_i) with FP32 collision and FP64 force,
compared with the FP64 path (which is bit-identical to the reference's CPU solver)."""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["f32", "f16s"])
def test_storage_round_trip(gpu, prec):
    """Sim::init writes equilibria; the download returns them rounded to the storage format."""
    V = gpu
    d = S.periodic_box(24, 20, collision="bgk")
    sim = S.product_sim(d, precision=prec)
    rho, ux, uy = S.swirl(24, 20)
    sim.init((rho, ux, uy))
    f = sim.populations()
    w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    ref = S.product_sim(d)
    ref.init((rho, ux, uy))
    fe = ref.populations()
    if prec == "f32":
        expect = fe.astype(np.float32).astype(np.float64)
    else:
        expect = (w[:, None, None].astype(np.float32)
                  + (fe.astype(np.float32) - w[:, None, None].astype(np.float32)).astype(np.float16).astype(np.float32)
                  ).astype(np.float64)
    assert np.array_equal(f, expect)


def test_f32_schafer_turek_2d2_matches_f64(gpu):
    """2D-2 at 20 cells per diameter, 60 convective units, statistics over the last 20: the FP32
    storage path stays within 2e-4 of the FP64 path on the force coefficients and St, and within
    1e-3 on the pressure drop (a difference of two nearly equal probe densities divided by u^2,
    sampled half a period after each lift peak, so its relative error is amplified)."""
    V = gpu
    runs = {p: V.cylinder.run_2d2(V.cylinder.Setup(n=20, precision=p), 60.0, 20.0) for p in ("f64", "f32")}
    a, b = runs["f64"], runs["f32"]
    for k, tol in (("cd_max", 2e-4), ("cd_min", 2e-4), ("cl_max", 2e-4), ("cl_min", 2e-4), ("st", 2e-4), ("dp", 1e-3)):
        va, vb = getattr(a, k), getattr(b, k)
        assert abs(vb - va) <= tol * abs(va), (k, va, vb)


@pytest.mark.parametrize("prec,tol", [("f32", 1e-6), ("f16s", 5e-4)])
def test_decaying_swirl_matches_f64(gpu, prec, tol):
    """Periodic box, TRT, 400 steps of a decaying swirl: velocity and density fields against FP64."""
    d = S.periodic_box(48, 36, 0.62, ("trt", 3.0 / 16.0))
    fields = []
    for p in ("f64", prec):
        sim = S.product_sim(d, precision=p)
        sim.init(S.swirl(48, 36))
        sim.step(400)
        fields.append(sim.macros_field())
        if p == prec:
            m = sim.total_mass()
    for a, b in zip(*fields):
        assert np.max(np.abs(a - b)) < tol
    assert abs(m / (48 * 36) - 1.0) < 10 * tol
