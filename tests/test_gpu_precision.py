"""Reduced-precision storage (FP32; 16-bit forms of f_i - w_i) with FP32 collision and FP64 force,
compared with the FP64 path (which is bit-identical to the reference's CPU solver)."""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


def c16_stored(v32, w32):
    """The value the custom 16-bit format (sign, 3-bit exponent, 12-bit mantissa of f_i - w_i) stores
    for FP32 populations v32 of weight w32, restated on the host: (v - w) 2^-118 rounded once to FP32,
    its bit pattern rounded to 12 mantissa bits (ties to even) and clamped, then decoded and w added
    back in one rounding."""
    y = ((v32.astype(np.float64) - w32.astype(np.float64)) * 2.0 ** -118).astype(np.float32)
    b = y.view(np.uint32).astype(np.uint64)
    mag = np.minimum(b & 0x7FFFFFFF, 0x03FFF800)
    r = (mag + 0x3FF + ((mag >> 11) & 1)) >> 11
    code = r | ((b >> 16) & 0x8000)
    bits = (((code & 0x7FFF) << 11) | ((code & 0x8000) << 16)).astype(np.uint32)
    x = bits.view(np.float32).astype(np.float64) * 2.0 ** 118
    return (x + w32.astype(np.float64)).astype(np.float32)


def q16_stored(v32, w32, up):
    """The value the 16-bit fixed-point format stores for FP32 populations v32 of weight w32 with
    scale `up` (2^18 for the axis directions, 2^19 otherwise), restated on the host: (v - w) up
    rounded once to FP32 (the scale is a power of two, so that is the FP32 difference scaled),
    rounded to the nearest integer (ties to even) and clamped to int16, then decoded and w added
    back in one FP32 rounding."""
    y = (v32 - w32).astype(np.float32) * np.float32(up)
    q = np.clip(np.rint(y), -32768, 32767).astype(np.float32)
    return (w32 + q * np.float32(1.0 / up)).astype(np.float32)


@pytest.mark.parametrize("prec", ["f32", "f16s", "f16c", "f16x"])
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
    elif prec == "f16c":
        w32 = np.broadcast_to(w[:, None, None].astype(np.float32), fe.shape)
        expect = c16_stored(fe.astype(np.float32), w32).astype(np.float64)
    elif prec == "f16x":
        w32 = np.broadcast_to(w[:, None, None].astype(np.float32), fe.shape)
        up = np.array([2.0 ** 19] + [2.0 ** 18] * 4 + [2.0 ** 19] * 4)[:, None, None]
        expect = np.stack([q16_stored(fe[i].astype(np.float32), w32[i], up[i, 0, 0]) for i in range(9)]).astype(np.float64)
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


@pytest.mark.parametrize("prec,tol", [("f32", 1e-6), ("f16s", 5e-4), ("f16c", 5e-4), ("f16x", 5e-4)])
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
