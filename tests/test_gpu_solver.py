"""The reference's solver-level tests (tests/solver.rs) run on the device, with the reference's
tolerances. Together with the oracle parity tests they show the kernels keep the invariants the
reference guarantees: conservation, Galilean-invariant wall forces, transparent open boundaries,
determinism and a working absorbing outlet."""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu

MODELS = ["bgk", ("trt", 3.0 / 16.0), ("trt", 0.25)]


@pytest.mark.parametrize("collision", MODELS)
def test_periodic_box_conserves_mass_and_momentum(gpu, collision):
    """tests/solver.rs:21-46."""
    sim = S.product_sim(S.periodic_box(48, 36, 0.62, collision))
    sim.init(S.swirl(48, 36))
    m0, p0 = sim.total_mass(), sim.total_momentum()
    sim.step(400)
    m1, p1 = sim.total_mass(), sim.total_momentum()
    assert abs(m1 - m0) < 2e-12
    assert abs(p1[0] - p0[0]) < 1e-12 and abs(p1[1] - p0[1]) < 1e-12
    assert sim.max_speed() < 0.07


def test_body_force_adds_exactly_its_impulse(gpu):
    """tests/solver.rs:48-61."""
    sim = S.product_sim(S.periodic_box(20, 16, 0.7, ("trt", 3.0 / 16.0), accel=(3e-5, -1e-5)))
    sim.init(S.swirl(20, 16))
    m, p0 = sim.total_mass(), sim.total_momentum()
    sim.step(250)
    p1 = sim.total_momentum()
    assert abs(p1[0] - p0[0] - 250.0 * 3e-5 * m) < 1e-11
    assert abs(p1[1] - p0[1] + 250.0 * 1e-5 * m) < 1e-11


@pytest.mark.parametrize("collision", MODELS)
def test_closed_box_with_halfway_walls_conserves_mass(gpu, collision):
    """tests/solver.rs:63-80."""
    d = dict(nx=34, ny=26, tau=0.58, collision=collision, kinds=[("wall", None, 0, None, None)],
             paint=[("rect", 0, 33, 0, 25, 1), ("rect", 1, 32, 1, 24, 0)])
    sim = S.product_sim(d)
    sim.init(S.swirl(34, 26))
    m0 = sim.total_mass()
    sim.step(600)
    assert abs(sim.total_mass() - m0) < 2e-12
    assert sim.max_speed() < 0.05


@pytest.mark.parametrize("collision", ["bgk", ("trt", 3.0 / 16.0)])
@pytest.mark.parametrize("frame", [0.0, 0.03, -0.05, 0.08])
def test_wall_shear_is_galilean_invariant(gpu, collision, frame):
    """tests/solver.rs:86-123 (Couette flow seen from sliding frames)."""
    shear, rows, nx = 0.04, 20, 6
    sim = S.product_sim(S.couette(frame, shear, collision, nx, rows))
    exact = lambda y: frame + shear * (y - 0.5) / rows  # noqa: E731
    ny = rows + 2
    ux = np.array([[exact(y)] * nx for y in range(ny)])
    sim.init((np.ones((ny, nx)), ux, np.zeros((ny, nx))))
    sim.step(20000)
    dev = max(abs(sim.macros(2, y)[1] - exact(y)) for y in range(1, rows + 1))
    f = sim.force
    low, top, normal = f[0, 0] / nx, f[1, 0] / nx, f[0, 1] / nx
    expected = (0.9 - 0.5) / 3.0 * shear / 20.0
    assert dev < 1e-12
    assert abs(low - expected) < 1e-12 * max(1.0, 1.0 / expected) * expected + 1e-13
    assert abs(top + expected) < 1e-13
    assert abs(normal + 1.0 / 3.0) < 1e-12


@pytest.mark.parametrize("collision", ["bgk", ("trt", 3.0 / 16.0)])
@pytest.mark.parametrize("u", [(0.06, 0.0), (0.0, -0.05), (0.04, 0.03), (-0.07, 0.02)])
@pytest.mark.parametrize("shape", [("circle", 20.3, 15.7, 6.4), ("section", 4, 0.1, 20.5, 16.5, 12.0, 0.3)])
def test_body_moving_with_the_stream_feels_no_force(gpu, collision, u, shape):
    """tests/solver.rs:125-159."""
    d = S.periodic_box(40, 32, 0.6, collision)
    d["kinds"] = [("wall", ("const", u[0], u[1]), 0, 0, shape)]
    d["paint"] = [("shape", 1)]
    sim = S.product_sim(d)
    sim.init((1.0, u[0], u[1]))
    sim.step(200)
    f = sim.force[0]
    assert abs(f[0]) < 1e-13 and abs(f[1]) < 1e-13
    _, ux, uy = sim.macros(3, 3)
    assert abs(ux - u[0]) < 1e-14 and abs(uy - u[1]) < 1e-14


def test_body_at_rest_in_fluid_at_rest_feels_no_force(gpu):
    """tests/solver.rs:161-173 (Builder default tau = 1, TRT 3/16)."""
    d = dict(nx=40, ny=32, periodic=(True, True), tau=1.0,
             kinds=[("wall", None, 0, 0, ("circle", 19.2, 16.9, 7.3))], paint=[("shape", 1)])
    sim = S.product_sim(d)
    sim.step(50)
    assert abs(sim.force[0, 0]) < 1e-14 and abs(sim.force[0, 1]) < 1e-14
    assert sim.max_speed() < 1e-15


def _open_channel(V, nx, rows, inflow, u, tau):
    """tests/solver.rs:176-199."""
    h = float(rows)
    kinds = [("wall", ("parabolic", u, h) if inflow == "parabolic" else ("const", u, 0.0), 0, None, None),
             ("pressure", 1.0),
             ("wall", None, 0, None, None) if inflow == "parabolic" else ("wall", ("const", u, 0.0), 0, None, None)]
    paint = [("rect", 0, 0, 0, rows + 1, 1), ("rect", nx - 1, nx - 1, 0, rows + 1, 2),
             ("rect", 0, nx - 1, 0, 0, 3), ("rect", 0, nx - 1, rows + 1, rows + 1, 3)]
    d = dict(nx=nx, ny=rows + 2, tau=tau, collision=("trt", 3.0 / 16.0), kinds=kinds, paint=paint)
    sim = S.product_sim(d)
    ys = np.arange(rows + 2, dtype=np.float64)
    if inflow == "parabolic":
        s = np.clip(ys - 0.5, 0.0, h)
        prof = 6.0 * u * s * (h - s) / (h * h)
    else:
        prof = np.full(rows + 2, u)
    sim.init((np.ones((rows + 2, nx)), np.repeat(prof[:, None], nx, axis=1), np.zeros((rows + 2, nx))))
    return sim


def test_uniform_stream_passes_through_inlet_and_outlet_unchanged(gpu):
    """tests/solver.rs:201-212."""
    sim = _open_channel(gpu, 40, 16, "uniform", 0.07, 0.55)
    sim.step(500)
    for (x, y) in [(1, 1), (20, 8), (38, 16), (38, 1)]:
        rho, ux, uy = sim.macros(x, y)
        assert abs(rho - 1.0) < 1e-13 and abs(ux - 0.07) < 1e-13 and abs(uy) < 1e-13


def test_inlet_and_outlet_drive_developed_channel_flow(gpu):
    """tests/solver.rs:214-253."""
    nx, rows, u_mean, tau = 82, 20, 0.005, 0.8
    sim = _open_channel(gpu, nx, rows, "parabolic", u_mean, tau)
    sim.step(40000)
    h = float(rows)
    rho, ux, uy = sim.macros_field()
    flux = lambda x: float(np.sum(rho[1:rows + 1, x] * ux[1:rows + 1, x])) / h / (1.0 + 0.5 / (h * h))  # noqa: E731
    mean_flux = flux(40)
    worst = 0.0
    for y in range(1, rows + 1):
        exact = 6.0 * mean_flux * (y - 0.5) * (h - y + 0.5) / (h * h)
        worst = max(worst, abs(rho[y, 40] * ux[y, 40] - exact), abs(uy[y, 40]))
    assert worst < 2e-4 * u_mean
    slope = (1.0 / 3.0) * (rho[10, 60] - rho[10, 20]) / 40.0
    exact = -12.0 * (tau - 0.5) / 3.0 * mean_flux / (h * h)
    assert abs(slope / exact - 1.0) < 1e-3
    u_max = 1.5 * u_mean
    assert abs(rho[10, nx - 2] - 1.0) < 6.0 * u_max * u_max
    assert abs(flux(2) / flux(nx - 3) - 1.0) < 1e-6
    crossing = mean_flux * (1.0 + 0.5 / (h * h))
    assert abs(crossing / u_mean - 1.0) < 1e-6


def test_absorbing_outlet_removes_sound_waves(gpu):
    """tests/solver.rs:293-327."""
    V = gpu

    def ripple(absorbing):
        spec = V.Spec(nx=302, ny=42, inflow=V.Inflow.Uniform(0.05), nu=0.02, collision=V.Collision.Trt(3.0 / 16.0),
                      body=V.Circle(60.5, 20.5, 4.0), ramp_steps=1)
        ch = V.Channel(spec)
        ch.sim.init((1.0, 0.0, 0.0))
        ch.absorbing_outlet = absorbing
        ch.step(6000)
        ch.sim.record(1200)
        ch.step(1200)
        cd = 2.0 / (0.05 * 0.05 * 8.0) * ch.sim.history()[:, 0]
        return (cd.max() - cd.min()) / cd.max()

    reflecting, absorbing = ripple(False), ripple(True)
    assert absorbing < 0.01
    assert reflecting > 10.0 * absorbing


def test_under_resolved_2d2_reports_divergence(gpu):
    """tests/validation.rs:92-94: at 10 cells per diameter case 2D-2 must diverge, not return numbers."""
    V = gpu
    with pytest.raises(V.VortexError, match="diverged"):
        V.cylinder.run_2d2(V.cylinder.Setup(n=10), 30.0, 5.0)
