"""The reference's solver-level tests (tests/solver.rs) and the validation cases of
tests/validation.rs that need no external data run on the device, with the reference's
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


def _poiseuille(rows, q, collision, tau=0.8):
    """src/cases/poiseuille.rs:41-90 on the device: the body-force channel run until the profile
    changes by less than 1e-13 u_max over 200 steps; relative L2 error against the parabola and
    wall drag over driving force."""
    d = S.poiseuille(rows=rows, tau=tau, q=q, collision=collision)
    sim = S.product_sim(d)
    y0, y1 = 1.0 - q, rows + q
    nu = (tau - 0.5) / 3.0
    umax = 0.1 * 16.0 / rows
    g = d["accel"][0]
    prev = np.zeros(rows + 2)
    while True:
        sim.step(200)
        u = sim.macros_field()[1][:, 1]
        change = np.max(np.abs(u[1:rows + 1] - prev[1:rows + 1]))
        prev = u
        if change < 1e-13 * umax or sim.t > 4_000_000:
            break
    y = np.arange(1, rows + 1, dtype=float)
    exact = g / (2.0 * nu) * (y - y0) * (y1 - y)
    num = float(np.sum((u[1:rows + 1] - exact) ** 2))
    den = float(np.sum(exact ** 2))
    return dict(rows=rows, q=q, l2=(num / den) ** 0.5, force_balance=sim.force[0][0] / (g * sim.total_mass()))


def test_poiseuille_is_second_order_and_exact_with_the_magic_parameter(gpu):
    """tests/validation.rs:19-36: second-order convergence of the driven channel for BGK and TRT
    with halfway and off-lattice walls; TRT with Lambda = 3/16 and halfway walls exact to rounding,
    with the wall drag balancing the driving force."""
    for collision, q in (("bgk", 0.5), (("trt", 0.25), 0.5), (("trt", 3.0 / 16.0), 0.25), (("trt", 3.0 / 16.0), 0.8)):
        out = [_poiseuille(h, q, collision) for h in (8, 16, 32)]
        for a, b in zip(out, out[1:]):
            h0, h1 = a["rows"] - 1.0 + 2.0 * a["q"], b["rows"] - 1.0 + 2.0 * b["q"]
            order = np.log(a["l2"] / b["l2"]) / np.log(h1 / h0)
            assert abs(order - 2.0) < 0.05, (collision, q, order)
        assert out[2]["l2"] < 2.5e-3, (collision, q, out[2]["l2"])
    for o in (_poiseuille(h, 0.5, ("trt", 3.0 / 16.0)) for h in (8, 16, 32)):
        assert o["l2"] < 1e-10, o
        assert abs(o["force_balance"] - 1.0) < 1e-9, o


def test_rounding_the_corners_lowers_drag_and_raises_the_shedding_frequency(gpu):
    """tests/validation.rs:96-124: a square of side 20 and the same square with corners rounded
    by 20 % in a towing tank at Re 100 (u 0.1, 10 % blockage), 70 convective units in 20 parts,
    statistics after 40."""
    V = gpu
    from vortexlab_b200.tunnel import Tunnel
    tn = Tunnel(d=20, re=100.0, u=0.1, upstream=6.0, downstream=12.0, height=10.0)
    cx, cy = tn.centre()

    def run(corner):
        ch = tn.build(V.section(corner, cx, cy, 20.0, 0.0))
        cd, cl = [], []
        for _ in range(20):
            s = tn.run(ch, 70.0 / 20.0)
            cd.append(s.cd)
            cl.append(s.cl)
        ch.close()
        return V.Series(s.dt, np.concatenate(cd), np.concatenate(cl)).stats(40.0)

    square, rounded = run(V.Corner.Sharp), run(V.Corner.Rounded(0.2))
    assert 1.45 < square.cd_mean < 1.75, square
    assert 0.14 < square.st < 0.17, square
    assert 0.1 < square.cl_rms < 0.35, square
    assert abs(square.st_crossings - square.st) <= 0.01 * abs(square.st), square
    assert abs(square.cl_mean) < 0.02, square
    assert rounded.cd_mean < 0.97 * square.cd_mean, (rounded, square)
    assert rounded.st > 1.02 * square.st, (rounded, square)


def test_nonfinite_force_is_recorded_on_the_device(gpu):
    """Failure detection without a GPU fault: NaN populations planted from the host into one
    boundary node reach the force of the next step; the device records that step (the step
    functions go on, as Sim::step does, and the case drivers then report divergence)."""
    d = S.periodic_box(48, 36, collision="bgk")
    d["kinds"] = [("wall", None, 0, 0, ("circle", 20.3, 15.7, 6.4))]
    d["paint"] = [("shape", 1)]
    sim = S.product_sim(d)
    sim.init((1.0, 0.02, 0.0))
    sim.step(5)
    assert sim.status() == (False, 0)
    f = sim.populations().copy()
    ys, xs = np.nonzero(sim.flags() == 1)
    f[:, ys[0], xs[0]] = np.nan
    sim.set_populations(f)
    sim.step(3)
    assert sim.status() == (True, 5)
    assert not np.all(np.isfinite(sim.force))


def test_nonfinite_force_is_recorded_per_tunnel_in_a_batch(gpu):
    """The same in a batch: a NaN start field in one tunnel is flagged for that tunnel only."""
    from vortexlab_b200.batch import Batch, seeded_tunnels
    cases = seeded_tunnels(seed=99, count=3, dmin=8, dmax=14, units=0.5)
    b = Batch("f32")
    for c in cases:
        b.add(c.tunnel.spec_warm(c.body), c.steps)
    b.build()
    i = b.info(1)
    rho = np.ones((i["ny"], i["nx"]))
    rho[:, :] = np.nan
    b.init(1, rho, 0.05, 0.0)
    b.run()
    assert [b.status(k)[1] for k in range(3)] == [False, True, False]
