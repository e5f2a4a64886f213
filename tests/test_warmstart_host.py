"""Host side of the learned warm start: the CPU FP64 restatement of the network (checked against
central finite differences, so that it can in turn check the device gradients), the field
encodings and the choice of the lift-maximum step. No GPU."""
import numpy as np
import pytest

from oracle import unet_ref as R


def _net(levels=2, c0=4, cin=3, cout=8, seed=0, mimic=False):
    rng = np.random.default_rng(seed)
    ws, bs = [], []
    for ci, co, s, relu, k in R.architecture(levels, c0, cin, cout):
        kp = R.kp_for(ci, k)
        fan = (9 if k == 3 else 1) * ci
        w = np.zeros((co, kp))
        w[:, :fan] = rng.standard_normal((co, fan)) * np.sqrt(2.0 / fan)
        ws.append(w)
        bs.append(0.1 * rng.standard_normal(co))
    return R.UNetRef(levels, c0, cin, cout, ws, bs, mimic_bf16=mimic)


def test_im2col_col2im_are_adjoint():
    rng = np.random.default_rng(1)
    for stride, (H, W) in ((1, (6, 10)), (2, (8, 12)), (2, (7, 9))):
        x = rng.standard_normal((2, H, W, 3))
        kp = R.kp_for(3, 3)
        cols = R.im2col(x, stride, kp)
        d = rng.standard_normal(cols.shape)
        d[:, 27:] = 0.0
        lhs = float((cols * d).sum())
        rhs = float((x * R.col2im(d, x.shape, stride)).sum())
        assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs))


def test_im2col_matches_direct_convolution():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((1, 5, 7, 2))
    w = rng.standard_normal((3, 3, 3, 2))     # cout, ky, kx, c
    cols = R.im2col(x, 2, 64)
    wm = np.zeros((3, 64))
    wm[:, :18] = w.reshape(3, 18)
    got = (cols @ wm.T).reshape(1, 3, 4, 3)
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    for oy in range(3):
        for ox in range(4):
            ref = np.einsum("oykc,ykc->o", w, xp[0, 2 * oy:2 * oy + 3, 2 * ox:2 * ox + 3])
            assert np.allclose(got[0, oy, ox], ref, atol=1e-12)


def test_reference_gradients_match_finite_differences():
    net = _net()
    rng = np.random.default_rng(3)
    x = rng.standard_normal((2, 8, 8, 3))
    tgt = rng.standard_normal((2 * 64, 8))
    w = (rng.random(2 * 64) > 0.3).astype(float)

    def loss():
        return net.loss_grad(net.forward(x), tgt, w, 3)[0]

    out = net.forward(x)
    _, dout = net.loss_grad(out, tgt, w, 3)
    gw, gb = net.backward(dout)
    eps = 1e-6
    for li, L in enumerate(net.layers):
        fan = (9 if L.k == 3 else 1) * L.cin
        for (o, j) in [(0, 0), (L.w.shape[0] - 1, fan - 1), (L.w.shape[0] // 2, fan // 2)]:
            keep = L.w[o, j]
            L.w[o, j] = keep + eps
            up = loss()
            L.w[o, j] = keep - eps
            dn = loss()
            L.w[o, j] = keep
            fd = (up - dn) / (2 * eps)
            assert abs(fd - gw[li][o, j]) <= 1e-6 * max(1e-3, abs(fd)), (li, o, j, fd, gw[li][o, j])
        keep = L.b[0]
        L.b[0] = keep + eps
        up = loss()
        L.b[0] = keep - eps
        dn = loss()
        L.b[0] = keep
        fd = (up - dn) / (2 * eps)
        assert abs(fd - gb[li][0]) <= 1e-6 * max(1e-3, abs(fd)), (li, fd, gb[li][0])


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -3.14159, 0.0])
    got = R.bf16(vals)
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == 1.0 + 2 ** -6 and got[3] == 1.0
    assert abs(got[4] + 3.14159) < 2 ** -6 and got[5] == 0.0


def test_encodings_round_trip():
    from vortexlab_b200 import warmstart as WS
    d, u = 20, 0.05
    nx, ny = 20 * d + 2, 10 * d + 2
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny))
    ux = u * (1.0 + 0.3 * np.sin(X / 37.0) * np.cos(Y / 23.0))
    uy = u * 0.2 * np.cos(X / 29.0)
    rho = 1.0 + 0.001 * np.sin(Y / 17.0)
    tgt = WS.encode_target(rho, ux, uy, d, u)
    r2, ux2, uy2 = WS.decode_to_lattice(tgt, nx, ny, d, u)
    inner = (slice(3, -3), slice(3, -3))
    assert np.max(np.abs(ux2 - ux)[inner]) < 2e-3 * u
    assert np.max(np.abs(uy2 - uy)[inner]) < 2e-3 * u
    assert np.max(np.abs(r2 - rho)[inner]) < 2e-6
    flags = np.zeros((ny, nx), np.uint8)
    flags[(X - 100.5) ** 2 + (Y - 100.5) ** 2 < 100] = 2
    inp = WS.encode_input(flags, d, 125.0)
    assert inp.shape == (WS.H, WS.W, WS.CIN) and 0.003 < inp[..., 0].mean() < 0.005
    assert np.all(inp[..., 1] == 0.0)


def test_next_lift_max_predicts_the_next_peak():
    """On a sinusoidal lift with a fast ripple and a slowly growing amplitude, the predicted stop
    lands within 4 % of a period of a true maximum of the underlying oscillation."""
    from vortexlab_b200 import warmstart as WS
    dt = 0.01
    t = np.arange(1, 8001) * dt
    f0 = 0.2
    base = (0.3 + 0.002 * t) * np.sin(2 * np.pi * f0 * t + 0.4) + 0.05
    cl = base + 0.004 * np.sin(2 * np.pi * 7.3 * t)
    for now in (4000, 4317, 5555):
        s = WS.next_lift_max(cl[:now], dt, now)
        assert now <= s <= now + int(1.05 / f0 / dt)
        phase = (2 * np.pi * f0 * s * dt + 0.4) / (2 * np.pi) % 1.0      # a maximum is at phase 0.25
        assert abs(phase - 0.25) < 0.04, (now, s, phase)
    assert WS.next_lift_max(np.full(4000, 0.02), dt, 4000) == 4000
