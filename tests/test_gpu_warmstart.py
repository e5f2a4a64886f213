"""The warm-start network's device kernels: the gathers and elementwise kernels against numpy, and
the whole network's forward pass and gradients (im2col + tcgen05 BF16 GEMMs, FP32 accumulation)
against the CPU FP64 restatement in oracle/unet_ref.py, itself checked by finite differences."""
import ctypes as C

import numpy as np
import pytest

from oracle import unet_ref as R

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _ok(V, rc):
    assert rc == 0, V._lib.last_error()


@pytest.mark.parametrize("stride,H,W,Cc", [(1, 8, 12, 4), (2, 8, 12, 8), (2, 6, 10, 3)])
def test_im2col_col2im(gpu, stride, H, W, Cc):
    V = gpu
    import torch
    from vortexlab_b200 import warmstart as WS
    rng = np.random.default_rng(stride * 100 + Cc)
    x = rng.standard_normal((2, H, W, Cc)).astype(np.float32)
    kp = R.kp_for(Cc, 3)
    xb = WS.bf16_upload(x)
    Ho, Wo = (H + stride - 1) // stride, (W + stride - 1) // stride
    cols = torch.zeros(2 * Ho * Wo, kp, dtype=torch.bfloat16, device="cuda")
    _ok(V, V.lib.vl_nn_im2col(_p(xb), 2, H, W, Cc, stride, kp, _p(cols), None))
    ref = R.im2col(R.bf16(x), stride, kp)
    assert np.array_equal(cols.float().cpu().numpy().astype(np.float64), ref)
    d = rng.standard_normal(ref.shape).astype(np.float32)
    dt = torch.from_numpy(d).cuda()
    dx = torch.full((2, H, W, Cc), 7.0, device="cuda")
    _ok(V, V.lib.vl_nn_col2im(_p(dt), 2, H, W, Cc, stride, kp, _p(dx), 0, None))
    dref = R.col2im(d.astype(np.float64), x.shape, stride)
    assert np.max(np.abs(dx.cpu().numpy() - dref)) < 1e-5
    _ok(V, V.lib.vl_nn_col2im(_p(dt), 2, H, W, Cc, stride, kp, _p(dx), 1, None))
    assert np.max(np.abs(dx.cpu().numpy() - 2 * dref)) < 2e-5


def test_input_gradient_by_mirrored_weights(gpu):
    """For a stride-1 3x3 layer, im2col(dZ) times the mirrored weights equals col2im(dZ W)."""
    V = gpu
    import torch
    from vortexlab_b200 import warmstart as WS
    rng = np.random.default_rng(21)
    B, H, W, cin, cout = 2, 8, 16, 24, 40
    kp, kpf = R.kp_for(cin, 3), R.kp_for(cout, 3)
    w = np.zeros((cout, kp), np.float32)
    w[:, :9 * cin] = rng.standard_normal((cout, 9 * cin))
    dz = rng.standard_normal((B * H * W, cout)).astype(np.float32)
    wb, dzb = WS.bf16_upload(w), WS.bf16_upload(dz)
    wf = torch.zeros(cin, kpf, dtype=torch.bfloat16, device="cuda")
    _ok(V, V.lib.vl_nn_flip_weights(_p(wb), cout, cin, kp, kpf, _p(wf), None))
    cols = torch.zeros(B * H * W, kpf, dtype=torch.bfloat16, device="cuda")
    _ok(V, V.lib.vl_nn_im2col(_p(dzb), B, H, W, cout, 1, kpf, _p(cols), None))
    dx = torch.zeros(B * H * W, cin, device="cuda")
    WS.gemm(cols, kpf, wf, kpf, B * H * W, cin, kpf, dx, cin)
    torch.cuda.synchronize()
    ref = R.col2im(R.bf16(dz) @ R.bf16(w), (B, H, W, cin), 1).reshape(-1, cin)
    assert _rel(dx.cpu().numpy(), ref) < 1e-5


def test_elementwise_kernels(gpu):
    V = gpu
    import torch
    from vortexlab_b200 import warmstart as WS
    rng = np.random.default_rng(7)
    B, H, W, Cc, ctot = 2, 4, 6, 5, 9
    x = rng.standard_normal((B, H, W, Cc)).astype(np.float32)
    xb = WS.bf16_upload(x)
    y = torch.zeros(B * 2 * H * 2 * W, ctot, dtype=torch.bfloat16, device="cuda")
    _ok(V, V.lib.vl_nn_up2(_p(xb), B, H, W, Cc, _p(y), ctot, 3, None))
    up = R.up2(R.bf16(x)).reshape(-1, Cc)
    assert np.array_equal(y.float().cpu().numpy()[:, 3:8], up)
    dy = rng.standard_normal((B * 4 * H * W, ctot)).astype(np.float32)
    dyt = torch.from_numpy(dy).cuda()
    dx = torch.zeros(B * H * W, Cc, device="cuda")
    _ok(V, V.lib.vl_nn_up2_bwd(_p(dyt), B, H, W, Cc, ctot, 3, _p(dx), 0, None))
    ref = R.up2_bwd(dy[:, 3:8].reshape(B, 2 * H, 2 * W, Cc).astype(np.float64)).reshape(-1, Cc)
    assert np.max(np.abs(dx.cpu().numpy() - ref)) < 1e-5
    # channel copy and slice
    z = torch.zeros(B * H * W, ctot, dtype=torch.bfloat16, device="cuda")
    _ok(V, V.lib.vl_nn_copy_channels(_p(xb), B * H * W, Cc, _p(z), ctot, 4, None))
    assert np.array_equal(z.float().cpu().numpy()[:, 4:9], R.bf16(x).reshape(-1, Cc))
    s = torch.ones(B * H * W, 3, device="cuda")
    _ok(V, V.lib.vl_nn_slice_channels(_p(dyt), B * H * W, ctot, 2, 3, _p(s), 1, None))
    assert np.allclose(s.cpu().numpy(), 1.0 + dy[:B * H * W, 2:5], atol=1e-6)
    # ReLU backward with the transposed copy, bias gradient, transpose
    Rn, Cn = 70, 40
    g = rng.standard_normal((Rn, Cn)).astype(np.float32)
    act = WS.bf16_upload(rng.standard_normal((Rn, Cn)).astype(np.float32))
    dz = torch.zeros(Rn, Cn, dtype=torch.bfloat16, device="cuda")
    dzt = torch.zeros(Cn, Rn, dtype=torch.bfloat16, device="cuda")
    gt = torch.from_numpy(g).cuda()
    colsum = torch.zeros(Cn, (Rn + 31) // 32, device="cuda")
    _ok(V, V.lib.vl_nn_act_bwd(_p(gt), _p(act), Rn, Cn, 1, _p(dz), _p(dzt), _p(colsum), None))
    expect = R.bf16(g * (act.float().cpu().numpy() > 0))
    assert np.array_equal(dz.float().cpu().numpy(), expect)
    assert np.array_equal(dzt.float().cpu().numpy(), expect.T)
    db = torch.zeros(Cn, device="cuda")
    _ok(V, V.lib.vl_nn_bias_grad(_p(colsum), Rn, Cn, _p(db), None))
    assert np.allclose(db.cpu().numpy(), expect.sum(axis=0), atol=1e-4)
    tt = torch.zeros(Rn, Cn, dtype=torch.bfloat16, device="cuda")
    _ok(V, V.lib.vl_nn_transpose_bf16(_p(dzt), Cn, Rn, _p(tt), None))
    assert torch.equal(tt, dz)


def test_mse_and_adam(gpu):
    V = gpu
    import torch
    rng = np.random.default_rng(9)
    Rn, Cc, cu = 1000, 8, 3
    out = rng.standard_normal((Rn, Cc)).astype(np.float32)
    tgt = rng.standard_normal((Rn, cu)).astype(np.float32)
    w = (rng.random(Rn) > 0.2).astype(np.float32)
    inv = 1.0 / (w.sum() * cu)
    dout = torch.zeros(Rn, Cc, device="cuda")
    part = torch.zeros(64, dtype=torch.float64, device="cuda")
    t = [torch.from_numpy(a).cuda() for a in (out, tgt, w)]
    _ok(V, V.lib.vl_nn_mse(_p(t[0]), _p(t[1]), _p(t[2]), Rn, Cc, cu, inv, _p(dout), _p(part), 64, None))
    d = out[:, :cu].astype(np.float64) - tgt
    assert abs(part.cpu().numpy().sum() - inv * (w[:, None] * d * d).sum()) < 1e-9
    ref = np.zeros((Rn, Cc))
    ref[:, :cu] = 2 * inv * w[:, None] * d
    assert np.max(np.abs(dout.cpu().numpy() - ref)) < 1e-6 * np.max(np.abs(ref))
    n = 1000
    wv, gv = rng.standard_normal(n).astype(np.float32), rng.standard_normal(n).astype(np.float32)
    m, v = np.zeros(n, np.float32), np.zeros(n, np.float32)
    tw, tg, tm, tv = (torch.from_numpy(a.copy()).cuda() for a in (wv, gv, m, v))
    wb = torch.zeros(n, dtype=torch.bfloat16, device="cuda")
    for step in (1, 2):
        _ok(V, V.lib.vl_nn_adam(_p(tw), _p(tg), _p(tm), _p(tv), n, 1e-2, 0.9, 0.999, 1e-8, step, _p(wb), None))
        m = 0.9 * m + 0.1 * gv
        v = 0.999 * v + 0.001 * gv * gv
        wv = wv - 1e-2 * (m / (1 - 0.9 ** step)) / (np.sqrt(v / (1 - 0.999 ** step)) + 1e-8)
    assert np.max(np.abs(tw.cpu().numpy() - wv)) < 1e-6
    assert np.array_equal(wb.float().cpu().numpy(), R.bf16(tw.cpu().numpy()))


def _unet_case(V, levels, c0, B, h, w, seed):
    import torch
    from vortexlab_b200 import warmstart as WS
    net = WS.UNet(levels=levels, c0=c0, cin=4, cout=8, seed=seed)
    for c in net.layers():       # non-zero biases so that the bias path is exercised
        c.b.copy_(torch.linspace(-0.1, 0.1, c.cout))
    net.alloc(B, h, w)
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((B, h, w, 4)).astype(np.float32)
    Rn = B * h * w
    tgt = rng.standard_normal((Rn, 3)).astype(np.float32)
    wt = (rng.random(Rn) > 0.25).astype(np.float32)
    inv = 1.0 / (wt.sum() * 3)
    out = net.forward(WS.bf16_upload(x))
    dout = torch.zeros(Rn, 8, device="cuda")
    part = torch.zeros(64, dtype=torch.float64, device="cuda")
    tt, wtt = torch.from_numpy(tgt).cuda(), torch.from_numpy(wt).cuda()
    _ok(V, V.lib.vl_nn_mse(_p(out), _p(tt), _p(wtt), Rn, 8, 3, inv, _p(dout), _p(part), 64, None))
    net.backward(dout)
    torch.cuda.synchronize()
    net.check_errors()
    got = dict(out=out.cpu().numpy().astype(np.float64), loss=float(part.cpu().numpy().sum()),
               gw=[c.gw.cpu().numpy() for c in net.layers()], gb=[c.gb.cpu().numpy() for c in net.layers()],
               net=net)
    weights = [c.wb.float().cpu().numpy() for c in net.layers()]
    biases = [c.b.cpu().numpy() for c in net.layers()]
    tpad = np.zeros((Rn, 8))
    tpad[:, :3] = tgt
    refs = {}
    for mimic in (True, False):
        ref = R.UNetRef(levels, c0, 4, 8, weights, biases, mimic_bf16=mimic)
        o = ref.forward(R.bf16(x))
        loss, d = ref.loss_grad(o, tpad, wt.astype(np.float64), 3)
        gw, gb = ref.backward(d)
        refs[mimic] = dict(out=o, loss=loss, gw=gw, gb=gb)
    return got, refs


@pytest.mark.parametrize("levels,c0,B,h,w", [(3, 8, 2, 16, 32)])
def test_unet_gradients_match_cpu_fp64(gpu, levels, c0, B, h, w):
    """Forward output, loss and every layer's weight and bias gradient of the device network
    against the FP64 restatement, relative L2 error. When the restatement rounds the same values to
    BF16 as the device (the layer outputs and the output gradients) everything agrees within 2e-3:
    the rest is FP32 against FP64 accumulation. Without that rounding the forward pass stays within
    2e-2, and the gradients within 0.25: a weight gradient is a sum over every pixel of products of
    both signs, so the 2^-9 relative rounding of each BF16 term is amplified by the cancellation
    (by about sqrt(pixels) for a network at its random initialisation)."""
    got, refs = _unet_case(gpu, levels, c0, B, h, w, seed=levels * 10 + c0)
    errs = {}
    for mimic in (True, False):
        ref = refs[mimic]
        errs[mimic] = dict(out=_rel(got["out"], ref["out"]), loss=abs(got["loss"] - ref["loss"]) / ref["loss"],
                           gw=[_rel(a, b) for a, b in zip(got["gw"], ref["gw"])],
                           gb=[_rel(a, b) for a, b in zip(got["gb"], ref["gb"])])
    e = errs[True]
    assert e["out"] < 2e-3 and e["loss"] < 2e-3 and max(e["gw"]) < 2e-3 and max(e["gb"]) < 2e-3, e
    e = errs[False]
    assert e["out"] < 2e-2 and e["loss"] < 2e-2 and max(e["gw"]) < 0.25 and max(e["gb"]) < 0.25, e


def test_training_fits_a_small_set(gpu):
    """Adam on the device kernels drives the masked MSE of 8 fixed samples down by 10x."""
    V = gpu
    import torch
    from vortexlab_b200 import warmstart as WS
    net = WS.UNet(levels=3, c0=16, cin=4, cout=8, seed=5)
    B, h, w = 8, 32, 64
    net.alloc(B, h, w)
    rng = np.random.default_rng(11)
    x = rng.standard_normal((B, h, w, 4)).astype(np.float32)
    X, Y = np.meshgrid(np.linspace(-1, 1, w), np.linspace(-1, 1, h))
    tgt = np.stack([np.stack([np.sin(3 * X + b), np.cos(2 * Y - b), X * Y], -1) for b in range(B)])
    tgt = tgt.reshape(-1, 3).astype(np.float32)
    Rn = B * h * w
    wt = np.ones(Rn, np.float32)
    xb = WS.bf16_upload(x)
    tt, wtt = torch.from_numpy(tgt).cuda(), torch.from_numpy(wt).cuda()
    dout = torch.zeros(Rn, 8, device="cuda")
    part = torch.zeros(64, dtype=torch.float64, device="cuda")
    losses = []
    for step in range(1, 301):
        out = net.forward(xb)
        _ok(V, V.lib.vl_nn_mse(_p(out), _p(tt), _p(wtt), Rn, 8, 3, 1.0 / (Rn * 3), _p(dout), _p(part), 64, None))
        net.backward(dout)
        net.adam(step, 2e-3)
        if step in (1, 300):
            losses.append(float(part.cpu().numpy().sum()))
    net.check_errors()
    assert losses[1] < 0.1 * losses[0], losses


def test_unet_layers_match_cpu_fp64_at_full_width(gpu):
    """The full-width network (4 levels, 32..256 channels, K up to 3456): every layer's output
    against the FP64 product of the layer's own device input and BF16 weights (at most one BF16
    rounding step apart), and every weight and bias gradient against the FP64 product of the
    layer's own device output gradient and input (FP32 accumulation: 1e-5). End to end, where
    rounding differences in one layer carry into the next, the output stays within 1e-2 and the
    gradients within 0.1 of the restatement that rounds like the device."""
    got, refs = _unet_case(gpu, 4, 32, 1, 16, 32, seed=4)
    import torch
    from vortexlab_b200 import warmstart as WS
    net = got["net"]
    for i, c in enumerate(net.layers()):
        x = c.x.float().cpu().numpy().astype(np.float64)
        Bn = x.size // (c.h * c.wd * c.cin)
        x = x.reshape(Bn, c.h, c.wd, c.cin)
        cols = R.im2col(x, c.stride, c.kp) if c.k == 3 else x.reshape(-1, c.cin)
        z = cols @ c.wb.float().cpu().numpy().astype(np.float64).T + c.b.cpu().numpy()
        y = c.y.float().cpu().numpy().astype(np.float64)
        if c.relu:
            ref = np.maximum(z, 0.0)
            assert np.all(np.abs(y - ref) <= 2.0 ** -8 * np.abs(ref) + 1e-6), i
        else:
            assert np.max(np.abs(y - z)) <= 1e-5 * max(1.0, np.max(np.abs(z))), i
        dz = c.dz.float().cpu().numpy().astype(np.float64)
        assert _rel(c.gw.cpu().numpy(), dz.T @ cols) < 1e-5, i
        assert _rel(c.gb.cpu().numpy(), dz.sum(axis=0)) < 1e-5, i
    ref = refs[True]
    assert _rel(got["out"], ref["out"]) < 1e-2
    assert max(_rel(a, b) for a, b in zip(got["gw"], ref["gw"])) < 0.1
