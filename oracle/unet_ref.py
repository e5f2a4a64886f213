"""CPU FP64 restatement of the warm-start network (test infrastructure only: the tests use it to
check the device forward pass and gradients; nothing in the product imports it).

The network has no counterpart in the reference (vortexlab starts every run from rest or from the
inflow profile through Sim::init, src/sim.rs:357-371); this file restates the device network's own
definition:

- activations NHWC, row r = (b * H + y) * W + x;
- 3x3 convolution, padding 1, stride 1 or 2 (output size ceil(H / s)); its weight matrix is
  [cout, kp] with columns in (ky, kx, c) order, zero-padded to kp (a multiple of 64); a 1x1
  convolution has kp = cin;
- encoder level l: conv(stride 1 if l == 0 else 2) + ReLU, conv + ReLU;
- decoder level l (from levels - 2 down to 0): nearest 2x upsampling of the level below,
  concatenated as [upsampled, encoder level l], conv + ReLU, conv + ReLU;
- head: 1x1 convolution without activation;
- loss: inv_count * sum over rows r and channels c < cuse of w_r (out - target)^2.

With ``mimic_bf16`` the values the device rounds to BF16 are rounded here too (the layer outputs
after ReLU, the output gradients dz of every layer); everything else stays FP64.
"""
from __future__ import annotations

import numpy as np


def bf16(a):
    """Round to the nearest BF16 value (ties to even), through FP32."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64).reshape(f.shape)


def kp_for(cin, k):
    return (9 * cin + 63) // 64 * 64 if k == 3 else cin


def im2col(x, stride, kp):
    B, H, W, C = x.shape
    Ho, Wo = (H + stride - 1) // stride, (W + stride - 1) // stride
    xp = np.zeros((B, H + 2, W + 2, C))
    xp[:, 1:-1, 1:-1] = x
    cols = np.zeros((B, Ho, Wo, kp))
    for ky in range(3):
        for kx in range(3):
            j = (ky * 3 + kx) * C
            cols[..., j:j + C] = xp[:, ky:ky + stride * (Ho - 1) + 1:stride, kx:kx + stride * (Wo - 1) + 1:stride, :]
    return cols.reshape(B * Ho * Wo, kp)


def col2im(dcols, shape, stride):
    B, H, W, C = shape
    Ho, Wo = (H + stride - 1) // stride, (W + stride - 1) // stride
    d = dcols.reshape(B, Ho, Wo, -1)
    dxp = np.zeros((B, H + 2, W + 2, C))
    for ky in range(3):
        for kx in range(3):
            j = (ky * 3 + kx) * C
            dxp[:, ky:ky + stride * (Ho - 1) + 1:stride, kx:kx + stride * (Wo - 1) + 1:stride, :] += d[..., j:j + C]
    return dxp[:, 1:-1, 1:-1]


def up2(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up2_bwd(d):
    B, H2, W2, C = d.shape
    return d.reshape(B, H2 // 2, 2, W2 // 2, 2, C).sum(axis=(2, 4))


class Layer:
    def __init__(self, w, b, cin, stride, relu, k):
        self.w, self.b, self.cin, self.stride, self.relu, self.k = w, b, cin, stride, relu, k


def architecture(levels, c0, cin, cout):
    """(cin, cout, stride, relu, k) of every layer, in the device network's order."""
    ch = [c0 * 2 ** l for l in range(levels)]
    out = []
    for l in range(levels):
        out.append((cin if l == 0 else ch[l - 1], ch[l], 1 if l == 0 else 2, True, 3))
        out.append((ch[l], ch[l], 1, True, 3))
    for l in range(levels - 2, -1, -1):
        out.append((ch[l + 1] + ch[l], ch[l], 1, True, 3))
        out.append((ch[l], ch[l], 1, True, 3))
    out.append((ch[0], cout, 1, False, 1))
    return out


class UNetRef:
    def __init__(self, levels, c0, cin, cout, weights, biases, mimic_bf16=False):
        self.levels, self.c0, self.cin, self.cout = levels, c0, cin, cout
        self.ch = [c0 * 2 ** l for l in range(levels)]
        self.mimic = mimic_bf16
        self.layers = [Layer(np.asarray(w, np.float64), np.asarray(b, np.float64), ci, s, r, k)
                       for (ci, co, s, r, k), w, b in zip(architecture(levels, c0, cin, cout), weights, biases)]

    def _r(self, a):
        return bf16(a) if self.mimic else a

    def _conv(self, L, x):
        B, H, W, _ = x.shape
        if L.k == 3:
            cols = im2col(x, L.stride, L.w.shape[1])
            Ho, Wo = (H + L.stride - 1) // L.stride, (W + L.stride - 1) // L.stride
        else:
            cols = x.reshape(B * H * W, -1)
            Ho, Wo = H, W
        z = cols @ L.w.T + L.b
        y = self._r(np.maximum(z, 0.0)) if L.relu else z
        return y.reshape(B, Ho, Wo, -1), (x, cols, y)

    def _conv_bwd(self, L, cache, dy):
        x, cols, y = cache
        dy = dy.reshape(y.shape)
        dz = dy * (y > 0) if L.relu else dy
        dz = self._r(dz)
        gw = dz.T @ cols
        gb = dz.sum(axis=0)
        dcols = dz @ L.w
        if L.k == 3:
            dx = col2im(dcols, x.shape, L.stride)
        else:
            dx = dcols.reshape(x.shape)
        return dx, gw, gb

    def forward(self, x):
        """x: [B, H, W, cin]. Returns [B * H * W, cout]."""
        self.caches = []
        Ls = iter(self.layers)
        e = []
        cur = x
        for l in range(self.levels):
            for _ in range(2):
                cur, c = self._conv(next(Ls), cur)
                self.caches.append(c)
            e.append(cur)
        d = e[-1]
        for l in range(self.levels - 2, -1, -1):
            cat = np.concatenate([up2(d), e[l]], axis=3)
            for _ in range(2):
                cat, c = self._conv(next(Ls), cat)
                self.caches.append(c)
            d = cat
        out, c = self._conv(next(Ls), d)
        self.caches.append(c)
        return out.reshape(-1, self.cout)

    def loss_grad(self, out, tgt, w, cuse):
        m = np.zeros_like(out)
        m[:, :cuse] = 1.0
        inv = 1.0 / (w.sum() * cuse)
        diff = (out - tgt) * m
        loss = inv * float((w[:, None] * diff * diff).sum())
        dout = 2.0 * inv * w[:, None] * diff
        return loss, dout

    def backward(self, dout):
        """Returns (gw, gb) lists in layer order for the last forward."""
        n = len(self.layers)
        gw, gb = [None] * n, [None] * n
        i = n - 1
        d, gw[i], gb[i] = self._conv_bwd(self.layers[i], self.caches[i], dout)
        skips = {}
        i -= 1
        for l in range(0, self.levels - 1):
            for _ in range(2):
                d, gw[i], gb[i] = self._conv_bwd(self.layers[i], self.caches[i], d)
                i -= 1
            cup = self.ch[l + 1]
            skips[l] = d[..., cup:]
            d = up2_bwd(d[..., :cup])
        for l in range(self.levels - 1, -1, -1):
            if l in skips:
                d = d + skips[l]
            for _ in range(2):
                d, gw[i], gb[i] = self._conv_bwd(self.layers[i], self.caches[i], d)
                i -= 1
        assert i == -1
        return gw, gb
