"""Learned warm start: a convolutional network that maps a tunnel's body mask and Reynolds number
to a developed wake (u_x, u_y, rho at a lift maximum), so that a run starts from it (Sim::init,
src/sim.rs:357-371, the equilibria of the predicted fields) instead of from rest with an inflow
ramp. The uniform start stays the fallback: a tunnel without a prediction runs as before.

Network: a U-Net of `levels` levels on a 256 x 128 grid (the tunnel's 20 D x 10 D fluid region
resampled). Level l has c0 * 2^l channels; each level is two 3x3 convolutions with ReLU (the first
of a lower level has stride 2); the decoder upsamples 2x (nearest), concatenates the encoder
level, and applies two 3x3 convolutions; a 1x1 convolution gives the output. With levels = 4 and
c0 = 32 it has 1.95 M parameters.

Every convolution is an im2col gather plus a BF16 GEMM on the tcgen05 tensor cores with FP32
accumulation (vl_nn_gemm_bf16); its backward pass is two more GEMMs (weights: cols^T dz, with both
operands read MN-major where they lie, no transposes; data: the im2col of dz times the mirrored
weights for stride-1 layers, dz W^T then col2im for stride 2).
Master weights and Adam moments are FP32. torch provides device memory only: every arithmetic
operation on the device runs in this library's kernels.

Inputs (4 channels): body mask, (Re - 125) / 75, x and y in [-1, 1]. Targets / outputs (the first
3 of COUT channels): u_x / u - 1, u_y / u, 2 (rho - 1) / (3 u^2).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time
from dataclasses import dataclass, field

import numpy as np

from ._lib import check, lib

H, W = 128, 256   # network grid (rows, columns)
CIN = 4           # input channels
COUT = 8          # output channels (the first NT are used; 8 keeps every row 16-byte aligned)
NT = 3            # target channels

EPI_ACCUM, EPI_BIAS, EPI_RELU, EPI_BF16 = 1, 2, 4, 8


def _t():
    import torch
    return torch


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _fp(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_float)) if t is not None else None


def _kp(k):
    return (k + 63) // 64 * 64


def _bn(n):
    for b in (32, 64, 128, 256):
        if n <= b:
            return b
    return 256


class _Err:
    """Device flag that a tensor-core GEMM tile sets when one of its bounded waits runs out."""

    def __init__(self):
        torch = _t()
        self.t = torch.zeros(1, dtype=torch.int32, device="cuda")

    def ptr(self):
        return C.cast(C.c_void_p(self.t.data_ptr()), C.POINTER(C.c_int))


A_MN, B_MN = 16, 32   # operand stored [K][M] / [K][N] (MN-major) instead of [M][K] / [N][K]


def gemm(a, lda, b, ldb, M, N, K, out, ldc, flags=0, bias=None, err=None):
    """out = epilogue(A B^T) on the tensor cores (all device tensors); A is a[M, K] (or a[K, M]
    with A_MN), B is b[N, K] (or b[K, N] with B_MN)."""
    bn = max(64, _bn(N)) if flags & B_MN else _bn(N)
    check(lib.vl_nn_gemm_bf16(_p(a), lda, _p(b), ldb, M, N, K, _p(out), ldc, _fp(bias), flags, bn,
                              err.ptr() if err is not None else None, None))


class Conv:
    """3x3 (padding 1, stride 1 or 2) or 1x1 convolution + bias (+ ReLU) over NHWC BF16
    activations. Weights W[cout, kp], columns in (ky, kx, c) order, zero-padded to kp. The FP32
    master copy, its gradient and the Adam moments are kept transposed, [kp, cout]: the weight
    gradient is then the GEMM colsT dzT^T with the long kp side on the tensor-core tile's 128 rows,
    and Adam writes the BF16 [kp, cout] operand directly."""

    def __init__(self, cin, cout, stride=1, relu=True, k=3, seed=0):
        torch = _t()
        self.cin, self.cout, self.stride, self.relu, self.k = cin, cout, stride, relu, k
        self.kp = _kp(9 * cin) if k == 3 else cin
        fan_in = (9 if k == 3 else 1) * cin
        g = torch.Generator().manual_seed(seed)
        w = torch.zeros(cout, self.kp)
        w[:, :fan_in] = torch.randn(cout, fan_in, generator=g) * math.sqrt(2.0 / fan_in) * (1.0 if relu else 0.1)
        self.wt = w.t().contiguous().cuda()          # FP32 master, [kp, cout]
        self.b = torch.zeros(cout, device="cuda")
        self.gwt = torch.zeros_like(self.wt)
        self.gb = torch.zeros_like(self.b)
        self.mw, self.vw = torch.zeros_like(self.wt), torch.zeros_like(self.wt)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)
        self.wb = torch.zeros(cout, self.kp, dtype=torch.bfloat16, device="cuda")
        self.wbt = torch.zeros(self.kp, cout, dtype=torch.bfloat16, device="cuda")
        self.sync_weights()

    @property
    def params(self):
        return self.cout * (9 if self.k == 3 else 1) * self.cin + self.cout

    @property
    def w(self):
        """FP32 weights [cout, kp] (a view of the transposed master copy)."""
        return self.wt.t()

    @property
    def gw(self):
        """Weight gradient [cout, kp] (a view)."""
        return self.gwt.t()

    def sync_weights(self):
        """BF16 copies of the FP32 master weights, [kp, cout] and transposed [cout, kp]."""
        check(lib.vl_nn_f32_to_bf16(_p(self.wt), self.wt.numel(), _p(self.wbt), None))
        check(lib.vl_nn_transpose_bf16(_p(self.wbt), self.kp, self.cout, _p(self.wb), None))

    def alloc(self, B, h, w):
        torch = _t()
        self.B, self.h, self.wd = B, h, w
        self.ho, self.wo = (h + self.stride - 1) // self.stride, (w + self.stride - 1) // self.stride
        self.rows = B * self.ho * self.wo
        bf = dict(dtype=torch.bfloat16, device="cuda")
        self.cols = torch.zeros(self.rows, self.kp, **bf) if self.k == 3 else None
        self.flip = self.k == 3 and self.stride == 1
        if self.flip:       # input gradient as a convolution of dz with mirrored weights
            self.kpf = _kp(9 * self.cout)
            self.dcols = torch.zeros(self.rows, self.kpf, **bf)
            self.wf = torch.zeros(self.cin, self.kpf, **bf)
        elif self.k == 3:   # stride 2: dz W^T, then col2im
            self.dcols = torch.zeros(self.rows, self.kp, dtype=torch.float32, device="cuda")
        self.y = torch.zeros(self.rows, self.cout, **bf) if self.relu else \
            torch.zeros(self.rows, self.cout, dtype=torch.float32, device="cuda")
        self.dz = torch.zeros(self.rows, self.cout, **bf)
        self.colsum = torch.zeros(self.cout, (self.rows + 31) // 32, dtype=torch.float32, device="cuda")

    def forward(self, x, err):
        """x: BF16 [B, h, w, cin] (contiguous). Returns y: BF16 (ReLU layers) or FP32 [rows, cout]."""
        self.x = x
        if self.k == 3:
            check(lib.vl_nn_im2col(_p(x), self.B, self.h, self.wd, self.cin, self.stride, self.kp, _p(self.cols), None))
            a = self.cols
        else:
            a = x
        flags = EPI_BIAS | ((EPI_RELU | EPI_BF16) if self.relu else 0)
        gemm(a, self.kp, self.wb, self.kp, self.rows, self.cout, self.kp, self.y, self.cout, flags, self.b, err)
        return self.y

    def backward(self, dy, dx, accumulate, err, need_dx=True):
        """dy: FP32 [rows, cout], the gradient of the layer output. Writes (or, with `accumulate`,
        adds) the input gradient into dx (FP32 [B, h, w, cin]); sets gw and gb."""
        check(lib.vl_nn_act_bwd(_p(dy), _p(self.y) if self.relu else None, self.rows, self.cout, int(self.relu),
                                _p(self.dz), None, _p(self.colsum), None))
        check(lib.vl_nn_bias_grad(_p(self.colsum), self.rows, self.cout, _p(self.gb), None))
        # weight gradient gw^T [kp, cout] = cols^T dz: both operands read MN-major as they lie
        a = self.cols if self.k == 3 else self.x
        gemm(a, self.kp, self.dz, self.cout, self.kp, self.cout, self.rows, self.gwt, self.cout, A_MN | B_MN, None, err)
        if not need_dx:
            return
        if self.flip:
            check(lib.vl_nn_flip_weights(_p(self.wb), self.cout, self.cin, self.kp, self.kpf, _p(self.wf), None))
            check(lib.vl_nn_im2col(_p(self.dz), self.B, self.ho, self.wo, self.cout, 1, self.kpf, _p(self.dcols), None))
            gemm(self.dcols, self.kpf, self.wf, self.kpf, self.rows, self.cin, self.kpf, dx, self.cin,
                 EPI_ACCUM if accumulate else 0, None, err)
        elif self.k == 3:
            gemm(self.dz, self.cout, self.wbt, self.cout, self.rows, self.kp, self.cout, self.dcols, self.kp, 0, None,
                 err)
            check(lib.vl_nn_col2im(_p(self.dcols), self.B, self.h, self.wd, self.cin, self.stride, self.kp, _p(dx),
                                   int(accumulate), None))
        else:
            gemm(self.dz, self.cout, self.wbt, self.cout, self.rows, self.kp, self.cout, dx, self.kp,
                 EPI_ACCUM if accumulate else 0, None, err)

    def adam(self, step, lr, b1=0.9, b2=0.999, eps=1e-8):
        check(lib.vl_nn_adam(_p(self.wt), _p(self.gwt), _p(self.mw), _p(self.vw), self.wt.numel(), lr, b1, b2, eps,
                             step, _p(self.wbt), None))
        check(lib.vl_nn_adam(_p(self.b), _p(self.gb), _p(self.mb), _p(self.vb), self.b.numel(), lr, b1, b2, eps,
                             step, None, None))
        check(lib.vl_nn_transpose_bf16(_p(self.wbt), self.kp, self.cout, _p(self.wb), None))


class UNet:
    """The warm-start network (see the module docstring); layers() gives the layer order shared
    with the CPU FP64 restatement used by the tests."""

    def __init__(self, levels=4, c0=32, cin=CIN, cout=COUT, seed=1):
        self.levels, self.c0, self.cin, self.cout = levels, c0, cin, cout
        ch = [c0 * (2 ** l) for l in range(levels)]
        self.ch = ch
        s = seed * 1000
        self.enc = []
        for l in range(levels):
            a = Conv(cin if l == 0 else ch[l - 1], ch[l], stride=1 if l == 0 else 2, seed=s + 2 * l)
            b = Conv(ch[l], ch[l], seed=s + 2 * l + 1)
            self.enc.append((a, b))
        self.dec = {}
        for l in range(levels - 2, -1, -1):
            a = Conv(ch[l + 1] + ch[l], ch[l], seed=s + 100 + 2 * l)
            b = Conv(ch[l], ch[l], seed=s + 101 + 2 * l)
            self.dec[l] = (a, b)
        self.head = Conv(ch[0], cout, k=1, relu=False, seed=s + 999)
        self.err = _Err()
        self.B = None

    def layers(self):
        out = []
        for a, b in self.enc:
            out += [a, b]
        for l in range(self.levels - 2, -1, -1):
            out += list(self.dec[l])
        return out + [self.head]

    @property
    def params(self):
        return sum(c.params for c in self.layers())

    def alloc(self, B, h=H, w=W):
        if h % (2 ** (self.levels - 1)) or w % (2 ** (self.levels - 1)):
            raise ValueError("the grid must halve evenly at every level")
        torch = _t()
        self.B, self.h, self.w = B, h, w
        hs = [h // (2 ** l) for l in range(self.levels)]
        ws = [w // (2 ** l) for l in range(self.levels)]
        self.hs, self.ws = hs, ws
        for l, (a, b) in enumerate(self.enc):
            a.alloc(B, hs[l - 1] if l else h, ws[l - 1] if l else w)
            b.alloc(B, hs[l], ws[l])
        self.cat, self.dcat = {}, {}
        for l, (a, b) in self.dec.items():
            ctot = self.ch[l + 1] + self.ch[l]
            self.cat[l] = torch.zeros(B * hs[l] * ws[l], ctot, dtype=torch.bfloat16, device="cuda")
            self.dcat[l] = torch.zeros(B * hs[l] * ws[l], ctot, dtype=torch.float32, device="cuda")
            a.alloc(B, hs[l], ws[l])
            b.alloc(B, hs[l], ws[l])
        self.head.alloc(B, h, w)
        f32 = dict(dtype=torch.float32, device="cuda")
        # FP32 gradients: (after the first conv, after the second conv) of every level
        self.g_enc = [(torch.zeros(B * hs[l] * ws[l], self.ch[l], **f32),
                       torch.zeros(B * hs[l] * ws[l], self.ch[l], **f32)) for l in range(self.levels)]
        self.g_dec = {l: (torch.zeros(B * hs[l] * ws[l], self.ch[l], **f32),
                          torch.zeros(B * hs[l] * ws[l], self.ch[l], **f32)) for l in self.dec}

    def forward(self, x):
        """x: BF16 [B, h, w, cin]. Returns FP32 [B * h * w, cout]."""
        err = self.err
        e = []
        cur = x
        for a, b in self.enc:
            cur = b.forward(a.forward(cur, err), err)
            e.append(cur)
        d = e[-1]
        for l in range(self.levels - 2, -1, -1):
            ctot = self.ch[l + 1] + self.ch[l]
            check(lib.vl_nn_up2(_p(d), self.B, self.hs[l + 1], self.ws[l + 1], self.ch[l + 1], _p(self.cat[l]), ctot, 0,
                                None))
            check(lib.vl_nn_copy_channels(_p(e[l]), self.B * self.hs[l] * self.ws[l], self.ch[l], _p(self.cat[l]), ctot,
                                          self.ch[l + 1], None))
            a, b = self.dec[l]
            d = b.forward(a.forward(self.cat[l], err), err)
        return self.head.forward(d, err)

    def backward(self, dout):
        """dout: FP32 [B * h * w, cout], the gradient of the loss with respect to the output."""
        err = self.err
        L = self.levels
        top = self.g_dec[0][1] if L > 1 else self.g_enc[0][1]
        self.head.backward(dout, top, False, err)
        for l in range(0, L - 1):
            a, b = self.dec[l]
            gmid, gout = self.g_dec[l]
            b.backward(gout, gmid, False, err)
            a.backward(gmid, self.dcat[l], False, err)
            R = self.B * self.hs[l] * self.ws[l]
            ctot = self.ch[l + 1] + self.ch[l]
            # concat split: the skip part is the first contribution to encoder level l's output
            check(lib.vl_nn_slice_channels(_p(self.dcat[l]), R, ctot, self.ch[l + 1], self.ch[l],
                                           _p(self.g_enc[l][1]), 0, None))
            # the upsampled part goes to the decoder output one level down (or the encoder bottom)
            dst = self.g_dec[l + 1][1] if (l + 1) in self.dec else self.g_enc[L - 1][1]
            check(lib.vl_nn_up2_bwd(_p(self.dcat[l]), self.B, self.hs[l + 1], self.ws[l + 1], self.ch[l + 1], ctot, 0,
                                    _p(dst), 0, None))
        for l in range(L - 1, -1, -1):
            a, b = self.enc[l]
            gmid, gout = self.g_enc[l]
            b.backward(gout, gmid, False, err)
            if l == 0:
                a.backward(gmid, None, False, err, need_dx=False)
            else:
                a.backward(gmid, self.g_enc[l - 1][1], True, err)

    def adam(self, step, lr):
        for c in self.layers():
            c.adam(step, lr)

    def check_errors(self):
        if int(self.err.t.item()) != 0:
            raise RuntimeError("a tensor-core GEMM tile gave up waiting for its operands")

    def state(self):
        out = {}
        for i, c in enumerate(self.layers()):
            out[f"w{i}"] = c.w.cpu().numpy()
            out[f"b{i}"] = c.b.cpu().numpy()
        return out

    def load(self, st):
        torch = _t()
        for i, c in enumerate(self.layers()):
            c.wt.copy_(torch.from_numpy(np.ascontiguousarray(np.asarray(st[f"w{i}"], np.float32).T)))
            c.b.copy_(torch.from_numpy(np.asarray(st[f"b{i}"], np.float32)))
            c.sync_weights()


PRETRAINED = os.path.join(os.path.dirname(__file__), "data", "warmstart_unet.npz")


def save_bf16(net, path):
    """Writes the network with its weights rounded to BF16 (the values its GEMMs use) and its FP32
    biases: inference from the file is identical to inference from the network."""
    out = {}
    for k, v in net.state().items():
        if k.startswith("w"):
            u = np.ascontiguousarray(v, np.float32).view(np.uint32).astype(np.uint64)
            out[k] = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
        else:
            out[k] = np.asarray(v, np.float32)
    out["config"] = np.array([net.levels, net.c0, net.cin, net.cout], np.int32)
    np.savez_compressed(path, **out)


def load_pretrained(path=PRETRAINED):
    """The network trained on solver-generated wakes (2000 tunnels of seed 0x7EA10001 at 50
    convective units, stopped on a lift peak): weights stored as BF16, biases FP32."""
    z = np.load(path)
    levels, c0, cin, cout = (int(v) for v in z["config"])
    net = UNet(levels=levels, c0=c0, cin=cin, cout=cout)
    st = {}
    for k in z.files:
        if k.startswith("w"):
            st[k] = (z[k].astype(np.uint32) << 16).view(np.float32)
        elif k.startswith("b"):
            st[k] = z[k]
    net.load(st)
    return net


# ---------------------------------------------------------------------------- data encodings
def grid_points(d):
    """Lattice coordinates (x, y) of the network grid's cell centres for a tunnel of frontal
    width d: the fluid region x in [0.5, 20 d + 0.5], y in [0.5, 10 d + 0.5]."""
    xs = 0.5 + (np.arange(W) + 0.5) * (20.0 * d / W)
    ys = 0.5 + (np.arange(H) + 0.5) * (10.0 * d / H)
    return xs, ys


def encode_input(flags, d, re):
    """(H, W, CIN) float32: mask (the nearest lattice cell is solid), Re feature, x and y."""
    xs, ys = grid_points(d)
    ny, nx = flags.shape
    ix = np.clip(np.rint(xs).astype(int), 0, nx - 1)
    iy = np.clip(np.rint(ys).astype(int), 0, ny - 1)
    mask = (flags[np.ix_(iy, ix)] == 2).astype(np.float32)
    out = np.zeros((H, W, CIN), np.float32)
    out[..., 0] = mask
    out[..., 1] = (re - 125.0) / 75.0
    out[..., 2] = np.linspace(-1, 1, W, dtype=np.float32)[None, :]
    out[..., 3] = np.linspace(-1, 1, H, dtype=np.float32)[:, None]
    return out


def _bilinear(f, xs, ys):
    """Samples a field f[ny, nx] at the points (xs[j], ys[i]), clamped to the grid."""
    ny, nx = f.shape
    x0 = np.clip(np.floor(xs).astype(int), 0, nx - 2)
    y0 = np.clip(np.floor(ys).astype(int), 0, ny - 2)
    fx = np.clip(xs - x0, 0, 1)[None, :]
    fy = np.clip(ys - y0, 0, 1)[:, None]
    f00 = f[np.ix_(y0, x0)]
    f01 = f[np.ix_(y0, x0 + 1)]
    f10 = f[np.ix_(y0 + 1, x0)]
    f11 = f[np.ix_(y0 + 1, x0 + 1)]
    return (1 - fy) * ((1 - fx) * f00 + fx * f01) + fy * ((1 - fx) * f10 + fx * f11)


def encode_target(rho, ux, uy, d, u):
    """(H, W, NT) float32 normalised target from lattice fields [ny, nx]."""
    xs, ys = grid_points(d)
    out = np.zeros((H, W, NT), np.float32)
    out[..., 0] = _bilinear(ux, xs, ys) / u - 1.0
    out[..., 1] = _bilinear(uy, xs, ys) / u
    out[..., 2] = 2.0 * (_bilinear(rho, xs, ys) - 1.0) / (3.0 * u * u)
    return out


def decode_to_lattice(pred, nx, ny, d, u):
    """Lattice start fields (rho, ux, uy), each [ny, nx], from a network output (H, W, >= NT)."""
    gx = (np.arange(nx) - 0.5) * (W / (20.0 * d)) - 0.5
    gy = (np.arange(ny) - 0.5) * (H / (10.0 * d)) - 0.5
    ux = u * (1.0 + _bilinear(pred[..., 0].astype(np.float64), gx, gy))
    uy = u * _bilinear(pred[..., 1].astype(np.float64), gx, gy)
    rho = 1.0 + 1.5 * u * u * _bilinear(pred[..., 2].astype(np.float64), gx, gy)
    return rho, ux, uy


# ---------------------------------------------------------------------------- data from the solver
def next_lift_max(cl, dt, now, units=10.0, rel_amp=1e-3):
    """Step count (>= now) at which the lift of a tunnel recorded up to step `now` (cl[i] is the
    lift of step i + 1) will next peak. The shedding period P0 comes from the lift spectrum of the
    trailing `units` convective units (src/signal.rs:92-107); the last complete peak is the lift
    maximum over [now - 1.25 P0, now - 0.25 P0), the one before it the maximum a period earlier,
    and their distance is the period used to step forward. Maxima over whole period-long windows
    are immune to the small fast ripples (pressure waves) riding on the lift. A lift that does not
    oscillate (range below rel_amp (|mean| + 0.01)) gives `now`."""
    from . import signal
    n = min(len(cl), now)
    m = min(n, int(units / dt))
    tail = np.asarray(cl[n - m:n], np.float64)
    if m < 8 or not np.all(np.isfinite(tail)) or np.ptp(tail) < rel_amp * (abs(np.mean(tail)) + 0.01):
        return now
    f = signal.dominant_frequency(tail, dt)[0]
    if not (f > 0 and np.isfinite(f)):
        return now
    p0 = 1.0 / f / dt
    if 2.5 * p0 > n:
        return now
    a, b = int(n - 1.25 * p0), int(n - 0.25 * p0)
    i1 = a + int(np.argmax(cl[a:b]))
    a0, b0 = max(0, int(i1 - 1.5 * p0)), int(i1 - 0.5 * p0)
    i0 = a0 + int(np.argmax(cl[a0:b0]))
    period = float(i1 - i0) if 0.7 * p0 < i1 - i0 < 1.3 * p0 else p0
    last = i1 + 1                          # step count of the last complete peak
    k = max(1, int(np.ceil((now - last) / period)))
    return int(round(last + k * period))


@dataclass
class Dataset:
    x: np.ndarray        # (N, H, W, CIN) float32
    y: np.ndarray        # (N, H, W, NT) float32
    w: np.ndarray        # (N, H, W) float32 (1 on fluid)
    meta: list = field(default_factory=list)
    seconds: float = 0.0

    def split(self, n):
        a = Dataset(self.x[:n], self.y[:n], self.w[:n], self.meta[:n])
        b = Dataset(self.x[n:], self.y[n:], self.w[n:], self.meta[n:])
        return a, b


def generate(cases, precision="f32", chunk=256, extra_units=12.0, log=None):
    """Fields of developed wakes at a lift maximum. Each case runs in a batch for its own length
    (its `steps`); at that step its lift history gives the step of the next lift peak, the tunnel is
    set to end there (vl_batch_set_steps) and the batch runs on until every tunnel has ended; the
    fields are then sampled onto the network grid. `extra_units` bounds the wait for the peak."""
    from .batch import Batch
    t0 = time.perf_counter()
    xs, ys, ws, meta = [], [], [], []
    for c0 in range(0, len(cases), chunk):
        part = cases[c0:c0 + chunk]
        b = Batch(precision)
        cap = [c.steps + int(extra_units * c.tunnel.steps_per_unit()) for c in part]
        for c, n in zip(part, cap):
            b.add(c.tunnel.spec(c.body), n)
        b.build()
        b.autotune(3)
        decide = [c.steps for c in part]
        stop = [None] * len(part)
        while True:
            s = b.global_step()
            for k, c in enumerate(part):
                if stop[k] is None and s >= decide[k]:
                    tn = c.tunnel
                    h = b.force_history(k)
                    cl = 2.0 / (tn.u * tn.u * tn.d) * h[:, 1]
                    stop[k] = min(max(next_lift_max(cl, 1.0 / tn.steps_per_unit(), s), s), cap[k])
                    b.set_steps(k, stop[k])
            pending = [decide[k] for k in range(len(part)) if stop[k] is None]
            if not pending:
                b.run()
                break
            b.run(min(pending) - s)
        for k, c in enumerate(part):
            t, nonfinite, _ = b.status(k)
            if nonfinite:
                continue
            tn = c.tunnel
            h = b.force_history(k)
            cl = h[:, 1]
            w = min(len(cl), int(tn.steps_per_unit() * 10))
            span = np.ptp(cl[-w:])
            phase_err = float((cl[-w:].max() - cl[-1]) / span) if span > 0 else 0.0
            rho, ux, uy = b.macros_field(k)
            x = encode_input(b.flags(k), tn.d, tn.re)
            xs.append(x)
            ys.append(encode_target(rho, ux, uy, tn.d, tn.u))
            ws.append(1.0 - x[..., 0])
            meta.append(dict(d=tn.d, re=tn.re, kind=c.kind, stop=int(t), steps=c.steps, peak_gap=phase_err))
        b.close()
        if log:
            log(f"generated {len(xs)} of {len(cases)} fields, {time.perf_counter() - t0:.1f} s")
    return Dataset(np.stack(xs), np.stack(ys), np.stack(ws).astype(np.float32), meta, time.perf_counter() - t0)


# ---------------------------------------------------------------------------- training / inference
@dataclass
class TrainLog:
    steps: int
    seconds: float
    loss: list


def bf16_upload(a):
    """Uploads a float32 array and rounds it to BF16 on the device with the library's kernel."""
    torch = _t()
    f = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    out = torch.empty(f.shape, dtype=torch.bfloat16, device="cuda")
    check(lib.vl_nn_f32_to_bf16(_p(f), f.numel(), _p(out), None))
    return out


def train(net, data: Dataset, epochs=20, batch=16, lr=1e-3, seed=0, seconds=None, log=None, lr_final=None):
    """Adam on the masked MSE; the dataset lives on the device (inputs BF16, targets FP32). The
    learning rate decays by cosine from lr to lr_final (default lr / 20) over the run."""
    torch = _t()
    n = len(data.x)
    if n < batch:
        raise ValueError("fewer samples than one batch")
    X = bf16_upload(data.x)
    T = torch.from_numpy(np.ascontiguousarray(data.y.reshape(n, -1), np.float32)).cuda()
    Wt = torch.from_numpy(np.ascontiguousarray(data.w.reshape(n, -1), np.float32)).cuda()
    counts = data.w.reshape(n, -1).sum(axis=1)
    net.alloc(batch)
    hw = H * W
    xb = torch.zeros(batch, H, W, CIN, dtype=torch.bfloat16, device="cuda")
    tb = torch.zeros(batch * hw * NT, dtype=torch.float32, device="cuda")
    wb = torch.zeros(batch * hw, dtype=torch.float32, device="cuda")
    dout = torch.zeros(batch * hw, net.cout, dtype=torch.float32, device="cuda")
    blocks = 296
    partial = torch.zeros(blocks, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(seed)
    steps_per_epoch = n // batch
    total = epochs * steps_per_epoch
    lr_final = lr / 20 if lr_final is None else lr_final
    step = 0
    losses = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    done = False
    for ep in range(epochs):
        perm = rng.permutation(n)
        for i in range(steps_per_epoch):
            idx = perm[i * batch:(i + 1) * batch]
            for j, s in enumerate(idx):        # device-to-device copies of the batch's samples
                xb[j].copy_(X[s])
                tb[j * hw * NT:(j + 1) * hw * NT].copy_(T[s])
                wb[j * hw:(j + 1) * hw].copy_(Wt[s])
            count = float(counts[idx].sum()) * NT
            out = net.forward(xb)
            check(lib.vl_nn_mse(_p(out), _p(tb), _p(wb), batch * hw, net.cout, NT, 1.0 / max(count, 1.0), _p(dout),
                                _p(partial), blocks, None))
            net.backward(dout)
            step += 1
            cur = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * min(step, total) / total))
            net.adam(step, cur)
            if step % 50 == 0 or step == 1:
                losses.append((step, float(partial.cpu().numpy().sum())))
                if log:
                    log(f"step {step}/{total} loss {losses[-1][1]:.5f} {time.perf_counter() - t0:.1f} s")
            if seconds is not None and time.perf_counter() - t0 > seconds:
                done = True
                break
        if done:
            break
    torch.cuda.synchronize()
    net.check_errors()
    return TrainLog(step, time.perf_counter() - t0, losses)


def predict(net, x, batch=16):
    """Network outputs (N, H, W, cout) float32 for inputs x (N, H, W, CIN) float32 (host)."""
    torch = _t()
    n = len(x)
    if net.B != batch:
        net.alloc(batch)
    out = np.zeros((n, H, W, net.cout), np.float32)
    X = bf16_upload(x)
    xb = torch.zeros(batch, H, W, CIN, dtype=torch.bfloat16, device="cuda")
    for i in range(0, n, batch):
        m = min(batch, n - i)
        xb.zero_()
        xb[:m].copy_(X[i:i + m])
        y = net.forward(xb)
        out[i:i + m] = y.reshape(batch, H, W, net.cout)[:m].cpu().numpy()
    net.check_errors()
    return out


def masked_mse(pred, data: Dataset):
    """Mean masked squared error of predictions (N, H, W, >= NT) against a dataset's targets."""
    d = (pred[..., :NT] - data.y) ** 2 * data.w[..., None]
    return float(d.sum() / (data.w.sum() * NT))


# ---------------------------------------------------------------------------- warm-started runs
def warm_batch(net, cases, precision="f32", batch=16, twins=False):
    """A built batch of the cases in their warm form (no ramp, no twist), every tunnel initialised
    from the network's prediction: inputs encoded on the host from the tunnels' flags, the network
    and the decode to lattice fields (vl_batch_init_grid) on the device. With `twins`, tunnels
    n .. 2n - 1 are the cases' uniform-start forms (inlet ramp and twist), held (vl_batch_hold)
    until a caller starts one as the fallback of its warm twin. Returns (batch, seconds spent on
    encoding, inference and initialisation)."""
    from .batch import Batch
    torch = _t()
    b = Batch(precision)
    for c in cases:
        b.add(c.tunnel.spec_warm(c.body), c.steps)
    if twins:
        for c in cases:
            b.add(c.tunnel.spec(c.body), c.steps)
    b.build()
    if twins:
        for k in range(len(cases), 2 * len(cases)):
            b.hold(k)
    if net.B != batch:          # the network's activation buffers: set-up, like building the batch
        net.alloc(batch)
    t0 = time.perf_counter()
    x = np.stack([encode_input(b.flags(k), c.tunnel.d, c.tunnel.re) for k, c in enumerate(cases)])
    X = bf16_upload(x)
    xb = torch.zeros(batch, H, W, CIN, dtype=torch.bfloat16, device="cuda")
    per = H * W * net.cout
    for i in range(0, len(cases), batch):
        m = min(batch, len(cases) - i)
        xb.zero_()
        xb[:m].copy_(X[i:i + m])
        y = net.forward(xb)
        torch.cuda.synchronize()
        for j in range(m):
            tn = cases[i + j].tunnel
            check(lib.vl_batch_init_grid(b._h, i + j, C.c_void_p(y.data_ptr() + 4 * j * per), H, W, net.cout,
                                         0.5, 20.0 * tn.d / W, 0.5, 10.0 * tn.d / H, tn.u))
    net.check_errors()
    return b, time.perf_counter() - t0


# ---------------------------------------------------------------------------- the study
TRAIN_SEED = 0x7EA10001     # training tunnels (disjoint from the held-out population's seed)
TEST_SEED = 0x5EED0004      # held-out tunnels: the seeded batched-tunnel population


def study(n_train=2000, n_test=200, gen_units=50.0, eval_units=100.0, train_seconds=360.0, epochs=60,
          batch=16, lr=1e-3, levels=4, c0=32, log=print, weights_out=None):
    """Trains the network on solver-generated wakes of `n_train` tunnels and measures, on `n_test`
    held-out tunnels, the time to converged c_D and St of the plain form (FP64, one tunnel at a
    time, uniform start), the batched FP32 form from a uniform start and the batched FP32 form from
    the network's warm start (convergence.warm_comparison)."""
    from . import convergence as CV
    from .batch import seeded_tunnels
    out = dict(config=dict(n_train=n_train, n_test=n_test, gen_units=gen_units, eval_units=eval_units,
                           train_seconds=train_seconds, epochs=epochs, batch=batch, lr=lr, levels=levels, c0=c0))
    cases = seeded_tunnels(seed=TRAIN_SEED, count=n_train, units=gen_units)
    data = generate(cases, log=log)
    gaps = [m["peak_gap"] for m in data.meta]
    out["generate"] = dict(seconds=data.seconds, samples=len(data.x), median_peak_gap=float(np.median(gaps)))
    log(f"generated {len(data.x)} samples in {data.seconds:.1f} s")
    ntr = len(data.x) - max(batch, len(data.x) // 20)
    tr, va = data.split(ntr)
    net = UNet(levels=levels, c0=c0)
    tl = train(net, tr, epochs=epochs, batch=batch, lr=lr, seconds=train_seconds, log=log)
    pv = predict(net, va.x, batch)
    out["train"] = dict(params=net.params, steps=tl.steps, seconds=tl.seconds, ms_per_step=1e3 * tl.seconds / tl.steps,
                        samples_per_s=tl.steps * batch / tl.seconds, loss=tl.loss,
                        val_mse=masked_mse(pv, va), val_mse_uniform=masked_mse(np.zeros_like(pv), va))
    log(f"trained {tl.steps} steps in {tl.seconds:.1f} s; validation MSE {out['train']['val_mse']:.5f} "
        f"(uniform start {out['train']['val_mse_uniform']:.5f})")
    if weights_out:
        save_bf16(net, weights_out)
    test = seeded_tunnels(seed=TEST_SEED, count=n_test, units=eval_units)
    t0 = time.perf_counter()
    cmp = CV.warm_comparison(net, test)
    out["comparison"] = cmp
    log(f"comparison in {time.perf_counter() - t0:.1f} s: {cmp['summary']}")
    return out


def compare(n_test=200, eval_units=100.0, log=print):
    """The time-to-converged comparison with the shipped network (no training): every run stops
    on-line from its own history, warm-start failures fall back to the uniform start, every tunnel
    is counted (online.comparison)."""
    from . import online as OL
    from .batch import seeded_tunnels
    test = seeded_tunnels(seed=TEST_SEED, count=n_test, units=eval_units)
    net = load_pretrained()
    predict(net, np.zeros((1, H, W, CIN), np.float32))     # resident network, kernels loaded
    t0 = time.perf_counter()
    out = OL.comparison(test, net, max_units=eval_units, log=log)
    log(f"comparison in {time.perf_counter() - t0:.1f} s: {out['summary']}")
    return dict(config=dict(n_test=n_test, eval_units=eval_units, network=PRETRAINED), comparison=out)


def profile_training(steps=6, fields=48, batch=16, seed=1):
    """Trains the full network for `steps` Adam steps on `fields` seeded random fields (synthetic
    inputs, targets and masks of the training shapes): the command the training-step profiles are
    taken on. Returns milliseconds per step over the timed run of `train` (after a first run that
    loads the kernels; device synchronised on both sides)."""
    torch = _t()
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((fields, H, W, CIN)).astype(np.float32)
    y = rng.standard_normal((fields, H, W, NT)).astype(np.float32)
    w = (rng.random((fields, H, W)) > 0.05).astype(np.float32)
    data = Dataset(x, y, w)
    net = UNet()
    train(net, data, epochs=1, batch=batch)                     # first step: set-up and module loading
    per_epoch = fields // batch
    log = train(net, data, epochs=max(1, -(-steps // per_epoch)), batch=batch)
    return 1e3 * log.seconds / max(log.steps, 1)


if __name__ == "__main__":
    # python -m vortexlab_b200.warmstart OUTDIR [n_train n_test gen_units eval_units train_seconds epochs]
    # python -m vortexlab_b200.warmstart compare OUTDIR [n_test eval_units]   (the shipped network)
    # python -m vortexlab_b200.warmstart profile [steps]   (training steps on random fields)
    import json
    import sys

    def log(m):
        print(m, flush=True)

    if sys.argv[1] == "profile":
        n = int(sys.argv[2]) if len(sys.argv) > 2 else 6
        print(json.dumps({"training_ms_per_step": round(profile_training(n), 3), "steps": n}), flush=True)
        sys.exit(0)
    if sys.argv[1] == "compare":
        outdir = sys.argv[2]
        os.makedirs(outdir, exist_ok=True)
        args = sys.argv[3:]
        res = compare(int(args[0]) if args else 200, float(args[1]) if len(args) > 1 else 100.0, log=log)
        with open(os.path.join(outdir, "warmstart_compare.json"), "w") as f:
            json.dump(res, f, default=float, indent=1)
        sys.exit(0)
    outdir = sys.argv[1]
    os.makedirs(outdir, exist_ok=True)
    names = ["n_train", "n_test", "gen_units", "eval_units", "train_seconds", "epochs"]
    kw = {k: (int(v) if k.startswith("n_") or k == "epochs" else float(v)) for k, v in zip(names, sys.argv[2:])}
    res = study(**kw, log=log, weights_out=os.path.join(outdir, "warmstart_unet.npz"))
    with open(os.path.join(outdir, "warmstart_study.json"), "w") as f:
        json.dump(res, f, default=float, indent=1)
