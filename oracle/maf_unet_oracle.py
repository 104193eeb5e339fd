"""CPU oracle of the warm-start U-net (magnumaf/unet.py, nn.cu) -- test
infrastructure only.

NumPy restatement of the network's forward pass, loss and backward pass in
float64, pixel-major (NHWC) like the device.  With ``bf16=True`` it rounds the
GEMM operands to BF16 (round to nearest even) where the device does -- the
im2col tiles of layer inputs, the weights, and the output gradients that feed
the data- and weight-gradient GEMMs -- so the device's gradients can be checked
on identical inputs; with ``bf16=False`` it is the exact network, whose
gradient a central finite-difference check pins.

Parameters: one flat vector, per layer W [cout][9][cin] (tap t = 3 (dy + 1) +
(dx + 1)) then b [cout], in the layer order of magnumaf.unet.UNet.
"""
from __future__ import annotations

import numpy as np


def bf16_round(a):
    """Round float32 values to BF16 (round to nearest even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def layer_spec(cin, widths=(32, 64, 128)):
    w1, w2, w3 = widths
    return [(cin, w1, True), (w1, w1, True), (w1, w2, True), (w2, w2, True), (w2, w3, True), (w3, w3, True),
            (w3 + w2, w2, True), (w2 + w1, w1, True), (w1, 3, False)]


def split_params(p, cin, widths=(32, 64, 128)):
    out, off = [], 0
    for ci, co, _ in layer_spec(cin, widths):
        W = p[off:off + co * 9 * ci].reshape(co, 9, ci)
        off += co * 9 * ci
        b = p[off:off + co]
        off += co
        out.append((W, b))
    return out


def im2col(a):
    """a [B][H][W][C] -> [B][H][W][9][C], zero padded, tap t = 3 (dy + 1) + (dx + 1)."""
    B, H, W, C = a.shape
    pad = np.zeros((B, H + 2, W + 2, C))
    pad[:, 1:-1, 1:-1] = a
    cols = np.empty((B, H, W, 9, C))
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        cols[:, :, :, t] = pad[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]
    return cols


def col2im(dcol):
    """Adjoint of im2col: [B][H][W][9][C] -> [B][H][W][C]."""
    B, H, W, _, C = dcol.shape
    pad = np.zeros((B, H + 2, W + 2, C))
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        pad[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W] += dcol[:, :, :, t]
    return pad[:, 1:-1, 1:-1]


def pool(a):
    return 0.25 * ((a[:, 0::2, 0::2] + a[:, 0::2, 1::2]) + (a[:, 1::2, 0::2] + a[:, 1::2, 1::2]))


def pool_bwd(d):
    return 0.25 * np.repeat(np.repeat(d, 2, axis=1), 2, axis=2)


def up(a):
    return np.repeat(np.repeat(a, 2, axis=1), 2, axis=2)


def up_bwd(d):
    return (d[:, 0::2, 0::2] + d[:, 0::2, 1::2]) + (d[:, 1::2, 0::2] + d[:, 1::2, 1::2])


class UNetOracle:
    def __init__(self, params, cin, widths=(32, 64, 128), bf16=True):
        self.cin, self.widths, self.bf16 = cin, widths, bf16
        self.layers = split_params(np.asarray(params, dtype=np.float64), cin, widths)
        self.spec = layer_spec(cin, widths)
        self.r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))

    def _conv(self, i, a):
        W, b = self.layers[i]
        relu = self.spec[i][2]
        col = im2col(self.r(a))
        y = np.einsum("bhwtc,otc->bhwo", col, self.r(W)) + b
        out = np.maximum(y, 0.0) if relu else y
        return out, col

    def forward(self, x):
        """x [B][cin][H][W] -> y [B][H][W][3]; keeps what the backward pass needs."""
        x = np.transpose(np.asarray(x, dtype=np.float64), (0, 2, 3, 1))
        self.m = x[..., :3]
        s = {}
        s[0] = x
        o0, c0 = self._conv(0, x)
        o1, c1 = self._conv(1, o0)
        p1 = pool(o1)
        o2, c2 = self._conv(2, p1)
        o3, c3 = self._conv(3, o2)
        p2 = pool(o3)
        o4, c4 = self._conv(4, p2)
        o5, c5 = self._conv(5, o4)
        cat6 = np.concatenate([up(o5), o3], axis=-1)
        o6, c6 = self._conv(6, cat6)
        cat7 = np.concatenate([up(o6), o1], axis=-1)
        o7, c7 = self._conv(7, cat7)
        d, c8 = self._conv(8, o7)
        self.outs = [o0, o1, o2, o3, o4, o5, o6, o7, d]
        self.cols = [c0, c1, c2, c3, c4, c5, c6, c7, c8]
        v = self.m + d
        self.n = np.linalg.norm(v, axis=-1, keepdims=True)
        self.y = v / self.n
        return self.y

    def loss(self, t):
        return float(np.mean(np.sum((self.y - t) ** 2, axis=-1)))

    def _conv_bwd(self, i, dA):
        W, _ = self.layers[i]
        relu = self.spec[i][2]
        dY = dA * (self.outs[i] > 0) if relu else dA
        db = dY.sum(axis=(0, 1, 2))
        dYr = self.r(dY)
        dW = np.einsum("bhwo,bhwtc->otc", dYr, self.cols[i])
        dx = col2im(np.einsum("bhwo,otc->bhwtc", dYr, self.r(W)))
        return dx, dW, db

    def backward(self, t):
        """Gradient of the loss (mean over pixels of |y - t|^2) w.r.t. the flat parameters."""
        P = self.y.shape[0] * self.y.shape[1] * self.y.shape[2]
        gy = 2.0 * (self.y - t) / P
        dot = np.sum(self.y * gy, axis=-1, keepdims=True)
        dd = (gy - self.y * dot) / self.n
        w1, w2, w3 = self.widths
        grads = [None] * 9
        dx, dW, db = self._conv_bwd(8, dd)
        grads[8] = (dW, db)
        dx, dW, db = self._conv_bwd(7, dx)
        grads[7] = (dW, db)
        dA6, dE1 = up_bwd(dx[..., :w2]), dx[..., w2:w2 + w1]
        dx, dW, db = self._conv_bwd(6, dA6)
        grads[6] = (dW, db)
        dA5, dE2 = up_bwd(dx[..., :w3]), dx[..., w3:w3 + w2]
        dx, dW, db = self._conv_bwd(5, dA5)
        grads[5] = (dW, db)
        dx, dW, db = self._conv_bwd(4, dx)
        grads[4] = (dW, db)
        dE2 = dE2 + pool_bwd(dx)
        dx, dW, db = self._conv_bwd(3, dE2)
        grads[3] = (dW, db)
        dx, dW, db = self._conv_bwd(2, dx)
        grads[2] = (dW, db)
        dE1 = dE1 + pool_bwd(dx)
        dx, dW, db = self._conv_bwd(1, dE1)
        grads[1] = (dW, db)
        _, dW, db = self._conv_bwd(0, dx)
        grads[0] = (dW, db)
        return np.concatenate([np.concatenate([g[0].ravel(), g[1].ravel()]) for g in grads])
