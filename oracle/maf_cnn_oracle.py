"""Oracle (test infrastructure, CPU, FP64 NumPy) for the warm-start network of
magnum.af_b200/csrc/cnn.cu: forward pass, loss and hand-derived backward pass.
Only tests import this module.  It is pinned by central finite differences
(tests/test_cnn_oracle.py), then used to check the device gradients.

Network: y = normalize(m + conv_L(relu(... relu(conv_1(x))))), 3x3 convolutions
with zero padding and dilation d_l per layer (taps at offsets -d, 0, +d; 1 by
default), x [B][cin][H][W] with m = x[:, :3]; loss = mean over the B*H*W cells
of |y - target|^2.  Parameters: one flat vector, per layer W[cout][cin][3][3]
then b[cout]."""
import numpy as np


def layout(cin, width, depth):
    ch = [cin] + [width] * (depth - 1) + [3]
    offs, off = [], 0
    for l in range(depth):
        offs.append(off)
        off += ch[l + 1] * ch[l] * 9 + ch[l + 1]
    return ch, offs, off


def unpack(p, cin, width, depth):
    ch, offs, _ = layout(cin, width, depth)
    out = []
    for l in range(depth):
        nw = ch[l + 1] * ch[l] * 9
        W = p[offs[l]:offs[l] + nw].reshape(ch[l + 1], ch[l], 3, 3)
        b = p[offs[l] + nw:offs[l] + nw + ch[l + 1]]
        out.append((W, b))
    return out


def conv(x, W, b, d=1):
    """out[b,co,y,x] = b[co] + sum W[co,ci,dy,dx] x[b,ci,y+(dy-1)d,x+(dx-1)d] (zero outside)."""
    B, C, H, Wd = x.shape
    xp = np.zeros((B, C, H + 2 * d, Wd + 2 * d))
    xp[:, :, d:d + H, d:d + Wd] = x
    out = np.zeros((B, W.shape[0], H, Wd)) + b[None, :, None, None]
    for dy in range(3):
        for dx in range(3):
            out += np.einsum("oc,bchw->bohw", W[:, :, dy, dx], xp[:, :, dy * d:dy * d + H, dx * d:dx * d + Wd])
    return out


def forward(p, x, cin, width, depth, dil=None):
    layers = unpack(p, cin, width, depth)
    dil = dil or [1] * depth
    acts = []
    a = x
    for l, (W, b) in enumerate(layers):
        z = conv(a, W, b, dil[l])
        a = np.maximum(z, 0.0) if l + 1 < depth else z
        acts.append(a)
    v = x[:, :3] + acts[-1]
    n = np.sqrt(np.sum(v * v, axis=1, keepdims=True))
    y = np.where(n > 0, v / np.where(n > 0, n, 1.0), 0.0)
    return y, acts, v, n


def loss(p, x, t, cin, width, depth, dil=None):
    y = forward(p, x, cin, width, depth, dil)[0]
    B, _, H, W = y.shape
    return float(np.sum((y - t) ** 2) / (B * H * W))


def loss_grad(p, x, t, cin, width, depth, dil=None):
    layers = unpack(p, cin, width, depth)
    dil = dil or [1] * depth
    ch, offs, npar = layout(cin, width, depth)
    y, acts, v, n = forward(p, x, cin, width, depth, dil)
    B, _, H, Wd = y.shape
    cells = B * H * Wd
    L = float(np.sum((y - t) ** 2) / cells)
    gy = 2.0 * (y - t) / cells
    inv = np.where(n > 0, 1.0 / np.where(n > 0, n, 1.0), 0.0)
    g = (gy - y * np.sum(y * gy, axis=1, keepdims=True)) * inv  # dL/dd, d = last layer output
    grad = np.zeros(npar)
    for l in range(depth - 1, -1, -1):
        W, _ = layers[l]
        d = dil[l]
        a_in = x if l == 0 else acts[l - 1]
        ap = np.zeros((B, ch[l], H + 2 * d, Wd + 2 * d))
        ap[:, :, d:d + H, d:d + Wd] = a_in
        gW = np.zeros_like(W)
        for dy in range(3):
            for dx in range(3):
                gW[:, :, dy, dx] = np.einsum("bohw,bchw->oc", g, ap[:, :, dy * d:dy * d + H, dx * d:dx * d + Wd])
        nw = W.size
        grad[offs[l]:offs[l] + nw] = gW.ravel()
        grad[offs[l] + nw:offs[l] + nw + ch[l + 1]] = np.sum(g, axis=(0, 2, 3))
        if l > 0:
            gp = np.zeros((B, W.shape[0], H + 2 * d, Wd + 2 * d))
            gp[:, :, d:d + H, d:d + Wd] = g
            gin = np.zeros((B, ch[l], H, Wd))
            for dy in range(3):
                for dx in range(3):
                    # input pixel (y, x) feeds output (y - (dy-1)d, x - (dx-1)d) through tap (dy, dx)
                    oy, ox = (2 - dy) * d, (2 - dx) * d
                    gin += np.einsum("oc,bohw->bchw", W[:, :, dy, dx], gp[:, :, oy:oy + H, ox:ox + Wd])
            g = gin * (acts[l - 1] > 0)
    return L, grad
