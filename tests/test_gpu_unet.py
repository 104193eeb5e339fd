"""The warm-start U-net on the device (magnumaf.unet.UNet: tensor-core BF16
GEMMs with FP32 accumulation, hand-written layer kernels) against the CPU
oracle on identical inputs (oracle/maf_unet_oracle.py with the device's BF16
roundings): forward output, loss and every parameter gradient; and a short
training run lowers the loss."""
import numpy as np
import pytest

import maf_unet_oracle as U

M = pytest.importorskip("magnumaf")
torch = pytest.importorskip("torch")
from magnumaf.unet import UNet  # noqa: E402

pytestmark = pytest.mark.gpu


def _sample(rng, B, cin, H, W):
    x = rng.normal(size=(B, cin, H, W)).astype(np.float32)
    x[:, :3] /= np.linalg.norm(x[:, :3], axis=1, keepdims=True)
    t = rng.normal(size=(B, H, W, 3))
    t /= np.linalg.norm(t, axis=-1, keepdims=True)
    return x, t.astype(np.float32)


def _np(t, shape=None):
    a = t.float().cpu().numpy().astype(np.float64)
    return a.reshape(shape) if shape is not None else a


@pytest.mark.parametrize("B,H,W,widths", [(2, 16, 16, (8, 16, 24)), (1, 32, 48, (32, 64, 128))])
def test_unet_layers_match_oracle(B, H, W, widths):
    """Every layer's forward and backward on the device's own layer inputs (so
    that BF16 rounding decisions are identical on both sides) against the
    oracle's layer functions, and the whole network end to end."""
    rng = np.random.default_rng(3)
    cin = 8
    net = UNet(cin, seed=1, widths=widths)
    p = net.get_params()
    last = net.layers[-1]
    p[last.woff:last.boff] = rng.normal(0, 0.05, last.boff - last.woff)  # a nonzero head
    net.set_params(p)
    x, t = _sample(rng, B, cin, H, W)
    xd = torch.from_numpy(x).cuda()
    td = torch.from_numpy(t.reshape(-1, 3)).cuda()
    loss = net.loss_grad(xd.data_ptr(), td.data_ptr(), B, H, W, True)
    torch.cuda.synchronize()
    g = net.grad.double().cpu().numpy()
    w1, w2, w3 = widths
    dims = [(H, W), (H // 2, W // 2), (H // 4, W // 4)]
    dx = {}
    for i, L in enumerate(net.layers):
        h, w = dims[L.level]
        Wl = p[L.woff:L.boff].astype(np.float64).reshape(L.cout, 9, L.cin)
        bl = p[L.boff:L.boff + L.cout].astype(np.float64)
        a = _np(net.inb[i], (B, h, w, L.cp))[..., :L.cin]  # BF16 values, exactly
        col = U.im2col(a)
        y = np.einsum("bhwtc,otc->bhwo", col, U.bf16_round(Wl)) + bl
        y = np.maximum(y, 0.0) if L.relu else y
        out = _np(net.out[i], (B, h, w, L.cout))
        assert np.linalg.norm(out - y) <= 1e-5 * np.linalg.norm(y) + 1e-30, ("forward", i)
        # backward from the device's output gradient
        dA = _np(net.dA[i], (B, h, w, L.cout))
        dY = dA * (out > 0) if L.relu else dA
        dYr = U.bf16_round(dY)
        dW = np.einsum("bhwo,bhwtc->otc", dYr, col)
        db = dY.sum(axis=(0, 1, 2))
        gw = g[L.woff:L.boff].reshape(L.cout, 9, L.cin)
        gb = g[L.boff:L.boff + L.cout]
        assert np.linalg.norm(gw - dW) <= 1e-5 * np.linalg.norm(dW) + 1e-30, ("dW", i)
        assert np.linalg.norm(gb - db) <= 1e-5 * np.linalg.norm(db) + 1e-30, ("db", i)
        if i > 0:
            dx[i] = U.col2im(np.einsum("bhwo,otc->bhwtc", dYr, U.bf16_round(Wl)))
    # the gradients the layers hand to each other
    chk = {7: dx[8], 4: dx[5], 2: dx[3], 0: dx[1],
           6: U.up_bwd(dx[7][..., :w2]), 5: U.up_bwd(dx[6][..., :w3]),
           3: dx[6][..., w3:w3 + w2] + U.pool_bwd(dx[4]), 1: dx[7][..., w2:w2 + w1] + U.pool_bwd(dx[2])}
    for i, ref in chk.items():
        L = net.layers[i]
        h, w = dims[L.level]
        got = _np(net.dA[i], (B, h, w, L.cout))
        assert np.linalg.norm(got - ref) <= 1e-5 * np.linalg.norm(ref) + 1e-30, ("dA", i)
    # end to end: rounding decisions may differ where FP32 and float64 values
    # straddle a BF16 boundary, so only closeness
    ora = U.UNetOracle(p, cin, widths, bf16=True)
    yo = ora.forward(x)
    go = ora.backward(t)
    y = net.y.double().cpu().numpy().reshape(B, H, W, 3)
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) < 1e-2
    assert abs(loss - ora.loss(t)) < 1e-2 * abs(ora.loss(t))
    assert np.linalg.norm(g - go) / np.linalg.norm(go) < 5e-2


def test_unet_training_lowers_the_loss():
    rng = np.random.default_rng(4)
    B, H, W, cin = 4, 32, 32, 8
    net = UNet(cin, seed=2, widths=(16, 32, 64))
    x, t = _sample(rng, B, cin, H, W)
    # a learnable target: a smooth rotation of the input magnetisation
    m = np.transpose(x[:, :3], (0, 2, 3, 1)).astype(np.float64)
    t = np.stack([m[..., 1], -m[..., 0], m[..., 2]], axis=-1)
    xd = torch.from_numpy(x).cuda()
    td = torch.from_numpy(t.reshape(-1, 3).astype(np.float32)).cuda()
    losses = [net.train_step(xd.data_ptr(), td.data_ptr(), B, H, W, 2e-3) for _ in range(150)]
    assert np.all(np.isfinite(losses))
    assert np.mean(losses[-10:]) < 0.5 * np.mean(losses[:5])
