"""The U-net oracle (oracle/maf_unet_oracle.py) in exact arithmetic against
central finite differences of its own loss: the analytic backward pass the
device reproduces is the gradient of the network."""
import numpy as np

import maf_unet_oracle as U


def test_exact_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    cin, widths = 8, (8, 8, 8)
    n = sum(co * 9 * ci + co for ci, co, _ in U.layer_spec(cin, widths))
    p = rng.normal(0, 0.3, n)
    x = rng.normal(size=(1, cin, 16, 16))
    x[:, :3] /= np.linalg.norm(x[:, :3], axis=1, keepdims=True)
    t = rng.normal(size=(1, 16, 16, 3))
    t /= np.linalg.norm(t, axis=-1, keepdims=True)
    net = U.UNetOracle(p, cin, widths, bf16=False)
    net.forward(x)
    g = net.backward(t)

    def loss(q):
        o = U.UNetOracle(q, cin, widths, bf16=False)
        o.forward(x)
        return o.loss(t)

    idx = rng.choice(n, 40, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros(n)
        e[i] = h
        fd = (loss(p + e) - loss(p - e)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1e-3, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e38], dtype=np.float32)
    r = U.bf16_round(a)
    assert r[0] == 1.0 and r[1] == 1.0  # a tie rounds to the even mantissa
    assert r[2] == 1.0 + 2 ** -7       # above the tie rounds up
    assert r[3] == -2.5
