"""The warm-start network's oracle (oracle/maf_cnn_oracle.py): the hand-derived
backward pass against central finite differences of the loss, on the CPU."""
import numpy as np

import maf_cnn_oracle as N


def _case(seed, B=2, H=5, W=6, cin=5, width=4, depth=3):
    rng = np.random.default_rng(seed)
    _, _, npar = N.layout(cin, width, depth)
    p = rng.normal(scale=0.4, size=npar)
    x = rng.normal(size=(B, cin, H, W))
    t = rng.normal(size=(B, 3, H, W))
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    return p, x, t, (cin, width, depth)


def test_gradient_matches_finite_differences():
    p, x, t, arch = _case(1)
    L, g = N.loss_grad(p, x, t, *arch)
    assert abs(L - N.loss(p, x, t, *arch)) < 1e-14
    eps = 1e-6
    idx = np.random.default_rng(2).choice(p.size, 60, replace=False)
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (N.loss(pp, x, t, *arch) - N.loss(pm, x, t, *arch)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-8, (i, fd, g[i])


def test_untrained_last_layer_zero_returns_normalised_m():
    p, x, t, arch = _case(3)
    ch, offs, npar = N.layout(*arch)
    p[offs[-1]:] = 0.0
    y = N.forward(p, x, *arch)[0]
    m = x[:, :3]
    np.testing.assert_allclose(y, m / np.linalg.norm(m, axis=1, keepdims=True), atol=1e-15)


def test_dilated_gradient_matches_finite_differences():
    """Dilated layers (taps at -d, 0, +d) with d larger than the image in one case."""
    p, x, t, arch = _case(4, H=7, W=8)
    dil = [1, 2, 9]
    L, g = N.loss_grad(p, x, t, *arch, dil=dil)
    assert abs(L - N.loss(p, x, t, *arch, dil=dil)) < 1e-14
    eps = 1e-6
    idx = np.random.default_rng(5).choice(p.size, 60, replace=False)
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (N.loss(pp, x, t, *arch, dil=dil) - N.loss(pm, x, t, *arch, dil=dil)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-8, (i, fd, g[i])
    # d = 1 everywhere is the undilated network
    L1, g1 = N.loss_grad(p, x, t, *arch, dil=[1, 1, 1])
    L0, g0 = N.loss_grad(p, x, t, *arch)
    assert L1 == L0 and np.array_equal(g1, g0)
