"""Learned warm start: the network's device kernels (csrc/cnn.cu) against the
oracle (oracle/maf_cnn_oracle.py), training, and the warm-started LBFGS
relaxation with plain LBFGS as fallback."""
import numpy as np
import pytest

import maf_cnn_oracle as N

M = pytest.importorskip("magnumaf")
torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

ARCH = (5, 4, 3)  # cin, width, depth


def _data(seed, B=2, H=7, W=9, cin=5):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(B, cin, H, W))
    t = rng.normal(size=(B, 3, H, W))
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    return x, t


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.mark.parametrize("dil", [None, [1, 2, 4], [3, 1, 10]])
def test_gradients_match_oracle(dil):
    net = M.ConvNet(*ARCH, seed=3, dilation=dil)
    rng = np.random.default_rng(4)
    p = rng.normal(scale=0.4, size=net.n_params).astype(np.float32)
    net.set_params(p)
    x, t = _data(5)
    xd, td = _dev(x), _dev(t)
    loss, g = net.loss_grad(xd.data_ptr(), td.data_ptr(), *x.shape[:1], x.shape[2], x.shape[3])
    x32, t32 = x.astype(np.float32).astype(np.float64), t.astype(np.float32).astype(np.float64)
    L_ref, g_ref = N.loss_grad(p.astype(np.float64), x32, t32, *ARCH, dil=dil)
    assert abs(loss - L_ref) <= 1e-5 * L_ref
    scale = np.abs(g_ref).max()
    np.testing.assert_allclose(g, g_ref, rtol=1e-3, atol=1e-5 * scale)


@pytest.mark.parametrize("dil", [None, [2, 3, 1]])
def test_forward_matches_oracle(dil):
    net = M.ConvNet(*ARCH, seed=1, dilation=dil)
    p = np.random.default_rng(6).normal(scale=0.4, size=net.n_params).astype(np.float32)
    net.set_params(p)
    x, _ = _data(7)
    xd = _dev(x)
    y = torch.empty((x.shape[0], 3, x.shape[2], x.shape[3]), dtype=torch.float32, device="cuda")
    net.forward(xd.data_ptr(), x.shape[0], x.shape[2], x.shape[3], y.data_ptr())
    y_ref = N.forward(p.astype(np.float64), x.astype(np.float32).astype(np.float64), *ARCH, dil=dil)[0]
    np.testing.assert_allclose(y.cpu().numpy(), y_ref, atol=2e-5)


def test_training_fits_a_teacher_network():
    """Targets from a fixed 'teacher' network of the same shape: Adam on the
    device kernels drives the loss down more than five-fold."""
    cin, width, depth = 5, 8, 3
    teacher = np.random.default_rng(8).normal(scale=0.3, size=N.layout(cin, width, depth)[2])
    x = np.random.default_rng(9).normal(size=(32, cin, 12, 12))
    t = N.forward(teacher, x, cin, width, depth)[0]
    net = M.ConvNet(cin, width, depth, seed=2)
    xd, td = _dev(x), _dev(t)
    losses = [net.train_step(xd.data_ptr(), td.data_ptr(), 32, 12, 12, 3e-3) for _ in range(400)]
    assert np.mean(losses[-10:]) < 0.2 * np.mean(losses[:10])


def test_warm_start_plumbing_and_fallback():
    from magnumaf import warmstart as WS

    rng = np.random.default_rng(11)
    p = WS.sample_params(rng)
    m0 = WS.smooth_random_m(rng, 16, 16)
    _, plain = WS.relax(m0, p, None)
    # untrained network: last layer zero, the proposal is m0 itself
    ident = M.ConvNet(WS.CIN, 8, 3, seed=0)
    _, same = WS.relax(m0, p, ident)
    assert same["used_proposal"] and abs(same["E"] - plain["E"]) <= 1e-12 * abs(plain["E"])
    # a proposal of higher energy than the initial state is discarded
    bad = M.ConvNet(WS.CIN, 8, 3, seed=0)
    q = bad.get_params()
    q[:] = np.random.default_rng(12).normal(scale=5.0, size=q.size)
    bad.set_params(q)
    _, fb = WS.relax(m0, p, bad)
    if not fb["used_proposal"]:
        assert abs(fb["E"] - plain["E"]) <= 1e-12 * abs(plain["E"])
    assert plain["torque"] < 1e-2
