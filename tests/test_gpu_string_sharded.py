"""The sharded string method's device adapter (one State and one LLGIntegrator
per image, magnumaf/string_sharded.py) on one GPU against the serial oracle
string method with the same per-image integrator policy."""
import numpy as np
import pytest

import maf_oracle as O
import maf_string_oracle as SO
from helpers import mesh_pair

M = pytest.importorskip("magnumaf")
from magnumaf import string_sharded as SS  # noqa: E402

pytestmark = pytest.mark.gpu

SHAPE = (16, 16, 1)
MS = 1.1e6


def test_device_images_follow_the_oracle():
    gm, om = mesh_pair(*SHAPE, 1e-9, 1e-9, 1e-9)
    d = M.DemagField(gm)
    g_terms = [d, M.ExchangeField(1.6e-11), M.DmiField(4e-3), M.UniaxialAnisotropyField(1e6)]
    o_terms = [O.DemagField(om, N_real=d.get_N(symmetric=True)), O.ExchangeField(1.6e-11), O.DmiField(4e-3),
               O.UniaxialAnisotropyField(1e6)]
    a = np.zeros(SHAPE + (3,))
    a[..., 2] = 1.0
    a[5:11, 5:11, 0, 2] = -1.0
    a[..., 0] += 0.1
    a = O.normalize(a)
    b = np.zeros(SHAPE + (3,))
    b[..., 0] = 0.1
    b[..., 2] = 1.0
    b = O.normalize(b)
    soa = lambda m: np.transpose(m, (3, 2, 1, 0)).reshape(-1).copy()  # noqa: E731
    n = 4
    imgs = SS.DeviceImages(gm, MS, range(n), lambda: M.LLGIntegrator(1.0, g_terms))
    sm = SS.ShardedStringMethod(imgs, n, 5e-14, [soa(a), soa(b)])
    ref = SO.StringMethod(O.State(om, MS, a), [a, b], n, 5e-14, O.LLGIntegrator(1.0, o_terms),
                          per_image_integrators=True)
    for _ in range(2):
        sm.step()
        ref.step()
    np.testing.assert_allclose(sm.x, ref.x, rtol=1e-8)
    np.testing.assert_allclose(sm.calc_E(), ref.calc_E(), rtol=1e-8)
    for i in range(n):
        np.testing.assert_allclose(imgs.get(i), soa(ref.images[i].m), atol=1e-8)
