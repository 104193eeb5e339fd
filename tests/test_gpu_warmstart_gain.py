"""What the trained warm start gains over plain LBFGS (the reference's
LBFGS_Minimizer, lbfgs_minimizer.cpp:55-198, is both fallback and arbiter): the
pretrained U-net (magnumaf/data/warmstart_unet_128.npz, trained by the
library's own tensor-core kernels on GPU-LBFGS relaxations) proposes relaxed
states for held-out 128 x 128 samples of the configuration (seeds never used in
training); LBFGS from the proposals needs far fewer iterations, and where both
starts reach the same minimum the final energies agree to 1e-6."""
import numpy as np
import pytest

M = pytest.importorskip("magnumaf")
pytest.importorskip("torch")

from magnumaf import warmstart as WS  # noqa: E402

pytestmark = pytest.mark.gpu


def test_pretrained_unet_cuts_lbfgs_iterations_on_held_out_samples():
    net = WS.pretrained_unet()
    res = WS.gain(net, 6, 128, 128, seed=20_000)
    assert res["proposals_used"] >= 5
    # fewer LBFGS iterations from the proposals, on average and on the samples
    # that end in the same minimum as plain LBFGS
    assert res["warm_iterations"] <= 0.5 * res["plain_iterations"], res
    assert res["equal_energy_1e-6"] >= 0.3, res
    assert res["warm_iterations_equal_energy"] <= 0.5 * res["plain_iterations_equal_energy"], res
    # the warm-started runs end at least as relaxed
    assert res["torque_warm_max"] <= max(res["torque_plain_max"], 1e-4), res


def test_untrained_unet_proposes_the_input_state():
    """An untrained net (zero last layer) returns the initial magnetisation, so
    the warm start can never be worse than the plain start by construction."""
    from magnumaf.unet import UNet

    rng = np.random.default_rng(0)
    p = WS.sample_params(rng, WS.PARAM_RANGES_128)
    m0 = WS.random_sphere_m(rng, 32, 32)
    prop = WS.propose(UNet(WS.CIN, seed=3), m0, p)
    np.testing.assert_allclose(prop, m0, atol=1e-6)
