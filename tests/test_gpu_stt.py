"""SpinTransferTorqueField (spin_transfer_torque_field.cpp) against the oracle,
and the mesh check of field terms with parameter arrays."""
import numpy as np
import pytest

import maf_oracle as O
from helpers import mesh_pair, random_m, rel_l2

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu

SHAPE = (12, 10, 3)


def _case(with_empty):
    gm, om = mesh_pair(*SHAPE, 2e-9, 3e-9, 1e-9)
    m = random_m(SHAPE, 4)
    pol = np.random.default_rng(5).normal(size=SHAPE + (3,))
    if with_empty:
        ms = np.full(SHAPE, 8e5)
        ms[::3, ::2, :] = 0.0
        m[ms == 0] = 0.0
    else:
        ms = 8e5
    return gm, om, m, pol, ms


@pytest.mark.parametrize("with_empty", [False, True])
def test_stt_field_and_energy_match_oracle(with_empty):
    gm, om, m, pol, ms = _case(with_empty)
    args = (0.3, 0.1, 2e10, 1.2e-9)
    g = M.SpinTransferTorqueField(pol, *args)
    o = O.SpinTransferTorqueField(pol, *args)
    gs = M.State(gm, ms, m)
    os_ = O.State(om, ms, m)
    H = g.H_in_Apm(gs)
    H_ref = o.H_in_Apm(os_)
    np.testing.assert_allclose(H, H_ref, rtol=1e-12, atol=1e-12 * np.abs(H_ref).max())
    assert abs(g.Energy_in_J(gs) - o.Energy_in_J(os_)) <= 1e-12 * abs(o.Energy_in_J(os_))
    s32 = M.State(gm, ms, m, precision="fp32_field")
    assert rel_l2(g.H_in_Apm(s32), H_ref) <= 1e-6


def test_parameter_field_of_another_mesh_is_rejected():
    gm, _, m, pol, _ = _case(False)
    other = np.ones((6, 5, 3, 3))
    t = M.SpinTransferTorqueField(other, 0.3, 0.1, 2e10, 1e-9)
    s = M.State(gm, 8e5, m)
    with pytest.raises(M.MafError):
        t.H_in_Apm(s)
    llg = M.LLGIntegrator(0.1, [M.ExchangeField(1e-11), t])
    with pytest.raises(M.MafError):
        llg.step(s)
