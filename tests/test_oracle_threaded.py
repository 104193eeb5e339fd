"""The threaded oracle evaluation (timed CPU baseline) against the plain oracle:
the same field, the local terms bit for bit (same element-wise arithmetic on
halo slabs), the demag term to the FFT libraries' rounding."""
import numpy as np
import pytest

import maf_oracle as O
import maf_oracle_threaded as OT
from helpers import random_m, rel_l2


@pytest.mark.parametrize("shape", [(24, 20, 4), (16, 9, 1), (5, 3, 2)])
def test_threaded_heff_matches_oracle(shape):
    mesh = O.Mesh(*shape, 3e-9, 3e-9, 3e-9)
    m = random_m(shape, 4)
    state = O.State(mesh, 8.6e5, m)
    hext = np.array([1e4, -2e4, 3e4])
    demag = O.DemagField(mesh, symmetric=True)
    local = [O.ExchangeField(1.3e-11), O.CubicAnisotropyField(-1e4), O.ExternalField(hext)]
    for t in local:
        np.testing.assert_array_equal(OT.heff_in_apm([t], state, workers=3), t.H_in_Apm(state))
    terms = [demag] + local
    ref = O.Heff_in_Apm(terms, state)
    got = OT.heff_in_apm(terms, state, workers=3)
    assert rel_l2(got, ref) < 1e-14


def test_threaded_falls_back_for_parameter_fields():
    shape = (8, 6, 2)
    mesh = O.Mesh(*shape, 1e-9, 1e-9, 1e-9)
    state = O.State(mesh, 8e5, random_m(shape, 5))
    zee = np.random.default_rng(1).normal(size=shape + (3,)) * 1e4
    t = O.ExternalField(zee)
    np.testing.assert_array_equal(OT.heff_in_apm([t], state, workers=2), t.H_in_Apm(state))
