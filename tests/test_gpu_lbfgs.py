"""LBFGS minimiser (magnumaf/src/solvers/lbfgs_minimizer.cpp) on the device
against the oracle's restatement, from identical random states."""
import numpy as np
import pytest

import maf_lbfgs_oracle as L
import maf_oracle as O
from helpers import mesh_pair, random_m

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu


def _terms(gm, om, with_demag):
    g = [M.ExchangeField(1.5e-11), M.DmiField(3e-3), M.UniaxialAnisotropyField(8e5),
         M.ExternalField.uniform(0.0, 0.0, 0.05 / O.mu0)]
    o = [O.ExchangeField(1.5e-11), O.DmiField(3e-3), O.UniaxialAnisotropyField(8e5),
         O.ExternalField(np.array([0.0, 0.0, 0.05 / O.mu0]))]
    if with_demag:
        d = M.DemagField(gm)
        g = [d] + g
        o = [O.DemagField(om, N_real=d.get_N(symmetric=True))] + o
    return g, o


@pytest.mark.parametrize("shape,with_demag", [((32, 32, 1), True), ((24, 20, 1), False)])
def test_lbfgs_matches_oracle(shape, with_demag):
    gm, om = mesh_pair(*shape, 2e-9, 2e-9, 1e-9)
    m0 = random_m(shape, 41)
    gterms, oterms = _terms(gm, om, with_demag)
    gs = M.State(gm, 8e5, m0)
    os_ = O.State(om, 8e5, m0)
    mini = M.LBFGS_Minimizer(gterms, tol=1e-6, maxiter=230)
    E = mini.minimize(gs)
    E_ref, it_ref = L.minimize(os_, oterms, tolerance=1e-6, maxIter=230)
    st = mini.stats()
    assert abs(E - E_ref) <= 1e-9 * abs(E_ref), (E, E_ref)
    assert abs(st["iterations"] - it_ref) <= 3, (st, it_ref)
    # the relaxed state: small residual torque, same configuration
    assert np.abs(gs.m - os_.m).max() < 1e-4
    assert E < O.Eeff_in_J(oterms, O.State(om, 8e5, m0))


def test_lbfgs_fp32_field_form():
    """The FP32-field form minimises to the same energy within FP32 field accuracy."""
    gm, om = mesh_pair(32, 32, 1, 2e-9, 2e-9, 1e-9)
    m0 = random_m((32, 32, 1), 42)
    gterms, oterms = _terms(gm, om, True)
    E64 = M.LBFGS_Minimizer(gterms).minimize(M.State(gm, 8e5, m0))
    E32 = M.LBFGS_Minimizer(gterms).minimize(M.State(gm, 8e5, m0, precision="fp32_field"))
    assert abs(E32 - E64) <= 1e-5 * abs(E64)
