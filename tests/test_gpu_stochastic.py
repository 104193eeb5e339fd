"""Stochastic LLG (Heun, semi-implicit Heun, deterministic RK4) against the
oracle, plus the statistics and the thermal equilibrium of the thermal field.

The reference draws its thermal field from ArrayFire's Philox engine seeded by
the wall clock (magnumaf/src/integrators/stochastic_integrator.cpp:81-84), so
its random stream is not reproducible and parity is pinned two ways: the
deterministic step arithmetic on the device's own thermal fields (fetched from
the library and fed to the oracle, 1e-12), and the statistics of the field and
of the stationary state it drives."""
import math

import numpy as np
import pytest

import maf_oracle as O
from helpers import mesh_pair, random_m, rel_max

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu


def _problem():
    gm, om = mesh_pair(16, 8, 2, 2e-9, 2e-9, 2e-9)
    m0 = random_m((16, 8, 2), 31)
    d = M.DemagField(gm)
    gterms = [d, M.ExchangeField(1.3e-11), M.UniaxialAnisotropyField(2e5, [0, 0, 1])]
    oterms = [O.DemagField(om, N_real=d.get_N(symmetric=True)), O.ExchangeField(1.3e-11),
              O.UniaxialAnisotropyField(2e5)]
    return gm, om, m0, gterms, oterms


def test_heun_matches_oracle():
    """stochastic_integrator.cpp:8-17: predictor with the previous step's field,
    corrector with the new one; five steps on the device's thermal fields."""
    gm, om, m0, gterms, oterms = _problem()
    alpha, T, dt = 0.1, 300.0, 1e-14
    gs = M.State(gm, 8e5, m0)
    os_ = O.State(om, 8e5, m0)
    st = M.Stochastic_LLG(alpha, T, dt, gs, gterms, "Heun", seed=7)
    for s in range(5):
        prev = st.thermal_field(gs, s)
        new = st.thermal_field(gs, s + 1)
        st.step(gs)
        O.heun_step(os_, oterms, alpha, dt, prev, new)
        assert rel_max(gs.m, os_.m) < 1e-12, s
    assert abs(gs.t - 5 * dt) < 1e-25 and st.calls == 5


def test_semi_implicit_heun_matches_oracle():
    gm, om, m0, gterms, oterms = _problem()
    alpha, T, dt = 0.2, 100.0, 5e-15
    gs = M.State(gm, 8e5, m0)
    os_ = O.State(om, 8e5, m0)
    st = M.Stochastic_LLG(alpha, T, dt, gs, gterms, "SemiHeun", seed=8)
    for s in range(3):
        h0 = st.thermal_field(gs, 2 * s)
        h1 = st.thermal_field(gs, 2 * s + 1)
        st.step(gs)
        O.semi_implicit_heun_step(os_, oterms, alpha, dt, h0, h1)
        assert rel_max(gs.m, os_.m) < 1e-12, s


def test_det_rk4_matches_oracle():
    gm, om, m0, gterms, oterms = _problem()
    alpha, dt = 0.5, 1e-14
    gs = M.State(gm, 8e5, m0)
    os_ = O.State(om, 8e5, m0)
    st = M.Stochastic_LLG(alpha, 300.0, dt, gs, gterms, "detRK4", seed=9)
    for s in range(3):
        st.step(gs)
        O.det_rk4_step(os_, oterms, alpha, dt)
        assert rel_max(gs.m, os_.m) < 1e-12, s


def test_thermal_field_statistics():
    """h_th = sqrt(2D/dt) N(0,1), D = alpha kB T / (gamma mu0 Ms dV): mean 0, the
    reference's variance, no correlation between components, noise indices or
    ensemble members, and identical fields for identical (seed, member, index)."""
    gm = M.Mesh(128, 128, 4, 2e-9, 2e-9, 2e-9)
    gs = M.State(gm, 8e5, random_m((128, 128, 4), 1))
    alpha, T, dt = 0.1, 300.0, 1e-13
    a = M.Stochastic_LLG(alpha, T, dt, gs, [M.ExchangeField(1e-11)], seed=123, member=0)
    b = M.Stochastic_LLG(alpha, T, dt, gs, [M.ExchangeField(1e-11)], seed=123, member=1)
    dV = 8e-27
    D = alpha * O.kb * T / (O.gamma * O.mu0 * 8e5 * dV)
    sigma = math.sqrt(2 * D / dt)
    h0 = a.thermal_field(gs, 0) / sigma
    h1 = a.thermal_field(gs, 1) / sigma
    hb = b.thermal_field(gs, 0) / sigma
    n = h0.size
    assert abs(h0.mean()) < 5 / math.sqrt(n)
    assert abs(h0.std() - 1.0) < 5 / math.sqrt(2 * n)
    for other in (h1, hb):
        assert abs(np.mean(h0 * other)) < 5 / math.sqrt(n)
    c01 = np.mean(h0[..., 0] * h0[..., 1])
    assert abs(c01) < 5 / math.sqrt(n / 3)
    # fourth moment of a normal variable is 3
    assert abs(np.mean(h0 ** 4) - 3.0) < 0.05
    assert np.array_equal(a.thermal_field(gs, 5), a.thermal_field(gs, 5))


@pytest.mark.slow
def test_langevin_equilibrium():
    """Independent macrospins in a field H along z (Zeeman only, one cell each):
    the stationary <m_z> of the stochastic LLG is the Langevin function
    L(x) = coth x - 1/x, x = mu0 Ms V H / (kB T)."""
    n = 64
    dx = 2e-9
    gm = M.Mesh(n, n, 1, dx, dx, dx)
    Ms, T = 8e5, 300.0
    x_target = 2.0
    H = x_target * O.kb * T / (O.mu0 * Ms * dx ** 3)
    m0 = np.zeros((n, n, 1, 3))
    m0[..., 2] = 1.0
    gs = M.State(gm, Ms, m0)
    st = M.Stochastic_LLG(1.0, T, 2e-14, gs, [M.ExternalField.uniform(0.0, 0.0, H)], "Heun", seed=11)
    st.steps(gs, 2000)
    samples = []
    for _ in range(100):
        st.steps(gs, 40)
        samples.append(gs.mean_m(2))
    mz = float(np.mean(samples))
    langevin = 1.0 / math.tanh(x_target) - 1.0 / x_target
    assert abs(mz - langevin) < 0.02, (mz, langevin)
