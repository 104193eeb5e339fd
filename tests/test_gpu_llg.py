"""LLG right-hand side, adaptive Runge-Kutta stepping and dense output of the
CUDA library against the FP64 oracle and the reference's trajectory goldens."""
import numpy as np
import pytest

import maf_oracle as O
from helpers import mesh_pair, random_m, rel_l2, rel_max

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu


def _sp4_initial():
    m = np.zeros((100, 25, 1, 3))
    m[1:-1, :, :, 0] = 1.0
    m[0, :, :, 1] = 1.0
    m[-1, :, :, 1] = 1.0
    return m


def _sp4_run(precision):
    """python/test/sp4.py:7-62 on the device: relax 1 ns at alpha = 1, then switch
    with the (-24.6, 4.3, 0) mT field at alpha = 0.02 until 2 ns."""
    mesh = M.Mesh(100, 25, 1, 5.e-7 / 100, 1.25e-7 / 25, 3.e-9)
    state = M.State(mesh, 8e5, _sp4_initial(), precision=precision)
    demag = M.DemagField(mesh)
    exch = M.ExchangeField(1.3e-11)
    llg = M.LLGIntegrator(1, [demag, exch])
    ix = iy = iz = 0.0
    while state.t < 1e-9:
        t1 = state.t
        llg.step(state)
        dt = state.t - t1
        mx, my, mz = state.mean_m()
        ix += mx * dt
        iy += my * dt
        iz += mz * dt
    relax = (ix, iy, iz)
    llg.alpha = 0.02
    zee = np.zeros((100, 25, 1, 3))
    zee[..., 0] = -24.6e-3 / M.Constants.mu0
    zee[..., 1] = +4.3e-3 / M.Constants.mu0
    llg.add_terms(M.ExternalField(zee))
    ix = iy = iz = 0.0
    while state.t < 2e-9:
        t1 = state.t
        llg.step(state)
        dt = state.t - t1
        mx, my, mz = state.mean_m()
        ix += mx * dt
        iy += my * dt
        iz += mz * dt
    return relax, (ix, iy, iz), llg.counters()


SP4_RELAX = (9.81206172824e-10, 9.14350283169e-11, -5.74381785359e-13)
SP4_SWITCH = (-6.41261165705e-10, 1.47353233738e-10, -1.78144535231e-11)


def test_sp4_golden_fp64():
    """The reference's own trajectory golden (python/test/sp4.py:34-36, 60-62), 1e-15 absolute."""
    relax, switch, cnt = _sp4_run("fp64")
    for v, g in zip(relax, SP4_RELAX):
        assert abs(v - g) < 1e-15, (relax, cnt)
    for v, g in zip(switch, SP4_SWITCH):
        assert abs(v - g) < 1e-15, (switch, cnt)


def test_sp4_fp32_field():
    """FP32-field form on the same problem.  The SP4 time integrals are sensitive to
    any field perturbation through the step-size controller (atol = rtol = 1e-6):
    the FP64 oracle with H merely rounded to FP32 moves the relaxation integral of
    <mx> by 4.7e-4 relative, with 1e-7 relative noise on H by 7.3e-4.  The bound,
    5e-3 of the largest component, is set from that measured sensitivity."""
    relax, switch, _ = _sp4_run("fp32_field")
    for v, g in zip(relax, SP4_RELAX):
        assert abs(v - g) < 5e-3 * abs(SP4_RELAX[0]), relax
    for v, g in zip(switch, SP4_SWITCH):
        assert abs(v - g) < 5e-3 * abs(SP4_SWITCH[0]), switch


def _rk_problem():
    gm, om = mesh_pair(24, 16, 2, 3e-9, 3e-9, 3e-9)
    m0 = random_m((24, 16, 2), 21)
    gs = M.State(gm, 8e5, m0)
    os_ = O.State(om, 8e5, m0)
    d = M.DemagField(gm)
    gterms = [d, M.ExchangeField(1.3e-11), M.UniaxialAnisotropyField(3e5, [0, 0, 1])]
    oterms = [O.DemagField(om, N_real=d.get_N(symmetric=True)), O.ExchangeField(1.3e-11),
              O.UniaxialAnisotropyField(3e5)]
    return gs, os_, gterms, oterms


@pytest.mark.parametrize("scheme", ["RKF45", "DP45", "BS23"])
@pytest.mark.parametrize("dt", [2e-14, 3e-13])
def test_rk_attempt_matches_oracle(scheme, dt):
    """One attempt at a fixed dt (adaptive_runge_kutta.cpp:75-173, 496-529): the
    candidate m + sumbk to 1e-12 and the scaled error norm to 1e-9 relative (the
    norm is a difference of nearly equal stage sums; 1e-9 is well above its
    rounding floor at these step sizes)."""
    gs, os_, gterms, oterms = _rk_problem()
    gl = M.LLGIntegrator(0.1, gterms, scheme)
    ol = O.LLGIntegrator(0.1, oterms, scheme)
    m_new, err = gl.rk_attempt(gs, scheme, dt)
    sumbk, err_ref = ol.attempt(os_, dt)
    ref = os_.m + sumbk
    assert rel_max(m_new, ref) < 1e-12
    assert abs(err - err_ref) < 1e-9 * err_ref


@pytest.mark.parametrize("scheme", ["RKF45", "DP45", "BS23"])
def test_rk_trajectory_matches_oracle(scheme):
    """25 adaptive steps from identical inputs.  The first step sizes are decided
    by error norms at the rounding floor (the first trial step is 1.01e-15 s), so
    t and m are compared to 1e-8; the accept/reject sequence must be identical."""
    gs, os_, gterms, oterms = _rk_problem()
    gl = M.LLGIntegrator(0.1, gterms, scheme)
    ol = O.LLGIntegrator(0.1, oterms, scheme)
    for i in range(25):
        gl.step(gs)
        ol.step(os_)
        assert abs(gs.t - os_.t) <= 1e-8 * abs(os_.t), (i, gs.t, os_.t)
        assert rel_max(gs.m, os_.m) < 1e-8, i
    assert gl.counters()["accepted"] == ol.controller.counter_accepted
    assert gl.counters()["rejected"] == ol.controller.counter_reject


def test_integrate_dense_matches_oracle():
    """integrate_dense (llg_integrator.cpp:68-104): RKF45 back-steps at each sample."""
    gm, om = mesh_pair(20, 10, 1, 5e-9, 5e-9, 3e-9)
    m0 = random_m((20, 10, 1), 22)
    gs = M.State(gm, 8e5, m0)
    os_ = O.State(om, 8e5, m0)
    d = M.DemagField(gm)
    gl = M.LLGIntegrator(0.5, [d, M.ExchangeField(1.3e-11)], "DP45")
    ol = O.LLGIntegrator(0.5, [O.DemagField(om, N_real=d.get_N(symmetric=True)), O.ExchangeField(1.3e-11)], "DP45")
    rows = gl.integrate_dense(gs, 2e-11, 2e-12)
    ref = ol.integrate_dense(os_, 2e-11, 2e-12)
    assert rows.shape == ref.shape
    np.testing.assert_allclose(rows[:, 0], ref[:, 0], rtol=1e-12, atol=0)
    np.testing.assert_allclose(rows[:, 1:], ref[:, 1:], rtol=0, atol=1e-12)
    assert abs(gs.t - os_.t) < 1e-12 * abs(os_.t)


def test_alpha_field_and_dissipation_only():
    gm, om = mesh_pair(12, 8, 2, 2e-9, 2e-9, 2e-9)
    m0 = random_m((12, 8, 2), 23)
    alpha = np.random.default_rng(24).uniform(0.01, 0.5, size=(12, 8, 2))
    gs = M.State(gm, 8e5, m0)
    os_ = O.State(om, 8e5, m0)
    for diss in (False, True):
        gl = M.LLGIntegrator(alpha, [M.ExchangeField(1.3e-11), M.UniaxialAnisotropyField(4e5)],
                             dissipation_term_only=diss)
        ol = O.LLGIntegrator(alpha, [O.ExchangeField(1.3e-11), O.UniaxialAnisotropyField(4e5)],
                             dissipation_term_only=diss)
        ref = ol.f(os_)
        np.testing.assert_allclose(gl.dmdt(gs), ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_nan_detected():
    """A NaN in m makes the error norm NaN; the step fails with MAF_ERR_NAN instead of
    running on (the reference never checks)."""
    gm, om = mesh_pair(8, 8, 1, 2e-9, 2e-9, 2e-9)
    m0 = random_m((8, 8, 1), 25)
    gs = M.State(gm, 8e5, m0)
    m_bad = gs.m
    m_bad[3, 3, 0, 0] = np.nan
    gs.m = m_bad
    llg = M.LLGIntegrator(0.1, [M.ExchangeField(1.3e-11)])
    with pytest.raises(M.MafError) as e:
        llg.step(gs)
    assert e.value.code == 4


def test_energy_relax_decreases():
    gm, om = mesh_pair(16, 16, 1, 3e-9, 3e-9, 3e-9)
    gs = M.State(gm, 8e5, random_m((16, 16, 1), 26))
    llg = M.LLGIntegrator(1.0, [M.DemagField(gm), M.ExchangeField(1.3e-11)])
    E0 = llg.Eeff_in_J(gs)
    llg.steps(gs, 50)
    assert llg.Eeff_in_J(gs) < E0
