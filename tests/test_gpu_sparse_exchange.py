"""SparseExchangeField / ExchangeFieldPBC (sparse_exchange_field.cpp,
exchange_field_pbc.cpp) and ExchangeField(A, mesh) against the oracle's
assembled matrix, plus the reference's own property tests of these terms
(magnumaf/test/micro_exch_sparse.cpp:36-84, magnumaf/test/micro_exch_pbc.cpp:34-92)."""
import numpy as np
import pytest

import maf_oracle as O
from helpers import mesh_pair, random_m, rel_l2, rel_max

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _A_field(shape, seed, zeros=True):
    rng = np.random.default_rng(seed)
    A = rng.uniform(0.5e-11, 2e-11, size=shape)
    if zeros:
        A[::4, 1::3, :] = 0.0
    return A


def _pair(kind, A, gm, om):
    if kind == "sparse":
        return M.SparseExchangeField(A, gm), O.SparseExchangeField(A, om)
    if kind == "pbc":
        return M.ExchangeFieldPBC(A, gm), O.ExchangeFieldPBC(A, om)
    return M.ExchangeField(A, gm), O.SparseExchangeField(A, om)


def _check(g, o, gs, os_):
    H = g.H_in_Apm(gs)
    H_ref = o.H_in_Apm(os_)
    np.testing.assert_allclose(H, H_ref, rtol=TOL, atol=TOL * np.abs(H_ref).max())
    E, E_ref = g.Energy_in_J(gs), o.Energy_in_J(os_)
    assert abs(E - E_ref) <= 1e-11 * max(abs(E_ref), 1e-300)
    return H_ref


@pytest.mark.parametrize("kind", ["sparse", "pbc", "exchange_mesh"])
@pytest.mark.parametrize("field_A", [False, True])
@pytest.mark.parametrize("shape", [(12, 10, 3), (5, 2, 1), (1, 7, 4)])
def test_matches_oracle(kind, field_A, shape):
    gm, om = mesh_pair(*shape, 2e-9, 3e-9, 1.5e-9)
    m = random_m(shape, 11)
    A = _A_field(shape, 12) if field_A else 1.3e-11
    g, o = _pair(kind, A, gm, om)
    H_ref = _check(g, o, M.State(gm, 8e5, m), O.State(om, 8e5, m))
    s32 = M.State(gm, 8e5, m, precision="fp32_field")
    assert rel_l2(g.H_in_Apm(s32), H_ref) <= 1e-6


@pytest.mark.parametrize("kind", ["sparse", "pbc"])
def test_ms_field_zero_cells(kind):
    shape = (9, 8, 2)
    gm, om = mesh_pair(*shape, 1e-9, 2e-9, 3e-9)
    m = random_m(shape, 13)
    ms = np.full(shape, 8e5)
    ms[::3, ::2, :] = 0.0
    m[ms == 0] = 0.0
    g, o = _pair(kind, _A_field(shape, 14), gm, om)
    _check(g, o, M.State(gm, ms, m), O.State(om, ms, m))


def test_sparse_homogeneous_cube_and_wall_are_exact():
    """micro_exch_sparse.cpp:36-84: H = 0 for a uniform m, and a wall between two
    z halves gives a field only in the two slices next to it."""
    n = 10
    mesh = M.Mesh(n, n, n, 1e-9, 1e-9, 1e-9)
    m = np.zeros((n, n, n, 3))
    m[..., 2] = 1.0
    t = M.SparseExchangeField(np.full((n, n, n), 1e-12), mesh)
    h = t.H_in_Apm(M.State(mesh, 8e5, m))
    assert np.all(h == 0.0)
    m[:, :, : n // 2, 2] = -1.0
    h2 = t.H_in_Apm(M.State(mesh, 8e5, m))
    assert np.all(h2[..., :2] == 0.0)
    assert np.all(h2[:, :, : n // 2 - 1, 2] == 0.0)
    assert np.all(h2[:, :, n // 2 + 1:, 2] == 0.0)
    assert np.abs(h2[:, :, n // 2 - 1: n // 2 + 1, 2]).min() > 0.0


def test_pbc_walls():
    """micro_exch_pbc.cpp:34-92: the periodic wrap puts a second wall between the
    slices 0 and nz-1."""
    n = 10
    mesh = M.Mesh(n, n, n, 1e-9, 1e-9, 1e-9)
    t = M.ExchangeFieldPBC(np.full((n, n, n), 1e-12), mesh)
    m = np.zeros((n, n, n, 3))
    m[..., 2] = 1.0
    s = M.State(mesh, 8e5, m)
    assert np.all(t.H_in_Apm(s) == 0.0)
    m[:, :, : n // 2, 2] = -1.0
    s.load_m(m)
    h2 = t.H_in_Apm(s)
    assert np.all(h2[:, :, 1: n // 2 - 1, 2] == 0.0)
    assert np.all(h2[:, :, n // 2 + 1: n - 1, 2] == 0.0)
    for sl in (0, n // 2 - 1, n // 2, n - 1):
        assert np.abs(h2[:, :, sl, 2]).min() > 0.0
    m3 = np.zeros((n, n, n, 3))
    m3[:, :, 0, 2] = 1.0
    s.load_m(m3)  # as state.m = ... in the reference: no Ms field
    h3 = t.H_in_Apm(s)
    assert np.all(h3[:, :, 2: n - 1, 2] == 0.0)
    assert np.abs(h3[:, :, 0:2, 2]).min() > 0.0
    assert np.abs(h3[:, :, n - 1, 2]).min() > 0.0


def test_exchange_field_array_without_mesh_is_an_error():
    with pytest.raises(RuntimeError):
        M.ExchangeField(np.full((3, 3, 3), 1e-11))


def test_mesh_of_another_size_is_rejected():
    t = M.SparseExchangeField(1e-11, M.Mesh(6, 5, 3, 1e-9, 1e-9, 1e-9))
    s = M.State(M.Mesh(12, 10, 3, 1e-9, 1e-9, 1e-9), 8e5, random_m((12, 10, 3), 1))
    with pytest.raises(M.MafError):
        t.H_in_Apm(s)


@pytest.mark.parametrize("dt", [2e-14, 1e-13])
def test_rk_attempt_with_sparse_exchange_matches_oracle(dt):
    """One RKF45 attempt at a fixed dt with demag + cell-wise exchange: the
    candidate m to 1e-12 and the scaled error norm to 1e-6 relative.  (Adaptive
    trajectories are not compared: the oracle's assembled matrix rounds the
    diagonal cancellation differently, which moves the first error norms, at the
    rounding floor, and with them the step sizes.)"""
    shape = (16, 8, 2)
    gm, om = mesh_pair(*shape, 2e-9, 2e-9, 2e-9)
    m = random_m(shape, 15)
    A = _A_field(shape, 16, zeros=False)
    d = M.DemagField(gm)
    gl = M.LLGIntegrator(0.5, [d, M.SparseExchangeField(A, gm)], "RKF45")
    ol = O.LLGIntegrator(0.5, [O.DemagField(om, N_real=d.get_N(symmetric=True)), O.SparseExchangeField(A, om)],
                         "RKF45")
    gs, os_ = M.State(gm, 8e5, m), O.State(om, 8e5, m)
    m_new, err = gl.rk_attempt(gs, "RKF45", dt)
    sumbk, err_ref = ol.attempt(os_, dt)
    assert rel_max(m_new, os_.m + sumbk) < 1e-12
    assert abs(err - err_ref) < 1e-6 * err_ref
