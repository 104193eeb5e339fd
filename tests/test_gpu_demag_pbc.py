"""DemagFieldPBC (demag_field_pbc.cpp) against the oracle, and the reference's
own tests of that term (magnumaf/test/micro_demag_pbc.cpp:5-70) run on the GPU."""
import numpy as np
import pytest

import maf_oracle as O
from helpers import mesh_pair, random_m, rel_l2, rel_max

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(8, 6, 4), (16, 10, 1), (12, 9, 5), (2, 3, 7), (30, 14, 3)])
@pytest.mark.parametrize("ms_field", [False, True])
def test_matches_oracle(shape, ms_field):
    gm, om = mesh_pair(*shape, 2e-9, 3e-9, 1.5e-9)
    m = random_m(shape, 31)
    if ms_field:
        ms = np.random.default_rng(32).uniform(4e5, 9e5, size=shape)
        ms[::3, ::2, :] = 0.0
        m[ms == 0] = 0.0
    else:
        ms = 8e5
    g, o = M.DemagFieldPBC(), O.DemagFieldPBC()
    gs, os_ = M.State(gm, ms, m), O.State(om, ms, m)
    H = g.H_in_Apm(gs)
    H_ref = o.H_in_Apm(os_)
    np.testing.assert_allclose(H, H_ref, rtol=1e-12, atol=1e-12 * np.abs(H_ref).max())
    E, E_ref = g.Energy_in_J(gs), o.Energy_in_J(os_)
    assert abs(E - E_ref) <= 1e-11 * abs(E_ref)
    s32 = M.State(gm, ms, m, precision="fp32_field")
    assert rel_l2(g.H_in_Apm(s32), H_ref) <= 1e-5


def _plane(mesh, Ms=8e5, m_layer=7, nm=0, err=0.04):
    m = np.zeros((mesh.nx, mesh.ny, mesh.nz, 3))
    m[:, :, m_layer:m_layer + nm + 1, 2] = 1.0
    h = M.DemagFieldPBC().H_in_Apm(M.State(mesh, Ms, m))
    hz = h[mesh.nx // 2, mesh.ny // 2, :, 2]
    for i in range(mesh.nz):
        if i < m_layer or i > m_layer + nm:
            assert abs(abs(hz[m_layer] - hz[i]) - Ms) <= err
    return hz[m_layer], hz[0]


def test_magnetic_xy_plane():
    """micro_demag_pbc.cpp:34-70 with the CPU backend's tolerances."""
    hzl_1, hz0_1 = _plane(M.Mesh(32, 18, 16, 1e-9, 1e-9, 1e-9))
    hzl_2, hz0_2 = _plane(M.Mesh(32, 18, 16, 1e-9, 1e-9, 2e-9))
    assert hzl_1 == hzl_2 and hz0_1 == hz0_2
    nz = 16
    mesh = M.Mesh(32, 18, nz, 1e-9, 1e-9, 1e-9)
    res = [_plane(mesh, nm=nm, err=e) for nm, e in [(0, 0.04), (1, 7e-2), (2, 0.2), (3, 0.2)]]
    for k, tol in [(1, 1e-7), (2, 2e-7), (3, 3e-7)]:
        assert abs(res[0][0] / res[k][0] - (nz - 1.0) / (nz - 1.0 - k)) <= tol
    for k, tol in [(0, 2e-5), (1, 1e-5), (2, 1e-5), (3, 1e-5)]:
        assert abs(abs(res[k][0] / res[k][1]) - (nz - 1.0 - k) / (k + 1.0)) <= tol


def test_odd_nx_is_unsupported():
    s = M.State(M.Mesh(7, 6, 4, 1e-9, 1e-9, 1e-9), 8e5, random_m((7, 6, 4), 2))
    with pytest.raises(M.MafError):
        M.DemagFieldPBC().H_in_Apm(s)


def test_one_term_on_two_meshes():
    """The term has no mesh of its own: each evaluation uses the state's."""
    t = M.DemagFieldPBC()
    for shape in [(8, 6, 4), (10, 4, 2), (8, 6, 4)]:
        gm, om = mesh_pair(*shape, 1e-9, 2e-9, 3e-9)
        m = random_m(shape, 33)
        H = t.H_in_Apm(M.State(gm, 8e5, m))
        H_ref = O.DemagFieldPBC().H_in_Apm(O.State(om, 8e5, m))
        np.testing.assert_allclose(H, H_ref, rtol=1e-12, atol=1e-12 * np.abs(H_ref).max())


@pytest.mark.parametrize("dt", [2e-14, 1e-13])
def test_rk_attempt_with_pbc_demag_matches_oracle(dt):
    shape = (16, 8, 4)
    gm, om = mesh_pair(*shape, 2e-9, 2e-9, 2e-9)
    m = random_m(shape, 34)
    gl = M.LLGIntegrator(0.5, [M.DemagFieldPBC(), M.ExchangeFieldPBC(1.3e-11, gm)], "RKF45")
    ol = O.LLGIntegrator(0.5, [O.DemagFieldPBC(), O.ExchangeFieldPBC(1.3e-11, om)], "RKF45")
    gs, os_ = M.State(gm, 8e5, m), O.State(om, 8e5, m)
    m_new, err = gl.rk_attempt(gs, "RKF45", dt)
    sumbk, err_ref = ol.attempt(os_, dt)
    assert rel_max(m_new, os_.m + sumbk) < 1e-12
    assert abs(err - err_ref) < 1e-6 * err_ref
