"""The oracle's DemagFieldPBC against the reference's own tests of that term
(magnumaf/test/micro_demag_pbc.cpp:5-70, python/test/micro_demag_pbc.py:7-16):
an infinite magnetic plane in xy has a field jump of Ms across the layer, the
field does not depend on dz, and the layer/outside fields scale with the number
of non-magnetic layers."""
import numpy as np
import pytest

import maf_oracle as O


def plane_fields(mesh, Ms=8e5, m_layer=7, nm=0, err=0.04):
    """micro_demag_pbc.cpp:5-31: m = z on layers [m_layer, m_layer + nm], zero
    elsewhere; returns (Hz in the layer, Hz in layer 0) at (nx/2, ny/2)."""
    m = np.zeros((mesh.nx, mesh.ny, mesh.nz, 3))
    m[:, :, m_layer:m_layer + nm + 1, 2] = 1.0
    h = O.DemagFieldPBC().H_in_Apm(O.State(mesh, Ms, m))
    hz = h[mesh.nx // 2, mesh.ny // 2, :, 2]
    for i in range(mesh.nz):
        if i < m_layer or i > m_layer + nm:
            assert abs(abs(hz[m_layer] - hz[i]) - Ms) <= err
    return hz[m_layer], hz[0]


def test_magnetic_xy_plane():
    hzl_1, hz0_1 = plane_fields(O.Mesh(32, 18, 16, 1e-9, 1e-9, 1e-9))
    hzl_2, hz0_2 = plane_fields(O.Mesh(32, 18, 16, 1e-9, 1e-9, 2e-9))
    assert hzl_1 == hzl_2 and hz0_1 == hz0_2  # dz scales by a power of two
    nz = 16
    mesh = O.Mesh(32, 18, nz, 1e-9, 1e-9, 1e-9)
    res = [plane_fields(mesh, nm=nm, err=e) for nm, e in [(0, 0.04), (1, 7e-2), (2, 0.2), (3, 0.2)]]
    for k, tol in [(1, 1e-7), (2, 2e-7), (3, 3e-7)]:
        assert abs(res[0][0] / res[k][0] - (nz - 1.0) / (nz - 1.0 - k)) <= tol
    for k, tol in [(0, 2e-5), (1, 1e-5), (2, 1e-5), (3, 1e-5)]:
        assert abs(abs(res[k][0] / res[k][1]) - (nz - 1.0 - k) / (k + 1.0)) <= tol


def test_python_homogen_m():
    """python/test/micro_demag_pbc.py:7-16."""
    mesh = O.Mesh(8, 10, 12, 1e-9, 2e-9, 3e-9)
    m = np.zeros((8, 10, 12, 3))
    m[:, :, 4:5, 2] = 1.0
    h = O.DemagFieldPBC().H_in_Apm(O.State(mesh, 1e5, m))
    assert float(np.sum(h)) != 0.0


def test_uniform_m_has_no_field():
    """Only the k = 0 mode is non-zero for a uniform m, and u(0) = 0."""
    mesh = O.Mesh(8, 6, 4, 1e-9, 2e-9, 3e-9)
    m = np.zeros((8, 6, 4, 3))
    m[..., 0] = 0.6
    m[..., 2] = 0.8
    h = O.DemagFieldPBC().H_in_Apm(O.State(mesh, 8e5, m))
    assert np.abs(h).max() <= 1e-9 * 8e5


def test_odd_nx_is_rejected():
    mesh = O.Mesh(7, 6, 4, 1e-9, 1e-9, 1e-9)
    with pytest.raises(ValueError):
        O.DemagFieldPBC().H_in_Apm(O.State(mesh, 8e5, np.ones((7, 6, 4, 3)) / np.sqrt(3)))
