"""The oracle's SparseExchangeField / ExchangeFieldPBC against the reference's own
tests of those terms (magnumaf/test/micro_exch_sparse.cpp:36-84,
magnumaf/test/micro_exch_pbc.cpp:34-92, python/test/micro_exchange_pbc.py:7-16)
and against the oracle's zero-padded ExchangeField, an independent restatement."""
import numpy as np

import maf_oracle as O
from helpers import random_m


def _sum3d(a):
    return float(np.sum(a))


def test_sparse_homogeneous_cube_and_wall():
    """micro_exch_sparse.cpp:36-84 (A field, COO assembly)."""
    n = 10
    mesh = O.Mesh(n, n, n, 1e-9, 1e-9, 1e-9)
    m = np.zeros((n, n, n, 3))
    m[..., 2] = 1.0
    t = O.SparseExchangeField(np.full((n, n, n), 1e-12), mesh)
    s = O.State(mesh, 8e5, m)
    h = t.H_in_Apm(s)
    scale = 2 * 1e-12 / (O.mu0 * 1e-18) / 8e5
    assert _sum3d(h[..., :2]) == 0.0
    assert abs(_sum3d(h[..., 2])) <= 1e-12 * scale * n ** 3
    m2 = m.copy()
    m2[:, :, : n // 2, 2] = -1.0
    h2 = t.H_in_Apm(O.State(mesh, 8e5, m2))
    assert _sum3d(h2[..., :2]) == 0.0
    assert np.abs(h2[:, :, : n // 2 - 1, 2]).max() <= 1e-12 * scale
    assert np.abs(h2[:, :, n // 2 + 1:, 2]).max() <= 1e-12 * scale
    assert _sum3d(np.abs(h2[:, :, n // 2 - 1: n // 2 + 1, 2])) != 0.0


def test_pbc_homogeneous_cube_and_walls():
    """micro_exch_pbc.cpp:34-92."""
    n = 10
    mesh = O.Mesh(n, n, n, 1e-9, 1e-9, 1e-9)
    t = O.ExchangeFieldPBC(np.full((n, n, n), 1e-12), mesh)
    scale = 2 * 1e-12 / (O.mu0 * 1e-18) / 8e5
    m = np.zeros((n, n, n, 3))
    m[..., 2] = 1.0
    h = t.H_in_Apm(O.State(mesh, 8e5, m))
    assert _sum3d(h[..., :2]) == 0.0
    assert np.abs(h).max() <= 1e-12 * scale
    m[:, :, : n // 2, 2] = -1.0
    h2 = t.H_in_Apm(O.State(mesh, 8e5, m))
    assert _sum3d(h2[..., :2]) == 0.0
    assert np.abs(h2[:, :, 1: n // 2 - 1, 2]).max() <= 1e-12 * scale
    assert np.abs(h2[:, :, n // 2 + 1: n - 1, 2]).max() <= 1e-12 * scale
    for sl in (0, n // 2 - 1, n // 2, n - 1):
        assert np.abs(h2[:, :, sl, 2]).min() > 1e-3 * scale  # the wrapped wall at 0 / nz-1 too
    # the reference sets state.m after construction, so no Ms field marks the empty cells
    s3 = O.State(mesh, 8e5, m)
    s3.m = np.zeros((n, n, n, 3))
    s3.m[:, :, 0, 2] = 1.0
    h3 = t.H_in_Apm(s3)
    assert np.abs(h3[:, :, 2: n - 1, 2]).max() == 0.0
    assert _sum3d(np.abs(h3[:, :, 0:2, 2])) != 0.0
    assert _sum3d(np.abs(h3[:, :, n - 1, 2])) != 0.0


def test_pbc_python_homogeneous():
    """python/test/micro_exchange_pbc.py:7-16 (scalar A)."""
    mesh = O.Mesh(8, 10, 12, 1e-9, 2e-9, 3e-9)
    m = np.zeros((8, 10, 12, 3))
    m[..., 2] = 1.0
    h = O.ExchangeFieldPBC(1e-12, mesh).H_in_Apm(O.State(mesh, 1e5, m))
    assert abs(float(np.sum(h))) < 0.5e-5


def test_scalar_sparse_is_exchange_without_the_diagonal():
    """The scalar matrix has no diagonal (sparse_exchange_field.cpp:25-101), so it
    differs from the zero-padded stencil (exchange_field.cpp:115-126) by
    2A/(mu0 Ms) * 2 (1/dx^2 + 1/dy^2 + 1/dz^2) m."""
    shape = (7, 5, 3)
    mesh = O.Mesh(*shape, 2e-9, 3e-9, 1.5e-9)
    m = random_m(shape, 3)
    s = O.State(mesh, 8e5, m)
    A = 1.3e-11
    hs = O.SparseExchangeField(A, mesh).H_in_Apm(s)
    he = O.ExchangeField(A).H_in_Apm(s)
    diag = 2 * A / (O.mu0 * 8e5) * 2 * (1 / mesh.dx ** 2 + 1 / mesh.dy ** 2 + 1 / mesh.dz ** 2)
    np.testing.assert_allclose(hs - he, diag * m, rtol=1e-9, atol=1e-9 * np.abs(hs).max())


def test_uniform_A_field_matches_exchange_inside():
    """With a uniform A field the harmonic weights are 2A/(mu0 d^2): interior
    cells equal the zero-padded stencil."""
    shape = (8, 6, 5)
    mesh = O.Mesh(*shape, 2e-9, 3e-9, 1.5e-9)
    m = random_m(shape, 4)
    s = O.State(mesh, 8e5, m)
    hs = O.SparseExchangeField(np.full(shape, 1e-11), mesh).H_in_Apm(s)
    he = O.ExchangeField(1e-11).H_in_Apm(s)
    np.testing.assert_allclose(hs[1:-1, 1:-1, 1:-1], he[1:-1, 1:-1, 1:-1], rtol=1e-9,
                               atol=1e-9 * np.abs(he).max())


def test_A_zero_rows_are_empty():
    shape = (6, 5, 4)
    mesh = O.Mesh(*shape, 1e-9, 1e-9, 1e-9)
    A = np.full(shape, 1e-11)
    A[2, 2, 1] = 0.0
    t = O.SparseExchangeField(A, mesh)
    h = t.H_in_Apm(O.State(mesh, 8e5, random_m(shape, 5)))
    assert np.all(h[2, 2, 1] == 0.0)
    # a neighbour with A = 0 contributes a zero weight
    assert t.matr[2 + 6 * (2 + 5 * 1), 3 + 6 * (2 + 5 * 1)] == 0.0
