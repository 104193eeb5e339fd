"""Pins the FP64 oracle to the reference's own known-answer tests and golden
vectors (CPU only).  Every test cites the reference test it restates."""
import math

import numpy as np
import pytest

import maf_oracle as O


def test_constants():
    """python/test/constants.py:8-10"""
    assert O.mu0 == 4e-7 * math.pi
    assert O.gamma == 221276.14886372554


def _sp4():
    mesh = O.Mesh(100, 25, 1, 5.e-7 / 100, 1.25e-7 / 25, 3.e-9)
    m = np.zeros((100, 25, 1, 3))
    m[1:-1, :, :, 0] = 1.0
    m[0, :, :, 1] = 1.0
    m[-1, :, :, 1] = 1.0
    return mesh, O.State(mesh, 8e5, m)


@pytest.mark.slow
def test_sp4_relax_and_switch():
    """muMAG SP4 (python/test/sp4.py:21-62): integrals of <m> over 0-1 ns (alpha=1)
    and 1-2 ns (alpha=0.02, -24.6/4.3 mT), RKF45 with the default controller,
    1e-15 absolute."""
    mesh, state = _sp4()
    llg = O.LLGIntegrator(1.0, [O.DemagField(mesh), O.ExchangeField(1.3e-11)])
    ix = iy = iz = 0.0
    while state.t < 1e-9:
        t1 = state.t
        llg.step(state)
        dt = state.t - t1
        mm = state.mean_m()
        ix += mm[0] * dt
        iy += mm[1] * dt
        iz += mm[2] * dt
    assert abs(ix - 9.81206172824e-10) < 1e-15
    assert abs(iy - 9.14350283169e-11) < 1e-15
    assert abs(iz + 5.74381785359e-13) < 1e-15
    llg.alpha = 0.02
    zee = np.zeros((100, 25, 1, 3))
    zee[..., 0] = -24.6e-3 / O.mu0
    zee[..., 1] = +4.3e-3 / O.mu0
    llg.terms.append(O.ExternalField(zee))
    ix = iy = iz = 0.0
    while state.t < 2e-9:
        t1 = state.t
        llg.step(state)
        dt = state.t - t1
        mm = state.mean_m()
        ix += mm[0] * dt
        iy += mm[1] * dt
        iz += mm[2] * dt
    assert abs(ix + 6.41261165705e-10) < 1e-15
    assert abs(iy - 1.47353233738e-10) < 1e-15
    assert abs(iz + 1.78144535231e-11) < 1e-15


@pytest.mark.parametrize("air", [False, True])
def test_demag_energy_homogeneous_cube(air):
    """magnumaf/test/micro_demag.cpp:6-55 (with and without an air box), 5.3e-8 relative."""
    x = y = z = 1.e-9
    if not air:
        nx, ny, nz = 8, 10, 12
        mesh = O.Mesh(nx, ny, nz, x / nx, y / ny, z / nz)
        m = np.zeros((nx, ny, nz, 3))
        m[..., 0] = 1
    else:
        nx, ny, nz = 12, 10, 8
        mesh = O.Mesh(2 * nx, 2 * ny, 2 * nz, x / nx, y / ny, z / nz)
        m = np.zeros((2 * nx, 2 * ny, 2 * nz, 3))
        m[nx // 2:2 * nx - nx // 2, ny // 2:2 * ny - ny // 2, nz // 2:2 * nz - nz // 2, 0] = 1
    Ms = 1e5
    state = O.State(mesh, Ms, m)
    demag = O.DemagField(mesh)
    E = demag.Energy_in_J(state)
    analytic = 1. / 6. * x * y * z * Ms ** 2 * O.mu0
    assert abs(E - analytic) < (E + analytic) / 2. * 5.3e-8


def test_newell_known_values():
    """Newell tensor properties pinned by magnumaf/test/nonequi_demag.cpp:84-95
    (Nxy vanishes on the x axis) and by the closed-form self-demag of a cube
    (Nxx = Nyy = Nzz = -1/3 at distance 0, trace -1) and Laplace's equation
    (trace 0 elsewhere)."""
    a = 2.0
    assert O.Nxy(2, 0, 0, a, a, a) == 0
    nxx = O.Nxx(0, 0, 0, a, a, a)
    assert abs(nxx + 1.0 / 3.0) < 1e-14
    for (i, j, k) in [(1, 0, 0), (1, 2, 3), (3, 1, 2)]:
        tr = O.Nxx(i, j, k, a, a, a) + O.Nxx(j, k, i, a, a, a) + O.Nxx(k, i, j, a, a, a)
        assert abs(tr) < 1e-13
    # point-dipole limit along x at moderate distance: Nxx -> 2/(4 pi r^3) (cell units)
    r = 10
    assert abs(O.Nxx(r, 0, 0, 1, 1, 1) - 2 / (4 * math.pi * r ** 3)) < 1e-3 * 2 / (4 * math.pi * r ** 3)


def test_newell_symmetry():
    """Nxx even, Nxy odd in x and y (the symmetries the reduced spectral tensor relies on).
    Mirrored entries are summed in a different order, so they agree only to the
    cancellation noise of the 27-point sums: eps * |f| / (4 pi dV), with |f| ~ r^3."""
    d = (1.0, 2.0, 3.0)
    for (i, j, k) in [(1, 2, 3), (4, 1, 0), (2, 5, 1)]:
        r3 = (i * d[0]) ** 2 + (j * d[1]) ** 2 + (k * d[2]) ** 2
        noise = 64 * 2.2e-16 * (r3 ** 1.5 + 1) / (4 * math.pi * d[0] * d[1] * d[2])
        assert abs(O.Nxx(i, j, k, *d) - O.Nxx(-i, -j, -k, *d)) < noise
        assert abs(O.Nxy(i, j, k, *d) + O.Nxy(-i, j, k, *d)) < noise
        assert abs(O.Nxy(i, j, k, *d) + O.Nxy(i, -j, k, *d)) < noise
        assert abs(O.Nxy(i, j, k, *d) - O.Nxy(i, j, -k, *d)) < noise


def test_cubic_constructor_axes():
    """magnumaf/test/cubic_anisotropy_field.cpp:6-15"""
    c = O.CubicAnisotropyField(1, 1, 1, (1, 1, 0), (-1, 1, 0))
    np.testing.assert_allclose(c.c1, [1 / math.sqrt(2), 1 / math.sqrt(2), 0], rtol=0, atol=1e-16)
    np.testing.assert_allclose(c.c2, [-1 / math.sqrt(2), 1 / math.sqrt(2), 0], rtol=0, atol=1e-16)
    np.testing.assert_allclose(c.c3, [0, 0, 1], rtol=0, atol=1e-16)
    with pytest.raises(ValueError):
        O.CubicAnisotropyField(1, 0, 0, (1, 0, 0), (1, 1, 0))


@pytest.mark.parametrize("K,z", [(1e6, 0.0), (-1e6, 0.0), (1e6, 0.5), (1e6, 1.0)])
def test_cubic_energy_rotation(K, z):
    """magnumaf/test/cubic_anisotropy_field.cpp:19-161: 64 in-plane angles,
    Kc1/Kc2/Kc3 energies against the analytic densities."""
    mesh = O.Mesh(2, 2, 2, 1e-9, 1e-9, 1e-9)
    ncells = 8
    dV = 1e-27
    Ms = np.full((2, 2, 2), 1 / O.mu0)
    for i in range(64):
        x = math.sin(2 * math.pi * i / 64)
        y = math.cos(2 * math.pi * i / 64)
        m = np.zeros((2, 2, 2, 3))
        m[..., 0], m[..., 1], m[..., 2] = x, y, z
        state = O.State(mesh, Ms, m)
        v = np.array([x, y, z]) / math.sqrt(x * x + y * y + z * z)
        c1m2, c2m2, c3m2 = v[0] ** 2, v[1] ** 2, v[2] ** 2
        e1 = ncells * K * (c1m2 * c2m2 + c1m2 * c3m2 + c2m2 * c3m2)
        E1 = O.CubicAnisotropyField(K, 0, 0).Energy_in_J(state)
        assert abs(E1 - e1 * dV) < 2e-36 and abs(E1 / dV - e1) < 2e-9
        e2 = ncells * K * (c1m2 * c2m2 * c3m2)
        E2 = O.CubicAnisotropyField(0, K, 0).Energy_in_J(state)
        assert abs(E2 - e2 * dV) < 1e-36 and abs(E2 / dV - e2) < 1e-10
        c1m4, c2m4, c3m4 = v[0] ** 4, v[1] ** 4, v[2] ** 4
        e3 = ncells * K * (c1m4 * c2m4 + c1m4 * c3m4 + c2m4 * c3m4)
        E3 = O.CubicAnisotropyField(0, 0, K).Energy_in_J(state)
        assert abs(E3 - e3 * dV) < 5e-37 and abs(E3 / dV - e3) < 5e-10


def test_cubic_energy_single_cell():
    """python/test/cubic_anisotropy_field.py:6-16: 250000 J/m^3 at m = (1,1,0)/sqrt(2)."""
    mesh = O.Mesh(1, 1, 1, 1e-9, 1e-9, 1e-9)
    m = np.zeros((1, 1, 1, 3))
    m[..., 0] = 1.
    m[..., 1] = 1.
    E = O.CubicAnisotropyField(1e6, 0, 0).Energy_in_J(O.State(mesh, 1.0, m))
    assert abs(E - 250000 * 1e-27) < 1e-36


def test_uniaxial_axis_field_exact():
    """python/test/micro_anisotropy.py:36-54"""
    axis = np.zeros((2, 1, 1, 3))
    axis[0, 0, 0, 0] = 1.
    axis[1, 0, 0, 1] = -1.
    m = np.zeros((2, 1, 1, 3))
    m[0, ..., 0] = 1.
    m[1, ..., 1] = 1.
    state = O.State(O.Mesh(2, 1, 1, 1, 1, 1), 1.0, m)
    h = O.UniaxialAnisotropyField(1.0, Ku1_axis_field=axis).H_in_Apm(state)
    assert h[0, 0, 0, 0] == 2 / O.mu0 and h[1, 0, 0, 1] == 2 / O.mu0
    assert h[0, 0, 0, 1] == 0 and h[0, 0, 0, 2] == 0 and h[1, 0, 0, 0] == 0 and h[1, 0, 0, 2] == 0


def test_zeeman_identity():
    """python/test/external_field.py:8-30"""
    mesh = O.Mesh(3, 1, 1, 1e-10, 1e-10, 1e-10)
    m = np.zeros((3, 1, 1, 3))
    m[..., 0] = 1.0
    zee = np.zeros((3, 1, 1, 3))
    zee[0, 0, 0, 0] = zee[1, 0, 0, 1] = zee[2, 0, 0, 2] = 1
    h = O.ExternalField(zee).H_in_Apm(O.State(mesh, 0.0, m))
    assert np.array_equal(h, zee)


def test_bulk_dmi_homogeneous_interior_zero():
    """python/test/micro_bulk_dmi_exchange_field.py:10-18"""
    mesh = O.Mesh(4, 5, 6, 0.1, 0.2, 0.3)
    m = np.zeros((4, 5, 6, 3))
    m[..., 0] = 1
    h = O.BulkDMIExchangeField(1, 1.3e-11).H_in_Apm(O.State(mesh, 8e5, m))
    assert abs(np.sum(h[1:-1, 1:-1, 1:-1])) < 1e-12


def test_central_difference_sign():
    """magnumaf/test/math.cpp:8-19: d/dx of iota is +1/h away from the edges
    (af::convolve is a true, flipped convolution)."""
    a = np.arange(10 * 5 * 4 * 6, dtype=np.float64).reshape((10, 5, 4, 6), order="F")
    d = O.central_diff(a, 2.0, 0)
    assert np.all(d[1:-1] == 0.5)


class _ODE(O.AdaptiveRungeKutta):
    def f(self, state):
        return state.t * np.sqrt(state.m)


@pytest.mark.parametrize("scheme,steps,tol", [("BS23", 200, 1e-12), ("DP45", 100, 1e-8), ("RKF45", 100, 1e-8)])
def test_adaptive_rk_analytic(scheme, steps, tol):
    """magnumaf/test/adaptive_runge_kutta.cpp:9-74: y' = t sqrt(y), y(0) = 1,
    y = (t^2 + 4)^2 / 16, normalize_ = false, Controller(1e-15, 1e15, 1e-10, 1e-10)."""
    rk = _ODE(scheme, O.Controller(1e-15, 1e15, 1e-10, 1e-10), normalize_=False)
    st = O.State.__new__(O.State)
    st.mesh = O.Mesh(1, 1, 1, 1, 1, 1)
    st.m = np.array([1.0, 0.0, 0.0]).reshape(1, 1, 1, 3)
    st.t = 0.0
    st.steps = 0
    st.Ms = 1.0
    st.Ms_field = None
    for _ in range(steps):
        rk.step(st)
        assert abs(st.m[0, 0, 0, 0] - (st.t ** 2 + 4) ** 2 / 16) < tol


def test_state_normalize_and_mean():
    """magnumaf/test/state.cpp:40-137"""
    mesh = O.Mesh(1, 1, 1, 1e-9, 1e-9, 1e-9)
    s = O.State(mesh, 1.0, np.ones((1, 1, 1, 3)))
    assert np.all(s.m == 1 / math.sqrt(3))
    mesh = O.Mesh(2, 2, 2, 1e-9, 1e-9, 1e-9)
    for c in range(3):
        m0 = np.zeros((2, 2, 2, 3))
        m0[0, :, :, c] = 1
        s = O.State(mesh, 1e6, m0)
        assert s.Ms_field is not None
        expect = [0.0, 0.0, 0.0]
        expect[c] = 1.0
        assert list(s.mean_m()) == expect


@pytest.mark.parametrize("args,bound", [((12, 10, 6, 2e-9, 2e-9, 3e-9), 1e-11), ((3, 5, 7, 1e-9, 1e-9, 1e-9), 1e-12),
                                        ((100, 25, 1, 5e-9, 5e-9, 3e-9), 1e-8)])
def test_symmetric_tensor_matches_reference_tensor(args, bound):
    """The parity-exact tensor changes the demag field on the mesh only by the
    rounding noise of the reference's own 27-point Newell sums (entries at
    |j| = P/2 never reach the truncated output; the others differ by the sum
    order of mirrored entries).  The bound is that noise, measured here."""
    mesh = O.Mesh(*args)
    rng = np.random.default_rng(9)
    m = rng.normal(size=args[:3] + (3,))
    state = O.State(mesh, 8e5, m)
    h_raw = O.DemagField(mesh).H_in_Apm(state)
    h_sym = O.DemagField(mesh, symmetric=True).H_in_Apm(state)
    assert np.linalg.norm(h_raw - h_sym) / np.linalg.norm(h_raw) < bound
