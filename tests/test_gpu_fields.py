"""Field-term parity of the CUDA library (through the C ABI) against the FP64 oracle.

Tolerances: the FP64 form must match the oracle to 1e-12 (relative L2 and
relative max norm) on identical inputs; the FP32-field form to 1e-5.  The
demag tensor is the one exception to "identical inputs": both sides assemble it
independently, and its far-field entries are dominated by the cancellation of
the 27-point Newell sums (magnumaf/src/field_terms/micro/demag_field.cpp:71-102),
so the device's and the oracle's libm differ there at the noise level.  The
convolution itself is therefore checked with the device's own tensor fed to the
oracle (1e-12), and the independently assembled field with a tolerance that
grows with the mesh as that noise does.
"""
import math

import numpy as np
import pytest

import maf_oracle as O
from helpers import mesh_pair, random_m, rel_l2, rel_max

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu

MESHES = [
    (6, 5, 4, 2e-9, 3e-9, 4e-9),
    (3, 5, 7, 1e-9, 1e-9, 1e-9),
    (16, 12, 1, 2e-9, 2e-9, 1e-9),
    (1, 1, 1, 1e-9, 1e-9, 1e-9),
    (1, 7, 3, 1e-9, 2e-9, 3e-9),
    (10, 1, 1, 3e-9, 3e-9, 3e-9),
]


def _pair_state(mesh_args, Ms=8e5, seed=0, precision="fp64", m=None):
    gm, om = mesh_pair(*mesh_args)
    if m is None:
        m = random_m((gm.nx, gm.ny, gm.nz), seed)
    return gm, om, M.State(gm, Ms, m, precision=precision), O.State(om, Ms, m)


LOCAL_TERMS = {
    "exchange": (lambda: M.ExchangeField(1.3e-11), lambda: O.ExchangeField(1.3e-11)),
    "dmi": (lambda: M.DmiField(3e-3, [0.2, -0.1, 1.0]), lambda: O.DmiField(3e-3, (0.2, -0.1, 1.0))),
    "uniaxial": (lambda: M.UniaxialAnisotropyField(1e6, [1, 2, 3]), lambda: O.UniaxialAnisotropyField(1e6, (1, 2, 3))),
    "cubic": (lambda: M.CubicAnisotropyField(-1e4, 2e3, 5e2, [1, 1, 0], [-1, 1, 0]),
              lambda: O.CubicAnisotropyField(-1e4, 2e3, 5e2, (1, 1, 0), (-1, 1, 0))),
}


@pytest.mark.parametrize("name", list(LOCAL_TERMS))
@pytest.mark.parametrize("mesh_args", MESHES)
def test_local_term_fp64(name, mesh_args):
    gm, om, gs, os_ = _pair_state(mesh_args, seed=1)
    gt, ot = LOCAL_TERMS[name][0](), LOCAL_TERMS[name][1]()
    h = gt.H_in_Apm(gs)
    ref = ot.H_in_Apm(os_)
    assert rel_l2(h, ref) < 1e-12 and rel_max(h, ref) < 1e-12
    e, eref = gt.Energy_in_J(gs), ot.Energy_in_J(os_)
    # energy scale: sum of |h.m| contributions (the exchange energy of a single cell
    # is an exact cancellation, so |eref| alone is no scale)
    dV = om.dx * om.dy * om.dz
    scale = O.mu0 * 8e5 * float(np.sum(np.abs(ref * os_.m))) * dV
    assert abs(e - eref) <= 1e-12 * max(abs(eref), scale)


@pytest.mark.parametrize("name", list(LOCAL_TERMS))
def test_local_term_fp32_field(name):
    gm, om, gs, os_ = _pair_state((24, 20, 3, 2e-9, 2e-9, 1e-9), seed=2, precision="fp32_field")
    gt, ot = LOCAL_TERMS[name][0](), LOCAL_TERMS[name][1]()
    h = gt.H_in_Apm_f32(gs)
    ref = ot.H_in_Apm(os_)
    assert rel_l2(h, ref) < 1e-5 and rel_max(h, ref) < 1e-5


@pytest.mark.parametrize("mesh_args", [(4, 5, 6, 0.1, 0.2, 0.3), (7, 3, 2, 1e-9, 2e-9, 3e-9)])
def test_bulk_dmi_exchange(mesh_args):
    gm, om, gs, os_ = _pair_state(mesh_args, seed=3)
    h = M.BulkDMIExchangeField(2e-3, 1.3e-11).H_in_Apm(gs)
    ref = O.BulkDMIExchangeField(2e-3, 1.3e-11).H_in_Apm(os_)
    assert rel_l2(h, ref) < 1e-12 and rel_max(h, ref) < 1e-12


def test_bulk_dmi_homogeneous_interior_zero():
    """python/test/micro_bulk_dmi_exchange_field.py:10-18"""
    mesh = M.Mesh(4, 5, 6, 0.1, 0.2, 0.3)
    m = np.zeros((4, 5, 6, 3))
    m[..., 0] = 1
    h = M.BulkDMIExchangeField(1, 1.3e-11).H_in_Apm(M.State(mesh, 8e5, m))
    assert abs(np.sum(h[1:-1, 1:-1, 1:-1])) < 1e-12


def test_zeeman_identity_and_energy():
    """python/test/external_field.py:8-30 plus the -mu0 Ms sum(h.m) dV energy."""
    gm, om, gs, os_ = _pair_state((3, 4, 2, 1e-9, 1e-9, 1e-9), seed=4)
    rng = np.random.default_rng(5)
    zee = rng.normal(size=(3, 4, 2, 3)) * 1e5
    t = M.ExternalField(zee)
    assert np.array_equal(t.H_in_Apm(gs), zee)
    assert abs(t.Energy_in_J(gs) - O.ExternalField(zee).Energy_in_J(os_)) <= 1e-12 * abs(
        O.ExternalField(zee).Energy_in_J(os_))
    u = M.ExternalField.uniform(1.0, -2.0, 3.0)
    hu = u.H_in_Apm(gs)
    assert np.all(hu[..., 0] == 1.0) and np.all(hu[..., 1] == -2.0) and np.all(hu[..., 2] == 3.0)


def test_uniaxial_axis_field_exact():
    """python/test/micro_anisotropy.py:36-54: h = 2 Ku/mu0 exactly."""
    axis = np.zeros((2, 1, 1, 3))
    axis[0, 0, 0, 0] = 1.0
    axis[1, 0, 0, 1] = -1.0
    aniso = M.UniaxialAnisotropyField(1.0, axis)
    m = np.zeros((2, 1, 1, 3))
    m[0, ..., 0] = 1.0
    m[1, ..., 1] = 1.0
    h = aniso.H_in_Apm(M.State(M.Mesh(2, 1, 1, 1, 1, 1), 1.0, m))
    assert h[0, 0, 0, 0] == 2 / M.Constants.mu0 and h[1, 0, 0, 1] == 2 / M.Constants.mu0
    assert h[0, 0, 0, 1] == 0 and h[0, 0, 0, 2] == 0 and h[1, 0, 0, 0] == 0 and h[1, 0, 0, 2] == 0


def test_spatial_parameter_fields():
    gm, om, gs, os_ = _pair_state((9, 7, 2, 1e-9, 1e-9, 1e-9), seed=6)
    rng = np.random.default_rng(7)
    Ku = rng.uniform(1e5, 1e6, size=(9, 7, 2))
    ax = rng.normal(size=(9, 7, 2, 3))
    h = M.UniaxialAnisotropyField(Ku, ax).H_in_Apm(gs)
    ref = O.UniaxialAnisotropyField(Ku, Ku1_axis_field=ax).H_in_Apm(os_)
    assert rel_l2(h, ref) < 1e-12
    D = rng.uniform(1e-3, 3e-3, size=(9, 7, 2))
    h = M.DmiField(D).H_in_Apm(gs)
    ref = O.DmiField(0.0, D_field=D).H_in_Apm(os_)
    assert rel_l2(h, ref) < 1e-12


def test_ms_field_zero_cells():
    """State with zero-norm cells creates an Ms_field (state.cpp:71-89); terms zero there."""
    m = random_m((6, 5, 2), 8)
    m[0, 0, 0] = 0.0
    m[3, 2, 1] = 0.0
    gm, om, gs, os_ = _pair_state((6, 5, 2, 1e-9, 1e-9, 1e-9), m=m)
    assert gs.Ms_field is not None and os_.Ms_field is not None
    assert np.array_equal(gs.Ms_field, os_.Ms_field)
    for name in ("exchange", "dmi", "uniaxial"):
        h = LOCAL_TERMS[name][0]().H_in_Apm(gs)
        ref = LOCAL_TERMS[name][1]().H_in_Apm(os_)
        assert rel_l2(h, ref) < 1e-12
    np.testing.assert_allclose(gs.mean_m(), os_.mean_m(), rtol=1e-13, atol=1e-15)


# --------------------------------------------------------------------- demag
@pytest.mark.parametrize("mesh_args", [(6, 5, 4, 2e-9, 3e-9, 4e-9), (3, 5, 7, 1e-9, 1e-9, 1e-9),
                                       (8, 6, 1, 1e-9, 1e-9, 1e-9), (1, 1, 1, 1e-9, 1e-9, 1e-9)])
def test_newell_real_tensor(mesh_args):
    """The device's FP64 Newell tensor (raw reference layout and the parity-exact
    one the spectral pipeline uses) against the oracle's, entry by entry."""
    gm, om = mesh_pair(*mesh_args)
    d = M.DemagField(gm)
    for N, ref in ((d.get_N(), O.demag_tensor_real(om)), (d.get_N(symmetric=True), O.demag_tensor_symmetric(om))):
        scale = np.abs(ref).max()
        assert np.abs(N - ref).max() < 1e-12 * scale


@pytest.mark.parametrize("mesh_args", [(12, 10, 6, 2e-9, 2e-9, 3e-9), (30, 20, 1, 3e-9, 3e-9, 3e-9),
                                       (3, 5, 7, 1e-9, 1e-9, 1e-9), (1, 1, 1, 1e-9, 1e-9, 1e-9),
                                       (1, 7, 3, 1e-9, 2e-9, 3e-9), (25, 1, 1, 1e-9, 1e-9, 1e-9),
                                       (16, 8, 4, 2e-9, 3e-9, 4e-9), (32, 16, 1, 3e-9, 3e-9, 2e-9),
                                       (64, 32, 16, 3e-9, 3e-9, 3e-9), (8, 64, 8, 1e-9, 2e-9, 1e-9)])
def test_demag_fp64_same_tensor(mesh_args):
    """Convolution parity on identical inputs: the oracle uses the device's tensor.
    Power-of-two meshes run the compile-time specialised passes, the others the
    generic mixed-radix ones."""
    gm, om, gs, os_ = _pair_state(mesh_args, seed=9)
    d = M.DemagField(gm)
    h = d.H_in_Apm(gs)
    ref = O.DemagField(om, N_real=d.get_N(symmetric=True)).H_in_Apm(os_)
    assert rel_l2(h, ref) < 1e-12 and rel_max(h, ref) < 1e-12


@pytest.mark.parametrize("mesh_args,tol", [((8, 6, 2, 2e-9, 2e-9, 3e-9), 1e-12),
                                           ((16, 12, 1, 2e-9, 2e-9, 1e-9), 1e-11),
                                           ((20, 16, 4, 3e-9, 3e-9, 3e-9), 1e-11)])
def test_demag_fp64_independent(mesh_args, tol):
    """Device and oracle each assemble the tensor (CUDA vs host libm asinh/atan);
    the tolerance is the measured rounding noise of the 27-point Newell sums at
    these sizes (it grows roughly as the fourth power of the mesh side)."""
    gm, om, gs, os_ = _pair_state(mesh_args, seed=10)
    h = M.DemagField(gm).H_in_Apm(gs)
    ref = O.DemagField(om, symmetric=True).H_in_Apm(os_)
    assert rel_l2(h, ref) < tol


def test_demag_energy_homogeneous_cube():
    """magnumaf/test/micro_demag.cpp:6-29: E = mu0 Ms^2 V / 6 within 5.3e-8."""
    x = y = z = 1e-9
    nx, ny, nz = 8, 10, 12
    mesh = M.Mesh(nx, ny, nz, x / nx, y / ny, z / nz)
    Ms = 1e5
    m = np.zeros((nx, ny, nz, 3))
    m[..., 0] = 1
    state = M.State(mesh, Ms, m)
    E = M.DemagField(mesh).Energy_in_J(state)
    analytic = 1.0 / 6.0 * x * y * z * Ms ** 2 * M.Constants.mu0
    assert abs(E - analytic) < (E + analytic) / 2 * 5.3e-8


def test_demag_energy_cube_with_airbox():
    """magnumaf/test/micro_demag.cpp:31-55"""
    x = y = z = 1e-9
    nx, ny, nz = 12, 10, 8
    mesh = M.Mesh(2 * nx, 2 * ny, 2 * nz, x / nx, y / ny, z / nz)
    Ms = 1e5
    m = np.zeros((2 * nx, 2 * ny, 2 * nz, 3))
    m[nx // 2:2 * nx - nx // 2, ny // 2:2 * ny - ny // 2, nz // 2:2 * nz - nz // 2, 0] = 1
    state = M.State(mesh, Ms, m)
    E = M.DemagField(mesh).Energy_in_J(state)
    analytic = 1.0 / 6.0 * x * y * z * Ms ** 2 * M.Constants.mu0
    assert abs(E - analytic) < (E + analytic) / 2 * 5.3e-8


@pytest.mark.parametrize("mesh_args", [(32, 24, 4, 3e-9, 3e-9, 3e-9), (40, 30, 1, 2e-9, 2e-9, 1e-9),
                                       (64, 32, 8, 3e-9, 3e-9, 3e-9), (128, 64, 1, 2e-9, 2e-9, 1e-9)])
def test_demag_fp32_field(mesh_args):
    gm, om, gs64, os_ = _pair_state(mesh_args, seed=11)
    gs32 = M.State(gm, 8e5, random_m((gm.nx, gm.ny, gm.nz), 11), precision="fp32_field")
    d = M.DemagField(gm)
    h64 = d.H_in_Apm(gs64)
    h32 = d.H_in_Apm_f32(gs32)
    assert rel_l2(h32, h64) < 1e-5 and rel_max(h32, h64) < 1e-5


def test_heff_sum_and_energy_fp64():
    """Demag + exchange + cubic + Zeeman (the metric's term set), summed in the LLG order."""
    gm, om, gs, os_ = _pair_state((20, 16, 4, 3e-9, 3e-9, 3e-9), Ms=8.6e5, seed=12)
    d = M.DemagField(gm)
    hz = (0.01 / O.mu0, -0.02 / O.mu0, 0.005 / O.mu0)
    gterms = [d, M.ExchangeField(1.3e-11), M.CubicAnisotropyField(-1e4), M.ExternalField.uniform(*hz)]
    oterms = [O.DemagField(om, N_real=d.get_N(symmetric=True)), O.ExchangeField(1.3e-11), O.CubicAnisotropyField(-1e4),
              O.ExternalField(np.broadcast_to(np.array(hz), (20, 16, 4, 3)))]
    llg = M.LLGIntegrator(0.01, gterms, "DP45")
    h = llg.H_in_Apm(gs)
    ref = O.Heff_in_Apm(oterms, os_)
    assert rel_l2(h, ref) < 1e-12 and rel_max(h, ref) < 1e-12
    E = llg.Eeff_in_J(gs)
    Eref = O.Eeff_in_J(oterms, os_)
    assert abs(E - Eref) < 1e-12 * abs(Eref)
    # dm/dt of LLGIntegrator::f
    oll = O.LLGIntegrator(0.01, oterms)
    np.testing.assert_allclose(llg.dmdt(gs), oll.f(os_), rtol=0, atol=1e-12 * np.abs(oll.f(os_)).max())


def test_heff_fp32_field_vs_fp64():
    gm, om = mesh_pair(32, 32, 4, 3e-9, 3e-9, 3e-9)
    m = random_m((32, 32, 4), 13)
    d = M.DemagField(gm)
    terms = [d, M.ExchangeField(1.3e-11), M.CubicAnisotropyField(-1e4), M.ExternalField.uniform(1e4, 2e4, -3e4)]
    llg = M.LLGIntegrator(0.01, terms, "DP45")
    h64 = llg.H_in_Apm(M.State(gm, 8.6e5, m))
    h32 = llg.H_in_Apm_f32(M.State(gm, 8.6e5, m, precision="fp32_field"))
    assert rel_l2(h32, h64) < 1e-5 and rel_max(h32, h64) < 1e-5


# ------------------------------------------------------------- error paths
def test_unsupported_fft_length():
    with pytest.raises(M.MafError) as e:
        M.DemagField(M.Mesh(17, 4, 1, 1e-9, 1e-9, 1e-9))
    assert e.value.code == 6


def test_cubic_axes_not_perpendicular():
    with pytest.raises(M.MafError) as e:
        M.CubicAnisotropyField(1e4, 0, 0, [1, 0, 0], [1, 1, 0])
    assert e.value.code == 1


def test_mesh_mismatch_rejected():
    gm, om, gs, os_ = _pair_state((6, 5, 4, 1e-9, 1e-9, 1e-9))
    d = M.DemagField(M.Mesh(6, 5, 3, 1e-9, 1e-9, 1e-9))
    with pytest.raises(M.MafError) as e:
        d.H_in_Apm(gs)
    assert e.value.code == 1
