"""String method (magnumaf/src/solvers/string_method.cpp) on the device
against the oracle's restatement: initial images, arc lengths, images and
energies after string steps, and run()'s lowest barrier and output files."""
import os

import numpy as np
import pytest

import maf_oracle as O
import maf_string_oracle as SO
from helpers import mesh_pair

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu

SHAPE = (16, 16, 1)
MS = 1.1e6


def _images():
    n = SHAPE[0]
    a = np.zeros(SHAPE + (3,))
    a[..., 2] = 1.0
    c = (n - 1) / 2.0
    for i in range(n):
        for j in range(n):
            if (i - c) ** 2 + (j - c) ** 2 <= 4.0 ** 2:
                a[i, j, 0, 2] = -1.0
    a[..., 0] += 0.1
    b = np.zeros(SHAPE + (3,))
    b[..., 0] = 0.1
    b[..., 2] = 1.0
    return O.normalize(a), O.normalize(b)


def _setup(n_interp, dt, reverse=False):
    gm, om = mesh_pair(*SHAPE, 1e-9, 1e-9, 1e-9)
    d = M.DemagField(gm)
    g_terms = [d, M.ExchangeField(1.6e-11), M.DmiField(4e-3), M.UniaxialAnisotropyField(1e6),
               M.ExternalField.uniform(0.0, 0.0, 0.01 / O.mu0)]
    o_terms = [O.DemagField(om, N_real=d.get_N(symmetric=True)), O.ExchangeField(1.6e-11), O.DmiField(4e-3),
               O.UniaxialAnisotropyField(1e6), O.ExternalField(np.array([0.0, 0.0, 0.01 / O.mu0]))]
    a, b = _images()
    if reverse:  # uniform first: the energy rises along the string, the barrier is positive
        a, b = b, a
    g_llg = M.LLGIntegrator(1.0, g_terms)
    o_llg = O.LLGIntegrator(1.0, o_terms)
    gs = M.State(gm, MS, a)
    os_ = O.State(om, MS, a)
    g = M.StringMethod(gs, [a, b], n_interp, dt, g_llg)
    o = SO.StringMethod(os_, [a, b], n_interp, dt, o_llg)
    return g, o


def test_initial_string_matches_oracle():
    g, o = _setup(5, 5e-14)
    x, xi = g.x()
    np.testing.assert_allclose(x[:2], o.x, rtol=1e-13)
    np.testing.assert_allclose(xi, o.x_interp, rtol=1e-13)
    for gi, oi in zip(g.images, o.images):
        np.testing.assert_allclose(gi.m, oi.m, rtol=0, atol=1e-14)
    E = g.calc_E()
    np.testing.assert_allclose(E, o.calc_E(), rtol=1e-11)


def test_string_steps_match_oracle():
    g, o = _setup(5, 5e-14)
    for _ in range(2):
        g.step()
        o.step()
        x, xi = g.x()
        np.testing.assert_allclose(x, o.x, rtol=1e-8)
        np.testing.assert_allclose(xi, o.x_interp, rtol=1e-8)
        for gi, oi in zip(g.images, o.images):
            np.testing.assert_allclose(gi.m, oi.m, rtol=0, atol=1e-8)
            assert abs(gi.t - oi.t) <= 1e-8 * oi.t
    np.testing.assert_allclose(g.calc_E(), o.calc_E(), rtol=1e-8)


def test_run_matches_oracle_and_writes_files(tmp_path):
    g, o = _setup(4, 5e-14, reverse=True)
    out = str(tmp_path) + os.sep
    dE = g.run(out, string_steps=3, verbose=False)
    dE_ref, it_ref, _ = o.run(string_steps=3)
    assert g.iterations == it_ref == 3
    assert dE_ref > 0
    assert abs(dE - dE_ref) <= 1e-7 * abs(dE_ref)
    for f in ("dE_over_iteration.dat", "E_curves.dat", "E_barrier.dat", "E_last_step.dat", "E_max_lowest.dat",
              "plot_string_method.gpi"):
        assert os.path.exists(out + f), f
    rows = [l for l in open(out + "dE_over_iteration.dat") if l.strip() and not l.startswith("#")]
    assert len(rows) == 3


def test_rejects_single_image():
    gm = M.Mesh(*SHAPE, 1e-9, 1e-9, 1e-9)
    a, _ = _images()
    llg = M.LLGIntegrator(1.0, [M.ExchangeField(1e-11)])
    with pytest.raises(RuntimeError):
        M.StringMethod(M.State(gm, MS, a), [a], 3, 1e-13, llg)


@pytest.mark.parametrize("substeps", [1, 4, 5])
def test_batched_string_matches_oracle(substeps):
    """maf_string_set_batched: every image advances its dt with `substeps` fixed
    RK4 steps, all images in one CUDA graph; images, arc lengths and energies
    after two string steps against the oracle's string with the same integration."""
    g, o = _setup(6, 6e-14)
    g.set_batched(substeps)
    o.rk4_substeps = substeps
    for _ in range(2):
        g.step()
        o.step()
    for gi, oi in zip(g.images, o.images):
        assert np.abs(np.asarray(gi.m) - oi.m).max() < 1e-12
        assert gi.t == pytest.approx(oi.t, rel=1e-14)
    x, xi = g.x()
    np.testing.assert_allclose(x, o.x, rtol=1e-11, atol=1e-15)
    np.testing.assert_allclose(g.calc_E(), o.calc_E(), rtol=1e-11)


def test_batched_string_run_and_back_to_reference_mode(tmp_path):
    g, _ = _setup(5, 5e-14, reverse=True)
    g.set_batched(2)
    dE = g.run(str(tmp_path) + os.sep, string_steps=30, verbose=False)
    assert np.isfinite(dE) and dE > 0
    assert os.path.exists(tmp_path / "E_barrier.dat")
    g.set_batched(0)  # the reference's sequential adaptive integration again
    g.step()
    with pytest.raises(M.MafError):
        g.set_batched(-1)
