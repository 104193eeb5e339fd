"""Parity of the kernels the benchmark runs, at sizes that instantiate them.

The throughput figure at 1024 x 1024 x 16 comes from compile-time kernels whose
template arguments depend on the transform lengths: the x passes of a 1024-cell
row (complex length 1024), the y passes of a 2048-point padded column and the
register-resident z convolution of a 16-layer mesh.  Smaller test meshes run
other instantiations, so these meshes are checked here against the FP64 oracle
(magnumaf/src/field_terms/micro/demag_field.cpp:215-264 and the local terms of
the metric's term set):

* 1024 x 1024 x 2 -- x length 1024, y length 2048 (every x/y kernel of the
  benchmark mesh, in both precisions and in every autotuner variant);
* 256 x 256 x 16 -- the z convolution of 16 layers (k_convz_reg<.,16,.>) and the
  shared-memory z variant.

The oracle gets the device's own tensor (parity on identical inputs; see
test_gpu_fields.py for why independently assembled tensors differ at the Newell
sums' rounding noise).  Tolerances: 1e-12 relative (L2 and max norm) for the
FP64 form, 1e-5 for the FP32-field form.
"""
import os

import numpy as np
import pytest

import maf_oracle as O
from helpers import random_m, rel_l2, rel_max

M = pytest.importorskip("magnumaf")

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

MS = 8.6e5
HEXT = (0.011 / O.mu0, -0.027 / O.mu0, 0.019 / O.mu0)


@pytest.fixture(autouse=True)
def _threaded_oracle():
    """The oracle's FFTs on all host cores (scipy.fft workers) for these sizes."""
    old = O.FFT_WORKERS
    O.FFT_WORKERS = os.cpu_count() or 1
    yield
    O.FFT_WORKERS = old


def _case(shape, seed):
    gm = M.Mesh(*shape, 3e-9, 3e-9, 3e-9)
    om = O.Mesh(*shape, 3e-9, 3e-9, 3e-9)
    m = random_m(shape, seed)
    d = M.DemagField(gm)
    gterms = [d, M.ExchangeField(1.3e-11), M.CubicAnisotropyField(-1e4), M.ExternalField.uniform(*HEXT)]
    od = O.DemagField(om, N_real=d.get_N(symmetric=True))
    oterms = [od, O.ExchangeField(1.3e-11), O.CubicAnisotropyField(-1e4), O.ExternalField(np.array(HEXT))]
    ref = O.Heff_in_Apm(oterms, O.State(om, MS, m))
    return gm, m, d, gterms, ref


# (cols_wide, convz_reg, xinv_run, cols_pipe, cols_plan): the defaults first, then
# every alternative of each pass
VARIANTS = [(0, 1, 2, 1, 0), (1, 1, 2, 1, 0), (0, 0, 4, 1, 0), (1, 0, 4, 0, 1), (0, 1, 2, 0, 1), (0, 1, 2, 1, 1),
            (0, 1, 2, 1, 2), (0, 1, 2, 0, 3)]


@pytest.mark.parametrize("shape", [(1024, 1024, 2), (256, 256, 16)])
def test_heff_headline_sizes_vs_oracle(shape):
    gm, m, d, gterms, ref = _case(shape, seed=21)
    llg = M.LLGIntegrator(0.01, gterms, "DP45")
    s64 = M.State(gm, MS, m)
    s32 = M.State(gm, MS, m, precision="fp32_field")
    for tune in VARIANTS:
        d.tune_ex = tune
        h64 = llg.H_in_Apm(s64)
        assert rel_l2(h64, ref) < 1e-12 and rel_max(h64, ref) < 1e-12, (tune, rel_l2(h64, ref), rel_max(h64, ref))
        h32 = llg.H_in_Apm_f32(s32)
        assert rel_l2(h32, ref) < 1e-5 and rel_max(h32, ref) < 1e-5, (tune, rel_l2(h32, ref), rel_max(h32, ref))


def test_demag_alone_headline_x_y_lengths():
    """The demag term by itself at 1024 x 1024 x 2 (no local terms to mask an
    error in the convolution), FP64 and FP32-field forms."""
    shape = (1024, 1024, 2)
    gm = M.Mesh(*shape, 3e-9, 3e-9, 3e-9)
    om = O.Mesh(*shape, 3e-9, 3e-9, 3e-9)
    m = random_m(shape, 22)
    d = M.DemagField(gm)
    ref = O.DemagField(om, N_real=d.get_N(symmetric=True)).H_in_Apm(O.State(om, MS, m))
    h64 = d.H_in_Apm(M.State(gm, MS, m))
    assert rel_l2(h64, ref) < 1e-12 and rel_max(h64, ref) < 1e-12
    h32 = d.H_in_Apm_f32(M.State(gm, MS, m, precision="fp32_field"))
    assert rel_l2(h32, ref) < 1e-5 and rel_max(h32, ref) < 1e-5
