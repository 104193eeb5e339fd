"""Compile-time passes for transform lengths of three times a power of two
(96 .. 1536: radix plans 16-3-2 .. 16-3-16-2 with a radix-3 stage) against the
FP64 oracle (magnumaf/src/field_terms/micro/demag_field.cpp:215-264 and the
local terms), with the device's own tensor fed to the oracle.  The meshes put
each new length into each pass: the x passes (complex length nx), the 3-D y
passes and the 2-D y convolution (length 2 ny); every kernel variant of the
autotuner runs.  Tolerances: 1e-12 relative (L2 and max norm) for the FP64 form,
1e-5 for the FP32-field form."""
import numpy as np
import pytest

import maf_oracle as O
from helpers import random_m, rel_l2, rel_max

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu

MS = 8.6e5
HEXT = (0.011 / O.mu0, -0.027 / O.mu0, 0.019 / O.mu0)

MESHES = [
    (96, 48, 1),    # x 96, y convolution 96
    (192, 96, 2),   # x 192, y passes 192
    (384, 24, 4),   # x 384
    (768, 12, 1),   # x 768
    (1536, 4, 1),   # x 1536
    (16, 384, 2),   # y passes 768
    (32, 192, 1),   # y convolution 384
    (8, 768, 1),    # y convolution 1536
    (8, 768, 2),    # y passes 1536
]

VARIANTS = [(0, 1, 2, 1, 0), (1, 0, 4, 0, 0), (0, 1, 4, 0, 0), (1, 1, 2, 1, 0)]


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


@pytest.mark.parametrize("shape", MESHES)
def test_heff_three_times_power_of_two_vs_oracle(shape):
    gm, m, d, gterms, ref = _case(shape, seed=31)
    llg = M.LLGIntegrator(0.01, gterms, "DP45")
    s64 = M.State(gm, MS, m)
    s32 = M.State(gm, MS, m, precision="fp32_field")
    for tune in VARIANTS:
        d.tune_ex = tune
        h64 = llg.H_in_Apm(s64)
        assert rel_l2(h64, ref) < 1e-12 and rel_max(h64, ref) < 1e-12, (tune, rel_l2(h64, ref), rel_max(h64, ref))
        h32 = llg.H_in_Apm_f32(s32)
        assert rel_l2(h32, ref) < 1e-5 and rel_max(h32, ref) < 1e-5, (tune, rel_l2(h32, ref), rel_max(h32, ref))


@pytest.mark.parametrize("shape", [(96, 48, 1), (192, 96, 2)])
def test_compile_time_and_generic_kernels_agree(shape):
    """The same field from the compile-time kernels and the run-time-plan ones
    (which ran these lengths before): FP64 to 1e-13."""
    gm = M.Mesh(*shape, 3e-9, 3e-9, 3e-9)
    m = random_m(shape, 32)
    d = M.DemagField(gm)
    llg = M.LLGIntegrator(0.01, [d, M.ExchangeField(1.3e-11)], "DP45")
    s = M.State(gm, MS, m)
    h_ct = np.asarray(llg.H_in_Apm(s))
    d.generic = True
    h_gen = np.asarray(llg.H_in_Apm(s))
    assert rel_l2(h_ct, h_gen) < 1e-13
