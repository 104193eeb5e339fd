"""maf_llg_heff_pipeline (overlapped host copies) against one maf_state_set_m +
maf_llg_heff(_f32) call per input: bit-identical fields, the state left at the
last input."""
import numpy as np
import pytest

from helpers import random_m

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32_field", "fp64"])
def test_pipeline_equals_single_calls(precision):
    shape = (64, 48, 4)
    mesh = M.Mesh(*shape, 3e-9, 3e-9, 3e-9)
    terms = [M.DemagField(mesh), M.ExchangeField(1.3e-11), M.CubicAnisotropyField(-1e4),
             M.ExternalField.uniform(1e4, -2e4, 3e4)]
    llg = M.LLGIntegrator(0.01, terms, "DP45")
    ms = [random_m(shape, 50 + i) for i in range(5)]
    s = M.State(mesh, 8.6e5, ms[0], precision=precision)
    f32 = precision == "fp32_field"
    ref = []
    for m in ms:
        s.m = m
        ref.append(llg.H_in_Apm_f32(s) if f32 else llg.H_in_Apm(s))
    # inputs/outputs in the library's [3][nz][ny][nx] layout (Fortran order of (nx,ny,nz,3))
    ins = [np.asfortranarray(m).ravel(order="F").copy() for m in ms]
    outs = [np.empty(3 * np.prod(shape), dtype=np.float32 if f32 else np.float64) for _ in ms]
    llg.heff_pipeline(s, [a.ctypes.data for a in ins], [o.ctypes.data for o in outs])
    for o, r in zip(outs, ref):
        assert np.array_equal(o, np.asarray(r).ravel(order="F"))
    np.testing.assert_array_equal(np.asarray(s.m), np.asarray(M.State(mesh, 8.6e5, ms[-1]).m))


@pytest.mark.parametrize("precision", ["fp32_field", "fp64"])
def test_pipeline_with_float32_inputs(precision):
    """maf_llg_heff_pipeline_m32: FP32 host magnetisations give exactly the fields
    of the same values passed in FP64 (the widening is exact)."""
    shape = (32, 24, 4)
    mesh = M.Mesh(*shape, 3e-9, 3e-9, 3e-9)
    llg = M.LLGIntegrator(0.01, [M.DemagField(mesh), M.ExchangeField(1.3e-11)], "DP45")
    ms = [random_m(shape, 60 + i).astype(np.float32) for i in range(3)]
    s = M.State(mesh, 8.6e5, ms[0], precision=precision)
    f32 = precision == "fp32_field"
    ins32 = [np.asfortranarray(m).ravel(order="F").copy() for m in ms]
    ins64 = [a.astype(np.float64) for a in ins32]
    out_t = np.float32 if f32 else np.float64
    outs32 = [np.empty(3 * np.prod(shape), dtype=out_t) for _ in ms]
    outs64 = [np.empty(3 * np.prod(shape), dtype=out_t) for _ in ms]
    llg.heff_pipeline(s, [a.ctypes.data for a in ins32], [o.ctypes.data for o in outs32], m_float32=True)
    llg.heff_pipeline(s, [a.ctypes.data for a in ins64], [o.ctypes.data for o in outs64])
    for a, b in zip(outs32, outs64):
        assert np.array_equal(a, b)
