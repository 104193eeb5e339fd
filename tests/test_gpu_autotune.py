"""Kernel-variant autotuner (maf_llg_autotune, DemagField.tune): every variant
computes the same field as the defaults up to rounding, and the autotuner
returns valid choices and keeps them in the DemagField."""
import numpy as np
import pytest

from helpers import random_m, rel_l2

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [("fp32_field", 2e-6), ("fp64", 1e-13)])
@pytest.mark.parametrize("shape", [(64, 32, 8), (32, 32, 16), (64, 64, 1)])
def test_variants_agree_and_autotune_picks_valid(precision, tol, shape):
    mesh = M.Mesh(*shape, 3e-9, 3e-9, 3e-9)
    d = M.DemagField(mesh)
    llg = M.LLGIntegrator(0.01, [d, M.ExchangeField(1.3e-11), M.CubicAnisotropyField(-1e4)])
    s = M.State(mesh, 8.6e5, random_m(shape, 3), precision=precision)
    f32 = precision == "fp32_field"
    field = (lambda: llg.H_in_Apm_f32(s)) if f32 else (lambda: llg.H_in_Apm(s))
    assert d.tune == (0, 1, 0)
    H0 = np.asarray(field(), dtype=np.float64)
    for choice in [(1, 1, 2), (0, 0, 4), (1, 0, 2)]:
        d.tune = choice
        H = np.asarray(field(), dtype=np.float64)
        assert rel_l2(H, H0) <= tol, (choice, rel_l2(H, H0))
    res = llg.autotune(s, reps=2)
    assert res["cols_wide"] in (0, 1) and res["convz_reg"] in (0, 1) and res["xinv_run"] in (2, 4)
    assert d.tune == (res["cols_wide"], res["convz_reg"], res["xinv_run"])
    assert rel_l2(np.asarray(field(), dtype=np.float64), H0) <= tol
    with pytest.raises(M.MafError):
        d.tune = (2, 1, 2)


@pytest.mark.parametrize("shape", [(64, 256, 4), (32, 1024, 2)])
def test_full_search_variants_agree_and_cache(shape):
    """Every radix sequence (both y passes, or only one of them) / pipelining / tile
    choice gives the field of the defaults to rounding, and the full search is
    cached per shape."""
    mesh = M.Mesh(*shape, 3e-9, 3e-9, 3e-9)
    d = M.DemagField(mesh)
    llg = M.LLGIntegrator(0.01, [d, M.ExchangeField(1.3e-11)])
    s = M.State(mesh, 8.6e5, random_m(shape, 4), precision="fp32_field")
    H0 = np.asarray(llg.H_in_Apm_f32(s), dtype=np.float64)
    for choice in [(0, 1, 2, 1, 1), (1, 1, 2, 0, 1), (0, 0, 4, 0, 0), (1, 0, 2, 1, 1), (0, 1, 2, 1, 2), (1, 0, 4, 0, 3)]:
        d.tune_ex = choice
        assert d.tune_ex == choice
        H = np.asarray(llg.H_in_Apm_f32(s), dtype=np.float64)
        assert rel_l2(H, H0) <= 2e-6, (choice, rel_l2(H, H0))
    res = llg.autotune_ex(s, reps=2)
    assert not res["cached"]
    assert d.tune_ex == tuple(res[k] for k in ("cols_wide", "convz_reg", "xinv_run", "cols_pipe", "cols_plan"))
    d2 = M.DemagField(mesh)
    llg2 = M.LLGIntegrator(0.01, [d2, M.ExchangeField(1.3e-11)])
    res2 = llg2.autotune_ex(s, reps=2)
    assert res2["cached"] and d2.tune_ex == d.tune_ex
    with pytest.raises(M.MafError):
        d.tune_ex = (0, 1, 2, 1, 4)  # cols_plan is 0..3
