"""Batched passes of a stochastic ensemble (StochasticBatch(fused=True),
maf_stoch_batch_set_fused): every pass of a step is one launch per transform
length over a device work table of (member, tile) pairs for members of uneven
2-D meshes -- the compile-time kernels' tile bodies where the length has them,
the run-time-plan kernels' for the others.  Each member's trajectory must
equal, bit for bit, the one its own integrator computes with the same kernels,
for odd and even step counts, after a member was stepped alone in between, and
in the FP32-field and FP64 forms and the three schemes."""
import numpy as np
import pytest

from helpers import random_m

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu

SIDES = [(64, 64), (96, 64), (128, 96), (40, 24), (33, 15)]


def _members(prec, scheme, generic, sides=SIDES, T=300.0):
    out = []
    for i, (nx, ny) in enumerate(sides):
        mesh = M.Mesh(nx, ny, 1, 2e-9, 2e-9, 1e-9)
        d = M.DemagField(mesh)
        d.generic = generic
        terms = [d, M.ExchangeField(1.5e-11), M.DmiField(2e-3), M.UniaxialAnisotropyField(6e5),
                 M.ExternalField.uniform(1e4, 0, 2e4)]
        st = M.State(mesh, 7e5, random_m((nx, ny, 1), 60 + i), precision=prec)
        it = M.Stochastic_LLG(0.1, T, 5e-14, st, terms, scheme, seed=11, member=i)
        out.append((it, st, terms))
    return out


@pytest.mark.parametrize("prec,scheme", [("fp32_field", "Heun"), ("fp64", "Heun"), ("fp32_field", "SemiHeun"),
                                         ("fp64", "detRK4")])
def test_fused_batch_matches_members_bitwise(prec, scheme):
    # both sides on the run-time-plan kernels: the batch's eager first step and
    # any odd last step run the members' own passes
    bm = _members(prec, scheme, generic=True)
    sm = _members(prec, scheme, generic=True)
    batch = M.StochasticBatch([(it, st) for it, st, _ in bm], fused=True)
    for n in (5, 4):
        batch.steps(n)
        assert batch.fused_active
        for it, st, _ in sm:
            it.steps(st, n)
        for (itb, stb, _), (its, sts, _) in zip(bm, sm):
            assert np.array_equal(np.asarray(stb.m), np.asarray(sts.m))
            assert stb.t == sts.t and itb.calls == its.calls
    bm[1][0].step(bm[1][1])  # a member alone: the next batch call captures again
    sm[1][0].step(sm[1][1])
    batch.steps(3)
    for it, st, _ in sm:
        it.steps(st, 3)
    for (_, stb, _), (_, sts, _) in zip(bm, sm):
        assert np.array_equal(np.asarray(stb.m), np.asarray(sts.m))


# power-of-two and other sides: each pass mixes compile-time classes (x length
# 64, 128, 32 / y length 128, 256) with members on the run-time-plan kernels
CT_SIDES = [(64, 64), (128, 96), (96, 64), (32, 128), (64, 128), (40, 24)]


@pytest.mark.parametrize("prec,scheme", [("fp32_field", "Heun"), ("fp64", "Heun"), ("fp32_field", "detRK4")])
def test_fused_batch_compile_time_kernels_bitwise(prec, scheme):
    """The default (compile-time) kernels: the batch groups the members by
    transform length and runs the per-state kernels' tile bodies, so every
    member's trajectory equals its own integrator's bit for bit."""
    bm = _members(prec, scheme, generic=False, sides=CT_SIDES)
    sm = _members(prec, scheme, generic=False, sides=CT_SIDES)
    batch = M.StochasticBatch([(it, st) for it, st, _ in bm], fused=True)
    for n in (5, 4):
        batch.steps(n)
        assert batch.fused_active
        for it, st, _ in sm:
            it.steps(st, n)
        for (itb, stb, _), (its, sts, _) in zip(bm, sm):
            assert np.array_equal(np.asarray(stb.m), np.asarray(sts.m))
            assert stb.t == sts.t and itb.calls == its.calls


def test_fused_batch_falls_back_for_3d_members():
    mesh = M.Mesh(16, 16, 2, 2e-9, 2e-9, 2e-9)
    st = M.State(mesh, 8e5, random_m((16, 16, 2), 3))
    it = M.Stochastic_LLG(0.1, 300.0, 5e-14, st, [M.DemagField(mesh), M.ExchangeField(1.3e-11)], "Heun", seed=2)
    batch = M.StochasticBatch([(it, st)], fused=True)
    batch.steps(3)
    assert not batch.fused_active
