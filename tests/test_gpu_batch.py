"""Batched stochastic ensemble (maf_stoch_batch_*): members of uneven meshes
advanced through one captured CUDA graph match the same members stepped one by
one, bit for bit, for odd and even step counts and after a member was stepped
on its own in between (the graph is then captured again)."""
import numpy as np
import pytest

from helpers import random_m

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu

SPECS = [  # (nx, ny, nz, precision, scheme, demag)
    (16, 16, 1, "fp32_field", "Heun", True),
    (24, 16, 1, "fp64", "Heun", False),
    (32, 32, 2, "fp32_field", "SemiHeun", False),
]


def _member(i, spec):
    nx, ny, nz, prec, scheme, demag = spec
    mesh = M.Mesh(nx, ny, nz, 2e-9, 2e-9, 2e-9)
    terms = [M.ExchangeField(1.3e-11), M.UniaxialAnisotropyField(4e5)]
    if demag:
        terms = [M.DemagField(mesh)] + terms
    st = M.State(mesh, 8e5, random_m((nx, ny, nz), 30 + i), precision=prec)
    it = M.Stochastic_LLG(0.2, 300.0, 2e-14, st, terms, scheme, seed=5, member=i)
    return it, st, terms


def _assert_same(batch_members, serial_members):
    for (it_b, st_b, _), (it_s, st_s, _) in zip(batch_members, serial_members):
        assert np.array_equal(np.asarray(st_b.m), np.asarray(st_s.m))
        assert st_b.t == st_s.t
        assert it_b.calls == it_s.calls


def test_batch_matches_serial_bitwise():
    bm = [_member(i, s) for i, s in enumerate(SPECS)]
    sm = [_member(i, s) for i, s in enumerate(SPECS)]
    batch = M.StochasticBatch([(it, st) for it, st, _ in bm])
    for n in (5, 4, 3):
        batch.steps(n)
        for it, st, _ in sm:
            it.steps(st, n)
        _assert_same(bm, sm)
    # a member stepped on its own between batch calls: the graph is captured again
    bm[0][0].step(bm[0][1])
    sm[0][0].step(sm[0][1])
    batch.steps(4)
    for it, st, _ in sm:
        it.steps(st, 4)
    _assert_same(bm, sm)


def test_batch_rejects_shared_state():
    it, st, _ = _member(0, SPECS[0])
    it2, _, _ = _member(1, SPECS[0])
    with pytest.raises(M.MafError):
        M.StochasticBatch([(it, st), (it2, st)])


def test_batch_rejects_a_shared_demag_plan():
    """Members run concurrently, so one DemagField (one set of spectral buffers)
    cannot serve two of them."""
    mesh = M.Mesh(16, 16, 1, 2e-9, 2e-9, 2e-9)
    d = M.DemagField(mesh)
    members = []
    for i in range(2):
        st = M.State(mesh, 8e5, random_m((16, 16, 1), 40 + i))
        members.append((M.Stochastic_LLG(0.2, 300.0, 2e-14, st, [d, M.ExchangeField(1.3e-11)], seed=5, member=i),
                        st))
    with pytest.raises(M.MafError):
        M.StochasticBatch(members)
