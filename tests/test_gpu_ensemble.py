"""Stochastic Heun ensemble members through magnumaf.ensemble: a member's
trajectory depends only on (seed, member), not on which members ran before it
on the same GPU, so the static assignment may place it on any rank."""
import numpy as np
import pytest

from helpers import random_m

M = pytest.importorskip("magnumaf")
from magnumaf import ensemble  # noqa: E402

pytestmark = pytest.mark.gpu


def _member(spec):
    nx, ny, steps, member = spec
    mesh = M.Mesh(nx, ny, 1, 2e-9, 2e-9, 2e-9)
    state = M.State(mesh, 8e5, random_m((nx, ny, 1), 100 + member), precision="fp32_field")
    terms = [M.ExchangeField(1.3e-11), M.UniaxialAnisotropyField(5e5)]
    st = M.Stochastic_LLG(0.1, 300.0, 1e-14, state, terms, "Heun", seed=11, member=member)
    st.steps(state, steps)
    return np.asarray(state.m)


def test_members_are_independent_of_order():
    specs = [(16, 16, 20, 0), (32, 16, 15, 1), (24, 24, 10, 2)]
    costs = [ensemble.member_cost(s[0], s[1], 1, s[2]) for s in specs]
    forward = ensemble.run_sharded(specs, costs, _member)
    backward = ensemble.run_sharded(specs[::-1], costs[::-1], _member)[::-1]
    for a, b in zip(forward, backward):
        assert np.array_equal(a, b)
    alone = _member(specs[1])
    assert np.array_equal(alone, forward[1])
