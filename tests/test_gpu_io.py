"""Checkpoint/resume through magnumaf.io with the step-size controller state:
a run resumed from a checkpoint takes the same steps as the uninterrupted run;
State.write_vti / read_vti round-trip the device magnetisation."""
import numpy as np
import pytest

from helpers import random_m

M = pytest.importorskip("magnumaf")
from magnumaf import io  # noqa: E402

pytestmark = pytest.mark.gpu

SHAPE = (24, 16, 2)


def _setup():
    mesh = M.Mesh(*SHAPE, 2e-9, 2e-9, 2e-9)
    terms = [M.DemagField(mesh), M.ExchangeField(1.3e-11), M.DmiField(3e-3), M.UniaxialAnisotropyField(5e5)]
    return mesh, terms


def test_resume_takes_the_same_steps(tmp_path):
    mesh, terms = _setup()
    m0 = random_m(SHAPE, 21)
    s = M.State(mesh, 8e5, m0)
    llg = M.LLGIntegrator(0.5, terms, "DP45")
    llg.steps(s, 15)
    ck = str(tmp_path / "ck.npz")
    io.save_checkpoint(ck, s, llg)
    llg.steps(s, 15)
    # a fresh state and integrator resumed from the checkpoint
    s2 = M.State(mesh, 8e5, m0)
    llg2 = M.LLGIntegrator(0.5, terms, "DP45")
    io.load_checkpoint(ck, s2, llg2)
    assert s2.steps == 15
    llg2.steps(s2, 15)
    assert np.array_equal(np.asarray(s.m), np.asarray(s2.m))
    assert s.t == s2.t and s.steps == s2.steps == 30
    assert llg.controller_state() == llg2.controller_state()


def test_state_vti_roundtrip(tmp_path):
    mesh, _ = _setup()
    s = M.State(mesh, 8e5, random_m(SHAPE, 22))
    fn = s.write_vti(str(tmp_path / "m"))
    s2 = M.State(mesh, 8e5, random_m(SHAPE, 23))
    s2.read_vti(fn)
    assert np.array_equal(np.asarray(s.m), np.asarray(s2.m))
