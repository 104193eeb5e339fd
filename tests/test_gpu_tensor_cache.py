"""Demag-tensor disk cache (DemagField(mesh, caching=True)): the first
construction writes the reduced spectral tensor, the next reads it and gives the
same field bit for bit; a damaged file is ignored and rewritten."""
import os

import numpy as np
import pytest

from helpers import random_m

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu


def test_cache_roundtrip_and_recovery(tmp_path, monkeypatch):
    monkeypatch.setenv("MAGNUMAF_CACHE", str(tmp_path))
    mesh = M.Mesh(24, 20, 6, 2e-9, 3e-9, 4e-9)
    s = M.State(mesh, 8e5, random_m((24, 20, 6), 1))
    ref = M.DemagField(mesh).H_in_Apm(s)
    d1 = M.DemagField(mesh, caching=True)  # computes and writes
    files = [f for f in os.listdir(tmp_path) if f.endswith(".npy")]
    assert len(files) == 1
    d2 = M.DemagField(mesh, caching=True)  # reads
    assert np.array_equal(d1.H_in_Apm(s), ref) and np.array_equal(d2.H_in_Apm(s), ref)
    assert np.array_equal(d2.spectral_tensor(), d1.spectral_tensor())
    with open(os.path.join(tmp_path, files[0]), "wb") as f:
        f.write(b"not a tensor")
    d3 = M.DemagField(mesh, caching=True)  # damaged: recomputed and rewritten
    assert np.array_equal(d3.H_in_Apm(s), ref)
    assert np.load(os.path.join(tmp_path, files[0])).shape == d1.spectral_tensor().shape
