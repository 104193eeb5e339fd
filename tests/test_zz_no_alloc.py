"""maf_mean_m_noalloc (static device scratch, no allocation) against
maf_state_mean_m on the same device field.  The file name sorts last so the
test also runs after every other GPU test in one session."""
import ctypes as C

import numpy as np
import pytest

from helpers import random_m

M = pytest.importorskip("magnumaf")

pytestmark = pytest.mark.gpu

MAX_CELLS = 1 << 25


def _noalloc_mean(state, ncells):
    p = state.device_m()
    out = np.zeros(3)
    rc = M.lib.maf_mean_m_noalloc(C.c_void_p(p), ncells, out.ctypes.data_as(C.POINTER(C.c_double)), None)
    return rc, out


@pytest.mark.parametrize("shape", [(1, 1, 1), (64, 48, 5), (256, 256, 8)])
def test_noalloc_mean_matches_state_mean(shape):
    mesh = M.Mesh(*shape, 2e-9, 2e-9, 2e-9)
    m0 = random_m(shape, 7)
    ms = np.full(shape, 8e5)
    if m0[..., 0].size > 1:  # empty cells: Ms = 0 and m = 0, left out of the count
        ms.reshape(-1)[::5] = 0.0
        m0.reshape(-1, 3)[::5] = 0.0
    s = M.State(mesh, ms, m0)
    ref = s.mean_m()
    assert np.all(np.isfinite(ref))
    n = int(np.prod(shape))
    for _ in range(2):
        rc, got = _noalloc_mean(s, n)
        assert rc == 0, M.lib.maf_last_error()
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-15)


def test_noalloc_rejects_oversized_and_bad_arguments():
    shape = (8, 8, 1)
    s = M.State(M.Mesh(*shape, 1e-9, 1e-9, 1e-9), 8e5, random_m(shape, 3))
    rc, _ = _noalloc_mean(s, MAX_CELLS + 1)
    assert rc == 1 and b"scratch limit" in M.lib.maf_last_error()
    rc, _ = _noalloc_mean(s, 0)
    assert rc == 1
    out = np.zeros(3)
    assert M.lib.maf_mean_m_noalloc(None, 64, out.ctypes.data_as(C.POINTER(C.c_double)), None) == 1
    # a rejected call leaves nothing behind: the next one is still correct
    rc, got = _noalloc_mean(s, 64)
    assert rc == 0
    np.testing.assert_allclose(got, s.mean_m(), rtol=1e-12, atol=1e-15)
