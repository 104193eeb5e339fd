"""maf_mean_m_noalloc (static device scratch, no allocation) against the mean
taken in NumPy from the state's host copy of m and against maf_state_mean_m on
the same device field, and a check that the call allocates no device memory.
The file name sorts last so the test also runs after every other GPU test in
one session; it also passes alone in a fresh process, where creating the first
state is what loads the entry point's module."""
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


def _numpy_mean(m):
    """<m> by the definition of maf_state_mean_m: sum / number of cells with |m| != 0."""
    flat = np.asarray(m, dtype=np.float64).reshape(-1, 3)
    n = np.count_nonzero(np.linalg.norm(flat, axis=1))
    return flat.sum(axis=0) / n


@pytest.mark.parametrize("shape", [(1, 1, 1), (64, 48, 5), (256, 256, 8)])
def test_noalloc_mean_matches_numpy_and_state_mean(shape):
    mesh = M.Mesh(*shape, 2e-9, 2e-9, 2e-9)
    m0 = random_m(shape, 7)
    ms = np.full(shape, 8e5)
    if m0[..., 0].size > 1:  # empty cells: Ms = 0 and m = 0, left out of the count
        ms.reshape(-1)[::5] = 0.0
        m0.reshape(-1, 3)[::5] = 0.0
    s = M.State(mesh, ms, m0)
    ref_np = _numpy_mean(s.m)
    ref = s.mean_m()  # also synchronises the state's stream before the field is read
    assert np.all(np.isfinite(ref))
    n = int(np.prod(shape))
    for _ in range(2):
        rc, got = _noalloc_mean(s, n)
        assert rc == 0, M.lib.maf_last_error()
        np.testing.assert_allclose(got, ref_np, rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-15)


def test_noalloc_mean_allocates_nothing_at_the_limit():
    """At the largest size the scratch allows (2^25 cells), device free memory
    is the same before and after repeated calls."""
    torch = pytest.importorskip("torch")
    shape = (1024, 1024, 32)
    assert int(np.prod(shape)) == MAX_CELLS
    rng = np.random.default_rng(5)
    m0 = np.zeros(shape + (3,))
    m0[..., 2] = 1.0
    m0[..., 0] = rng.uniform(-0.5, 0.5, size=shape)
    s = M.State(M.Mesh(*shape, 1e-9, 1e-9, 1e-9), 8e5, m0)
    ref_np = _numpy_mean(s.m)
    s.mean_m()
    torch.cuda.mem_get_info(0)  # initialises torch's view of the device first
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        rc, got = _noalloc_mean(s, MAX_CELLS)
        assert rc == 0, M.lib.maf_last_error()
        np.testing.assert_allclose(got, ref_np, rtol=1e-12, atol=1e-15)
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)


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
    np.testing.assert_allclose(got, _numpy_mean(s.m), rtol=1e-12, atol=1e-15)
