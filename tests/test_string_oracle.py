"""The string-method oracle (magnumaf/src/solvers/string_method.cpp) on the
CPU: initial interpolation in closed form, the reference's copy branch, and
re-interpolation to equal arc lengths."""
import numpy as np
import pytest

import maf_oracle as O
import maf_string_oracle as SO


def _disk(n, r):
    m = np.zeros((n, n, 1, 3))
    m[..., 2] = 1.0
    c = (n - 1) / 2.0
    for i in range(n):
        for j in range(n):
            if (i - c) ** 2 + (j - c) ** 2 <= r * r:
                m[i, j, 0, 2] = -1.0
    m[..., 0] += 0.05  # no exactly antiparallel pairs: the interpolation passes no zero vector
    return O.normalize(m)


def _setup(n_interp, inputs):
    mesh = O.Mesh(8, 8, 1, 1e-9, 1e-9, 1e-9)
    state = O.State(mesh, 8e5, inputs[0])
    llg = O.LLGIntegrator(1.0, [O.ExchangeField(1.5e-11)])
    return mesh, state, llg


def test_initial_images_follow_the_straight_path():
    a = _disk(8, 2.5)
    b = O.normalize(np.tile([0.05, 0.0, 1.0], (8, 8, 1, 1)))
    _, state, llg = _setup(5, [a, b])
    sm = SO.StringMethod(state, [a, b], 5, 1e-13, llg)
    X = O.FrobeniusNorm(b - a)
    assert sm.x == pytest.approx([0.0, X], rel=1e-15)
    for i, img in enumerate(sm.images):
        f = i / 4.0
        np.testing.assert_allclose(img.m, O.normalize(a + f * (b - a)), rtol=0, atol=1e-14)
    np.testing.assert_allclose(sm.images[0].m, a, atol=1e-15)
    np.testing.assert_allclose(sm.images[-1].m, b, atol=1e-15)


def test_copy_branch_when_bracket_reaches_the_last_interpolation_index():
    """With more input images than n_interp the bracket index can reach
    n_interp - 1; the reference then copies input image j (string_method.cpp:37-41)."""
    rng = np.random.default_rng(3)
    ins = [O.normalize(rng.normal(size=(8, 8, 1, 3))) for _ in range(4)]
    _, state, llg = _setup(2, ins)
    sm = SO.StringMethod(state, ins, 2, 1e-13, llg)
    # x_interp = [0, X]: the search stops at j = n_interp = 2 and steps back to
    # j = 1 = n_interp - 1, so image 1 is a copy of input image 1
    assert sm._bracket(1) == 1
    np.testing.assert_allclose(sm.images[0].m, ins[0], atol=1e-15)
    np.testing.assert_allclose(sm.images[1].m, ins[1], atol=1e-15)


def test_reinterpolation_equalises_arc_lengths_of_a_straight_string():
    """Images on a straight line (no normalisation effect: all cells rotate in a
    plane by small angles) are redistributed to nearly equal spacing."""
    n = 6
    base = np.zeros((8, 8, 1, 3))
    base[..., 2] = 1.0
    angles = [0.0, 0.02, 0.03, 0.09, 0.1, 0.2]
    ms = [np.concatenate([np.full((8, 8, 1, 1), np.sin(t)), np.zeros((8, 8, 1, 1)),
                          np.full((8, 8, 1, 1), np.cos(t))], axis=3) for t in angles]
    _, state, llg = _setup(n, ms)
    sm = SO.StringMethod(state, ms, n, 1e-13, llg)
    sm._calc_x([img.m for img in sm.images])
    d = np.diff(sm.x)
    assert np.max(np.abs(d - d.mean())) < 1e-3 * d.mean()
