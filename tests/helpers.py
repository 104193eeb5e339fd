"""Shared helpers of the parity tests: seeded inputs and error metrics."""
import numpy as np

import maf_oracle as O


def random_m(shape, seed):
    """Uniform random directions, (nx, ny, nz, 3)."""
    rng = np.random.default_rng(seed)
    m = rng.normal(size=tuple(shape) + (3,))
    return m / np.linalg.norm(m, axis=3, keepdims=True)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d


def rel_max(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.abs(b).max()
    return np.abs(a - b).max() / n if n > 0 else np.abs(a - b).max()


def mesh_pair(nx, ny, nz, dx, dy, dz):
    import magnumaf as M
    return M.Mesh(nx, ny, nz, dx, dy, dz), O.Mesh(nx, ny, nz, dx, dy, dz)
