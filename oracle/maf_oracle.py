"""CPU FP64 oracle for the magnum.af effective-field / time-step path.

TEST INFRASTRUCTURE ONLY.  This module is the checker that the CUDA product is
compared against; it is imported by ``tests/``, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` and by
nothing else.  The product path (``magnum.af_b200``) never calls it.

It is a plain NumPy restatement of the reference algorithm, written from the
reference sources (paths relative to the magnum.af project root).  Arrays use
the reference's ArrayFire index order: a vector field is ``m[x, y, z, c]`` with
shape ``(nx, ny, nz, 3)``; a scalar field is ``(nx, ny, nz)``.  In memory a
Fortran-ordered ``(nx, ny, nz, 3)`` array is the same bytes as the C-ABI's
structure-of-arrays ``[3][nz][ny][nx]`` layout (see ``to_soa`` / ``from_soa``).

The reference's ArrayFire dependency (FFT/convolve/reductions, version not
pinned by the project) is replaced by ``numpy.fft`` and explicit stencils.
Parity is pinned by the reference's own known-answer tests (see
``tests/test_oracle_golden.py``): the muMAG standard problem 4 time integrals
(python/test/sp4.py:34-36,60-62), the homogeneous-cube demag energy
(magnumaf/test/micro_demag.cpp:6-55), Newell tensor closed forms, cubic and
uniaxial anisotropy values, the Zeeman identity, the bulk-DMI interior zero,
the analytic ODE for the adaptive Runge-Kutta schemes and the central
difference sign.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

# ---------------------------------------------------------------------------
# constants  (magnumaf/include/magnumaf/constants.hpp:9-20)
# ---------------------------------------------------------------------------
mu0 = 4e-7 * math.pi
gamma = 1.760859644e11 * mu0
kb = 1.38064852e-23
mu_b = 9.274009994e-24
e_abs = 1.6021766208e-19
hbar = 1.0545718e-34
e_neg = -1.6021766208e-19


def to_soa(a: np.ndarray) -> np.ndarray:
    """(nx,ny,nz,3) -> C-contiguous [3][nz][ny][nx] (the device layout)."""
    if a.ndim == 3:
        return np.ascontiguousarray(a.transpose(2, 1, 0))
    return np.ascontiguousarray(a.transpose(3, 2, 1, 0))


def from_soa(a: np.ndarray) -> np.ndarray:
    """C-contiguous [3][nz][ny][nx] -> (nx,ny,nz,3) view."""
    if a.ndim == 3:
        return a.transpose(2, 1, 0)
    return a.transpose(3, 2, 1, 0)


# ---------------------------------------------------------------------------
# Mesh / State   (magnumaf/include/magnumaf/mesh.hpp:11-20, state.hpp:11-78,
#                 magnumaf/src/state.cpp:39-111)
# ---------------------------------------------------------------------------
@dataclass
class Mesh:
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float

    @property
    def dims_v(self):
        return (self.nx, self.ny, self.nz, 3)

    @property
    def dims_s(self):
        return (self.nx, self.ny, self.nz)


def vecnorm(a):
    """magnumaf/src/util/util.cpp:44"""
    return np.sqrt(np.sum(a * a, axis=3))


def normalize_even_zero_vectors(a):
    """magnumaf/src/util/util.cpp:34 (0/0 -> NaN kept, like the reference)."""
    with np.errstate(invalid="ignore", divide="ignore"):
        return a / np.sqrt(np.sum(a * a, axis=3))[..., None]


def normalize(a):
    """normalize_handle_zero_vectors, magnumaf/src/util/util.cpp:37-42."""
    n = vecnorm(a)[..., None]
    with np.errstate(invalid="ignore", divide="ignore"):
        out = a / n
    return np.where(n != 0, out, 0.0)


class State:
    """State(Mesh, Ms or Ms_field, m): m normalised on construction
    (magnumaf/src/state.cpp:91-94); an Ms_field is created when some |m| == 0
    (state.cpp:71-89)."""

    def __init__(self, mesh: Mesh, Ms, m, t: float = 0.0):
        self.mesh = mesh
        self.m = normalize(np.array(m, dtype=np.float64))
        self.t = t
        self.steps = 0
        if np.ndim(Ms) == 0:
            self.Ms = float(Ms)
            self.Ms_field = None
            if vecnorm(self.m).min() == 0:
                nzero = vecnorm(self.m) != 0
                self.Ms_field = self.Ms * nzero.astype(np.float64)
        else:
            self.Ms = float("nan")
            Ms = np.asarray(Ms, dtype=np.float64)
            if Ms.ndim == 4:
                Ms = Ms[..., 0]
            self.Ms_field = Ms

    def copy(self):
        s = State.__new__(State)
        s.mesh, s.m, s.t, s.steps = self.mesh, self.m.copy(), self.t, self.steps
        s.Ms, s.Ms_field = self.Ms, self.Ms_field
        return s

    def Ms_v(self):
        """Ms as a (nx,ny,nz,1) broadcastable array or scalar."""
        if self.Ms_field is None:
            return self.Ms
        return self.Ms_field[..., None]

    def mean_m(self):
        """state.cpp:32-43: sum over cells / number of cells with |m| != 0."""
        n = np.count_nonzero(vecnorm(self.m) != 0)
        return np.sum(self.m, axis=(0, 1, 2)) / n


def _replace_ms_zero(h, state):
    """af::replace(h, Ms_field != 0, 0): zero where Ms_field == 0."""
    if state.Ms_field is None:
        return h
    return np.where(state.Ms_field[..., None] != 0, h, 0.0)


def _inv_Ms(state):
    if state.Ms_field is None:
        return 1.0 / state.Ms
    with np.errstate(divide="ignore"):
        return 1.0 / state.Ms_field[..., None]


# ---------------------------------------------------------------------------
# energies  (micro_term.hpp:18-30, external_field.cpp:40-48)
# ---------------------------------------------------------------------------
def micro_energy(state, h, factor=-mu0 / 2.0):
    dV = state.mesh.dx * state.mesh.dy * state.mesh.dz
    if state.Ms_field is None:
        return factor * state.Ms * float(np.sum(h * state.m)) * dV
    return factor * float(np.sum(state.Ms_field[..., None] * h * state.m)) * dV


class FieldTerm:
    def H_in_Apm(self, state) -> np.ndarray:
        raise NotImplementedError

    def Energy_in_J(self, state, h=None) -> float:
        if h is None:
            h = self.H_in_Apm(state)
        return micro_energy(state, h)


# ---------------------------------------------------------------------------
# Newell demag tensor (magnumaf/src/field_terms/micro/demag_field.cpp:14-121)
# ---------------------------------------------------------------------------
def nx_exp(n):
    return 2 * n


def nz_exp(n):
    return 1 if n == 1 else 2 * n


def newell_f(x, y, z):
    """demag_field.cpp:20-40 (vectorised, same term order)."""
    x = np.abs(x)
    y = np.abs(y)
    z = np.abs(z)
    R = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    xx, yy, zz = x ** 2, y ** 2, z ** 2
    result = 1.0 / 6.0 * (2.0 * xx - yy - zz) * R
    with np.errstate(all="ignore"):
        t = y / 2.0 * (zz - xx) * np.arcsinh(y / np.sqrt(xx + zz))
        result = result + np.where(xx + zz > 0, t, 0.0)
        t = z / 2.0 * (yy - xx) * np.arcsinh(z / np.sqrt(xx + yy))
        result = result + np.where(xx + yy > 0, t, 0.0)
        t = -x * y * z * np.arctan(y * z / (x * R))
        result = result + np.where(x * R > 0, t, 0.0)
    return result


def newell_g(x, y, z):
    """demag_field.cpp:42-69 (vectorised, same term order)."""
    z = np.abs(z)
    R = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    xx, yy, zz = x ** 2, y ** 2, z ** 2
    result = -x * y * R / 3.0
    with np.errstate(all="ignore"):
        t = x * y * z * np.arcsinh(z / np.sqrt(xx + yy))
        result = result + np.where(xx + yy > 0, t, 0.0)
        t = y / 6.0 * (3.0 * zz - yy) * np.arcsinh(x / np.sqrt(yy + zz))
        result = result + np.where(yy + zz > 0, t, 0.0)
        t = x / 6.0 * (3.0 * zz - xx) * np.arcsinh(y / np.sqrt(xx + zz))
        result = result + np.where(xx + zz > 0, t, 0.0)
        t = -(z ** 3) / 6.0 * np.arctan(x * y / (z * R))
        result = result + np.where(z * R > 0, t, 0.0)
        t = -z * yy / 2.0 * np.arctan(x * z / (y * R))
        result = result + np.where(y * R != 0, t, 0.0)
        t = -z * xx / 2.0 * np.arctan(y * z / (x * R))
        result = result + np.where(x * R != 0, t, 0.0)
    return result


# the 27 stencil points in the reference's summation order (demag_field.cpp:75-83)
_NEWELL_STENCIL = (
    [(8.0, 0, 0, 0)]
    + [(-4.0, 1, 0, 0), (-4.0, -1, 0, 0), (-4.0, 0, 1, 0), (-4.0, 0, -1, 0), (-4.0, 0, 0, 1), (-4.0, 0, 0, -1)]
    + [(2.0, 1, 1, 0), (2.0, 1, -1, 0), (2.0, -1, 1, 0), (2.0, -1, -1, 0),
       (2.0, 1, 0, 1), (2.0, 1, 0, -1), (2.0, -1, 0, 1), (2.0, -1, 0, -1),
       (2.0, 0, 1, 1), (2.0, 0, 1, -1), (2.0, 0, -1, 1), (2.0, 0, -1, -1)]
    + [(-1.0, 1, 1, 1), (-1.0, 1, 1, -1), (-1.0, 1, -1, 1), (-1.0, 1, -1, -1),
       (-1.0, -1, 1, 1), (-1.0, -1, 1, -1), (-1.0, -1, -1, 1), (-1.0, -1, -1, -1)]
)


def _newell_27(fn, ix, iy, iz, dx, dy, dz):
    x = dx * np.asarray(ix, dtype=np.float64)
    y = dy * np.asarray(iy, dtype=np.float64)
    z = dz * np.asarray(iz, dtype=np.float64)
    result = 0.0
    for w, a, b, c in _NEWELL_STENCIL:
        xa = x if a == 0 else (x + dx if a > 0 else x - dx)
        yb = y if b == 0 else (y + dy if b > 0 else y - dy)
        zc = z if c == 0 else (z + dz if c > 0 else z - dz)
        result = result + w * fn(xa, yb, zc)
    return -result / (4.0 * math.pi * dx * dy * dz)


def Nxx(ix, iy, iz, dx, dy, dz):
    """demag_field.cpp:71-85"""
    return _newell_27(newell_f, ix, iy, iz, dx, dy, dz)


def Nxy(ix, iy, iz, dx, dy, dz):
    """demag_field.cpp:87-102"""
    return _newell_27(newell_g, ix, iy, iz, dx, dy, dz)


def newell_wrapped_index(i, P):
    """j = (i + P/2) % P - P/2  (demag_field.cpp:106-110)"""
    return (i + P // 2) % P - P // 2


def demag_tensor_real(mesh: Mesh) -> np.ndarray:
    """setup_N (demag_field.cpp:104-121): real tensor [Px, Py, Pz, 6] with the
    component order xx, xy, xz, yy, yz, zz."""
    Px, Py, Pz = nx_exp(mesh.nx), nx_exp(mesh.ny), nz_exp(mesh.nz)
    j0 = newell_wrapped_index(np.arange(Px), Px)
    j1 = newell_wrapped_index(np.arange(Py), Py)
    j2 = newell_wrapped_index(np.arange(Pz), Pz)
    J0, J1, J2 = np.meshgrid(j0, j1, j2, indexing="ij")
    dx, dy, dz = mesh.dx, mesh.dy, mesh.dz
    N = np.empty((Px, Py, Pz, 6))
    N[..., 0] = Nxx(J0, J1, J2, dx, dy, dz)
    N[..., 1] = Nxy(J0, J1, J2, dx, dy, dz)
    N[..., 2] = Nxy(J0, J2, J1, dx, dz, dy)
    N[..., 3] = Nxx(J1, J2, J0, dy, dz, dx)
    N[..., 4] = Nxy(J1, J2, J0, dy, dz, dx)
    N[..., 5] = Nxx(J2, J0, J1, dz, dx, dy)
    return N


_ODD_AXES = {0: (), 1: (0, 1), 2: (0, 2), 3: (), 4: (1, 2), 5: ()}


def _octant_chunk(args):
    """Newell values on the octant planes a0 in [a0_lo, a0_hi) (process-pool worker)."""
    a0_lo, a0_hi, ny1, nz1, dx, dy, dz = args
    A0, A1, A2 = np.meshgrid(np.arange(a0_lo, a0_hi), np.arange(ny1), np.arange(nz1), indexing="ij")
    out = np.empty(A0.shape + (6,))
    out[..., 0] = Nxx(A0, A1, A2, dx, dy, dz)
    out[..., 1] = Nxy(A0, A1, A2, dx, dy, dz)
    out[..., 2] = Nxy(A0, A2, A1, dx, dz, dy)
    out[..., 3] = Nxx(A1, A2, A0, dy, dz, dx)
    out[..., 4] = Nxy(A1, A2, A0, dy, dz, dx)
    out[..., 5] = Nxx(A2, A0, A1, dz, dx, dy)
    return out


def demag_tensor_symmetric(mesh: Mesh, workers: int = 0) -> np.ndarray:
    """The parity-exact tensor: the reference formula evaluated at
    (|j0|, |j1|, |j2|), multiplied by each component's parity sign (xy odd in
    x and y, xz odd in x and z, yz odd in y and z), with odd components set to
    zero where they vanish in exact arithmetic (j = 0 along an odd axis) and
    on their Nyquist planes j = -P/2.  Entries with |j| = P/2 never reach the
    truncated output of the zero-padded convolution, so the field on the mesh
    equals the reference's up to the rounding noise of its 27-point sums,
    while the spectrum becomes exactly real and even/odd.  The octant
    |j| <= P/2 is evaluated once (workers > 1: in a spawned process pool)."""
    Px, Py, Pz = nx_exp(mesh.nx), nx_exp(mesh.ny), nz_exp(mesh.nz)
    P = (Px, Py, Pz)
    n1 = (Px // 2 + 1, Py // 2 + 1, Pz // 2 + 1)
    args = (mesh.dx, mesh.dy, mesh.dz)
    if workers and workers > 1:
        import concurrent.futures as cf
        import multiprocessing as mp
        step = max(1, n1[0] // (4 * workers))
        chunks = [(a, min(a + step, n1[0]), n1[1], n1[2]) + args for a in range(0, n1[0], step)]
        with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            octant = np.concatenate(list(ex.map(_octant_chunk, chunks)), axis=0)
    else:
        octant = _octant_chunk((0, n1[0], n1[1], n1[2]) + args)
    j = [newell_wrapped_index(np.arange(p), p) for p in P]
    N = octant[np.abs(j[0])][:, np.abs(j[1])][:, :, np.abs(j[2])]
    for c, axes in _ODD_AXES.items():
        sign = np.ones(P)
        for ax in axes:
            shape = [1, 1, 1]
            shape[ax] = P[ax]
            jj = j[ax].reshape(shape)
            s = np.where(jj < 0, -1.0, 1.0)
            s = np.where(jj == 0, 0.0, s)
            if P[ax] > 1:
                s = np.where(jj == -(P[ax] // 2), 0.0, s)
            sign = sign * s
        N[..., c] = N[..., c] * sign
    return N


# Number of host threads for the oracle's FFTs.  None: numpy.fft (single
# thread, used by the tests); an int: scipy.fft with that many workers (used
# when the oracle is timed as the CPU baseline on all host cores).
FFT_WORKERS: Optional[int] = None


def _rfft3(a, P):
    """ArrayFire fftR2C over dims 0..2 of a [x,y,z,...] array: halves dim 0."""
    if FFT_WORKERS:
        import scipy.fft as sf
        return sf.rfftn(a, s=(P[1], P[2], P[0]), axes=(1, 2, 0), workers=FFT_WORKERS)
    return np.fft.rfftn(a, s=(P[1], P[2], P[0]), axes=(1, 2, 0))


def _irfft3(a, P):
    """ArrayFire fftC2R with the 1/N normalisation (demag_field.cpp:251-257)."""
    if FFT_WORKERS:
        import scipy.fft as sf
        return sf.irfftn(a, s=(P[1], P[2], P[0]), axes=(1, 2, 0), workers=FFT_WORKERS)
    return np.fft.irfftn(a, s=(P[1], P[2], P[0]), axes=(1, 2, 0))


class DemagField(FieldTerm):
    """Open-boundary demag by zero-padded FFT convolution
    (demag_field.cpp:144-147, 211-264).  ``N_real`` lets a test feed a tensor
    computed elsewhere (e.g. the device's) so that the convolution is checked
    on identical inputs."""

    def __init__(self, mesh: Mesh, N_real: Optional[np.ndarray] = None, symmetric: bool = False,
                 Nfft: Optional[np.ndarray] = None):
        self.mesh = mesh
        self.P = (nx_exp(mesh.nx), nx_exp(mesh.ny), nz_exp(mesh.nz))
        if Nfft is not None:
            # spectral tensor supplied directly ([Px/2+1, Py, Pz, 6]); used by the timed CPU baseline
            self.N_real = None
            self.Nfft = Nfft
            return
        if N_real is None:
            N_real = demag_tensor_symmetric(mesh) if symmetric else demag_tensor_real(mesh)
        self.N_real = N_real
        self.Nfft = _rfft3(N_real, self.P)

    def H_in_Apm(self, state):
        nx, ny, nz = state.mesh.nx, state.mesh.ny, state.mesh.nz
        Msm = state.m * state.Ms_v()
        mfft = _rfft3(Msm, self.P)
        N = self.Nfft
        hfft = np.empty_like(mfft)
        hfft[..., 0] = N[..., 0] * mfft[..., 0] + N[..., 1] * mfft[..., 1] + N[..., 2] * mfft[..., 2]
        hfft[..., 1] = N[..., 1] * mfft[..., 0] + N[..., 3] * mfft[..., 1] + N[..., 4] * mfft[..., 2]
        hfft[..., 2] = N[..., 2] * mfft[..., 0] + N[..., 4] * mfft[..., 1] + N[..., 5] * mfft[..., 2]
        h = _irfft3(hfft, self.P)
        return np.ascontiguousarray(h[:nx, :ny, :nz, :])


# ---------------------------------------------------------------------------
# stencils
# ---------------------------------------------------------------------------
def _shift(a, axis, s):
    """b[i] = a[i+s] along axis, zero outside (zero-padded convolution)."""
    out = np.zeros_like(a)
    n = a.shape[axis]
    if abs(s) >= n:
        return out
    src = [slice(None)] * a.ndim
    dst = [slice(None)] * a.ndim
    if s > 0:
        src[axis] = slice(s, n)
        dst[axis] = slice(0, n - s)
    else:
        src[axis] = slice(0, n + s)
        dst[axis] = slice(-s, n)
    out[tuple(dst)] = a[tuple(src)]
    return out


def laplace_zero_padded(m, dx, dy, dz):
    """3x3x3 convolution with the 7-point Laplacian filter including the
    centre -2/dx^2-2/dy^2-2/dz^2 (exchange_field.cpp:115-126)."""
    c = -2.0 / dx ** 2 - 2.0 / dy ** 2 - 2.0 / dz ** 2
    out = c * m
    out = out + (_shift(m, 0, 1) + _shift(m, 0, -1)) / dx ** 2
    out = out + (_shift(m, 1, 1) + _shift(m, 1, -1)) / dy ** 2
    out = out + (_shift(m, 2, 1) + _shift(m, 2, -1)) / dz ** 2
    return out


def central_diff(a, h, axis):
    """math::central_diff (magnumaf/src/math.cpp:42-66): (a[i+1]-a[i-1])/(2h),
    zero padded; a true convolution, pinned by magnumaf/test/math.cpp:8-19."""
    return (_shift(a, axis, 1) - _shift(a, axis, -1)) * (0.5 / h)


class ExchangeField(FieldTerm):
    """exchange_field.cpp:115-157 (H) and :14-60 (E with h_withedges)."""

    def __init__(self, A: float):
        self.A = A

    def H_in_Apm(self, state):
        mesh = state.mesh
        exch = laplace_zero_padded(state.m, mesh.dx, mesh.dy, mesh.dz)
        if state.Ms_field is None:
            return (2.0 * self.A) / (mu0 * state.Ms) * exch
        with np.errstate(divide="ignore", invalid="ignore"):
            h = (2.0 * self.A) / (mu0 * state.Ms_field[..., None]) * exch
        return _replace_ms_zero(h, state)

    def h_withedges(self, state):
        mesh = state.mesh
        m = state.m
        exch = laplace_zero_padded(m, mesh.dx, mesh.dy, mesh.dz)
        exch[0] += m[0] / mesh.dx ** 2
        exch[-1] += m[-1] / mesh.dx ** 2
        exch[:, 0] += m[:, 0] / mesh.dy ** 2
        exch[:, -1] += m[:, -1] / mesh.dy ** 2
        exch[:, :, 0] += m[:, :, 0] / mesh.dz ** 2
        exch[:, :, -1] += m[:, :, -1] / mesh.dz ** 2
        h = (2.0 * self.A) / mu0 * _inv_Ms(state) * exch
        return _replace_ms_zero(h, state)

    def Energy_in_J(self, state, h=None):
        return micro_energy(state, self.h_withedges(state))


class DmiField(FieldTerm):
    """Interface DMI, dmi_field.cpp:41-110: H = 2D/(mu0 Ms) [n div m - grad(n.m)]
    with zero-padded central differences and no DMI boundary condition."""

    def __init__(self, D: float, D_axis=(0.0, 0.0, 1.0), D_field=None):
        self.D = D
        self.D_axis = tuple(float(v) for v in D_axis)
        self.D_field = D_field

    def H_in_Apm(self, state):
        mesh = state.mesh
        m = state.m
        nrm = math.sqrt(sum(v * v for v in self.D_axis))
        n = np.array(self.D_axis) / nrm
        div = (central_diff(m[..., 0], mesh.dx, 0) + central_diff(m[..., 1], mesh.dy, 1)) + central_diff(
            m[..., 2], mesh.dz, 2)
        first = n[None, None, None, :] * div[..., None]
        nm = m[..., 0] * n[0] + m[..., 1] * n[1] + m[..., 2] * n[2]
        second = np.stack([central_diff(nm, mesh.dx, 0), central_diff(nm, mesh.dy, 1), central_diff(nm, mesh.dz, 2)],
                          axis=3)
        D = self.D if self.D_field is None else np.asarray(self.D_field)[..., None]
        h = (2.0 * D) / mu0 * _inv_Ms(state) * (first - second)
        return _replace_ms_zero(h, state)


class BulkDMIExchangeField(FieldTerm):
    """bulk_dmi_exchange_field.cpp:11-119: ghost cells carrying the coupled
    DMI/exchange boundary condition, then curl and Laplacian (math.cpp:86-122)."""

    def __init__(self, D: float, A: float):
        self.D = D
        self.A = A

    def ghost(self, m, dx, dy, dz):
        D, A = self.D, self.A
        nx, ny, nz, _ = m.shape
        g = np.zeros((nx + 2, ny + 2, nz + 2, 3))
        g[1:-1, 1:-1, 1:-1] = m
        for (d, axis) in ((dx, 0), (dy, 1), (dz, 2)):
            c = 2.0 * d * D / (2.0 * A)
            for plus in (False, True):
                i = -1 if plus else 0
                io = -2 if plus else 1
                sign = 1.0 if plus else -1.0
                sl_m = [slice(None)] * 3
                sl_m_in = [slice(None)] * 3
                sl_g = [slice(1, -1)] * 3
                sl_m[axis] = i
                sl_m_in[axis] = io
                sl_g[axis] = i
                mi = m[tuple(sl_m)]
                mo = m[tuple(sl_m_in)]
                gs = g[tuple(sl_g)]
                if axis == 0:
                    gs[..., 0] = mo[..., 0]
                    gs[..., 1] = mo[..., 1] + c * (sign * -1.0 * mi[..., 2])
                    gs[..., 2] = mo[..., 2] + c * (sign * mi[..., 1])
                elif axis == 1:
                    gs[..., 0] = mo[..., 0] + c * (sign * mi[..., 2])
                    gs[..., 1] = mo[..., 1]
                    gs[..., 2] = mo[..., 2] + c * (sign * -1.0 * mi[..., 0])
                else:
                    gs[..., 0] = mo[..., 0] + c * (sign * -1.0 * mi[..., 1])
                    gs[..., 1] = mo[..., 1] + c * (sign * mi[..., 0])
                    gs[..., 2] = mo[..., 2]
                g[tuple(sl_g)] = gs
        return g

    def H_in_Apm(self, state):
        mesh = state.mesh
        g = self.ghost(state.m, mesh.dx, mesh.dy, mesh.dz)
        ddx = central_diff(g, mesh.dx, 0)[1:-1, 1:-1, 1:-1]
        ddy = central_diff(g, mesh.dy, 1)[1:-1, 1:-1, 1:-1]
        ddz = central_diff(g, mesh.dz, 2)[1:-1, 1:-1, 1:-1]
        curl = np.stack([ddy[..., 2] - ddz[..., 1], ddz[..., 0] - ddx[..., 2], ddx[..., 1] - ddy[..., 0]], axis=3)
        lap = laplace_zero_padded(g, mesh.dx, mesh.dy, mesh.dz)[1:-1, 1:-1, 1:-1]
        result = 2.0 * self.D * curl + (-2.0 * self.A) * lap
        if state.Ms_field is None:
            return result / (-mu0 * state.Ms)
        with np.errstate(all="ignore"):
            return result / (-mu0 * state.Ms_field[..., None])


def normalize_vector(v):
    v = np.asarray(v, dtype=np.float64)
    return v / math.sqrt(float(np.sum(v * v)))


class UniaxialAnisotropyField(FieldTerm):
    """uniaxial_anisotropy_field.cpp:58-89: H = 2Ku/(mu0 Ms) e (e.m)."""

    def __init__(self, Ku1, Ku1_axis=(0.0, 0.0, 1.0), Ku1_axis_field=None):
        self.Ku1 = Ku1  # scalar or (nx,ny,nz) field
        self.Ku1_axis = normalize_vector(Ku1_axis)
        self.Ku1_axis_field = None if Ku1_axis_field is None else normalize(np.asarray(Ku1_axis_field, np.float64))

    def H_in_Apm(self, state):
        eu = self.Ku1_axis[None, None, None, :] if self.Ku1_axis_field is None else self.Ku1_axis_field
        an = np.sum(eu * state.m, axis=3)[..., None]
        Ku = self.Ku1 if np.ndim(self.Ku1) == 0 else np.asarray(self.Ku1)[..., None]
        h = 2.0 * Ku / mu0 * _inv_Ms(state) * (eu * an)
        return _replace_ms_zero(h, state)


class CubicAnisotropyField(FieldTerm):
    """cubic_anisotropy_field.cpp:61-113 (scalar constants and lab-fixed axes)."""

    def __init__(self, Kc1, Kc2=0.0, Kc3=0.0, c1=(1.0, 0.0, 0.0), c2=(0.0, 1.0, 0.0)):
        # UnitVectorOrArray normalises the axes (unit_vector_or_array.hpp:14)
        c1 = normalize_vector(c1)
        c2 = normalize_vector(c2)
        if abs(float(np.dot(c1, c2))) > 1e-12:
            raise ValueError("CubicAnisotropyField: c1 and c2 are not perpendicular")
        self.Kc1, self.Kc2, self.Kc3 = Kc1, Kc2, Kc3
        self.c1 = c1
        self.c2 = c2
        self.c3 = normalize_vector(np.cross(c1, c2))

    def h_1to3(self, state):
        m = state.m
        c1, c2, c3 = (c[None, None, None, :] for c in (self.c1, self.c2, self.c3))
        c1m = np.sum(c1 * m, axis=3)[..., None]
        c2m = np.sum(c2 * m, axis=3)[..., None]
        c3m = np.sum(c3 * m, axis=3)[..., None]
        c1m2, c2m2, c3m2 = c1m ** 2, c2m ** 2, c3m ** 2
        c1m4, c2m4, c3m4 = c1m ** 4, c2m ** 4, c3m ** 4
        c1m3, c2m3, c3m3 = c1m ** 3, c2m ** 3, c3m ** 3
        if state.Ms_field is None:
            Ms = state.Ms
        else:
            Ms = state.Ms_field[..., None]
        with np.errstate(all="ignore"):
            h1 = -2 / (mu0 * Ms) * self.Kc1 * ((c2m2 + c3m2) * c1m * c1 + (c1m2 + c3m2) * c2m * c2
                                              + (c1m2 + c2m2) * c3m * c3)
            h2 = -2 / (mu0 * Ms) * self.Kc2 * (c2m2 * c3m2 * c1m * c1 + c1m2 * c3m2 * c2m * c2
                                              + c1m2 * c2m2 * c3m * c3)
            h3 = -4 / (mu0 * Ms) * self.Kc3 * ((c2m4 + c3m4) * c1m3 * c1 + (c1m4 + c3m4) * c2m3 * c2
                                              + (c1m4 + c2m4) * c3m3 * c3)
        return h1, h2, h3

    def H_in_Apm(self, state):
        h1, h2, h3 = self.h_1to3(state)
        return h1 + h2 + h3

    def Energy_in_J(self, state, h=None):
        h1, h2, h3 = self.h_1to3(state)
        Ms = state.Ms if state.Ms_field is None else state.Ms_field[..., None]
        dV = state.mesh.dx * state.mesh.dy * state.mesh.dz
        return mu0 * float(np.sum(Ms * (-1 / 4.0 * h1 - 1 / 6.0 * h2 - 1 / 8.0 * h3) * state.m)) * dV


class ExternalField(FieldTerm):
    """external_field.cpp:28-48: returns the stored field; E = -mu0 Ms sum(h.m) dV."""

    def __init__(self, zee):
        self.zee = np.asarray(zee, dtype=np.float64)

    def H_in_Apm(self, state):
        return np.broadcast_to(self.zee, state.m.shape).copy()

    def Energy_in_J(self, state, h=None):
        if h is None:
            h = self.H_in_Apm(state)
        return micro_energy(state, h, factor=-mu0)


class SpinTransferTorqueField(FieldTerm):
    """spin_transfer_torque_field.cpp:7-28: H = -j_e hbar / (2 e mu0 Ms d) (eta_d m x p + eta_f p),
    p = normalize(polarization); zero where Ms_field == 0; default micro energy."""

    def __init__(self, pol, eta_damping, eta_field, j_e, fl_thickness):
        self.pol = normalize(np.asarray(pol, dtype=np.float64))
        self.eta_damping, self.eta_field = float(eta_damping), float(eta_field)
        self.j_e, self.fl_thickness = float(j_e), float(fl_thickness)

    def H_in_Apm(self, state):
        pre = -self.j_e * hbar / (2.0 * e_neg * mu0 * self.fl_thickness)
        h = pre * _inv_Ms(state) * (self.eta_damping * cross4(state.m, self.pol) + self.eta_field * self.pol)
        return _replace_ms_zero(np.nan_to_num(h, nan=0.0, posinf=0.0, neginf=0.0), state)


def exchange_matrix(mesh, A, A_field=None, periodic=False):
    """One component block (N x N, cell index i0 + nx*(i1 + ny*i2)) of the 3N x 3N
    exchange matrix of SparseExchangeField / ExchangeFieldPBC, assembled as COO
    triplets and summed into CSR like the reference:
      scalar A, open (sparse_exchange_field.cpp:25-101): neighbours inside the
        mesh in the order +x,-x,+y,-y,+z,-z, value (2A)/mu0/d^2, no diagonal;
      A field (sparse_exchange_field.cpp:289-330) or periodic
        (exchange_field_pbc.cpp:126-163): value lapA(A_i, A_nb, d) =
        2A_i/(mu0 d^2) * 2A_nb/(A_nb+A_i) (sparse_exchange_field.cpp:183-185),
        periodic neighbours wrapped (i+n) % n, then the diagonal -sum; rows of
        cells with A_i = 0 are left empty.
    The three component blocks of the reference's matrix are identical."""
    import scipy.sparse as sp

    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    N = nx * ny * nz
    i0, i1, i2 = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    row = (i0 + nx * (i1 + ny * i2)).reshape(-1, order="F")
    Af = np.full((nx, ny, nz), float(A)) if A_field is None else np.asarray(A_field, dtype=np.float64)
    Ai = Af.reshape(-1, order="F")
    harmonic = periodic or A_field is not None
    rows, cols, vals = [], [], []
    m_self = np.zeros(N)
    dirs = [(0, 1, mesh.dx), (0, -1, mesh.dx), (1, 1, mesh.dy), (1, -1, mesh.dy), (2, 1, mesh.dz), (2, -1, mesh.dz)]
    for axis, s, d in dirs:
        idx = [i0, i1, i2]
        n = (nx, ny, nz)[axis]
        j = idx[axis] + s
        if periodic:
            j = (j + n) % n
            valid = np.ones_like(j, dtype=bool)
        else:
            valid = (j >= 0) & (j < n)
        idx[axis] = np.where(valid, j, 0)
        nb = (idx[0] + nx * (idx[1] + ny * idx[2])).reshape(-1, order="F")
        valid = valid.reshape(-1, order="F")
        if harmonic:
            Anb = Ai[nb]
            with np.errstate(divide="ignore", invalid="ignore"):
                w = 2.0 * Ai / (mu0 * d ** 2) * 2.0 * Anb / (Anb + Ai)
            keep = valid & (Ai != 0.0)
            m_self[keep] -= w[keep]
        else:
            w = np.full(N, (2.0 * float(A)) / mu0 / d ** 2)
            keep = valid
        rows.append(row[keep])
        cols.append(nb[keep])
        vals.append(w[keep])
    if harmonic:
        keep = Ai != 0.0
        rows.append(row[keep])
        cols.append(row[keep])
        vals.append(m_self[keep])
    coo = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    return coo.tocsr()


class SparseExchangeField(FieldTerm):
    """sparse_exchange_field.cpp:8-18: H = matr * flat(m) / Ms, zero where
    Ms_field == 0; default micro energy (micro_term.hpp:18)."""

    periodic = False

    def __init__(self, A, mesh):
        if np.ndim(A) == 0:
            self.matr = exchange_matrix(mesh, float(A), None, self.periodic)
        else:
            self.matr = exchange_matrix(mesh, 0.0, np.asarray(A, dtype=np.float64), self.periodic)

    def H_in_Apm(self, state):
        m = state.m
        exch = np.stack([(self.matr @ m[..., c].reshape(-1, order="F")).reshape(m.shape[:3], order="F")
                         for c in range(3)], axis=3)
        with np.errstate(divide="ignore", invalid="ignore"):
            h = exch * _inv_Ms(state)
        return _replace_ms_zero(h, state)


class ExchangeFieldPBC(SparseExchangeField):
    """exchange_field_pbc.cpp:9-19: the harmonic-mean matrix with periodic
    neighbours in x, y and z."""

    periodic = True


class DemagFieldPBC(FieldTerm):
    """demag_field_pbc.cpp:10-71: periodic demag through the scalar potential on
    the mesh's own grid.  R2C of Ms*m (x halved), K_a = 2 pi k_a / n_a,
    div = sum_a (1 - exp(-i K_a)) M_a / d_a, u = -div / sum_a 4/d_a^2 sin^2(K_a/2)
    with u(0,0,0) = 0, H_a = (1 - exp(i K_a)) u / d_a, then C2R with the 1/N
    normalisation (the fftC2R default).  The C2R returns 2*(nx//2) columns
    (is_odd = false), so only even nx gives the mesh's shape."""

    def H_in_Apm(self, state):
        mesh = state.mesh
        nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
        if nx % 2:
            raise ValueError("DemagFieldPBC: nx must be even")
        ms = state.Ms if state.Ms_field is None else state.Ms_field[..., None]
        M = np.fft.rfftn(ms * state.m, axes=(1, 2, 0))  # real transform along x
        kx = (2.0 * math.pi * np.arange(nx // 2 + 1) / nx)[:, None, None]
        ky = (2.0 * math.pi * np.arange(ny) / ny)[None, :, None]
        kz = (2.0 * math.pi * np.arange(nz) / nz)[None, None, :]
        div = ((1.0 - np.exp(-1j * kx)) * M[..., 0] / mesh.dx + (1.0 - np.exp(-1j * ky)) * M[..., 1] / mesh.dy
               + (1.0 - np.exp(-1j * kz)) * M[..., 2] / mesh.dz)
        den = (4.0 / mesh.dx ** 2 * np.sin(kx / 2.0) ** 2 + 4.0 / mesh.dy ** 2 * np.sin(ky / 2.0) ** 2
               + 4.0 / mesh.dz ** 2 * np.sin(kz / 2.0) ** 2)
        with np.errstate(divide="ignore", invalid="ignore"):
            u = -div / den
        u[0, 0, 0] = 0.0
        h = np.stack([(1.0 - np.exp(1j * kx)) * u / mesh.dx, (1.0 - np.exp(1j * ky)) * u / mesh.dy,
                      (1.0 - np.exp(1j * kz)) * u / mesh.dz], axis=3)
        return np.fft.irfftn(h, s=(ny, nz, nx), axes=(1, 2, 0))


def Heff_in_Apm(terms: Sequence[FieldTerm], state):
    """sequential_Heff_in_Apm, field_term.hpp:116-119."""
    h = terms[0].H_in_Apm(state)
    for t in terms[1:]:
        h = h + t.H_in_Apm(state)
    return h


def Eeff_in_J(terms, state):
    return sum(t.Energy_in_J(state) for t in terms)


# ---------------------------------------------------------------------------
# LLG (equations.hpp:19-33, math.cpp:10-19)
# ---------------------------------------------------------------------------
def cross4(a, b):
    c = np.empty(np.broadcast_shapes(a.shape, b.shape))
    c[..., 0] = a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1]
    c[..., 1] = a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2]
    c[..., 2] = a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]
    return c


def LLG(alpha, m, h, dissipation_term_only=False):
    mxh = cross4(m, h)
    damp = -alpha * gamma / (1.0 + alpha ** 2) * cross4(m, mxh)
    if dissipation_term_only:
        return damp
    return -gamma / (1.0 + alpha ** 2) * mxh + damp


# ---------------------------------------------------------------------------
# Controller  (controller.hpp:11-61, controller.cpp:36-95)
# ---------------------------------------------------------------------------
class Controller:
    beta = 0.4 / 5.0
    alpha = 0.2 - 0.75 * beta
    headroom = 0.9
    minscale = 0.2
    maxscale = 10.0

    def __init__(self, hmin=1e-15, hmax=3.5e-10, atol=1e-6, rtol=1e-6):
        self.hmin, self.hmax, self.atol, self.rtol = hmin, hmax, atol, rtol
        self.reject = False
        self.errold = 1.0e-4
        self.hnext = 0.0
        self.counter_reject = 0
        self.counter_accepted = 0
        self.counter_hmax = 0
        self.counter_hmin = 0

    def givescale(self, a):
        return self.atol + self.rtol * np.abs(a)

    def success(self, err, h):
        """returns (accepted, h)"""
        if err <= 1.0:
            if err == 0.0:
                scale = self.maxscale
            else:
                scale = self.headroom * err ** (-self.alpha) * self.errold ** self.beta
                scale = min(max(scale, self.minscale), self.maxscale)
            if self.reject:
                self.hnext = h * min(scale, 1.0)
            else:
                self.hnext = h * scale
            if self.hnext <= self.hmin:
                self.hnext = self.hmin
                self.counter_hmin += 1
            elif self.hnext >= self.hmax:
                self.hnext = self.hmax
                self.counter_hmax += 1
            self.errold = max(err, 1.0e-4)
            self.reject = False
            self.counter_accepted += 1
            return True, h
        scale = max(self.headroom * err ** (-self.alpha), self.minscale)
        h = h * scale
        if h <= self.hmin:
            self.counter_hmin += 1
            return True, self.hmin
        if h >= self.hmax:
            self.counter_hmax += 1
            return True, self.hmax
        self.reject = True
        self.counter_reject += 1
        return False, h


# Butcher tableaus (adaptive_runge_kutta.cpp:75-173, 496-529)
RKF45_A = [
    [],
    [1. / 4.],
    [3. / 32., 9 / 32.],
    [1932. / 2197., -7200. / 2197., 7296. / 2197.],
    [439. / 216., -8., 3680. / 513., -845. / 4104.],
    [-8. / 27., 2., -3544. / 2565., 1859. / 4104., -11. / 40.],
]
RKF45_C = [0.0, 1. / 4., 3. / 8., 12. / 13., 1.0, 1. / 2.]


def _dp45_tableau():
    a = [[0.0] * 7 for _ in range(8)]
    e = [0.0] * 8
    c = [0.0] * 8
    c[2], c[3], c[4], c[5], c[6], c[7] = 0.2, 0.3, 0.8, 8.0 / 9.0, 1, 1
    e[1], e[3], e[4], e[5], e[6], e[7] = 71.0 / 57600.0, -71.0 / 16695.0, 71.0 / 1920.0, -17253.0 / 339200.0, \
        22.0 / 525.0, -1.0 / 40.0
    a[2][1] = 0.2
    a[3][1], a[3][2] = 3.0 / 40.0, 9.0 / 40.0
    a[4][1], a[4][2], a[4][3] = 44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0
    a[5][1], a[5][2], a[5][3], a[5][4] = 19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0
    a[6][1], a[6][2], a[6][3], a[6][4], a[6][5] = 9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, \
        -5103.0 / 18656.0
    a[7][1], a[7][3], a[7][4], a[7][5], a[7][6] = 35.0 / 384.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, \
        11.0 / 84.0
    return a, e, c


DP45_A, DP45_E, DP45_C = _dp45_tableau()


class AdaptiveRungeKutta:
    """adaptive_runge_kutta.cpp:39-71 step loop; the schemes below keep the
    reference's expression order.  ``f(state) -> dm/dt``."""

    def __init__(self, scheme="RKF45", controller: Optional[Controller] = None, normalize_=True):
        if scheme not in ("RKF45", "DP45", "BS23"):
            raise ValueError("Integration method not found: " + scheme)
        self.scheme = scheme
        self.controller = controller if controller is not None else Controller()
        self.normalize_ = normalize_
        self.h = 1.01e-15
        self.k_FSAL = None
        self.step_calls = 0
        self.accumulated_steps = 0

    def f(self, state):
        raise NotImplementedError

    def _scale_err(self, state, sumbk, rk_error):
        return float(np.max(np.abs(rk_error / self.controller.givescale(np.maximum(state.m, state.m + sumbk)))))

    def RKF45(self, state, dt):
        a, c = RKF45_A, RKF45_C
        tmp = state.copy()
        k = [dt * self.f(state)]
        for s in range(1, 6):
            tmp.t = state.t + c[s] * dt
            acc = state.m
            for j, aj in enumerate(a[s]):
                # 'm - 8/27 k1' of stage 6 equals 'm + (-8/27) k1' exactly
                acc = acc + aj * k[j]
            tmp.m = acc
            k.append(dt * self.f(tmp))
        k1, k2, k3, k4, k5, k6 = k
        sumbk = 16. / 135. * k1 + 6656. / 12825. * k3 + 28561. / 56430. * k4 - 9. / 50. * k5 + 2. / 55. * k6
        rk_error = sumbk - (25. / 216. * k1 + 1408. / 2565. * k3 + 2197. / 4104. * k4 - 1. / 5. * k5)
        return sumbk, self._scale_err(state, sumbk, rk_error)

    def DP45(self, state, dt):
        a, e, c = DP45_A, DP45_E, DP45_C
        tmp = state.copy()
        if self.controller.reject or self.normalize_ or state.steps == 0 or self.k_FSAL is None:
            k1 = dt * self.f(tmp)
        else:
            k1 = self.k_FSAL
        k = [None, k1]
        for s in range(2, 8):
            tmp.t = state.t + c[s] * dt
            acc = state.m
            for j in range(1, s):
                acc = acc + a[s][j] * k[j]
            tmp.m = acc
            k.append(dt * self.f(tmp))
        self.k_FSAL = k[7]
        sumbk = a[7][1] * k[1]
        for j in range(2, 7):
            sumbk = sumbk + a[7][j] * k[j]
        rk_error = e[1] * k[1]
        for j in range(2, 8):
            rk_error = rk_error + e[j] * k[j]
        return sumbk, self._scale_err(state, sumbk, rk_error)

    def BS23(self, state, dt):
        tmp = state.copy()
        if self.controller.reject or self.normalize_ or self.step_calls == 0 or self.k_FSAL is None:
            k1 = self.f(tmp)
        else:
            k1 = self.k_FSAL
        tmp.t = state.t + 1. / 2. * dt
        tmp.m = state.m + dt * (1. / 2. * k1)
        k2 = self.f(tmp)
        tmp.t = state.t + 3. / 4. * dt
        tmp.m = state.m + dt * 3. / 4. * k2
        k3 = self.f(tmp)
        sumbk = dt * (2. / 9. * k1 + 1. / 3. * k2 + 4. / 9. * k3)
        tmp.t = state.t + dt
        tmp.m = state.m + sumbk
        self.k_FSAL = self.f(tmp)
        rk_error = sumbk - dt * (7. / 24. * k1 + 1. / 4. * k2 + 1. / 3. * k3 + 1. / 8. * self.k_FSAL)
        return sumbk, self._scale_err(state, sumbk, rk_error)

    def attempt(self, state, h):
        return getattr(self, self.scheme)(state, h)

    def step(self, state):
        while True:
            mtemp, err = self.attempt(state, self.h)
            ok, self.h = self.controller.success(err, self.h)
            if ok:
                break
        state.t += self.h
        self.h = self.controller.hnext
        state.m = state.m + mtemp
        if self.normalize_:
            if state.Ms_field is None:
                state.m = normalize_even_zero_vectors(state.m)
            else:
                state.m = normalize(state.m)
        state.steps += 1
        self.step_calls += 1
        self.accumulated_steps += 1


class LLGIntegrator(AdaptiveRungeKutta):
    """llg_integrator.hpp:26-82, llg_integrator.cpp:11-104."""

    def __init__(self, alpha, terms, scheme="RKF45", controller=None, dissipation_term_only=False):
        super().__init__(scheme, controller)
        self.alpha = alpha  # scalar or (nx,ny,nz) field
        self.terms = list(terms)
        self.dissipation_term_only = dissipation_term_only

    def fheff(self, state):
        return Heff_in_Apm(self.terms, state)

    def f(self, state):
        alpha = self.alpha if np.ndim(self.alpha) == 0 else np.asarray(self.alpha)[..., None]
        return LLG(alpha, state.m, self.fheff(state), self.dissipation_term_only)

    def E(self, state):
        return Eeff_in_J(self.terms, state)

    def integrate_dense(self, state, time_in_s, write_every_dt_in_s):
        """llg_integrator.cpp:68-104; returns the rows (t, <mx>, <my>, <mz>)."""
        rows = [(state.t, *state.mean_m())]
        time_init = state.t
        time_final = time_init + time_in_s
        t_next = time_init + write_every_dt_in_s
        while state.t < time_final:
            self.step(state)
            if state.t >= t_next:
                backstep = t_next - state.t
                if t_next >= time_final - 1e-20:
                    dm, _ = self.RKF45(state, backstep)
                    state.m = state.m + dm
                    state.t += backstep
                    rows.append((state.t, *state.mean_m()))
                    break
                cur = state.copy()
                dm, _ = self.RKF45(cur, backstep)
                cur.m = cur.m + dm
                cur.t += backstep
                rows.append((cur.t, *cur.mean_m()))
                t_next += write_every_dt_in_s
                while t_next < state.t:
                    t_next += write_every_dt_in_s
        return np.array(rows)


# ---------------------------------------------------------------------------
# stochastic Heun  (stochastic_integrator.cpp:8-17, 42-57; stochastic_llg.cpp:19-22)
# ---------------------------------------------------------------------------
def thermal_sigma(alpha, T, dt, Ms, mesh):
    D = (alpha * kb * T) / (gamma * mu0 * Ms * mesh.dx * mesh.dy * mesh.dz)
    return math.sqrt((2.0 * D) / dt)


def heun_step(state, terms, alpha, dt, h_th_prev, h_th):
    """One Heun step with given thermal fields: predictor uses the previous
    step's noise, corrector the new one (stochastic_integrator.cpp:13-15)."""
    k1 = dt * LLG(alpha, state.m, Heff_in_Apm(terms, state) + h_th_prev)
    s2 = state.copy()
    s2.m = state.m + k1
    k2 = dt * LLG(alpha, s2.m, Heff_in_Apm(terms, s2) + h_th)
    state.m = normalize(state.m + (k1 + k2) / 2.0)
    state.t += dt


def semi_implicit_heun_step(state, terms, alpha, dt, h_th_init, h_th):
    """stochastic_integrator.cpp:19-32 with given thermal fields."""
    def f(m, h):
        s = state.copy()
        s.m = m
        return LLG(alpha, m, Heff_in_Apm(terms, s) + h)
    m1 = dt / 2. * f(state.m, h_th_init)
    m2 = dt / 2. * f(state.m + m1, h_th)
    m3 = dt / 2. * f(state.m + m2, h_th)
    m4 = dt / 2. * f(state.m + m3, h_th)
    m5 = dt / 2. * f(state.m + m4, h_th)
    res = dt * f(state.m + m5, h_th)
    state.m = normalize(state.m + res)
    state.t += dt


def det_rk4_step(state, terms, alpha, dt):
    """stochastic_integrator.cpp:34-40 (deterministic RK4 reference)."""
    def f(m):
        s = state.copy()
        s.m = m
        return LLG(alpha, m, Heff_in_Apm(terms, s))
    k1 = dt * f(state.m)
    k2 = dt * f(state.m + 1. / 2. * k1)
    k3 = dt * f(state.m + 1. / 2. * k2)
    k4 = dt * f(state.m + k3)
    state.m = normalize(state.m + (k1 + 2. * k2 + 2. * k3 + k4) / 6.)
    state.t += dt


# ---------------------------------------------------------------------------
# util reductions (util.cpp:30-55)
# ---------------------------------------------------------------------------
def FrobeniusNorm(a):
    return math.sqrt(float(np.mean(a * a)))


def full_inner_product(a, b):
    return float(np.sum(a * b))


def max_4d_abs(a):
    return float(np.max(np.abs(a)))


def spectral_tensor_from_reduced(Nred: np.ndarray, mesh: Mesh) -> np.ndarray:
    """Expand the device's symmetry-reduced real spectral tensor
    [ncomp][kz][ky][kx] to the full half spectrum [Px/2+1, Py, Pz, 6] that
    DemagField.Nfft holds, using the parities of the components (xy odd in ky,
    xz odd in kz, yz odd in ky and kz).  Setup helper of the timed CPU baseline
    (the oracle's own tensor assembly at 1024^2 x 16 would take far longer than
    the field evaluation being timed)."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    Py, Pz = 2 * ny, nz_exp(nz)
    ky = np.arange(Py)
    kyr = np.where(ky <= ny, ky, Py - ky)
    sy = np.where(ky <= ny, 1.0, -1.0)
    kz = np.arange(Pz)
    if nz > 1:
        kzr = np.where(kz <= nz, kz, Pz - kz)
        sz = np.where(kz <= nz, 1.0, -1.0)
        comps = [(0, 0, 0), (1, 1, 0), (2, 0, 1), (3, 0, 0), (4, 1, 1), (5, 0, 0)]  # (slot, odd y, odd z)
    else:
        kzr = np.zeros(1, dtype=int)
        sz = np.ones(1)
        comps = [(0, 0, 0), (1, 1, 0), (None, 0, 0), (2, 0, 0), (None, 0, 0), (3, 0, 0)]
    out = np.zeros((nx + 1, Py, Pz, 6), dtype=np.complex128)
    for c, (slot, oy, oz) in enumerate(comps):
        if slot is None:
            continue
        blk = Nred[slot][kzr][:, kyr]  # (Pz, Py, nxh)
        sign = np.ones((Pz, Py))
        if oy:
            sign = sign * sy[None, :]
        if oz:
            sign = sign * sz[:, None]
        out[..., c] = (blk * sign[..., None]).transpose(2, 1, 0)
    return out
