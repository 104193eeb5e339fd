"""Threaded evaluation of the FP64 oracle's effective field, for the timed CPU
baseline at the benchmark's full mesh.

Test infrastructure: only tests/ and bench.py's CPU legs use it.  The
arithmetic is maf_oracle's, element for element; only the work is split over
host threads (NumPy releases the GIL inside its array operations):

* the demag convolution (maf_oracle.DemagField.H_in_Apm, the reference's
  demag_field.cpp:215-264) runs its FFTs with scipy.fft workers and its
  3 x 3 tensor product on slabs of kx;
* local field terms (exchange, anisotropies, Zeeman, ...) are evaluated on slabs
  of y rows with a one-row halo on each side -- their stencils reach one cell,
  so every kept row sees its true neighbours -- and the halo rows are dropped;
* the terms are summed in list order (field_term.hpp:116-119), slab by slab.
"""
from __future__ import annotations

import concurrent.futures as cf
import os

import numpy as np

import maf_oracle as O


def _pool(workers):
    return cf.ThreadPoolExecutor(max_workers=workers)


def _spans(n, parts):
    parts = max(1, min(n, parts))
    edges = np.linspace(0, n, parts + 1).astype(int)
    return [(int(a), int(b)) for a, b in zip(edges[:-1], edges[1:]) if b > a]


def _sub_state(state, y0, y1):
    """State over rows [y0, y1) of the mesh (views, no renormalisation)."""
    mesh = state.mesh
    sub = O.State.__new__(O.State)
    sub.mesh = O.Mesh(mesh.nx, y1 - y0, mesh.nz, mesh.dx, mesh.dy, mesh.dz)
    sub.m = state.m[:, y0:y1]
    sub.t, sub.steps = state.t, state.steps
    sub.Ms = state.Ms
    sub.Ms_field = None if state.Ms_field is None else state.Ms_field[:, y0:y1]
    return sub


def _local_into(term, state, out, ex, parts):
    ny = state.mesh.ny

    def one(span):
        y0, y1 = span
        lo, hi = max(0, y0 - 1), min(ny, y1 + 1)
        h = term.H_in_Apm(_sub_state(state, lo, hi))
        out[:, y0:y1] = h[:, y0 - lo:y0 - lo + (y1 - y0)]

    list(ex.map(one, _spans(ny, parts)))


def _demag_into(term, state, out, ex, parts, workers):
    nx, ny, nz = state.mesh.nx, state.mesh.ny, state.mesh.nz
    old = O.FFT_WORKERS
    O.FFT_WORKERS = workers
    try:
        Msm = state.m * state.Ms_v()
        mfft = O._rfft3(Msm, term.P)
        del Msm
        N = term.Nfft
        hfft = np.empty_like(mfft)

        def prod(span):
            a, b = span
            n, mf, hf = N[a:b], mfft[a:b], hfft[a:b]
            hf[..., 0] = n[..., 0] * mf[..., 0] + n[..., 1] * mf[..., 1] + n[..., 2] * mf[..., 2]
            hf[..., 1] = n[..., 1] * mf[..., 0] + n[..., 3] * mf[..., 1] + n[..., 4] * mf[..., 2]
            hf[..., 2] = n[..., 2] * mf[..., 0] + n[..., 4] * mf[..., 1] + n[..., 5] * mf[..., 2]

        list(ex.map(prod, _spans(mfft.shape[0], parts)))
        del mfft
        h = O._irfft3(hfft, term.P)
        del hfft

        def crop(span):
            y0, y1 = span
            out[:, y0:y1] = h[:nx, y0:y1, :nz, :]

        list(ex.map(crop, _spans(ny, parts)))
    finally:
        O.FFT_WORKERS = old


def _splittable(term):
    """Terms whose field at a cell depends only on m within one cell of it and on
    scalar parameters (a per-cell parameter array would need slicing too)."""
    if isinstance(term, (O.ExchangeField, O.CubicAnisotropyField)):
        return True
    if isinstance(term, O.ExternalField):
        return term.zee.ndim == 1
    return False


def heff_in_apm(terms, state, workers=None):
    """maf_oracle.Heff_in_Apm(terms, state) on `workers` host threads."""
    workers = workers or os.cpu_count() or 1
    parts = 4 * workers
    shape = state.m.shape
    total = None
    with _pool(workers) as ex:
        for term in terms:
            h = np.empty(shape)
            if isinstance(term, O.DemagField):
                _demag_into(term, state, h, ex, parts, workers)
            elif _splittable(term):
                _local_into(term, state, h, ex, parts)
            else:
                h[...] = term.H_in_Apm(state)
            if total is None:
                total = h
            else:
                def add(span, total=total, h=h):
                    y0, y1 = span
                    total[:, y0:y1] += h[:, y0:y1]

                list(ex.map(add, _spans(shape[1], parts)))
    return total
