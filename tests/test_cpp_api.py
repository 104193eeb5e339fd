"""The C++ host interface (include/magnumaf_b200.hpp) compiles reference-style
host code: the muMAG SP4 example written like magnumaf/examples/sp4.cpp.  On a
GPU it reproduces the reference's SP4 golden integrals (python/test/sp4.py)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "magnum.af_b200", "examples", "sp4.cpp")
LIBDIR = os.path.join(ROOT, "magnum.af_b200", "lib")


TERMS_SRC = os.path.join(ROOT, "magnum.af_b200", "examples", "field_terms.cpp")


def _build(tmp_path, src=SRC, name="sp4"):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / name)
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), src, "-L" + LIBDIR, "-lmafb200",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_example_compiles(tmp_path):
    _build(tmp_path)
    _build(tmp_path, TERMS_SRC, "field_terms")


@pytest.mark.gpu
def test_cpp_field_terms(tmp_path):
    """The further terms through the C++ classes: for a uniform m the periodic
    demag (only the k = 0 mode, which is dropped) and both exchange forms with
    a diagonal vanish exactly; the two-domain m gives fields and energies that
    match the Python API on the same library."""
    import numpy as np

    exe = _build(tmp_path, TERMS_SRC, "field_terms")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = {line.split()[0]: [float(v) for v in line.split()[1:]] for line in r.stdout.splitlines()}
    assert got["DemagFieldPBC"][0] <= 1e-9 * 8e5
    assert got["SparseExchangeField"][0] == 0.0 and got["ExchangeFieldPBC"][0] == 0.0
    assert got["SpinTransferTorqueField"][0] > 0.0
    import magnumaf as M

    nx, ny, nz = 16, 8, 4
    mesh = M.Mesh(nx, ny, nz, 2e-9, 2e-9, 2e-9)
    m = np.zeros((nx, ny, nz, 3))
    m[..., 2] = np.where(np.arange(nz) < nz // 2, -1.0, 1.0)[None, None, :]
    s = M.State(mesh, 8e5, m)
    pol = np.zeros((nx, ny, nz, 3))
    pol[..., 0] = 1.0
    py = {"DemagFieldPBC": M.DemagFieldPBC(),
          "SparseExchangeField": M.SparseExchangeField(np.full((nx, ny, nz), 1.3e-11), mesh),
          "ExchangeFieldPBC": M.ExchangeFieldPBC(1.3e-11, mesh),
          "SpinTransferTorqueField": M.SpinTransferTorqueField(pol, 0.3, 0.1, 2e10, 1e-9)}
    for name, t in py.items():
        assert got[name][1] == float(np.abs(t.H_in_Apm(s)).max()), name
        assert got[name][2] == t.Energy_in_J(s), name


@pytest.mark.gpu
def test_cpp_sp4_golden(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe, str(tmp_path / "m.dat")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    vals = {}
    for line in r.stdout.splitlines():
        k, *v = line.split()
        vals[k] = [float(x) for x in v]
    for got, want in zip(vals["relax"], (9.81206172824e-10, 9.14350283169e-11, -5.74381785359e-13)):
        assert abs(got - want) < 1e-15
    for got, want in zip(vals["switch"], (-6.41261165705e-10, 1.47353233738e-10, -1.78144535231e-11)):
        assert abs(got - want) < 1e-15
    rows = open(tmp_path / "m.dat").read().splitlines()
    assert len(rows) > 1000
