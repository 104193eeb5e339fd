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


def _build(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "sp4")
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), SRC, "-L" + LIBDIR, "-lmafb200",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_example_compiles(tmp_path):
    _build(tmp_path)


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
