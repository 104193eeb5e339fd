"""The C-ABI library loads and exports every entry point that include/*.h
declares; without a GPU every compute call fails loudly (no CPU path)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "magnum.af_b200", "lib", "libmafb200.so")


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_ ]+\*?\s*\**(maf_[A-Za-z0-9_]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "maf_state_create" in names and "maf_llg_step" in names and "maf_term_demag_create" in names
    assert len(names) >= 40


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_symbol():
    import magnumaf as M
    names = declared_functions()
    assert set(M._SIGS) == set(names)


def test_no_cpu_fallback_without_gpu():
    import magnumaf as M
    if M.device_count() > 0:
        pytest.skip("a GPU is present")
    m = np.zeros((2, 2, 1, 3))
    m[..., 0] = 1
    with pytest.raises(M.MafError) as e:
        M.State(M.Mesh(2, 2, 1, 1e-9, 1e-9, 1e-9), 8e5, m)
    assert e.value.code == 7
    with pytest.raises(M.MafError) as e:
        M.DemagField(M.Mesh(2, 2, 1, 1e-9, 1e-9, 1e-9))
    assert e.value.code == 7
