"""Checkpoint and exchange formats (magnumaf/io.py) on the CPU: VTI and ASCII
round trips, and VTI files laid out the way VTK's own XML writer lays them out
(appended raw data, zlib-compressed blocks, UInt32 headers)."""
import base64
import os
import struct
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "magnum.af_b200", "python"))
from magnumaf import io  # noqa: E402


def _field(shape=(5, 4, 3, 3), seed=0):
    return np.random.default_rng(seed).normal(size=shape)


def test_vti_roundtrip(tmp_path):
    a = _field()
    fn = io.write_vti(a, 1e-9, 2e-9, 3e-9, str(tmp_path / "m"))
    assert fn.endswith(".vti")
    b, sp = io.read_vti(fn)
    assert np.array_equal(a, b) and sp == (1e-9, 2e-9, 3e-9)


def test_vti_scalar_field_roundtrip(tmp_path):
    a = _field((6, 2, 1))
    b, _ = io.read_vti(io.write_vti(a, 1.0, 1.0, 1.0, str(tmp_path / "s.vti")))
    assert np.array_equal(a[..., None], b)


def _vtk_style(a, path, compressed, header="UInt32"):
    nx, ny, nz, n = a.shape
    raw = np.transpose(a, (2, 1, 0, 3)).reshape(-1).astype("<f8").tobytes()
    h = "<I" if header == "UInt32" else "<Q"
    if compressed:
        bs = 1000
        blocks = [raw[i:i + bs] for i in range(0, len(raw), bs)]
        comp = [zlib.compress(b) for b in blocks]
        blob = struct.pack("<" + h[-1] * (3 + len(comp)), len(comp), bs, len(blocks[-1]), *[len(c) for c in comp])
        blob += b"".join(comp)
    else:
        blob = struct.pack(h, len(raw)) + raw
    comp_attr = ' compressor="vtkZLibDataCompressor"' if compressed else ""
    xml = ('<?xml version="1.0"?>\n<VTKFile type="ImageData" version="1.0" byte_order="LittleEndian" '
           'header_type="%s"%s>\n<ImageData WholeExtent="0 %d 0 %d 0 %d" Origin="0 0 0" Spacing="2e-09 2e-09 1e-09">\n'
           '<Piece Extent="0 %d 0 %d 0 %d"><PointData/><CellData Scalars="ImageScalars">\n'
           '<DataArray type="Float64" Name="ImageScalars" NumberOfComponents="%d" format="appended" '
           'RangeMin="0" RangeMax="1" offset="0"/>\n</CellData></Piece></ImageData>\n'
           '<AppendedData encoding="raw">\n_' % (header, comp_attr, nx, ny, nz, nx, ny, nz, n))
    with open(path, "wb") as f:
        f.write(xml.encode() + blob + b"\n</AppendedData>\n</VTKFile>\n")


def test_vti_reads_vtk_writer_layouts(tmp_path):
    a = _field((7, 5, 2, 3), 3)
    for compressed in (False, True):
        for header in ("UInt32", "UInt64"):
            p = str(tmp_path / ("v_%d_%s.vti" % (compressed, header)))
            _vtk_style(a, p, compressed, header)
            b, sp = io.read_vti(p)
            assert np.array_equal(a, b) and sp == (2e-9, 2e-9, 1e-9)


def test_ascii_roundtrip(tmp_path):
    a = _field((4, 3, 2, 3), 5)
    p = str(tmp_path / "m.dat")
    io.write_ascii(a, 1e-9, 2e-9, 3e-9, p, precision=17)
    b, sp = io.read_ascii(p)
    assert np.array_equal(a, b) and sp == (1e-9, 2e-9, 3e-9)
    with open(p) as f:
        assert f.readline().split()[1:5] == ["4", "3", "2", "3"]
