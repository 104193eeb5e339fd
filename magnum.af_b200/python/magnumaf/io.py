"""Checkpoint and exchange formats of magnum.af, on the host (NumPy).

* VTK XML ImageData (.vti), the reference's vti_writer_micro / vti_reader
  (magnumaf/src/util/vtk_io.cpp:52-118, 178-255): a cell-centred image of
  (nx+1) x (ny+1) x (nz+1) points, origin 0, spacing (dx, dy, dz), one
  Float64 cell array "ImageScalars" with one tuple per cell, x fastest.
  The writer emits base64 "binary" data (readable by ParaView/VTK); the reader
  also takes "ascii" and "appended" data, raw or zlib-compressed, with UInt32
  or UInt64 block headers -- what VTK's own writer produces.
* The ASCII format of write_ascii / read_ascii
  (magnumaf/src/util/ascii_io.cpp:17-159): a header "# nx ny nz n dx dy dz",
  comment lines, then one line per cell, ix outer, iz inner, with the cell's
  position and its n values.
* Integrator checkpoints: m, t, steps and the step-size controller state in one
  .npz file, so an adaptive run resumes with the same next step size.

Arrays are (nx, ny, nz, n) like the rest of the Python API.
"""
from __future__ import annotations

import base64
import struct
import xml.etree.ElementTree as ET
import zlib
from typing import Tuple

import numpy as np


# --------------------------------------------------------------------- VTI
def write_vti(a: np.ndarray, dx: float, dy: float, dz: float, filename: str) -> str:
    """Util.write_vti(array, dx, dy, dz, filename); returns the file name written
    ('.vti' is appended unless present, vtk_io.cpp:86-87)."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 3:
        a = a[..., None]
    nx, ny, nz, n = a.shape
    fn = filename if filename.endswith(".vti") else filename + ".vti"
    # tuples in cell order (x fastest), components interleaved
    flat = np.transpose(a, (2, 1, 0, 3)).reshape(-1).astype("<f8")
    raw = flat.tobytes()
    blob = base64.b64encode(struct.pack("<Q", len(raw)) + raw).decode("ascii")
    with open(fn, "w") as f:
        f.write('<?xml version="1.0"?>\n')
        f.write('<VTKFile type="ImageData" version="1.0" byte_order="LittleEndian" header_type="UInt64">\n')
        f.write('  <ImageData WholeExtent="0 %d 0 %d 0 %d" Origin="0 0 0" Spacing="%r %r %r">\n'
                % (nx, ny, nz, float(dx), float(dy), float(dz)))
        f.write('    <Piece Extent="0 %d 0 %d 0 %d">\n' % (nx, ny, nz))
        f.write('      <PointData>\n      </PointData>\n')
        f.write('      <CellData Scalars="ImageScalars">\n')
        f.write('        <DataArray type="Float64" Name="ImageScalars" NumberOfComponents="%d" format="binary">\n'
                % n)
        f.write("          " + blob + "\n")
        f.write("        </DataArray>\n      </CellData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n")
    return fn


_TYPES = {"Float64": "<f8", "Float32": "<f4", "Int32": "<i4", "Int64": "<i8", "UInt8": "u1", "UInt32": "<u4",
          "UInt64": "<u8"}


def _decode_blocks(data: bytes, pos: int, hdr: str, compressed: bool) -> Tuple[bytes, int]:
    """One binary data block at data[pos:]: [size] raw, or the compressed layout
    [nblocks, blocksize, lastsize, csize_0..] followed by the zlib blocks."""
    hs = struct.calcsize(hdr)
    w = hdr[-1]  # 'I' (UInt32) or 'Q' (UInt64), little-endian
    if not compressed:
        (size,) = struct.unpack_from(hdr, data, pos)
        pos += hs
        return data[pos:pos + size], pos + size
    (nb,) = struct.unpack_from(hdr, data, pos)
    blocksize, lastsize = struct.unpack_from("<" + w * 2, data, pos + hs)
    csizes = struct.unpack_from("<" + w * nb, data, pos + 3 * hs)
    pos += (3 + nb) * hs
    out = bytearray()
    for c in csizes:
        out += zlib.decompress(data[pos:pos + c])
        pos += c
    return bytes(out), pos


def read_vti(filename: str):
    """vti_reader: returns (array (nx, ny, nz, n), (dx, dy, dz))."""
    text = open(filename, "rb").read()
    # appended raw data follows '<AppendedData encoding="raw">' and a '_' marker
    appended = None
    k = text.find(b"<AppendedData")
    if k >= 0:
        u = text.find(b"_", text.find(b">", k)) + 1
        appended = text[u:]
        xml_part = text[:k] + b"</VTKFile>"
        enc = b'encoding="base64"' in text[k:u]
    else:
        xml_part = text
        enc = False
    root = ET.fromstring(xml_part)
    hdr = "<Q" if root.get("header_type", "UInt32") == "UInt64" else "<I"
    compressed = root.get("compressor") is not None
    if root.get("byte_order", "LittleEndian") != "LittleEndian":
        raise ValueError("read_vti: only little-endian files are supported")
    img = root.find("ImageData")
    ext = [int(v) for v in img.get("WholeExtent").split()]
    nx, ny, nz = ext[1] - ext[0], ext[3] - ext[2], ext[5] - ext[4]
    spacing = tuple(float(v) for v in img.get("Spacing").split())
    arr = img.find("Piece/CellData/DataArray")
    if arr is None:
        raise ValueError("read_vti: no cell data")
    n = int(arr.get("NumberOfComponents", "1"))
    dt = np.dtype(_TYPES[arr.get("type")])
    fmt = arr.get("format")
    if fmt == "ascii":
        vals = np.array(arr.text.split(), dtype=np.float64)
    elif fmt == "binary":
        raw = base64.b64decode("".join(arr.text.split()))
        if compressed:
            body, _ = _decode_blocks(raw, 0, hdr, True)
        else:
            body, _ = _decode_blocks(raw, 0, hdr, False)
        vals = np.frombuffer(body, dtype=dt).astype(np.float64)
    elif fmt == "appended":
        off = int(arr.get("offset", "0"))
        data = appended
        if enc:
            data = base64.b64decode(data.split(b"</AppendedData>")[0].strip())
        body, _ = _decode_blocks(data, off, hdr, compressed)
        vals = np.frombuffer(body, dtype=dt).astype(np.float64)
    else:
        raise ValueError("read_vti: unknown data format %r" % fmt)
    a = vals[: nx * ny * nz * n].reshape(nz, ny, nx, n).transpose(2, 1, 0, 3)
    return np.ascontiguousarray(a), spacing


# ------------------------------------------------------------------- ASCII
def write_ascii(a: np.ndarray, dx: float, dy: float, dz: float, filename: str, precision: int = 12):
    """write_ascii (ascii_io.cpp:17-94)."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 3:
        a = a[..., None]
    nx, ny, nz, n = a.shape
    w = precision + 4
    with open(filename, "w") as f:
        f.write("# %d %d %d %d %r %r %r\n" % (nx, ny, nz, n, float(dx), float(dy), float(dz)))
        f.write("# magnum.af ascii-encoded %dd spacial field\n" % n)
        f.write("#\n")
        cols = ["# x-position[m]", "y-position[m]", "z-position[m]"]
        cols += ["mx[a.u.]", "my[a.u.]", "mz[a.u.]"] if n == 3 else ["%d-component" % i for i in range(n)]
        f.write("\t".join(c.ljust(w) for c in cols).rstrip() + "\n")
        fmt = "%-" + str(w) + "." + str(precision) + "g"
        for ix in range(nx):
            for iy in range(ny):
                for iz in range(nz):
                    vals = [ix * dx, iy * dy, iz * dz] + list(a[ix, iy, iz])
                    f.write("\t".join(fmt % v for v in vals) + "\n")


def read_ascii(filename: str):
    """read_ascii (ascii_io.cpp:95-157): returns (array (nx, ny, nz, n), (dx, dy, dz))."""
    with open(filename) as f:
        head = f.readline()[2:].split()
        nx, ny, nz, n = (int(v) for v in head[:4])
        dx, dy, dz = (float(v) for v in head[4:7])
        rows = [line.split() for line in f if line.strip() and not line.startswith("#")]
    vals = np.array([[float(v) for v in r[3:3 + n]] for r in rows], dtype=np.float64)
    if vals.shape[0] != nx * ny * nz:
        raise ValueError("read_ascii: %d cells in the file, header says %d" % (vals.shape[0], nx * ny * nz))
    return vals.reshape(nx, ny, nz, n), (dx, dy, dz)


# -------------------------------------------------------------- checkpoint
def save_checkpoint(filename: str, state, llg=None):
    """m, t and steps of a State, plus the integrator's step size and controller
    state when llg (an LLGIntegrator) is given."""
    data = {"m": np.asarray(state.m), "t": state.t, "steps": state.steps,
            "mesh": np.array([state.mesh.nx, state.mesh.ny, state.mesh.nz, state.mesh.dx, state.mesh.dy,
                              state.mesh.dz])}
    if llg is not None:
        data["controller"] = np.array(llg.controller_state(), dtype=np.float64)
    np.savez(filename, **data)


def load_checkpoint(filename: str, state, llg=None):
    """Restores what save_checkpoint wrote into an existing State of the same mesh
    (and LLGIntegrator)."""
    d = np.load(filename if filename.endswith(".npz") else filename + ".npz")
    mesh = d["mesh"]
    if tuple(int(v) for v in mesh[:3]) != (state.mesh.nx, state.mesh.ny, state.mesh.nz):
        raise ValueError("load_checkpoint: mesh differs")
    state.load_m(d["m"])  # bit-exact: no normalisation
    state.t = float(d["t"])
    state.steps = int(d["steps"])
    if llg is not None and "controller" in d:
        llg.set_controller_state(d["controller"].tolist())
