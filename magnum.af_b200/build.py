"""Build libmafb200.so (sm_100a) in-tree: magnum.af_b200/lib/libmafb200.so.

    python magnum.af_b200/build.py [--force]

Every translation unit is compiled by nvcc for `-gencode arch=compute_100a,code=sm_100a`
with -lineinfo; the Newell tensor file is compiled with -fmad=false so that its
cancellation-prone sums are not contracted into multiply-adds.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libmafb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + INCLUDE]
# object name -> (source, extra nvcc options); fields_ct.cu is compiled once per
# group of its template instantiations (see the end of that file) so that the
# groups build in parallel
SOURCES = {
    "fields.o": ("fields.cu", []),
    "llg.o": ("llg.cu", []),
    "newell.o": ("newell.cu", ["-fmad=false"]),
    "capi.o": ("capi.cu", []),
    "noalloc.o": ("noalloc.cu", []),
    "cnn.o": ("cnn.cu", []),
    "batch.o": ("batch.cu", []),
    "umma.o": ("umma.cu", []),
    "nn.o": ("nn.cu", []),
}
for _part in (1, 2, 3):
    for _real in (4, 8):
        SOURCES["fields_ct_%d_%d.o" % (_part, _real)] = (
            "fields_ct.cu", ["-DMAF_CT_PART=%d" % _part, "-DMAF_CT_REAL=%d" % _real])


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps_mtime() -> float:
    mt = 0.0
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            mt = max(mt, os.path.getmtime(os.path.join(d, f)))
    return max(mt, os.path.getmtime(__file__))


def _headers_mtime() -> float:
    """Newest header (csrc/*.cuh, *.hpp, include/*) or this script."""
    mt = os.path.getmtime(__file__)
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if not f.endswith(".cu"):
                mt = max(mt, os.path.getmtime(os.path.join(d, f)))
    return mt


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps_mtime():
        return LIB
    nv = nvcc()
    hdr = _headers_mtime()
    user = os.environ.get("MAF_NVCC_EXTRA", "")

    def compile_one(item):
        objname, (src, extra) = item
        obj = os.path.join(OBJDIR, objname)
        # an object is rebuilt when its source, a header or this script is newer
        # (always with --force or extra user options)
        if (not force and not user and os.path.exists(obj)
                and os.path.getmtime(obj) >= max(hdr, os.path.getmtime(os.path.join(CSRC, src)))):
            return obj
        # MAF_NVCC_EXTRA: additional nvcc options, e.g. -DMAF_COLS_TILE_F32=16384 (tile sizes)
        cmd = [nv, *COMMON, *ARCH, *extra, *user.split(), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        return obj

    with ThreadPoolExecutor(max_workers=min(12, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, SOURCES.items()))
    tmp = LIB + ".tmp"
    cmd = [nv, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-cudart", "static", *objs, "-o", tmp]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    sys.exit(0)
