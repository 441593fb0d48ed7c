"""Build ``libbrkga_b200.so`` in-tree with nvcc for sm_100a.

    python -m brkga_fft2_b200.build [--force] [-v]

The library is plain CUDA C++ behind the C ABI of ``include/brkga_b200.h``
(cudart linked statically), loaded with ctypes by :mod:`brkga_fft2_b200.abi`.

Build identity: the SHA-256 of every source and header together with the
nvcc command line is the build id.  It is compiled into the library
(``brkga_build_id()``) and written beside it (``libbrkga_b200.so.buildid``);
the library is rebuilt whenever the id of the current tree differs from the
stamp, and :func:`brkga_fft2_b200.abi.load_library` refuses a library whose
compiled-in id is not the current tree's.
"""
from __future__ import annotations

import glob
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
SOURCES = sorted(glob.glob(os.path.join(PKG, "csrc", "*.cu")))
HEADERS = sorted(glob.glob(os.path.join(REPO, "include", "*.h"))) + sorted(glob.glob(os.path.join(PKG, "csrc", "*.cuh")))
LIB = os.path.join(PKG, "libbrkga_b200.so")
STAMP = LIB + ".buildid"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-shared"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build_id() -> str:
    """SHA-256 (first 16 hex digits) of the sources, headers and nvcc flags."""
    h = hashlib.sha256()
    for path in SOURCES + HEADERS:
        h.update(os.path.relpath(path, REPO).encode())
        h.update(b"\0")
        with open(path, "rb") as f:
            h.update(f.read())
        h.update(b"\0")
    h.update(" ".join(ARCH + FLAGS).encode())
    return h.hexdigest()[:16]


def decoder_source_id() -> str:
    """Hash (16 hex digits) of what the decode kernel is compiled from: its
    source, the headers it includes and the nvcc flags.  A profile of the
    decode kernel (instruction counts, DRAM bytes) stays valid while this id
    does, whatever else in the library changes."""
    h = hashlib.sha256()
    names = ["brkga_decoder.cu", "corr_i8.cuh", "umma_core.cuh"]
    for path in [os.path.join(PKG, "csrc", n) for n in names] + sorted(glob.glob(os.path.join(REPO, "include", "*.h"))):
        h.update(os.path.relpath(path, REPO).encode())
        h.update(b"\0")
        with open(path, "rb") as f:
            h.update(f.read())
        h.update(b"\0")
    h.update(" ".join(ARCH + FLAGS).encode())
    return h.hexdigest()[:16]


def stamped_id() -> str:
    try:
        with open(STAMP) as f:
            return f.read().strip()
    except OSError:
        return ""


def build(force: bool = False, verbose: bool = False) -> str:
    bid = build_id()
    if not force and os.path.exists(LIB) and stamped_id() == bid:
        return LIB
    tmp = LIB + f".tmp{os.getpid()}"
    cmd = [nvcc(), *ARCH, *FLAGS, f"-DBRKGA_BUILD_ID=\"{bid}\"", "-I", os.path.join(REPO, "include"), "-o", tmp,
           *SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    with open(STAMP + f".tmp{os.getpid()}", "w") as f:
        f.write(bid + "\n")
    os.replace(STAMP + f".tmp{os.getpid()}", STAMP)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
