"""ctypes wrapper of ``oracle/brkga_oracle.c`` — test infrastructure only.

The C file restates the reference's sequential decoder (placement.py,
binClassNew.py, numba_utils.py, collision_backend.py; file:line citations
in the C source).  It is built with plain gcc into ``oracle/liboracle.so``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

from brkga_fft2_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "brkga_oracle.c")
HDR = os.path.join(os.path.dirname(HERE), "include", "brkga_b200.h")
LIB = os.path.join(HERE, "liboracle.so")
_lock = threading.Lock()
_lib = None


def oracle_lib_path() -> str:
    return LIB


def build_oracle(force: bool = False) -> str:
    """Compile the oracle with gcc (-O2, pthreads) unless it is up to date."""
    with _lock:
        newest = max(os.path.getmtime(SRC), os.path.getmtime(HDR))
        if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
            tmp = LIB + f".tmp{os.getpid()}"
            cmd = ["gcc", "-O2", "-std=c11", "-shared", "-fPIC", "-pthread", "-o", tmp, SRC, "-lm"]
            subprocess.run(cmd, check=True)
            os.replace(tmp, LIB)
    return LIB


def _load():
    global _lib
    if _lib is None:
        build_oracle()
        lib = ctypes.CDLL(LIB)
        lib.oracle_decode.restype = ctypes.c_int
        lib.oracle_decode.argtypes = [ctypes.POINTER(abi.BrkgaProblemDesc), ctypes.POINTER(ctypes.c_float),
                                      ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p,
                                      ctypes.c_int]
        _lib = lib
    return _lib


def oracle_decode(packed, chromosomes: np.ndarray, n_threads: int = 1, with_log: bool = False):
    """Decode host chromosomes [P, 2N] with the CPU oracle.

    Returns ``makespans`` (float64 [P]) or ``(makespans, log)`` where ``log`` is
    a structured array [P, M, N] of (gene, bin, x, y, rot).
    """
    lib = _load()
    chrom = np.ascontiguousarray(chromosomes, dtype=np.float32)
    if chrom.ndim != 2 or chrom.shape[1] != 2 * packed.n_genes:
        raise ValueError("chromosomes must be [P, 2N] float32")
    P = chrom.shape[0]
    out = np.zeros(P, np.float64)
    log = np.zeros((P, packed.n_machines, packed.n_genes), abi.PLACEMENT_DTYPE) if with_log else None
    st = lib.oracle_decode(ctypes.byref(packed.desc), abi.ptr(chrom, ctypes.c_float), P,
                           abi.ptr(out, ctypes.c_double),
                           log.ctypes.data_as(ctypes.c_void_p) if with_log else None, int(n_threads))
    abi.check(st, "oracle_decode")
    return (out, log) if with_log else out


def oracle_initial_solution(packed, order):
    """Greedy initial placements on the CPU (oracle_initial_solution in brkga_oracle.c)."""
    lib = _load()
    if not hasattr(lib, "_init_sol_declared"):
        lib.oracle_initial_solution.restype = ctypes.c_int
        lib.oracle_initial_solution.argtypes = [ctypes.POINTER(abi.BrkgaProblemDesc), ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib._init_sol_declared = True
    order = np.ascontiguousarray(order, dtype=np.int32)
    n = order.size
    machine = np.zeros(max(n, 1), np.int32)
    place = np.zeros(max(n, 1), abi.PLACEMENT_DTYPE)
    mk = np.zeros(packed.n_machines, np.float64)
    st = lib.oracle_initial_solution(ctypes.byref(packed.desc), order.ctypes.data_as(ctypes.c_void_p), n,
                                     machine.ctypes.data_as(ctypes.c_void_p), place.ctypes.data_as(ctypes.c_void_p),
                                     mk.ctypes.data_as(ctypes.c_void_p))
    abi.check(st, "oracle_initial_solution")
    return machine[:n], place[:n], mk
