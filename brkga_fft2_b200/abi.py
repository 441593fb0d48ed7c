"""ctypes mirror of ``include/brkga_b200.h`` (structs, status codes, loader).

Only plain ctypes: the shared library ``libbrkga_b200.so`` is built in-tree
by :mod:`brkga_fft2_b200.build` and loaded from the package directory.  The
loader raises when the library is missing — there is no fallback path.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

ABI_VERSION = 1
NOALLOC_SCRATCH_BYTES = 64 << 20  # BRKGA_NOALLOC_SCRATCH_BYTES
MAX_INSTANCES = 64  # BRKGA_MAX_INSTANCES

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_BAD_INSTANCE = 2
ERR_CUDA = 3
ERR_WORKSPACE = 4
ERR_CAPACITY = 5
ERR_NEW_BIN_UNFIT = 6
ERR_NO_DEVICE = 7
ERR_INTERNAL = 8

STATUS_NAMES = {
    OK: "ok",
    ERR_INVALID_ARGUMENT: "invalid argument",
    ERR_BAD_INSTANCE: "bad instance",
    ERR_CUDA: "CUDA error",
    ERR_WORKSPACE: "workspace too small",
    ERR_CAPACITY: "bin pool exhausted",
    ERR_NEW_BIN_UNFIT: "new plate received a rotation that does not fit",
    ERR_NO_DEVICE: "no CUDA device",
    ERR_INTERNAL: "device consistency check failed",
}


class BrkgaError(RuntimeError):
    """A non-zero BrkgaStatus returned by the native library."""

    def __init__(self, status: int, what: str = ""):
        self.status = int(status)
        msg = STATUS_NAMES.get(self.status, f"status {status}")
        super().__init__(f"{what}: {msg}" if what else msg)


class BrkgaProblemDesc(ctypes.Structure):
    _fields_ = [
        ("n_genes", ctypes.c_int32),
        ("n_machines", ctypes.c_int32),
        ("n_types", ctypes.c_int32),
        ("threshold_mode", ctypes.c_int32),
        ("gene_type", ctypes.POINTER(ctypes.c_int32)),
        ("thresholds", ctypes.POINTER(ctypes.c_double)),
        ("bin_length", ctypes.POINTER(ctypes.c_int32)),
        ("bin_width", ctypes.POINTER(ctypes.c_int32)),
        ("bin_area", ctypes.POINTER(ctypes.c_double)),
        ("setup_time", ctypes.POINTER(ctypes.c_double)),
        ("proc_time", ctypes.POINTER(ctypes.c_double)),
        ("proc_time_height", ctypes.POINTER(ctypes.c_double)),
        ("part_area", ctypes.POINTER(ctypes.c_double)),
        ("part_nrot", ctypes.POINTER(ctypes.c_int32)),
        ("part_best_rot", ctypes.POINTER(ctypes.c_int32)),
        ("rot_h", ctypes.POINTER(ctypes.c_int32)),
        ("rot_w", ctypes.POINTER(ctypes.c_int32)),
        ("rot_mask_offset", ctypes.POINTER(ctypes.c_int64)),
        ("masks", ctypes.POINTER(ctypes.c_uint8)),
        ("masks_bytes", ctypes.c_int64),
    ]


class BrkgaPlacement(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("gene", "bin", "x", "y", "rot")]


COLLISION_BITSET = 0
COLLISION_INT8_TC = 1
# BrkgaChunkTest: plate, out (device pointers), machine, part_type, rot, ty_hi
CHUNK_TEST_DTYPE = np.dtype([("plate", "<u8"), ("out", "<u8"), ("machine", "<i4"), ("part_type", "<i4"),
                             ("rot", "<i4"), ("ty_hi", "<i4")])

PLACEMENT_DTYPE = np.dtype([("gene", "<i4"), ("bin", "<i4"), ("x", "<i4"), ("y", "<i4"), ("rot", "<i4")])


def ptr(arr: np.ndarray, ctype):
    if not arr.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return arr.ctypes.data_as(ctypes.POINTER(ctype))


PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libbrkga_b200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)

_lib = None


def load_library(path: str = LIB_PATH):
    """Load ``libbrkga_b200.so`` and declare its entry points.

    Raises ``RuntimeError`` when the library has not been built: the decoder
    has no CPU fallback.
    """
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build the CUDA library first "
            "(python -m brkga_fft2_b200.build); there is no CPU fallback")
    lib = ctypes.CDLL(path)
    c_int, c_i32, c_i64, c_sz, vp = ctypes.c_int, ctypes.c_int32, ctypes.c_int64, ctypes.c_size_t, ctypes.c_void_p
    P = ctypes.POINTER
    sig = {
        "brkga_abi_version": (c_int, []),
        "brkga_status_string": (ctypes.c_char_p, [c_int]),
        "brkga_build_id": (ctypes.c_char_p, []),
        "brkga_problem_create": (c_int, [P(BrkgaProblemDesc), P(vp)]),
        "brkga_problem_destroy": (None, [vp]),
        "brkga_workspace_bytes": (c_int, [vp, c_i32, c_i64, P(c_sz)]),
        "brkga_decode": (c_int, [vp, vp, c_i32, vp, vp, vp, vp, c_sz, c_i64, vp]),
        "brkga_decode_stage": (c_int, [c_i32, vp, vp, c_i32, vp, vp, vp, vp, c_sz, c_i64, vp]),
        "brkga_decode_noalloc": (c_int, [vp, vp, c_i32, vp, vp, vp, vp]),
        "brkga_initial_solution_host": (c_int, [vp, vp, c_i32, vp, vp, vp]),
        "brkga_ga_init_population": (c_int, [vp, c_i32, c_i32, ctypes.c_uint64, c_i32, vp]),
        "brkga_ga_rank": (c_int, [vp, c_i32, vp, vp]),
        "brkga_ga_breed": (c_int, [vp, vp, vp, c_i32, c_i32, c_i32, c_i32, ctypes.c_float, ctypes.c_uint64, vp, vp,
                                   vp, vp]),
        "brkga_ga_breed_pool": (c_int, [vp, vp, vp, c_i32, c_i32, c_i32, c_i32, c_i32, ctypes.c_float,
                                        ctypes.c_uint64, vp, vp, vp, vp]),
        "brkga_ga_breed_families": (c_int, [vp, vp, vp, c_i32, c_i32, c_i32, c_i32, c_i32, c_i32, ctypes.c_float,
                                            ctypes.c_uint64, vp, vp, vp, vp]),
        "brkga_ga_select_families": (c_int, [vp, c_i32, c_i32, vp, vp]),
        "brkga_ga_gather": (c_int, [vp, vp, c_i32, c_i32, vp, vp]),
        "brkga_ga_screen_stats": (c_int, [vp, vp, vp, vp, c_i32, vp, vp, c_i32, vp, vp]),
        "brkga_ga_track": (c_int, [vp, vp, c_i32, c_i32, vp, vp, c_i32, vp, vp, vp]),
        "brkga_ga_audit": (c_int, [vp, vp, vp, c_i32, c_i32, vp, c_i32, vp, vp, vp]),
        "brkga_gemm_bf16": (c_int, [vp, c_i32, vp, c_i32, vp, c_i32, c_i32, c_i32, c_i32, vp, vp]),
        "brkga_surrogate_create": (c_int, [vp, c_i32, c_i32, ctypes.c_uint64, P(vp)]),
        "brkga_surrogate_create_ex": (c_int, [vp, c_i32, c_i32, ctypes.c_uint64, c_i32, P(vp)]),
        "brkga_surrogate_destroy": (None, [vp]),
        "brkga_surrogate_reset": (c_int, [vp]),
        "brkga_surrogate_dims": (c_int, [vp, P(c_i32), P(c_i32), P(c_i64)]),
        "brkga_surrogate_predict": (c_int, [vp, vp, c_i32, vp, vp]),
        "brkga_surrogate_observe": (c_int, [vp, vp, vp, c_i32, vp]),
        "brkga_surrogate_train": (c_int, [vp, c_i32, c_i32, ctypes.c_float, vp]),
        "brkga_surrogate_features": (c_int, [vp, vp, c_i32, vp]),
        "brkga_surrogate_load_batch": (c_int, [vp, vp, vp, c_i32, c_i32, vp]),
        "brkga_surrogate_gradients": (c_int, [vp, c_i32, vp]),
        "brkga_surrogate_adam": (c_int, [vp, ctypes.c_float, vp]),
        "brkga_surrogate_buffers": (c_int, [vp, vp, vp, vp, vp, vp, vp, vp]),
        "brkga_surrogate_io": (c_int, [vp, c_i32, vp, c_i64, c_i32]),
        "brkga_problem_create_multi": (c_int, [P(BrkgaProblemDesc), c_i32, P(vp)]),
        "brkga_problem_instances": (c_int, [vp, P(c_i32)]),
        "brkga_workspace_bytes_multi": (c_int, [vp, P(c_i32), c_i64, P(c_sz)]),
        "brkga_decode_multi": (c_int, [vp, vp, P(c_i32), vp, vp, vp, vp, c_sz, c_i64, vp]),
        "brkga_decode_multi_stage": (c_int, [c_i32, vp, vp, P(c_i32), vp, vp, vp, vp, c_sz, c_i64, vp]),
        "brkga_decode_multi_at": (c_int, [c_i32, vp, vp, P(c_i64), P(c_i32), vp, P(c_i64), vp, vp, vp, c_sz, c_i64,
                                          vp]),
        "brkga_set_launch_config": (c_int, [vp, c_i32, c_i32, c_i32, c_i32]),
        "brkga_get_launch_config": (c_int, [vp, c_i64, P(c_i32), P(c_i32), P(c_i32), P(c_i32), P(c_i32)]),
        "brkga_evaluate_host": (c_int, [vp, P(ctypes.c_float), c_i32, P(ctypes.c_double), vp]),
        "brkga_last_counters": (c_int, [vp, P(c_i64), P(c_i64), P(c_i64), P(c_i64)]),
        "brkga_probe_smem_stream": (c_int, [c_i32, c_i32, c_i32, vp, vp, vp]),
        "brkga_chunk_free": (c_int, [vp, c_i32, vp, c_i32, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.brkga_abi_version() != ABI_VERSION:
        raise RuntimeError("libbrkga_b200.so ABI version mismatch; rebuild it")
    if path == LIB_PATH:
        from .build import build_id
        have, want = lib.brkga_build_id().decode(), build_id()
        if have != want:
            raise RuntimeError(f"{path} was built from other sources (build id {have}, the tree's is {want}); "
                               "rebuild it (python -m brkga_fft2_b200.build)")
    _lib = lib
    return lib


def library_build_id() -> str:
    """Build id compiled into the loaded library (hash of its sources and flags)."""
    return load_library().brkga_build_id().decode()


def check(status: int, what: str = "") -> None:
    if status != OK:
        raise BrkgaError(status, what)
