"""CPU-side checks of the C ABI: the library loads, exports every entry point
declared in include/brkga_b200.h, and validates descriptors before touching a
device.  No decode runs here (no GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from brkga_fft2_b200 import abi, build, instances, pack_problem

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return abi.load_library()


def declared_functions():
    text = open(os.path.join(REPO, "include", "brkga_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(brkga_[a-z_0-9]+)\s*\(", text)))


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert "brkga_decode" in names and "brkga_evaluate_host" in names
    for n in names:
        assert hasattr(lib, n), n


def test_version_and_status_strings(lib):
    assert lib.brkga_abi_version() == abi.ABI_VERSION
    for code, name in abi.STATUS_NAMES.items():
        assert lib.brkga_status_string(code).decode() == name


def _packed():
    inst = instances.small(1, n_parts=6)
    return pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                        inst.instance_parts)


def _create(lib, packed):
    h = ctypes.c_void_p()
    st = lib.brkga_problem_create(ctypes.byref(packed.desc), ctypes.byref(h))
    if st == abi.OK:
        lib.brkga_problem_destroy(h)
    return st


def test_create_rejects_bad_descriptors(lib):
    pk = _packed()
    assert lib.brkga_problem_create(None, ctypes.byref(ctypes.c_void_p())) == abi.ERR_INVALID_ARGUMENT
    pk.arrays["gene_type"][0] = 99
    assert _create(lib, pk) == abi.ERR_BAD_INSTANCE
    pk = _packed()
    pk.arrays["part_area"][0] = 0.0
    assert _create(lib, pk) == abi.ERR_BAD_INSTANCE
    pk = _packed()
    pk.arrays["masks"][0] = 2
    assert _create(lib, pk) == abi.ERR_BAD_INSTANCE
    pk = _packed()
    pk.arrays["part_best_rot"][0] = 4
    assert _create(lib, pk) == abi.ERR_BAD_INSTANCE
    pk = _packed()
    pk.desc.threshold_mode = 7
    assert _create(lib, pk) == abi.ERR_INVALID_ARGUMENT


def test_create_without_gpu_reports_no_device(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert _create(lib, _packed()) == abi.ERR_NO_DEVICE


def test_null_problem_arguments(lib):
    n = ctypes.c_size_t()
    assert lib.brkga_workspace_bytes(None, 10, 0, ctypes.byref(n)) == abi.ERR_INVALID_ARGUMENT
    assert lib.brkga_decode(None, None, 1, None, None, None, None, 0, 0, None) == abi.ERR_INVALID_ARGUMENT
    assert lib.brkga_evaluate_host(None, None, 1, None, None) == abi.ERR_INVALID_ARGUMENT
    lib.brkga_problem_destroy(None)


def test_multi_instance_arguments(lib):
    pk = [_packed(), _packed()]
    descs = (abi.BrkgaProblemDesc * 2)(*[p.desc for p in pk])
    h = ctypes.c_void_p()
    assert lib.brkga_problem_create_multi(descs, 0, ctypes.byref(h)) == abi.ERR_INVALID_ARGUMENT
    assert lib.brkga_problem_create_multi(descs, abi.MAX_INSTANCES + 1, ctypes.byref(h)) == abi.ERR_INVALID_ARGUMENT
    assert lib.brkga_problem_create_multi(None, 1, ctypes.byref(h)) == abi.ERR_INVALID_ARGUMENT
    pk[1].arrays["part_area"][0] = 0.0  # a bad second instance is caught before any device work
    assert lib.brkga_problem_create_multi(descs, 2, ctypes.byref(h)) == abi.ERR_BAD_INSTANCE
    pops = np.array([3, 4], np.int32)
    n = ctypes.c_size_t()
    assert lib.brkga_workspace_bytes_multi(None, abi.ptr(pops, ctypes.c_int32), 0, ctypes.byref(n)) == \
        abi.ERR_INVALID_ARGUMENT
    assert lib.brkga_set_launch_config(None, 4, 1, 0, -1) == abi.ERR_INVALID_ARGUMENT
    assert lib.brkga_get_launch_config(None, 0, None, None, None, None, None) == abi.ERR_INVALID_ARGUMENT


def test_header_status_codes_match_the_python_mirror():
    """Every BrkgaStatus value of include/brkga_b200.h has the same value in abi.py."""
    import os
    import re
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "brkga_b200.h")).read()
    enum = hdr[hdr.index("typedef enum BrkgaStatus"):hdr.index("} BrkgaStatus;")]
    codes = dict((name, int(v)) for name, v in re.findall(r"BRKGA_(OK|ERR_[A-Z_]+)\s*=\s*(\d+)", enum))
    assert codes and len(codes) == len(abi.STATUS_NAMES)
    for name, value in codes.items():
        assert getattr(abi, name) == value, name


def test_no_cpu_fallback(tmp_path):
    """Without the CUDA library or without a GPU the product path raises; it never
    decodes on the CPU."""
    import pytest as _pytest
    import torch
    from brkga_fft2_b200 import instances
    with _pytest.raises(RuntimeError, match="no CPU fallback"):
        _load_missing(tmp_path)
    if torch.cuda.is_available():
        return
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator
    inst = instances.small(2)
    with _pytest.raises(RuntimeError):
        B200DecoderEvaluator(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)


def _load_missing(tmp_path):
    """abi.load_library on a path with no library, the loaded one put back after."""
    saved = abi._lib
    abi._lib = None
    try:
        return abi.load_library(str(tmp_path / "missing.so"))
    finally:
        abi._lib = saved


def test_library_carries_the_build_id_of_this_tree(lib):
    """The loaded library was compiled from the sources now in the tree: its
    compiled-in id is the hash of the sources, headers and nvcc flags, and the
    stamp beside it says the same (a stale library is rebuilt, never reused)."""
    bid = build.build_id()
    assert len(bid) == 16
    assert lib.brkga_build_id().decode() == bid
    assert build.stamped_id() == bid
    assert abi.library_build_id() == bid
