"""The C ABI from C: tests/c_abi_client.c includes include/brkga_b200.h, links
libbrkga_b200.so and decodes a population through brkga_evaluate_host, as a
C or C++ host replacing the reference's native decoder would.  Compiling it
is a CPU test; running it needs the GPU and must match the oracle bit for bit."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from brkga_fft2_b200 import abi, build, instances, pack_problem

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def compile_client(out_dir):
    gcc = shutil.which("gcc") or shutil.which("cc")
    if gcc is None:
        pytest.fail("no C compiler")
    lib = build.build()
    exe = os.path.join(out_dir, "c_abi_client")
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-O1", "-I", os.path.join(REPO, "include"),
                    os.path.join(HERE, "c_abi_client.c"), "-o", exe, "-L", os.path.dirname(lib), "-lbrkga_b200",
                    "-Wl,-rpath," + os.path.dirname(lib)], check=True)
    return exe


def write_instance(packed, path):
    a = packed.arrays
    with open(path, "wb") as f:
        np.array([packed.n_genes, packed.n_machines, packed.n_types, packed.threshold_mode], np.int32).tofile(f)
        np.array([a["masks"].size], np.int64).tofile(f)
        for key, dt in (("gene_type", np.int32), ("thresholds", np.float64), ("bin_length", np.int32),
                        ("bin_width", np.int32), ("bin_area", np.float64), ("setup_time", np.float64),
                        ("proc_time", np.float64), ("proc_time_height", np.float64), ("part_area", np.float64),
                        ("part_nrot", np.int32), ("part_best_rot", np.int32), ("rot_h", np.int32),
                        ("rot_w", np.int32), ("rot_mask_offset", np.int64), ("masks", np.uint8)):
            arr = np.ascontiguousarray(a[key], dtype=dt)
            if key == "thresholds":
                arr = arr[: max(packed.n_machines - 1, 0)]
            arr.tofile(f)


def test_header_compiles_as_c_and_links(tmp_path):
    exe = compile_client(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_c_client_matches_oracle(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from oracle import oracle_decode
    exe = compile_client(str(tmp_path))
    inst = instances.p100m4(3)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    ch = instances.chromosomes(40, inst.nb_parts, 21)
    write_instance(pk, str(tmp_path / "inst.bin"))
    with open(tmp_path / "pop.bin", "wb") as f:
        np.array([ch.shape[0]], np.int32).tofile(f)
        ch.tofile(f)
    res = subprocess.run([exe, str(tmp_path / "inst.bin"), str(tmp_path / "pop.bin"), str(tmp_path / "out.bin")],
                         capture_output=True, text=True)
    assert res.returncode == abi.OK, res.stderr
    got = np.fromfile(tmp_path / "out.bin", dtype=np.float64)
    np.testing.assert_array_equal(got, oracle_decode(pk, ch, n_threads=8))
