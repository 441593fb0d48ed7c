"""Helpers to load the golden fixtures (written by tests/golden/make_golden.py)."""
import glob
import os

import numpy as np

from brkga_fft2_b200 import THRESH_F32, pack_problem
from brkga_fft2_b200.instance_io import load_instance

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names(prefix=""):
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def load(name, threshold_mode=THRESH_F32):
    pdata, n, m, thr, inst, z = load_instance(os.path.join(GOLDEN, name + ".npz"))
    packed = pack_problem(pdata, n, m, thr, inst, threshold_mode)
    return packed, pdata, z


def part_ids_of_log(packed, log):
    """Oracle/CUDA log [P, M, N] (gene indices) -> part ids int64 [P, M, N, 5] like the goldens."""
    out = -np.ones(log.shape + (5,), np.int64)
    g = log["gene"]
    ok = g >= 0
    inst_type = packed.type_ids[packed.arrays["gene_type"]]
    out[..., 0] = np.where(ok, inst_type[np.clip(g, 0, None)], -1)
    for k, f in enumerate(("bin", "x", "y", "rot"), start=1):
        out[..., k] = np.where(ok, log[f], -1)
    return out
