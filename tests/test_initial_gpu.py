"""Greedy initial solution on the GPU (brkga_initial_solution_host) against
the reference's greedy: the same placements, makespan and chromosome."""
import random

import numpy as np
import pytest

from tests import goldens
from tests.test_initial_cpu import ref_records

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", goldens.names("greedy_"))
def test_device_greedy_matches_reference(name):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required")
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator
    from brkga_fft2_b200.initial import initial_solution
    from brkga_fft2_b200.instance_io import load_instance
    pdata, n, m, thr, inst, z = load_instance(f"{goldens.GOLDEN}/{name}.npz")
    ev = B200DecoderEvaluator(pdata, n, m, thr, inst)
    heights = dict(zip(z["height_ids"].tolist(), z["heights"].tolist()))
    areas = {p: pdata.parts[p].area for p in pdata.parts}
    for i, seed in enumerate(z["greedy_seeds"]):
        chrom, mk, (machine, place) = initial_solution(ev._native, inst, heights, areas, thr,
                                                       random.Random(int(seed)))
        np.testing.assert_array_equal(ref_records(ev.packed, machine, place), z["greedy_placements"][i])
        assert mk == z["greedy_makespans"][i]
        np.testing.assert_array_equal(chrom, z["greedy_chromosomes"][i])
        # the chromosome is a valid GA individual: the decoder scores it
        assert ev.evaluate_batch(chrom[None].astype(np.float32))[0] < 1e15
