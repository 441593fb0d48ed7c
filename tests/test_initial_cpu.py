"""Greedy initial solution (BRKGA_alg3.py:445-603): the CPU oracle and the
chromosome encoding against the reference's own greedy, run on the same
instances (tests/golden/greedy_*.npz)."""
import random

import numpy as np
import pytest

from brkga_fft2_b200.initial import encode, greedy_order
from oracle import oracle_initial_solution
from tests import goldens


def ref_records(packed, machine, place):
    """(machine, plate, part id, x, y, rot) per placement, like the golden."""
    pid = packed.type_ids[packed.arrays["gene_type"][place["gene"]]]
    return np.stack([machine, place["bin"], pid, place["x"], place["y"], place["rot"]], axis=1).astype(np.int64)


@pytest.mark.parametrize("name", goldens.names("greedy_"))
def test_oracle_greedy_matches_reference(name):
    packed, pdata, z = goldens.load(name)
    heights = dict(zip(z["height_ids"].tolist(), z["heights"].tolist()))
    areas = {p: pdata.parts[p].area for p in pdata.parts}
    order = greedy_order(z["instance_parts"], heights, areas)
    machine, place, mk = oracle_initial_solution(packed, order)
    for i, seed in enumerate(z["greedy_seeds"]):
        np.testing.assert_array_equal(ref_records(packed, machine, place), z["greedy_placements"][i])
        assert mk.max() == z["greedy_makespans"][i]
        chrom = encode(machine, place, z["instance_parts"], packed.type_ids, packed.arrays["gene_type"],
                       packed.n_machines, [float(v) for v in z["thresholds"]], random.Random(int(seed)))
        np.testing.assert_array_equal(chrom, z["greedy_chromosomes"][i])
