"""The host-side problem layer (brkga_fft2_b200/problem.py, instance_io.py):
the reference's part precompute (BRKGA_alg3.py:332-386), the packing of a
ProblemData into descriptor tables, its argument checks, and the fixture
file round trip."""
import numpy as np
import pytest

from brkga_fft2_b200 import THRESH_F32, THRESH_F64, instances, make_part_data, pack_problem
from brkga_fft2_b200.instance_io import load_instance, save_instance
from tests.edge_shapes import EDGE_INSTANCES


def test_part_precompute_follows_the_reference():
    # not symmetric under a half turn: four rotations, counter-clockwise np.rot90
    m = np.array([[1, 1, 1], [1, 0, 0]], np.uint8)
    pd = make_part_data(7, m)
    assert pd.nrot == 4 and pd.area == 4.0
    for r in range(4):
        np.testing.assert_array_equal(pd.rotations[r], np.rot90(m, r))
    assert pd.shapes == [(2, 3), (3, 2), (2, 3), (3, 2)]
    assert pd.best_rotation == 0  # first of the lowest rotations
    assert [list(d) for d in pd.densities[:2]] == [[3, 1], [1, 1, 2]]  # longest run of ones per row
    # symmetric under a half turn: two rotations
    sym = np.array([[1, 0], [0, 1]], np.uint8)
    assert make_part_data(1, sym).nrot == 2
    # a tall part: the lying rotation is the best one
    assert make_part_data(2, np.ones((5, 2), np.uint8)).best_rotation == 1
    with pytest.raises(ValueError):
        make_part_data(3, np.array([[0, 2]], np.uint8))


def test_pack_problem_checks_its_arguments():
    inst = instances.small(3)
    args = (inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    pk = pack_problem(*args)
    assert pk.n_genes == inst.nb_parts and pk.n_machines == inst.nb_machines
    with pytest.raises(ValueError):
        pack_problem(inst.problem_data, inst.nb_parts + 1, inst.nb_machines, inst.thresholds, inst.instance_parts)
    with pytest.raises(ValueError):
        pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines + 1, inst.thresholds, inst.instance_parts)
    with pytest.raises(ValueError):
        pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, [], inst.instance_parts)
    with pytest.raises(ValueError):
        pack_problem(*args, threshold_mode=7)
    assert pack_problem(*args, threshold_mode=THRESH_F64).threshold_mode == THRESH_F64


@pytest.mark.parametrize("name", ["EdgeWords", "EdgeFlat"])
def test_fixture_round_trip_keeps_the_tables(tmp_path, name):
    inst = EDGE_INSTANCES[name]()
    path = str(tmp_path / "inst.npz")
    save_instance(path, inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts,
                  extra={"note": np.array([1])})
    pdata, n, m, thr, ip, z = load_instance(path)
    assert (n, m) == (inst.nb_parts, inst.nb_machines) and list(z["note"]) == [1]
    a = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts,
                     THRESH_F32)
    b = pack_problem(pdata, n, m, thr, ip, THRESH_F32)
    assert set(a.arrays) == set(b.arrays)
    for key in a.arrays:
        np.testing.assert_array_equal(a.arrays[key], b.arrays[key], err_msg=key)
