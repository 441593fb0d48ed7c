"""The placement-log checker (tests/placement_check.py) and the hand-built
edge instances (tests/edge_shapes.py), on the CPU.

The checker must accept every decode of the oracle — which the reference's
golden vectors pin — on the golden instances and on the edge instances, in
both threshold modes and with adversarial keys, and it must reject each kind
of mistake planted into a copy of an oracle result."""
import numpy as np
import pytest

from brkga_fft2_b200 import THRESH_F32, THRESH_F64, instances, pack_problem
from oracle import oracle_decode
from tests import goldens
from tests.edge_shapes import EDGE_INSTANCES
from tests.placement_check import PlacementError, rotation_masks, check_rows, machine_of


def special_keys(inst, P, seed):
    """Seeded chromosomes with ties, signed zeros and machine keys on the thresholds."""
    rng = np.random.default_rng(seed)
    ch = instances.chromosomes(P, inst.nb_parts, seed)
    N = inst.nb_parts
    thr32 = np.asarray(inst.thresholds, np.float32)
    for i in range(P):
        if i % 4 == 1:  # ties: a few distinct sequencing keys only
            ch[i, :N] = rng.choice(np.array([0.25, 0.5, 0.75], np.float32), N)
        if i % 4 == 2:  # signed zeros among the sequencing keys
            ch[i, rng.choice(N, N // 2, replace=False)] = np.float32(-0.0)
            ch[i, rng.choice(N, N // 3, replace=False)] = np.float32(0.0)
        if i % 4 == 3 and thr32.size:  # machine keys exactly at float32(threshold)
            pick = rng.choice(N, max(1, N // 2), replace=False)
            ch[i, N + pick] = rng.choice(thr32, pick.size)
    return ch


def edge_pack(name, mode):
    inst = EDGE_INSTANCES[name]()
    return inst, pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                              inst.instance_parts, mode)


@pytest.mark.parametrize("name", list(EDGE_INSTANCES))
@pytest.mark.parametrize("mode", [THRESH_F32, THRESH_F64])
def test_checker_accepts_oracle_on_edge_instances(name, mode):
    inst, pk = edge_pack(name, mode)
    ch = np.concatenate([instances.chromosomes(48, inst.nb_parts, 9), special_keys(inst, 32, 10)])
    ms, log = oracle_decode(pk, ch, n_threads=8, with_log=True)
    assert check_rows(pk, ch, ms, log, range(len(ms))) > 0


@pytest.mark.parametrize("name", goldens.names("real_") + goldens.names("syn_"))
def test_checker_accepts_oracle_on_goldens(name):
    pk, _, z = goldens.load(name)
    ms, log = oracle_decode(pk, z["chromosomes"], n_threads=8, with_log=True)
    np.testing.assert_array_equal(ms, z["makespans"])
    check_rows(pk, z["chromosomes"], ms, log, range(len(ms)))


def test_threshold_modes_differ_on_float32_thresholds():
    """A key equal to float32(1/3) is above the float64 threshold 1/3: the
    float32 mode keeps it on machine 0, the float64 mode sends it to 1."""
    thr = np.array([1 / 3, 2 / 3])
    k = np.array([np.float32(1 / 3), np.float32(2 / 3), np.float32(0.0), np.float32(1.0)], np.float32)
    assert machine_of(k, thr, 3, THRESH_F32).tolist() == [0, 1, 0, 2]
    assert machine_of(k, thr, 3, THRESH_F64).tolist() == [1, 2, 0, 2]
    assert machine_of(np.array([np.nan], np.float32), thr, 3, THRESH_F32).tolist() == [3]
    assert machine_of(np.array([np.nan], np.float32), thr[:0], 1, THRESH_F32).tolist() == [0]


@pytest.fixture(scope="module")
def words():
    inst, pk = edge_pack("EdgeWords", THRESH_F32)
    ch = instances.chromosomes(64, inst.nb_parts, 9)
    ms, log = oracle_decode(pk, ch, n_threads=8, with_log=True)
    check_rows(pk, ch, ms, log, range(len(ms)))
    return pk, ch, ms, log


def _planted(words, plant):
    pk, ch, ms, log = words
    ms2, log2 = ms.copy(), log.copy()
    row = plant(pk, ch, ms2, log2)
    with pytest.raises(PlacementError):
        check_rows(pk, ch, ms2, log2, [row])


def _entry_on_old_plate(log):
    """(row, machine, k) of a part placed into an already open plate."""
    for row in range(log.shape[0]):
        for m in range(log.shape[1]):
            lg = log[row, m]
            for k in range(1, lg.shape[0]):
                if lg["gene"][k] >= 0 and (lg["bin"][:k] == lg["bin"][k]).any():
                    return row, m, k
    raise AssertionError("no part shares a plate")


def test_checker_rejects_a_changed_makespan(words):
    def plant(pk, ch, ms, log):
        ms[3] = np.nextafter(ms[3], np.inf)
        return 3
    _planted(words, plant)


def test_checker_rejects_swapped_decode_order(words):
    def plant(pk, ch, ms, log):
        lg = log[5, 0]
        lg[[0, 1]] = lg[[1, 0]]
        return 5
    _planted(words, plant)


def test_checker_rejects_an_overlap(words):
    def plant(pk, ch, ms, log):
        row, m, k = _entry_on_old_plate(log)
        lg = log[row, m]
        a = pk.arrays
        L, W = int(a["bin_length"][m]), int(a["bin_width"][m])
        masks = rotation_masks(pk)
        occ = np.zeros((L, W), bool)  # the plate before entry k
        for j in np.flatnonzero(lg["bin"][:k] == lg["bin"][k]):
            t, r = int(a["gene_type"][lg["gene"][j]]), int(lg["rot"][j])
            mk = masks[t * 4 + r]
            y, x = int(lg["y"][j]), int(lg["x"][j])
            occ[y - mk.shape[0] + 1:y + 1, x:x + mk.shape[1]] |= mk
        t, r = int(a["gene_type"][lg["gene"][k]]), int(lg["rot"][k])
        mk = masks[t * 4 + r]
        h, w = mk.shape
        my, mx = (int(v[0]) for v in np.nonzero(mk))
        for py, px in zip(*np.nonzero(occ)):  # put the mask's first cell on an occupied cell
            ty, x = int(py) - my, int(px) - mx
            if 0 <= ty and ty + h <= L and 0 <= x and x + w <= W:
                lg["x"][k], lg["y"][k] = x, ty + h - 1
                return row
        raise AssertionError("no overlapping position in bounds")
    _planted(words, plant)


def test_checker_rejects_leaving_the_plate(words):
    def plant(pk, ch, ms, log):
        row, m, k = _entry_on_old_plate(log)
        log[row, m]["x"][k] = int(pk.arrays["bin_width"][m])
        return row
    _planted(words, plant)


def test_checker_rejects_a_skipped_plate_index(words):
    def plant(pk, ch, ms, log):
        lg = log[7, 1]
        lg["bin"][0] = 1
        return 7
    _planted(words, plant)


def test_checker_rejects_a_moved_new_plate(words):
    def plant(pk, ch, ms, log):
        log[9, 0]["x"][0] = 1
        return 9
    _planted(words, plant)


def test_checker_rejects_a_missing_infeasible_score():
    inst, pk = edge_pack("EdgeFlat", THRESH_F32)
    ch = instances.chromosomes(64, inst.nb_parts, 4)
    ms, log = oracle_decode(pk, ch, n_threads=4, with_log=True)
    bad = np.flatnonzero(ms == 1e16)
    assert bad.size
    check_rows(pk, ch, ms, log, range(len(ms)))
    ms[bad[0]] = 1.0
    with pytest.raises(PlacementError):
        check_rows(pk, ch, ms, log, [bad[0]])
