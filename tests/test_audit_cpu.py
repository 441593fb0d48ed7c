"""Audit output (brkga_fft2_b200/audit.py) in the reference's formats, on the
oracle's logs: plates rebuilt from the log equal the reference's own plate
dumps (results/inspection_output, P50M2-0 chromosome 462), the text dump
round-trips, the golden-solution record matches the reference's golden
placements, and per-machine makespans rebuild the decoded makespan."""
import json

import numpy as np
import pytest

from brkga_fft2_b200 import audit, instances, pack_problem
from oracle import oracle_decode
from tests import goldens


def reference_plates(z):
    out = {}
    for key in z.files:
        if key.startswith("plate_") and not key.endswith("_shape"):
            m, b = (int(s[1:]) for s in key[len("plate_"):].split("_"))
            shape = tuple(z[key + "_shape"])
            out[(m, b)] = np.unpackbits(z[key], axis=1)[:, : shape[1]]
    return out


def test_plates_from_log_equal_reference_dumps(tmp_path):
    packed, _, z = goldens.load("real_P50M2-0")
    ms, log = oracle_decode(packed, z["chromosomes"], with_log=True)
    plates = audit.plates_from_log(packed, log[0])
    ref = reference_plates(z)
    assert ref and set(ref) <= set(plates)
    for k, grid in ref.items():
        assert (plates[k] == grid).all(), k
    paths = audit.write_plate_dumps(str(tmp_path), plates)
    assert len(paths) == len(plates)
    for (m, b), grid in plates.items():
        path = tmp_path / f"bin_m{m}_b{b}.txt"
        np.testing.assert_array_equal(audit.read_plate_dump(str(path)), grid)
        first = path.read_text().splitlines()[0]
        assert first == " ".join(f"{int(v):2d}" for v in grid[0])  # binClassNew.py:39-42


def test_solution_record_matches_reference_golden():
    packed, _, z = goldens.load("real_P75M2-0")
    ms, log = oracle_decode(packed, z["chromosomes"], with_log=True)
    rec = audit.solution_record(packed, z["chromosomes"][0], ms[0], log[0], instance="P75M2-0", inst_number=0)
    json.dumps(rec)
    assert rec["makespan"] == round(float(z["makespans"][0]), 6)
    ref = z["logs"][0]  # [M, N, 5] part id, bin, x, y, rot
    for m in range(packed.n_machines):
        got = [[p["part_id"], p["bin_idx"], p["col"], p["row"], p["rot"]] for p in rec["machines"][str(m)]["placements"]]
        want = [list(r) for r in ref[m] if r[0] >= 0]
        assert got == want, m
        assert rec["machines"][str(m)]["n_bins"] == len({r[1] for r in want})
    assert max(rec["machines"][str(m)]["makespan"] for m in range(packed.n_machines)) == rec["makespan"]


@pytest.mark.parametrize("maker", [instances.p50m2, instances.p100m4])
def test_machine_makespans_rebuild_the_makespan(maker):
    inst = maker(0)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    ch = instances.chromosomes(12, inst.nb_parts, 33)
    ms, log = oracle_decode(pk, ch, n_threads=4, with_log=True)
    for i in range(len(ms)):
        if ms[i] < 1e15:
            assert max(audit.machine_makespans(pk, log[i])) == ms[i]
