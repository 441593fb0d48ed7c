"""Pin the CPU oracle to the reference's own known answers and to golden
vectors produced by running the reference's decoder (tests/golden)."""
import numpy as np
import pytest

from oracle import oracle_decode
from tests import goldens


def test_p75m2_0_reference_golden():
    """results/golden/P75M2-0: makespan 358657.39113 and the 75 ordered placements."""
    packed, _, z = goldens.load("real_P75M2-0")
    ms, log = oracle_decode(packed, z["chromosomes"], with_log=True)
    assert abs(ms[0] - float(z["golden_makespan"][0])) < 1e-6 * 358657  # verify_correctness.py:149 tolerance 1e-6 rel-ish
    assert ms[0] == float(z["makespans"][0])  # bit-exact vs the reference run here
    assert (goldens.part_ids_of_log(packed, log) == z["logs"]).all()


def test_p50m2_0_chromosome_462_and_plate_dumps():
    """verify_native_vs_pp.py:31-32 (448166.8336) and results/inspection_output/pp_bin_m*_b*.txt."""
    packed, pdata, z = goldens.load("real_P50M2-0")
    ms, log = oracle_decode(packed, z["chromosomes"], with_log=True)
    assert round(ms[0], 4) == 448166.8336
    assert ms[0] == float(z["makespans"][0])
    assert (goldens.part_ids_of_log(packed, log) == z["logs"]).all()
    # rebuild the final plates from the log and compare with the reference's dumps
    plates = [k for k in z.files if k.startswith("plate_") and not k.endswith("_shape")]
    assert plates
    for key in plates:
        m, b = (int(s[1:]) for s in key[len("plate_"):].split("_"))
        shape = tuple(z[key + "_shape"])
        grid = np.zeros(shape, np.uint8)
        for rec in log[0, m]:
            if rec["gene"] < 0 or rec["bin"] != b:
                continue
            pid = packed.type_ids[packed.arrays["gene_type"][rec["gene"]]]
            mask = pdata.parts[int(pid)].rotations[rec["rot"]]
            h, w = mask.shape
            grid[rec["y"] - h + 1: rec["y"] + 1, rec["x"]: rec["x"] + w] += mask.astype(np.uint8)
        ref = np.unpackbits(z[key], axis=1)[:, : shape[1]]
        assert grid.max() <= 1
        assert (grid == ref).all(), key


@pytest.mark.parametrize("name", goldens.names("fp_"))
def test_benchmark_fingerprints(name):
    """benchmarks/20260422_*.json: first five feasible makespans (%.6f) of rep 4."""
    packed, _, z = goldens.load(name)
    ms, log = oracle_decode(packed, z["chromosomes"], n_threads=4, with_log=True)
    feas = ms[ms < 1e15]
    assert len(feas) == 5
    assert [f"{v:.6f}" for v in feas] == [f"{v:.6f}" for v in z["fingerprint"]]
    assert (ms == z["makespans"]).all()
    ok = ms < 1e15
    assert (goldens.part_ids_of_log(packed, log)[ok] == z["logs"][ok]).all()


@pytest.mark.parametrize("name", goldens.names("fp_"))
def test_benchmark_feasible_counts(name):
    """n_feasible / n_infeasible of the whole rep-4 population (benchmark JSON)."""
    packed, _, z = goldens.load(name)
    n = packed.n_genes
    pop = np.random.default_rng(int(z["pop_seed"])).random((int(z["pop_mult"]) * n, 2 * n)).astype(np.float32)
    a = packed.arrays
    M = packed.n_machines
    thr = np.float32(a["thresholds"][: M - 1])
    mv = pop[:, n:]
    mach = np.zeros(mv.shape, np.int64)
    for k in range(M - 1):
        mach += mv > thr[k]
    t = a["gene_type"]
    h0 = a["rot_h"][t * 4]
    w0 = a["rot_w"][t * 4]
    L = a["bin_length"][mach]
    W = a["bin_width"][mach]
    unfit = ((h0 > L) | (w0 > W)) & ((w0 > L) | (h0 > W))
    infeasible = unfit.any(axis=1)
    assert int((~infeasible).sum()) == int(z["n_feasible"])
    assert int(infeasible.sum()) == int(z["n_infeasible"])


@pytest.mark.parametrize("name", goldens.names("syn_"))
def test_synthetic_goldens(name):
    """Seeded synthetic instances decoded by the reference (makespans + placements)."""
    packed, _, z = goldens.load(name)
    ms, log = oracle_decode(packed, z["chromosomes"], n_threads=4, with_log=True)
    np.testing.assert_array_equal(ms, z["makespans"])
    ok = ms < 1e15
    assert (goldens.part_ids_of_log(packed, log)[ok] == z["logs"][ok]).all()


def test_six_machine_golden_exercises_the_float32_thresholds():
    """syn_P200M6_s0 puts machine keys on f32(k/6) and the float above it.
    placement.py:122-127 compares them with k/6 in float32, the reference's
    C++ decoder in float64: the two modes must assign some of those genes
    differently, so the golden really pins the float32 choice (hazard H1)."""
    from brkga_fft2_b200 import THRESH_F64
    z = np.load(f"{goldens.GOLDEN}/syn_P200M6_s0.npz")
    ch = z["chromosomes"]
    n = ch.shape[1] // 2
    on = np.zeros(ch.shape[0], bool)
    for k in range(1, 6):
        t = np.float32(k / 6)
        on |= (ch[:, n:] == t).any(axis=1)
        assert (np.float64(t) != k / 6) == (k != 3)  # only 3/6 is exact in float32
    assert on.all()
    p32, _, _ = goldens.load("syn_P200M6_s0")
    p64, _, _ = goldens.load("syn_P200M6_s0", THRESH_F64)
    m32 = oracle_decode(p32, ch, n_threads=4)
    m64 = oracle_decode(p64, ch, n_threads=4)
    np.testing.assert_array_equal(m32, z["makespans"])
    assert (m32 != m64).any()


def test_oracle_results_do_not_depend_on_threads():
    """The oracle's threads take rows from a shared counter: any thread count
    gives the same makespans and placement logs, row for row."""
    from brkga_fft2_b200 import instances, pack_problem
    from oracle import oracle_decode
    inst = instances.p50m2(0)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    ch = instances.chromosomes(37, inst.nb_parts, 5)
    ms1, log1 = oracle_decode(pk, ch, n_threads=1, with_log=True)
    for nt in (3, 8, 64):
        ms, log = oracle_decode(pk, ch, n_threads=nt, with_log=True)
        np.testing.assert_array_equal(ms, ms1)
        assert (log == log1).all()


@pytest.mark.parametrize("tag,step", [("refms_bench_P100M4_step0", 5), ("refms_bench_P100M4_step19", 24)])
def test_benchmark_population_against_reference(tag, step):
    """All 500 rows of the populations bench.py times first and last (with its
    default 5 warm-up and 20 timed steps): the oracle's makespans equal the
    reference's own (its sequential decoder run over a process pool by
    tests/golden/make_golden.py).  bench.py compares the GPU with the oracle
    on the same two populations every run, so the benchmarked rows are tied
    to the reference row for row."""
    import os
    import bench
    from brkga_fft2_b200 import instances
    z = np.load(f"{goldens.GOLDEN}/{tag}.npz")
    assert int(z["pop"]) == bench.POP and int(z["seed"]) == bench.chrom_seed(0, step)
    assert int(z["instance_seed"]) == bench.INSTANCE_SEED
    inst, packed = bench.load_workload()
    rows = instances.chromosomes(int(z["pop"]), inst.nb_parts, int(z["seed"]))
    np.testing.assert_array_equal(rows[0], z["first_row"])
    assert rows.astype(np.float64).sum() == float(z["rows_sum"])
    ms = oracle_decode(packed, rows, n_threads=os.cpu_count() or 1)
    np.testing.assert_array_equal(ms, z["makespans"])


@pytest.mark.parametrize("tag,maker", [("refms_P200M6_s13", "p200m6"), ("refms_P400M8_s14", "p400m8")])
def test_large_workload_rows_against_reference(tag, maker):
    """The rows that the GPU tests compare with the oracle at the 200- and
    400-part sizes (tests/test_decoder_gpu.py, test_benchmark_workloads_vs_oracle):
    the oracle's makespans equal the reference's own."""
    import os
    from brkga_fft2_b200 import instances, pack_problem
    z = np.load(f"{goldens.GOLDEN}/{tag}.npz")
    inst = getattr(instances, maker)(int(z["instance_seed"]))
    packed = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    rows = instances.chromosomes(int(z["pop"]), inst.nb_parts, int(z["seed"]))
    np.testing.assert_array_equal(rows[0], z["first_row"])
    assert rows.astype(np.float64).sum() == float(z["rows_sum"])
    ms = oracle_decode(packed, rows, n_threads=os.cpu_count() or 1)
    np.testing.assert_array_equal(ms, z["makespans"])


def test_uneven_instance_rows_against_reference():
    """The rows of the uneven multi-instance GPU test (tests/test_multi_gpu.py,
    instance k = uneven(k) with rows of seed 100 + k): the oracle's makespans
    equal the reference's own on every instance with at least two machines."""
    import os
    from brkga_fft2_b200 import instances, pack_problem
    z = np.load(f"{goldens.GOLDEN}/refms_uneven.npz")
    done = 0
    for k, P in enumerate(z["pops"].tolist()):
        if f"makespans_{k}" not in z:
            continue
        inst = instances.uneven(k)
        packed = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                              inst.instance_parts)
        rows = instances.chromosomes(P, inst.nb_parts, 100 + k)
        assert rows.astype(np.float64).sum() == float(z[f"rows_sum_{k}"])
        ms = oracle_decode(packed, rows, n_threads=os.cpu_count() or 1)
        np.testing.assert_array_equal(ms, z[f"makespans_{k}"], err_msg=f"instance {k}")
        done += 1
    assert done == 5
