"""Parity of the CUDA decoder with the reference (golden fixtures) and with
the CPU oracle.  Bit-exact: makespans compared with ==, placements (gene,
plate, x, y, rotation) element-wise."""
import numpy as np
import pytest

from brkga_fft2_b200 import THRESH_F64, instances, pack_problem
from oracle import oracle_decode
from tests import goldens

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from brkga_fft2_b200 import build
    build.build()
    return torch


def evaluator_for(name, torch_cuda, mode=0):
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator
    from brkga_fft2_b200.instance_io import load_instance
    pdata, n, m, thr, inst, z = load_instance(f"{goldens.GOLDEN}/{name}.npz")
    ev = B200DecoderEvaluator(pdata, n, m, thr, inst, None, "cuda", threshold_mode=mode)
    return ev, z


@pytest.mark.parametrize("name", goldens.names("real_") + goldens.names("fp_") + goldens.names("syn_"))
def test_golden_makespans_and_placements(name, torch_cuda):
    ev, z = evaluator_for(name, torch_cuda)
    ms, log = ev.evaluate_batch(z["chromosomes"], return_log=True)
    ms = np.asarray(ms)
    np.testing.assert_array_equal(ms, z["makespans"])
    ok = ms < 1e15
    got = goldens.part_ids_of_log(ev.packed, log)
    assert (got[ok] == z["logs"][ok]).all()
    assert (log["gene"][~ok] == -1).all()


def test_reference_p75m2_golden_value(torch_cuda):
    ev, z = evaluator_for("real_P75M2-0", torch_cuda)
    ms = ev.evaluate_batch(z["chromosomes"])
    assert abs(ms[0] - 358657.39113) < 1e-5


def test_fingerprint_strings(torch_cuda):
    for name in goldens.names("fp_"):
        ev, z = evaluator_for(name, torch_cuda)
        ms = np.asarray(ev.evaluate_batch(z["chromosomes"]))
        assert [f"{v:.6f}" for v in ms[ms < 1e15]] == [f"{v:.6f}" for v in z["fingerprint"]], name


@pytest.mark.parametrize("maker,P,seed", [(instances.p50m2, 100, 11), (instances.p100m4, 64, 12),
                                          (instances.p200m6, 24, 13), (instances.p400m8, 8, 14)])
def test_benchmark_workloads_vs_oracle(maker, P, seed, torch_cuda):
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator
    inst = maker(0)
    ev = B200DecoderEvaluator(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                              inst.instance_parts)
    ch = instances.chromosomes(P, inst.nb_parts, seed)
    ms, log = ev.evaluate_batch(ch, return_log=True)
    ref, rlog = oracle_decode(ev.packed, ch, n_threads=8, with_log=True)
    np.testing.assert_array_equal(np.asarray(ms), ref)
    assert (log == rlog).all()


def test_float64_threshold_mode(torch_cuda):
    """Machine keys on f32(1/3): placement.py (float32) and the C++ decoder (float64) differ."""
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator
    from brkga_fft2_b200.instance_io import load_instance
    pdata, n, m, thr, inst, z = load_instance(f"{goldens.GOLDEN}/syn_three_machines.npz")
    ev = B200DecoderEvaluator(pdata, n, m, thr, inst, threshold_mode=THRESH_F64)
    ms = np.asarray(ev.evaluate_batch(z["chromosomes"]))
    np.testing.assert_array_equal(ms, oracle_decode(ev.packed, z["chromosomes"]))
    ev32, _ = evaluator_for("syn_three_machines", torch_cuda)
    assert not np.array_equal(ms, np.asarray(ev32.evaluate_batch(z["chromosomes"])))


def test_determinism_and_batch_position_independence(torch_cuda):
    """verify_native_vs_pp.py Parts A-D as properties: same chromosome, same
    result, whatever the batch size, position or repetition."""
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator
    inst = instances.p50m2(0)
    ev = B200DecoderEvaluator(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                              inst.instance_parts)
    ch = instances.chromosomes(300, inst.nb_parts, 21)
    a = np.asarray(ev.evaluate_batch(ch))
    b = np.asarray(ev.evaluate_batch(ch))
    np.testing.assert_array_equal(a, b)
    perm = np.random.default_rng(0).permutation(300)
    c = np.asarray(ev.evaluate_batch(ch[perm]))
    np.testing.assert_array_equal(c, a[perm])
    for k in (1, 7, 64):
        np.testing.assert_array_equal(np.asarray(ev.evaluate_batch(ch[:k])), a[:k])
    d = np.asarray(ev.evaluate_batch(np.repeat(ch[5:6], 50, axis=0)))
    assert (d == a[5]).all()


def test_device_decoder_matches_host_path(torch_cuda):
    torch = torch_cuda
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator, DeviceDecoder
    inst = instances.p100m4(0)
    ev = B200DecoderEvaluator(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                              inst.instance_parts)
    dd = DeviceDecoder(ev.packed, max_pop=128)
    ch = instances.chromosomes(128, inst.nb_parts, 5)
    dev = torch.from_numpy(ch).cuda()
    out = dd.decode(dev)
    torch.cuda.synchronize()
    assert int(dd.status.item()) == 0
    np.testing.assert_array_equal(out.cpu().numpy(), np.asarray(ev.evaluate_batch(ch)))
    tests, chunks, bins, scan = dd.counters()
    assert tests > 0 and chunks > 0 and bins > 0 and scan > 0


def test_pool_overflow_is_reported_then_retried(torch_cuda):
    """A one-plate pool overflows (status BRKGA_ERR_CAPACITY, NaN makespans);
    the host entry point grows its pool and returns exact results."""
    torch = torch_cuda
    from brkga_fft2_b200 import abi
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator, DeviceDecoder
    inst = instances.make_instance("many", 40, [(60, 60), (64, 56)], 3, bbox_min=12, bbox_max=40)
    ev = B200DecoderEvaluator(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                              inst.instance_parts)
    ch = instances.chromosomes(32, inst.nb_parts, 9)
    ref = oracle_decode(ev.packed, ch)
    np.testing.assert_array_equal(np.asarray(ev.evaluate_batch(ch)), ref)
    dd = DeviceDecoder(ev.packed, max_pop=32, pool_bins=1)
    out = dd.decode(torch.from_numpy(ch).cuda())
    torch.cuda.synchronize()
    assert int(dd.status.item()) == abi.ERR_CAPACITY
    o = out.cpu().numpy()
    assert np.isnan(o).any()
    fine = ~np.isnan(o)
    np.testing.assert_array_equal(o[fine], ref[fine])


def test_rejects_bad_shapes(torch_cuda):
    ev, z = evaluator_for("syn_edge", torch_cuda)
    with pytest.raises(RuntimeError):
        ev.evaluate_batch(np.zeros(10, np.float32))
    with pytest.raises(RuntimeError):
        ev.evaluate_batch(np.zeros((2, 5), np.float32))
    assert ev.evaluate_batch(np.zeros((0, 2 * ev.nb_parts), np.float32)) == []


def test_single_machine_and_nan_keys(torch_cuda):
    """M = 1 puts every part on the one machine (as the C++ decoder does); a NaN
    machine key drops the gene (every threshold comparison is false)."""
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator
    inst = instances.make_instance("one", 15, [(64, 64)], 4, bbox_min=6, bbox_max=30)
    ev = B200DecoderEvaluator(inst.problem_data, 15, 1, [], inst.instance_parts)
    ch = instances.chromosomes(20, 15, 1)
    np.testing.assert_array_equal(np.asarray(ev.evaluate_batch(ch)), oracle_decode(ev.packed, ch))
    inst2 = instances.small(4, n_parts=12)
    ev2 = B200DecoderEvaluator(inst2.problem_data, 12, 2, inst2.thresholds, inst2.instance_parts)
    ch2 = instances.chromosomes(20, 12, 2)
    ch2[::3, 12 + 2] = np.nan
    ch2[1::4, 5] = np.nan
    np.testing.assert_array_equal(np.asarray(ev2.evaluate_batch(ch2)), oracle_decode(ev2.packed, ch2))


def test_audit_output_from_the_device_log(torch_cuda):
    """Plates rebuilt from the CUDA decoder's log equal the reference's own plate
    dumps (P50M2-0 chromosome 462), and the solution record's machines rebuild
    the makespan."""
    from brkga_fft2_b200 import audit
    from tests.test_audit_cpu import reference_plates
    ev, z = evaluator_for("real_P50M2-0", torch_cuda)
    ms, log = ev.evaluate_batch(z["chromosomes"], return_log=True)
    plates = audit.plates_from_log(ev.packed, log[0])
    for k, grid in reference_plates(z).items():
        assert (plates[k] == grid).all(), k
    rec = audit.solution_record(ev.packed, z["chromosomes"][0], ms[0], log[0], instance="P50M2-0")
    assert max(m["makespan"] for m in rec["machines"].values()) == rec["makespan"] == round(ms[0], 6)
