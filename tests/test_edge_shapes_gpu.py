"""The CUDA decoder on the hand-built edge instances (tests/edge_shapes.py)
and on the full-size large-stress population, bit for bit against the oracle.

Edge instances: every row, makespans and placements, in both threshold modes,
with adversarial keys (ties, signed zeros, machine keys on the float32
thresholds), under launch shapes that take every path of the plate search —
1-, 2- and 4-warp CTAs, plates in shared memory and in the global pool, the
(candidate, word) pairs dealt across lanes and, with task_max 0, each lane
testing its own candidate.  Full size: P400M8 (400 parts up to 240x240
cells, 8 plates of 600x600) at population 4096 in one launch — every 8th row
goes through the size-independent placement checker and a spread sample of
16 rows is compared with the oracle."""
import numpy as np
import pytest

from brkga_fft2_b200 import THRESH_F32, THRESH_F64, abi, instances, pack_problem
from oracle import oracle_decode
from tests.edge_shapes import EDGE_INSTANCES
from tests.placement_check import check_rows
from tests.test_placement_check_cpu import special_keys

pytestmark = pytest.mark.gpu

# (warps per item, CTAs per SM, plates in shared memory, task_max); 0 / -1 = automatic
SHAPES = [(0, 0, -1, -1), (2, 0, -1, -1), (4, 0, 0, 0), (4, 1, -1, 64), (1, 0, -1, -1)]


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from brkga_fft2_b200 import build
    build.build()
    return torch


def decode_with_log(torch, dec, ch):
    P = ch.shape[0]
    M, N = dec.packed.n_machines, dec.packed.n_genes
    log = torch.full((P, M, N, 5), -7, dtype=torch.int32, device="cuda")
    out = dec.decode(torch.from_numpy(ch).cuda(), log=log)
    torch.cuda.synchronize()
    assert int(dec.status.item()) == 0
    return out.cpu().numpy(), log.cpu().numpy().reshape(-1).view(abi.PLACEMENT_DTYPE).reshape(P, M, N)


@pytest.mark.parametrize("mode", [THRESH_F32, THRESH_F64])
@pytest.mark.parametrize("name", list(EDGE_INSTANCES))
def test_edge_instances_match_oracle(torch, name, mode):
    from brkga_fft2_b200.evaluator import DeviceDecoder
    inst = EDGE_INSTANCES[name]()
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts,
                      mode)
    P = 256 if name == "EdgeFlat" else 96  # EdgeFlat: most rows are infeasible by design
    ch = np.concatenate([instances.chromosomes(P - 32, inst.nb_parts, 21), special_keys(inst, 32, 22)])
    ref, rlog = oracle_decode(pk, ch, n_threads=8, with_log=True)
    dec = DeviceDecoder(pk, max_pop=P)
    for shape in SHAPES:
        dec.set_launch_config(*shape)
        ms, log = decode_with_log(torch, dec, ch)
        np.testing.assert_array_equal(ms, ref, err_msg=f"{name} {shape}")
        ok = ref < 1e15
        assert (log[ok] == rlog[ok]).all(), f"{name} {shape}"
        assert (log["gene"][~ok] == -1).all()
        check_rows(pk, ch, ms, log, range(P))


def test_full_size_large_stress_population(torch):
    """P400M8 at population 4096, one launch: every 8th row through the
    checker, 16 rows spread over the population against the oracle."""
    from brkga_fft2_b200.evaluator import DeviceDecoder
    inst = instances.p400m8(0)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    P = 4096
    ch = instances.chromosomes(P, inst.nb_parts, 4096)
    dec = DeviceDecoder(pk, max_pop=P)
    ms, log = decode_with_log(torch, dec, ch)
    assert np.isfinite(ms).all() and (ms > 0).all()
    assert check_rows(pk, ch, ms, log, range(0, P, 8)) == P // 8 * inst.nb_parts
    sample = np.linspace(0, P - 1, 16).astype(int)
    ref, rlog = oracle_decode(pk, ch[sample], n_threads=16, with_log=True)
    np.testing.assert_array_equal(ms[sample], ref)
    assert (log[sample] == rlog).all()


def test_bench_workload_every_row(torch):
    """P100M4 at population 500 (the throughput workload): every row through the checker."""
    from brkga_fft2_b200.evaluator import DeviceDecoder
    inst = instances.p100m4(0)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    ch = instances.chromosomes(500, inst.nb_parts, 500)
    ms, log = decode_with_log(torch, DeviceDecoder(pk, max_pop=500), ch)
    assert check_rows(pk, ch, ms, log, range(500)) == 500 * inst.nb_parts
