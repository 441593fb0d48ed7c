"""Several independent instances decoded in one launch (brkga_decode_multi).

Uneven instances (25-200 parts, 1-6 machines, plates 150x150 to 500x500
cells) with different population sizes, one of them empty, go through one
launch of each kernel; every row must equal the oracle's decode of that
instance alone, makespans and placements bit for bit, whatever the launch
shape of the decode kernel.
"""
import ctypes

import numpy as np
import pytest

from brkga_fft2_b200 import abi, instances, pack_problem
from oracle import oracle_decode

pytestmark = pytest.mark.gpu

POPS = [12, 0, 9, 16, 3, 7]


@pytest.fixture(scope="module")
def multi():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from brkga_fft2_b200 import build
    build.build()
    from brkga_fft2_b200.evaluator import MultiDecoder
    insts = [instances.uneven(s) for s in range(len(POPS))]
    packs = [pack_problem(i.problem_data, i.nb_parts, i.nb_machines, i.thresholds, i.instance_parts)
             for i in insts]
    chroms = [instances.chromosomes(p, i.nb_parts, 100 + k) for k, (p, i) in enumerate(zip(POPS, insts))]
    ref = [oracle_decode(pk, ch, n_threads=8, with_log=True) for pk, ch in zip(packs, chroms)]
    md = MultiDecoder(packs, max_pops=POPS)
    return torch, insts, packs, chroms, ref, md


def _run(torch, md, chroms, pops):
    flat = torch.from_numpy(np.concatenate([c.reshape(-1) for c in chroms])).cuda()
    n_log = sum(p * m * n for p, m, n in zip(pops, md.n_machines, md.n_genes))
    log = torch.full((n_log * 5,), -7, dtype=torch.int32, device="cuda")
    out = md.decode_concat(flat, pops, log=log)
    torch.cuda.synchronize()
    assert int(md.status.item()) == 0
    return out.cpu().numpy(), log.cpu().numpy()


def _check(md, pops, out, log, ref):
    r0 = l0 = 0
    for k, (p, (rms, rlog)) in enumerate(zip(pops, ref)):
        M, N = md.n_machines[k], md.n_genes[k]
        np.testing.assert_array_equal(out[r0:r0 + p], rms, err_msg=f"instance {k}")
        got = log[l0 * 5:(l0 + p * M * N) * 5].view(abi.PLACEMENT_DTYPE).reshape(p, M, N)
        assert (got == rlog).all(), f"instance {k}"
        r0 += p
        l0 += p * M * N


def test_uneven_instances_match_oracle(multi):
    torch, insts, packs, chroms, ref, md = multi
    assert {i.nb_machines for i in insts} != {insts[0].nb_machines} or len(insts) == 1
    out, log = _run(torch, md, chroms, POPS)
    _check(md, POPS, out, log, ref)


CONFIGS = [(4, 1, 0, -1), (4, 2, 1, 0), (2, 4, -1, 64), (4, 8, 0, 8192), (2, 16, 0, 1), (0, 0, -1, -1),
           (2, 0, -1, -1), (4, 0, 2, -1)]


@pytest.mark.parametrize("cfg", CONFIGS)
def test_launch_configs_give_identical_results(multi, cfg):
    torch, insts, packs, chroms, ref, md = multi
    md.set_launch_config(*cfg)
    warps, ctas, plates, grid, task_max = md.launch_config()
    if cfg[0]:
        assert warps == cfg[0]
    if cfg[1]:
        assert ctas == cfg[1]
    if cfg[2] >= 0:
        assert plates == cfg[2]
    assert task_max == (cfg[3] if cfg[3] >= 0 else 8192)
    out, log = _run(torch, md, chroms, POPS)
    _check(md, POPS, out, log, ref)
    md.set_launch_config()


def test_automatic_warps_follow_item_count(multi):
    torch, insts, packs, chroms, ref, md = multi
    md.set_launch_config()
    w_small, _, _, slots4, _ = md.launch_config(items=1)
    assert w_small == 4
    assert md.launch_config(items=3 * slots4)[0] == 4
    assert md.launch_config(items=3 * slots4 + 1)[0] == 2


def test_unresident_shape_is_refused(multi):
    torch, insts, packs, chroms, ref, md = multi
    before = md.launch_config()
    with pytest.raises(abi.BrkgaError) as e:
        md.set_launch_config(4, 32, 8)  # 32 CTAs with 8 plates each cannot share one SM
    assert e.value.status == abi.ERR_INVALID_ARGUMENT
    with pytest.raises(abi.BrkgaError):
        md.set_launch_config(0, 8, 0)  # a CTA count needs an explicit CTA size
    assert md.launch_config() == before


def test_single_instance_entry_points_refuse_multi(multi):
    torch, insts, packs, chroms, ref, md = multi
    lib, h = md.lib, md.native.handle
    nbytes = ctypes.c_size_t()
    assert lib.brkga_workspace_bytes(h, 4, 0, ctypes.byref(nbytes)) == abi.ERR_INVALID_ARGUMENT
    K = ctypes.c_int32()
    assert lib.brkga_problem_instances(h, ctypes.byref(K)) == abi.OK and K.value == len(POPS)


def test_per_instance_tensors_and_graph_replay(multi):
    """decode() on a list of tensors, and the same launch captured in a CUDA graph."""
    torch, insts, packs, chroms, ref, md = multi
    outs = md.decode([torch.from_numpy(c).cuda() for c in chroms])
    for k, o in enumerate(outs):
        np.testing.assert_array_equal(o.cpu().numpy(), ref[k][0])
    flat = torch.from_numpy(np.concatenate([c.reshape(-1) for c in chroms])).cuda()
    out = torch.empty(sum(POPS), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        md.decode_concat(flat, POPS, out=out)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        md.decode_concat(flat, POPS, out=out)
    out.fill_(-1.0)
    g.replay()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), np.concatenate([r[0] for r in ref]))
