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

POPS = [12, 0, 9, 16, 3, 7, 5]  # instance 6 has one machine


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
    assert len({i.nb_machines for i in insts}) > 1 and 1 in {i.nb_machines for i in insts}
    out, log = _run(torch, md, chroms, POPS)
    _check(md, POPS, out, log, ref)


CONFIGS = [(4, 1, 0, -1), (4, 2, 1, 0), (2, 4, -1, 64), (4, 8, 0, 8192), (2, 16, 0, 1), (0, 0, -1, -1),
           (2, 0, -1, -1), (4, 0, 2, -1), (1, 0, -1, -1), (1, 4, 1, 64), (1, 32, 0, 0)]


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
    w2, _, _, slots2, _ = md.launch_config(items=3 * slots4 + 1)
    assert w2 == 2
    assert md.launch_config(items=16 * slots2)[0] == 2
    assert md.launch_config(items=16 * slots2 + 1)[0] == 1


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


def test_decode_at_explicit_offsets(multi):
    """Each instance's rows at its own place in a block layout with gaps (the
    GA's elites stay untouched); makespans written only where asked."""
    torch, insts, packs, chroms, ref, md = multi
    skip = [2, 0, 1, 5, 0, 3, 1]  # leading rows of each block that are not decoded
    blocks = [np.concatenate([np.full((s, c.shape[1]), 0.5, np.float32), c]) for s, c in zip(skip, chroms)]
    sizes = [b.size for b in blocks]
    chrom_off = np.cumsum([0] + sizes)[:-1] + np.array([s * 2 * n for s, n in zip(skip, md.n_genes)])
    rows = [b.shape[0] for b in blocks]
    out_off = np.cumsum([0] + rows)[:-1] + np.array(skip)
    flat = torch.from_numpy(np.concatenate([b.reshape(-1) for b in blocks])).cuda()
    out = torch.full((sum(rows),), -3.0, dtype=torch.float64, device="cuda")
    md.decode_at(flat, chrom_off, POPS, out, out_off)
    torch.cuda.synchronize()
    assert int(md.status.item()) == 0
    got = out.cpu().numpy()
    r0 = 0
    for k, (s, p) in enumerate(zip(skip, POPS)):
        np.testing.assert_array_equal(got[r0:r0 + s], -3.0)
        np.testing.assert_array_equal(got[r0 + s:r0 + s + p], ref[k][0], err_msg=f"instance {k}")
        r0 += s + p
    bad = np.array(chrom_off, np.int64)
    bad[1] = -1
    lib = md.lib
    pops = np.ascontiguousarray(POPS, np.int32)
    oo = np.ascontiguousarray(out_off, np.int64)
    st = lib.brkga_decode_multi_at(0, md.native.handle, ctypes.c_void_p(flat.data_ptr()), abi.ptr(bad, ctypes.c_int64),
                                   abi.ptr(pops, ctypes.c_int32), ctypes.c_void_p(out.data_ptr()),
                                   abi.ptr(oo, ctypes.c_int64), None, ctypes.c_void_p(md.status.data_ptr()),
                                   ctypes.c_void_p(md.workspace.data_ptr()), md.ws_bytes, 0, None)
    assert st == abi.ERR_INVALID_ARGUMENT


def test_pool_exhaustion_is_reported(multi):
    """A plate pool too small for the launch: BRKGA_ERR_CAPACITY on the device
    status and NaN for the items that could not open a plate, never a fault."""
    torch, insts, packs, chroms, ref, md = multi
    from brkga_fft2_b200.evaluator import MultiDecoder
    small = MultiDecoder(packs, max_pops=POPS, pool_bins=1)
    small.set_launch_config(4, 0, 0, -1)  # no plates in shared memory: every plate comes from the pool
    flat = torch.from_numpy(np.concatenate([c.reshape(-1) for c in chroms])).cuda()
    out = small.decode_concat(flat, POPS)
    torch.cuda.synchronize()
    assert int(small.status.item()) == abi.ERR_CAPACITY
    assert np.isnan(out.cpu().numpy()).any()


def test_large_batch_takes_the_one_warp_tier():
    """64 uneven instances x 256 chromosomes (some 50,000 items, past sixteen
    waves of 2-warp CTAs) decode with the automatic shape — 1 warp per item —
    and two rows of every instance equal the oracle's decode."""
    import torch
    from brkga_fft2_b200.evaluator import MultiDecoder
    insts = [instances.uneven(s) for s in range(64)]
    packs = [pack_problem(i.problem_data, i.nb_parts, i.nb_machines, i.thresholds, i.instance_parts) for i in insts]
    pops = [256] * 64
    md = MultiDecoder(packs, max_pops=pops)
    items = sum(p * pk.n_machines for p, pk in zip(pops, packs))
    assert md.launch_config(items=items)[0] == 1
    chroms = [instances.chromosomes(p, i.nb_parts, 500 + k) for k, (p, i) in enumerate(zip(pops, insts))]
    out = md.decode_concat(torch.from_numpy(np.concatenate([c.reshape(-1) for c in chroms])).cuda(), pops)
    torch.cuda.synchronize()
    assert int(md.status.item()) == 0
    got = out.cpu().numpy().reshape(64, 256)
    for k, (pk, ch) in enumerate(zip(packs, chroms)):
        rows = [0, 255 - k]
        np.testing.assert_array_equal(got[k, rows], oracle_decode(pk, ch[rows], n_threads=2), err_msg=f"instance {k}")
