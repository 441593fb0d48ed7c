"""The INT8 tensor-core correlation against the bit-packed search, chunk by chunk.

Both collision paths of brkga_chunk_free must give the same free-position
words on the decoder's own chunks: plates recovered from P400M8 decode logs
(600 x 600 plates, masks up to 240 x 240) and P200M6 ones, every rotation of
the placed part with a side of at least 64 cells, the bottom three chunk
levels.  A few chunks are also checked against a direct numpy correlation
(overlap count == 0, the reference's test, collision_backend.py:109-128)."""
import numpy as np
import pytest
from numpy.lib.stride_tricks import sliding_window_view

from brkga_fft2_b200 import abi, collision, instances, pack_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from brkga_fft2_b200 import build
    build.build()
    return torch


def decoded_cases(torch, maker, P, seed, limit):
    from brkga_fft2_b200.evaluator import DeviceDecoder
    inst = maker(0)
    packed = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    dd = DeviceDecoder(packed, max_pop=P)
    chrom = torch.from_numpy(instances.chromosomes(P, inst.nb_parts, seed)).cuda()
    log = torch.empty((P, inst.nb_machines, inst.nb_parts, 5), dtype=torch.int32, device="cuda")
    dd.decode(chrom, log=log)
    torch.cuda.synchronize()
    assert int(dd.status.item()) == 0
    log = log.cpu().numpy().view(abi.PLACEMENT_DTYPE).reshape(P, inst.nb_machines, inst.nb_parts)
    cases = collision.chunk_cases(packed, log, min_side=64, levels=(0, 1, 2), limit=limit)
    return packed, dd, cases


def direct_words(grid, mask, ty_hi):
    """Free-position words [32, nwo] by a direct overlap count (numpy)."""
    L, W = grid.shape
    h, w = mask.shape
    nx = W - w + 1
    cnt = np.zeros((32, nx), np.float32)
    rows = np.zeros((L + 32, W), np.float32)
    rows[32:] = grid
    for i in range(h):
        # candidate n has top row ty_hi - n: its mask row i sits on plate row ty_hi - n + i
        band = rows[32 + ty_hi - 31 + i: 32 + ty_hi + i + 1][::-1]  # row n = plate row ty_hi - n + i
        cnt += sliding_window_view(band, w, axis=1) @ mask[i].astype(np.float32)
    free = cnt == 0
    for n in range(32):
        if ty_hi - n < 0:
            free[n] = False
    nwo = (nx + 31) // 32
    by = np.packbits(free, axis=1, bitorder="little")
    out = np.zeros((32, nwo * 4), np.uint8)
    out[:, : by.shape[1]] = by
    return out.view("<u4")


@pytest.mark.parametrize("maker,P,seed,limit", [(instances.p400m8, 4, 21, 240), (instances.p200m6, 8, 22, 160)])
def test_int8_correlation_equals_bitset_search(torch_cuda, maker, P, seed, limit):
    torch = torch_cuda
    packed, dd, cases = decoded_cases(torch, maker, P, seed, limit)
    assert len(cases) >= 50
    batch = collision.ChunkBatch(dd.native, packed, cases)
    batch.out.fill_(-1)
    batch.run(abi.COLLISION_BITSET)
    torch.cuda.synchronize()
    assert int(batch.status.item()) == 0
    ref = [batch.words(i) for i in range(len(cases))]
    batch.out.fill_(-1)
    batch.run(abi.COLLISION_INT8_TC)
    torch.cuda.synchronize()
    assert int(batch.status.item()) == 0
    n_free = 0
    for i, c in enumerate(cases):
        got = batch.words(i)
        assert np.array_equal(got, ref[i]), (i, c["machine"], c["type"], c["rot"], c["ty_hi"])
        n_free += int(np.unpackbits(got.view(np.uint8)).sum())
    assert n_free > 0  # some chunks do have free placements
    # independent check of both: a direct overlap count on a few chunks, the largest masks among them
    pick = sorted(range(len(cases)), key=lambda i: -cases[i]["h"] * cases[i]["w"])[:2] + [0, len(cases) // 2]
    for i in pick:
        c = cases[i]
        mask = collision._rotation(packed, c["type"], c["rot"])
        assert np.array_equal(direct_words(c["grid"], mask, c["ty_hi"]), ref[i]), i


def test_int8_correlation_chunk_near_the_top_and_empty_plate(torch_cuda):
    """Candidates above the plate's first row come out empty; on an empty
    plate every column of every valid candidate is free (both paths)."""
    torch = torch_cuda
    packed, dd, cases = decoded_cases(torch, instances.p400m8, 2, 23, 16)
    c = dict(cases[0])
    c["ty_hi"] = 5  # candidates 6..31 would start above row 0
    e = dict(cases[1])
    e["grid"] = np.zeros_like(e["grid"])
    batch = collision.ChunkBatch(dd.native, packed, [c, e])
    for path in (abi.COLLISION_BITSET, abi.COLLISION_INT8_TC):
        batch.out.fill_(-1)
        batch.run(path)
        torch.cuda.synchronize()
        assert int(batch.status.item()) == 0
        w0 = batch.words(0)
        assert (w0[6:] == 0).all()
        mask = collision._rotation(packed, c["type"], c["rot"])
        assert np.array_equal(w0, direct_words(c["grid"], mask, 5))
        w1 = batch.words(1)
        W = int(packed.arrays["bin_width"][e["machine"]])
        nx = W - e["w"] + 1
        full = np.unpackbits(w1.view(np.uint8), axis=1, bitorder="little")[:, :nx]
        assert full.all()


def test_malformed_chunk_is_refused(torch_cuda):
    torch = torch_cuda
    packed, dd, cases = decoded_cases(torch, instances.p200m6, 2, 24, 8)
    bad = dict(cases[0])
    bad["ty_hi"] = int(packed.arrays["bin_length"][bad["machine"]])  # beyond L - h
    batch = collision.ChunkBatch(dd.native, packed, [bad])
    for path in (abi.COLLISION_BITSET, abi.COLLISION_INT8_TC):
        batch.status.zero_()
        batch.out.fill_(-1)
        batch.run(path)
        torch.cuda.synchronize()
        assert int(batch.status.item()) == abi.ERR_INVALID_ARGUMENT
        assert (batch.out == -1).all()
