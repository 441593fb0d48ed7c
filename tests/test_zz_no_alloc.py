"""brkga_decode_noalloc: decoding for callers that cannot allocate device memory.

Some callers own every device byte themselves (a plugin host or an embedded
scheduler with a fixed budget) or run loops that must never reach cudaMalloc
or cudaFree, which can synchronise the whole device.  For them the library
keeps a fixed 64 MiB scratch array in device memory and decodes into it; the
caller passes only its inputs and outputs.  This test checks that path against
the ordinary workspace path, bit for bit, on two calls in a row (the second
call reuses the array the first one left behind).  It lives in its own file,
collected last, so that a failure here never hides the other tests.
"""
import ctypes

import numpy as np
import pytest

from brkga_fft2_b200 import abi, instances, pack_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from brkga_fft2_b200 import build
    build.build()
    from brkga_fft2_b200.evaluator import DeviceDecoder
    inst = instances.p100m4(0)
    packed = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                          inst.instance_parts)
    return torch, inst, DeviceDecoder(packed, max_pop=500)


def _noalloc(torch, dd, chrom, out, log, status):
    s = torch.cuda.current_stream()
    return dd.lib.brkga_decode_noalloc(dd.native.handle, ctypes.c_void_p(chrom.data_ptr()), chrom.shape[0],
                                       ctypes.c_void_p(out.data_ptr()),
                                       ctypes.c_void_p(log.data_ptr()) if log is not None else None,
                                       ctypes.c_void_p(status.data_ptr()), ctypes.c_void_p(s.cuda_stream))


def test_noalloc_matches_workspace_decode_two_calls(setup):
    torch, inst, dd = setup
    N, M = inst.nb_parts, inst.nb_machines
    for call, seed in enumerate((31, 32)):
        chrom = torch.from_numpy(instances.chromosomes(500, N, seed)).cuda()
        ref_log = torch.full((500, M, N, 5), -7, dtype=torch.int32, device="cuda")
        ref = dd.decode(chrom, log=ref_log)
        out = torch.full((500,), -1.0, dtype=torch.float64, device="cuda")
        log = torch.full((500, M, N, 5), -7, dtype=torch.int32, device="cuda")
        status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        assert _noalloc(torch, dd, chrom, out, log, status) == abi.OK
        torch.cuda.synchronize()
        assert int(status.item()) == abi.OK, f"call {call}"
        assert int(dd.status.item()) == abi.OK
        assert torch.equal(out, ref), f"call {call}: makespans differ"
        assert torch.equal(log, ref_log), f"call {call}: placements differ"
        assert bool(torch.isfinite(out).all())


def test_noalloc_rejects_population_beyond_scratch(setup):
    """A population whose tables alone exceed the 64 MiB scratch is refused
    before anything is launched."""
    torch, inst, dd = setup
    dummy = torch.zeros(2 * inst.nb_parts, dtype=torch.float32, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    st = dd.lib.brkga_decode_noalloc(dd.native.handle, ctypes.c_void_p(dummy.data_ptr()), 200_000,
                                     ctypes.c_void_p(out.data_ptr()), None, ctypes.c_void_p(status.data_ptr()),
                                     ctypes.c_void_p(s.cuda_stream))
    assert st == abi.ERR_WORKSPACE
    assert abi.NOALLOC_SCRATCH_BYTES == 64 << 20


def test_noalloc_full_plate_pool_reports_capacity(setup):
    """Tables that fit but plates that do not: 600x600 plates (51 KB each, so
    about 1,300 of them in the scratch array) for 96 P400M8 chromosomes, whose
    768 items open several plates each.  The device status says
    BRKGA_ERR_CAPACITY, the rows with an item that ran out are NaN, every other
    row equals the workspace decode, and a smaller batch afterwards decodes in
    full."""
    torch, _, _ = setup
    from brkga_fft2_b200.evaluator import DeviceDecoder
    inst = instances.p400m8(0)
    packed = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                          inst.instance_parts)
    N, M = inst.nb_parts, inst.nb_machines
    dd = DeviceDecoder(packed, max_pop=96, pool_bins=8 * 96 * M)  # room for 8 plates per item
    chrom = torch.from_numpy(instances.chromosomes(96, N, 41)).cuda()
    ref = dd.decode(chrom).clone()
    torch.cuda.synchronize()
    assert int(dd.status.item()) == abi.OK
    out = torch.full((96,), -1.0, dtype=torch.float64, device="cuda")
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    assert _noalloc(torch, dd, chrom, out, None, status) == abi.OK
    torch.cuda.synchronize()
    assert int(status.item()) == abi.ERR_CAPACITY
    nan = torch.isnan(out)
    assert bool(nan.any()), "the pool should have run out for some rows"
    assert torch.equal(out[~nan], ref[~nan])
    small = chrom[:8].contiguous()
    out8 = torch.full((8,), -1.0, dtype=torch.float64, device="cuda")
    status.fill_(-1)
    assert _noalloc(torch, dd, small, out8, None, status) == abi.OK
    torch.cuda.synchronize()
    assert int(status.item()) == abi.OK
    assert torch.equal(out8, ref[:8])
