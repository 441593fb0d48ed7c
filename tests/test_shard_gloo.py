"""The multi-process path on the CPU: world_size 2 over gloo.  Each rank
decodes its row range with the CPU oracle (standing in for the GPU decoder)
and the all-gathered makespans equal a single-process decode; the timing
reduction returns the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from brkga_fft2_b200 import shard


def test_row_ranges_cover_population():
    for total in (0, 1, 7, 500):
        for world in (1, 2, 3, 8):
            spans = [shard.row_range(total, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            assert max(e - s for s, e in spans) - min(e - s for s, e in spans) <= 1
    with pytest.raises(ValueError):
        shard.row_range(5, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    import torch
    import torch.distributed as dist
    from brkga_fft2_b200 import instances, pack_problem
    from oracle import oracle_decode
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        inst = instances.small(8, n_parts=10)
        pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
        pop = torch.from_numpy(instances.chromosomes(23, inst.nb_parts, 5))
        fit = shard.ShardedDecode(lambda rows: oracle_decode(pk, rows.numpy()), dist)(pop)
        t = shard.max_over_ranks(1.0 + rank, dist)
        if rank == 0:
            np.savez(out_path, fit=fit.numpy(), t=t)
    finally:
        dist.destroy_process_group()


def test_sharded_decode_two_ranks(tmp_path):
    from brkga_fft2_b200 import instances, pack_problem
    from oracle import oracle_decode, build_oracle
    build_oracle()
    out = str(tmp_path / "r0.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    z = np.load(out)
    inst = instances.small(8, n_parts=10)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    ref = oracle_decode(pk, instances.chromosomes(23, inst.nb_parts, 5))
    np.testing.assert_array_equal(z["fit"], ref)
    assert float(z["t"]) == 2.0
    assert shard.weak_throughput(500, 2, 0.5) == 2000.0
