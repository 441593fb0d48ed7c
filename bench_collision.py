#!/usr/bin/env python
"""Collision-test paths timed side by side on the decoder's own chunks.

    python bench_collision.py [--workload P400M8] [--pop 8] [--limit 512] [--levels 0,1,2]

Decodes ``pop`` seeded chromosomes with placement logs, replays the plates
each part met, and times brkga_chunk_free on the resulting 32-row candidate
chunks (rotations with a side of at least 64 cells) through both paths — the
bit-packed run-dilation search (every word tested to the end) and the INT8
tensor-core correlation (tcgen05.mma kind::i8) — per mask-size bucket, after
checking that both give identical free-position words; each bucket's
chunks are repeated until one launch holds ``--target-chunks`` of them, so
the figures are throughput (GPU ns per chunk, and SM microseconds per
chunk), not the latency of a handful of chunks.  Beside the table:
the decode kernel's own GPU time per placement test on a population of 256
(one placement test = one rotation of one part on one plate; the kernel
stops at the first free placement of the bottom-most candidate).  Prints one
JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="P400M8")
    ap.add_argument("--pop", type=int, default=8)
    ap.add_argument("--limit", type=int, default=512)
    ap.add_argument("--levels", default="0,1,2")
    ap.add_argument("--repeats", type=int, default=5)
    ap.add_argument("--target-chunks", type=int, default=4736,
                    help="chunks per timed launch (each bucket's chunks repeated to fill the GPU)")
    args = ap.parse_args()
    import torch
    from brkga_fft2_b200 import abi, build, collision, instances, pack_problem
    from brkga_fft2_b200.evaluator import DeviceDecoder
    build.build()
    inst = instances.WORKLOADS[args.workload](0)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    P, N, M = args.pop, inst.nb_parts, inst.nb_machines
    dd = DeviceDecoder(pk, max_pop=max(P, 256))
    chrom = torch.from_numpy(instances.chromosomes(P, N, 77)).cuda()
    log = torch.empty((P, M, N, 5), dtype=torch.int32, device="cuda")
    dd.decode(chrom, log=log)
    torch.cuda.synchronize()
    log = log.cpu().numpy().view(abi.PLACEMENT_DTYPE).reshape(P, M, N)
    levels = tuple(int(v) for v in args.levels.split(","))
    cases = collision.chunk_cases(pk, log, min_side=64, levels=levels, limit=args.limit)
    table = collision.bucket_table(dd.native, pk, cases, target_chunks=args.target_chunks, repeats=args.repeats)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for r in table:  # SM time per chunk at throughput
        r["bitset_sm_us_per_chunk"] = r["bitset_ns_per_chunk"] * sms / 1e3
        r["int8_tc_sm_us_per_chunk"] = r["int8_tc_ns_per_chunk"] * sms / 1e3
    w = [r["chunks"] for r in table]
    mean_bit = float(np.average([r["bitset_ns_per_chunk"] for r in table], weights=w))
    mean_i8 = float(np.average([r["int8_tc_ns_per_chunk"] for r in table], weights=w))
    # the decode kernel's own rate: GPU time per placement test on 256 chromosomes
    pop = torch.from_numpy(instances.chromosomes(256, N, 78)).cuda()
    out = torch.empty(256, dtype=torch.float64, device="cuda")
    for _ in range(2):
        dd.decode(pop, out)
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dd.decode(pop, out, kernel_events=(k0, k1))
    torch.cuda.synchronize()
    tests = dd.counters()[0]
    kms = k0.elapsed_time(k1)
    print(json.dumps({
        "workload": args.workload, "chunks": len(cases), "levels": list(levels), "identical_words": True,
        "table": table, "all_buckets": {"bitset_ns_per_chunk": mean_bit, "int8_tc_ns_per_chunk": mean_i8,
                                        "int8_over_bitset": mean_i8 / mean_bit},
        "decoder_pop256": {"kernel_ms": kms, "placement_tests": tests, "ns_per_test": 1e6 * kms / tests,
                           "sm_us_per_test": 1e3 * kms * sms / tests},
        "build_id": abi.library_build_id()}))


if __name__ == "__main__":
    main()
