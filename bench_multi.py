"""Uneven batched decode: many independent instances, one launch per generation.

    python bench_multi.py [--instances 64] [--pop 256] [--generations 100] [--no-tune]

Workload: 64 seeded instances (part counts U[25,200], machines U[1,6],
square plates of 150 to 500 cells a side, per-machine time constants
x U(0.8,1.2)), population 256 each, elites 20 %, mutants 15 %, rho 0.7.
Every generation of all 64 GAs — 64 ranks, 64 breeds, one decode of the
non-elite rows of all instances, 64 statistics — is one CUDA graph replay.
The decode kernel's launch shape comes from the autotuner (timed on one
random population per instance) unless --no-tune.

Prints one JSON line: decodes/s over the whole GA run (device time), the
device time per generation, the one-launch decode throughput of a full
population per instance, the chosen launch shape with the autotuner's table,
and a cross-check of a 1 % sample of the final populations against each
instance decoded alone (single-instance problem, host-to-host entry point).
Bit-exactness against the reference decoder is the tests' job
(tests/test_multi_gpu.py, tests/test_multi_ga_gpu.py).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--pop", type=int, default=256)
    ap.add_argument("--generations", type=int, default=100)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--tune-cache", default=None)
    args = ap.parse_args()

    import torch
    from brkga_fft2_b200 import build, instances, pack_problem
    from brkga_fft2_b200.autotune import autotune
    from brkga_fft2_b200.evaluator import MultiDecoder
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator
    from brkga_fft2_b200.multi_ga import MultiBRKGA

    build.build()
    K, P, G = args.instances, args.pop, args.generations
    insts = [instances.uneven(s) for s in range(K)]
    packs = [pack_problem(i.problem_data, i.nb_parts, i.nb_machines, i.thresholds, i.instance_parts) for i in insts]
    pops = [P] * K
    chroms = [instances.chromosomes(P, i.nb_parts, 1000 + k) for k, i in enumerate(insts)]
    flat = torch.from_numpy(np.concatenate([c.reshape(-1) for c in chroms])).cuda()

    # one launch over full populations: throughput and autotuning
    md = MultiDecoder(packs, max_pops=pops, pool_bins=4 * sum(P * i.nb_machines for i in insts))
    tune = None
    if not args.no_tune:
        tune = autotune(md, flat, pops, cache_path=args.tune_cache)
    shape = md.launch_config()
    out = torch.empty(K * P, dtype=torch.float64, device="cuda")
    times, ktimes = [], []
    for it in range(6):
        e0, e1, k0, k1 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record()
        md.decode_concat(flat, pops, out=out, kernel_events=(k0, k1))
        e1.record()
        torch.cuda.synchronize()
        if it >= 2:
            times.append(e0.elapsed_time(e1))
            ktimes.append(k0.elapsed_time(k1))
    launch_ms, kernel_ms = float(np.median(times)), float(np.median(ktimes))
    counters = md.counters()

    ga = MultiBRKGA(packs, num_generations=G, num_individuals=P, eliteCProb=0.7, seed=args.seed,
                    launch_config=(shape[0], shape[1], shape[2], shape[4]) if tune else None)
    t0 = time.perf_counter()
    ga.prepare()
    prep_s = time.perf_counter() - t0
    ga.fit()
    gen_ms = float(np.sum(ga.generation_ms))
    decoded = sum(P - e for e in ga.ne) * G
    # a 1 % sample of the final populations, each instance decoded alone
    rng = np.random.default_rng(7)
    n_ok = n_chk = 0
    for k, inst in enumerate(insts):
        rows = rng.choice(P, size=max(1, round(0.01 * P)), replace=False)
        alone = B200DecoderEvaluator(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                                     inst.instance_parts)
        ref = np.asarray(alone.evaluate_batch(ga.populations[k][rows]))
        alone.close()
        n_chk += rows.size
        n_ok += int(np.sum(ref == ga.fitness[k][rows]))
    line = {
        "metric": "decodes/s, uneven batched GA (instances x pop, one graph per generation)",
        "value": decoded / (gen_ms / 1000.0),
        "unit": "decodes/s",
        "instances": K, "pop": P, "generations": G,
        "ms_per_generation": gen_ms / G,
        "initial_ms": ga.initial_ms,
        "graph_capture_s": prep_s,
        "one_launch": {"rows": K * P, "ms": launch_ms, "decode_kernel_ms": kernel_ms,
                       "decodes_per_s": K * P / (launch_ms / 1000.0),
                       "placement_tests": counters[0], "plates": counters[2]},
        "launch_config": {"warps_per_item": shape[0], "ctas_per_sm": shape[1], "smem_plates": shape[2],
                          "resident_ctas": shape[3], "task_max": shape[4]},
        "autotune": None if tune is None else {"table": tune["table"], "cached": tune["cached"]},
        "sample_matches_single_instance_decode": f"{n_ok}/{n_chk}",
        "parts": [i.nb_parts for i in insts], "machines": [i.nb_machines for i in insts],
        "data": "synthetic (seeded generator)",
    }
    print(json.dumps(line))
    if n_ok != n_chk:
        sys.exit(1)


if __name__ == "__main__":
    main()
