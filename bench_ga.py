#!/usr/bin/env python
"""Surrogate screening benchmark: time for the screened GPU GA to reach the
best makespan the plain GPU GA finds in its first G generations.

    python bench_ga.py [--workload P200M6] [--pop 1000] [--generations 200] [--seeds 3]

Both runs use the same instance, GA parameters (elites ceil(0.1 pop), mutants
ceil(0.15 pop), rho 0.7 as BRKGA_alg3.py:618) and decoder; each generation is
a CUDA-graph replay, timed with CUDA events on the GPU timeline.  The screened
run breeds an oversampled pool and decodes exactly only the best-predicted
rows; every makespan either run reports comes from the exact decoder.
Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="P200M6")
    ap.add_argument("--pop", type=int, default=1000)
    ap.add_argument("--generations", type=int, default=200)
    ap.add_argument("--seeds", type=int, default=3)
    ap.add_argument("--oversample", type=int, default=5)
    ap.add_argument("--train-steps", type=int, default=8)
    args = ap.parse_args()
    import torch
    from brkga_fft2_b200 import build, instances, pack_problem
    from brkga_fft2_b200.ga import DeviceBRKGA
    build.build()
    inst = instances.WORKLOADS[args.workload](0)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    P = args.pop
    ne, nm = math.ceil(0.1 * P), math.ceil(0.15 * P)
    runs = []
    for seed in range(args.seeds):
        plain = DeviceBRKGA(None, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts,
                            num_generations=args.generations, num_individuals=P, num_elites=ne, num_mutants=nm,
                            eliteCProb=0.7, seed=seed, packed=pk)
        plain.fit()
        target = plain.best_fitness
        t_plain = plain.history["time"][-1]
        scr = DeviceBRKGA(None, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts,
                          num_generations=args.generations, num_individuals=P, num_elites=ne, num_mutants=nm,
                          eliteCProb=0.7, seed=seed, packed=pk, screening=True, oversample=args.oversample,
                          train_steps=args.train_steps, target=target)
        scr.fit()
        mins = np.array(scr.history["min"])
        hit = np.flatnonzero(mins <= target)
        t_scr = scr.history["time"][int(hit[0])] if hit.size else float("inf")
        # best makespan of each run at the plain run's wall time
        sp = np.array(scr.history["spearman"][1:])
        runs.append({"seed": seed, "target": target, "plain_s": t_plain, "plain_gen_ms": 1000 * t_plain / args.generations,
                     "screened_s": t_scr, "screened_generations": int(hit[0]) if hit.size else None,
                     "screened_best": float(mins.min()), "ratio": t_scr / t_plain,
                     "screened_gen_ms": 1000 * scr.history["time"][-1] / max(len(mins) - 1, 1),
                     "screen_fraction": float(np.mean([m == "screen" for m in scr.history["mode"][1:]])),
                     "spearman_median": float(np.nanmedian(sp)) if np.isfinite(sp).any() else None,
                     "mae_median": float(np.nanmedian(scr.history["mae"][1:]))})
        torch.cuda.empty_cache()
    ratios = [r["ratio"] for r in runs]
    print(json.dumps({"metric": "time to plain-GA best makespan, screened vs plain", "workload": args.workload,
                      "pop": P, "generations": args.generations, "oversample": args.oversample,
                      "ratio_median": float(np.median(ratios)), "runs": runs}))


if __name__ == "__main__":
    main()
