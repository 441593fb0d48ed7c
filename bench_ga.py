#!/usr/bin/env python
"""Surrogate screening benchmark: time for the screened GPU GA to reach the
best makespan the plain GPU GA finds in its first G generations.

    python bench_ga.py [--workload P200M6] [--pop 1000] [--generations 200] [--seeds 3]
                       [--screened-limit 2.0] [--train-steps 8] [--explore 0] [--overlap 1]
                       [--features decode]

``--train-steps``, ``--explore``, ``--overlap`` and ``--features`` take comma
lists: every combination runs its own screened GA against the same plain run
per seed, and ``by_variant`` holds each one's medians.  ``--features``: the
surrogate's input, "decode" (per part in decode order its machine, proc time
and height time, plus per machine its loads) or "order" (per part its
sequencing key, area and height, parts sorted by key).  ``--screen-mode``:
"family" (every offspring slot's parent pair makes ``--oversample``
children and the surrogate keeps its best-predicted one) or "pool" (the
best-predicted rows of the whole oversampled pool; ``--screen-mutants`` and
``--explore`` apply there).

Both runs use the same instance, GA parameters (elites ceil(0.1 pop), mutants
ceil(0.15 pop), rho 0.7 as BRKGA_alg3.py:618) and decoder; each generation is
a CUDA-graph replay, timed with CUDA events on the GPU timeline.  The screened
run breeds an oversampled pool and decodes exactly only the best-predicted
rows; every makespan either run reports comes from the exact decoder.  The
screened run stops at the target or after screened-limit x generations; a run
that never reaches the target has ratio Infinity.

``ratio`` is the metric as specified: the screened run's time to the plain
run's 200-generation best over the plain run's time for all 200 generations.
When the plain run finds that best early and then stalls, a run identical to
it (screening never on: the screened GA then replays the plain GA exactly)
scores the same early fraction.  ``ratio_vs_plain_hit`` therefore divides by
the time at which the plain run itself first reached that makespan: below 1
only when screening got there sooner.  Prints one JSON line.
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
    ap.add_argument("--train-steps", default="8",
                    help="surrogate training steps per generation; a comma list runs one screened GA per value "
                         "against the same plain run")
    ap.add_argument("--explore", default="0",
                    help="share of the decoded rows spread over the lower-ranked pool; a comma list runs one "
                         "screened GA per value (and per training budget)")
    ap.add_argument("--overlap", default="1",
                    help="1: surrogate training beside the decode on a second stream, 0: after it; a comma list "
                         "runs one screened GA per value")
    ap.add_argument("--train-batch", type=int, default=512, help="rows per surrogate training step (multiple of 128)")
    ap.add_argument("--lr", type=float, default=1e-3, help="the surrogate's Adam learning rate")
    ap.add_argument("--spearman-threshold", type=float, default=0.3,
                    help="screening runs while the surrogate's recent Spearman is at least this")
    ap.add_argument("--check-every", type=int, default=5, help="generations between screening decisions")
    ap.add_argument("--warmup-generations", type=int, default=5, help="generations before screening may start")
    ap.add_argument("--screen-mode", default="family",
                    help="family: the surrogate picks one child per parent pair; pool: the best rows of the pool")
    ap.add_argument("--screen-mutants", type=int, default=0,
                    help="1: the surrogate screens mutants with the offspring; 0: mutants enter unscreened")
    ap.add_argument("--features", default="decode",
                    help="surrogate input: decode or order; a comma list runs one screened GA per value")
    ap.add_argument("--screened-limit", type=float, default=2.0,
                    help="the screened run may use up to this many times the plain run's generations")
    args = ap.parse_args()
    from brkga_fft2_b200 import build
    build.build()
    variants = [(int(t), float(x), int(o), f) for t in str(args.train_steps).split(",")
                for x in str(args.explore).split(",") for o in str(args.overlap).split(",")
                for f in str(args.features).split(",")]
    print(json.dumps(time_to_target(args.workload, args.pop, args.generations, args.seeds, args.oversample,
                                    variants, args.screened_limit, bool(args.screen_mutants), args.screen_mode,
                                    args.train_batch, args.lr,
                                    gate=(args.spearman_threshold, args.check_every, args.warmup_generations))))


def time_to_target(workload, P, generations, seeds, oversample=5, variants=((8, 0.0, 1, "decode"),),
                   screened_limit=2.0, screen_mutants=False, screen_mode="family", train_batch=512, lr=1e-3,
                   gate=(0.3, 5, 5)):
    """Plain GPU GA for `generations` generations, then each screened variant
    (train_steps, explore, overlap, surrogate features) against its best
    makespan, per seed; the record printed by this script (medians per
    variant and every run)."""
    import torch
    from brkga_fft2_b200 import instances, pack_problem
    from brkga_fft2_b200.ga import DeviceBRKGA
    inst = instances.WORKLOADS[workload](0)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    ne, nm = math.ceil(0.1 * P), math.ceil(0.15 * P)
    variants = [tuple(v) for v in variants]
    runs = []
    for seed in range(seeds):
        plain = DeviceBRKGA(None, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts,
                            num_generations=generations, num_individuals=P, num_elites=ne, num_mutants=nm,
                            eliteCProb=0.7, seed=seed, packed=pk)
        plain.fit()
        target = plain.best_fitness
        t_plain = plain.history["time"][-1]
        p_hit = int(np.flatnonzero(np.array(plain.history["min"]) <= target)[0])
        t_plain_hit = plain.history["time"][p_hit]
        del plain
        torch.cuda.empty_cache()
        for ts, ex, ov, ft in variants:
            runs.append(screened_run(generations, screened_limit, oversample, inst, pk, P, ne, nm, seed, ts, ex, ov,
                                     ft, target, t_plain, p_hit, t_plain_hit, screen_mutants, screen_mode,
                                     train_batch, lr, gate))
            torch.cuda.empty_cache()
    by_variant = {}
    for ts, ex, ov, ft in variants:
        rs = [r for r in runs if (r["train_steps"], r["explore"], r["overlap"], r["features"]) == (ts, ex, ov, ft)]
        by_variant[f"train_steps={ts},explore={ex:g},overlap={ov},features={ft}"] = {
            "ratio_median": float(np.median([r["ratio"] for r in rs])),
            "ratio_vs_plain_hit_median": float(np.median([r["ratio_vs_plain_hit"] for r in rs])),
            "spearman_median": float(np.nanmedian([r["spearman_median"] if r["spearman_median"] is not None
                                                   else np.nan for r in rs])),
            "screened_gen_ms_median": float(np.median([r["screened_gen_ms"] for r in rs])),
            "reached": sum(math.isfinite(r["ratio"]) for r in rs)}
    first = by_variant["train_steps={},explore={:g},overlap={},features={}".format(*variants[0])]
    return {"metric": "time to plain-GA best makespan, screened vs plain", "workload": workload,
            "pop": P, "generations": generations, "oversample": oversample,
            "screened_limit": screened_limit, "screen_mode": screen_mode, "screen_mutants": screen_mutants,
            "train_batch": train_batch, "lr": lr,
            "gate": {"spearman_threshold": gate[0], "check_every": gate[1], "warmup_generations": gate[2]},
            "train_steps": variants[0][0],
            "explore": variants[0][1], "overlap": variants[0][2], "features": variants[0][3], "seeds": seeds,
            "reached": first["reached"],
            "ratio_median": first["ratio_median"],
            "ratio_vs_plain_hit_median": first["ratio_vs_plain_hit_median"],
            "by_variant": by_variant, "runs": runs}


def screened_run(generations, screened_limit, oversample, inst, pk, P, ne, nm, seed, train_steps, explore, overlap,
                 features, target, t_plain, p_hit, t_plain_hit, screen_mutants=False, screen_mode="family",
                 train_batch=512, lr=1e-3, gate=(0.3, 5, 5)):
    """One screened GA against the plain run's target; a dict for the JSON line."""
    from brkga_fft2_b200.ga import DeviceBRKGA
    scr = DeviceBRKGA(None, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts,
                      num_generations=max(1, int(round(generations * screened_limit))),
                      num_individuals=P, num_elites=ne, num_mutants=nm,
                      eliteCProb=0.7, seed=seed, packed=pk, screening=True, oversample=oversample,
                      train_steps=train_steps, explore=explore, overlap_training=bool(overlap), target=target,
                      surrogate_features=features, screen_mutants=screen_mutants, screen_mode=screen_mode,
                      train_batch=train_batch, lr=lr, spearman_threshold=gate[0], check_every=gate[1],
                      warmup_generations=gate[2])
    scr.fit()
    mins = np.array(scr.history["min"])
    hit = np.flatnonzero(mins <= target)
    t_scr = scr.history["time"][int(hit[0])] if hit.size else float("inf")
    sp = np.array(scr.history["spearman"][1:])
    return {"seed": seed, "train_steps": train_steps, "explore": explore, "overlap": overlap, "features": features,
            "target": target,
            "plain_s": t_plain,
            "plain_gen_ms": 1000 * t_plain / generations,
            "screened_s": t_scr, "screened_generations": int(hit[0]) if hit.size else None,
            "screened_best": float(mins.min()), "ratio": t_scr / t_plain,
            "plain_hit_generation": p_hit, "plain_hit_s": t_plain_hit,
            "ratio_vs_plain_hit": t_scr / t_plain_hit if t_plain_hit > 0 else float("inf"),
            "screened_gen_ms": 1000 * scr.history["time"][-1] / max(len(mins) - 1, 1),
            "screen_fraction": float(np.mean([m == "screen" for m in scr.history["mode"][1:]])),
            "spearman_median": float(np.nanmedian(sp)) if np.isfinite(sp).any() else None,
            "mae_median": float(np.nanmedian(scr.history["mae"][1:]))}


if __name__ == "__main__":
    main()
