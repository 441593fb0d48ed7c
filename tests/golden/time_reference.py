"""Time the reference's own CPU decoder beside the oracle port on the rows the
benchmark times, one core each, and check that the two agree on them.

    python tests/golden/time_reference.py --reference /root/reference [--rows 12]

Only where the reference can be imported (its scripts, numba and torch): it
runs the reference's ``placementProcedure`` with the ``torch_cpu`` collision
backend and ``parallel=False`` (placement.py:94-165, collision_backend.py),
the path the reference's GA runs per chromosome, on the first rows of the
population of the benchmark's first timed step (P100M4, seeded synthetic
instance).  The first row is decoded once untimed (numba compiles on first
use).  The oracle (``oracle/brkga_oracle.c``) decodes the same rows on one
thread.  Prints one JSON line: both rates in decodes/s per core, their ratio,
and whether every makespan (==) and every placement agree.

With ``--workers W`` it also times the reference the way its GA spreads a
population over the host cores (``eval_mode="process"``, BRKGA_alg3.py:149-154):
a process pool of W workers, each holding its own copy of the problem (built,
and numba compiled, before the clock starts, so the pool's start-up and the
per-generation pickling the reference pays are left out), mapping the first
``--pool-rows`` rows of the same population; and the oracle on W threads on
those rows.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from make_golden import Reference, _pool_decode, bench_pool, log_to_array  # noqa: E402
from tests.goldens import part_ids_of_log  # noqa: E402


def pool_rates(reference, rows, workers, packed):
    """(reference rows/s over a process pool of `workers`, oracle rows/s on as many threads, equal?)."""
    from oracle import oracle_decode
    with bench_pool(reference, workers) as ex:
        list(ex.map(_pool_decode, rows[:workers]))  # every worker started and compiled
        t0 = time.perf_counter()
        ref_ms = np.array(list(ex.map(_pool_decode, rows)), np.float64)
        ref_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    ora_ms = oracle_decode(packed, rows, n_threads=workers)
    ora_s = time.perf_counter() - t0
    return len(rows) / ref_s, len(rows) / ora_s, bool(np.array_equal(ref_ms, ora_ms))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--rows", type=int, default=12)
    ap.add_argument("--workers", type=int, default=0)
    ap.add_argument("--pool-rows", type=int, default=96)
    args = ap.parse_args()
    import bench
    from brkga_fft2_b200 import instances
    from oracle import oracle_decode

    inst, packed = bench.load_workload()
    N, M = inst.nb_parts, inst.nb_machines
    # the population of the first timed step of `bench.py` (its default warm-up is 5 steps)
    rows = instances.chromosomes(bench.POP, N, bench.chrom_seed(0, 5))[: args.rows + 1]

    ref = Reference(args.reference)
    t0 = time.perf_counter()
    rpd = ref.problem(inst.problem_data, M)
    setup_s = time.perf_counter() - t0
    ref_ms, ref_logs = [], []
    ms, log = ref.decode(rpd, N, M, inst.thresholds, rows[0], inst.instance_parts)  # numba compiles here
    ref_ms.append(ms)
    ref_logs.append(log_to_array(log, M, N))
    t0 = time.perf_counter()
    for r in rows[1:]:
        ms, log = ref.decode(rpd, N, M, inst.thresholds, r, inst.instance_parts)
        ref_ms.append(ms)
        ref_logs.append(log_to_array(log, M, N))
    ref_s = time.perf_counter() - t0

    oracle_decode(packed, rows[:1], n_threads=1)
    t0 = time.perf_counter()
    ora_ms, ora_log = oracle_decode(packed, rows[1:], n_threads=1, with_log=True)
    ora_s = time.perf_counter() - t0
    ora_ms = np.concatenate([oracle_decode(packed, rows[:1], n_threads=1), ora_ms])
    _, log0 = oracle_decode(packed, rows[:1], n_threads=1, with_log=True)
    ora_log = np.concatenate([log0, ora_log]).reshape(len(rows), M, N)

    ref_ms = np.asarray(ref_ms, np.float64)
    ref_logs = np.stack(ref_logs)  # [rows, M, N, 5]: part, plate, x, bottom row, rotation; -1 past the count
    ours = part_ids_of_log(packed, ora_log)
    feasible = ref_ms < 1e15
    n = len(rows) - 1
    pool = {}
    if args.workers > 0:
        prow = instances.chromosomes(bench.POP, N, bench.chrom_seed(0, 5))[: args.pool_rows]
        r_rate, o_rate, same = pool_rates(args.reference, prow, args.workers, packed)
        pool = {"pool": {"workers": args.workers, "rows": len(prow),
                         "reference_decodes_per_s": r_rate, "oracle_decodes_per_s": o_rate,
                         "port_over_reference": o_rate / r_rate, "makespans_equal": same}}
    print(json.dumps({
        "workload": "P100M4 pop 500, rows 0..%d of the first timed step" % n,
        "reference": {"code": "placement.py placementProcedure, torch_cpu backend, parallel=False",
                      "decodes_per_s_per_core": n / ref_s, "rows_timed": n, "seconds": ref_s,
                      "problem_setup_s": setup_s},
        "oracle_port": {"code": "oracle/brkga_oracle.c, 1 thread", "decodes_per_s_per_core": n / ora_s,
                        "rows_timed": n, "seconds": ora_s},
        "port_over_reference": (n / ora_s) / (n / ref_s),
        "makespans_equal": bool(np.array_equal(ref_ms, ora_ms)),
        "placements_equal": bool((ref_logs[feasible] == ours[feasible]).all()),
        "feasible_rows": int(feasible.sum()), "rows": len(rows), **pool,
    }))


if __name__ == "__main__":
    main()
