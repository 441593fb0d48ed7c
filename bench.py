#!/usr/bin/env python
"""Decoder throughput benchmark: decodes/s at P100M4, population 500.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step decodes one population of 500 seeded synthetic chromosomes of the
P100M4 workload (100 parts with masks up to 120x120 cells, two 300x300 and
two 250x250 plates).  ``value`` times the device path with the populations
already in HBM (CUDA events, L2 flushed by a 256 MiB write between steps);
``e2e`` times the drop-in ``evaluate_batch`` call with host buffers (H2D copy
of the chromosomes and D2H of the makespans inside the timed region).  Under
torchrun every rank decodes its own populations (weak scaling, no data-path
collective); the time is the max over ranks.

``--impl reference`` times the CPU restatement of the reference decoder on the
host cores instead (the reference itself is Python and cannot be shipped).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

WORKLOAD = "P100M4"
METRIC = "decodes/s at P100M4 pop 500"
UNIT = "decodes/s"
POP = 500
INSTANCE_SEED = 0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pop", type=int, default=POP)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def chrom_seed(rank: int, step: int) -> int:
    from brkga_fft2_b200.shard import rank_seed
    return rank_seed(rank, step)


def load_workload():
    from brkga_fft2_b200 import instances, pack_problem
    inst = instances.p100m4(INSTANCE_SEED)
    packed = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                          inst.instance_parts)
    return inst, packed


def workload_config(pop: int, world: int) -> dict:
    """The `config` record both arms print: the same workload, whichever arm runs it."""
    return {"workload": f"{WORKLOAD} pop {pop}", "parts": 100, "machines": 4, "plates": "2x300x300 + 2x250x250",
            "mask_bbox_max": 120, "l2": "flushed (256 MiB write) between timed steps",
            "parallelism": f"dp{world} (shards)"}


def measured_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_rate(packed, n_parts, seconds, threads, seed=12345):
    """Decodes/s of the CPU oracle on a bounded sample of the workload."""
    from brkga_fft2_b200 import instances
    from oracle import oracle_decode
    probe = instances.chromosomes(threads, n_parts, seed)
    t0 = time.perf_counter()
    oracle_decode(packed, probe, n_threads=threads)
    dt = time.perf_counter() - t0
    n = int(max(threads, min(20 * threads * 50, threads * round(seconds / max(dt, 1e-3)))))
    sample = instances.chromosomes(n, n_parts, seed + 1)
    t0 = time.perf_counter()
    oracle_decode(packed, sample, n_threads=threads)
    dt = time.perf_counter() - t0
    return n / dt, n, dt


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples (every 20 ms, timestamped)
    around the timed region; only the samples taken inside it are reported."""
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        self.t0 = self.t1 = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "20", "-i", str(gpu_index)],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        deadline = time.time() + 5.0  # the first sample shows the sampler is running before the timing starts
        while time.time() < deadline and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
            time.sleep(0.01)

    def mark_start(self):
        self.t0 = datetime.datetime.now()

    def mark_end(self):
        self.t1 = datetime.datetime.now()

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.05)  # one more sample after the region
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f")
                rows.append((ts, float(parts[2]), float(parts[3]), parts[6:10]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        inside = [r for r in rows if self.t0 is not None and self.t1 is not None and self.t0 <= r[0] <= self.t1]
        use = inside or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, _, r in use for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[1] for r in use), "sm_max_mhz": max(r[2] for r in use),
                "reasons": reasons, "samples": len(use), "in_timed_region": bool(inside),
                "interval_ms": 20}


def profile_traffic():
    """dram bytes per decode-kernel launch from the committed ncu summary, if any."""
    path = os.path.join(HERE, "profiles", "decode_kernel_P100M4.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_launch")
    return None


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle_decode
    from brkga_fft2_b200 import instances
    inst, packed = load_workload()
    threads = os.cpu_count() or 1
    # size each step for ~2 s of CPU work
    probe = instances.chromosomes(threads, inst.nb_parts, 99)
    t0 = time.perf_counter()
    oracle_decode(packed, probe, n_threads=threads)
    rate = threads / (time.perf_counter() - t0)
    n = int(min(args.pop, max(threads, threads * round(2.0 * rate / threads))))
    for s in range(args.warmup):
        oracle_decode(packed, instances.chromosomes(n, inst.nb_parts, chrom_seed(0, s)), n_threads=threads)
    total = 0.0
    for s in range(args.steps):
        ch = instances.chromosomes(n, inst.nb_parts, chrom_seed(0, args.warmup + s))
        t0 = time.perf_counter()
        oracle_decode(packed, ch, n_threads=threads)
        total += time.perf_counter() - t0
    value = n * args.steps / total
    sample = f"{n} of the {args.pop} chromosomes per step ({WORKLOAD}, instance seed {INSTANCE_SEED})"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator, P100M4 shapes)",
        "config": workload_config(args.pop, args.gpus),
        "sample_per_step": n,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    from brkga_fft2_b200 import build as libbuild
    libbuild.build()
    from brkga_fft2_b200 import instances
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator, DeviceDecoder

    inst, packed = load_workload()
    P, N = args.pop, inst.nb_parts
    dd = DeviceDecoder(packed, max_pop=P)
    host = [instances.chromosomes(P, N, chrom_seed(rank, s)) for s in range(args.warmup + args.steps)]
    dev = [torch.from_numpy(h).cuda() for h in host]
    out = torch.empty(P, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    for s in range(args.warmup):
        dd.decode(dev[s], out)
    torch.cuda.synchronize()
    if int(dd.status.item()) != 0:
        raise RuntimeError(f"decode status {int(dd.status.item())}")

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    sampler = ClockSampler(local)
    barrier()
    sampler.mark_start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    tests = chunks = scan = 0
    for s in range(args.steps):
        flush.fill_(s & 0xFF)  # evict the previous step's data from the 126 MB L2
        e0, k0, k1, e1 = ev[s]
        e0.record(stream)
        dd.decode(dev[args.warmup + s], out, kernel_events=(k0, k1))
        e1.record(stream)
    torch.cuda.synchronize()
    sampler.mark_end()
    step_ms = [e0.elapsed_time(e1) for e0, _, _, e1 in ev]
    kern_ms = [k0.elapsed_time(k1) for _, k0, k1, _ in ev]
    barrier()
    clocks = sampler.stop()
    status = int(dd.status.item())
    tests, chunks, bins, scan = dd.counters()  # counters of the last step

    from brkga_fft2_b200.shard import max_over_ranks, weak_throughput
    total_ms = max_over_ranks(sum(step_ms), dist, "cuda")
    value = weak_throughput(P * args.steps, world, total_ms / 1000.0)

    # e2e through the drop-in evaluator (host buffers, pinned input)
    evaluator = B200DecoderEvaluator(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                                     inst.instance_parts)
    pinned = [torch.from_numpy(h).pin_memory().numpy() for h in host]
    for s in range(args.warmup):
        evaluator.evaluate_batch(pinned[s])
    barrier()
    e2e_t = 0.0
    last = None
    for s in range(args.steps):
        flush.fill_(s & 0xFF)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        last = evaluator.evaluate_batch(pinned[args.warmup + s])
        e2e_t += time.perf_counter() - t0
    e2e_value = weak_throughput(P * args.steps, world, max_over_ranks(e2e_t, dist, "cuda"))
    ref_last = out.cpu().numpy()
    same = bool(np.array_equal(np.asarray(last), ref_last))

    if rank == 0:
        hbm_peak, peak_kind = measured_peaks()
        kern_avg_s = statistics.mean(kern_ms) / 1000.0
        achieved = scan / kern_avg_s / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generator, P100M4 shapes)",
            "config": workload_config(P, world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": profile_traffic(),
                         "kernel": "decode_kernel", "kernel_ms": statistics.mean(kern_ms),
                         "algorithmic_bytes_per_launch": scan, "tests_per_launch": tests,
                         "placement_tests_per_s": tests / kern_avg_s,
                         "peak_source": peak_kind,
                         "note": "algorithmic bytes = per placement test one read of the bit-packed plate "
                                 "and rotated mask, 4*(L*ceil(W/32)+h*ceil(w/32))"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": P * 2 * N * 4,
                    "d2h_bytes_per_step": P * 8, "matches_device_path": same},
            "gpu_launches": 4 * args.steps,  # assign_sort, order_items, decode, reduce per step
            "kernel_share": statistics.mean(kern_ms) / statistics.mean(step_ms),
            "counters_last_step": {"tests": tests, "row_chunks": chunks, "plates": bins},
            "status": status,
        }
        if clocks:
            line["clocks"] = clocks
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            rate, n, dt = cpu_rate(packed, N, args.cpu_seconds, threads)
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                    "sample": f"{n} seeded {WORKLOAD} chromosomes decoded by the C oracle "
                                              f"on {threads} threads in {dt:.1f} s"}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
