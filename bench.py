#!/usr/bin/env python
"""Decoder throughput benchmark: decodes/s at P100M4, population 500.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step decodes one population of 500 seeded synthetic chromosomes of the
P100M4 workload (100 parts with masks up to 120x120 cells, two 300x300 and
two 250x250 plates).  ``value`` times the device path with the populations
already in HBM (CUDA events, L2 flushed by a 256 MiB write between steps).
``e2e`` times the drop-in ``evaluate_batch`` call the way the reference's GA
makes it (BRKGA_alg3.py:119-123: a fresh pageable ``np.array`` of the
population), host-to-device copy of the chromosomes and device-to-host copy
of the makespans inside the timed region; ``e2e_pinned`` is the same call on
page-locked input.  ``parity`` decodes the rows of the first and the last
timed step again with placement logs and compares makespans and every
placement with the CPU oracle (the run fails on any difference); the oracle's
time on those rows is the ``cpu_baseline``.  ``roofline`` scores the decode
kernel against the resource that bounds it, integer-ALU issue on chip, with
its on-chip scan rate against the shared-memory bandwidth measured by this
library's own streaming probe beside it, and HBM traffic as a check that
memory does not bound it.  ``time_to_target`` runs the plain GPU GA for 200
generations and the surrogate-screened GA (family screening: 8 children per
parent pair, the best-predicted one kept; 6 training steps a generation)
against its best makespan, eleven seeds (the median of a few seeds moves with
any change of the surrogate's arithmetic, which changes every screened
trajectory).
Under torchrun every rank decodes its own populations (weak scaling, no
data-path collective); the time is the max over ranks.

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
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the oracle leg (parity check of the timed rows and the CPU baseline)")
    ap.add_argument("--no-ttt", action="store_true", help="skip the time-to-target record")
    ap.add_argument("--ttt-seeds", type=int, default=11)
    ap.add_argument("--ttt-generations", type=int, default=200)
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


# What the CPU figures time, said in the JSON line itself.
CPU_CODE = "oracle/brkga_oracle.c"
CPU_NOTE = ("the C restatement (port) of the reference's sequential decoder, placement.py:94-165 with "
            "binClassNew.py:45-174; not the reference's own Python placementProcedure + numba + torch_cpu path, "
            "which cannot be installed or shipped to this box; on one core of the build host and this "
            "benchmark's own first rows that path decodes 1.45 rows/s and the port 5.53, with equal makespans "
            "and placements, and on its 8 cores 11.1 rows/s through the reference's process pool against "
            "41.7 for the port on 8 threads (tests/golden/time_reference.py): the port is about 3.8x faster; "
            "on the reference's real P100M4-0 instance the path's single-core rate is 1.33 decodes/s")


def measured_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_peaks_bf16():
    """Dense bf16 tensor-core peak in TFLOP/s: the burst figure of MEASURED_PEAKS.json, else the fallback."""
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["bf16_tflops"])
    return 1590.0


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples (every 5 ms asked, as fast
    as nvidia-smi answers; timestamped) around the timed region; only the
    samples taken inside it are reported."""
    INTERVAL_MS = 5
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
                                          "-lms", str(self.INTERVAL_MS), "-i", str(gpu_index)],
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
                "interval_ms": self.INTERVAL_MS}


def decode_profile():
    """Per-launch counters of the decode kernel on this workload from the
    committed ncu summary (instruction counts, DRAM bytes, pipe peaks), or {}."""
    path = os.path.join(HERE, "profiles", "decode_kernel_P100M4.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def smem_probe(torch, lib, sm_count):
    """Shared-memory bandwidth of this GPU from the library's streaming probe
    (brkga_probe_smem_stream): GB/s over the whole GPU and bytes per SM clock."""
    import ctypes
    blocks, threads, iters = 2 * sm_count, 1024, 1024
    sink = torch.empty(blocks * threads, dtype=torch.int32, device="cuda")
    cycles = torch.empty(blocks, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()

    def launch():
        st = lib.brkga_probe_smem_stream(blocks, threads, iters, ctypes.c_void_p(sink.data_ptr()),
                                         ctypes.c_void_p(cycles.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        if st != 0:
            raise RuntimeError(f"brkga_probe_smem_stream: status {st}")

    for _ in range(3):
        launch()
    times = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launch()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1000.0)
    nbytes = blocks * threads * iters * 128
    gbs = nbytes / statistics.median(times) / 1e9
    # per SM and clock: one CTA's bytes over its own load-loop cycles (CTAs of
    # 1024 threads run one at a time per SM)
    per_clk = threads * iters * 128 / float(cycles.max().item())
    return {"gbs": gbs, "bytes_per_clk_per_sm": per_clk, "kernel": "smem_stream_kernel", "bytes_per_launch": nbytes,
            "launch": f"{blocks}x{threads}"}


def roofline_record(prof, kern_s, scan, tests, sm_count, sm_mhz, smem, hbm_peak, peak_kind, build_id):
    """The decode kernel against the resource that bounds it: integer-ALU issue.

    achieved = ALU-pipe warp instructions of one launch (ncu count of this
    workload, committed in profiles/) over the launch's live CUDA-event time;
    peak = SMs x the ALU pipe's warp instructions per SM cycle (ncu's peak
    for this pipe) x the SM clock sampled during the timed region.  The
    profile holds for the decoder sources it was captured from
    (`profile_matches_build` compares their hash).  Beside it:
    all warp instructions against the 4-per-cycle issue limit of an SM, the
    on-chip scan bytes against the measured shared-memory bandwidth, and the
    DRAM traffic against HBM."""
    rec = {"bound": "int_alu", "unit": "G warp-instructions/s", "kernel": "decode_kernel",
           "kernel_ms": kern_s * 1000.0, "tests_per_launch": tests, "placement_tests_per_s": tests / kern_s}
    alu = prof.get("alu_warp_inst_per_launch")
    alu_peak = prof.get("alu_peak_warp_inst_per_cycle_per_sm")
    clock_hz = (sm_mhz or prof.get("sm_mhz", 1965.0)) * 1e6
    if alu and alu_peak:
        achieved = alu / kern_s / 1e9
        peak = sm_count * alu_peak * clock_hz / 1e9
        rec.update({"achieved": achieved, "peak": peak, "frac": achieved / peak,
                    "alu_warp_inst_per_launch": alu, "alu_peak_warp_inst_per_cycle_per_sm": alu_peak,
                    "sm_clock_mhz": clock_hz / 1e6})
    else:
        rec.update({"achieved": None, "peak": None, "frac": None,
                    "note_missing": "no ALU instruction count in profiles/decode_kernel_P100M4.json"})
    inst = prof.get("warp_inst_per_launch")
    if inst:
        issue = inst / kern_s / 1e9
        issue_peak = sm_count * 4 * clock_hz / 1e9
        rec["issue"] = {"achieved": issue, "peak": issue_peak, "frac": issue / issue_peak,
                        "unit": "G warp-instructions/s", "warp_inst_per_launch": inst}
    scan_gbs = scan / kern_s / 1e9
    rec["smem"] = {"achieved": scan_gbs, "peak": smem["gbs"], "frac": scan_gbs / smem["gbs"], "unit": "GB/s",
                   "algorithmic_bytes_per_launch": scan, "peak_source": "measured (brkga_probe_smem_stream)",
                   "note": "algorithmic bytes = per placement test one read of the bit-packed plate and rotated "
                           "mask, 4*(L*ceil(W/32)+h*ceil(w/32)); the kernel stops early, so this is a scan "
                           "rate, not traffic"}
    if prof.get("smem_bytes_per_launch"):  # bytes the shared-memory instructions moved (ncu), not the scan model
        rec["smem"]["actual_bytes_per_launch"] = prof["smem_bytes_per_launch"]
        rec["smem"]["actual_gbs"] = prof["smem_bytes_per_launch"] / kern_s / 1e9
        rec["smem"]["actual_frac"] = rec["smem"]["actual_gbs"] / smem["gbs"]
    if prof.get("l2_bytes_per_launch"):
        rec["l2"] = {"achieved": prof["l2_bytes_per_launch"] / kern_s / 1e9, "unit": "GB/s",
                     "bytes_per_launch": prof["l2_bytes_per_launch"],
                     "l1_global_bytes_per_launch": prof.get("l1_global_bytes_per_launch"),
                     "note": "L2 requests (lts__t_bytes); no measured L2 peak on this pool"}
    traffic = prof.get("dram_bytes_per_launch")
    rec["traffic"] = traffic
    if traffic:
        rec["hbm"] = {"achieved": traffic / kern_s / 1e9, "peak": hbm_peak, "frac": traffic / kern_s / 1e9 / hbm_peak,
                      "unit": "GB/s", "peak_source": peak_kind, "dram_bytes_per_launch": traffic}
    from brkga_fft2_b200.build import decoder_source_id
    rec["profile_build_id"] = prof.get("build_id")
    rec["profile_decoder_source_id"] = prof.get("decoder_source_id")
    rec["profile_matches_build"] = prof.get("decoder_source_id") == decoder_source_id()
    return rec


def surrogate_record(torch, dd, inst, bf16_peak, steps=6, batch=512, n_pred=3600):
    """The surrogate's tensor-core work on this workload, timed alone as CUDA
    graph replays: `steps` training steps of `batch` rows (five tcgen05 GEMMs
    each) and one prediction of `n_pred` rows (two), as FLOP/s of their GEMMs
    against the dense bf16 peak."""
    from brkga_fft2_b200 import instances
    from brkga_fft2_b200.surrogate import Surrogate
    sur = Surrogate(dd.native, max_batch=4096, buffer_capacity=20000, seed=11)
    rows = torch.from_numpy(instances.chromosomes(4096, inst.nb_parts, 777)).cuda()
    ms = torch.empty(4096, dtype=torch.float64, device="cuda")
    for off in range(0, 4096, dd.max_pop):
        dd.decode(rows[off:off + dd.max_pop], ms[off:off + dd.max_pop])
    sur.observe(rows, ms)
    side = torch.cuda.Stream()
    pred = torch.empty(n_pred, dtype=torch.float64, device="cuda")
    I = sur.in_pad
    jobs = {"train": (lambda: sur.train(steps, batch, 1e-3, stream=side),
                      steps * 2.0 * batch * (2 * 512 * I + 3 * 256 * 512)),
            "predict": (lambda: sur.predict(rows[:n_pred], out=pred, stream=side), 2.0 * n_pred * (512 * I + 256 * 512))}
    rec = {"workload": f"P100M4 features ({I} inputs), MLP {I}-512-256-1 bf16, fp32 accumulation",
           "peak_tflops": bf16_peak, "peak_source": "measured bf16 burst (MEASURED_PEAKS.json)"}
    torch.cuda.synchronize()
    for name, (fn, flops) in jobs.items():
        with torch.cuda.stream(side):
            fn()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            fn()
        for _ in range(3):
            g.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(side)
        with torch.cuda.stream(side):
            for _ in range(20):
                g.replay()
        e1.record(side)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1000.0 / 20
        tf = flops / sec / 1e12
        rec[name] = {"us": sec * 1e6, "gemm_flops": flops, "tflops": tf,
                     "frac": tf / bf16_peak if bf16_peak else None}
    rec["train"]["steps"], rec["train"]["batch"] = steps, batch
    rec["predict"]["rows"] = n_pred
    sur.close()
    return rec


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle_decode
    from brkga_fft2_b200 import instances
    inst, packed = load_workload()
    threads = os.cpu_count() or 1
    # size each step for ~3 s of CPU work, from a probe of four rows per thread
    probe = instances.chromosomes(4 * threads, inst.nb_parts, 99)
    t0 = time.perf_counter()
    oracle_decode(packed, probe, n_threads=threads)
    rate = 4 * threads / (time.perf_counter() - t0)
    n = int(min(args.pop, max(threads, threads * round(3.0 * rate / threads))))
    for s in range(args.warmup):
        oracle_decode(packed, instances.chromosomes(n, inst.nb_parts, chrom_seed(0, s)), n_threads=threads)
    total = 0.0
    for s in range(args.steps):
        ch = instances.chromosomes(n, inst.nb_parts, chrom_seed(0, args.warmup + s))
        t0 = time.perf_counter()
        oracle_decode(packed, ch, n_threads=threads)
        total += time.perf_counter() - t0
    value = n * args.steps / total
    sample = (f"the first {n} of the {args.pop} chromosomes of each step ({WORKLOAD}, instance seed "
              f"{INSTANCE_SEED}), {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator, P100M4 shapes)",
        "config": workload_config(args.pop, args.gpus),
        "sample_per_step": n,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "code": CPU_CODE,
                         "note": CPU_NOTE, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# The reference's own makespans of the populations of the first and last timed
# steps under the default warm-up and step counts (populations 5 and 24), made
# by running the reference's decoder (tests/golden/make_golden.py).
REFERENCE_FIXTURES = {5: "refms_bench_P100M4_step0", 24: "refms_bench_P100M4_step19"}


def reference_anchor(step_makespans):
    """Compare GPU makespans of whole timed populations, given as (population
    index, makespans) pairs, with the reference's own where a fixture holds that
    population (same seed and size); other populations are skipped."""
    import numpy as np
    rows = exact = 0
    used = []
    for step, ms in step_makespans:
        tag = REFERENCE_FIXTURES.get(int(step))
        path = os.path.join(HERE, "tests", "golden", f"{tag}.npz") if tag else ""
        if not path or not os.path.exists(path):
            continue
        z = np.load(path)
        ms = np.asarray(ms, np.float64)
        if int(z["seed"]) != chrom_seed(0, int(step)) or int(z["pop"]) != ms.shape[0]:
            continue
        rows += ms.shape[0]
        exact += int((ms == z["makespans"]).sum())
        used.append(tag)
    return {"rows": rows, "exact": exact, "fixtures": used,
            "checked": "GPU makespans (==) against the reference's own sequential decoder (placement.py "
                       "placementProcedure, torch_cpu backend) run on the same rows when the fixtures were made"}


def parity_and_cpu(dd, packed, host_rows, P, M, N, torch, step_ids=()):
    """Decode the given host populations again on the GPU with placement logs
    and with the CPU oracle on all host threads; compare every makespan and
    every placement, and the makespans with the reference's own where a
    fixture holds the population (``step_ids``: their population indices).
    Returns (parity record, cpu_baseline record)."""
    import numpy as np
    from oracle import oracle_decode
    threads = os.cpu_count() or 1
    rows = exact = placements_bad = 0
    cpu_s = 0.0
    gpu_ms = []
    for h in host_rows:
        dev = torch.from_numpy(h).cuda()
        log = torch.empty((P, M, N, 5), dtype=torch.int32, device="cuda")
        ms = dd.decode(dev, log=log).cpu().numpy()
        gpu_ms.append(ms)
        glog = log.cpu().numpy()
        t0 = time.perf_counter()
        rms, rlog = oracle_decode(packed, h, n_threads=threads, with_log=True)
        cpu_s += time.perf_counter() - t0
        rl = np.stack([rlog[f] for f in ("gene", "bin", "x", "y", "rot")], axis=-1)
        same_row = np.array([np.array_equal(a, b) for a, b in zip(ms, rms)])
        same_log = (glog == rl).reshape(P, -1).all(axis=1)
        rows += P
        exact += int(same_row.sum())
        placements_bad += int((~same_log).sum())
    parity = {"rows": rows, "exact": exact, "placements_exact": placements_bad == 0,
              "rows_with_placement_differences": placements_bad,
              "checked": "every makespan (==) and every placement (gene, plate, x, bottom row y, rotation) of "
                         "the first and last timed steps' populations against the CPU oracle"}
    try:
        parity["reference"] = reference_anchor(list(zip(step_ids, gpu_ms)))
    except Exception as exc:  # a report, never a reason to lose the bench line
        parity["reference"] = {"error": f"{type(exc).__name__}: {exc}"}
    cpu = {"value": rows / cpu_s, "unit": UNIT, "cores": threads, "kind": "port", "code": CPU_CODE,
           "note": CPU_NOTE,
           "sample": f"the {rows} chromosomes of the parity check (the first and last timed steps), decoded "
                     f"with placement logs on {threads} threads in {cpu_s:.1f} s"}
    return parity, cpu


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
    from brkga_fft2_b200 import abi, build as libbuild
    libbuild.build()
    from brkga_fft2_b200 import instances
    from brkga_fft2_b200.evaluator import B200DecoderEvaluator, DeviceDecoder

    inst, packed = load_workload()
    P, N, M = args.pop, inst.nb_parts, inst.nb_machines
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
    device_last = out.cpu().numpy()

    from brkga_fft2_b200.shard import max_over_ranks, weak_throughput
    total_ms = max_over_ranks(sum(step_ms), dist, "cuda")
    value = weak_throughput(P * args.steps, world, total_ms / 1000.0)

    # e2e through the drop-in evaluator with host buffers: a fresh pageable array
    # per call as the reference's GA passes it, and page-locked input beside it
    evaluator = B200DecoderEvaluator(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                                     inst.instance_parts)

    def e2e_time(inputs):
        for s in range(args.warmup):
            evaluator.evaluate_batch(inputs[s])
        barrier()
        t, last = 0.0, None
        for s in range(args.steps):
            flush.fill_(s & 0xFF)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            last = evaluator.evaluate_batch(inputs[args.warmup + s])
            t += time.perf_counter() - t0
        return weak_throughput(P * args.steps, world, max_over_ranks(t, dist, "cuda")), last

    pageable = [np.array(h) for h in host]
    e2e_value, last_pageable = e2e_time(pageable)
    pinned = [torch.from_numpy(h).pin_memory().numpy() for h in host]
    e2e_pinned, last_pinned = e2e_time(pinned)
    same = bool(np.array_equal(np.asarray(last_pageable), device_last) and
                np.array_equal(np.asarray(last_pinned), device_last))
    failed = False

    if rank == 0:
        hbm_peak, peak_kind = measured_peaks()
        lib = abi.load_library()
        bid = abi.library_build_id()
        sm_count = torch.cuda.get_device_properties(local).multi_processor_count
        smem = smem_probe(torch, lib, sm_count)
        kern_avg_s = statistics.mean(kern_ms) / 1000.0
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generator, P100M4 shapes)",
            "config": workload_config(P, world),
            "roofline": roofline_record(decode_profile(), kern_avg_s, scan, tests, sm_count,
                                        clocks["sm_mhz"] if clocks else None, smem, hbm_peak, peak_kind, bid),
            "smem_probe": smem,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": P * 2 * N * 4,
                    "d2h_bytes_per_step": P * 8, "input": "pageable (a fresh np.array per call, as "
                                                          "BRKGA_alg3.py:119-123 passes it)",
                    "matches_device_path": same},
            "e2e_pinned": {"value": e2e_pinned, "unit": UNIT, "h2d_bytes_per_step": P * 2 * N * 4,
                           "d2h_bytes_per_step": P * 8, "input": "page-locked"},
            "gpu_launches": 4 * args.steps,  # assign_sort, order_items, decode, reduce per step
            "kernel_share": statistics.mean(kern_ms) / statistics.mean(step_ms),
            "counters_last_step": {"tests": tests, "row_chunks": chunks, "plates": bins},
            "status": status,
            "build_id": bid,
        }
        if clocks:
            line["clocks"] = clocks
        if not args.no_cpu_baseline:
            ids = [args.warmup] + ([args.warmup + args.steps - 1] if args.steps > 1 else [])
            parity, cpu = parity_and_cpu(dd, packed, [host[i] for i in ids], P, M, N, torch, step_ids=ids)
            line["parity"] = parity
            if world == 1:
                line["cpu_baseline"] = cpu
            failed = parity["exact"] != parity["rows"] or not parity["placements_exact"]
        if world == 1 and not args.no_ttt:
            line["surrogate"] = surrogate_record(torch, dd, inst, measured_peaks_bf16())
            import bench_ga
            # family screening: 8 children per parent pair, the surrogate keeps the best-predicted one;
            # 6 training steps of 512 rows per generation beside the decode
            line["time_to_target"] = bench_ga.time_to_target(WORKLOAD, P, args.ttt_generations, args.ttt_seeds,
                                                             oversample=8, variants=((6, 0.0, 1, "decode"),),
                                                             screen_mode="family")
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and failed:
        raise SystemExit("parity check failed: the timed rows differ from the CPU oracle")


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
