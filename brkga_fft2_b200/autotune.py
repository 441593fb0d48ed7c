"""Launch-shape autotuner for the decode kernel.

The decode kernel has four knobs (``brkga_set_launch_config``).  Warps per
item (1, 2 or 4) trade the latency of one (chromosome, machine) item against
throughput: 4 finish an item sooner, 2 waste fewer lanes on speculative row
chunks, so 2 win once the items fill several waves of resident CTAs, and 1
(no CTA barrier at all) wins by a few per cent only when they fill some 20
waves (measured: 64 uneven instances x 256 chromosomes, 52,000 items, 33.0
against 35.4 ms); the automatic choice follows these tiers.  More
resident CTAs per SM hide more latency, more plates per item in shared
memory keep more collision searches off the global pool, and both draw on
the same 228 KB of shared memory per SM, whose share per plate grows with
the plate grid (a 500 x 500 plate is 36 KB as bit-packed rows, a 150 x 150
one 3.6 KB).  The fourth, ``task_max``, decides when a warp
deals (candidate row, 32-column word) pairs of the exact collision test
across its lanes instead of giving each lane one candidate row: dealing wins
while the pairs are few, loses on wide plates with many surviving candidates
(long, uneven chains), so its best value depends on the grid and masks.
``autotune`` times the shapes first (``task_max`` at its default), then the
``task_max`` values at the best shape, each on the caller's own population
(CUDA events around the decode kernel alone), keeps the fastest, and
remembers it per device and grid size in a JSON cache, so later runs on the
same plate grids skip the search.

The reference has no counterpart (its kernels use fixed launch shapes,
full_native_decoder.py:2570-2755).
"""
from __future__ import annotations

import json
import os
from typing import Iterable, Optional, Sequence, Tuple

import numpy as np

from . import abi

# (warps per item, CTAs per SM, plates per item in shared memory)
DEFAULT_SHAPES: Tuple[Tuple[int, int, int], ...] = ((4, 8, 0), (4, 8, 1), (4, 8, 2), (4, 6, 1), (4, 6, 2),
                                                    (2, 16, 0), (2, 16, 1), (2, 12, 1), (2, 12, 2), (2, 8, 2),
                                                    (1, 32, 0))
DEFAULT_TASK_MAX: Tuple[int, ...] = (0, 64, 256, 1024, 8192)


def grid_key(packs: Sequence, device_index: int = 0) -> str:
    """Cache key: device, SM count, the largest plate grid, genes and machines."""
    import torch
    props = torch.cuda.get_device_properties(device_index)
    L = max(int(max(p.arrays["bin_length"])) for p in packs)
    W = max(int(max(p.arrays["bin_width"])) for p in packs)
    N = max(p.n_genes for p in packs)
    M = max(p.n_machines for p in packs)
    return f"{props.name}|sm{props.multi_processor_count}|grid{L}x{W}|N{N}|M{M}|K{len(packs)}"


def _time_decode(decoder, run, repeats: int) -> float:
    import torch
    times = []
    for _ in range(repeats + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        run((e0, e1))
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    st = int(decoder.status.item())
    if st != 0:
        raise abi.BrkgaError(st, "decode during autotuning")
    return float(np.median(times[1:]))


def autotune(decoder, chrom, pops=None, shapes: Optional[Iterable[Tuple[int, int, int]]] = None,
             task_max_values: Optional[Iterable[int]] = None, repeats: int = 2, cache_path: Optional[str] = None,
             key: Optional[str] = None) -> dict:
    """Pick the fastest decode-kernel configuration for ``decoder``.

    ``decoder`` is a ``DeviceDecoder`` (``chrom``: float32 CUDA [P, 2N]) or a
    ``MultiDecoder`` (``chrom``: the flat concatenated rows, ``pops``: rows per
    instance).  ``shapes`` are (warps per item, CTAs per SM, plates in shared
    memory) triples; those that cannot be resident are skipped.  Returns
    ``{"key", "config": (warps, ctas_per_sm, smem_plates, task_max), "ms",
    "table": [(warps, ctas_per_sm, smem_plates, task_max, ms), ...],
    "cached"}`` and leaves the decoder on the chosen configuration.
    """
    import torch
    packs = decoder.packs if hasattr(decoder, "packs") else [decoder.packed]
    key = key or grid_key(packs, decoder.device.index or 0)
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
    if key in cache:
        w, c, s, t = cache[key]["config"]
        decoder.set_launch_config(w, c, s, t)
        return {"key": key, "config": (w, c, s, t), "ms": cache[key]["ms"], "table": cache[key]["table"],
                "cached": True}

    if pops is None:
        out = torch.empty(chrom.shape[0], dtype=torch.float64, device=chrom.device)
        run = lambda ev: decoder.decode(chrom, out=out, kernel_events=ev)  # noqa: E731
    else:
        out = torch.empty(int(np.sum(pops)), dtype=torch.float64, device=chrom.device)
        run = lambda ev: decoder.decode_concat(chrom, pops, out=out, kernel_events=ev)  # noqa: E731
    reference = []
    table = []

    def trial(w, c, s, t):
        try:
            decoder.set_launch_config(w, c, s, t)
        except abi.BrkgaError:
            return
        ms = _time_decode(decoder, run, repeats)
        if not reference:
            reference.append(out.clone())
        elif not torch.equal(out, reference[0]):
            raise RuntimeError(f"launch configuration {(w, c, s, t)} changed the makespans")
        table.append((w, c, s, t, ms))

    for w, c, s in (shapes or DEFAULT_SHAPES):
        trial(w, c, s, -1)
    if not table:
        raise RuntimeError("no launch shape could be resident")
    w, c, s, _, _ = min(table, key=lambda r: r[4])
    for t in (task_max_values if task_max_values is not None else DEFAULT_TASK_MAX):
        trial(w, c, s, t)
    w, c, s, t, ms = min(table, key=lambda r: r[4])
    decoder.set_launch_config(w, c, s, t)
    t = decoder.launch_config()[4]
    if cache_path:
        cache[key] = {"config": [w, c, s, t], "ms": ms, "table": table}
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return {"key": key, "config": (w, c, s, t), "ms": ms, "table": table, "cached": False}


def collision_paths(decoder, chrom, limit: int = 512, levels=(0, 1, 2), repeats: int = 5,
                    cache_path: Optional[str] = None, key: Optional[str] = None) -> dict:
    """Time the two collision-test paths per mask-size bucket on the decoder's own chunks.

    ``chrom`` (float32 CUDA [P, 2N]) is decoded once with placement logs; the
    plates each part met are replayed (:func:`collision.chunk_cases`) and the
    chunks of every rotation with a side of at least 64 cells are timed
    through both paths of ``brkga_chunk_free``: the bit-packed search and the
    INT8 tensor-core correlation, each bucket's chunks repeated until a launch
    fills the GPU (throughput, not the latency of a few chunks).  Returns ``{"key", "table": [per bucket:
    chunks, ms and ns per chunk of each path, "choice"], "choices":
    {bucket: path}, "cached"}``; buckets without chunks are absent.  The
    decode kernel runs the bit-packed search; the tensor-core path would be
    taken for a bucket only where it is timed faster.
    """
    import torch
    from . import collision
    key = (key or grid_key([decoder.packed], decoder.device.index or 0)) + "|collision"
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
    if key in cache:
        return {"key": key, "table": cache[key]["table"], "choices": cache[key]["choices"], "cached": True}
    P, pk = chrom.shape[0], decoder.packed
    log = torch.empty((P, pk.n_machines, pk.n_genes, 5), dtype=torch.int32, device=chrom.device)
    decoder.decode(chrom, log=log)
    torch.cuda.synchronize()
    if int(decoder.status.item()) != 0:
        raise abi.BrkgaError(int(decoder.status.item()), "decode before the collision-path timing")
    log = log.cpu().numpy().view(abi.PLACEMENT_DTYPE).reshape(P, pk.n_machines, pk.n_genes)
    cases = collision.chunk_cases(pk, log, min_side=64, levels=levels, limit=limit)
    if not cases:
        return {"key": key, "table": [], "choices": {}, "cached": False}
    table = collision.bucket_table(decoder.native, pk, cases, repeats=repeats, device=chrom.device)
    choices = {r["bucket"]: r["choice"] for r in table}
    if cache_path:
        cache[key] = {"table": table, "choices": choices}
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return {"key": key, "table": table, "choices": choices, "cached": False}
