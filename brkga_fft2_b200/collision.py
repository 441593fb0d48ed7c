"""The two collision-test paths, chunk by chunk, on plates the decoder met.

The reference tests a rotated part mask against a plate with an FFT
correlation (collision_backend.py:109-128): rounded overlap count == 0 is a
free position.  This library has two exact integer replacements for it,
``brkga_chunk_free`` (include/brkga_b200.h) runs either on a batch of
32-row candidate chunks:

* ``abi.COLLISION_BITSET`` — the decode kernel's bit-packed run-dilation
  search (every output word tested to the end here; inside the decoder it
  stops at the first free placement of the bottom-most candidate);
* ``abi.COLLISION_INT8_TC`` — a dense INT8 tensor-core correlation
  (tcgen05.mma kind::i8 with INT32 accumulation, csrc/corr_i8.cuh).

``chunk_cases`` replays placement logs to recover the plates exactly as they
were when each part was tested, so the chunks are the decoder's own;
``ChunkBatch`` uploads them, runs a path, returns the free-position words and
times launches; ``path_table`` times both paths per mask-size bucket, which
is what :func:`brkga_fft2_b200.autotune.collision_paths` decides with.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import abi
from .problem import PackedProblem

# mask-size buckets (largest side of the rotation, cells): the tensor-core
# path is offered from 64 x 64 up; the last bucket ends at its limit (256)
BUCKETS: Tuple[Tuple[int, int], ...] = ((64, 96), (96, 128), (128, 160), (160, 192), (192, 257))


def pack_plate(grid: np.ndarray) -> np.ndarray:
    """A 0/1 plate [L, W] in the decoder's format: L rows of ceil(W/32) + 2
    uint32 words, bit c of a row = column c, zero past column W."""
    L, W = grid.shape
    rs = (W + 31) // 32 + 2
    by = np.packbits(grid.astype(bool), axis=1, bitorder="little")
    out = np.zeros((L, rs * 4), np.uint8)
    out[:, : by.shape[1]] = by
    return out.view("<u4").reshape(L, rs)


def _rotation(packed: PackedProblem, t: int, r: int) -> np.ndarray:
    a = packed.arrays
    i = t * 4 + r
    h, w, off = int(a["rot_h"][i]), int(a["rot_w"][i]), int(a["rot_mask_offset"][i])
    return a["masks"][off: off + h * w].reshape(h, w)


def chunk_cases(packed: PackedProblem, log: np.ndarray, min_side: int = 64, levels: Sequence[int] = (0,),
                limit: int = 0) -> List[dict]:
    """Chunk tests as the decoder meets them, from placement logs [P, M, N].

    For every part placed on a plate that was already open, the plate as it
    was just before, each rotation of the part that fits the plate with a
    largest side of at least ``min_side``, and the chunks at ``levels``
    (0 = the bottom-most 32 candidate top rows, which the decoder tests
    first).  ``limit`` > 0 keeps that many cases spread evenly.  Each case:
    {machine, type, rot, ty_hi, h, w, grid (uint8 [L, W])}."""
    a = packed.arrays
    cases: List[dict] = []
    for row in log:
        for m in range(packed.n_machines):
            L, W = int(a["bin_length"][m]), int(a["bin_width"][m])
            plates: Dict[int, np.ndarray] = {}
            for rec in row[m]:
                g = int(rec["gene"])
                if g < 0:
                    continue
                t, b = int(a["gene_type"][g]), int(rec["bin"])
                if b in plates:
                    for r in range(int(a["part_nrot"][t])):
                        h, w = int(a["rot_h"][t * 4 + r]), int(a["rot_w"][t * 4 + r])
                        if h > L or w > W or max(h, w) < min_side:
                            continue
                        for lv in levels:
                            ty_hi = L - h - 32 * lv
                            if ty_hi >= 0:
                                cases.append({"machine": m, "type": t, "rot": r, "ty_hi": ty_hi, "h": h, "w": w,
                                              "grid": plates[b].copy()})
                mask = _rotation(packed, t, int(rec["rot"]))
                h, w = mask.shape
                grid = plates.setdefault(b, np.zeros((L, W), np.uint8))
                grid[int(rec["y"]) - h + 1: int(rec["y"]) + 1, int(rec["x"]): int(rec["x"]) + w] |= mask
    if limit and len(cases) > limit:
        cases = [cases[i] for i in np.linspace(0, len(cases) - 1, limit).astype(int)]
    return cases


def bucket_of(side: int) -> int:
    for i, (lo, hi) in enumerate(BUCKETS):
        if lo <= side < hi:
            return i
    return -1


class ChunkBatch:
    """Chunk cases on the device: plates, output words and the item array.

    With ``copies`` > 1 every case is listed that many times in a row (same
    plate, its own output words), so that one launch over a bucket holds
    enough chunks to fill the GPU and times throughput, not the latency of
    a few chunks.  Ranges given to ``run`` / ``time`` count cases."""

    def __init__(self, native, packed: PackedProblem, cases: List[dict], device=None, copies: int = 1):
        import torch
        self.torch = torch
        self.native = native
        self.lib = native.lib
        self.cases = cases
        self.copies = max(1, int(copies))
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        a = packed.arrays
        plates, pofs, oofs, self.nwo = [], [], [], []
        p = o = 0
        for c in cases:
            pw = pack_plate(c["grid"])
            plates.append(pw.reshape(-1))
            pofs.append(p)
            p += pw.size
            nwo = (int(a["bin_width"][c["machine"]]) - c["w"] + 1 + 31) // 32
            self.nwo.append(nwo)
            oofs.append(o)
            o += 32 * nwo * self.copies
        self.plates = torch.from_numpy(np.concatenate(plates).view(np.int32)).to(dev)
        self.out = torch.zeros(max(o, 1), dtype=torch.int32, device=dev)
        self.out_offsets = oofs
        items = np.zeros(len(cases) * self.copies, abi.CHUNK_TEST_DTYPE)
        pb, ob = self.plates.data_ptr(), self.out.data_ptr()
        for i, c in enumerate(cases):
            for k in range(self.copies):
                items[i * self.copies + k] = (pb + 4 * pofs[i], ob + 4 * (oofs[i] + 32 * self.nwo[i] * k), c["machine"],
                                              c["type"], c["rot"], c["ty_hi"])
        self.items = torch.from_numpy(items.view(np.uint8)).to(dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)

    def run(self, path: int, first: int = 0, count: int = -1, stream=None):
        torch = self.torch
        n = (len(self.cases) - first if count < 0 else count) * self.copies
        s = stream if stream is not None else torch.cuda.current_stream()
        ptr = self.items.data_ptr() + first * self.copies * abi.CHUNK_TEST_DTYPE.itemsize
        abi.check(self.lib.brkga_chunk_free(self.native.handle, path, ctypes.c_void_p(ptr), n,
                                            ctypes.c_void_p(self.status.data_ptr()), ctypes.c_void_p(s.cuda_stream)),
                  "brkga_chunk_free")

    def words(self, i: int, copy: int = 0) -> np.ndarray:
        """Free-position words [32, nwo] of case i (synchronises)."""
        nwo = self.nwo[i]
        o = self.out_offsets[i] + 32 * nwo * copy
        return self.out[o: o + 32 * nwo].cpu().numpy().view(np.uint32).reshape(32, nwo)

    def time(self, path: int, first: int = 0, count: int = -1, repeats: int = 5) -> float:
        """Median ms of one launch over cases [first, first + count)."""
        torch = self.torch
        self.run(path, first, count)
        times = []
        for _ in range(repeats):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self.run(path, first, count)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        st = int(self.status.item())
        if st:
            raise abi.BrkgaError(st, "brkga_chunk_free")
        return float(np.median(times))


def sort_by_bucket(cases: List[dict]) -> Tuple[List[dict], Dict[int, Tuple[int, int]]]:
    """Cases grouped by mask-size bucket, and each bucket's (first, count)."""
    keyed = sorted((bucket_of(max(c["h"], c["w"])), i) for i, c in enumerate(cases))
    out = [cases[i] for b, i in keyed if b >= 0]
    spans: Dict[int, Tuple[int, int]] = {}
    for j, (b, _) in enumerate(k for k in keyed if k[0] >= 0):
        f, n = spans.get(b, (j, 0))
        spans[b] = (f, n + 1)
    return out, spans


def path_table(batch: ChunkBatch, spans: Dict[int, Tuple[int, int]], repeats: int = 5) -> List[dict]:
    """Per mask-size bucket: distinct chunks, chunks per launch (with the
    batch's copies), ms per launch and GPU ns per chunk of each path."""
    rows = []
    for b, (first, n) in sorted(spans.items()):
        t_bit = batch.time(abi.COLLISION_BITSET, first, n, repeats)
        t_i8 = batch.time(abi.COLLISION_INT8_TC, first, n, repeats)
        lo, hi = BUCKETS[b]
        per = n * batch.copies
        rows.append({"bucket": f"{lo}-{hi - 1}", "chunks": n, "chunks_per_launch": per, "bitset_ms": t_bit,
                     "int8_tc_ms": t_i8, "bitset_ns_per_chunk": 1e6 * t_bit / per,
                     "int8_tc_ns_per_chunk": 1e6 * t_i8 / per, "int8_over_bitset": t_i8 / t_bit,
                     "choice": "int8_tc" if t_i8 < t_bit else "bitset"})
    return rows


def bucket_table(native, packed: PackedProblem, cases: List[dict], target_chunks: int = 4736, repeats: int = 5,
                 device=None) -> List[dict]:
    """Both paths timed per mask-size bucket at throughput: each bucket's cases
    are repeated until one launch holds about ``target_chunks`` chunks (by
    default four waves of the bit-packed path's 4-warp CTAs on 148 SMs at 8
    per SM), and both paths' words are compared on the way."""
    cases, spans = sort_by_bucket(cases)
    rows = []
    for b, (first, n) in sorted(spans.items()):
        sub = cases[first: first + n]
        copies = max(1, -(-target_chunks // n))
        batch = ChunkBatch(native, packed, sub, device=device, copies=copies)
        batch.run(abi.COLLISION_BITSET)
        ref = [batch.words(i) for i in range(n)]
        batch.out.fill_(-1)
        batch.run(abi.COLLISION_INT8_TC)
        if not all(np.array_equal(batch.words(i, copies - 1), ref[i]) for i in range(n)):
            raise RuntimeError(f"bucket {BUCKETS[b]}: the two paths differ")
        rows += path_table(batch, {b: (0, n)}, repeats)
        del batch
    return rows
