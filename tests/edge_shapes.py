"""Hand-built instances aimed at the edge paths of the decoder.

The seeded star polygons of ``brkga_fft2_b200.instances`` reach these only by
chance; here every instance is built to hit them:

* plate widths at and around the 32-column word boundaries (31, 32, 33, 63,
  64, 65, 96, 97), plates of 1 and 3 rows, and the largest extents the
  selection key allows (8191 rows, 8191 columns: 256 output words);
* parts that fill a plate exactly, lines of one cell width, single cells;
* runs of ones of length 1..W, in particular 32 / 33 / 64 / 65 / 96 / 97
  (the doubling dilation below 33 cells, the range test above it);
* combs with many runs per row, hollow frames, parts with empty interior rows
  (two blobs), staircases whose rows have every length, masks taller than the
  32 rows the vacancy pre-filter samples.

Each instance satisfies the reference's precondition that a plate which can
take a part in some orientation can take its new-plate rotation
(placement.py:72-78 places that rotation without a fit check); a part that
fits no orientation of a machine makes every chromosome that sends it there
infeasible (placement.py:47-53), which some instances use on purpose.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Sequence, Tuple

import numpy as np

from brkga_fft2_b200.instances import HT_S_PER_MM, ST_S, VT_S_PER_MM3, Instance
from brkga_fft2_b200.problem import (MachineData, MachinePartData, ProblemData, default_thresholds,
                                     make_part_data)


def rect(h: int, w: int) -> np.ndarray:
    return np.ones((h, w), np.uint8)


def frame(h: int, w: int, t: int) -> np.ndarray:
    m = rect(h, w)
    m[t:h - t, t:w - t] = 0
    return m


def comb(h: int, w: int, period: int, teeth: int = 1) -> np.ndarray:
    """Columns ``c % period < teeth`` set, plus a full bottom row (a comb)."""
    m = np.zeros((h, w), np.uint8)
    m[:, (np.arange(w) % period) < teeth] = 1
    m[-1, :] = 1
    return m


def staircase(h: int, w: int) -> np.ndarray:
    """Row i holds the first ceil((i + 1) * w / h) cells: every run length up to w."""
    m = np.zeros((h, w), np.uint8)
    for i in range(h):
        m[i, :max(1, -(-(i + 1) * w // h))] = 1
    return m


def inverted_staircase(h: int, w: int) -> np.ndarray:
    return staircase(h, w)[::-1].copy()


def two_blobs(h: int, w: int, gap: int) -> np.ndarray:
    """Two rectangles stacked with ``gap`` empty rows between them."""
    m = np.zeros((h, w), np.uint8)
    top = (h - gap) // 2
    m[:top, : max(1, w // 2)] = 1
    m[top + gap:, w // 3:] = 1
    return m


def u_shape(h: int, w: int, t: int) -> np.ndarray:
    m = rect(h, w)
    m[: h - t, t:w - t] = 0
    return m


def checker(h: int, w: int, cell: int) -> np.ndarray:
    ii, jj = np.meshgrid(np.arange(h) // cell, np.arange(w) // cell, indexing="ij")
    m = ((ii + jj) % 2 == 0).astype(np.uint8)
    m[-1, :] = 1  # keep it one piece
    m[:, 0] = 1
    return m


def random_blob(rng: np.random.Generator, h: int, w: int, p: float = 0.75) -> np.ndarray:
    """Random cells, cropped so the first and last row and column are occupied."""
    m = (rng.random((h, w)) < p).astype(np.uint8)
    m[0, rng.integers(w)] = 1
    m[-1, rng.integers(w)] = 1
    m[rng.integers(h), 0] = 1
    m[rng.integers(h), -1] = 1
    return m


def build(name: str, plates: Sequence[Tuple[int, int]], masks: List[np.ndarray], seed: int,
          repeat: Sequence[int] = ()) -> Instance:
    """An instance from explicit masks.  ``repeat`` lists mask indices that
    get a second gene of the same part type (instance_parts holds a part id
    twice), so the decoder's type tables are shared between genes."""
    rng = np.random.default_rng(seed)
    parts, heights, volumes = {}, [], []
    for p, m in enumerate(masks):
        pd = make_part_data(p, m)
        hb, wb = pd.shapes[pd.best_rotation]
        for L, W in plates:
            h0, w0 = pd.shapes[0]
            fits_any = not ((h0 > L or w0 > W) and (w0 > L or h0 > W))
            if fits_any and not (hb <= L and wb <= W):
                raise ValueError(f"{name}: part {p} fits plate {L}x{W} but its new-plate rotation does not")
        parts[p] = pd
        heights.append(rng.uniform(5.0, 300.0))
        volumes.append(float(m.sum()) * heights[-1] * rng.uniform(0.3, 0.8))
    machines = []
    for L, W in plates:
        f = rng.uniform(0.8, 1.2, size=3)
        mp = {p: MachinePartData(ffts=None, proc_time=volumes[p] * VT_S_PER_MM3 * f[1],
                                 proc_time_height=heights[p] * HT_S_PER_MM * f[2]) for p in parts}
        machines.append(MachineData(bin_length=int(L), bin_width=int(W), bin_area=float(L * W),
                                    setup_time=float(ST_S * f[0]), parts=mp))
    inst_parts = np.concatenate([np.arange(len(masks)), np.asarray(list(repeat), np.int64)]).astype(np.int64)
    uniq = np.arange(len(masks), dtype=np.int64)
    pdata = ProblemData(parts=parts, machines=machines, instance_parts=inst_parts, instance_parts_unique=uniq)
    M = len(plates)
    return Instance(name, pdata, int(inst_parts.size), M, default_thresholds(M), inst_parts, masks,
                    np.asarray(heights))


def word_boundaries() -> Instance:
    """Plates 64 x 64 (two words exactly) and 66 x 65; a full-plate part, runs of 32/33/64."""
    masks = [rect(64, 64), rect(1, 64), rect(32, 32), rect(33, 33), rect(2, 33), rect(1, 1), rect(64, 1),
             comb(20, 63, 2), comb(12, 64, 5, 3), staircase(40, 64), inverted_staircase(33, 64),
             frame(30, 60, 3), two_blobs(40, 50, 6), u_shape(45, 31, 4), checker(36, 36, 4), rect(31, 63)]
    return build("EdgeWords", [(64, 64), (66, 65)], masks, 1, repeat=(1, 5, 5, 2))


def long_runs() -> Instance:
    """Plates 40 x 97 and 40 x 96; runs of 65, 96 and 97 cells (range test across words)."""
    rng = np.random.default_rng(2)
    masks = [rect(3, 96), rect(2, 65), rect(40, 96), staircase(35, 96), inverted_staircase(38, 90),
             frame(20, 96, 2), comb(10, 95, 7, 5), rect(1, 66), rect(5, 64), u_shape(39, 97 - 31, 10),
             random_blob(rng, 12, 80, 0.9), two_blobs(30, 96, 2)]
    return build("EdgeLong", [(40, 97), (40, 96)], masks, 2, repeat=(1, 7))


def narrow() -> Instance:
    """Plates 33 x 31 and 31 x 33 (non-square, under one word wide) and 40 x 32."""
    rng = np.random.default_rng(3)
    masks = [rect(31, 31), rect(1, 31), rect(31, 1), comb(10, 31, 3), staircase(30, 31), frame(20, 25, 2),
             two_blobs(24, 20, 3), checker(15, 15, 2), rect(1, 1), random_blob(rng, 9, 13, 0.8),
             inverted_staircase(31, 31), u_shape(18, 30, 3)]
    return build("EdgeNarrow", [(33, 31), (31, 33), (40, 32)], masks, 3, repeat=(8, 8, 8, 1))


def flat_plates() -> Instance:
    """Plates of 1 and 3 rows: lines only; taller parts make a machine infeasible."""
    masks = [rect(1, 50), rect(1, 1), rect(1, 17), rect(1, 33), rect(2, 3), rect(3, 3), rect(1, 100),
             np.array([[1, 0, 1, 1, 0, 0, 1]], np.uint8), rect(3, 50)]
    return build("EdgeFlat", [(1, 100), (3, 50)], masks, 4, repeat=(1, 1, 2))


def extreme_extent() -> Instance:
    """The largest extents of the selection key: 8191 x 40 and 60 x 8191 plates."""
    rng = np.random.default_rng(5)
    masks = [rect(30, 40), staircase(40, 40), rect(1, 40), frame(40, 40, 5), random_blob(rng, 25, 39, 0.85),
             comb(20, 40, 4, 2), rect(40, 1), two_blobs(40, 33, 4), rect(1, 1), inverted_staircase(33, 40)]
    return build("EdgeExtent", [(8191, 40), (60, 8191)], masks, 5, repeat=(8, 8, 8, 8, 2))


def wide_plates() -> Instance:
    """Plates 60 x 8191 and 50 x 8000: runs thousands of cells long, up to 256 output words per row."""
    rng = np.random.default_rng(6)
    masks = [rect(1, 8000), rect(2, 4100), staircase(50, 8000), frame(40, 3000, 7), comb(30, 2000, 97, 40),
             rect(10, 10), random_blob(rng, 20, 300, 0.9), rect(50, 1), two_blobs(40, 5000, 10),
             inverted_staircase(45, 1000)]
    return build("EdgeWide", [(60, 8191), (50, 8000)], masks, 6, repeat=(5, 5, 7, 1))


EDGE_INSTANCES: Dict[str, Callable[[], Instance]] = {
    "EdgeWords": word_boundaries,
    "EdgeLong": long_runs,
    "EdgeNarrow": narrow,
    "EdgeFlat": flat_plates,
    "EdgeExtent": extreme_extent,
    "EdgeWide": wide_plates,
}
