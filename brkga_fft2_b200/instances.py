"""Seeded synthetic instances for the decoder's benchmark and test workloads.

The reference measures on its own instance files (``data/Instances``, masks
in ``data/partsMatrices``); no public suite is involved.  These generators
stand in for them with the shapes the workloads name:

* part = a random star-shaped simple polygon with 6-12 vertices whose bounding
  box is drawn U[bbox_min, bbox_max] x U[bbox_min, bbox_max] cells, rasterised
  at cell centres and cropped to its occupied rows/columns; accepted when its
  fill (ones / bounding box) lies in [0.5, 0.9];
* part height U[5, 300] mm, volume = area_mm2 * height * U(0.3, 0.8), support 0;
* time model per machine: setup 1 h, 0.03 h/cm3 of volume, 0.7 h/cm of the
  tallest part (in seconds: ST 3600 s, VT 0.108 s/mm3, HT 252 s/mm, SPT 0),
  optionally each constant scaled by U(0.8, 1.2) per machine;
* every gene is its own part type (instance_parts = 0..N-1).

The per-part precompute and the processing-time formulas follow the
reference's ``BRKGA_alg3.py:332-431`` (``proc_time = volume*VT + support*SPT``,
``proc_time_height = height*HT``).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .problem import (MachineData, MachinePartData, ProblemData, default_thresholds,
                      make_part_data)

ST_S = 3600.0          # 1.0 h setup
VT_S_PER_MM3 = 0.108   # 0.03 h/cm3
HT_S_PER_MM = 252.0    # 0.7 h/cm
SPT_S_PER_MM3 = 0.0


@dataclass
class Instance:
    name: str
    problem_data: ProblemData
    nb_parts: int
    nb_machines: int
    thresholds: List[float]
    instance_parts: np.ndarray
    masks: List[np.ndarray]
    heights: Optional[np.ndarray] = None  # part height in mm (the greedy initial solution sorts by it)


def _star_polygon(rng: np.random.Generator, h: int, w: int) -> np.ndarray:
    k = int(rng.integers(6, 13))
    base = np.sort(rng.uniform(0.0, 2.0 * np.pi, size=k))
    radii = rng.uniform(0.45, 1.0, size=k)
    ys = radii * np.sin(base)
    xs = radii * np.cos(base)
    # stretch the vertices onto the whole bounding box so the raster spans it
    eps = 1e-3
    ys = eps + (ys - ys.min()) / max(ys.max() - ys.min(), 1e-9) * (h - 2 * eps)
    xs = eps + (xs - xs.min()) / max(xs.max() - xs.min(), 1e-9) * (w - 2 * eps)
    return np.stack([ys, xs], axis=1)


def _rasterize(poly: np.ndarray, h: int, w: int) -> np.ndarray:
    py = np.arange(h)[:, None] + 0.5
    px = np.arange(w)[None, :] + 0.5
    inside = np.zeros((h, w), dtype=bool)
    n = len(poly)
    for i in range(n):
        y0, x0 = poly[i]
        y1, x1 = poly[(i + 1) % n]
        if y0 == y1:
            continue
        cond = (y0 > py) != (y1 > py)
        xint = x0 + (py - y0) * (x1 - x0) / (y1 - y0)
        inside ^= cond & (px < xint)
    return inside


def random_part_mask(rng: np.random.Generator, bbox_min: int = 10, bbox_max: int = 80,
                     fill_lo: float = 0.5, fill_hi: float = 0.9) -> np.ndarray:
    """One uint8 0/1 mask with fill in [fill_lo, fill_hi] (rejection sampled)."""
    h = int(rng.integers(bbox_min, bbox_max + 1))
    w = int(rng.integers(bbox_min, bbox_max + 1))
    for _ in range(1000):
        m = _rasterize(_star_polygon(rng, h, w), h, w)
        rows = np.flatnonzero(m.any(axis=1))
        cols = np.flatnonzero(m.any(axis=0))
        if rows.size == 0:
            continue
        m = m[rows[0]:rows[-1] + 1, cols[0]:cols[-1] + 1]
        fill = m.mean()
        if fill_lo <= fill <= fill_hi:
            return m.astype(np.uint8)
    raise RuntimeError("could not draw a part mask with the requested fill")


def make_instance(name: str, n_parts: int, plates: Sequence[Tuple[int, int]], seed: int,
                  bbox_min: int = 10, bbox_max: int = 80, cell_mm: float = 1.0,
                  scale_machines: bool = False,
                  time_constants: Optional[Sequence[Tuple[float, float, float, float]]] = None,
                  fill: Tuple[float, float] = (0.5, 0.9), allow_unfit: bool = False) -> Instance:
    """Build one instance.  ``plates`` is a list of (L rows, W columns) per machine.

    With ``allow_unfit`` a part may be too large for some plates (the decoder
    then scores chromosomes that send it there as infeasible); it must still
    fit the largest plate.  In every case a plate that can take the part in
    some orientation can take its new-plate rotation (placement.py:72-78 places
    that rotation without a fit check).
    """
    rng = np.random.default_rng(seed)
    M = len(plates)
    min_side = min(min(L, W) for L, W in plates)
    max_side = max(max(L, W) for L, W in plates)
    masks: List[np.ndarray] = []
    parts = {}
    heights = np.zeros(n_parts)
    volumes = np.zeros(n_parts)
    for p in range(n_parts):
        while True:
            m = random_part_mask(rng, bbox_min, min(bbox_max, max_side if allow_unfit else min_side),
                                 fill[0], fill[1])
            pd = make_part_data(p, m)
            hb, wb = pd.shapes[pd.best_rotation]
            h0, w0 = pd.shapes[0]
            best_fits = [hb <= L and wb <= W for L, W in plates]
            any_fits = [not ((h0 > L or w0 > W) and (w0 > L or h0 > W)) for L, W in plates]
            if allow_unfit:
                ok = any(best_fits) and all(b or not a for a, b in zip(any_fits, best_fits))
            else:
                ok = all(best_fits)
            if ok:
                break
        masks.append(m)
        parts[p] = pd
        area_mm2 = float(m.sum()) * cell_mm * cell_mm
        heights[p] = rng.uniform(5.0, 300.0)
        volumes[p] = area_mm2 * heights[p] * rng.uniform(0.3, 0.8)
    machines = []
    for mi, (L, W) in enumerate(plates):
        if time_constants is not None:
            st, vt, spt, ht = time_constants[mi]
        else:
            st, vt, spt, ht = ST_S, VT_S_PER_MM3, SPT_S_PER_MM3, HT_S_PER_MM
            if scale_machines:
                f = rng.uniform(0.8, 1.2, size=3)
                st, vt, ht = st * f[0], vt * f[1], ht * f[2]
        mp = {}
        for p in range(n_parts):
            mp[p] = MachinePartData(ffts=None,
                                    proc_time=volumes[p] * vt + 0.0 * spt,
                                    proc_time_height=heights[p] * ht)
        machines.append(MachineData(bin_length=int(L), bin_width=int(W), bin_area=float(L * W),
                                    setup_time=float(st), parts=mp))
    inst_parts = np.arange(n_parts, dtype=np.int64)
    pdata = ProblemData(parts=parts, machines=machines, instance_parts=inst_parts,
                        instance_parts_unique=inst_parts.copy())
    return Instance(name, pdata, n_parts, M, default_thresholds(M), inst_parts, masks, heights)


# Named workloads (sizes from the benchmark configurations).
def p50m2(seed: int = 0) -> Instance:
    """50 parts (bbox <= 80), 2 machines with 250x250 plates."""
    return make_instance("P50M2", 50, [(250, 250)] * 2, seed, bbox_max=80)


def p100m4(seed: int = 0) -> Instance:
    """100 parts (bbox <= 120), 2 x 300x300 + 2 x 250x250 plates, constants x U(0.8,1.2)."""
    return make_instance("P100M4", 100, [(300, 300), (300, 300), (250, 250), (250, 250)], seed,
                         bbox_max=120, scale_machines=True)


def p200m6(seed: int = 0) -> Instance:
    """200 parts, 6 machines with 400x400 plates."""
    return make_instance("P200M6", 200, [(400, 400)] * 6, seed, bbox_max=80)


def p400m8(seed: int = 0) -> Instance:
    """400 parts with masks up to 240x240 cells at 0.5 mm/cell, 8 x 600x600 plates."""
    return make_instance("P400M8", 400, [(600, 600)] * 8, seed, bbox_min=20, bbox_max=240,
                         cell_mm=0.5)


def uneven(seed: int) -> Instance:
    """One of the uneven batch: U[25,200] parts, U[1,6] machines, plates 150..500."""
    rng = np.random.default_rng(10_000 + seed)
    n = int(rng.integers(25, 201))
    M = int(rng.integers(1, 7))
    plates = [(int(s), int(s)) for s in rng.integers(150, 501, size=M)]
    return make_instance(f"U{seed}", n, plates, seed, bbox_max=80, scale_machines=True)


def small(seed: int = 0, n_parts: int = 12, plates=((60, 60), (50, 70)), bbox_max: int = 24) -> Instance:
    """Tiny instance for fast parity tests (non-square plates allowed)."""
    return make_instance(f"S{seed}", n_parts, list(plates), seed, bbox_min=3, bbox_max=bbox_max)


def chromosomes(n: int, nb_parts: int, seed: int) -> np.ndarray:
    """``default_rng(seed).random((n, 2N), float64).astype(float32)`` (benchmark_harness.py:171-185)."""
    return np.random.default_rng(seed).random((n, 2 * nb_parts), dtype=np.float64).astype(np.float32)


WORKLOADS = {"P50M2": p50m2, "P100M4": p100m4, "P200M6": p200m6, "P400M8": p400m8}
