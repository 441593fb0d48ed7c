"""Audit output of decoded chromosomes, in the reference's formats.

From a placement log (``evaluate_batch(..., return_log=True)``, or
``DeviceDecoder.decode(..., log=...)``) and the packed instance:

* ``plates_from_log`` rebuilds every plate's occupancy grid (cells 0/1, rows
  top to bottom) — the ``BuildingPlate.grid`` the reference ends with;
* ``write_plate_dumps`` writes them as the reference's plate text files
  (``BuildingPlate.save_plate_to_file``, binClassNew.py:39-42: one line per
  row, each cell ``f'{val:2d}'``, separated by single spaces), one file
  ``{prefix}_m{machine}_b{plate}.txt`` per plate;
* ``machine_makespans`` recomputes each machine's build time from the log
  with the reference's model (placement.py:86-89: per plate processing time
  plus the tallest part's height time plus the setup time, summed over the
  machine's plates in order);
* ``solution_record`` returns the reference's golden-solution record
  (create_golden.py:194-210): instance label, sizes, the chromosome, the
  makespan and per machine its makespan, plate count and ordered placements
  ``{part_id, bin_idx, col, row, rot}`` (``col`` = left column x, ``row`` =
  bottom row y), ready for ``json.dump``.

Everything here runs on the host over arrays the decoder already returned.
"""
from __future__ import annotations

import os
from typing import Dict, List, Optional, Tuple

import numpy as np

from .problem import PackedProblem


def _rotation_mask(packed: PackedProblem, t: int, r: int) -> np.ndarray:
    a = packed.arrays
    i = t * 4 + r
    h, w, off = int(a["rot_h"][i]), int(a["rot_w"][i]), int(a["rot_mask_offset"][i])
    return a["masks"][off: off + h * w].reshape(h, w)


def plates_from_log(packed: PackedProblem, log_row: np.ndarray) -> Dict[Tuple[int, int], np.ndarray]:
    """Occupancy grids {(machine, plate): uint8 [L, W]} of one chromosome's log [M, N]."""
    a = packed.arrays
    out: Dict[Tuple[int, int], np.ndarray] = {}
    for m in range(packed.n_machines):
        L, W = int(a["bin_length"][m]), int(a["bin_width"][m])
        for rec in log_row[m]:
            g = int(rec["gene"])
            if g < 0:
                continue
            t = int(a["gene_type"][g])
            mask = _rotation_mask(packed, t, int(rec["rot"]))
            h, w = mask.shape
            y, x, b = int(rec["y"]), int(rec["x"]), int(rec["bin"])
            grid = out.setdefault((m, b), np.zeros((L, W), np.uint8))
            grid[y - h + 1: y + 1, x: x + w] += mask
    return out


def write_plate_dumps(directory: str, plates: Dict[Tuple[int, int], np.ndarray], prefix: str = "bin") -> List[str]:
    """Write each plate as the reference's text dump; returns the paths written."""
    os.makedirs(directory, exist_ok=True)
    paths = []
    for (m, b), grid in sorted(plates.items()):
        path = os.path.join(directory, f"{prefix}_m{m}_b{b}.txt")
        with open(path, "w") as f:
            for row in grid:
                f.write(" ".join(f"{int(v):2d}" for v in row) + "\n")
        paths.append(path)
    return paths


def read_plate_dump(path: str) -> np.ndarray:
    """A plate text dump back as an int array [L, W]."""
    with open(path) as f:
        return np.array([[int(v) for v in line.split()] for line in f if line.strip()], dtype=np.int64)


def machine_makespans(packed: PackedProblem, log_row: np.ndarray) -> List[float]:
    """Build time of every machine from one chromosome's log (0.0 for a machine with no plate)."""
    a = packed.arrays
    M, T = packed.n_machines, packed.n_types
    pt, pth = a["proc_time"].reshape(M, T), a["proc_time_height"].reshape(M, T)
    out = []
    for m in range(M):
        ptb: Dict[int, float] = {}
        pthb: Dict[int, float] = {}
        for rec in log_row[m]:
            g = int(rec["gene"])
            if g < 0:
                continue
            t, b = int(a["gene_type"][g]), int(rec["bin"])
            ptb[b] = ptb.get(b, 0.0) + float(pt[m, t])
            v = float(pth[m, t])
            if v > pthb.get(b, 0.0):
                pthb[b] = v
            else:
                pthb.setdefault(b, 0.0)
        ms = 0.0
        for b in range(len(ptb)):
            ms += (ptb[b] + pthb[b]) + float(a["setup_time"][m])
        out.append(ms)
    return out


def solution_record(packed: PackedProblem, chromosome: np.ndarray, makespan: float, log_row: np.ndarray,
                    instance: Optional[str] = None, inst_number: Optional[int] = None,
                    chromosome_idx: Optional[int] = None) -> dict:
    """The reference's golden-solution record of one decoded chromosome."""
    a = packed.arrays
    machines = {}
    per_machine = machine_makespans(packed, log_row)
    for m in range(packed.n_machines):
        placements = []
        bins = set()
        for rec in log_row[m]:
            g = int(rec["gene"])
            if g < 0:
                continue
            bins.add(int(rec["bin"]))
            placements.append({"part_id": int(packed.type_ids[a["gene_type"][g]]), "bin_idx": int(rec["bin"]),
                               "col": int(rec["x"]), "row": int(rec["y"]), "rot": int(rec["rot"])})
        machines[str(m)] = {"makespan": round(per_machine[m], 6), "n_bins": len(bins), "placements": placements}
    return {
        "instance": instance,
        "nbParts": int(packed.n_genes),
        "nbMachines": int(packed.n_machines),
        "instNumber": inst_number,
        "chromosome_idx": chromosome_idx,
        "chromosome": np.asarray(chromosome, np.float32).tolist(),
        "makespan": round(float(makespan), 6),
        "machines": machines,
    }
