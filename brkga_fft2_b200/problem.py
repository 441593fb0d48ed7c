"""Problem model for the BRKGA decoder: parts, machines and their packing.

The dataclasses mirror the reference's ``data_structures.py`` (``PartData``
:13-58, ``MachinePartData`` :61-69, ``MachineData`` :72-81, ``ProblemData``
:84-105) field for field, so a ``ProblemData`` built by the reference's
``BRKGA_alg3.py`` can be handed to :class:`brkga_fft2_b200.B200DecoderEvaluator`
unchanged (duck typing: only the attributes used below are read).  The
per-rotation FFTs the reference stores in ``MachinePartData.ffts`` are not
needed here — the decoder's collision test is an exact integer correlation —
so our own constructors leave that field empty.

``make_part_data`` restates the per-part precompute of ``BRKGA_alg3.py:332-386``:
``nrot`` = 2 when the mask equals its 180-degree rotation else 4, rotation r
is ``np.rot90(mask, r)`` (counter-clockwise), density = longest run of ones in
each row, ``best_rotation`` = first rotation of minimum height.

``pack_problem`` flattens a problem into the C-ABI descriptor
(``BrkgaProblemDesc`` in ``include/brkga_b200.h``); it plays the role of the
reference's ``_pack_problem_data`` (``full_native_decoder.py:2788-2926``).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import abi

THRESH_F32 = 0  # placement.py: float32 keys compared with Python-float thresholds (NumPy >= 2 keeps float32)
THRESH_F64 = 1  # full_native_decoder.py / wave_batch_evaluator.py: comparison in float64

INFEASIBLE_PENALTY = 1e16  # placement.py:9


@dataclass
class PartData:
    """Geometry of one part type; same fields as the reference's ``PartData``."""

    id: int
    area: float
    nrot: int
    rotations: List[np.ndarray]
    shapes: List[Tuple[int, int]]
    densities: List[np.ndarray]
    best_rotation: int
    rotations_gpu: Optional[List[Any]] = None
    rotations_uint8: Optional[List[np.ndarray]] = None


@dataclass
class MachinePartData:
    """Machine-specific data of one part type (``ffts`` unused by this decoder)."""

    ffts: Optional[List[Any]]
    proc_time: float
    proc_time_height: float


@dataclass
class MachineData:
    """One machine: plate of ``bin_length`` rows by ``bin_width`` columns."""

    bin_length: int
    bin_width: int
    bin_area: float
    setup_time: float
    parts: Dict[int, MachinePartData] = field(default_factory=dict)


@dataclass
class ProblemData:
    parts: Dict[int, PartData]
    machines: List[MachineData]
    instance_parts: np.ndarray
    instance_parts_unique: np.ndarray


def row_max_runs(mask: np.ndarray) -> np.ndarray:
    """Longest run of ones per row (``BRKGA_alg3.py:350-360``)."""
    m = np.asarray(mask)
    padded = np.pad(m.astype(np.int8), ((0, 0), (1, 1)), constant_values=0)
    diffs = np.diff(padded, axis=1)
    starts = np.where(diffs == 1)
    ends = np.where(diffs == -1)
    out = np.zeros(m.shape[0], dtype=np.int32)
    if len(starts[0]) > 0:
        np.maximum.at(out, starts[0], ends[1] - starts[1])
    return out


def make_part_data(part_id: int, mask: np.ndarray, area: Optional[float] = None) -> PartData:
    """Rotations, shapes, densities and best rotation of one part mask.

    Follows ``BRKGA_alg3.py:332-386``.  ``area`` defaults to the mask's cell
    count (the reference reads it from ``polygon_areas.xlsx``).
    """
    m = np.ascontiguousarray(np.asarray(mask).astype(np.int32))
    if m.ndim != 2 or m.shape[0] < 1 or m.shape[1] < 1:
        raise ValueError("part mask must be a non-empty 2-D array")
    if not np.isin(m, (0, 1)).all():
        raise ValueError("part mask must hold only 0 and 1")
    nrot = 2 if np.array_equal(m, np.rot90(m, 2)) else 4
    rotations, shapes, densities = [], [], []
    for r in range(nrot):
        rr = np.ascontiguousarray(np.rot90(m, r))
        rotations.append(rr)
        shapes.append((int(rr.shape[0]), int(rr.shape[1])))
        densities.append(row_max_runs(rr))
    best = int(np.argmin([s[0] for s in shapes]))
    return PartData(
        id=int(part_id),
        area=float(m.sum()) if area is None else float(area),
        nrot=nrot,
        rotations=rotations,
        shapes=shapes,
        densities=densities,
        best_rotation=best,
        rotations_uint8=[r.astype(np.uint8) for r in rotations],
    )


def default_thresholds(nb_machines: int) -> List[float]:
    """Machine-assignment thresholds ``t/M`` (``BRKGA_alg3.py:442``)."""
    return [t / nb_machines for t in range(1, nb_machines)]


class PackedProblem:
    """Flat arrays of one problem instance plus the ctypes descriptor over them.

    The arrays are owned here; ``desc`` points into them, so keep this object
    alive while the descriptor is in use.
    """

    def __init__(self, arrays: Dict[str, np.ndarray], n_genes: int, n_machines: int,
                 n_types: int, threshold_mode: int, type_ids: np.ndarray):
        self.arrays = arrays
        self.n_genes = int(n_genes)
        self.n_machines = int(n_machines)
        self.n_types = int(n_types)
        self.threshold_mode = int(threshold_mode)
        self.type_ids = type_ids
        a = arrays
        d = abi.BrkgaProblemDesc()
        d.n_genes = self.n_genes
        d.n_machines = self.n_machines
        d.n_types = self.n_types
        d.threshold_mode = self.threshold_mode
        d.gene_type = abi.ptr(a["gene_type"], ctypes.c_int32)
        d.thresholds = abi.ptr(a["thresholds"], ctypes.c_double)
        d.bin_length = abi.ptr(a["bin_length"], ctypes.c_int32)
        d.bin_width = abi.ptr(a["bin_width"], ctypes.c_int32)
        d.bin_area = abi.ptr(a["bin_area"], ctypes.c_double)
        d.setup_time = abi.ptr(a["setup_time"], ctypes.c_double)
        d.proc_time = abi.ptr(a["proc_time"], ctypes.c_double)
        d.proc_time_height = abi.ptr(a["proc_time_height"], ctypes.c_double)
        d.part_area = abi.ptr(a["part_area"], ctypes.c_double)
        d.part_nrot = abi.ptr(a["part_nrot"], ctypes.c_int32)
        d.part_best_rot = abi.ptr(a["part_best_rot"], ctypes.c_int32)
        d.rot_h = abi.ptr(a["rot_h"], ctypes.c_int32)
        d.rot_w = abi.ptr(a["rot_w"], ctypes.c_int32)
        d.rot_mask_offset = abi.ptr(a["rot_mask_offset"], ctypes.c_int64)
        d.masks = abi.ptr(a["masks"], ctypes.c_uint8)
        d.masks_bytes = int(a["masks"].size)
        self.desc = d

    @property
    def max_bin_width(self) -> int:
        return int(self.arrays["bin_width"].max())

    @property
    def max_bin_length(self) -> int:
        return int(self.arrays["bin_length"].max())

    def save(self, path: str) -> None:
        np.savez_compressed(path, n_genes=self.n_genes, n_machines=self.n_machines,
                            n_types=self.n_types, threshold_mode=self.threshold_mode,
                            type_ids=self.type_ids, **self.arrays)

    @classmethod
    def load(cls, path: str) -> "PackedProblem":
        z = np.load(path)
        keys = ("gene_type", "thresholds", "bin_length", "bin_width", "bin_area", "setup_time",
                "proc_time", "proc_time_height", "part_area", "part_nrot", "part_best_rot",
                "rot_h", "rot_w", "rot_mask_offset", "masks")
        arrays = {k: np.ascontiguousarray(z[k]) for k in keys}
        return cls(arrays, int(z["n_genes"]), int(z["n_machines"]), int(z["n_types"]),
                   int(z["threshold_mode"]), np.asarray(z["type_ids"]))


def pack_problem(problem_data, nb_parts: int, nb_machines: int, thresholds: Sequence[float],
                 instance_parts, threshold_mode: int = THRESH_F32) -> PackedProblem:
    """Flatten a (reference-compatible) ``ProblemData`` into descriptor arrays.

    Masks are taken from ``PartData.rotations[0]`` and re-rotated here, so the
    four rotation slots always follow ``np.rot90``; ``nrot`` and
    ``best_rotation`` are taken from the part data as the reference does.
    """
    inst = np.asarray(instance_parts, dtype=np.int64).reshape(-1)
    if inst.size != nb_parts:
        raise ValueError(f"instance_parts has {inst.size} entries, expected nb_parts={nb_parts}")
    if len(problem_data.machines) < nb_machines:
        raise ValueError("problem_data has fewer machines than nb_machines")
    thr = np.asarray(list(thresholds), dtype=np.float64).reshape(-1)
    if nb_machines > 1 and thr.size < nb_machines - 1:
        raise ValueError(f"need {nb_machines - 1} thresholds, got {thr.size}")
    if threshold_mode not in (THRESH_F32, THRESH_F64):
        raise ValueError("threshold_mode must be THRESH_F32 or THRESH_F64")
    type_ids = np.unique(inst)
    tindex = {int(p): i for i, p in enumerate(type_ids)}
    T = len(type_ids)
    gene_type = np.array([tindex[int(p)] for p in inst], dtype=np.int32)

    part_area = np.zeros(T, np.float64)
    part_nrot = np.zeros(T, np.int32)
    part_best = np.zeros(T, np.int32)
    rot_h = np.zeros(T * 4, np.int32)
    rot_w = np.zeros(T * 4, np.int32)
    rot_off = np.zeros(T * 4, np.int64)
    blobs = []
    off = 0
    for ti, pid in enumerate(type_ids):
        pd = problem_data.parts[int(pid)] if int(pid) in problem_data.parts else problem_data.parts[pid]
        base = np.ascontiguousarray(np.asarray(pd.rotations[0]).astype(np.uint8))
        part_area[ti] = float(pd.area)
        part_nrot[ti] = int(pd.nrot)
        part_best[ti] = int(pd.best_rotation)
        if part_nrot[ti] not in (2, 4):
            raise ValueError(f"part {pid}: nrot must be 2 or 4")
        for r in range(4):
            rr = np.ascontiguousarray(np.rot90(base, r)).astype(np.uint8)
            rot_h[ti * 4 + r], rot_w[ti * 4 + r] = rr.shape
            rot_off[ti * 4 + r] = off
            blobs.append(rr.reshape(-1))
            off += rr.size
    masks = np.concatenate(blobs) if blobs else np.zeros(1, np.uint8)

    M = nb_machines
    bin_length = np.zeros(M, np.int32)
    bin_width = np.zeros(M, np.int32)
    bin_area = np.zeros(M, np.float64)
    setup = np.zeros(M, np.float64)
    pt = np.zeros((M, T), np.float64)
    pth = np.zeros((M, T), np.float64)
    for m in range(M):
        md = problem_data.machines[m]
        bin_length[m] = int(md.bin_length)
        bin_width[m] = int(md.bin_width)
        bin_area[m] = float(md.bin_area)
        setup[m] = float(md.setup_time)
        for ti, pid in enumerate(type_ids):
            mp = md.parts[int(pid)] if int(pid) in md.parts else md.parts[pid]
            pt[m, ti] = float(mp.proc_time)
            pth[m, ti] = float(mp.proc_time_height)

    arrays = dict(
        gene_type=gene_type,
        thresholds=np.ascontiguousarray(thr[: max(M - 1, 0)]) if M > 1 else np.zeros(1, np.float64),
        bin_length=bin_length, bin_width=bin_width, bin_area=bin_area, setup_time=setup,
        proc_time=np.ascontiguousarray(pt.reshape(-1)),
        proc_time_height=np.ascontiguousarray(pth.reshape(-1)),
        part_area=part_area, part_nrot=part_nrot, part_best_rot=part_best,
        rot_h=rot_h, rot_w=rot_w, rot_mask_offset=rot_off, masks=np.ascontiguousarray(masks),
    )
    return PackedProblem(arrays, nb_parts, M, T, threshold_mode, type_ids)
