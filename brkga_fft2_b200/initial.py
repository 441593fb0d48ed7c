"""Greedy initial solution for the GA's first individual.

Restates the reference's construction in ``BRKGA_alg3.py:445-603``: parts
sorted by height, then area, both descending (:447-452); each part placed
where the largest machine makespan grows least (the placement itself runs on
the GPU, ``brkga_initial_solution_host``); then the chromosome is encoded
(:571-600): every part of machine m gets one machine key drawn uniformly from
m's threshold interval, and sequencing keys ``linspace(0, 1, count)`` in the
order the parts sit on m's plates.
"""
from __future__ import annotations

import ctypes
import random as _random
from typing import Optional, Sequence

import numpy as np

from . import abi


def greedy_order(instance_parts, heights_by_part, areas_by_part) -> np.ndarray:
    """Gene indices sorted by (height, area) descending, ties in gene order (BRKGA_alg3.py:447-452)."""
    inst = np.asarray(instance_parts)
    h = np.array([float(heights_by_part[int(p)]) for p in inst])
    a = np.array([float(areas_by_part[int(p)]) for p in inst])
    return np.lexsort((-a, -h)).astype(np.int32)


def greedy_placements(native_problem, order: np.ndarray):
    """Run the device greedy; returns (machine [n], placements [n] structured, machine makespans [M])."""
    lib = abi.load_library()
    order = np.ascontiguousarray(order, dtype=np.int32)
    n = order.size
    M = native_problem.packed.n_machines
    machine = np.zeros(max(n, 1), np.int32)
    place = np.zeros(max(n, 1), abi.PLACEMENT_DTYPE)
    mk = np.zeros(M, np.float64)
    abi.check(lib.brkga_initial_solution_host(native_problem.handle, order.ctypes.data_as(ctypes.c_void_p), n,
                                              machine.ctypes.data_as(ctypes.c_void_p),
                                              place.ctypes.data_as(ctypes.c_void_p),
                                              mk.ctypes.data_as(ctypes.c_void_p)), "brkga_initial_solution_host")
    return machine[:n], place[:n], mk


def encode(machine, place, instance_parts, type_ids, gene_type, nb_machines: int,
           thresholds: Sequence[float], rng=None) -> np.ndarray:
    """Chromosome of a greedy packing (BRKGA_alg3.py:571-600), float64 [2N]."""
    rng = _random if rng is None else rng
    inst = np.asarray(instance_parts)
    N = inst.size
    array = np.zeros(2 * N)
    used = set()
    for m in range(nb_machines):
        ks = [k for k in range(len(machine)) if machine[k] == m]
        ks.sort(key=lambda k: (int(place[k]["bin"]), k))  # plates in creation order, parts in insertion order
        parts_machine = [int(type_ids[gene_type[int(place[k]["gene"])]]) for k in ks]
        positions = []
        for value in parts_machine:
            for idx, val in enumerate(inst):
                if val == value and idx not in used:
                    positions.append(idx)
                    used.add(idx)
                    break
        pos = np.array(positions, dtype=np.int64)
        if nb_machines == 1:
            key = rng.uniform(0, 1)
        elif m == 0:
            key = rng.uniform(0, thresholds[m])
        elif m == nb_machines - 1:
            key = rng.uniform(thresholds[m - 1] + 0.0001, 1 - 0.0001)
        else:
            key = rng.uniform(thresholds[m - 1] + 0.0001, thresholds[m] - 0.0001)
        array[pos + N] = key
        values = np.linspace(0, 1, len(pos), endpoint=False)
        for i, p in enumerate(pos):
            array[p] = values[i]
    return array


def initial_solution(native_problem, instance_parts, heights_by_part, areas_by_part, thresholds,
                     rng: Optional[object] = None):
    """(chromosome float64 [2N], greedy makespan, (machine, placements)) for ``population[0]``."""
    pk = native_problem.packed
    order = greedy_order(instance_parts, heights_by_part, areas_by_part)
    machine, place, mk = greedy_placements(native_problem, order)
    chrom = encode(machine, place, instance_parts, pk.type_ids, pk.arrays["gene_type"], pk.n_machines, thresholds, rng)
    return chrom, float(mk.max()) if mk.size else 0.0, (machine, place)
