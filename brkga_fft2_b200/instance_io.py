"""Compact on-disk form of an instance (masks + times + plates), used by fixtures.

Only rotation 0 of each part mask is stored; rotations, densities and the
best rotation are re-derived with :func:`make_part_data` on load, which is
the reference's precompute (``BRKGA_alg3.py:332-386``).
"""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np

from .problem import MachineData, MachinePartData, ProblemData, make_part_data


def save_instance(path: str, problem_data, nb_parts: int, nb_machines: int, thresholds,
                  instance_parts, extra: Optional[Dict[str, np.ndarray]] = None) -> None:
    inst = np.asarray(instance_parts, dtype=np.int64)
    types = np.unique(inst)
    out = {
        "nb_parts": np.int64(nb_parts), "nb_machines": np.int64(nb_machines),
        "thresholds": np.asarray(list(thresholds), np.float64),
        "instance_parts": inst, "types": types,
        "area": np.array([float(problem_data.parts[int(t)].area) for t in types], np.float64),
        "nrot": np.array([int(problem_data.parts[int(t)].nrot) for t in types], np.int64),
        "best_rot": np.array([int(problem_data.parts[int(t)].best_rotation) for t in types], np.int64),
        "bin_length": np.array([int(problem_data.machines[m].bin_length) for m in range(nb_machines)], np.int64),
        "bin_width": np.array([int(problem_data.machines[m].bin_width) for m in range(nb_machines)], np.int64),
        "bin_area": np.array([float(problem_data.machines[m].bin_area) for m in range(nb_machines)], np.float64),
        "setup_time": np.array([float(problem_data.machines[m].setup_time) for m in range(nb_machines)], np.float64),
        "proc_time": np.array([[float(problem_data.machines[m].parts[int(t)].proc_time) for t in types]
                               for m in range(nb_machines)], np.float64),
        "proc_time_height": np.array([[float(problem_data.machines[m].parts[int(t)].proc_time_height) for t in types]
                                      for m in range(nb_machines)], np.float64),
    }
    for t in types:
        out[f"mask_{int(t)}"] = np.asarray(problem_data.parts[int(t)].rotations[0]).astype(np.uint8)
    if extra:
        out.update(extra)
    np.savez_compressed(path, **out)


def load_instance(path: str):
    """Returns (problem_data, nb_parts, nb_machines, thresholds, instance_parts, npz)."""
    z = np.load(path)
    types = z["types"]
    parts = {}
    for i, t in enumerate(types):
        pd = make_part_data(int(t), z[f"mask_{int(t)}"], float(z["area"][i]))
        if pd.nrot != int(z["nrot"][i]) or pd.best_rotation != int(z["best_rot"][i]):
            raise ValueError(f"part {t}: derived nrot/best rotation differ from the stored ones")
        parts[int(t)] = pd
    M = int(z["nb_machines"])
    machines = []
    for m in range(M):
        mp = {int(t): MachinePartData(None, float(z["proc_time"][m, i]), float(z["proc_time_height"][m, i]))
              for i, t in enumerate(types)}
        machines.append(MachineData(int(z["bin_length"][m]), int(z["bin_width"][m]), float(z["bin_area"][m]),
                                    float(z["setup_time"][m]), mp))
    inst = z["instance_parts"]
    pdata = ProblemData(parts, machines, inst, np.unique(inst))
    return pdata, int(z["nb_parts"]), M, [float(v) for v in z["thresholds"]], inst, z
