"""B200-native BRKGA chromosome decoder (sm_100a CUDA behind a C ABI).

Drop-in for the evaluator call of paulonasc7/BRKGA_FFT2's GA loop
(``BRKGA.cal_fitness`` -> ``evaluate_batch``, BRKGA_alg3.py:119-123).
"""
from .problem import (  # noqa: F401
    INFEASIBLE_PENALTY, THRESH_F32, THRESH_F64, MachineData, MachinePartData, PackedProblem,
    PartData, ProblemData, default_thresholds, make_part_data, pack_problem,
)

__all__ = [
    "INFEASIBLE_PENALTY", "THRESH_F32", "THRESH_F64", "MachineData", "MachinePartData",
    "PackedProblem", "PartData", "ProblemData", "default_thresholds", "make_part_data",
    "pack_problem",
]


def __getattr__(name):
    # The evaluator pulls in torch and the CUDA library; import it lazily.
    if name in ("B200DecoderEvaluator", "DeviceDecoder"):
        from . import evaluator
        return getattr(evaluator, name)
    raise AttributeError(name)
