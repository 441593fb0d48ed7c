"""CPU oracle for the BRKGA decoder — test infrastructure only.

Imported by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` as the checker the CUDA decoder is compared against.  The
product package (``brkga_fft2_b200``) never imports this package.
"""
from .oracle import build_oracle, oracle_decode, oracle_initial_solution, oracle_lib_path  # noqa: F401
