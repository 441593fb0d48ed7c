"""Population evaluators over the CUDA decoder.

``B200DecoderEvaluator`` is the drop-in for the reference's
``FullNativeDecoderEvaluator`` (``full_native_decoder.py:2937-2981``) and
``WaveBatchEvaluator`` (``wave_batch_evaluator.py:109-191``): same constructor
arguments, ``evaluate_batch(np.ndarray [P, 2N]) -> list[float]`` with 1e16 for
infeasible chromosomes, ``RuntimeError`` on bad input.  It goes through the
host-to-host entry point ``brkga_evaluate_host`` of the C ABI.

``DeviceDecoder`` decodes populations that are already on the GPU (torch
tensors), stream-ordered and without host synchronisation, through
``brkga_decode`` with a preallocated workspace — the form the GA loop and the
throughput benchmark use.  ``MultiDecoder`` does the same for several
independent instances (own parts, machines and plate sizes) in one launch of
each kernel, through ``brkga_decode_multi(_at)``.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import abi
from .problem import THRESH_F32, PackedProblem, pack_problem


class _NativeProblem:
    """Owns one ``BrkgaProblem*`` (device-resident tables of one or more instances)."""

    def __init__(self, packed):
        self.lib = abi.load_library()
        self.packed = packed
        handle = ctypes.c_void_p()
        if isinstance(packed, (list, tuple)):
            descs = (abi.BrkgaProblemDesc * len(packed))(*[p.desc for p in packed])
            st = self.lib.brkga_problem_create_multi(descs, len(packed), ctypes.byref(handle))
            abi.check(st, "brkga_problem_create_multi")
        else:
            st = self.lib.brkga_problem_create(ctypes.byref(packed.desc), ctypes.byref(handle))
            abi.check(st, "brkga_problem_create")
        self.handle = handle

    def launch_config(self, items: int = 0):
        """(warps per item, CTAs per SM, plates per item in shared memory, resident CTAs, task_max)
        of a decode launch of ``items`` (chromosome, machine) items."""
        w, c, s, r, t = (ctypes.c_int32() for _ in range(5))
        abi.check(self.lib.brkga_get_launch_config(self.handle, int(items), ctypes.byref(w), ctypes.byref(c),
                                                   ctypes.byref(s), ctypes.byref(r), ctypes.byref(t)))
        return w.value, c.value, s.value, r.value, t.value

    def set_launch_config(self, warps_per_item: int = 0, ctas_per_sm: int = 0, smem_plates: int = -1,
                          task_max: int = -1):
        abi.check(self.lib.brkga_set_launch_config(self.handle, int(warps_per_item), int(ctas_per_sm),
                                                   int(smem_plates), int(task_max)), "brkga_set_launch_config")

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.brkga_problem_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class B200DecoderEvaluator:
    """Drop-in evaluator: ``evaluate_batch(population) -> list of makespans``.

    Arguments follow ``FullNativeDecoderEvaluator.__init__``
    (``full_native_decoder.py:2940-2963``); ``collision_backend`` is accepted
    and ignored, as there.  ``threshold_mode`` picks how machine keys are
    compared with the thresholds: ``THRESH_F32`` is ``placement.py``'s
    behaviour (float32 under NumPy >= 2), ``THRESH_F64`` the C++ decoder's.
    """

    def __init__(self, problem_data, nb_parts: int, nb_machines: int, thresholds, instance_parts,
                 collision_backend=None, device: str = "cuda", threshold_mode: int = THRESH_F32):
        del collision_backend
        self._set_device(device)
        self.nb_parts = int(nb_parts)
        self.nb_machines = int(nb_machines)
        self.packed = pack_problem(problem_data, nb_parts, nb_machines, thresholds, instance_parts,
                                   threshold_mode)
        self._native = _NativeProblem(self.packed)
        self._lib = self._native.lib
        self._counters = (0, 0, 0, 0)
        self._totals = [0, 0, 0, 0]

    @staticmethod
    def _set_device(device: str):
        if device is None or not str(device).startswith("cuda"):
            raise RuntimeError("B200DecoderEvaluator needs a CUDA device (no CPU path)")
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA is not available")
        dev = torch.device(device)
        torch.cuda.set_device(dev.index if dev.index is not None else 0)
        torch.cuda.init()

    def _check_input(self, chromosomes) -> np.ndarray:
        chrom = np.ascontiguousarray(chromosomes, dtype=np.float32)
        if chrom.ndim != 2:
            raise RuntimeError("chromosomes must be a 2D float32 array")  # full_native_decoder.py:567-569
        if chrom.shape[1] != 2 * self.nb_parts:
            raise RuntimeError("chromosomes second dimension must be 2 * nb_parts")  # :571-573
        return chrom

    def evaluate_batch(self, chromosomes: np.ndarray, return_log: bool = False):
        """Makespans of a population (list of float; 1e16 = infeasible)."""
        chrom = self._check_input(chromosomes)
        P = chrom.shape[0]
        out = np.zeros(P, np.float64)
        log = np.zeros((P, self.nb_machines, self.nb_parts), abi.PLACEMENT_DTYPE) if return_log else None
        st = self._lib.brkga_evaluate_host(self._native.handle, abi.ptr(chrom, ctypes.c_float), P,
                                           abi.ptr(out, ctypes.c_double),
                                           log.ctypes.data_as(ctypes.c_void_p) if return_log else None)
        if st != abi.OK:
            raise RuntimeError(f"brkga_evaluate_host failed: {abi.STATUS_NAMES.get(st, st)}")
        t, r, b, sb = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self._lib.brkga_last_counters(self._native.handle, ctypes.byref(t), ctypes.byref(r), ctypes.byref(b),
                                      ctypes.byref(sb))
        self._counters = (t.value, r.value, b.value, sb.value)
        self._totals[0] += P
        self._totals[1] += t.value
        self._totals[2] += r.value
        self._totals[3] += b.value
        return (out.tolist(), log) if return_log else out.tolist()

    @property
    def last_counters(self):
        """(placement tests, 32-row chunks searched, plates opened, scan bytes) of the last call."""
        return self._counters

    def get_profile_summary(self) -> str:
        """Counterpart of ``FullNativeDecoderEvaluator.get_profile_summary`` (:2970-2975)."""
        d, t, r, b = self._totals
        return (f"decodes={d} placement_tests={t} row_chunks={r} plates={b} "
                f"tests_per_decode={t / max(d, 1):.1f}")

    def reset_profile(self) -> None:
        self._totals = [0, 0, 0, 0]

    def close(self):
        self._native.close()


class DeviceDecoder:
    """Stream-ordered decoding of device-resident populations (torch tensors).

    Holds a workspace sized for up to ``max_pop`` chromosomes; ``decode`` is
    asynchronous (no host synchronisation, no allocation) and therefore safe
    to capture in a CUDA graph.  Check ``status`` (a device int32) for
    BRKGA_ERR_CAPACITY after a run when plates may overflow the pool.
    """

    def __init__(self, packed: PackedProblem, max_pop: int, pool_bins: int = 0, device=None):
        import torch
        self.torch = torch
        self.packed = packed
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        with torch.cuda.device(self.device):
            torch.cuda.init()
            self.native = _NativeProblem(packed)
            self.lib = self.native.lib
            self.max_pop = int(max_pop)
            self.pool_bins = int(pool_bins)
            nbytes = ctypes.c_size_t()
            abi.check(self.lib.brkga_workspace_bytes(self.native.handle, self.max_pop, self.pool_bins,
                                                     ctypes.byref(nbytes)), "brkga_workspace_bytes")
            self.ws_bytes = nbytes.value
            self.workspace = torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.device)
            self.status = torch.zeros(1, dtype=torch.int32, device=self.device)

    def workspace_bytes(self, P: int) -> int:
        nbytes = ctypes.c_size_t()
        abi.check(self.lib.brkga_workspace_bytes(self.native.handle, int(P), self.pool_bins, ctypes.byref(nbytes)))
        return nbytes.value

    def launch_config(self, items: Optional[int] = None):
        """(warps per item, CTAs per SM, plates per item in shared memory, resident CTAs, task_max) of a
        decode launch of ``items`` items (default: a full population, ``max_pop`` x machines)."""
        return self.native.launch_config(self.max_pop * self.packed.n_machines if items is None else items)

    def set_launch_config(self, warps_per_item: int = 0, ctas_per_sm: int = 0, smem_plates: int = -1,
                          task_max: int = -1):
        """Change the decode kernel's launch configuration (defaults: automatic)
        and regrow the workspace when the new shape needs more."""
        self.native.set_launch_config(warps_per_item, ctas_per_sm, smem_plates, task_max)
        need = self.workspace_bytes(self.max_pop)
        if need > self.ws_bytes:
            self.workspace = self.torch.empty(need, dtype=self.torch.uint8, device=self.device)
        self.ws_bytes = max(need, self.ws_bytes)

    def decode(self, chrom, out=None, log=None, stream=None, kernel_events=None):
        """Decode ``chrom`` (cuda float32 [P, 2N]) into ``out`` (cuda float64 [P]).

        ``kernel_events`` = (start, end) torch.cuda.Event pair recorded on the
        launch stream right around the decode kernel (stage 2).
        """
        torch = self.torch
        if chrom.dtype != torch.float32 or chrom.dim() != 2 or chrom.shape[1] != 2 * self.packed.n_genes:
            raise RuntimeError("chromosomes must be a float32 [P, 2N] CUDA tensor")
        if not chrom.is_cuda or not chrom.is_contiguous():
            raise RuntimeError("chromosomes must be a contiguous CUDA tensor")
        P = chrom.shape[0]
        if P > self.max_pop:
            raise RuntimeError(f"population {P} exceeds the workspace capacity {self.max_pop}")
        if out is None:
            out = torch.empty(P, dtype=torch.float64, device=chrom.device)
        if log is not None and (log.dtype != torch.int32 or tuple(log.shape) != (P, self.packed.n_machines,
                                                                                  self.packed.n_genes, 5)):
            raise RuntimeError("log must be int32 [P, M, N, 5]")
        s = stream if stream is not None else torch.cuda.current_stream(chrom.device)
        args = (self.native.handle, ctypes.c_void_p(chrom.data_ptr()), P, ctypes.c_void_p(out.data_ptr()),
                ctypes.c_void_p(log.data_ptr()) if log is not None else None,
                ctypes.c_void_p(self.status.data_ptr()), ctypes.c_void_p(self.workspace.data_ptr()),
                self.ws_bytes, self.pool_bins, ctypes.c_void_p(s.cuda_stream))
        if kernel_events is None:
            abi.check(self.lib.brkga_decode(*args), "brkga_decode")
        else:
            abi.check(self.lib.brkga_decode_stage(1, *args), "brkga_decode_stage")
            kernel_events[0].record(s)
            abi.check(self.lib.brkga_decode_stage(2, *args), "brkga_decode_stage")
            kernel_events[1].record(s)
            abi.check(self.lib.brkga_decode_stage(3, *args), "brkga_decode_stage")
        return out

    def counters(self):
        """(placement tests, row chunks, plates, scan bytes) of the last decode (synchronises)."""
        c = self.workspace[8:8 + 32].view(self.torch.int64).cpu().tolist()
        return tuple(int(v) for v in c)


class MultiDecoder:
    """Decodes populations of several independent instances in one launch.

    ``packs`` is a list of ``PackedProblem`` (up to ``abi.MAX_INSTANCES``),
    each with its own parts, machines and plate sizes; ``max_pops[k]`` bounds
    the rows of instance k per call.  ``decode`` takes one CUDA float32
    tensor [P_k, 2 N_k] per instance (``decode_concat`` the rows already
    concatenated) and returns the makespans of all rows, instance after
    instance, from one launch of each kernel: every (chromosome, machine)
    item of every instance goes to the same persistent decode kernel.
    Stream-ordered, no allocation: capturable in a CUDA graph.
    """

    def __init__(self, packs, max_pops, pool_bins: int = 0, device=None):
        import torch
        self.torch = torch
        self.packs = list(packs)
        if len(max_pops) != len(self.packs):
            raise ValueError("one population bound per instance")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.n_genes = [p.n_genes for p in self.packs]
        self.n_machines = [p.n_machines for p in self.packs]
        with torch.cuda.device(self.device):
            torch.cuda.init()
            self.native = _NativeProblem(self.packs)
            self.lib = self.native.lib
            self.max_pops = np.ascontiguousarray(max_pops, dtype=np.int32)
            self.pool_bins = int(pool_bins)
            self.ws_bytes = self.workspace_bytes(self.max_pops)
            self.workspace = torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.device)
            self.status = torch.zeros(1, dtype=torch.int32, device=self.device)

    @property
    def n_instances(self) -> int:
        return len(self.packs)

    def workspace_bytes(self, pops) -> int:
        pops = np.ascontiguousarray(pops, dtype=np.int32)
        nbytes = ctypes.c_size_t()
        abi.check(self.lib.brkga_workspace_bytes_multi(self.native.handle, abi.ptr(pops, ctypes.c_int32),
                                                       self.pool_bins, ctypes.byref(nbytes)),
                  "brkga_workspace_bytes_multi")
        return nbytes.value

    def launch_config(self, items: Optional[int] = None):
        """Launch configuration for ``items`` items (default: every instance at ``max_pops``)."""
        if items is None:
            items = int(sum(int(p) * m for p, m in zip(self.max_pops, self.n_machines)))
        return self.native.launch_config(items)

    def set_launch_config(self, warps_per_item: int = 0, ctas_per_sm: int = 0, smem_plates: int = -1,
                          task_max: int = -1):
        self.native.set_launch_config(warps_per_item, ctas_per_sm, smem_plates, task_max)
        need = self.workspace_bytes(self.max_pops)
        if need > self.ws_bytes:
            self.workspace = self.torch.empty(need, dtype=self.torch.uint8, device=self.device)
        self.ws_bytes = max(need, self.ws_bytes)

    def _check_pops(self, pops) -> np.ndarray:
        pops = np.ascontiguousarray(pops, dtype=np.int32)
        if pops.shape != (self.n_instances,) or (pops < 0).any() or (pops > self.max_pops).any():
            raise RuntimeError("population sizes must be 0 <= P_k <= max_pops[k], one per instance")
        return pops

    def decode_concat(self, chrom, pops, out=None, log=None, stream=None, kernel_events=None):
        """Decode rows already concatenated instance after instance (flat
        float32 CUDA tensor of sum_k P_k * 2 N_k keys) into ``out`` (float64 [sum P_k])."""
        torch = self.torch
        pops = self._check_pops(pops)
        n_keys = int(sum(int(p) * 2 * n for p, n in zip(pops, self.n_genes)))
        if chrom.dtype != torch.float32 or not chrom.is_cuda or not chrom.is_contiguous() or chrom.numel() != n_keys:
            raise RuntimeError(f"chromosomes must be a contiguous float32 CUDA tensor of {n_keys} keys")
        rows = int(pops.sum())
        if out is None:
            out = torch.empty(rows, dtype=torch.float64, device=chrom.device)
        n_log = int(sum(int(p) * m * n for p, m, n in zip(pops, self.n_machines, self.n_genes)))
        if log is not None and (log.dtype != torch.int32 or log.numel() != n_log * 5):
            raise RuntimeError(f"log must be int32 with {n_log} x 5 entries")
        s = stream if stream is not None else torch.cuda.current_stream(chrom.device)
        args = (self.native.handle, ctypes.c_void_p(chrom.data_ptr()), abi.ptr(pops, ctypes.c_int32),
                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(log.data_ptr()) if log is not None else None,
                ctypes.c_void_p(self.status.data_ptr()), ctypes.c_void_p(self.workspace.data_ptr()),
                self.ws_bytes, self.pool_bins, ctypes.c_void_p(s.cuda_stream))
        if kernel_events is None:
            abi.check(self.lib.brkga_decode_multi(*args), "brkga_decode_multi")
        else:
            abi.check(self.lib.brkga_decode_multi_stage(1, *args), "brkga_decode_multi_stage")
            kernel_events[0].record(s)
            abi.check(self.lib.brkga_decode_multi_stage(2, *args), "brkga_decode_multi_stage")
            kernel_events[1].record(s)
            abi.check(self.lib.brkga_decode_multi_stage(3, *args), "brkga_decode_multi_stage")
        return out

    def decode_at(self, chrom, chrom_offsets, pops, out, out_offsets, stream=None, kernel_events=None):
        """Decode instance k's ``pops[k]`` rows starting at float ``chrom_offsets[k]``
        of ``chrom`` into ``out`` from element ``out_offsets[k]`` (one launch of
        each kernel; both tensors are flat CUDA buffers the caller lays out)."""
        torch = self.torch
        pops = self._check_pops(pops)
        co = np.ascontiguousarray(chrom_offsets, dtype=np.int64)
        oo = np.ascontiguousarray(out_offsets, dtype=np.int64)
        if co.shape != pops.shape or oo.shape != pops.shape:
            raise RuntimeError("one chromosome offset and one makespan offset per instance")
        for k, p in enumerate(pops):
            if p and (co[k] < 0 or co[k] + int(p) * 2 * self.n_genes[k] > chrom.numel() or oo[k] < 0
                      or oo[k] + int(p) > out.numel()):
                raise RuntimeError(f"instance {k}: rows outside the buffers")
        if chrom.dtype != torch.float32 or out.dtype != torch.float64 or not (chrom.is_cuda and out.is_cuda):
            raise RuntimeError("chrom must be float32 and out float64 CUDA tensors")
        s = stream if stream is not None else torch.cuda.current_stream(chrom.device)
        args = (self.native.handle, ctypes.c_void_p(chrom.data_ptr()), abi.ptr(co, ctypes.c_int64),
                abi.ptr(pops, ctypes.c_int32), ctypes.c_void_p(out.data_ptr()), abi.ptr(oo, ctypes.c_int64), None,
                ctypes.c_void_p(self.status.data_ptr()), ctypes.c_void_p(self.workspace.data_ptr()),
                self.ws_bytes, self.pool_bins, ctypes.c_void_p(s.cuda_stream))
        if kernel_events is None:
            abi.check(self.lib.brkga_decode_multi_at(0, *args), "brkga_decode_multi_at")
        else:
            abi.check(self.lib.brkga_decode_multi_at(1, *args), "brkga_decode_multi_at")
            kernel_events[0].record(s)
            abi.check(self.lib.brkga_decode_multi_at(2, *args), "brkga_decode_multi_at")
            kernel_events[1].record(s)
            abi.check(self.lib.brkga_decode_multi_at(3, *args), "brkga_decode_multi_at")
        return out

    def decode(self, chroms, stream=None):
        """Makespans (list of float64 CUDA tensors, one per instance) of one
        population per instance (float32 CUDA tensors [P_k, 2 N_k])."""
        torch = self.torch
        if len(chroms) != self.n_instances:
            raise RuntimeError("one population per instance")
        for c, n in zip(chroms, self.n_genes):
            if c.dim() != 2 or c.shape[1] != 2 * n:
                raise RuntimeError("population k must be [P_k, 2 N_k]")
        pops = [int(c.shape[0]) for c in chroms]
        flat = torch.cat([c.reshape(-1) for c in chroms]).contiguous()
        out = self.decode_concat(flat, pops, stream=stream)
        return list(torch.split(out, pops))

    def counters(self):
        """(placement tests, row chunks, plates, scan bytes) of the last decode (synchronises)."""
        c = self.workspace[8:8 + 32].view(self.torch.int64).cpu().tolist()
        return tuple(int(v) for v in c)

    def close(self):
        self.native.close()
