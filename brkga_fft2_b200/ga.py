"""BRKGA on the GPU: the reference's GA loop with every generation on the device.

``DeviceBRKGA`` mirrors ``BRKGA_alg3.BRKGA`` (``BRKGA_alg3.py:23-281``): the
same constructor parameters (``num_generations``, ``num_individuals``,
``num_elites``, ``num_mutants``, ``eliteCProb``, ``initialSol``), ``fit()``,
``history`` with ``mean`` / ``min`` / ``time`` per generation, ``best_fitness``
and ``solution``.  Population and fitness stay in device memory; one
generation — rank, elite copy, Philox mutants, rho-biased crossover, decode of
the non-elite rows, statistics — is a fixed sequence of kernels on one stream,
captured once into a CUDA graph per buffer parity and replayed.  Nothing is
read back to the host until ``fit`` returns.
"""
from __future__ import annotations

import ctypes
import time
from typing import Optional

import numpy as np

from . import abi
from .evaluator import DeviceDecoder
from .problem import THRESH_F32, PackedProblem, pack_problem


class DeviceBRKGA:
    def __init__(self, problem_data, nbParts, nbMachines, thresholds, instanceParts, initialSol=None,
                 collision_backend=None, eval_mode="b200", eval_workers=0, eval_chunksize=1,
                 num_generations=200, num_individuals=100, num_elites=12, num_mutants=18, eliteCProb=0.7,
                 seed: int = 0, use_graph: bool = True, threshold_mode: int = THRESH_F32,
                 packed: Optional[PackedProblem] = None, device=None):
        import torch
        del collision_backend, eval_mode, eval_workers, eval_chunksize
        self.torch = torch
        self.N = int(nbParts)
        self.nbMachines = int(nbMachines)
        self.num_generations = int(num_generations)
        self.num_individuals = int(num_individuals)
        self.num_elites = int(num_elites)
        self.num_mutants = int(num_mutants)
        self.num_gene = 2 * self.N
        self.eliteCProb = float(eliteCProb)
        self.seed = int(seed)
        self.use_graph = bool(use_graph)
        self.initialSol = None if initialSol is None else np.asarray(initialSol, np.float32)
        if not (1 <= self.num_elites and self.num_elites + self.num_mutants <= self.num_individuals):
            raise ValueError("need 1 <= num_elites and num_elites + num_mutants <= num_individuals")
        if self.num_individuals > 8192:
            raise ValueError("num_individuals must be <= 8192 (single-CTA rank)")
        self.packed = packed if packed is not None else pack_problem(
            problem_data, nbParts, nbMachines, thresholds, instanceParts, threshold_mode)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        P, K = self.num_individuals, self.num_gene
        self.decoder = DeviceDecoder(self.packed, max_pop=P, pool_bins=max(1024, 4 * P * self.nbMachines),
                                     device=self.device)
        self.lib = self.decoder.lib
        dev = self.device
        self.pop = [torch.zeros(P, K, dtype=torch.float32, device=dev) for _ in range(2)]
        self.fitness_buf = [torch.zeros(P, dtype=torch.float64, device=dev) for _ in range(2)]
        self.order = torch.zeros(P, dtype=torch.int32, device=dev)
        self.generation = torch.zeros(1, dtype=torch.int64, device=dev)
        self.history_dev = torch.zeros(self.num_generations + 1, 2, dtype=torch.float64, device=dev)
        self.best_fit = torch.full((1,), float("inf"), dtype=torch.float64, device=dev)
        self.best_sol = torch.zeros(K, dtype=torch.float32, device=dev)
        self.history = {"mean": [], "min": [], "time": []}
        self.best_fitness = -1
        self.solution = None
        self.used_bins = -1
        self._graphs = None

    # ---- kernels of one generation ------------------------------------------------
    @staticmethod
    def _ptr(t):
        return ctypes.c_void_p(t.data_ptr())

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def _track(self, cur):
        abi.check(self.lib.brkga_ga_track(self._ptr(self.fitness_buf[cur]), self._ptr(self.pop[cur]),
                                          self.num_individuals, self.num_gene, self._ptr(self.generation),
                                          self._ptr(self.history_dev), self.num_generations + 1,
                                          self._ptr(self.best_fit), self._ptr(self.best_sol), self._stream()),
                  "brkga_ga_track")

    def _step(self, cur):
        nxt = 1 - cur
        P, K, ne, nm = self.num_individuals, self.num_gene, self.num_elites, self.num_mutants
        abi.check(self.lib.brkga_ga_rank(self._ptr(self.fitness_buf[cur]), P, self._ptr(self.order), self._stream()),
                  "brkga_ga_rank")
        abi.check(self.lib.brkga_ga_breed(self._ptr(self.pop[cur]), self._ptr(self.fitness_buf[cur]), self._ptr(self.order),
                                          P, K, ne, nm, ctypes.c_float(self.eliteCProb), ctypes.c_uint64(self.seed),
                                          self._ptr(self.generation), self._ptr(self.pop[nxt]),
                                          self._ptr(self.fitness_buf[nxt]), self._stream()), "brkga_ga_breed")
        if P > ne:
            self.decoder.decode(self.pop[nxt][ne:], out=self.fitness_buf[nxt][ne:])
        self._track(nxt)

    def _initial(self):
        P, K = self.num_individuals, self.num_gene
        skip = 1 if self.initialSol is not None else 0
        abi.check(self.lib.brkga_ga_init_population(self._ptr(self.pop[0]), P, K, ctypes.c_uint64(self.seed), skip,
                                                    self._stream()), "brkga_ga_init_population")
        if skip:
            self.pop[0][0].copy_(self.torch.from_numpy(self.initialSol))
        self.decoder.decode(self.pop[0], out=self.fitness_buf[0])
        self._track(0)

    def _capture(self):
        torch = self.torch
        graphs = []
        side = torch.cuda.Stream(self.device)
        # the first step runs eagerly (warm-up) inside fit(); capture both parities here
        for cur in (0, 1):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=side):
                self._step(cur)
            graphs.append(g)
        return graphs

    # ---- public ---------------------------------------------------------------------
    def fit(self, verbose: bool = False):
        """Run ``num_generations`` generations (BRKGA_alg3.py:210-281)."""
        torch = self.torch
        with torch.cuda.device(self.device):
            self.generation.zero_()
            self.best_fit.fill_(float("inf"))
            start = time.perf_counter()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev0.record()
            self._initial()
            events = []
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            events.append(e)
            cur = 0
            G = self.num_generations
            if self.use_graph and G >= 1:
                # generation 1 eagerly: warms up the library before capture
                self._step(cur)
                cur = 1 - cur
                e = torch.cuda.Event(enable_timing=True)
                e.record()
                events.append(e)
                if G > 1:
                    # capture records the launches without running them
                    torch.cuda.synchronize()
                    if self._graphs is None:
                        self._graphs = self._capture()
                    graphs = self._graphs
                    for _ in range(G - 1):
                        graphs[cur].replay()
                        cur = 1 - cur
                        e = torch.cuda.Event(enable_timing=True)
                        e.record()
                        events.append(e)
            else:
                for _ in range(G):
                    self._step(cur)
                    cur = 1 - cur
                    e = torch.cuda.Event(enable_timing=True)
                    e.record()
                    events.append(e)
            torch.cuda.synchronize()
            wall = time.perf_counter() - start
            if int(self.decoder.status.item()) != 0:
                raise RuntimeError(f"decoder status {int(self.decoder.status.item())} during the GA run")
            hist = self.history_dev.cpu().numpy()
            self.history = {"min": [float(v) for v in hist[:G + 1, 0]],
                            "mean": [float(v) for v in hist[:G + 1, 1]],
                            "time": [ev0.elapsed_time(e) / 1000.0 for e in events]}
            self.best_fitness = float(self.best_fit.item())
            self.solution = self.best_sol.cpu().numpy()
            self.used_bins = int(np.floor(self.best_fitness))
            self.population = self.pop[cur].cpu().numpy()
            self.fitness = self.fitness_buf[cur].cpu().numpy()
            self.wall_time = wall
            if verbose:
                for g in range(G + 1):
                    print(f"Generation {g}: Best={self.history['min'][g]:.4f} Mean={self.history['mean'][g]:.4f} "
                          f"Time={self.history['time'][g]:.3f}s")
        return "feasible"
