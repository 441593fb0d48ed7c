"""Many independent BRKGAs on one GPU, one decode launch per generation for all.

``MultiBRKGA`` runs the reference's GA loop (``BRKGA_alg3.py:210-265``) on K
instances at once (up to ``abi.MAX_INSTANCES``; own parts, machines, plate
sizes and population sizes).  Instance k evolves exactly as
``DeviceBRKGA`` would with seed ``seed + k``: the same Philox streams, rank,
elite copy, mutants, rho-biased crossover and statistics kernels run on its
slice of one flat population buffer.  What is shared is the decode: the
non-elite rows of all K populations go to one ``brkga_decode_multi_at``
launch, so the persistent decode kernel sees every (chromosome, machine)
item of every instance at once and starts the longest first.  One
generation — K ranks, K breeds, one decode, K statistics — is captured once
per buffer parity as a CUDA graph and replayed.

The reference has no multi-instance driver: it runs one ``BRKGA`` per
instance and process (``BRKGA_alg3.py:605-624``).
"""
from __future__ import annotations

import ctypes
import time
from typing import Optional, Sequence

import numpy as np

from . import abi
from .evaluator import MultiDecoder
from .ga import MAX_RANK


def _per_instance(v, K, name):
    if np.isscalar(v):
        return [v] * K
    if len(v) != K:
        raise ValueError(f"{name}: one value per instance")
    return list(v)


class MultiBRKGA:
    def __init__(self, packs: Sequence, num_generations: int = 100, num_individuals=256, num_elites=None,
                 num_mutants=None, eliteCProb: float = 0.7, seed: int = 0, use_graph: bool = True, device=None,
                 launch_config: Optional[tuple] = None):
        import torch
        self.torch = torch
        self.packs = list(packs)
        K = self.K = len(self.packs)
        if not 1 <= K <= abi.MAX_INSTANCES:
            raise ValueError(f"1 to {abi.MAX_INSTANCES} instances")
        self.num_generations = int(num_generations)
        self.P = [int(p) for p in _per_instance(num_individuals, K, "num_individuals")]
        ne = _per_instance(num_elites, K, "num_elites") if num_elites is not None else [max(1, p // 5) for p in self.P]
        nm = (_per_instance(num_mutants, K, "num_mutants") if num_mutants is not None
              else [int(round(0.15 * p)) for p in self.P])
        self.ne, self.nm = [int(v) for v in ne], [int(v) for v in nm]
        for P, e, m in zip(self.P, self.ne, self.nm):
            if not (1 <= e and e + m <= P <= MAX_RANK):
                raise ValueError(f"need 1 <= num_elites, num_elites + num_mutants <= num_individuals <= {MAX_RANK}")
        self.rho = float(eliteCProb)
        if not 0.0 <= self.rho <= 1.0 or self.num_generations < 0:
            raise ValueError("need 0 <= eliteCProb <= 1 and num_generations >= 0")
        self.seed = int(seed)
        self.use_graph = bool(use_graph)
        self.nkeys = [2 * p.n_genes for p in self.packs]
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        # flat layout: instance k's population block [P_k, 2N_k] at pop_off[k] floats, fitness at fit_off[k]
        self.pop_off = np.cumsum([0] + [P * n for P, n in zip(self.P, self.nkeys)])[:-1].astype(np.int64)
        self.fit_off = np.cumsum([0] + self.P)[:-1].astype(np.int64)
        self.sol_off = np.cumsum([0] + self.nkeys)[:-1].astype(np.int64)
        n_keys = int(sum(P * n for P, n in zip(self.P, self.nkeys)))
        n_rows = int(sum(self.P))
        items = int(sum(P * p.n_machines for P, p in zip(self.P, self.packs)))
        self.decoder = MultiDecoder(self.packs, max_pops=self.P, pool_bins=max(1024, 4 * items), device=self.device)
        if launch_config is not None:
            self.decoder.set_launch_config(*launch_config)
        self.lib = self.decoder.lib
        dev = self.device
        G1 = self.num_generations + 1
        self.pop = [torch.zeros(n_keys, dtype=torch.float32, device=dev) for _ in range(2)]
        self.fit_buf = [torch.zeros(n_rows, dtype=torch.float64, device=dev) for _ in range(2)]
        self.order = torch.zeros(n_rows, dtype=torch.int32, device=dev)
        self.generation = torch.zeros(K, dtype=torch.int64, device=dev)
        self.history_dev = torch.zeros(K, G1, 2, dtype=torch.float64, device=dev)
        self.best_fit = torch.full((K,), float("inf"), dtype=torch.float64, device=dev)
        self.best_sol = torch.zeros(int(sum(self.nkeys)), dtype=torch.float32, device=dev)
        # decode of the non-elite rows of every block, in place
        self.dec_chrom_off = np.array([o + e * n for o, e, n in zip(self.pop_off, self.ne, self.nkeys)], np.int64)
        self.dec_out_off = np.array([o + e for o, e in zip(self.fit_off, self.ne)], np.int64)
        self.dec_pops = np.array([P - e for P, e in zip(self.P, self.ne)], np.int32)
        self._graphs = {}
        self._prepared = False
        self.history = None

    # ---- pointers into the flat buffers ------------------------------------------------
    @staticmethod
    def _at(t, offset=0):
        return ctypes.c_void_p(t.data_ptr() + int(offset) * t.element_size())

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def _track(self, cur):
        G1 = self.num_generations + 1
        for k in range(self.K):
            abi.check(self.lib.brkga_ga_track(
                self._at(self.fit_buf[cur], self.fit_off[k]), self._at(self.pop[cur], self.pop_off[k]), self.P[k],
                self.nkeys[k], self._at(self.generation, k), self._at(self.history_dev, k * G1 * 2), G1,
                self._at(self.best_fit, k), self._at(self.best_sol, self.sol_off[k]), self._stream()),
                "brkga_ga_track")

    def _step(self, cur):
        nxt = 1 - cur
        s = self._stream()
        for k in range(self.K):
            fo, po = self.fit_off[k], self.pop_off[k]
            abi.check(self.lib.brkga_ga_rank(self._at(self.fit_buf[cur], fo), self.P[k], self._at(self.order, fo), s),
                      "brkga_ga_rank")
            abi.check(self.lib.brkga_ga_breed(
                self._at(self.pop[cur], po), self._at(self.fit_buf[cur], fo), self._at(self.order, fo), self.P[k],
                self.nkeys[k], self.ne[k], self.nm[k], ctypes.c_float(self.rho), ctypes.c_uint64(self.seed + k),
                self._at(self.generation, k), self._at(self.pop[nxt], po), self._at(self.fit_buf[nxt], fo), s),
                "brkga_ga_breed")
        self.decoder.decode_at(self.pop[nxt], self.dec_chrom_off, self.dec_pops, self.fit_buf[nxt], self.dec_out_off)
        self._track(nxt)

    def _initial(self):
        s = self._stream()
        for k in range(self.K):
            abi.check(self.lib.brkga_ga_init_population(self._at(self.pop[0], self.pop_off[k]), self.P[k],
                                                        self.nkeys[k], ctypes.c_uint64(self.seed + k), 0, s),
                      "brkga_ga_init_population")
        self.decoder.decode_at(self.pop[0], self.pop_off, self.P, self.fit_buf[0], self.fit_off)
        self._track(0)

    def prepare(self):
        """Load every kernel with one eager generation per parity, then capture
        one CUDA graph per parity; ``fit`` afterwards only replays them."""
        torch = self.torch
        with torch.cuda.device(self.device):
            self.generation.zero_()
            self._initial()
            self._step(0)
            self._step(1)
            torch.cuda.synchronize()
            side = torch.cuda.Stream(self.device)
            for cur in (0, 1):
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=side):
                    self._step(cur)
                self._graphs[cur] = g
            torch.cuda.synchronize()
        self._prepared = True

    def fit(self):
        """``num_generations`` generations of every instance.  Sets ``history``
        (per instance ``min`` / ``mean`` per generation), ``best_fitness`` [K],
        ``solutions`` (list of best chromosomes), ``populations`` / ``fitness``
        (final, per instance), ``generation_ms`` (device time per generation)."""
        torch = self.torch
        if self.use_graph and not self._prepared:
            self.prepare()
        with torch.cuda.device(self.device):
            self.generation.zero_()
            self.best_fit.fill_(float("inf"))
            self.decoder.status.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(self.num_generations + 2)]
            ev[0].record()
            self._initial()
            ev[1].record()
            cur = 0
            for g in range(1, self.num_generations + 1):
                if self.use_graph:
                    self._graphs[cur].replay()
                else:
                    self._step(cur)
                ev[g + 1].record()
                cur = 1 - cur
            torch.cuda.synchronize()
            self.wall_time = time.perf_counter() - t0
            st = int(self.decoder.status.item())
            if st != 0:
                raise abi.BrkgaError(st, "decoder status during the GA run")
            self.generation_ms = [ev[g].elapsed_time(ev[g + 1]) for g in range(1, self.num_generations + 1)]
            self.initial_ms = ev[0].elapsed_time(ev[1])
            hist = self.history_dev.cpu().numpy()
            self.history = [{"min": hist[k, :, 0].tolist(), "mean": hist[k, :, 1].tolist()} for k in range(self.K)]
            self.best_fitness = self.best_fit.cpu().numpy()
            sol = self.best_sol.cpu().numpy()
            self.solutions = [sol[o:o + n] for o, n in zip(self.sol_off, self.nkeys)]
            pop, fit = self.pop[cur].cpu().numpy(), self.fit_buf[cur].cpu().numpy()
            self.populations = [pop[o:o + P * n].reshape(P, n) for o, P, n in zip(self.pop_off, self.P, self.nkeys)]
            self.fitness = [fit[o:o + P] for o, P in zip(self.fit_off, self.P)]
        return self
