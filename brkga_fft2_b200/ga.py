"""BRKGA on the GPU: the reference's GA loop with every generation on the device.

With ``screening=True`` each generation breeds an ``oversample``-times larger
candidate pool, ranks it with the online-trained surrogate
(:mod:`brkga_fft2_b200.surrogate`) and decodes exactly only the best-predicted
``num_individuals - num_elites`` rows; the surrogate then learns from those
exact makespans.  Its Spearman correlation and mean absolute error on the
decoded rows are logged for every generation (``history['spearman']``,
``history['mae']``), and screening is switched off while the mean Spearman of
the last ``check_every`` generations stays below ``spearman_threshold``
(the surrogate keeps learning from plain generations meanwhile).  With
``explore > 0`` that share of the decoded rows is not the surrogate's top but
spread evenly over the rest of the ranked pool, which keeps lower-ranked
offspring in the population.  With ``overlap_training`` (the default) the
surrogate trains on a second stream while the decode kernel runs, on the
rows observed up to the previous generation.  ``surrogate_features`` picks
the surrogate's input: "decode" (per part in decode order its machine, proc
time and height time, then per machine its loads) or "order" (per part its
sequencing key, area and height, the parts sorted by key).  With
``screen_mutants=False`` (the default) the mutants of a screened generation
enter unscreened, as in the plain GA, and only the crossover offspring are
oversampled and ranked (a surrogate ranks random-key mutants low, so
screening them too removes BRKGA's diversity injection); ``True`` screens
mutants and offspring together.  ``screen_mode="family"`` (the default)
keeps the plain GA's parents: every offspring slot's (elite, non-elite) pair
makes ``oversample`` children and the surrogate keeps the best-predicted one,
the mutants entering unscreened; ``"pool"`` ranks the whole oversampled pool
and keeps its best-predicted rows (``screen_mutants`` and ``explore`` apply
there).  Ranking the whole pool picks children that resemble the current
elites and measurably collapses the population at P100M4 (screened runs
stalling above the plain GA's best); choosing among siblings does not change
who breeds with whom.

With ``audit_fraction > 0`` every generation also copies an evenly spaced
sample of the rows it decoded (that fraction of them), with their exact
makespans, into ``audit`` = (chromosomes [G+1, n, 2N], makespans [G+1, n]),
so a run can be checked against an independent decoder afterwards without
stopping the graph replays.

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

MAX_RANK = 65536  # brkga_ga_rank


class DeviceBRKGA:
    def __init__(self, problem_data, nbParts, nbMachines, thresholds, instanceParts, initialSol=None,
                 collision_backend=None, eval_mode="b200", eval_workers=0, eval_chunksize=1,
                 num_generations=200, num_individuals=100, num_elites=12, num_mutants=18, eliteCProb=0.7,
                 seed: int = 0, use_graph: bool = True, threshold_mode: int = THRESH_F32,
                 packed: Optional[PackedProblem] = None, device=None, screening: bool = False,
                 oversample: int = 5, train_steps: int = 8, train_batch: int = 512, lr: float = 1e-3,
                 spearman_threshold: float = 0.3, check_every: int = 5, warmup_generations: int = 5,
                 buffer_capacity: int = 200_000, target: Optional[float] = None, audit_fraction: float = 0.0,
                 explore: float = 0.0, overlap_training: bool = True, surrogate_features: str = "decode",
                 screen_mutants: bool = False, screen_mode: str = "family"):
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
        if self.num_individuals > MAX_RANK:
            raise ValueError(f"num_individuals must be <= {MAX_RANK} (device rank)")
        if self.num_generations < 0:
            raise ValueError("num_generations must be >= 0")
        if not 0.0 <= self.eliteCProb <= 1.0:
            raise ValueError("eliteCProb must be in [0, 1]")
        if not 0.0 <= float(audit_fraction) <= 1.0:
            raise ValueError("audit_fraction must be in [0, 1]")
        if screening and (int(oversample) < 1 or not 0.0 <= float(explore) <= 1.0 or int(train_steps) < 0
                          or int(train_batch) < 1):
            raise ValueError("screening needs oversample >= 1, 0 <= explore <= 1, train_steps >= 0 and "
                             "train_batch >= 1")
        if screening and screen_mode not in ("family", "pool"):
            raise ValueError('screen_mode must be "family" or "pool"')
        if screening and screen_mode == "family" and (screen_mutants or float(explore) > 0):
            raise ValueError("screen_mutants and explore apply to screen_mode='pool'")
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
        self._graphs = {}
        self._prepared = False
        self.target = target
        # audit sample: evenly spaced rows among those decoded every generation, kept with their makespans
        self.audit = None
        n_dec = P - self.num_elites
        self.n_audit = min(n_dec, max(1, int(np.ceil(audit_fraction * n_dec)))) if audit_fraction > 0 and n_dec else 0
        if self.n_audit:
            idx = self.num_elites + (np.arange(self.n_audit) * n_dec) // self.n_audit
            self.audit_index = torch.from_numpy(idx.astype(np.int32)).to(dev)
            self.audit_pop = torch.zeros(self.num_generations + 1, self.n_audit, K, dtype=torch.float32, device=dev)
            self.audit_fit = torch.zeros(self.num_generations + 1, self.n_audit, dtype=torch.float64, device=dev)
        self.screening = bool(screening)
        self.overlap_training = False
        if self.screening:
            from .surrogate import Surrogate
            self.oversample = int(oversample)
            self.train_steps, self.train_batch, self.lr = int(train_steps), int(train_batch), float(lr)
            self.spearman_threshold = float(spearman_threshold)
            self.check_every = max(1, int(check_every))
            self.warmup_generations = int(warmup_generations)
            rows = P - self.num_elites
            # rows that enter every screened generation as they are: the elites
            # and, unless screen_mutants, the mutants; the rest are offspring
            # chosen from an oversampled candidate pool by the surrogate
            self.screen_mode = screen_mode
            self.screen_mutants = bool(screen_mutants)
            self.n_fixed = self.num_elites + (0 if self.screen_mutants else self.num_mutants)
            n_screen = P - self.n_fixed
            self.pool_rows = self.n_fixed + self.oversample * n_screen
            if self.pool_rows - self.n_fixed > MAX_RANK:
                raise ValueError(f"oversampled pool too large for the device rank ({MAX_RANK} rows)")
            self.pool = torch.zeros(self.pool_rows, K, dtype=torch.float32, device=dev)
            self.pool_fit = torch.zeros(self.pool_rows, dtype=torch.float64, device=dev)
            self.pred = torch.zeros(max(self.pool_rows - self.n_fixed, 1), dtype=torch.float64, device=dev)
            self.order_pool = torch.zeros(max(self.pool_rows - self.n_fixed, 1), dtype=torch.int32, device=dev)
            self.pred_sel = torch.zeros(max(rows, 1), dtype=torch.float64, device=dev)
            self.o_pred = torch.zeros(max(rows, 1), dtype=torch.int32, device=dev)
            self.o_exact = torch.zeros(max(rows, 1), dtype=torch.int32, device=dev)
            self.stat_scratch = torch.zeros(2 * max(rows, 1), dtype=torch.int32, device=dev)
            self.stats_dev = torch.full((self.num_generations + 1, 2), float("nan"), dtype=torch.float64, device=dev)
            # one prediction batch covers the whole candidate pool
            batch = max(self.train_batch, self.pool_rows - self.n_fixed, rows, 128)
            self.surrogate = Surrogate(self.decoder.native, max_batch=(batch + 127) // 128 * 128,
                                       buffer_capacity=buffer_capacity, seed=self.seed ^ 0x5EED,
                                       features=surrogate_features)
            # Training runs on a second stream while the decode kernel runs (on the rows
            # observed up to the previous generation), joined before the next prediction.
            self.overlap_training = bool(overlap_training)
            self._train_stream = torch.cuda.Stream(dev) if self.overlap_training else None
            # the surrogate's quality statistics (two ranks, Spearman, MAE) run on a third
            # stream beside the example-ring update; they only read the predictions and makespans
            self._stats_stream = torch.cuda.Stream(dev)
            # exploration: that share of the decoded rows is spread evenly over the
            # pool's lower-ranked candidates instead of taken from its top
            cand = self.pool_rows - self.n_fixed
            self.n_explore = min(n_screen, max(0, int(round(float(explore) * n_screen))))
            if self.n_explore:
                top = n_screen - self.n_explore
                sel = np.arange(n_screen, dtype=np.int64)
                sel[top:] = top + (np.arange(self.n_explore) * (cand - top)) // self.n_explore
                self.sel_idx = torch.from_numpy(sel).to(dev)
                self.order_sel = torch.zeros(n_screen, dtype=torch.int32, device=dev)

    # ---- kernels of one generation ------------------------------------------------
    @staticmethod
    def _ptr(t):
        return ctypes.c_void_p(t.data_ptr())

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def _track(self, cur):
        if self.n_audit:
            abi.check(self.lib.brkga_ga_audit(self._ptr(self.pop[cur]), self._ptr(self.fitness_buf[cur]),
                                              self._ptr(self.audit_index), self.n_audit, self.num_gene,
                                              self._ptr(self.generation), self.num_generations + 1,
                                              self._ptr(self.audit_pop), self._ptr(self.audit_fit), self._stream()),
                      "brkga_ga_audit")
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

    def _rank(self, values, n, order):
        abi.check(self.lib.brkga_ga_rank(self._ptr(values), n, self._ptr(order), self._stream()), "brkga_ga_rank")

    def _train_fork(self):
        """Start this generation's surrogate training beside the decode (overlap mode)."""
        if self.overlap_training:
            self._train_stream.wait_stream(self.torch.cuda.current_stream(self.device))
            self.surrogate.train(self.train_steps, self.train_batch, self.lr, stream=self._train_stream)

    def _train_join(self):
        if self.overlap_training:
            self.torch.cuda.current_stream(self.device).wait_stream(self._train_stream)

    def _monitor_and_learn(self, nxt, screened=False):
        """Surrogate quality on this generation's decoded rows, then learn from them
        (the training itself ran beside the decode in overlap mode).  In a
        screened generation the quality is that of the predictions that chose
        the screened rows (already in pred_sel, nothing is predicted again);
        otherwise the decoded rows are predicted now."""
        ne, P = self.num_elites, self.num_individuals
        if P - ne < 1:
            return
        decoded = self.pop[nxt][ne:]
        first = self.n_fixed if screened else ne
        rows = P - first
        if rows < 1:
            return
        exact = self.fitness_buf[nxt][first:]
        if not screened:
            self.surrogate.predict(decoded, out=self.pred_sel[:rows])
        main = self.torch.cuda.current_stream(self.device)
        self._stats_stream.wait_stream(main)
        with self.torch.cuda.stream(self._stats_stream):
            self._rank(self.pred_sel, rows, self.o_pred)
            self._rank(exact, rows, self.o_exact)
            abi.check(self.lib.brkga_ga_screen_stats(self._ptr(self.pred_sel), self._ptr(exact),
                                                     self._ptr(self.o_pred), self._ptr(self.o_exact), rows,
                                                     self._ptr(self.generation), self._ptr(self.stats_dev),
                                                     self.num_generations + 1, self._ptr(self.stat_scratch),
                                                     self._stream()), "brkga_ga_screen_stats")
        self.surrogate.observe(decoded, self.fitness_buf[nxt][ne:])
        if not self.overlap_training:
            self.surrogate.train(self.train_steps, self.train_batch, self.lr)
        main.wait_stream(self._stats_stream)

    def _step_learn(self, cur):
        """Plain generation that also measures and trains the surrogate."""
        nxt = 1 - cur
        P, K, ne, nm = self.num_individuals, self.num_gene, self.num_elites, self.num_mutants
        self._rank(self.fitness_buf[cur], P, self.order)
        abi.check(self.lib.brkga_ga_breed(self._ptr(self.pop[cur]), self._ptr(self.fitness_buf[cur]),
                                          self._ptr(self.order), P, K, ne, nm, ctypes.c_float(self.eliteCProb),
                                          ctypes.c_uint64(self.seed), self._ptr(self.generation),
                                          self._ptr(self.pop[nxt]), self._ptr(self.fitness_buf[nxt]),
                                          self._stream()), "brkga_ga_breed")
        self._train_fork()
        if P > ne:
            self.decoder.decode(self.pop[nxt][ne:], out=self.fitness_buf[nxt][ne:])
        self._train_join()
        self._monitor_and_learn(nxt)
        self._track(nxt)

    def _step_screened(self, cur):
        """Oversampled pool -> surrogate ranking -> exact decode of the best-predicted rows."""
        nxt = 1 - cur
        P, K, ne, nm = self.num_individuals, self.num_gene, self.num_elites, self.num_mutants
        rows, nf = P - ne, self.n_fixed
        self._rank(self.fitness_buf[cur], P, self.order)
        family = self.oversample if self.screen_mode == "family" else 1
        pool_mutants = nm * self.oversample if self.screen_mutants else nm
        abi.check(self.lib.brkga_ga_breed_families(self._ptr(self.pop[cur]), self._ptr(self.fitness_buf[cur]),
                                                   self._ptr(self.order), P, self.pool_rows, K, ne, pool_mutants,
                                                   family, ctypes.c_float(self.eliteCProb),
                                                   ctypes.c_uint64(self.seed), self._ptr(self.generation),
                                                   self._ptr(self.pool), self._ptr(self.pool_fit), self._stream()),
                  "brkga_ga_breed_families")
        cand = self.pool_rows - nf
        if P > nf:
            self.surrogate.predict(self.pool[nf:], out=self.pred[:cand])
            if self.screen_mode == "family":  # the best-predicted child of every parent pair
                abi.check(self.lib.brkga_ga_select_families(self._ptr(self.pred), P - nf, family,
                                                            self._ptr(self.order_pool), self._stream()),
                          "brkga_ga_select_families")
                order = self.order_pool
            else:  # the best-predicted rows of the whole pool
                self._rank(self.pred, cand, self.order_pool)
                order = self.order_pool
                if self.n_explore:
                    self.torch.index_select(self.order_pool, 0, self.sel_idx, out=self.order_sel)
                    order = self.order_sel
            abi.check(self.lib.brkga_ga_gather(self._ptr(self.pool[nf:]), self._ptr(order), P - nf, K,
                                               self._ptr(self.pop[nxt][nf:]), self._stream()), "brkga_ga_gather")
            self.torch.index_select(self.pred[:cand], 0, order[:P - nf], out=self.pred_sel[:P - nf])
        self.pop[nxt][:nf].copy_(self.pool[:nf])
        self.fitness_buf[nxt][:ne].copy_(self.pool_fit[:ne])
        self._train_fork()
        if rows > 0:
            self.decoder.decode(self.pop[nxt][ne:], out=self.fitness_buf[nxt][ne:])
        self._train_join()
        self._monitor_and_learn(nxt, screened=P > nf)
        self._track(nxt)

    def _initial(self):
        P, K = self.num_individuals, self.num_gene
        skip = 1 if self.initialSol is not None else 0
        abi.check(self.lib.brkga_ga_init_population(self._ptr(self.pop[0]), P, K, ctypes.c_uint64(self.seed), skip,
                                                    self._stream()), "brkga_ga_init_population")
        if skip:
            self.pop[0][0].copy_(self.torch.from_numpy(self.initialSol))
        self.decoder.decode(self.pop[0], out=self.fitness_buf[0])
        if self.screening:
            self.surrogate.observe(self.pop[0], self.fitness_buf[0])
            self.surrogate.train(self.train_steps, self.train_batch, self.lr)
        self._track(0)

    def _step_fn(self, mode):
        return {"plain": self._step, "learn": self._step_learn, "screen": self._step_screened}[mode]

    def _modes(self):
        return ("learn", "screen") if self.screening else ("plain",)

    def prepare(self):
        """Run each kind of generation once eagerly (loads the kernels), capture
        one CUDA graph per kind and buffer parity, then reset the surrogate:
        afterwards ``fit`` only replays graphs."""
        torch = self.torch
        with torch.cuda.device(self.device):
            self.generation.zero_()
            self._initial()
            for mode in self._modes():
                self._step_fn(mode)(0)
                self._step_fn(mode)(1)
            torch.cuda.synchronize()
            side = torch.cuda.Stream(self.device)
            for mode in self._modes():
                for cur in (0, 1):
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g, stream=side):  # records the launches without running them
                        self._step_fn(mode)(cur)
                    self._graphs[(mode, cur)] = g
            torch.cuda.synchronize()
            if self.screening:
                self.surrogate.reset()
        self._prepared = True

    # ---- public ---------------------------------------------------------------------
    def fit(self, verbose: bool = False):
        """Run ``num_generations`` generations (BRKGA_alg3.py:210-281)."""
        torch = self.torch
        if self.use_graph and not self._prepared:
            self.prepare()
        with torch.cuda.device(self.device):
            self.generation.zero_()
            self.best_fit.fill_(float("inf"))
            if self.screening:
                self.stats_dev.fill_(float("nan"))
            torch.cuda.synchronize()
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
            base_mode = "learn" if self.screening else "plain"
            screening_on = False
            modes = []
            done = 0
            for g in range(1, G + 1):
                mode = "screen" if screening_on else base_mode
                if self.use_graph:
                    self._graphs[(mode, cur)].replay()
                else:
                    self._step_fn(mode)(cur)
                modes.append(mode)
                cur = 1 - cur
                e = torch.cuda.Event(enable_timing=True)
                e.record()
                events.append(e)
                done = g
                if (self.screening or self.target is not None) and g % (self.check_every if self.screening else 5) == 0:
                    if self.screening:
                        st = self.stats_dev[max(1, g - self.check_every + 1):g + 1, 0].cpu().numpy()
                        rho = float(np.nanmean(st)) if np.isfinite(st).any() else float("nan")
                        screening_on = g >= self.warmup_generations and rho >= self.spearman_threshold
                    if self.target is not None and float(self.best_fit.item()) <= self.target:
                        break
            G = done
            torch.cuda.synchronize()
            wall = time.perf_counter() - start
            if int(self.decoder.status.item()) != 0:
                raise RuntimeError(f"decoder status {int(self.decoder.status.item())} during the GA run")
            hist = self.history_dev.cpu().numpy()
            self.history = {"min": [float(v) for v in hist[:G + 1, 0]],
                            "mean": [float(v) for v in hist[:G + 1, 1]],
                            "time": [ev0.elapsed_time(e) / 1000.0 for e in events],
                            "mode": ["initial"] + modes}
            if self.screening:
                st = self.stats_dev.cpu().numpy()
                self.history["spearman"] = [float(v) for v in st[:G + 1, 0]]
                self.history["mae"] = [float(v) for v in st[:G + 1, 1]]
            self.best_fitness = float(self.best_fit.item())
            self.solution = self.best_sol.cpu().numpy()
            self.used_bins = int(np.floor(self.best_fitness))
            self.population = self.pop[cur].cpu().numpy()
            if self.n_audit:
                self.audit = (self.audit_pop[:G + 1].cpu().numpy(), self.audit_fit[:G + 1].cpu().numpy())
            self.fitness = self.fitness_buf[cur].cpu().numpy()
            self.wall_time = wall
            if verbose:
                for g in range(G + 1):
                    print(f"Generation {g}: Best={self.history['min'][g]:.4f} Mean={self.history['mean'][g]:.4f} "
                          f"Time={self.history['time'][g]:.3f}s")
        return "feasible"
