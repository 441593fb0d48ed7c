"""Device GA step vs the NumPy oracle of the same operators: bit-exact
populations, fitness, history and best solution; CUDA-graph replay equals
eager execution."""
import ctypes
import os

import numpy as np
import pytest

from brkga_fft2_b200 import abi, instances, pack_problem
from oracle import ga_oracle as go

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required")
    from brkga_fft2_b200 import build
    build.build()
    return torch


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def test_kernels_match_oracle(torch):
    lib = abi.load_library()
    P, K, ne, nm, seed = 300, 42, 30, 45, 0x1234_5678_9ABC
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    pop = torch.zeros(P, K, dtype=torch.float32, device="cuda")
    assert lib.brkga_ga_init_population(_p(pop), P, K, ctypes.c_uint64(seed), 0, s) == 0
    np.testing.assert_array_equal(pop.cpu().numpy(), go.init_population(P, K, seed))
    rng = np.random.default_rng(1)
    fit_h = np.round(rng.random(P) * 50)            # many ties
    fit_h[7] = np.nan
    fit = torch.from_numpy(fit_h).cuda()
    order = torch.zeros(P, dtype=torch.int32, device="cuda")
    assert lib.brkga_ga_rank(_p(fit), P, _p(order), s) == 0
    np.testing.assert_array_equal(order.cpu().numpy(), go.rank(fit_h))
    gen = torch.full((1,), 17, dtype=torch.int64, device="cuda")
    nxt = torch.zeros_like(pop)
    nfit = torch.zeros_like(fit)
    assert lib.brkga_ga_breed(_p(pop), _p(fit), _p(order), P, K, ne, nm, ctypes.c_float(0.7), ctypes.c_uint64(seed),
                              _p(gen), _p(nxt), _p(nfit), s) == 0
    ref, rfit = go.breed(go.init_population(P, K, seed), fit_h, go.rank(fit_h), ne, nm, 0.7, seed, 17)
    np.testing.assert_array_equal(nxt.cpu().numpy(), ref)
    np.testing.assert_array_equal(nfit.cpu().numpy()[:ne], rfit[:ne])


def test_family_breed_and_selection_match_oracle(torch):
    """Offspring in families of 4 siblings per parent pair (the plain breed's
    pair for that slot), then the best-predicted child of each family."""
    lib = abi.load_library()
    P, K, ne, nm, k, seed = 300, 42, 30, 45, 4, 0x2468
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    pop_h = go.init_population(P, K, seed)
    fit_h = np.round(np.random.default_rng(2).random(P) * 50)
    pop, fit = torch.from_numpy(pop_h).cuda(), torch.from_numpy(fit_h).cuda()
    order = torch.from_numpy(go.rank(fit_h).astype(np.int32)).cuda()
    gen = torch.full((1,), 5, dtype=torch.int64, device="cuda")
    R = ne + nm + (P - ne - nm) * k
    pool = torch.zeros(R, K, dtype=torch.float32, device="cuda")
    pfit = torch.zeros(R, dtype=torch.float64, device="cuda")
    assert lib.brkga_ga_breed_families(_p(pop), _p(fit), _p(order), P, R, K, ne, nm, k, ctypes.c_float(0.7),
                                       ctypes.c_uint64(seed), _p(gen), _p(pool), _p(pfit), s) == 0
    ref, _ = go.breed(pop_h, fit_h, go.rank(fit_h), ne, nm, 0.7, seed, 5, out_rows=R, family=k)
    np.testing.assert_array_equal(pool.cpu().numpy(), ref)
    # family = 1 is the plain breed
    plain, _ = go.breed(pop_h, fit_h, go.rank(fit_h), ne, nm, 0.7, seed, 5)
    one = torch.zeros(P, K, dtype=torch.float32, device="cuda")
    assert lib.brkga_ga_breed_families(_p(pop), _p(fit), _p(order), P, P, K, ne, nm, 1, ctypes.c_float(0.7),
                                       ctypes.c_uint64(seed), _p(gen), _p(one), _p(pfit[:P]), s) == 0
    np.testing.assert_array_equal(one.cpu().numpy(), plain)
    nf = P - ne - nm
    pred_h = np.round(np.random.default_rng(3).random(nf * k) * 9)  # ties inside families
    pred_h[5] = np.nan
    pred_h[8:12] = np.nan
    idx = torch.full((nf,), -1, dtype=torch.int32, device="cuda")
    assert lib.brkga_ga_select_families(_p(torch.from_numpy(pred_h).cuda()), nf, k, _p(idx), s) == 0
    want = []
    for f in range(nf):
        blk = pred_h[f * k:(f + 1) * k]
        best = 0
        for j in range(1, k):
            if blk[j] < blk[best] or (np.isnan(blk[best]) and not np.isnan(blk[j])):
                best = j
        want.append(f * k + best)
    np.testing.assert_array_equal(idx.cpu().numpy(), want)


@pytest.mark.parametrize("P", [8192, 8193, 20000, 65536])
def test_rank_large_populations(torch, P):
    """Above 8192 rows the rank counts instead of sorting; same order (ties by index, NaN last)."""
    lib = abi.load_library()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(P)
    fit_h = np.round(rng.random(P) * 300)  # many ties
    fit_h[rng.choice(P, 5, replace=False)] = np.nan
    fit_h[rng.choice(P, 5, replace=False)] = -0.0
    fit = torch.from_numpy(fit_h).cuda()
    order = torch.full((P,), -1, dtype=torch.int32, device="cuda")
    assert lib.brkga_ga_rank(_p(fit), P, _p(order), s) == 0
    np.testing.assert_array_equal(order.cpu().numpy(), go.rank(fit_h))


def test_rank_refuses_beyond_limit(torch):
    lib = abi.load_library()
    fit = torch.zeros(65537, dtype=torch.float64, device="cuda")
    order = torch.zeros(65537, dtype=torch.int32, device="cuda")
    assert lib.brkga_ga_rank(_p(fit), 65537, _p(order), None) == abi.ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("use_graph", [False, True])
def test_ga_run_matches_oracle(torch, use_graph):
    from brkga_fft2_b200.ga import DeviceBRKGA
    inst = instances.small(5, n_parts=14, plates=((64, 64), (56, 72)), bbox_max=28)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    P, ne, nm, G, seed = 64, 8, 10, 6, 99
    ga = DeviceBRKGA(None, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts,
                     num_generations=G, num_individuals=P, num_elites=ne, num_mutants=nm, eliteCProb=0.7,
                     seed=seed, use_graph=use_graph, packed=pk)
    assert ga.fit() == "feasible"
    pop, fit, hist, best, sol = go.run(pk, P, ne, nm, 0.7, seed, G)
    np.testing.assert_array_equal(np.array([ga.history["min"], ga.history["mean"]]).T, hist)
    np.testing.assert_array_equal(ga.population, pop)
    np.testing.assert_array_equal(ga.fitness, fit)
    assert ga.best_fitness == best
    np.testing.assert_array_equal(ga.solution, sol)
    assert len(ga.history["time"]) == G + 1 and all(np.diff(ga.history["time"]) >= 0)


def test_ga_initial_solution_kept(torch):
    from brkga_fft2_b200.ga import DeviceBRKGA
    inst = instances.small(6, n_parts=12)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    init = instances.chromosomes(1, 12, 3)[0]
    ga = DeviceBRKGA(None, 12, inst.nb_machines, inst.thresholds, inst.instance_parts, initialSol=init,
                     num_generations=3, num_individuals=30, num_elites=4, num_mutants=5, packed=pk, seed=1)
    ga.fit()
    pop, fit, hist, best, sol = go.run(pk, 30, 4, 5, 0.7, 1, 3, initial=init)
    np.testing.assert_array_equal(np.array(ga.history["min"]), hist[:, 0])
    assert ga.best_fitness == best


@pytest.mark.parametrize("mode,explore,screen_mutants", [("family", 0.0, False), ("pool", 0.0, False),
                                                         ("pool", 0.3, False), ("pool", 0.0, True)])
def test_screened_ga_reports_exact_makespans(torch, mode, explore, screen_mutants):
    """With surrogate screening (mutants unscreened or screened with the
    offspring, and an exploration share of the decoded rows taken from the
    lower-ranked pool) every reported makespan still comes from the exact
    decoder; Spearman and MAE are logged for every generation."""
    from brkga_fft2_b200.ga import DeviceBRKGA
    from oracle import oracle_decode
    inst = instances.p50m2(0)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    ga = DeviceBRKGA(None, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts,
                     num_generations=20, num_individuals=200, num_elites=20, num_mutants=30, packed=pk, seed=3,
                     screening=True, oversample=4, warmup_generations=4, check_every=2, spearman_threshold=-1.0,
                     explore=explore, screen_mutants=screen_mutants, screen_mode=mode)
    ga.fit()
    np.testing.assert_array_equal(ga.fitness, oracle_decode(pk, ga.population, n_threads=8))
    assert ga.best_fitness == min(ga.history["min"])
    assert oracle_decode(pk, ga.solution[None])[0] == ga.best_fitness
    assert "screen" in ga.history["mode"]
    assert np.isfinite(ga.history["spearman"][1:]).all() and np.isfinite(ga.history["mae"][1:]).all()
    assert (np.diff(ga.history["min"]) <= 0).all()


@pytest.mark.parametrize("maker,P,G,frac", [(instances.p50m2, 200, 12, 0.02), (instances.p400m8, 48, 2, 0.01),
                                             (instances.p400m8, 4096, 3, 0.01)])
def test_audit_sample_of_every_generation_is_exact(torch, maker, P, G, frac):
    """The audit sample (1-2 % of the rows decoded in every generation, screening on)
    matches the oracle bit for bit, generation by generation — at the
    large-stress size too (P400M8, population 4096: 37 rows a generation)."""
    from brkga_fft2_b200.ga import DeviceBRKGA
    from oracle import oracle_decode
    inst = maker(0)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    ne = max(1, P // 10)
    ga = DeviceBRKGA(None, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts,
                     num_generations=G, num_individuals=P, num_elites=ne, num_mutants=P // 6, packed=pk, seed=5,
                     screening=True, oversample=3, warmup_generations=1, check_every=1, spearman_threshold=-1.0,
                     audit_fraction=frac)
    ga.fit()
    chrom, fit = ga.audit
    assert chrom.shape[:2] == (G + 1, ga.n_audit) and ga.n_audit >= 1
    ref = oracle_decode(pk, chrom.reshape(-1, chrom.shape[-1]), n_threads=min(16, os.cpu_count() or 1)
                        ).reshape(fit.shape)
    np.testing.assert_array_equal(fit, ref)
    assert "screen" in ga.history["mode"]
