"""Lockstep GA over several instances (MultiBRKGA) and the launch-shape
autotuner.  Instance k of a MultiBRKGA must evolve exactly as the GA oracle
with seed + k — populations, fitness, per-generation min/mean and best
solution bit for bit — although all instances share one decode launch per
generation.  The autotuner may only change speed, never a makespan."""
import numpy as np
import pytest

from brkga_fft2_b200 import instances, pack_problem
from oracle import ga_oracle as go
from oracle import oracle_decode

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required")
    from brkga_fft2_b200 import build
    build.build()
    return torch


def _packs(specs):
    out = []
    for seed, n, plates, bbox in specs:
        inst = instances.small(seed, n_parts=n, plates=plates, bbox_max=bbox)
        out.append(pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds,
                                inst.instance_parts))
    return out


SPECS = [(21, 14, ((64, 64), (56, 72)), 28), (22, 9, ((48, 48),), 20), (23, 18, ((70, 60), (64, 64), (80, 80)), 30)]


@pytest.mark.parametrize("use_graph", [False, True])
def test_multi_ga_matches_oracle_per_instance(torch, use_graph):
    from brkga_fft2_b200.multi_ga import MultiBRKGA
    packs = _packs(SPECS)
    P, ne, nm, G, seed = [48, 40, 64], [6, 5, 9], [8, 6, 10], 5, 1234
    ga = MultiBRKGA(packs, num_generations=G, num_individuals=P, num_elites=ne, num_mutants=nm, eliteCProb=0.7,
                    seed=seed, use_graph=use_graph).fit()
    for k, pk in enumerate(packs):
        pop, fit, hist, best, best_sol = go.run(pk, P[k], ne[k], nm[k], 0.7, seed + k, G, n_threads=4)
        np.testing.assert_array_equal(ga.populations[k], pop, err_msg=f"instance {k}")
        np.testing.assert_array_equal(ga.fitness[k], fit, err_msg=f"instance {k}")
        np.testing.assert_array_equal(np.array(ga.history[k]["min"]), hist[:, 0])
        np.testing.assert_array_equal(np.array(ga.history[k]["mean"]), hist[:, 1])
        assert ga.best_fitness[k] == best
        np.testing.assert_array_equal(ga.solutions[k], best_sol)
    assert len(ga.generation_ms) == G


def test_autotune_picks_a_shape_and_keeps_results(torch, tmp_path):
    from brkga_fft2_b200.autotune import autotune
    from brkga_fft2_b200.evaluator import MultiDecoder
    insts = [instances.uneven(s) for s in (40, 41, 42)]
    packs = [pack_problem(i.problem_data, i.nb_parts, i.nb_machines, i.thresholds, i.instance_parts) for i in insts]
    pops = [24, 16, 20]
    chroms = [instances.chromosomes(p, i.nb_parts, 300 + k) for k, (p, i) in enumerate(zip(pops, insts))]
    ref = np.concatenate([oracle_decode(pk, ch, n_threads=8) for pk, ch in zip(packs, chroms)])
    md = MultiDecoder(packs, max_pops=pops)
    flat = torch.from_numpy(np.concatenate([c.reshape(-1) for c in chroms])).cuda()
    cache = str(tmp_path / "tune.json")
    shapes = [(4, 2, 0), (4, 4, 1), (2, 16, 0), (0, 0, -1), (4, 32, 8)]  # the last cannot be resident
    res = autotune(md, flat, pops, shapes=shapes, task_max_values=(0, 256), cache_path=cache)
    assert not res["cached"] and len(res["table"]) == 6
    assert res["config"] in [(w, c, s, t if t >= 0 else 8192) for w, c, s, t, _ in res["table"]]
    w, c, s, _, t = md.launch_config()
    assert t == res["config"][3]
    if res["config"][0]:
        assert w == res["config"][0]
    if res["config"][1]:
        assert c == res["config"][1]
    np.testing.assert_array_equal(md.decode_concat(flat, pops).cpu().numpy(), ref)
    md.set_launch_config()
    again = autotune(md, flat, pops, shapes=shapes, cache_path=cache)
    assert again["cached"] and again["config"] == res["config"]
    assert md.launch_config()[4] == res["config"][3]
    np.testing.assert_array_equal(md.decode_concat(flat, pops).cpu().numpy(), ref)
