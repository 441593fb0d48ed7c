"""GA oracle checks on the CPU: Philox4x32-10 known answers and the
operators of BRKGA_alg3.py:178-265 as restated for the device GA."""
import numpy as np
import pytest

from brkga_fft2_b200 import instances, pack_problem
from oracle import ga_oracle as go


def test_philox_known_answers():
    """Known-answer vectors of Philox4x32-10 (Random123 distribution, kat_vectors)."""
    kat = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
           ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for c, k, want in kat:
        got = tuple(int(v) for v in go.philox(*c, seed=k[0] | (k[1] << 32)))
        assert got == want


def test_breed_structure():
    rng = np.random.default_rng(0)
    P, K, ne, nm = 40, 18, 6, 8
    pop = rng.random((P, K)).astype(np.float32)
    fit = rng.random(P) * 100
    order = go.rank(fit)
    assert (np.diff(fit[order]) >= 0).all()
    nxt, nfit = go.breed(pop, fit, order, ne, nm, 0.7, seed=5, gen=3)
    np.testing.assert_array_equal(nxt[:ne], pop[order[:ne]])       # elites, best first
    np.testing.assert_array_equal(nfit[:ne], fit[order[:ne]])
    assert ((nxt[ne:ne + nm] >= 0) & (nxt[ne:ne + nm] < 1)).all()    # mutants
    elites, others = set(order[:ne]), set(order[ne:])
    frac = []
    for r in range(ne + nm, P):                                    # each offspring key from its two parents
        child = nxt[r]
        from_e = [e for e in elites if np.isin(child, pop[e]).sum() > 0]
        assert from_e
        frac.append(np.mean([np.any(pop[list(elites)][:, g] == child[g]) for g in range(K)]))
    assert 0.5 < np.mean(frac) <= 1.0


def test_small_run_history():
    inst = instances.small(2, n_parts=10)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    pop, fit, hist, best, sol = go.run(pk, P=24, ne=4, nm=5, rho=0.7, seed=3, generations=4)
    assert hist.shape == (5, 2)
    assert (np.diff(hist[:, 0]) <= 0).all()       # elites survive: the minimum never increases
    assert best == hist[-1, 0] == fit.min()
    from oracle import oracle_decode
    assert oracle_decode(pk, sol[None])[0] == best


@pytest.mark.parametrize("kwargs", [dict(num_elites=0), dict(num_elites=5, num_mutants=96), dict(num_individuals=70000),
                                    dict(num_generations=-1), dict(eliteCProb=1.5), dict(audit_fraction=2.0),
                                    dict(screening=True, oversample=0), dict(screening=True, explore=-0.1),
                                    dict(screening=True, explore=1.5), dict(screening=True, train_batch=0),
                                    dict(screening=True, screen_mode="rows"),
                                    dict(screening=True, explore=0.3), dict(screening=True, screen_mutants=True)])
def test_device_ga_refuses_bad_arguments_before_any_gpu_work(kwargs):
    """Argument errors surface as ValueError on the host, before a decoder or
    any device buffer exists (an oversample below 1 would otherwise gather
    more rows than the pool holds)."""
    from brkga_fft2_b200.ga import DeviceBRKGA
    args = dict(num_generations=2, num_individuals=100, num_elites=10, num_mutants=15)
    args.update(kwargs)
    with pytest.raises(ValueError):
        DeviceBRKGA(None, 10, 2, [0.5], np.arange(10), **args)


@pytest.mark.parametrize("kwargs", [dict(eliteCProb=-0.1), dict(num_generations=-2), dict(num_elites=0),
                                    dict(num_individuals=[10, 10]), dict(num_mutants=300)])
def test_multi_ga_refuses_bad_arguments_before_any_gpu_work(kwargs):
    from brkga_fft2_b200.multi_ga import MultiBRKGA
    inst = instances.small(1)
    pk = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    with pytest.raises(ValueError):
        MultiBRKGA([pk], **dict(dict(num_generations=2, num_individuals=100), **kwargs))


def test_breed_equals_the_reference_operators_on_the_same_draws():
    """One generation of the reference's own partition, mating and mutants
    (BRKGA_alg3.py:178-208, the new population of :246-250), run by
    tests/golden/make_golden.py with numpy's random draws replaced by this
    GA's Philox draws (the same parents, crossover uniforms and mutants):
    the oracle's breed gives the same population, row for row and key for key,
    and carries the same elite fitness.  Cases: 10/15 % elites/mutants, one
    elite and no mutants, and no offspring at all."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "ga_ops.npz"))
    for i, (P, N, ne, nm, rho, seed, gen) in enumerate(z["cases"].tolist()):
        P, ne, nm, seed, gen = int(P), int(ne), int(nm), int(seed), int(gen)
        pop, fit = z[f"pop_{i}"], z[f"fit_{i}"]
        nxt, nfit = go.breed(pop, fit, go.rank(fit), ne, nm, rho, seed, gen)
        assert nxt.dtype == np.float32 and nxt.shape == z[f"next_{i}"].shape
        np.testing.assert_array_equal(nxt, z[f"next_{i}"], err_msg=f"case {i}")
        np.testing.assert_array_equal(nfit[:ne], z[f"elite_fit_{i}"], err_msg=f"case {i}")
