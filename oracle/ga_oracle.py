"""CPU oracle of the device GA step — test infrastructure only.

Restates ``brkga_fft2_b200/csrc/brkga_ga.cu`` in NumPy (the operators follow
the reference's ``BRKGA_alg3.py:178-265``; the random stream is
Philox4x32-10 of Salmon et al., SC'11, restated here from the paper) so that
tests can check populations, fitness and history bit for bit.  Fitness comes
from the C decoder oracle.
"""
from __future__ import annotations

import numpy as np

from .oracle import oracle_decode

MASK = np.uint64(0xFFFFFFFF)
TAG_INIT, TAG_MUTANT, TAG_MASK, TAG_PARENTS = 0, 1, 2, 3


def philox(c0, c1, c2, c3, seed: int):
    """Philox4x32-10 on arrays of 32-bit counters; returns four uint64 arrays of 32-bit outputs."""
    c0, c1, c2, c3 = (np.asarray(v, dtype=np.uint64) & MASK for v in (c0, c1, c2, c3))
    c0, c1, c2, c3 = np.broadcast_arrays(c0, c1, c2, c3)
    k0 = np.uint64(seed & 0xFFFFFFFF)
    k1 = np.uint64((seed >> 32) & 0xFFFFFFFF)
    for r in range(10):
        if r:
            k0 = (k0 + np.uint64(0x9E3779B9)) & MASK
            k1 = (k1 + np.uint64(0xBB67AE85)) & MASK
        p0 = np.uint64(0xD2511F53) * c0
        p1 = np.uint64(0xCD9E8D57) * c2
        c0, c1, c2, c3 = ((p1 >> np.uint64(32)) ^ c1 ^ k0, p1 & MASK, (p0 >> np.uint64(32)) ^ c3 ^ k1, p0 & MASK)
    return c0, c1, c2, c3


def unit_float(v):
    return (np.asarray(v) >> np.uint64(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)


def mulhi(a, n):
    return ((np.asarray(a, dtype=np.uint64) * np.uint64(n)) >> np.uint64(32)).astype(np.int64)


def keys_block(rows, K, gen, tag, seed):
    """[len(rows), K] uniform floats from the (block, row, gen, tag) counters."""
    rows = np.asarray(rows, dtype=np.uint64)
    nb = (K + 3) // 4
    b = np.arange(nb, dtype=np.uint64)
    out = philox(b[None, :], rows[:, None], np.uint64(gen), np.uint64(tag), seed)
    vals = np.stack([unit_float(o) for o in out], axis=-1).reshape(len(rows), nb * 4)
    return vals[:, :K]


def init_population(P, K, seed, skip_rows=0):
    pop = keys_block(np.arange(P), K, 0, TAG_INIT, seed)
    pop[:skip_rows] = 0.0
    return pop


def rank(fit):
    return np.argsort(np.asarray(fit, dtype=np.float64), kind="stable").astype(np.int32)


def breed(pop, fit, order, ne, nm, rho, seed, gen, out_rows=None, family=1):
    """Next population (or candidate pool of ``out_rows`` rows): elites,
    mutants, then offspring in families of ``family`` rows sharing the parent
    pair that the plain breed draws for row ne + nm + family index."""
    P, K = pop.shape
    R = P if out_rows is None else out_rows
    nxt = np.empty((R, K), pop.dtype)
    nfit = np.zeros(R, np.float64)
    nxt[:ne] = pop[order[:ne]]
    nfit[:ne] = fit[order[:ne]]
    if nm:
        nxt[ne:ne + nm] = keys_block(np.arange(ne, ne + nm), K, gen, TAG_MUTANT, seed)
    rows = np.arange(ne + nm, R)
    if rows.size:
        pr = philox(0, ne + nm + (rows - ne - nm) // family, gen, TAG_PARENTS, seed)
        e = order[mulhi(pr[0], ne)]
        o = order[ne + mulhi(pr[1], P - ne)]
        u = keys_block(rows, K, gen, TAG_MASK, seed)
        nxt[ne + nm:] = np.where(u < np.float32(rho), pop[e], pop[o])
    return nxt, nfit


def track_stats(fit, threads=1024):
    """(min, argmin, mean) with the device reduction order: per-thread strided
    sums, then a halving tree over the 1024 partial sums."""
    fit = np.asarray(fit, dtype=np.float64)
    P = fit.size
    part = np.zeros(threads, np.float64)
    for t in range(threads):
        acc = 0.0
        for i in range(t, P, threads):
            acc += float(fit[i])
        part[t] = acc
    h = threads // 2
    while h:
        for t in range(h):
            part[t] = part[t] + part[t + h]
        h //= 2
    return float(fit.min()), int(np.argmin(fit)), part[0] / P


def run(packed, P, ne, nm, rho, seed, generations, initial=None, n_threads=4):
    """The device GA's sequence of populations on the CPU; returns
    (final population, final fitness, history [G+1, 2], best fitness, best row)."""
    K = 2 * packed.n_genes
    pop = init_population(P, K, seed, 1 if initial is not None else 0)
    if initial is not None:
        pop[0] = np.asarray(initial, np.float32)
    fit = oracle_decode(packed, pop, n_threads=n_threads)
    hist = []
    best, best_sol = np.inf, None
    mn, arg, mean = track_stats(fit)
    hist.append((mn, mean))
    if mn < best:
        best, best_sol = mn, pop[arg].copy()
    for g in range(1, generations + 1):
        order = rank(fit)
        pop, nfit = breed(pop, fit, order, ne, nm, rho, seed, g)
        nfit[ne:] = oracle_decode(packed, pop[ne:], n_threads=n_threads)
        fit = nfit
        mn, arg, mean = track_stats(fit)
        hist.append((mn, mean))
        if mn < best:
            best, best_sol = mn, pop[arg].copy()
    return pop, fit, np.array(hist), best, best_sol
