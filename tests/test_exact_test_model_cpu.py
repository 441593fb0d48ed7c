"""A CPU model of one round of the decode kernel's exact collision test
(search_plate in brkga_fft2_b200/csrc/brkga_decoder.cu), checked against the
direct per-pair result on random rounds.

A round holds up to 32 (candidate, 32-column word) pairs in key order.  Each
pair's open columns F start full and every run of the mask clears the columns
it would overlap; the round's answer is the first pair whose F stays non-empty
(its lowest set bit is the leftmost free x).  The kernel gets there in two
phases: a solo phase in which lane i walks at most `solo` runs of pair i, two
runs per step, and a shared phase in which the pairs still open with runs
left are finished one at a time in task order — only those before the first
pair the solo phase already proved free — each lane taking every 32nd
remaining run, the lanes' results ANDed.  The model follows those steps and
must give the same pair and the same open columns as walking every pair's
runs directly, for any run count, density and solo length."""
import numpy as np
import pytest

LANES = 32


def direct(pairs):
    for i, (f0, blocks) in enumerate(pairs):
        f = f0
        for b in blocks:
            f &= ~b
        if f:
            return i, f
    return None


def two_phase(pairs, solo):
    F = [0] * LANES
    q = [0] * LANES
    n = [0] * LANES
    for lane, (f0, blocks) in enumerate(pairs):  # solo phase, two runs per step
        n[lane] = len(blocks)
        qend = min(n[lane], solo)
        f, qq = f0, 0
        while qq < qend and f:
            f &= ~blocks[qq]
            if qq + 1 < qend:
                f &= ~blocks[qq + 1]
            qq += 2
        F[lane], q[lane] = f, min(qq, qend)
    open_mask = sum(1 << i for i in range(LANES) if F[i] and q[i] < n[i])
    done_free = sum(1 << i for i in range(LANES) if F[i] and q[i] >= n[i])
    rem = open_mask & (((done_free & -done_free) - 1) if done_free else (1 << LANES) - 1)
    win = (done_free & -done_free).bit_length() - 1 if done_free else -1
    fw = F[win] if win >= 0 else 0
    while rem:  # shared phase, in task order
        l = (rem & -rem).bit_length() - 1
        rem &= rem - 1
        parts = []
        for lane in range(LANES):
            f, qq = F[l], q[l] + lane
            while qq < n[l] and f:
                f &= ~pairs[l][1][qq]
                qq += LANES
            parts.append(f)
        fp = (1 << 32) - 1
        for p in parts:  # the kernel's five shfl_xor steps
            fp &= p
        if fp:
            win, fw = l, fp
            break
    return (win, fw) if win >= 0 else None


@pytest.mark.parametrize("solo", [2, 8, 13, 20])
def test_two_phase_round_equals_direct_walk(solo):
    rng = np.random.default_rng(solo)
    for _ in range(1500):
        npairs = int(rng.integers(1, LANES + 1))
        dens = float(rng.choice([0.02, 0.08, 0.25, 0.6]))
        pairs = []
        for _ in range(npairs):
            nruns = int(rng.integers(1, 130))
            f0 = int(rng.integers(1, 1 << 32))
            bits = rng.random((nruns, 32)) < dens
            blocks = [int(np.packbits(row[::-1]).view(">u4")[0]) for row in bits]
            pairs.append((f0, blocks))
        assert two_phase(pairs, solo) == direct(pairs)
