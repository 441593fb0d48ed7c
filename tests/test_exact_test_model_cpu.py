"""CPU models of the decode kernel's exact collision test (search_plate in
brkga_fft2_b200/csrc/brkga_decoder.cu): one round of the two-phase test,
checked against the direct per-pair result on random rounds, and the key
order of the dealt pairs on which the kernel's early stops rely.

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


def key_of(newlen, y, x, r):
    """The kernel's selection key (smaller is better): newLen, then larger y, smaller x, lower rotation."""
    return (newlen << 28) | ((8191 - y) << 15) | (x << 2) | r


def test_pairs_come_in_key_order():
    """The decode kernel stops a chunk's rounds, and the shared phase's pairs,
    as soon as the next pair cannot beat the best key found.  That is exact
    because pairs are dealt in key order: for survivors from the bottom up and
    words from the left, every key a pair can produce is at least its own
    bound, and the bounds never decrease along the dealing order."""
    rng = np.random.default_rng(7)
    for _ in range(3000):
        L = int(rng.integers(2, 600))
        h = int(rng.integers(1, L + 1))
        W = int(rng.integers(1, 600))
        w = int(rng.integers(1, W + 1))
        enc = int(rng.integers(0, L + 1))
        r = int(rng.integers(0, 4))
        level = int(rng.integers(0, max(1, (L - h) // 32 + 1)))
        ty_hi = L - h - 32 * level
        if ty_hi < 0:
            continue
        lanes = sorted(set(int(v) for v in rng.integers(0, min(32, ty_hi + 1), size=int(rng.integers(1, 33)))))
        nwo = (W - w + 1 + 31) // 32
        bounds, worst = [], []
        for sl in lanes:  # survivors in lane order = bottom-most candidate first
            ty = ty_hi - sl
            for k in range(nwo):
                nl = max(enc, L - ty)
                bounds.append(key_of(nl, ty + h - 1, 32 * k, r))
                worst.append(key_of(nl, ty + h - 1, min(32 * k + 31, W - w), r))
        assert all(b1 <= b2 for b1, b2 in zip(bounds, bounds[1:]))
        assert all(hi <= b for hi, b in zip(worst, bounds[1:]))  # a pair's worst key is below the next bound
