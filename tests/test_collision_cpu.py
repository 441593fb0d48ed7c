"""Host side of the collision-path comparison (brkga_fft2_b200.collision), on
the CPU: plates packed in the decoder's format, and chunk cases replayed from
placement logs (here the oracle's) with each plate exactly as it was before
the part was placed."""
import numpy as np

from brkga_fft2_b200 import collision, instances, pack_problem
from oracle import oracle_decode


def test_pack_plate_bit_layout():
    rng = np.random.default_rng(3)
    for L, W in ((5, 31), (4, 32), (3, 33), (2, 600)):
        g = (rng.random((L, W)) < 0.4).astype(np.uint8)
        p = collision.pack_plate(g)
        rs = (W + 31) // 32 + 2
        assert p.shape == (L, rs) and p.dtype == np.dtype("<u4")
        for y in range(L):
            for x in range(W):
                assert ((int(p[y, x >> 5]) >> (x & 31)) & 1) == g[y, x]
        assert all(int(p[y, k]) == 0 for y in range(L) for k in range((W + 31) // 32, rs))
        tail = W & 31
        if tail:
            assert all((int(p[y, W >> 5]) >> tail) == 0 for y in range(L))


def test_chunk_cases_replay_the_plates_before_each_placement():
    inst = instances.p200m6(0)
    packed = pack_problem(inst.problem_data, inst.nb_parts, inst.nb_machines, inst.thresholds, inst.instance_parts)
    ch = instances.chromosomes(2, inst.nb_parts, 5)
    _, log = oracle_decode(packed, ch, n_threads=2, with_log=True)
    cases = collision.chunk_cases(packed, log, min_side=1, levels=(0,))
    assert cases
    a = packed.arrays
    # the plate of every case holds exactly the parts placed on it before: the
    # part's own placement was free on it, and a case with that plate exists
    seen = 0
    for row in log:
        for m in range(packed.n_machines):
            recs = [r for r in row[m] if r["gene"] >= 0]
            for k, rec in enumerate(recs):
                prev = [r for r in recs[:k] if r["bin"] == rec["bin"]]
                if not prev:
                    continue
                t = int(a["gene_type"][rec["gene"]])
                mask = collision._rotation(packed, t, int(rec["rot"]))
                h, w = mask.shape
                L, W = int(a["bin_length"][m]), int(a["bin_width"][m])
                grid = np.zeros((L, W), np.uint8)
                for r in prev:
                    mk = collision._rotation(packed, int(a["gene_type"][r["gene"]]), int(r["rot"]))
                    grid[r["y"] - mk.shape[0] + 1: r["y"] + 1, r["x"]: r["x"] + mk.shape[1]] |= mk
                y, x = int(rec["y"]), int(rec["x"])
                assert not (grid[y - h + 1: y + 1, x: x + w] & mask).any()
                match = [c for c in cases if c["machine"] == m and c["type"] == t and np.array_equal(c["grid"], grid)]
                assert match
                seen += 1
    assert seen > 0
    assert all(c["ty_hi"] == int(a["bin_length"][c["machine"]]) - c["h"] for c in cases)


def test_buckets_and_sorting():
    assert collision.bucket_of(63) == -1 and collision.bucket_of(64) == 0 and collision.bucket_of(256) == 4
    assert collision.bucket_of(257) == -1
    cases = [{"h": s, "w": 10} for s in (200, 70, 100, 70, 300, 130)]
    out, spans = collision.sort_by_bucket(cases)
    assert [c["h"] for c in out] == [70, 70, 100, 130, 200]
    assert spans == {0: (0, 2), 1: (2, 1), 2: (3, 1), 4: (4, 1)}
