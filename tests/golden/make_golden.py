"""Generate the golden fixtures in tests/golden from the reference itself.

Run in a container where the reference checkout is available (read-only):

    python tests/golden/make_golden.py --reference /root/reference

It imports the reference's sequential decoder (placement.py / binClassNew.py /
numba_utils.py / collision_backend.py with the ``torch_cpu`` backend) and
records, per chromosome, the makespan and every placement (part id, plate,
column x, bottom row y, rotation).  Outputs:

* ``real_<inst>.npz`` / ``fp_<inst>.npz`` — reference instances rebuilt from ``data/`` (masks from
  ``data/partsMatrices``, part/machine specs and polygon areas parsed from the
  xlsx files as raw XML, never from the pickle), with the reference's own
  known answers:
    - P75M2-0: ``results/golden/P75M2-0`` (chromosome 688, makespan and the 75
      ordered placements);
    - P50M2-0: chromosome 462 of ``np.random.seed(42)`` uniform (500, 100)
      -> 448166.8336 (``verify_native_vs_pp.py:31-32``) and the final plate
      grids ``results/inspection_output/pp_bin_m*_b*.txt`` (bit-packed here);
    - the 8 instances of ``benchmarks/20260422_*.json``: the first five
      feasible makespans of rep 4 (population ``default_rng(127)``) and the
      feasible / infeasible counts of the whole population.
* ``syn_<name>.npz`` — seeded synthetic instances (brkga_fft2_b200.instances)
  with reference makespans and placement logs for a batch of chromosomes.
* ``refms_bench_P100M4_step0.npz`` / ``_step19.npz`` — the reference's
  makespans of all 500 rows of the populations bench.py times first and last
  (decoded over a process pool of all host cores; the rows are regenerated
  from their seed);
  ``refms_P200M6_s13.npz`` / ``refms_P400M8_s14.npz`` — the same for the rows
  the GPU tests compare with the oracle at the 200- and 400-part sizes;
  ``refms_uneven.npz`` — and for the rows of the uneven multi-instance test.
* ``ga_ops.npz`` — one generation of the reference's GA operators (partition,
  mating, mutants) on seeded populations, its random draws replaced by the
  device GA's Philox draws, so the GA oracle's breed can be compared with it.

Nothing under tests/ reads the reference at run time; only this script does.
"""
from __future__ import annotations

import argparse
import glob
import textwrap
import json
import os
import sys
import threading
import time
import xml.etree.ElementTree as ET
import zipfile

os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/brkga_numba_cache")
sys.dont_write_bytecode = True

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from brkga_fft2_b200 import instances as syn  # noqa: E402
from brkga_fft2_b200.instance_io import save_instance  # noqa: E402
from brkga_fft2_b200.problem import MachineData, MachinePartData, ProblemData, make_part_data  # noqa: E402

NS = {"m": "http://schemas.openxmlformats.org/spreadsheetml/2006/main"}
RID = "{http://schemas.openxmlformats.org/officeDocument/2006/relationships}id"


def read_xlsx(path):
    """Sheets of an xlsx file as lists of {column letter: value} rows (raw XML)."""
    z = zipfile.ZipFile(path)
    sst = []
    if "xl/sharedStrings.xml" in z.namelist():
        for si in ET.fromstring(z.read("xl/sharedStrings.xml")).findall("m:si", NS):
            sst.append("".join(t.text or "" for t in si.iter("{%s}t" % NS["m"])))
    wb = ET.fromstring(z.read("xl/workbook.xml"))
    rels = {r.get("Id"): r.get("Target") for r in ET.fromstring(z.read("xl/_rels/workbook.xml.rels"))}
    out = {}
    for s in wb.find("m:sheets", NS):
        root = ET.fromstring(z.read("xl/" + rels[s.get(RID)]))
        rows = []
        for r in root.find("m:sheetData", NS).findall("m:row", NS):
            d = {}
            for c in r.findall("m:c", NS):
                v = c.find("m:v", NS)
                if v is None:
                    continue
                col = "".join(ch for ch in c.get("r") if ch.isalpha())
                d[col] = sst[int(v.text)] if c.get("t") == "s" else float(v.text)
            rows.append(d)
        out[s.get("name")] = rows
    return out


class Reference:
    """The reference's CPU decoder, imported read-only, with a placement logger."""

    def __init__(self, root):
        self.root = root
        sys.path.insert(0, root)
        import torch
        torch.set_num_threads(1)
        import placement
        import binClassNew
        from collision_backend import create_collision_backend
        import data_structures
        self.placement = placement
        self.binClassNew = binClassNew
        self.ds = data_structures
        self.backend = create_collision_backend("torch_cpu")
        self._orig_insert = binClassNew.BuildingPlate.insert
        self._orig_machine = placement._process_single_machine
        self._tls = threading.local()
        ref = self

        def insert(plate, x, y, partMatrix, shapes, partArea, gpu_tensor=None):
            st = getattr(ref._tls, "state", None)
            if st is not None:
                pid, rot = st["rot_of"][id(partMatrix)]
                bins = st["bins"]
                if id(plate) not in bins:
                    bins[id(plate)] = len(bins)
                st["log"][st["machine"]].append((pid, bins[id(plate)], int(x), int(y), rot))
            return ref._orig_insert(plate, x, y, partMatrix, shapes, partArea, gpu_tensor=gpu_tensor)

        def machine(args):
            st = getattr(ref._tls, "state", None)
            if st is not None:
                st["machine"] = args[0]
                st["bins"] = {}
            return ref._orig_machine(args)

        binClassNew.BuildingPlate.insert = insert
        placement._process_single_machine = machine

    def problem(self, ours: ProblemData, nb_machines):
        """Reference ProblemData (with torch_cpu FFTs) from one of ours."""
        ds = self.ds
        parts = {}
        for pid, p in ours.parts.items():
            rd = ds.PartData(id=pid, area=p.area, nrot=p.nrot, rotations=[r.astype(np.int32) for r in p.rotations],
                             shapes=list(p.shapes), densities=list(p.densities), best_rotation=p.best_rotation,
                             rotations_gpu=None, rotations_uint8=[r.astype(np.uint8) for r in p.rotations])
            rd.prepare_jit_data()
            parts[pid] = rd
        machines = []
        for m in range(nb_machines):
            md = ours.machines[m]
            L, W = int(md.bin_length), int(md.bin_width)
            mp = {}
            for pid in ours.parts:
                ffts = [self.backend.prepare_part_fft(parts[pid].rotations[r], L, W) for r in range(parts[pid].nrot)]
                # numpy scalars, as BRKGA_alg3.py:411-417 gets them from pandas: CPython >= 3.12
                # sums exact Python floats with compensation but numpy float64 items naively,
                # which is what the reference's pipeline (and its C++ decoder) does.
                mp[pid] = ds.MachinePartData(ffts=ffts, proc_time=np.float64(md.parts[pid].proc_time),
                                             proc_time_height=np.float64(md.parts[pid].proc_time_height))
            st = md.setup_time
            st = np.int64(st) if float(st).is_integer() else np.float64(st)
            machines.append(ds.MachineData(bin_length=L, bin_width=W, bin_area=md.bin_area,
                                           setup_time=st, parts=mp))
        return ds.ProblemData(parts=parts, machines=machines, instance_parts=ours.instance_parts,
                              instance_parts_unique=ours.instance_parts_unique)

    def decode(self, rpd, nb_parts, nb_machines, thresholds, chrom, inst_parts, stable=False):
        rot_of = {}
        for pid, p in rpd.parts.items():
            for r, arr in enumerate(p.rotations_uint8):
                rot_of[id(arr)] = (int(pid), r)
        self._tls.state = {"rot_of": rot_of, "log": {m: [] for m in range(nb_machines)}, "machine": 0, "bins": {}}
        orig_argsort = np.argsort
        try:
            if stable:
                np.argsort = lambda a, *k, **kw: orig_argsort(a, kind="stable")
            ms = self.placement.placementProcedure(rpd, nb_parts, nb_machines, list(thresholds),
                                                   np.asarray(chrom, np.float32), np.asarray(inst_parts),
                                                   self.backend, parallel=False)
        finally:
            np.argsort = orig_argsort
            log = self._tls.state["log"]
            self._tls.state = None
        return float(ms), log


def reference_greedy(ref, root, rpd, nb_parts, nb_machines, thresholds, inst_parts, heights, areas, seed):
    """Run the reference's own greedy initial solution (the block of BRKGA_alg3.py
    from its "CREATE INITIAL SOLUTION" marker to its "CALL BRKGA" marker) on
    our instance; returns (chromosome, makespan, placements in order as
    (machine, plate, part, x, y, rot))."""
    import random
    import pandas
    import binClassInitialSol
    src = open(os.path.join(root, "BRKGA_alg3.py")).read()
    q3 = "'" * 3
    a = src.rindex("\n", 0, src.index(q3 + " CREATE INITIAL SOLUTION " + q3)) + 1
    b = src.rindex("\n", 0, src.index(q3 + " CALL BRKGA" + q3)) + 1
    block = textwrap.dedent(src[a:b])  # the block is indented under `if __name__ == "__main__":`
    ids = sorted(set(int(p) for p in inst_parts))

    class PandasWithAreas:  # the block reads polygon areas with pd.read_excel; serve the same numbers
        def __getattr__(self, name):
            return getattr(pandas, name)

        def read_excel(self, *a, **k):
            return pandas.DataFrame({"Area": [areas[i] for i in ids]}, index=pandas.Index(ids, name="part ID"))

    rot_of = {}
    for pid, p in rpd.parts.items():
        for r, arr in enumerate(p.rotations_uint8):
            rot_of[id(arr)] = (int(pid), r)
    rec = []
    orig = binClassInitialSol.BuildingPlate.insert

    def insert(plate, x, y, partMatrix, shapes, partArea, gpu_tensor=None):
        rec.append((plate, int(x), int(y)) + rot_of[id(partMatrix)])
        return orig(plate, x, y, partMatrix, shapes, partArea, gpu_tensor=gpu_tensor)

    binClassInitialSol.BuildingPlate.insert = insert
    jobSpec = pandas.DataFrame({"height(mm)": [heights[i] for i in ids]}, index=pandas.Index(ids))
    ns = {"np": np, "pd": PandasWithAreas(), "random": random, "problem_data": rpd, "nbMachines": nb_machines,
          "nbParts": nb_parts, "instanceParts": np.asarray(inst_parts), "jobSpec": jobSpec,
          "collision_backend": ref.backend, "BuildingPlate": binClassInitialSol.BuildingPlate,
          "thresholds": list(thresholds), "print": lambda *a, **k: None}
    random.seed(seed)
    try:
        exec(compile(block, "BRKGA_alg3.py:initial-solution", "exec"), ns)
    finally:
        binClassInitialSol.BuildingPlate.insert = orig
    plates = {}
    for m in range(nb_machines):
        for b, batch in enumerate(ns["machines_dict"][f"machine_{m}"]["batches"]):
            plates[id(batch)] = (m, b)
    out = np.array([plates[id(pl)] + (pid, x, y, r) for pl, x, y, pid, r in rec], np.int64)
    return np.asarray(ns["array"], np.float64), float(ns["best_makespan"]), out


def log_to_array(log, nb_machines, nb_parts):
    """Per machine ordered placements -> int64 [M, N, 5] (part, bin, x, y, rot), -1 padded."""
    out = -np.ones((nb_machines, nb_parts, 5), np.int64)
    for m in range(nb_machines):
        for k, rec in enumerate(log[m]):
            out[m, k] = rec
    return out


_POOL = {}


def _pool_init(root, maker="p100m4", inst_seed=0):
    """A process of the reference pool: the reference decoder and the problem of
    a synthetic workload (default: the benchmark's, P100M4 instance seed 0),
    numba compiled on one row."""
    inst = getattr(syn, maker)(inst_seed)
    ref = Reference(root)
    rpd = ref.problem(inst.problem_data, inst.nb_machines)
    _POOL.update(ref=ref, rpd=rpd, inst=inst)
    ref.decode(rpd, inst.nb_parts, inst.nb_machines, inst.thresholds,
               syn.chromosomes(1, inst.nb_parts, 7)[0], inst.instance_parts)


def _pool_decode(row):
    """The reference's makespan of one benchmark chromosome (in a pool process)."""
    p = _POOL
    inst = p["inst"]
    return p["ref"].decode(p["rpd"], inst.nb_parts, inst.nb_machines, inst.thresholds, row, inst.instance_parts)[0]


def bench_pool(root, workers, maker="p100m4", inst_seed=0):
    """A process pool decoding rows of a synthetic workload with the reference,
    the way its GA spreads a population over the host cores (eval_mode="process",
    BRKGA_alg3.py:149-154), every worker started with its own problem."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    return ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"), initializer=_pool_init,
                               initargs=(root, maker, inst_seed))


def reference_ga_step(root, pop, fit, ne, nm, rho, seed, gen):
    """One generation of the reference's GA operators (BRKGA_alg3.py:178-208 and
    the new population of :246-250: partition, mating, mutants) on (pop, fit),
    numpy's random draws replaced by the device GA's Philox draws for (seed,
    gen) — every offspring's elite and non-elite parent (mapped into the
    reference's elite and non-elite arrays), its crossover uniforms, and the
    mutants.  Returns the next population and the elites' carried fitness."""
    from types import SimpleNamespace
    sys.path.insert(0, root)
    import BRKGA_alg3
    sys.path.insert(0, REPO)
    from oracle import ga_oracle as go
    P, K = pop.shape
    ns = SimpleNamespace(num_elites=ne, num_individuals=P, num_mutants=nm, num_gene=K, eliteCProb=rho)
    order = go.rank(fit)
    non_elite_rows = np.argpartition(np.asarray(fit), ne)[ne:]  # the reference's non-elite order
    rows = np.arange(ne + nm, P)
    pr = go.philox(0, rows, gen, go.TAG_PARENTS, seed)
    e_idx = go.mulhi(pr[0], ne)
    o_rows = order[ne + go.mulhi(pr[1], P - ne)]
    pos = {int(r): j for j, r in enumerate(non_elite_rows)}
    o_idx = np.array([pos[int(r)] for r in o_rows], np.int64)
    ints = [e_idx, o_idx]
    unis = [go.keys_block(rows, K, gen, go.TAG_MASK, seed), go.keys_block(np.arange(ne, ne + nm), K, gen,
                                                                          go.TAG_MUTANT, seed)]

    def randint(low, high=None, size=None):
        v = ints.pop(0)
        assert low == 0 and v.shape == (size,) and (v < high).all()
        return v

    def uniform(low=0.0, high=1.0, size=None):
        v = unis.pop(0)
        assert low == 0.0 and high == 1.0 and v.shape == tuple(size)
        return v

    saved = np.random.randint, np.random.uniform
    np.random.randint, np.random.uniform = randint, uniform
    try:
        elites, non_elites, elite_fit = BRKGA_alg3.BRKGA.partition(ns, pop, fit)
        offspring = BRKGA_alg3.BRKGA.mating(ns, elites, non_elites)
        mutants = BRKGA_alg3.BRKGA.mutants(ns)
    finally:
        np.random.randint, np.random.uniform = saved
    assert not ints and not unis
    return np.concatenate((elites, mutants, offspring), axis=0), np.asarray(elite_fit, np.float64)


def real_heights(root):
    spec = read_xlsx(os.path.join(root, "data/PartsMachines/part-machine-information.xlsx"))
    return {int(r["A"]): r["D"] for r in spec["part"][1:]}


def real_problem(root, nb_parts, nb_machines, inst):
    spec = read_xlsx(os.path.join(root, "data/PartsMachines/part-machine-information.xlsx"))
    areas = read_xlsx(os.path.join(root, "data/PartsMachines/polygon_areas.xlsx"))
    part_rows = {int(r["A"]): r for r in spec["part"][1:]}
    mach_rows = spec["machine"][1:]
    area = {int(r["A"]): r["B"] for r in list(areas.values())[0][1:]}
    with open(os.path.join(root, f"data/Instances/P{nb_parts}M{nb_machines}-{inst}.txt")) as f:
        inst_parts = np.array([int(v) for v in f.read().split()], np.int64)
    uniq = np.unique(inst_parts)
    parts = {int(p): make_part_data(int(p), np.load(os.path.join(root, f"data/partsMatrices/matrix_{p}.npy")),
                                    area[int(p)]) for p in uniq}
    machines = []
    for m in range(nb_machines):
        mr = mach_rows[m]  # columns: B W(mm), C L(mm), E ST, F VT, G SPT, H HT (BRKGA_alg3.py:389-417)
        L, W = int(mr["C"]), int(mr["B"])
        mp = {int(p): MachinePartData(None,
                                      part_rows[int(p)]["E"] * mr["F"] + part_rows[int(p)]["F"] * mr["G"],
                                      part_rows[int(p)]["D"] * mr["H"]) for p in uniq}
        machines.append(MachineData(L, W, float(L * W), float(int(mr["E"])), mp))
    pd = ProblemData(parts, machines, inst_parts, uniq)
    return pd, inst_parts, [t / nb_machines for t in range(1, nb_machines)]


def read_plate(path):
    rows = [list(map(int, line.split())) for line in open(path) if line.strip()]
    return np.packbits(np.array(rows, np.uint8) != 0, axis=1), np.array(rows).shape


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    root = args.reference
    ref = Reference(root)
    only = set(filter(None, args.only.split(",")))

    def want(tag):
        return not only or tag in only

    t0 = time.time()
    # --- reference golden P75M2-0 (results/golden/P75M2-0) -------------------
    if want("real_P75M2-0"):
        g = json.load(open(os.path.join(root, "results/golden/P75M2-0")))
        pd, ip, thr = real_problem(root, 75, 2, 0)
        rpd = ref.problem(pd, 2)
        ms, log = ref.decode(rpd, 75, 2, thr, np.array(g["chromosome"], np.float32), ip)
        gl = -np.ones((2, 75, 5), np.int64)
        for m in range(2):
            for k, p in enumerate(g["machines"][str(m)]["placements"]):
                gl[m, k] = (p["part_id"], p["bin_idx"], p["col"], p["row"], p["rot"])
        ours = log_to_array(log, 2, 75)
        assert (ours == gl).all(), "reference run here differs from results/golden/P75M2-0"
        save_instance(os.path.join(args.out, "real_P75M2-0.npz"), pd, 75, 2, thr, ip, extra={
            "chromosomes": np.array([g["chromosome"]], np.float32),
            "golden_makespan": np.array([g["makespan"]], np.float64),
            "machine_makespan": np.array([g["machines"][str(m)]["makespan"] for m in range(2)], np.float64),
            "makespans": np.array([ms], np.float64), "logs": gl[None]})
        print(f"real_P75M2-0: {ms} (golden {g['makespan']})  [{time.time() - t0:.1f}s]")

    # --- P50M2-0 chromosome 462 + plate dumps ----------------------------------
    if want("real_P50M2-0"):
        pd, ip, thr = real_problem(root, 50, 2, 0)
        rpd = ref.problem(pd, 2)
        np.random.seed(42)
        pop = np.random.uniform(0.0, 1.0, size=(500, 100)).astype(np.float32)
        ms, log = ref.decode(rpd, 50, 2, thr, pop[462], ip)
        extra = {"chromosomes": pop[462:463], "golden_makespan": np.array([448166.8336]),
                 "makespans": np.array([ms]), "logs": log_to_array(log, 2, 50)[None]}
        for path in sorted(glob.glob(os.path.join(root, "results/inspection_output/pp_bin_m*_b*.txt"))):
            tag = os.path.basename(path)[len("pp_bin_"):-4]
            bits, shape = read_plate(path)
            extra[f"plate_{tag}"] = bits
            extra[f"plate_{tag}_shape"] = np.array(shape)
        save_instance(os.path.join(args.out, "real_P50M2-0.npz"), pd, 50, 2, thr, ip, extra=extra)
        print(f"real_P50M2-0 #462: {ms}  [{time.time() - t0:.1f}s]")

    # --- benchmark fingerprints (benchmark_harness.py:171-195) -----------------
    bench = json.load(open(sorted(glob.glob(os.path.join(root, "benchmarks/*.json")))[0]))
    seen = set()
    for res in bench["results"]:
        name = res["instance"]
        if name in seen or not want("fp_" + name):
            continue
        seen.add(name)
        n, mm, k = res["nb_parts"], res["nb_machines"], res["inst_idx"]
        pd, ip, thr = real_problem(root, n, mm, k)
        pop = np.random.default_rng(bench["seed"] + bench["n_reps"] - 1).random(
            (bench["mult"] * n, 2 * n), dtype=np.float64).astype(np.float32)
        fp = np.array([float(v) for v in res["fingerprint"]], np.float64)
        # reference pp run on the first chromosomes, until five feasible ones are decoded
        rpd = ref.problem(pd, mm)
        rows, mss, logs = [], [], []
        for i in range(pop.shape[0]):
            ms, log = ref.decode(rpd, n, mm, thr, pop[i], ip)
            rows.append(i)
            mss.append(ms)
            logs.append(log_to_array(log, mm, n))
            if sum(1 for v in mss if v < 1e15) == 5:
                break
        feas = np.array([v for v in mss if v < 1e15])
        assert np.allclose(feas, fp, rtol=0, atol=5e-7), (name, feas, fp)
        save_instance(os.path.join(args.out, f"fp_{name}.npz"), pd, n, mm, thr, ip, extra={
            "pop_seed": np.int64(bench["seed"] + bench["n_reps"] - 1), "pop_mult": np.int64(bench["mult"]),
            "fingerprint": fp, "n_feasible": np.int64(res["n_feasible"]),
            "n_infeasible": np.int64(res["n_infeasible"]), "rows": np.array(rows),
            "chromosomes": pop[rows], "makespans": np.array(mss), "logs": np.stack(logs)})
        print(f"fp_{name}: fingerprint ok over {len(rows)} chromosomes  [{time.time() - t0:.1f}s]")

    # --- synthetic instances ----------------------------------------------------
    def syn_case(tag, inst, chrom, stable=False):
        if not want(tag):
            return
        rpd = ref.problem(inst.problem_data, inst.nb_machines)
        mss, logs = [], []
        for c in chrom:
            ms, log = ref.decode(rpd, inst.nb_parts, inst.nb_machines, inst.thresholds, c, inst.instance_parts,
                                 stable=stable)
            mss.append(ms)
            logs.append(log_to_array(log, inst.nb_machines, inst.nb_parts))
        save_instance(os.path.join(args.out, f"{tag}.npz"), inst.problem_data, inst.nb_parts, inst.nb_machines,
                      inst.thresholds, inst.instance_parts,
                      extra={"chromosomes": np.asarray(chrom, np.float32), "makespans": np.array(mss),
                             "logs": np.stack(logs), "stable_ties": np.int64(stable)})
        print(f"{tag}: {len(chrom)} chromosomes  [{time.time() - t0:.1f}s]")

    i50 = syn.p50m2(0)
    syn_case("syn_P50M2_s0", i50, syn.chromosomes(32, 50, 1))
    i100 = syn.p100m4(0)
    syn_case("syn_P100M4_s0", i100, syn.chromosomes(8, 100, 1))
    # the benchmark's own rows: the first 16 chromosomes of the population of
    # bench.py's first timed step (P100M4 population 500, default warm-up of 5)
    if want("syn_bench_P100M4_rows"):
        import bench as bench_py
        ch = syn.chromosomes(bench_py.POP, 100, bench_py.chrom_seed(0, 5))[:16]
        syn_case("syn_bench_P100M4_rows", syn.p100m4(bench_py.INSTANCE_SEED), ch)
    # six machines: the thresholds 1/6, 2/6, 4/6, 5/6 are not float32-exact
    # (placement.py:122-127 compares in float32); some machine keys sit on
    # f32(k/6) and on the next float above it
    if want("syn_P200M6_s0"):
        i200 = syn.p200m6(0)
        ch = syn.chromosomes(4, 200, 1)
        for r in range(4):
            for k in range(1, 6):
                t = np.float32(k / 6)
                ch[r, 200 + (7 * k + 11 * r) % 200] = t
                ch[r, 200 + (7 * k + 11 * r + 3) % 200] = np.nextafter(t, np.float32(1))
        syn_case("syn_P200M6_s0", i200, ch)
    # the large stress geometry: 600x600 plates, masks up to 240x240 cells
    if want("syn_P400M8_s0"):
        syn_case("syn_P400M8_s0", syn.p400m8(0), syn.chromosomes(2, 400, 1))
    small = syn.small(3, n_parts=14, plates=((64, 48), (40, 72)), bbox_max=30)
    syn_case("syn_small_nonsquare", small, syn.chromosomes(48, 14, 2))
    # infeasible parts: machine 1's plate is smaller than some masks (placement.py:47-53)
    tight = syn.make_instance("tight", 10, [(90, 90), (26, 30)], 5, bbox_min=8, bbox_max=40, allow_unfit=True)
    syn_case("syn_infeasible", tight, syn.chromosomes(40, 10, 3))
    # three machines: thresholds 1/3, 2/3 are not float32-exact; keys placed on f32(t)
    m3 = syn.make_instance("M3", 18, [(70, 70), (60, 80), (80, 60)], 7, bbox_min=6, bbox_max=32)
    ch = syn.chromosomes(24, 18, 4)
    f13, f23 = np.float32(1 / 3), np.float32(2 / 3)
    for r in range(0, 24, 2):
        ch[r, 18 + (r % 18)] = f13
        ch[r, 18 + ((r + 5) % 18)] = f23
        ch[r, 18 + ((r + 9) % 18)] = np.nextafter(f13, np.float32(1))
    syn_case("syn_three_machines", m3, ch)
    # equal sequencing keys: reference run with a stable argsort (ties keep gene order)
    ties = syn.make_instance("ties", 16, [(64, 64), (56, 56)], 9, bbox_min=6, bbox_max=28)
    ch = syn.chromosomes(24, 16, 6)
    ch[:, :16] = np.floor(ch[:, :16] * 4) / 4
    syn_case("syn_ties_stable", ties, ch, stable=True)
    # full-row and single-cell masks, plates barely larger than the parts
    edge = syn.make_instance("edge", 12, [(24, 24), (20, 31)], 11, bbox_min=1, bbox_max=18, fill=(0.3, 1.0))
    syn_case("syn_edge", edge, syn.chromosomes(48, 12, 8))
    # --- greedy initial solutions (BRKGA_alg3.py:445-603) ------------------------
    def greedy_case(tag, pd, nb_parts, nb_machines, thr, ip, heights, areas, seeds):
        if not want(tag):
            return
        rpd = ref.problem(pd, nb_machines)
        chroms, mks, recs = [], [], []
        for sd in seeds:
            c, mk, out = reference_greedy(ref, root, rpd, nb_parts, nb_machines, thr, ip, heights, areas, sd)
            chroms.append(c)
            mks.append(mk)
            recs.append(out)
        ids = sorted(set(int(p) for p in ip))
        save_instance(os.path.join(args.out, f"{tag}.npz"), pd, nb_parts, nb_machines, thr, ip, extra={
            "greedy_seeds": np.array(seeds), "greedy_chromosomes": np.stack(chroms), "greedy_makespans": np.array(mks),
            "greedy_placements": np.stack(recs), "height_ids": np.array(ids),
            "heights": np.array([heights[i] for i in ids], np.float64)})
        print(f"{tag}: {len(seeds)} greedy runs  [{time.time() - t0:.1f}s]")

    # the reference's makespans of the whole populations of bench.py's first and
    # last timed steps with its defaults (warm-up 5, 20 steps: populations 5 and
    # 24; 500 P100M4 rows each, regenerated from their seed by the test) — the
    # two steps whose rows bench.py checks against the oracle
    for tag, step in (("refms_bench_P100M4_step0", 5), ("refms_bench_P100M4_step19", 24)):
        if not want(tag):
            continue
        import bench as bench_py
        seed = bench_py.chrom_seed(0, step)
        rows = syn.chromosomes(bench_py.POP, 100, seed)
        with bench_pool(root, os.cpu_count() or 1) as ex:
            mss = np.array(list(ex.map(_pool_decode, rows, chunksize=4)), np.float64)
        np.savez(os.path.join(args.out, f"{tag}.npz"), makespans=mss,
                 pop=np.int64(bench_py.POP), seed=np.int64(seed), instance_seed=np.int64(bench_py.INSTANCE_SEED),
                 rows_sum=np.float64(rows.astype(np.float64).sum()), first_row=rows[0])
        print(f"{tag}: {len(rows)} makespans  [{time.time() - t0:.1f}s]")
    # the rows the GPU tests compare with the oracle at the larger configurations
    # (tests/test_decoder_gpu.py, test_benchmark_workloads_vs_oracle): P200M6 24
    # rows of seed 13, P400M8 8 rows of seed 14 (workers bounded by memory: the
    # reference keeps every rotation's plate-sized FFT, ~3 GB and ~18 GB a process)
    for maker, P, seed, workers in (("p200m6", 24, 13, 4), ("p400m8", 8, 14, 2)):
        tag = f"refms_{maker.upper()}_s{seed}"
        if not want(tag):
            continue
        inst = getattr(syn, maker)(0)
        rows = syn.chromosomes(P, inst.nb_parts, seed)
        with bench_pool(root, workers, maker, 0) as ex:
            mss = np.array(list(ex.map(_pool_decode, rows)), np.float64)
        np.savez(os.path.join(args.out, f"{tag}.npz"), makespans=mss, pop=np.int64(P), seed=np.int64(seed),
                 instance_seed=np.int64(0), rows_sum=np.float64(rows.astype(np.float64).sum()), first_row=rows[0])
        print(f"{tag}: {len(rows)} makespans  [{time.time() - t0:.1f}s]")
    # the rows of the uneven multi-instance GPU test (tests/test_multi_gpu.py:
    # instance k = instances.uneven(k), POPS[k] rows of seed 100 + k), except
    # the one-machine instance, which the reference cannot decode (placement.py
    # reads thresholds[0] of an empty list)
    if want("refms_uneven"):
        pops = [12, 0, 9, 16, 3, 7, 5]
        out = {"pops": np.array(pops, np.int64)}
        for k, P in enumerate(pops):
            inst = syn.uneven(k)
            if P == 0 or inst.nb_machines < 2:
                continue
            rows = syn.chromosomes(P, inst.nb_parts, 100 + k)
            with bench_pool(root, min(4, P), "uneven", k) as ex:
                out[f"makespans_{k}"] = np.array(list(ex.map(_pool_decode, rows)), np.float64)
            out[f"rows_sum_{k}"] = np.float64(rows.astype(np.float64).sum())
        np.savez(os.path.join(args.out, "refms_uneven.npz"), **out)
        print(f"refms_uneven: {sorted(k for k in out if k.startswith('makespans'))}  [{time.time() - t0:.1f}s]")

    # the reference's GA operators on seeded populations, fed the device GA's
    # random draws: (P, N, elites, mutants, rho, seed, generation) per case —
    # the reference's proportions, the 10/15 % of BRKGA_alg3.py:608-618, one
    # elite and no mutants, and no offspring at all
    if want("ga_ops"):
        cases = [(40, 10, 6, 8, 0.7, 123, 3), (100, 25, 10, 15, 0.7, 7, 1), (57, 13, 1, 0, 0.5, 99, 200),
                 (64, 8, 13, 51, 0.9, 5, 2)]
        out = {"cases": np.array(cases, np.float64)}
        rng = np.random.default_rng(2024)
        for i, (P, N, ne, nm, rho, seed, gen) in enumerate(cases):
            pop = rng.random((P, 2 * N)).astype(np.float32)
            fit = rng.permutation(P).astype(np.float64) * 1000.0 + rng.random(P)  # no ties
            nxt, efit = reference_ga_step(root, pop, fit, ne, nm, rho, seed, gen)
            out.update({f"pop_{i}": pop, f"fit_{i}": fit, f"next_{i}": nxt, f"elite_fit_{i}": efit})
        np.savez(os.path.join(args.out, "ga_ops.npz"), **out)
        print(f"ga_ops: {len(cases)} cases  [{time.time() - t0:.1f}s]")

    hts = real_heights(root)
    for (n, mm, k) in ((50, 2, 0), (75, 2, 0), (100, 4, 0)):
        pd, ip, thr = real_problem(root, n, mm, k)
        greedy_case(f"greedy_P{n}M{mm}-{k}", pd, n, mm, thr, ip, hts, {p: pd.parts[p].area for p in pd.parts},
                    [1, 2])
    for inst in (syn.p50m2(0), syn.p100m4(0)):
        hd = {p: float(inst.heights[p]) for p in range(inst.nb_parts)}
        greedy_case(f"greedy_syn_{inst.name}", inst.problem_data, inst.nb_parts, inst.nb_machines,
                    inst.thresholds, inst.instance_parts, hd, {p: inst.problem_data.parts[p].area for p in hd}, [3])
    print(f"done in {time.time() - t0:.1f}s")


if __name__ == "__main__":
    main()
