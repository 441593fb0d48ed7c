"""bench.py's output contract, on the CPU: the reference arm prints one JSON
line with the same metric, unit and workload config as the GPU arm, a
cpu_baseline record and an e2e record without host-device traffic; the clock
sampler keeps only the samples taken inside the timed region."""
import datetime
import importlib.util
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_arm_prints_the_contract_line():
    res = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1", "--pop", "16"], capture_output=True, text=True, timeout=600, cwd=REPO)
    assert res.returncode == 0, res.stderr
    line = json.loads(res.stdout.strip().splitlines()[-1])
    bench = load_bench()
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT and line["higher_is_better"] is True
    assert line["config"] == bench.workload_config(16, 1)
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 1
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_clock_sampler_keeps_the_timed_region(tmp_path):
    bench = load_bench()
    cs = bench.ClockSampler.__new__(bench.ClockSampler)
    cs.path = str(tmp_path / "clocks.csv")
    now = datetime.datetime(2026, 1, 1, 12, 0, 0)

    def row(ms, mhz, power_cap):
        ts = (now + datetime.timedelta(milliseconds=ms)).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
        cap = "Active" if power_cap else "Not Active"
        return f"{ts}, 0, {mhz}, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, {cap}"

    lines = [row(0, 1200, True), row(20, 1965, False), row(40, 1950, False), row(60, 1965, True), row(80, 1100, False)]
    with open(cs.path, "w") as f:
        f.write("\n".join(lines) + "\n")

    class Proc:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            pass

    cs.proc = Proc()
    cs.t0 = now + datetime.timedelta(milliseconds=10)
    cs.t1 = now + datetime.timedelta(milliseconds=70)
    got = cs.stop()
    assert got["in_timed_region"] and got["samples"] == 3
    assert got["sm_mhz"] == 1965.0 and got["reasons"] == ["sw_power_cap"]
    assert not os.path.exists(cs.path)


def test_reference_anchor_compares_with_the_reference_fixtures():
    """bench.py's parity record compares the GPU makespans of the first and last
    timed populations with the reference's own (tests/golden/refms_bench_*):
    fed the reference's makespans it counts every row exact, one changed row
    is counted, and populations without a fixture (other step counts or sizes)
    are skipped."""
    import numpy as np
    bench = load_bench()
    z0 = np.load(os.path.join(HERE, "golden", "refms_bench_P100M4_step0.npz"))
    z19 = np.load(os.path.join(HERE, "golden", "refms_bench_P100M4_step19.npz"))
    rec = bench.reference_anchor([(5, z0["makespans"]), (24, z19["makespans"])])
    assert rec["rows"] == 1000 and rec["exact"] == 1000
    assert rec["fixtures"] == ["refms_bench_P100M4_step0", "refms_bench_P100M4_step19"]
    bad = z19["makespans"].copy()
    bad[7] += 1.0
    assert bench.reference_anchor([(5, z0["makespans"]), (24, bad)])["exact"] == 999
    assert bench.reference_anchor([(6, z0["makespans"])])["rows"] == 0
    assert bench.reference_anchor([(5, z0["makespans"][:100])])["rows"] == 0
    json.dumps(rec)


def test_parity_record_with_a_stand_in_decoder():
    """bench.parity_and_cpu end to end on the CPU: a stand-in for the device
    decoder (the oracle, behind numpy-backed stand-ins of the few torch calls
    the function makes) gives every row exact, every placement exact, and no
    reference rows for a population without a fixture."""
    import numpy as np
    bench = load_bench()
    from brkga_fft2_b200 import instances
    from oracle import oracle_decode
    inst, packed = bench.load_workload()

    class T:  # a host array standing in for a device tensor
        def __init__(self, a):
            self.a = a

        def cuda(self):
            return self

        def cpu(self):
            return self

        def numpy(self):
            return self.a

    class FakeTorch:
        int32 = np.int32

        @staticmethod
        def from_numpy(h):
            return T(h)

        @staticmethod
        def empty(shape, dtype=None, device=None):
            return T(np.zeros(shape, np.int32))

    class Decoder:
        def decode(self, dev, log=None):
            ms, lg = oracle_decode(packed, dev.a, n_threads=2, with_log=True)
            log.a[...] = np.stack([lg[f] for f in ("gene", "bin", "x", "y", "rot")], axis=-1)
            return T(ms)

    P, N, M = 8, inst.nb_parts, inst.nb_machines
    rows = [instances.chromosomes(P, N, bench.chrom_seed(0, s)) for s in (3, 4)]
    parity, cpu = bench.parity_and_cpu(Decoder(), packed, rows, P, M, N, FakeTorch, step_ids=[3, 4])
    assert parity["rows"] == 16 and parity["exact"] == 16 and parity["placements_exact"]
    assert parity["reference"]["rows"] == 0 and parity["reference"]["fixtures"] == []
    assert cpu["kind"] == "port" and cpu["value"] > 0
    json.dumps(parity)
    json.dumps(cpu)
