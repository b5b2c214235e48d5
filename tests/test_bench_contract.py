"""bench.py pieces that run without a GPU: the reference arm's JSON line (the oracle port on the
host cores), the clock summary that rejects throttled runs, and the algorithmic-bytes formula of
the roofline."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_reference_arm_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "config1",
                        "--steps", "1", "--warmup", "3", "--ref-step-seconds", "0.2"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["warmup"] >= 3
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    # the arm maps the oracle's library only, never the product's
    assert line["libraries_mapped"] == ["oracle/liboracle.so"], line["libraries_mapped"]


def test_reference_arm_workload_equals_product_workload(G, O):
    """The reference arm makes its inputs with the generator compiled into liboracle.so and a
    GFA parse of its own: the same reads, and the same distances as on the product loader's
    graph (whose vertex numbering differs)."""
    for kind, n in (("config1", 200), ("config2", 100), ("config3", 100)):
        w = G.load_workload(kind, n=n)
        wo = O.synth_workload(G.workload_spec(kind, n))
        end = int(w["offs"][-1] + w["lens"][-1])
        assert np.array_equal(w["offs"], wo["offs"]) and np.array_equal(w["lens"], wo["lens"])
        assert np.array_equal(w["cat"][:end], wo["cat"][:end])
        d1, _, _ = O.OracleGraph.from_graph(w["graph"]).ed_batch(w["cat"], w["offs"], w["lens"], w["v0"],
                                                                  stats=False)
        d2, _, _ = wo["graph"].ed_batch(wo["cat"], wo["offs"], wo["lens"], wo["v0"], stats=False)
        assert np.array_equal(d1, d2)


def test_clock_summary_reports_throttle_reasons():
    import bench
    c = bench.ClockSampler(0)
    c.lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1900, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1950, 1965, 990.0, 0x8, Active, Not Active, Not Active, Not Active",
               "garbage"]
    s = c.summary()
    assert s["sm_mhz"] == 1950 and s["sm_max_mhz"] == 1965 and s["samples"] == 3
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]
    c.lines = []
    assert c.summary()["samples"] == 0


def test_algorithmic_bytes():
    import bench
    lens = np.array([1000, 2000])
    W = np.array([10, 20])
    E = np.array([100, 200])
    assert bench.algorithmic_bytes(lens, W, E) == (1000 + 4 + 320 + 200) + (2000 + 4 + 640 + 400)


def test_serving_request_split_and_fifo_replay(G):
    """The serving benchmark's request split covers every read once, in order, in requests of
    1..256 reads; the plain baseline's FIFO replay queues requests behind each other."""
    import bench
    w = G.load_workload("config1", n=1000)
    reqs = bench.make_requests(w, np.random.default_rng(55))
    lens = [len(v0) for _, v0 in reqs]
    assert sum(lens) == 1000 and all(1 <= k <= 256 for k in lens)
    offs = np.concatenate([reads[1] for reads, _ in reqs])
    assert np.array_equal(offs, w["offs"])
    lat = bench.fifo_replay([0.0, 0.0, 5.0], [2.0, 2.0, 1.0])
    assert list(lat) == [2.0, 4.0, 1.0]
