"""TEST INFRASTRUCTURE ONLY: times the reference's own CUDA kernel (gwf-ed.cu, sm_100a build in
oracle/_ref/gwf-ref-harness, with the reference driver's 16-stream scheduling restated and a
per-read v0) on the benchmark workloads, on the same GPU.

Reads that the oracle flags as unsafe for the reference (arena overflow, non-termination) are
left out so the reference is never given an input that can fault or hang; the count is reported.

    python oracle/run_ref_gpu.py config2 [config1 config3 config4] > ref_gpu.json
    python oracle/run_ref_gpu.py config4:2000      # the first 2,000 reads of a workload
"""
import importlib.util
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def pkg():
    d = os.path.join(ROOT, "gwfa-cuda-version_b200")
    spec = importlib.util.spec_from_file_location("gwfa_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules["gwfa_b200"] = m
    spec.loader.exec_module(m)
    return m


def main():
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import oracle as O
    G = pkg()
    harness = os.path.join(ROOT, "oracle", "_ref", "gwf-ref-harness")
    out = []
    for arg in sys.argv[1:] or ["config2"]:
        kind, _, n = arg.partition(":")
        w = G.load_workload(kind, n=int(n) if n else None)
        og = O.OracleGraph.from_graph(w["graph"])
        t0 = time.perf_counter()
        d_or, st, threads = og.ed_batch(w["cat"], w["offs"], w["lens"], w["v0"])
        t_or = time.perf_counter() - t0
        flags = O.stats_arrays(st, len(w["lens"]))["flags"]
        keep = np.nonzero((flags & O.F_UNSAFE_MASK) == 0)[0]
        with tempfile.TemporaryDirectory() as td:
            open(os.path.join(td, "g.gfa"), "wb").write(w["synth"].gfa)
            with open(os.path.join(td, "r.fa"), "wb") as f:
                for i in keep:
                    o, l = int(w["offs"][i]), int(w["lens"][i])
                    f.write(b">r\n" + w["cat"][o:o + l].tobytes() + b"\n")
            np.savetxt(os.path.join(td, "v0.txt"), w["v0"][keep], fmt="%d")
            res = subprocess.run([harness, os.path.join(td, "g.gfa"), os.path.join(td, "r.fa"),
                                  os.path.join(td, "v0.txt")], capture_output=True, text=True, timeout=3000)
        if res.returncode != 0:
            raise SystemExit(kind + ": harness failed: " + res.stderr[-2000:])
        timing = json.loads(res.stderr.strip().splitlines()[-1])
        d_ref = np.array([int(x) for x in res.stdout.split()])
        line = {"workload": arg, "reads": int(len(w["lens"])), "reads_run": int(len(keep)),
                "reference_gpu_seconds": timing["seconds"], "reference_gpu_reads_per_s": timing["reads_per_s"],
                "reference_launches": timing["launches"], "reference_streams": timing["streams"],
                "oracle_threads": threads, "oracle_seconds": t_or,
                "reference_equals_oracle": int(np.sum(d_ref == d_or[keep])),
                "timing_scope": "wall clock from the first memset/copy to the last result copy (all streams)"}
        print(json.dumps(line), flush=True)
        out.append(line)


if __name__ == "__main__":
    main()
