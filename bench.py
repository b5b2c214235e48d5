"""Benchmark of the GWFA sequence-to-graph edit-distance path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload config3] [--impl ours|reference]

One step = one pass of the path over the whole workload (default: the mixed-length batch, 200,000
reads with lognormal lengths of median 2 kbp in [500, 10000] bp and error rates U[1%, 10%], on the
100 kbp bubble graph; synthetic and seeded), in the persistent form, beside the plain form on the
same reads. `value` is reads/s with the reads already resident in HBM (CUDA events on the
library's stream, L2 flushed between steps); `e2e` is the same metric through gwf_ed_batch_concat
from pinned host memory, with the copies in the timed region. Under torchrun every rank aligns
its own workload (weak scaling, no data-path collective); timings are the max over ranks.
`--impl reference` times the reference algorithm on the host cores instead (the reference ships
no CPU gwf_ed; its CPU restatement in oracle/ stands in for it, on inputs made by the same seeded
generator compiled into oracle/liboracle.so, so that arm maps no library of the product).
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "reads/sec and Gbases/sec (bit-exact), persistent-batched vs plain kernel; serving p50/p99"
WORKLOAD_DESC = {
    "config1": "config1: 1,000 reads x 1 kbp at 1% on the 100 kbp bubble graph",
    "config2": "config2: 100,000 reads x 1 kbp (50,000 at 5%, 50,000 at 10%) on the 100 kbp bubble graph",
    "config3": "config3: 200,000 reads, lognormal length (median 2 kbp, sigma 0.6, 500-10000 bp), error U[1%,10%]",
    "config4": "config4: 20,000 reads x 10 kbp at 5% on the 5 Mbp graph (variant every 50 bp, SV every 50 kbp)",
}


def pkg():
    import importlib.util
    d = os.path.join(ROOT, "gwfa-cuda-version_b200")
    if "gwfa_b200" in sys.modules:
        return sys.modules["gwfa_b200"]
    spec = importlib.util.spec_from_file_location("gwfa_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules["gwfa_b200"] = m
    spec.loader.exec_module(m)
    return m


def oracle_mod():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def shard_seed(workload, rank):
    """Per-rank seed: rank 0 uses the published workload seeds, others shift them."""
    return None if rank == 0 else 1000 + 17 * rank


def reduce_max(x, dist=None, device="cuda"):
    """Max of a per-rank timing over all ranks (the rank's own value without a process group)."""
    if dist is None or not dist.is_initialized():
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks during the timed region (one sample every 200 ms)."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(lens, W, E):
    """Bytes per read: ql + 4 + 32 W + 2 E (query, result, one 16-byte state read and written
    per wavefront diagonal per step, one graph and one query byte per compared character)."""
    return float(np.sum(lens.astype(np.float64) + 4 + 32.0 * W + 2.0 * E))


def cpu_oracle_run(w, max_seconds=30.0, threads=0):
    """Oracle over the workload with all host threads. Runs the whole workload when a probe
    predicts it finishes within max_seconds, else a prefix sample of each error class."""
    O = oracle_mod()
    og = O.OracleGraph.from_graph(w["graph"])
    n = len(w["lens"])
    probe = min(n, 2000)
    idx_probe = np.linspace(0, n - 1, probe).astype(np.int64)
    t0 = time.perf_counter()
    _, _, used = og.ed_batch(w["cat"], w["offs"][idx_probe], w["lens"][idx_probe], w["v0"][idx_probe],
                             stats=False, threads=threads)
    tp = time.perf_counter() - t0
    est = tp * n / probe
    if est <= max_seconds:
        sel = np.arange(n)
    else:
        m = max(probe, int(n * max_seconds / est))
        sel = np.linspace(0, n - 1, m).astype(np.int64)
    t0 = time.perf_counter()
    dist, st, used = og.ed_batch(w["cat"], w["offs"][sel], w["lens"][sel], w["v0"][sel], stats=True,
                                 threads=threads)
    el = time.perf_counter() - t0
    s = O.stats_arrays(st, len(sel))
    return {"sel": sel, "dist": dist, "W": s["W"], "E": s["E"], "flags": s["flags"], "seconds": el,
            "threads": used, "full": len(sel) == n}


def mapped_libraries():
    """Shared objects of this repository mapped into the process (from /proc/self/maps)."""
    out = set()
    try:
        for line in open("/proc/self/maps"):
            f = line.split()
            if len(f) >= 6 and f[-1].endswith(".so") and f[-1].startswith(ROOT):
                out.add(os.path.relpath(f[-1], ROOT))
    except OSError:
        pass
    return sorted(out)


def run_reference(args, rank, world):
    """Reference arm: the reference algorithm on the host cores (oracle port, all threads). The
    workload comes from the same seeded generator compiled into liboracle.so, so this process
    maps no library of the product."""
    if rank != 0:
        return
    spec = pkg().workload_spec(args.workload)  # plain data: the package's library is not loaded
    O = oracle_mod()
    w = O.synth_workload(spec)
    og = w["graph"]
    n = len(w["lens"])
    # each step aligns a bounded, evenly spread sample so the whole run takes a few minutes
    budget_s = args.ref_step_seconds
    probe = np.linspace(0, n - 1, min(n, 1000)).astype(np.int64)
    t0 = time.perf_counter()
    _, _, threads = og.ed_batch(w["cat"], w["offs"][probe], w["lens"][probe], w["v0"][probe], stats=False)
    per_read = (time.perf_counter() - t0) / len(probe)
    m = int(min(n, max(len(probe), budget_s / max(per_read, 1e-9))))
    sel = np.linspace(0, n - 1, m).astype(np.int64)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        og.ed_batch(w["cat"], w["offs"][sel], w["lens"][sel], w["v0"][sel], stats=False)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    ms = 1000.0 * statistics.mean(times)
    rps = m / (ms / 1000.0)
    bases = float(np.sum(w["lens"][sel]))
    line = {
        "impl": "reference", "metric": METRIC, "value": rps, "unit": "reads/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": WORKLOAD_DESC[args.workload], "reads_per_gpu": n,
                   "l2": "not applicable: host cores",
                   "parallelism": "all host threads, one process (an evenly spread sample per step)"},
        "gbases_per_s": bases / (ms / 1000.0) / 1e9,
        "cpu_baseline": {"value": rps, "unit": "reads/s", "cores": threads, "kind": "port",
                         "sample": "%d of %d reads per step, evenly spread" % (m, n)},
        "e2e": {"value": rps, "unit": "reads/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "libraries_mapped": mapped_libraries(),
    }
    print(json.dumps(line), flush=True)


def make_requests(w, rng, max_reads=256):
    """Split the workload's reads into consecutive requests of U{1..max_reads} reads."""
    n = len(w["lens"])
    reqs, i = [], 0
    while i < n:
        m = int(rng.integers(1, max_reads + 1))
        idx = np.arange(i, min(n, i + m))
        reqs.append(((w["cat"], np.ascontiguousarray(w["offs"][idx]), np.ascontiguousarray(w["lens"][idx])),
                     np.ascontiguousarray(w["v0"][idx])))
        i += m
    return reqs


def serve_stream(srv, reqs, rate_rps, rng):
    """Submits requests at seeded Poisson arrival times (rate in requests/s; 0 = all at once) and
    waits for all. Returns per-request latency (done - submit) and the span from the first
    submit to the last completion."""
    gaps = rng.exponential(1.0 / rate_rps, len(reqs)) if rate_rps > 0 else np.zeros(len(reqs))
    ids = []
    t_next = time.perf_counter()
    for (reads, v0), gap in zip(reqs, gaps):
        t_next += gap
        d = t_next - time.perf_counter()
        if d > 0:
            time.sleep(d)
        ids.append(srv.submit(reads, v0))
    lat, first, last = [], None, None
    for rid, k in ids:
        _, st = srv.wait(rid, k, timeout_s=600)
        if not (st == 0).all():
            raise RuntimeError("serving request %d: read status %s" % (rid, np.unique(st)))
        ts, _, td = srv.times(rid)
        lat.append(td - ts)
        first = ts if first is None else min(first, ts)
        last = td if last is None else max(last, td)
    return np.array(lat), last - first


def fifo_replay(arrivals, service):
    """Latency of a single FIFO server (one launch per request, one after another)."""
    lat, free = [], 0.0
    for a, s in zip(arrivals, service):
        start = max(a, free)
        free = start + s
        lat.append(free - a)
    return np.array(lat)


def run_serving(args):
    """Serving on the 5 Mbp graph (resident): requests of U{1..256} reads, ql U[500, 20000],
    error U[1%, 10%], seeded Poisson arrivals at 50/70/90% of the measured peak, admission by a
    fixed arena budget. Plain baseline: one plain launch per request, served FIFO."""
    G = pkg()
    w = G.load_workload("config5", n=args.serve_reads)
    g = w["graph"]
    g.index()
    budget = int(args.serve_budget_gib * (1 << 30))
    srv = G.Server(g, arena_budget_bytes=budget, warps_per_read=args.serve_warps)
    rng = np.random.default_rng(55)
    reqs = make_requests(w, rng)
    nreads = [len(r[1]) for r in reqs]
    mean_req = float(np.mean(nreads))
    # warm-up, then peak: every request submitted at once
    serve_stream(srv, reqs[:4], 0, rng)
    with ClockSampler(0) as clk:
        _, span = serve_stream(srv, reqs, 0, rng)
        peak = sum(nreads) / span
        print("serving peak %.1f reads/s over %.1f s" % (peak, span), file=sys.stderr, flush=True)
        levels = {}
        for frac in (0.5, 0.7, 0.9):
            rate = frac * peak / mean_req
            lat, span = serve_stream(srv, reqs, rate, np.random.default_rng(int(frac * 100)))
            key = "%d%%" % int(frac * 100)
            levels[key] = {"offered_reads_per_s": frac * peak, "reads_per_s": sum(nreads) / span,
                           "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                           "requests": len(reqs)}
            print("serving at %s: %s" % (key, levels[key]), file=sys.stderr, flush=True)
    stats = srv.stats()
    srv.close()
    # plain one-launch-per-request: measured launch times on a sample, FIFO replay per level
    sample = reqs[:args.plain_sample]
    svc = []
    for reads, v0 in sample:
        t0 = time.perf_counter()
        g.ed_batch(reads, v0, mode=G.MODE_PLAIN)
        svc.append(time.perf_counter() - t0)
        print("plain request of %d reads: %.2f s" % (len(v0), svc[-1]), file=sys.stderr, flush=True)
    plain_cap = sum(nreads[:len(sample)]) / sum(svc)
    service = [svc[i % len(svc)] for i in range(len(reqs))]
    plain = {"reads_per_s_capacity": plain_cap, "sample_requests": len(sample)}
    for frac in (0.5, 0.7, 0.9):
        rate = frac * peak / mean_req
        arr = np.cumsum(np.random.default_rng(int(frac * 100)).exponential(1.0 / rate, len(reqs)))
        lat = fifo_replay(arr, service)
        plain["%d%%" % int(frac * 100)] = {"p50_s": float(np.percentile(lat, 50)),
                                           "p99_s": float(np.percentile(lat, 99))}
    line = {
        "metric": "serving p50/p99 request latency and reads/s at 50/70/90% of peak offered load",
        "value": levels["70%"]["p99_s"], "unit": "s (p99 at 70% of peak)", "n_gpus": 1,
        "higher_is_better": False, "dtype": "int32", "data": "synthetic",
        "config": {"workload": "config5: 5 Mbp graph resident; requests of U{1..256} reads, ql U[500,20000], "
                               "error U[1%,10%]; seeded Poisson arrivals", "reads": int(sum(nreads)),
                   "requests": len(reqs), "arena_budget_gib": args.serve_budget_gib,
                   "warps_per_read": args.serve_warps or 8},
        "peak_reads_per_s": peak, "levels": levels, "server": stats,
        "plain_one_launch_per_request": plain,
        "plain_note": "plain capacity from measured per-request launches; latency by FIFO replay of the same "
                      "arrivals (the sample's launch times, cycled)",
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_features(args):
    """The options beyond the reference, each timed end to end (host arrays in, results out) on
    one GPU: traceback (paths, then paths and CIGARs) against distances alone, opt-in lag
    pruning against exact distances, and lag pruning in the serving loop. One JSON line."""
    G = pkg()

    def best_of(fn, k=3):
        fn()
        ts = []
        for _ in range(k):
            t0 = time.perf_counter()
            res = fn()
            ts.append(time.perf_counter() - t0)
        return min(ts), res

    out = {"metric": "options beyond the reference: traceback, lag pruning, serving with lag pruning",
           "unit": "reads/s", "n_gpus": 1, "dtype": "int32", "data": "synthetic"}
    trace = {}
    for name, n, max_nv, max_ops in (("config2", 100000, 64, 256), ("config4", 2000, 1024, 2048)):
        w = G.load_workload(name, n=n)
        g = w["graph"]
        g.index()
        reads = (w["cat"], w["offs"], w["lens"])
        t_d, _ = best_of(lambda: g.ed_batch(reads, w["v0"], mode=G.MODE_PLAIN))
        t_p, rp = best_of(lambda: g.ed_path(reads, w["v0"], max_nv=max_nv, as_arrays=True))
        t_c, rc = best_of(lambda: g.ed_path(reads, w["v0"], max_nv=max_nv, as_arrays=True, max_ops=max_ops))
        trace[name] = {"reads": n, "distance_only": n / t_d, "paths": n / t_p, "paths_and_cigars": n / t_c,
                       "mean_path_vertices": float(np.mean(rp[3])), "cigars": int((rc[6] > 0).sum())}
        g.close()
    out["traceback"] = trace
    lag = {}
    for name, n in (("config3", 50000), ("config4", 2000)):
        w = G.load_workload(name, n=n)
        g = w["graph"]
        g.index()
        reads = (w["cat"], w["offs"], w["lens"])
        t0, d0 = best_of(lambda: g.ed_batch(reads, w["v0"], mode=G.MODE_PERSISTENT)[0])
        row = {"reads": n, "exact": n / t0}
        for m in (5, 20):
            t, d = best_of(lambda: g.ed_batch(reads, w["v0"], mode=G.MODE_PERSISTENT, flags=G.GWF_F_MAX_LAG,
                                              max_lag=m)[0])
            row["lag%d" % m] = {"reads_per_s": n / t, "worse": int(((d != d0) & (d >= 0)).sum()),
                                "none": int((d < 0).sum())}
        lag[name] = row
        g.close()
    out["lag_pruning"] = lag
    w = G.load_workload("config5", n=3000)
    g = w["graph"]
    g.index()
    reqs = make_requests(w, np.random.default_rng(55))
    srv_rows, dists = {}, {}
    for label, kw in (("exact", {}), ("lag20", {"flags": G.GWF_F_MAX_LAG, "max_lag": 20})):
        srv = G.Server(g, arena_budget_bytes=int(args.serve_budget_gib * (1 << 30)), **kw)
        serve_stream(srv, reqs[:3], 0, np.random.default_rng(1))
        t0 = time.perf_counter()
        ids = [srv.submit(reads, v0) for reads, v0 in reqs]
        lat, ds = [], []
        for rid, k in ids:
            d, st = srv.wait(rid, k, timeout_s=600)
            ts, _, td = srv.times(rid)
            lat.append(td - ts)
            ds.append(d)
        span = time.perf_counter() - t0
        srv.close()
        srv_rows[label] = {"reads_per_s": len(w["lens"]) / span, "p50_s": float(np.percentile(lat, 50)),
                           "p99_s": float(np.percentile(lat, 99))}
        dists[label] = np.concatenate(ds)
    srv_rows["requests"] = len(reqs)
    srv_rows["same_distances"] = int((dists["exact"] == dists["lag20"]).sum())
    srv_rows["reads"] = len(w["lens"])
    out["serving_all_at_once"] = srv_rows
    print(json.dumps(out), flush=True)


def run_case(args):
    """Small fixed cases, one kernel each, sized for profiler captures (a few GB on the device):
    config3-4k   k_align_persistent: 20,000 config-3 reads of at most 4 kbp, one warp per read,
                 four launches;
    classes      k_align_classes: 100 config-4 reads (10 kbp, 5 Mbp graph), warps per read by
                 default (eight here), two batches;
    cigar        k_cigar: 400 config-2 reads with paths and CIGARs, two batches;
    serve        k_serve: four requests of ten config-5 reads on a one-warp server, 1 GiB budget."""
    G = pkg()
    c = args.case
    if c == "config3-4k":
        w = G.load_workload("config3", n=30000)
        sel = np.nonzero(w["lens"] <= 4000)[0][:20000]
        g = w["graph"]
        g.index()
        b = G.ResidentBatch(g, w["cat"], np.ascontiguousarray(w["offs"][sel]), np.ascontiguousarray(w["lens"][sel]),
                            np.ascontiguousarray(w["v0"][sel]), mode=G.MODE_PERSISTENT)
        ms = [b.run(warps_per_read=1, use_graph=0) for _ in range(4)]
        _, st = b.results()
        out = {"reads": len(sel), "bases": int(w["lens"][sel].sum()), "ms": ms}
    elif c == "classes":
        w = G.load_workload("config4", n=100)
        g = w["graph"]
        g.index()
        for _ in range(2):
            _, st = g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"], mode=G.MODE_PERSISTENT)
        out = {"reads": 100}
    elif c == "cigar":
        w = G.load_workload("config2", n=400)
        g = w["graph"]
        g.index()
        for _ in range(2):
            r = g.ed_path((w["cat"], w["offs"], w["lens"]), w["v0"], max_nv=64, as_arrays=True, max_ops=256)
        st = r[1]
        out = {"reads": 400, "cigars": int((r[6] > 0).sum())}
    else:
        w = G.load_workload("config5", n=40)
        g = w["graph"]
        g.index()
        srv = G.Server(g, arena_budget_bytes=1 << 30, warps_per_read=1)
        ids = [srv.submit((w["cat"], np.ascontiguousarray(w["offs"][a:a + 10]), np.ascontiguousarray(w["lens"][a:a + 10])),
                          np.ascontiguousarray(w["v0"][a:a + 10])) for a in range(0, 40, 10)]
        st = np.concatenate([srv.wait(rid, k, timeout_s=300)[1] for rid, k in ids])
        srv.close()
        out = {"reads": 40}
    if not (np.asarray(st) == 0).all():
        raise SystemExit("case %s: per-read errors" % c)
    out["case"] = c
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="config3", choices=sorted(WORKLOAD_DESC))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="persistent", choices=["persistent", "plain"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-form comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--ref-step-seconds", type=float, default=6.0)
    ap.add_argument("--ctas-per-sm", type=int, default=0, help="persistent grid; 0 = occupancy limit")
    ap.add_argument("--graph", type=int, default=1, help="1 = persistent runs replay a captured CUDA graph")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--split", action="store_true",
                    help="strong scaling: every rank holds the same workload, aligns its cost-balanced "
                         "range (partition_reads) and the distances are all-gathered")
    ap.add_argument("--reads", type=int, default=0,
                    help="the first N reads of the workload (small profiling cases); 0 = all")
    ap.add_argument("--serving", action="store_true", help="serving benchmark (config5) instead")
    ap.add_argument("--features", action="store_true",
                    help="time traceback, lag pruning and serving with lag pruning instead")
    ap.add_argument("--serve-reads", type=int, default=6000)
    ap.add_argument("--serve-budget-gib", type=float, default=64.0)
    ap.add_argument("--plain-sample", type=int, default=6)
    ap.add_argument("--warps-per-read", type=int, default=0,
                    help="persistent form: 1, 2, 4 or 8 warps per read; 0 = per read by its share of the work")
    ap.add_argument("--case", choices=["config3-4k", "classes", "cigar", "serve"],
                    help="run one small fixed case of one kernel (profiler captures) instead")
    ap.add_argument("--serve-warps", type=int, default=0, help="serving: warps per read (0 = the library default, 8)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.case:
        run_case(args)
        return
    if args.serving:
        run_serving(args)
        return
    if args.features:
        run_features(args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import torch
    torch.cuda.set_device(local)
    G = pkg()
    mode = G.MODE_PERSISTENT if args.mode == "persistent" else G.MODE_PLAIN
    seed = None if args.split else shard_seed(args.workload, rank)
    w = G.load_workload(args.workload, n=args.reads or None, seed=seed, pinned=True)
    g = w["graph"]
    g.index()
    n_total = len(w["lens"])
    # weak scaling: this rank's own workload; --split: this rank's range of the shared workload
    lo, hi = G.partition_reads(w["lens"], world)[rank] if args.split else (0, n_total)
    r_offs, r_lens, r_v0 = (np.ascontiguousarray(w[k][lo:hi]) for k in ("offs", "lens", "v0"))
    n = hi - lo
    bases = float(np.sum(r_lens))
    job_reads = n_total if args.split else world * n
    job_bases = float(np.sum(w["lens"])) if args.split else world * bases
    batch = G.ResidentBatch(g, w["cat"], r_offs, r_lens, r_v0, mode=mode)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_max(x, dist, "cuda")

    use_graph = args.graph if mode == G.MODE_PERSISTENT else 0
    for _ in range(args.warmup):
        batch.run(mode=mode, ctas_per_sm=args.ctas_per_sm, use_graph=use_graph, warps_per_read=args.warps_per_read)
    dist_gpu, status = batch.results()
    launches = 0
    times = []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()              # evict L2 between steps (256 MB > 126 MB L2)
            torch.cuda.synchronize()
            times.append(batch.run(mode=mode, ctas_per_sm=args.ctas_per_sm, use_graph=use_graph,
                                   warps_per_read=args.warps_per_read))
            launches += batch.launches()
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(statistics.mean(times))
    value = job_reads / (ms / 1000.0)

    # the other form on the same reads, for the persistent-vs-plain comparison
    forms = {}
    if not args.no_plain:
        other = G.MODE_PLAIN if mode == G.MODE_PERSISTENT else G.MODE_PERSISTENT
        batch.run(mode=other)
        t2 = []
        for _ in range(max(1, min(args.steps, 3))):
            flush.zero_()
            torch.cuda.synchronize()
            t2.append(batch.run(mode=other))
        d2, _ = batch.results()
        ms2 = max_over_ranks(statistics.mean(t2))
        forms = {args.mode: n / (ms / 1000.0),
                 ("plain" if other == G.MODE_PLAIN else "persistent"): n / (ms2 / 1000.0),
                 "forms_identical": bool(np.array_equal(d2, dist_gpu))}
        forms["persistent_over_plain"] = forms["persistent"] / forms["plain"]

    # end to end through the public batch call, pinned host buffers, copies in the timed region
    e2e_t = []
    dist_full = None  # --split: every read's distance, gathered from all ranks
    if not args.no_e2e:
        def e2e_call():
            if args.split:
                return G.align_sharded(g, (w["cat"], w["offs"], w["lens"]), w["v0"], mode=mode)[0]
            g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"], mode=mode, warps_per_read=args.warps_per_read)
        for _ in range(2):
            e2e_call()
        barrier()
        for _ in range(args.steps):
            t0 = time.perf_counter()
            dist_full = e2e_call()
            e2e_t.append(time.perf_counter() - t0)
        barrier()
    e2e_s = max_over_ranks(statistics.mean(e2e_t)) if e2e_t else None
    # bytes of the whole job per step: read bytes plus per-read offsets, lengths, v0 and queue
    # metadata in, distance and status out
    h2d = int(job_bases) + job_reads * (8 + 4 + 4 + 8 + 4)
    d2h = job_reads * 8 + 4

    line = {
        "metric": METRIC, "value": value, "unit": "reads/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong" if args.split else "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": WORKLOAD_DESC[args.workload], "reads_per_gpu": n,
                   "l2": "flushed between steps (256 MB write)",
                   "parallelism": ("one batch split by cost over the ranks, distances all-gathered, graph replicated"
                                   if args.split else "reads sharded by rank, graph replicated")},
        "form": args.mode, "cuda_graph": bool(use_graph), "warps_per_read": args.warps_per_read or "by share of work",
        "gbases_per_s": job_bases / (ms / 1000.0) / 1e9,
        "e2e": ({"value": job_reads / e2e_s, "unit": "reads/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
                if e2e_s else None),
        "gpu_launches": launches,
        "status_ok": bool((status == 0).all()),
        "clocks": clk.summary(),
    }
    if forms:
        line["forms"] = forms

    if rank == 0 and not args.no_cpu:
        cpu = cpu_oracle_run(w)
        sel = cpu["sel"]
        if args.split and dist_full is not None:
            chk, got = np.ones(len(sel), dtype=bool), dist_full[sel]
        else:  # this rank's reads
            chk = (sel >= lo) & (sel < hi)
            got = dist_gpu[sel[chk] - lo]
        line["bit_exact_vs_oracle"] = {"reads_checked": int(chk.sum()),
                                       "mismatches": int(np.sum(cpu["dist"][chk] != got))}
        line["cpu_baseline"] = {"value": len(sel) / cpu["seconds"], "unit": "reads/s", "cores": cpu["threads"],
                                "kind": "port",
                                "sample": ("whole workload" if cpu["full"] else "%d evenly spread reads" % len(sel))
                                + ", oracle/gwf_oracle.c restatement of gwf-ed.cu, all host threads"}
        scale = n / len(sel)
        alg = algorithmic_bytes(w["lens"][sel], cpu["W"], cpu["E"]) * scale
        peak, src = measured_peak()
        achieved = alg / (ms / 1000.0) / 1e9
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic_%s.json" % args.workload)
        if os.path.exists(tp):
            traffic = json.load(open(tp)).get("dram_bytes_per_launch")
        line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": traffic,
                            "peak_source": src + " hbm_gbs (burst)",
                            "algorithmic_bytes_per_step": alg,
                            "note": "B_read = ql + 4 + 32 W + 2 E per read, W/E from the oracle"
                                    + ("" if cpu["full"] else " sample, scaled")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    batch.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
