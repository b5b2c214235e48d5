"""Generates the golden fixtures of tests/golden/ from the reference itself.

Stages (run in order):
  prepare   (CPU, needs the reference tree): copies the reference's exposed fixtures
            (graph_1000.gfa, grafo_test.gfa, the first 200 reads of reads_1000.fa) into
            tests/golden/, records the reference loader's `gwf-test -p` dumps, and writes the
            synthetic read sets to _work/golden_inputs/ as FASTA + per-read v0. Reads that the
            oracle flags as unsafe for the reference (arena overflow, non-termination) are
            left out, so the reference kernel is never given an input that can fault or hang.
  run       (a machine with a B200): runs oracle/_ref/gwf-test and oracle/_ref/gwf-ref-harness
            (the reference's own CUDA code, built by `make -C oracle ref`) on those inputs;
            writes OUTDIR/*.txt.
  collect   (CPU): copies the reference outputs from OUTDIR into tests/golden/ref_*.txt.

    python tests/golden/make_golden.py prepare [SET ...]
    python tests/golden/make_golden.py run OUTDIR [SET ...]       # on the GPU machine
    python tests/golden/make_golden.py collect OUTDIR [SET ...]   # OUTDIR brought back here

SET names one synthetic set (default: all of them, plus the reference's exposed fixture); the
overlap_* sets are graphs whose GFA links carry overlaps (tests/golden/overlap_graph.py).
"""
import importlib.util
import json
import os
import shutil
import subprocess
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
GOLD = os.path.join(ROOT, "tests", "golden")
INP = os.path.join(ROOT, "_work", "golden_inputs")
OUT = None  # the reference outputs' directory, from the command line
REF = os.environ.get("GWF_REFERENCE_DIR", "/root/reference")  # the reference source tree

# synthetic sets: name -> (workload, n reads); the overlap_* sets come from overlap_graph.py
SYNTH = {"config1": ("config1", 1000), "config2": ("config2", 2000), "config3": ("config3", 600),
         "config4": ("config4", 200), "config5": ("config5", 100),
         "overlap_uniform": ("uniform", 300), "overlap_mixed": ("mixed", 300)}
SETS = list(SYNTH)  # the sets a stage works on (command line)


def build_set(G, name):
    """(GFA text, product Graph, cat, offs, lens, v0) of one synthetic set; v0 in the loader's
    vertex numbering, which is the reference's (gwf_gfa2gwf from the first segment)."""
    kind, n = SYNTH[name]
    if name.startswith("overlap_"):
        sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
        from overlap_graph import overlap_gfa, overlap_reads
        text, seqs, links = overlap_gfa(5 if kind == "uniform" else 7, mode=kind)
        g = G.Graph.from_gfa_text(text)
        seg2v = g.vertex_of_segment()
        reads, starts = overlap_reads(6 if kind == "uniform" else 8, seqs, links, n)
        cat, offs, lens = G.pack_reads(reads)
        return text, g, cat, offs, lens, np.array([seg2v[v] for v in starts], dtype=np.int32)
    w = G.load_workload(kind, n=n)
    return w["synth"].gfa, w["graph"], w["cat"], w["offs"], w["lens"], w["v0"]


def pkg():
    spec = importlib.util.spec_from_file_location(
        "gwfa_b200", os.path.join(ROOT, "gwfa-cuda-version_b200", "__init__.py"),
        submodule_search_locations=[os.path.join(ROOT, "gwfa-cuda-version_b200")])
    m = importlib.util.module_from_spec(spec)
    sys.modules["gwfa_b200"] = m
    spec.loader.exec_module(m)
    return m


def oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as o
    return o


def read_fasta(path, limit=None):
    reads = []
    for line in open(path, "rb"):
        line = line.rstrip(b"\r\n")
        if line.startswith(b">"):
            if limit is not None and len(reads) >= limit:
                break
            reads.append(b"")
        elif reads:
            reads[-1] += line
    return reads


def write_fasta(path, reads):
    with open(path, "wb") as f:
        for i, r in enumerate(reads):
            f.write(b">r%d\n%s\n" % (i, r))


def prepare():
    G, O = pkg(), oracle()
    os.makedirs(INP, exist_ok=True)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all", "ref", "REF=" + REF], check=True)
    gwf_test = os.path.join(ROOT, "oracle", "_ref", "gwf-test")
    if SETS == list(SYNTH):
        prepare_exposed(G, O, gwf_test)
    # synthetic sets
    mpath = os.path.join(INP, "manifest.json")
    manifest = json.load(open(mpath)) if os.path.exists(mpath) else {}
    for name in SETS:
        text, g, cat, offs, lens, v0 = build_set(G, name)
        n = len(lens)
        og = O.OracleGraph.from_graph(g)
        d, st, _ = og.ed_batch(cat, offs, lens, v0)
        flags = O.stats_arrays(st, n)["flags"]
        keep = np.nonzero((flags & O.F_UNSAFE_MASK) == 0)[0]
        open(os.path.join(INP, name + ".gfa"), "wb").write(text)
        rr = [cat[offs[i]:offs[i] + lens[i]].tobytes() for i in keep]
        write_fasta(os.path.join(INP, name + ".fa"), rr)
        np.savetxt(os.path.join(INP, name + ".v0.txt"), v0[keep], fmt="%d")
        manifest[name] = {"workload": SYNTH[name][0], "n": n, "kept": keep.tolist()}
    json.dump(manifest, open(mpath, "w"))
    print("prepared", {k: len(manifest[k]["kept"]) for k in SETS})


def prepare_exposed(G, O, gwf_test):
    shutil.copy(os.path.join(REF, "exposed_testing/1000_reads/graph_1000.gfa"), GOLD)
    shutil.copy(os.path.join(REF, "exposed_testing/generated/grafo_test.gfa"), GOLD)
    reads = read_fasta(os.path.join(REF, "exposed_testing/1000_reads/reads_1000.fa"), limit=200)
    write_fasta(os.path.join(GOLD, "reads_200.fa"), reads)
    for name in ("graph_1000", "grafo_test"):
        dump = subprocess.run([gwf_test, "-p", os.path.join(GOLD, name + ".gfa")], capture_output=True).stdout
        open(os.path.join(GOLD, name + ".ref_dump.txt"), "wb").write(dump)
    # exposed reads: all start at the first segment (gwf-test's default v0)
    g = G.Graph.from_gfa(os.path.join(GOLD, "graph_1000.gfa"))
    og = O.OracleGraph.from_graph(g)
    cat, offs, lens = G.pack_reads(reads)
    d, st, _ = og.ed_batch(cat, offs, lens, 0)
    flags = O.stats_arrays(st, len(lens))["flags"]
    assert not (flags & O.F_UNSAFE_MASK).any(), "exposed reads unsafe for the reference"


def run():
    os.makedirs(OUT, exist_ok=True)
    R = os.path.join(ROOT, "oracle", "_ref")
    if SETS == list(SYNTH):
        res = subprocess.run([os.path.join(R, "gwf-test"), os.path.join(GOLD, "graph_1000.gfa"),
                              os.path.join(GOLD, "reads_200.fa")], capture_output=True, text=True, timeout=600)
        if res.returncode != 0:
            raise SystemExit("gwf-test failed: " + res.stderr[-2000:])
        open(os.path.join(OUT, "exposed_gwf_test.txt"), "w").write(res.stdout)
    for name in SETS:
        res = subprocess.run([os.path.join(R, "gwf-ref-harness"), os.path.join(INP, name + ".gfa"),
                              os.path.join(INP, name + ".fa"), os.path.join(INP, name + ".v0.txt")],
                             capture_output=True, text=True, timeout=900)
        if res.returncode != 0:
            raise SystemExit(name + " harness failed: " + res.stderr[-2000:])
        open(os.path.join(OUT, name + ".txt"), "w").write(res.stdout)
        open(os.path.join(OUT, name + ".timing.json"), "w").write(res.stderr.strip().splitlines()[-1])
    print("ran reference on", SETS)


def collect():
    if SETS == list(SYNTH):
        # gwf-test prints a header, one distance per read, then a timing line (main.cu:470, 747-750)
        lines = open(os.path.join(OUT, "exposed_gwf_test.txt")).read().split("\n")
        vals = [int(x) for x in lines if x.strip().lstrip("-").isdigit()]
        with open(os.path.join(GOLD, "ref_exposed_200.txt"), "w") as f:
            f.write("# reference gwf-test (sm_100a build of the reference sources) on graph_1000.gfa + reads_200.fa\n")
            f.write("\n".join(str(v) for v in vals) + "\n")
    man = json.load(open(os.path.join(INP, "manifest.json")))
    for name in SETS:
        vals = [int(x) for x in open(os.path.join(OUT, name + ".txt")).read().split()]
        kept = man[name]["kept"]
        assert len(vals) == len(kept)
        with open(os.path.join(GOLD, "ref_%s.txt" % name), "w") as f:
            src = ("overlap_graph.py %s links, %d reads" % (man[name]["workload"], man[name]["n"])
                   if name.startswith("overlap_") else "load_workload(%r, n=%d)" % (man[name]["workload"], man[name]["n"]))
            f.write("# reference gwf_ed (gwf-ed.cu via oracle/_ref/gwf-ref-harness) on %s;"
                    " columns: read index, distance\n" % src)
            for i, v in zip(kept, vals):
                f.write("%d %d\n" % (i, v))
    print("collected")


if __name__ == "__main__":
    rest = sys.argv[2:]
    if sys.argv[1] in ("run", "collect"):
        OUT = os.path.abspath(rest[0])
        rest = rest[1:]
    if rest:
        assert all(r in SYNTH for r in rest), rest
        SETS = rest
    {"prepare": prepare, "run": run, "collect": collect}[sys.argv[1]]()
