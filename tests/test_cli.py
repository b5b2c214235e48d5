"""gwf-b200, the command-line driver with gwf-test's interface (main.cu:360-750): graph dumps
byte-identical to the reference's `gwf-test -p`, and on a GPU the reference's own distances for
its exposed fixture (tolerance 0: int32 distances)."""
import gzip
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLD, PKG_DIR, read_golden

CLI = os.path.join(PKG_DIR, "gwf-b200")


def run(*args, check=True):
    return subprocess.run([CLI, *args], capture_output=True, text=True, check=check, timeout=600)


@pytest.fixture(scope="module", autouse=True)
def built(G):
    G.lib()  # builds the library and the driver when only sources are present
    assert os.access(CLI, os.X_OK)


@pytest.mark.parametrize("name", ["graph_1000", "grafo_test"])
def test_print_graph_equals_reference_dump(name):
    out = run("-p", os.path.join(GOLD, name + ".gfa")).stdout
    assert out == open(os.path.join(GOLD, name + ".ref_dump.txt")).read()


def test_usage_and_bad_arguments():
    assert run(check=False).returncode == 1
    assert run("-m", "nope", "a.gfa", "b.fa", check=False).returncode == 1
    r = run(os.path.join(GOLD, "missing.gfa"), os.path.join(GOLD, "reads_200.fa"), check=False)
    assert r.returncode == 1 and "ERROR" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["persistent", "plain"])
def test_scores_equal_reference_gwf_test(form, tmp_path):
    _, ref = read_golden("ref_exposed_200.txt")
    gfa = os.path.join(GOLD, "graph_1000.gfa")
    reads = os.path.join(GOLD, "reads_200.fa")
    out = run("-m", form, gfa, reads).stdout.split()
    assert np.array_equal(np.array(out, dtype=np.int64), np.asarray(ref))
    # the same reads gzip-compressed, as FASTQ
    fq = tmp_path / "r.fq.gz"
    names, seqs = [], []
    for line in open(reads):
        line = line.strip()
        if line.startswith(">"):
            names.append(line[1:]), seqs.append("")
        elif line:
            seqs[-1] += line
    with gzip.open(fq, "wt") as f:
        for n, s in zip(names, seqs):
            f.write("@%s\n%s\n+\n%s\n" % (n, s, "I" * len(s)))
    out2 = run(gfa, str(fq)).stdout.split()
    assert out2 == out


@pytest.mark.gpu
def test_traceback_option(G):
    """-t: the distance column equals the plain output; each path starts at vertex 0, follows arcs
    of the converted graph, and ends at a valid offset of its last vertex; each CIGAR consumes the
    read and costs at most the distance."""
    gfa = os.path.join(GOLD, "graph_1000.gfa")
    reads = os.path.join(GOLD, "reads_200.fa")
    plain = run(gfa, reads).stdout.split()
    lines = run("-t", gfa, reads).stdout.splitlines()
    reads_seq = [s for s in open(reads).read().split("\n") if s and not s.startswith(">")]
    assert [ln.split("\t")[0] for ln in lines] == plain
    g = G.Graph.from_gfa(gfa)
    g.index()
    arcs = {(v, w) for v, w, _ in g.arcs()}
    lens = g.lens()
    assert len(lines) == len(reads_seq)
    for ln, seq in zip(lines, reads_seq):
        d, eo, path, cigar = ln.split("\t")
        verts = [int(x) for x in path.split(",")]
        assert verts[0] == 0 and all((a, b) in arcs for a, b in zip(verts, verts[1:]))
        assert 0 <= int(eo) < lens[verts[-1]]
        ops = re.findall(r"(\d+)([=XID])", cigar)
        assert "".join(n + o for n, o in ops) == cigar
        assert sum(int(n) for n, o in ops if o in "=XI") == len(seq)
        assert sum(int(n) for n, o in ops if o in "XID") <= int(d)


@pytest.mark.gpu
def test_lag_option(G):
    """-l alone is ignored, as in the reference; -l with -P prunes (distances never below)."""
    gfa = os.path.join(GOLD, "graph_1000.gfa")
    reads = os.path.join(GOLD, "reads_200.fa")
    base = np.array(run(gfa, reads).stdout.split(), dtype=np.int64)
    assert np.array_equal(np.array(run("-l", "3", gfa, reads).stdout.split(), dtype=np.int64), base)
    pruned = np.array(run("-l", "3", "-P", gfa, reads).stdout.split(), dtype=np.int64)
    assert ((pruned >= base) | (pruned == -1)).all()


@pytest.mark.gpu
def test_both_strands_option(tmp_path):
    """-b: the reads as given align on strand + with the plain distances; their reverse
    complements align on strand - at the same distances."""
    gfa = os.path.join(GOLD, "graph_1000.gfa")
    reads = os.path.join(GOLD, "reads_200.fa")
    plain = run(gfa, reads).stdout.split()
    rows = [ln.split("\t") for ln in run("-b", gfa, reads).stdout.splitlines()]
    assert all(s in "+-*" for _, s in rows)
    assert all(int(d) <= int(p) for (d, _), p in zip(rows, plain))
    comp = str.maketrans("ACGTacgt", "TGCAtgca")
    rc = tmp_path / "rc.fa"
    with open(rc, "w") as f:
        seq = None
        for line in open(reads).read().split("\n") + [">"]:
            if line.startswith(">"):
                if seq is not None:
                    f.write(">r\n%s\n" % seq.translate(comp)[::-1])
                seq = ""
            else:
                seq += line.strip()
    rows_rc = [ln.split("\t") for ln in run("-b", gfa, str(rc)).stdout.splitlines()]
    # the same two strands swapped: the same distances; a strand - becomes + (a tie stays +)
    assert [d for d, _ in rows_rc] == [d for d, _ in rows]
    for (_, s), (_, t) in zip(rows, rows_rc):
        assert (s == "*") == (t == "*") and (s != "-" or t == "+")
    assert sum(s == "+" for _, s in rows) > 0.9 * len(rows) and sum(t == "-" for _, t in rows_rc) > 0.8 * len(rows)
    assert run("-b", "-t", gfa, reads, check=False).returncode == 1
