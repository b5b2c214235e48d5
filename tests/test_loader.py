"""GFA loader parity: the product loader's gwf_graph_print dump equals the reference
`gwf-test -p` output (tests/golden/*.ref_dump.txt, from the reference binary)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLD


@pytest.mark.parametrize("name", ["graph_1000", "grafo_test"])
def test_dump_matches_reference(G, name):
    g = G.Graph.from_gfa(os.path.join(GOLD, name + ".gfa"))
    ref = open(os.path.join(GOLD, name + ".ref_dump.txt"), "rb").read()
    assert g.dump() == ref


def test_in_memory_load_equals_file_load(G):
    text = open(os.path.join(GOLD, "graph_1000.gfa"), "rb").read()
    a = G.Graph.from_gfa_text(text).dump()
    b = G.Graph.from_gfa(os.path.join(GOLD, "graph_1000.gfa")).dump()
    assert a == b


def test_synthetic_graph_is_topologically_ordered(G):
    sg = G.SynthGraph(20_000, 100, 0.7, 10, 5000, 1000, 2000, seed=7)
    g = G.Graph.from_gfa_text(sg.gfa)
    assert g.n_vtx == G.lib().gwf_synth_graph_nseg(sg.ptr)
    for v, w, o in g.arcs():
        assert v < w and o == 0
    assert sum(len(s) for s in g.seqs()) == int(g.lens().sum())


def test_start_segment_and_orientation(G):
    gfa = b"S\ta\tAAAC\nS\tb\tGGT\nS\tc\tTTA\nL\ta\t+\tb\t+\t0M\nL\tb\t+\tc\t-\t0M\n"
    g = G.Graph.from_gfa_text(gfa, start_seg="b")
    # b first, then c on its reverse strand (reverse complement, main.cu:320-326)
    assert g.seqs() == [b"GGT", b"TAA"]
    assert g.arcs() == [(0, 1, 0)]
    with pytest.raises(G.GwfError):
        G.Graph.from_gfa_text(gfa, start_seg="zz")
    # a strand suffix picks the start strand: "b+" is the default, "c+" walks c+ -> b- -> a-
    assert G.Graph.from_gfa_text(gfa, start_seg="b+").seqs() == g.seqs()
    gc = G.Graph.from_gfa_text(gfa, start_seg="c+")
    assert gc.seqs() == [b"TTA", b"ACC", b"GTTT"] and gc.arcs() == [(0, 1, 0), (1, 2, 0)]
    gb = G.Graph.from_gfa_text(gfa, start_seg="b-")
    assert gb.seqs() == [b"ACC", b"GTTT"] and gb.arcs() == [(0, 1, 0)]
    assert G.Graph.from_gfa_text(gfa, start_seg="c-").seqs() == [b"TAA"]
    with pytest.raises(G.GwfError):
        G.Graph.from_gfa_text(gfa, start_seg="zz-")


def test_overlap_cigar_and_missing_overlap(G):
    gfa = b"S\ta\tAAACG\nS\tb\tCGTTT\nS\tc\tGG\nL\ta\t+\tb\t+\t2M\nL\tb\t+\tc\t+\n"
    g = G.Graph.from_gfa_text(gfa)
    assert (0, 1, 2) in g.arcs() and (1, 2, 0) in g.arcs()


def test_fasta_as_graph(G):
    g = G.Graph.from_gfa_text(b">x desc\nACGT\nAC\n>y\nTT\n")
    assert g.n_vtx == 1 and g.seqs() == [b"ACGTAC"]


def test_truncated_dump_returns_full_length(G):
    g = G.Graph.from_gfa(os.path.join(GOLD, "graph_1000.gfa"))
    full = g.dump()
    buf = ctypes.create_string_buffer(100)
    n = G.lib().gwf_graph_dump(g.ptr, buf, 100)
    assert n == len(full) and buf.raw[:100] == full[:100]


REF_GWF_TEST = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "gwf-test")


def _random_gfa(rng):
    """Names of 1-24 characters, redefined segments, LN tags, lower case and N, links on both
    strands with 0M / * / short M overlaps, links to segments that are never defined. (The
    reference crashes on '*' sequences, so none are generated here.)"""
    n = int(rng.integers(2, 60))
    names = []
    while len(names) < n:
        k = int(rng.integers(1, 25))
        nm = "".join(rng.choice(list("abcxyz0123456789_"), size=k))
        if nm not in names:
            names.append(nm)
    lines, lens = [], {}
    order = list(rng.permutation(n))
    for i in order + list(rng.choice(n, size=int(rng.integers(0, 4)))):
        L = int(rng.integers(1, 40))
        seq = "".join(rng.choice(list("ACGTACGTACGTacgtN"), size=L))
        lines.append("S\t%s\t%s" % (names[i], seq) + ("\tLN:i:%d" % L if rng.random() < 0.3 else ""))
        lens[names[i]] = L
    ghosts = ["ghost%d" % j for j in range(int(rng.integers(1, 3)))] if rng.random() < 0.2 else []
    for _ in range(int(rng.integers(n, 3 * n))):
        if rng.random() < 0.7:  # mostly forward along the S-line order: large reachable parts
            x = int(rng.integers(n - 1))
            a, b = names[order[x]], names[order[x + 1 + int(rng.integers(min(3, n - 1 - x)))]]
        else:
            a, b = names[int(rng.integers(n))], names[int(rng.integers(n))]
        if ghosts and rng.random() < 0.05:
            a = ghosts[0]
        r = rng.random()
        if r < 0.7:
            ov = "0M"
        elif r < 0.85:
            ov = "*"
        else:
            m = min(lens.get(a, 1), lens.get(b, 1))
            ov = "%dM" % int(rng.integers(0, m + 1))
        lines.append("L\t%s\t%s\t%s\t%s\t%s" % (a, "+-"[rng.random() < 0.3], b, "+-"[rng.random() < 0.3], ov))
    return ("\n".join(lines) + "\n").encode()


@pytest.mark.skipif(not os.path.exists(REF_GWF_TEST), reason="reference gwf-test not built")
@pytest.mark.parametrize("threads", ["1", "3"])
def test_random_gfa_dumps_match_reference_binary(G, tmp_path, monkeypatch, threads):
    """Random GFA texts through the reference's own loader (gwf-test -p, built from its sources) and
    through the product loader, parsing on one thread and on three: identical dumps."""
    monkeypatch.setenv("GWF_GFA_THREADS", threads)
    rng = np.random.default_rng(99)
    checked = 0
    for t in range(60):
        text = _random_gfa(rng)
        path = tmp_path / ("g%d.gfa" % t)
        path.write_bytes(text)
        ref = subprocess.run([REF_GWF_TEST, "-p", str(path)], capture_output=True, timeout=60)
        if ref.returncode != 0:
            # the reference crashes on links to undefined segments, and on subgraphs whose arc
            # count changes between its traversal and its extraction (main.cu:338 assertion)
            assert b"not defined on an S-line" in ref.stderr or b"unusual bubble chain" in ref.stderr
            continue
        if b"unusual bubble chain" in ref.stderr:
            continue  # fewer arcs extracted than counted: the reference dumps uninitialised arcs
        assert G.Graph.from_gfa(str(path)).dump() == ref.stdout, text.decode()
        checked += ref.stdout.count(b"S\t") > 3
    assert checked > 30


@pytest.mark.skipif(not os.path.exists(REF_GWF_TEST), reason="reference gwf-test not built")
def test_large_graph_parallel_parse_matches_reference(G, tmp_path, monkeypatch):
    """A 2 Mbp graph (~100,000 segments): the parallel parse, the sequential parse and the
    reference's gwf-test -p give the same dump."""
    sg = G.SynthGraph(2_000_000, 50, 0.7, 20, 50_000, 1000, 5000, seed=9)
    path = tmp_path / "g.gfa"
    path.write_bytes(sg.gfa)
    ref = subprocess.run([REF_GWF_TEST, "-p", str(path)], capture_output=True, timeout=120).stdout
    monkeypatch.setenv("GWF_GFA_THREADS", "8")
    par = G.Graph.from_gfa(str(path)).dump()
    monkeypatch.setenv("GWF_GFA_THREADS", "1")
    seq = G.Graph.from_gfa(str(path)).dump()
    assert par == seq == ref and ref.count(b"\nS\t") > 50_000


def test_gzip_input_equals_plain(G, tmp_path):
    import gzip
    src = os.path.join(GOLD, "graph_1000.gfa")
    gz = tmp_path / "g.gfa.gz"
    with gzip.open(gz, "wb") as f:
        f.write(open(src, "rb").read())
    assert G.Graph.from_gfa(str(gz)).dump() == G.Graph.from_gfa(src).dump()


def test_segment_without_sequence_becomes_n(G):
    """An S line with '*' and an LN tag: the reference's conversion reads a null sequence there
    (it crashes); this loader spells the segment as N bases and records an error message."""
    text = b"S\ta\tACGT\nS\tb\t*\tLN:i:5\nS\tc\tGG\nL\ta\t+\tb\t+\t0M\nL\tb\t+\tc\t+\t0M\n"
    g = G.Graph.from_gfa_text(text)
    assert g.seqs() == [b"ACGT", b"NNNNN", b"GG"]
    assert "without a sequence" in G.last_error()
