"""The oracle (CPU restatement of gwf-ed.cu) against the independent DP and against the
reference's own outputs (tests/golden/ref_*.txt, produced by the reference CUDA code)."""
import os

import numpy as np
import pytest

from conftest import GOLD, read_fasta, read_golden
from randgraph import cases


def test_oracle_exact_start_equals_dp(O):
    """With the start-state quirk disabled and v1 = -1, the restated GWFA is the exact
    sequence-to-graph edit distance (cycles, N bytes, 1-base vertices included)."""
    n = 0
    for seqs, arcs, v0, v1, q in cases(101, 600):
        g = O.OracleGraph(seqs, arcs)
        d, st = g.ed(q, v0, -1, exact_start=True)
        assert d == g.dp(q, v0, -1), (seqs, arcs, v0, q)
        n += 1
    assert n == 600


def test_oracle_uniform_overlaps_equal_dp(O):
    """Arcs entering their targets at a non-zero offset (GFA "nM" links), the same offset for
    every arc into a vertex: the reference's arrival key (vertex, query position) names one graph
    position, the library's entry-keyed rule gives the same result, and both equal the DP."""
    for seqs, arcs, v0, v1, q in cases(111, 600, overlap="uniform"):
        g = O.OracleGraph(seqs, arcs)
        d, _ = g.ed(q, v0, -1, exact_start=True)
        de, _ = g.ed(q, v0, -1, exact_start=True, entry_key=True)
        assert d == de == g.dp(q, v0, -1), (seqs, arcs, v0, q)
        for v1_ in (v1, -1):  # also with the reference's start state and with targets
            assert g.ed(q, v0, v1_)[0] == g.ed(q, v0, v1_, entry_key=True)[0]


def test_oracle_mixed_overlaps_entry_key_is_exact(O):
    """Arcs into one vertex with different overlaps: the reference keys arrivals by (vertex,
    query position), so an arrival through one arc can hide one through another that enters at a
    different offset, and its result depends on its FIFO order (gwf-ed.cu:1196, 1106-1255). The
    entry-keyed rule the library uses equals the DP; the reference's result is never below it."""
    n_worse = 0
    for seqs, arcs, v0, v1, q in cases(112, 1500, overlap="mixed"):
        g = O.OracleGraph(seqs, arcs)
        d, st = g.ed(q, v0, -1, exact_start=True)
        de, _ = g.ed(q, v0, -1, exact_start=True, entry_key=True)
        assert de == g.dp(q, v0, -1), (seqs, arcs, v0, q)
        assert d >= de
        n_worse += d > de
    assert n_worse > 0  # the inputs do reach the order-dependent case


@pytest.mark.parametrize("kind,seeds", [("uniform", (5, 6)), ("mixed", (7, 8))])
def test_oracle_matches_reference_on_overlap_links(G, O, kind, seeds):
    """GFA links with overlaps ("L a + b + nM", tests/golden/overlap_graph.py) through the
    product loader: the restatement equals the reference's own CUDA routine on every read it was
    given (tests/golden/ref_overlap_*.txt), also where the links into a segment differ."""
    import sys
    sys.path.insert(0, GOLD)
    from overlap_graph import overlap_gfa, overlap_reads
    idx, ref = read_golden("ref_overlap_%s.txt" % kind)
    text, seqs, links = overlap_gfa(seeds[0], mode=kind)
    g = G.Graph.from_gfa_text(text)
    seg2v = g.vertex_of_segment()
    reads, starts = overlap_reads(seeds[1], seqs, links, 300)
    cat, offs, lens = G.pack_reads(reads)
    v0 = np.array([seg2v[v] for v in starts], dtype=np.int32)
    og = O.OracleGraph.from_graph(g)
    d, _, _ = og.ed_batch(cat, offs, lens, v0, stats=False)
    assert list(d[np.array(idx)]) == ref
    e, _, _ = og.ed_batch(cat, offs, lens, v0, stats=False, entry_key=True)
    assert (e <= d).all()
    if kind == "uniform":
        assert np.array_equal(e, d)
    assert any(o > 0 for _, _, o in g.arcs())


def test_oracle_quirk_adds_cost_on_short_start_vertex(O):
    """gwf-ed.cu:809,833: k=-1 against an unsigned max_k: a start vertex shorter than 32 bases
    does not extend at s=0, so a perfect match costs 1."""
    g = O.OracleGraph([b"ACG", b"TTTTACGATCGATCGATCGGATCGATCGATCGA"], [(0, 1, 0)])
    q = b"ACGTTTTACGATCG"
    assert g.dp(q, 0) == 0
    assert g.ed(q, 0, exact_start=True)[0] == 0
    assert g.ed(q, 0, exact_start=False)[0] == 1
    # a long start vertex extends normally
    g2 = O.OracleGraph([b"ACGT" * 10], [])
    assert g2.ed(b"ACGT" * 8, 0)[0] == 0


def test_oracle_target_vertex_is_an_upper_bound(O):
    """v1 >= 0: the reference skips the end-of-vertex insertion when every arc matches
    (gwf-ed.cu:1225), which is exact only for v1 < 0; the result is never below the DP."""
    for seqs, arcs, v0, v1, q in cases(202, 300, v1_prob=1.0):
        g = O.OracleGraph(seqs, arcs)
        d, st = g.ed(q, v0, v1, exact_start=True)
        t = g.dp(q, v0, v1)
        if t < 0:
            assert d < 0 or d >= 0  # unreachable target: both give no or some alignment
        else:
            assert d == -1 or d >= t


def test_oracle_empty_query_flags_nontermination(O):
    g = O.OracleGraph([b"ACGT"], [])
    d, st = g.ed(b"", 0)
    assert st.flags & O.F_NONTERM


def test_oracle_batch_matches_single(O):
    seqs = [b"ACGTACGTAC", b"GGG", b"TTT", b"ACGTAAACCC"]
    arcs = [(0, 1, 0), (0, 2, 0), (1, 3, 0), (2, 3, 0)]
    g = O.OracleGraph(seqs, arcs)
    reads = [b"ACGTACGTACGGGACGTAAACCC", b"ACGTACGTACTTTACGTAAACC", b"ACGAACGTACGGTACGTAAACCC"]
    cat = np.frombuffer(b"".join(reads), np.uint8)
    offs = np.cumsum([0] + [len(r) for r in reads[:-1]])
    lens = np.array([len(r) for r in reads], np.int32)
    d, st, _ = g.ed_batch(cat, offs, lens, 0, threads=2)
    assert list(d) == [g.ed(r, 0)[0] for r in reads]


def test_oracle_matches_reference_on_exposed_reads(G, O):
    """Pins the oracle to the reference's own gwf-test output (all reads start at the first
    segment, main.cu:370)."""
    _, ref = read_golden("ref_exposed_200.txt")
    reads = read_fasta(os.path.join(GOLD, "reads_200.fa"))
    assert len(ref) == len(reads) == 200
    g = G.Graph.from_gfa(os.path.join(GOLD, "graph_1000.gfa"))
    og = O.OracleGraph.from_graph(g)
    cat, offs, lens = G.pack_reads(reads)
    d, st, _ = og.ed_batch(cat, offs, lens, 0)
    assert list(d) == ref


@pytest.mark.parametrize("name", ["config1", "config2", "config3", "config4", "config5"])
def test_oracle_matches_reference_on_synthetic(G, O, name):
    """Pins the oracle to the reference gwf_ed device routine run with per-read v0 (configs 4
    and 5: 10 kbp and up to 20 kbp reads on the 5 Mbp graph, the reads whose arena the
    reference can hold)."""
    idx, ref = read_golden("ref_%s.txt" % name)
    n = {"config1": 1000, "config2": 2000, "config3": 600, "config4": 200, "config5": 100}[name]
    w = G.load_workload(name, n=n)
    og = O.OracleGraph.from_graph(w["graph"])
    sel = np.array(idx)
    d, st, _ = og.ed_batch(w["cat"], w["offs"][sel], w["lens"][sel], w["v0"][sel])
    assert list(d) == ref


def test_lag_pruning_bounds(G, O):
    """The lag pruning that GWF_F_MAX_LAG enables: a lag beyond the read length changes nothing,
    and a smaller lag can only raise the distance (or leave no alignment, -1)."""
    w = G.load_workload("config2", n=300)
    og = O.OracleGraph.from_graph(w["graph"])
    grew = 0
    for i in range(0, 300, 3):
        q = bytes(w["cat"][w["offs"][i]:w["offs"][i] + w["lens"][i]])
        v0 = int(w["v0"][i])
        full, _ = og.ed(q, v0)
        assert og.ed(q, v0, max_lag=len(q) + 1)[0] == full
        for lag in (2, 5, 20, 100):
            d, _ = og.ed(q, v0, max_lag=lag)
            assert d == -1 or d >= full
            grew += d != full
    assert grew > 0  # small lags do prune something on 5-10% error reads
    for seqs, arcs, v0, v1, q in cases(515, 150, v1_prob=0.3):
        og2 = O.OracleGraph(seqs, arcs)
        full, st = og2.ed(q, v0, v1)
        if st.flags & O.F_NONTERM:
            continue
        for lag in (1, 3):
            d, st2 = og2.ed(q, v0, v1, max_lag=lag)
            if not st2.flags & O.F_NONTERM:
                assert d == -1 or full == -1 or d >= full
