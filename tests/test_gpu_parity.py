"""GPU parity: every int32 distance from the sm_100a kernels equals the oracle (CPU restatement
of gwf-ed.cu) and the reference's own CUDA outputs, bit for bit. All calls go through the C ABI
of libgwfa_b200.so."""
import os
import sys

import numpy as np
import pytest

from conftest import GOLD, read_fasta, read_golden
from randgraph import cases

sys.path.insert(0, GOLD)

pytestmark = pytest.mark.gpu


def _indexed(G, g):
    err = g.index()
    assert g.indexed
    return g


def test_exposed_reads_match_reference(G, O):
    _, ref = read_golden("ref_exposed_200.txt")
    reads = read_fasta(os.path.join(GOLD, "reads_200.fa"))
    g = _indexed(G, G.Graph.from_gfa(os.path.join(GOLD, "graph_1000.gfa")))
    for mode in (G.MODE_PLAIN, G.MODE_PERSISTENT):
        d, st = g.ed_batch(reads, 0, mode=mode)
        assert (st == 0).all()
        assert list(d) == ref


@pytest.mark.parametrize("name,n", [("config1", 1000), ("config2", 2000), ("config3", 600), ("config4", 200),
                                    ("config5", 100)])
def test_synthetic_match_reference_and_oracle(G, O, name, n):
    idx, ref = read_golden("ref_%s.txt" % name)
    w = G.load_workload(name, n=n)
    g = _indexed(G, w["graph"])
    sel = np.array(idx)
    for mode in (G.MODE_PLAIN, G.MODE_PERSISTENT):
        d, st = g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"], mode=mode)
        assert (st == 0).all()
        assert list(d[sel]) == ref
        og = O.OracleGraph.from_graph(w["graph"])
        od, _, _ = og.ed_batch(w["cat"], w["offs"], w["lens"], w["v0"], stats=False)
        assert np.array_equal(d, od)


@pytest.mark.parametrize("exact", [False, True])
def test_random_graphs_match_oracle(G, O, exact):
    """Small DAGs and cyclic graphs, 1-base vertices (start-state quirk), N and lower-case
    bytes (byte-compare path), v1 >= 0 targets."""
    flags = G.GWF_F_EXACT_START if exact else 0
    checked = 0
    for t, (seqs, arcs, v0, v1, q) in enumerate(cases(303 + exact, 250, v1_prob=0.25)):
        g = _indexed(G, G.Graph.from_arrays(seqs, arcs))
        og = O.OracleGraph(seqs, arcs)
        od, ost = og.ed(q, v0, v1, exact_start=exact)
        if ost.flags & O.F_NONTERM:
            continue
        d, st = g.ed_batch([q], [v0], v1=v1, flags=flags, mode=G.MODE_PLAIN if t % 2 else G.MODE_PERSISTENT)
        assert st[0] == 0 and d[0] == od, (seqs, arcs, v0, v1, q, d[0], od)
        if exact and v1 < 0:
            assert d[0] == og.dp(q, v0, v1)
        checked += 1
        g.close()
    assert checked > 200


@pytest.mark.parametrize("exact", [False, True])
@pytest.mark.parametrize("overlap", ["uniform", "mixed"])
def test_random_graphs_with_overlaps(G, O, overlap, exact):
    """Arcs that enter their target at a non-zero offset (GFA "nM" links): cyclic and acyclic
    graphs, v1 targets, both forms. With one overlap per target (uniform) the kernels equal the
    reference restatement; with different overlaps into one vertex (mixed) they equal the
    oracle under the library's entry-keyed arrival rule, which is the DP's exact distance and
    never above the reference's queue-order-dependent result."""
    flags = G.GWF_F_EXACT_START if exact else 0
    checked = 0
    seed = 404 + 2 * (overlap == "mixed") + exact
    for t, (seqs, arcs, v0, v1, q) in enumerate(cases(seed, 250, v1_prob=0.25, overlap=overlap)):
        og = O.OracleGraph(seqs, arcs)
        od, ost = og.ed(q, v0, v1, exact_start=exact, entry_key=True)
        rd, rst = og.ed(q, v0, v1, exact_start=exact)
        if (ost.flags | rst.flags) & O.F_NONTERM:
            continue
        g = _indexed(G, G.Graph.from_arrays(seqs, arcs))
        d, st = g.ed_batch([q], [v0], v1=v1, flags=flags, mode=G.MODE_PLAIN if t % 2 else G.MODE_PERSISTENT)
        assert st[0] == 0 and d[0] == od, (seqs, arcs, v0, v1, q, d[0], od)
        if overlap == "uniform":
            assert d[0] == rd
        if exact and v1 < 0:
            assert d[0] == og.dp(q, v0, v1) and d[0] <= rd
        checked += 1
        g.close()
    assert checked > 200


def _overlap_set(G, kind, n=300):
    """The overlap golden sets of tests/golden/make_golden.py: GFA links "L a + b + nM"."""
    from overlap_graph import overlap_gfa, overlap_reads
    text, seqs, links = overlap_gfa(5 if kind == "uniform" else 7, mode=kind)
    g = G.Graph.from_gfa_text(text)
    seg2v = g.vertex_of_segment()
    reads, starts = overlap_reads(6 if kind == "uniform" else 8, seqs, links, n)
    cat, offs, lens = G.pack_reads(reads)
    return g, (cat, offs, lens), np.array([seg2v[v] for v in starts], dtype=np.int32)


@pytest.mark.parametrize("kind", ["uniform", "mixed"])
def test_overlap_links_match_reference(G, O, kind):
    """GFA links with overlaps, through the loader: with one overlap per target segment the
    kernels equal the reference's own CUDA routine (golden) and its restatement, in both forms
    and with groups of warps; with mixed overlaps they equal the entry-keyed rule, never above
    the reference, whose own results equal the restatement of its queue order."""
    idx, ref = read_golden("ref_overlap_%s.txt" % kind)
    g, reads, v0 = _overlap_set(G, kind)
    _indexed(G, g)
    og = O.OracleGraph.from_graph(g)
    cat, offs, lens = reads
    fifo, _, _ = og.ed_batch(cat, offs, lens, v0, stats=False)
    entry, _, _ = og.ed_batch(cat, offs, lens, v0, stats=False, entry_key=True)
    sel = np.array(idx)
    assert list(fifo[sel]) == ref  # the restatement of the reference, pinned by the reference
    for mode, nw in ((G.MODE_PLAIN, 0), (G.MODE_PERSISTENT, 1), (G.MODE_PERSISTENT, 4)):
        d, st = g.ed_batch(reads, v0, mode=mode, warps_per_read=nw)
        assert (st == 0).all() and np.array_equal(d, entry)
        if kind == "uniform":
            assert list(d[sel]) == ref
        else:
            assert (d[sel] <= np.array(ref)).all()


def test_lag_pruning_random_graphs_with_overlaps(G, O):
    checked = 0
    for t, (seqs, arcs, v0, v1, q) in enumerate(cases(921, 150, v1_prob=0.3, overlap="uniform")):
        lag = 1 + t % 4
        og = O.OracleGraph(seqs, arcs)
        od, ost = og.ed(q, v0, v1, max_lag=lag)
        if ost.flags & O.F_NONTERM:
            continue
        g = _indexed(G, G.Graph.from_arrays(seqs, arcs))
        d, st = g.ed_batch([q], [v0], v1=v1, flags=G.GWF_F_MAX_LAG, max_lag=lag)
        assert st[0] == 0 and d[0] == od, (seqs, arcs, v0, v1, q, lag, d[0], od)
        checked += 1
        g.close()
    assert checked > 100


def test_single_read_entry_point(G, O):
    w = G.load_workload("config1", n=20)
    g = _indexed(G, w["graph"])
    og = O.OracleGraph.from_graph(w["graph"])
    for i in range(20):
        q = w["cat"][w["offs"][i]:w["offs"][i] + w["lens"][i]].tobytes()
        assert g.ed(q, int(w["v0"][i])) == og.ed(q, int(w["v0"][i]))[0]
    # max_lag is accepted and ignored, as in the reference; traceback is not implemented
    q = w["cat"][:w["lens"][0]].tobytes()
    assert g.ed(q, int(w["v0"][0]), max_lag=7) == og.ed(q, int(w["v0"][0]))[0]
    with pytest.raises(G.GwfError):
        g.ed(q, int(w["v0"][0]), traceback=1)


def test_pointer_array_batch_equals_concat(G):
    w = G.load_workload("config1", n=64)
    g = _indexed(G, w["graph"])
    a, _ = g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"], concat=True)
    b, _ = g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"], concat=False)
    assert np.array_equal(a, b)


def test_edge_cases(G, O):
    seqs, arcs = [b"ACGTACGT", b"TTTT"], [(0, 1, 0)]
    g = _indexed(G, G.Graph.from_arrays(seqs, arcs))
    og = O.OracleGraph(seqs, arcs)
    d, st = g.ed_batch([b"", b"ACGT", b"N", b"ACGTACGTTTTTGGGG"], [0, 5, 0, 0])
    assert st[0] == G.GWF_E_BAD_INPUT and st[1] == G.GWF_E_BAD_INPUT
    assert st[2] == 0 and st[3] == 0
    # the 8-base start vertex does not extend at score 0 (reference start-state rule): +1
    assert d[3] == og.ed(b"ACGTACGTTTTTGGGG", 0)[0] == og.dp(b"ACGTACGTTTTTGGGG", 0) + 1 == 5
    d, st = g.ed_batch([b"ACGTACGTTTTTGGGG"], [0], flags=G.GWF_F_EXACT_START)
    assert d[0] == 4
    d, st = g.ed_batch([], [], mode=G.MODE_PERSISTENT)
    assert len(d) == 0
    # a read that can only be aligned with insertions past the graph end
    q = b"ACGTACGTTTTT" + b"C" * 30
    d, st = g.ed_batch([q], [0], flags=G.GWF_F_EXACT_START)
    assert st[0] == 0 and d[0] == 30 == og.dp(q, 0)


def test_long_reads_dense_graph_and_retries(G, O):
    """10 kbp reads on the 5 Mbp dense graph (config 4 shapes): large wavefronts, arrival sets
    of ~10^5 keys; reads whose arena overflows are re-run at a larger class."""
    w = G.load_workload("config4", n=24)
    g = _indexed(G, w["graph"])
    d, st = g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"])
    assert (st == 0).all()
    og = O.OracleGraph.from_graph(w["graph"])
    od, _, _ = og.ed_batch(w["cat"], w["offs"], w["lens"], w["v0"], stats=False)
    assert np.array_equal(d, od)


def test_serving_reads_match_oracle(G, O):
    """Config 5 shapes (reads of U[500, 20000] bp at U[1%, 10%] on the 5 Mbp graph), the longest
    the benchmarks use, through both batch forms, against the oracle."""
    w = G.load_workload("config5", n=16)
    g = _indexed(G, w["graph"])
    og = O.OracleGraph.from_graph(w["graph"])
    od, _, _ = og.ed_batch(w["cat"], w["offs"], w["lens"], w["v0"], stats=False)
    for mode in (G.MODE_PERSISTENT, G.MODE_PLAIN):
        d, st = g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"], mode=mode)
        assert (st == 0).all()
        assert np.array_equal(d, od)


def test_resident_batch_runs_are_repeatable(G):
    w = G.load_workload("config1", n=500)
    g = _indexed(G, w["graph"])
    b = G.ResidentBatch(g, w["cat"], w["offs"], w["lens"], w["v0"])
    ms = b.run()
    d1, _ = b.results()
    b.run(mode=G.MODE_PLAIN)
    d2, _ = b.results()
    assert ms > 0 and np.array_equal(d1, d2)
    assert b.launches() >= 2
    assert (b.steps() == d1 + 1).all()


def test_graph_captured_runs_equal_stream_runs(G):
    """use_graph = 1: the level-0 sequence (pack, persistent kernel, overflow count) replays as one
    CUDA graph; results equal the stream-launched run, across replays and with arena retries
    (reads unrelated to the graph overflow the first arena class)."""
    w = G.load_workload("config1", n=300)
    g = _indexed(G, w["graph"])
    rng = np.random.default_rng(4)
    junk = [bytes(rng.choice(list(b"ACGT"), size=600).astype(np.uint8)) for _ in range(4)]
    reads = [bytes(w["cat"][o:o + l]) for o, l in zip(w["offs"], w["lens"])] + junk
    v0 = np.concatenate([w["v0"], np.zeros(len(junk), np.int32)]).astype(np.int32)
    cat, offs, lens = G.pack_reads(reads)
    b = G.ResidentBatch(g, cat, offs, lens, v0)
    b.run(use_graph=0)
    d0, s0 = b.results()
    for _ in range(3):
        b.run(use_graph=1)
        d1, s1 = b.results()
        assert np.array_equal(d0, d1) and np.array_equal(s0, s1)
    d2, s2 = g.ed_batch((cat, offs, lens), v0, use_graph=1)
    assert np.array_equal(d0, d2) and np.array_equal(s0, s2)
    b.close()


@pytest.mark.parametrize("lag", [2, 5, 20])
def test_lag_pruning_matches_oracle(G, O, lag):
    """GWF_F_MAX_LAG: the kernels' pruned distances equal the oracle's with the same rule, in both
    forms and through the captured CUDA graph; without the flag max_lag stays ignored."""
    w = G.load_workload("config2", n=1000)
    g = _indexed(G, w["graph"])
    og = O.OracleGraph.from_graph(w["graph"])
    reads = (w["cat"], w["offs"], w["lens"])
    od = [og.ed(bytes(w["cat"][o:o + l]), int(v), max_lag=lag)[0] for o, l, v in zip(w["offs"], w["lens"], w["v0"])]
    for mode, use_graph in ((G.MODE_PLAIN, 0), (G.MODE_PERSISTENT, 0), (G.MODE_PERSISTENT, 1)):
        d, st = g.ed_batch(reads, w["v0"], mode=mode, flags=G.GWF_F_MAX_LAG, max_lag=lag, use_graph=use_graph)
        assert (st == 0).all() and list(d) == od
    full, _ = g.ed_batch(reads, w["v0"], max_lag=lag)  # flag off: ignored, as in the reference
    d0, _ = g.ed_batch(reads, w["v0"])
    assert np.array_equal(full, d0)


def test_lag_pruning_random_graphs(G, O):
    checked = 0
    for t, (seqs, arcs, v0, v1, q) in enumerate(cases(919, 200, v1_prob=0.3)):
        lag = 1 + t % 4
        og = O.OracleGraph(seqs, arcs)
        od, ost = og.ed(q, v0, v1, max_lag=lag)
        if ost.flags & O.F_NONTERM:
            continue
        g = _indexed(G, G.Graph.from_arrays(seqs, arcs))
        d, st = g.ed_batch([q], [v0], v1=v1, flags=G.GWF_F_MAX_LAG, max_lag=lag)
        assert st[0] == 0 and d[0] == od, (seqs, arcs, v0, v1, q, lag, d[0], od)
        checked += 1
        g.close()
    assert checked > 150
