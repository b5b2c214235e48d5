"""Both-strand alignment (GWF_F_BOTH_STRANDS, gwf_ed_batch_strand): each read and its reverse
complement are aligned from the same v0 in one launch; the read keeps the smaller distance and
the strand that gave it. Checked against the oracle run on both strands."""
import numpy as np
import pytest

from randgraph import cases

pytestmark = pytest.mark.gpu

COMP = bytes.maketrans(b"ACGTacgtRYKMBVDHrykmbvdhUu", b"TGCAtgcaYRMKVBHDyrmkbvhdAa")


def revcomp(q):
    return bytes(q).translate(COMP)[::-1]


def oracle_both(og, q, v0, v1=-1, exact=False):
    df, sf = og.ed(q, v0, v1, exact_start=exact, entry_key=True)
    dr, sr = og.ed(revcomp(q), v0, v1, exact_start=exact, entry_key=True)
    if df >= 0 and (dr < 0 or df <= dr):
        return df, 0, (sf.flags | sr.flags)
    if dr >= 0:
        return dr, 1, (sf.flags | sr.flags)
    return -1, -1, (sf.flags | sr.flags)


def test_both_strands_config_reads(G, O):
    """Half the reads are given reverse-complemented: they align as the reverse complement
    (strand 1) at the distance of the original read."""
    w = G.load_workload("config3", n=400)
    g = w["graph"]
    g.index()
    reads = [bytes(w["cat"][o:o + l]) for o, l in zip(w["offs"], w["lens"])]
    flip = np.arange(len(reads)) % 2 == 1
    given = [revcomp(r) if f else r for r, f in zip(reads, flip)]
    d_fwd, _ = g.ed_batch(reads, w["v0"], mode=G.MODE_PERSISTENT)
    og = O.OracleGraph.from_graph(g)
    exp = [oracle_both(og, q, int(v)) for q, v in zip(given, w["v0"])]
    for mode, nw in ((G.MODE_PERSISTENT, 0), (G.MODE_PERSISTENT, 4), (G.MODE_PLAIN, 0)):
        d, st, strand = g.ed_strand(given, w["v0"], mode=mode, warps_per_read=nw)
        assert (st == 0).all()
        assert list(d) == [e[0] for e in exp] and list(strand) == [e[1] for e in exp]
        assert (d <= d_fwd).all()
        assert (strand[flip] == 1).mean() > 0.95
    # the flag on the plain batch call gives the same distances
    d2, _ = g.ed_batch(given, w["v0"], flags=G.GWF_F_BOTH_STRANDS)
    assert list(d2) == [e[0] for e in exp]


def test_both_strands_random_graphs(G, O):
    """IUPAC, N and lower-case bytes (the complement table), cycles, overlaps, v1 targets."""
    checked = 0
    for t, (seqs, arcs, v0, v1, q) in enumerate(cases(1313, 150, v1_prob=0.25, overlap="uniform")):
        exact = t % 2 == 0
        og = O.OracleGraph(seqs, arcs)
        ed, es, fl = oracle_both(og, q, v0, v1, exact)
        if fl & O.F_NONTERM:
            continue
        g = G.Graph.from_arrays(seqs, arcs)
        g.index()
        d, st, strand = g.ed_strand([q], [v0], v1=v1, flags=G.GWF_F_EXACT_START if exact else 0)
        assert st[0] == 0 and (d[0], strand[0]) == (ed, es), (seqs, arcs, v0, v1, q, d[0], strand[0], ed, es)
        checked += 1
        g.close()
    assert checked > 120


def test_both_strands_resident_batch(G, O):
    w = G.load_workload("config1", n=100)
    g = w["graph"]
    g.index()
    b = G.ResidentBatch(g, w["cat"], w["offs"], w["lens"], w["v0"], mode=G.MODE_PERSISTENT,
                        flags=G.GWF_F_BOTH_STRANDS)
    b.run(use_graph=1)
    d, st = b.results()
    e, _, _ = g.ed_strand((w["cat"], w["offs"], w["lens"]), w["v0"])
    assert (st == 0).all() and np.array_equal(d, e)
    assert len(b.steps()) == 100
    b.close()


def test_both_strands_serving(G):
    """A both-strand server: each read's reverse complement is queued as a read of its own; the
    request's results equal the batch call's, distance and strand."""
    w = G.load_workload("config3", n=90)
    g = w["graph"]
    g.index()
    reads = [bytes(w["cat"][o:o + l]) for o, l in zip(w["offs"], w["lens"])]
    given = [revcomp(r) if i % 3 == 0 else r for i, r in enumerate(reads)]
    e_d, e_s, e_k = g.ed_strand(given, w["v0"])
    srv = G.Server(g, arena_budget_bytes=1 << 30, flags=G.GWF_F_BOTH_STRANDS)
    try:
        ids = [srv.submit(given[a:a + 30], w["v0"][a:a + 30]) for a in (0, 30, 60)]
        for a, (rid, k) in zip((0, 30, 60), ids):
            d, st = srv.wait(rid, k, timeout_s=120)
            assert (st == 0).all() and np.array_equal(d, e_d[a:a + 30])
            assert np.array_equal(srv.strand(rid, k), e_k[a:a + 30])
    finally:
        srv.close()
