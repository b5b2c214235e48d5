"""Several warps per read: the persistent form's read classes, where groups of 2, 4 or 8 warps of
one CTA align one read together (k_align_classes, gwf_group.cuh). Every distance must equal the
one-warp kernel's and the oracle's, bit for bit, on every workload shape and option the one-warp
path supports."""
import numpy as np
import pytest

from randgraph import cases

pytestmark = pytest.mark.gpu

NWS = [2, 4, 8]


@pytest.mark.parametrize("name,n", [("config1", 300), ("config2", 600), ("config3", 300), ("config4", 24),
                                    ("config5", 16)])
def test_groups_equal_one_warp_and_oracle(G, O, name, n):
    w = G.load_workload(name, n=n)
    g = w["graph"]
    g.index()
    reads = (w["cat"], w["offs"], w["lens"])
    d1, s1 = g.ed_batch(reads, w["v0"], mode=G.MODE_PERSISTENT, warps_per_read=1)
    assert (s1 == 0).all()
    od, _, _ = O.OracleGraph.from_graph(g).ed_batch(w["cat"], w["offs"], w["lens"], w["v0"], stats=False)
    assert np.array_equal(d1, od)
    for nw in NWS:
        for use_graph in (0, 1):
            d, s = g.ed_batch(reads, w["v0"], mode=G.MODE_PERSISTENT, warps_per_read=nw, use_graph=use_graph)
            assert (s == 0).all(), (nw, use_graph, np.unique(s))
            assert np.array_equal(d, d1), (nw, use_graph, np.nonzero(d != d1)[0][:10])


@pytest.mark.parametrize("overlap", ["zero", "uniform", "mixed"])
def test_groups_random_graphs(G, O, overlap):
    """Cyclic and acyclic graphs, 1-base vertices, N and lower-case bytes (byte compares), arc
    overlaps, v1 targets, both start-state rules; group sizes in turn."""
    checked = 0
    for t, (seqs, arcs, v0, v1, q) in enumerate(cases(707 + len(overlap), 240, v1_prob=0.25, overlap=overlap)):
        exact = t % 3 == 0
        og = O.OracleGraph(seqs, arcs)
        od, ost = og.ed(q, v0, v1, exact_start=exact, entry_key=True)
        if ost.flags & O.F_NONTERM:
            continue
        g = G.Graph.from_arrays(seqs, arcs)
        g.index()
        nw = NWS[t % 3]
        d, st = g.ed_batch([q], [v0], v1=v1, flags=G.GWF_F_EXACT_START if exact else 0, mode=G.MODE_PERSISTENT,
                           warps_per_read=nw)
        assert st[0] == 0 and d[0] == od, (seqs, arcs, v0, v1, q, nw, d[0], od)
        checked += 1
        g.close()
    assert checked > 200


@pytest.mark.parametrize("lag", [3, 20])
def test_groups_lag_pruning(G, O, lag):
    w = G.load_workload("config3", n=200)
    g = w["graph"]
    g.index()
    og = O.OracleGraph.from_graph(g)
    od = [og.ed(bytes(w["cat"][o:o + l]), int(v), max_lag=lag)[0] for o, l, v in zip(w["offs"], w["lens"], w["v0"])]
    for nw in NWS:
        d, st = g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"], mode=G.MODE_PERSISTENT, flags=G.GWF_F_MAX_LAG,
                           max_lag=lag, warps_per_read=nw)
        assert (st == 0).all() and list(d) == od


def test_groups_retry_overflowing_reads(G):
    """Reads unrelated to the graph overflow their group's arena and are re-run at larger classes;
    the results equal the one-warp form's, and reads of every class share the launch."""
    w = G.load_workload("config3", n=200)
    g = w["graph"]
    g.index()
    rng = np.random.default_rng(9)
    junk = [bytes(rng.choice(list(b"ACGT"), size=int(L)).astype(np.uint8)) for L in (700, 2500, 4000)]
    reads = [bytes(w["cat"][o:o + l]) for o, l in zip(w["offs"], w["lens"])] + junk
    v0 = np.concatenate([w["v0"], np.zeros(len(junk), np.int32)]).astype(np.int32)
    cat, offs, lens = G.pack_reads(reads)
    d1, s1 = g.ed_batch((cat, offs, lens), v0, mode=G.MODE_PERSISTENT, warps_per_read=1)
    for nw in NWS:
        d, s = g.ed_batch((cat, offs, lens), v0, mode=G.MODE_PERSISTENT, warps_per_read=nw)
        assert np.array_equal(s, s1) and np.array_equal(d, d1)


def test_groups_resident_batch_steps(G):
    w = G.load_workload("config3", n=400)
    g = w["graph"]
    g.index()
    b = G.ResidentBatch(g, w["cat"], w["offs"], w["lens"], w["v0"], mode=G.MODE_PERSISTENT)
    b.run(warps_per_read=1)
    d1, _ = b.results()
    s1 = b.steps()
    for nw in NWS:
        ms = b.run(warps_per_read=nw, use_graph=1)
        d, st = b.results()
        assert ms > 0 and (st == 0).all() and np.array_equal(d, d1)
        assert np.array_equal(b.steps(), s1)


def test_groups_option_checked(G):
    w = G.load_workload("config1", n=4)
    g = w["graph"]
    g.index()
    with pytest.raises(G.GwfError):
        g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"], warps_per_read=3)
