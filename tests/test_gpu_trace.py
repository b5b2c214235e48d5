"""Traceback (gwf_ed_batch_path): the distances equal the distance-only kernels', and every
returned path is checked on the CPU: its arcs exist, and the read aligned end to end against the
text the path spells costs at most the distance (exactly the distance, which is then the graph
optimum, with GWF_F_EXACT_START and v1 = -1)."""
import numpy as np
import pytest

from randgraph import cases

pytestmark = pytest.mark.gpu


def edit_distance(q, t):
    """Global edit distance (unit costs) of byte strings q and t, row by row."""
    a = np.frombuffer(q, dtype=np.uint8)
    b = np.frombuffer(t, dtype=np.uint8)
    ar = np.arange(len(b) + 1, dtype=np.int64)
    row = ar.copy()
    for i in range(len(a)):
        cand = np.empty_like(row)
        cand[0] = row[0] + 1
        cand[1:] = np.minimum(row[1:] + 1, row[:-1] + (b != a[i]))
        row = np.minimum.accumulate(cand - ar) + ar  # insertions along the row
    return int(row[-1])


def path_text(g, seqs, arcs, verts, arc_ids, end_off):
    """The text a path spells, after checking that each arc joins its two vertices."""
    assert len(verts) >= 1
    if len(verts) == 1:
        return seqs[verts[0]][:end_off + 1]
    parts = [seqs[verts[0]]]
    for j in range(1, len(verts)):
        v, w, o = arcs[arc_ids[j]]
        assert (v, w) == (verts[j - 1], verts[j])
        parts.append(seqs[w][o:end_off + 1] if j == len(verts) - 1 else seqs[w][o:])
    return b"".join(parts)


def check_paths(g, reads, v0, dist, st, end_off, paths, exact, v1=-1):
    seqs, arcs = g.seqs(), g.arcs()
    for i, q in enumerate(reads):
        if st[i] != 0 or dist[i] < 0:
            assert len(paths[i][0]) == 0 and end_off[i] == -1
            continue
        verts, arc_ids = paths[i]
        assert verts[0] == v0[i] and arc_ids[0] == -1
        if v1 >= 0:
            assert verts[-1] == v1 and end_off[i] == len(seqs[v1]) - 1
        cost = edit_distance(q, path_text(g, seqs, arcs, verts, arc_ids, end_off[i]))
        if exact and v1 < 0:
            assert cost == dist[i], (i, cost, dist[i])
        else:
            assert cost <= dist[i], (i, cost, dist[i])


def _reads(w, n):
    return [bytes(w["cat"][o:o + l]) for o, l in zip(w["offs"][:n], w["lens"][:n])]


@pytest.mark.parametrize("exact", [True, False])
def test_paths_on_bubble_graph(G, exact):
    w = G.load_workload("config2", n=400)
    g = w["graph"]
    g.index()
    flags = G.GWF_F_EXACT_START if exact else 0
    reads = (w["cat"], w["offs"], w["lens"])
    d0, s0 = g.ed_batch(reads, w["v0"], flags=flags)
    d, st, eo, paths = g.ed_path(reads, w["v0"], flags=flags)
    assert np.array_equal(d, d0) and np.array_equal(st, s0) and (st == 0).all()
    sel = np.arange(0, 400, 4)
    check_paths(g, [_reads(w, 400)[i] for i in sel], w["v0"][sel], d[sel], st[sel], eo[sel],
                [paths[i] for i in sel], exact)


def test_paths_on_random_graphs(G, O):
    """Small DAGs and cyclic graphs with v1 >= 0 targets, against the oracle's distance and DP."""
    checked = 0
    for t, (seqs, arcs, v0, v1, q) in enumerate(cases(707, 200, v1_prob=0.3)):
        exact = bool(t & 1)
        og = O.OracleGraph(seqs, arcs)
        od, ost = og.ed(q, v0, v1, exact_start=exact)
        if ost.flags & O.F_NONTERM:
            continue
        g = G.Graph.from_arrays(seqs, arcs)
        g.index()
        d, st, eo, paths = g.ed_path([q], [v0], v1=v1, flags=G.GWF_F_EXACT_START if exact else 0)
        assert st[0] == 0 and d[0] == od
        check_paths(g, [q], [v0], d, st, eo, paths, exact, v1)
        if d[0] >= 0 and v1 < 0:
            assert edit_distance(q, path_text(g, g.seqs(), g.arcs(), paths[0][0], paths[0][1], eo[0])) >= og.dp(q, v0, v1)
        checked += 1
        g.close()
    assert checked > 150


def test_long_reads_with_arena_retries(G):
    """10 kbp reads on the 5 Mbp graph; the trace arenas of some overflow and are re-run."""
    w = G.load_workload("config4", n=6)
    g = w["graph"]
    g.index()
    reads = (w["cat"], w["offs"], w["lens"])
    d0, _ = g.ed_batch(reads, w["v0"], flags=G.GWF_F_EXACT_START)
    d, st, eo, paths = g.ed_path(reads, w["v0"], flags=G.GWF_F_EXACT_START)
    assert (st == 0).all() and np.array_equal(d, d0)
    check_paths(g, _reads(w, 6), w["v0"], d, st, eo, paths, True)


def test_truncated_rows_and_failed_reads(G):
    w = G.load_workload("config1", n=20)
    g = w["graph"]
    g.index()
    reads = _reads(w, 20)
    _, _, eo, full = g.ed_path(reads, w["v0"], max_nv=4096)
    d, st, eo2, cut = g.ed_path(reads, w["v0"], max_nv=2)
    assert np.array_equal(eo, eo2)
    for (fv, fa), (cv, ca) in zip(full, cut):
        assert np.array_equal(cv, fv[:2]) and np.array_equal(ca, fa[:2])
    _, _, _, pn, pv, pa = g.ed_path(reads, w["v0"], max_nv=4096, as_arrays=True)
    for i, (fv, fa) in enumerate(full):
        assert pn[i] == len(fv) and np.array_equal(pv[i, :pn[i]], fv) and np.array_equal(pa[i, :pn[i]], fa)
    # an empty read is a per-read error: no path
    d, st, eo, paths = g.ed_path([b"", reads[0]], [0, int(w["v0"][0])])
    assert st[0] == G.GWF_E_BAD_INPUT and eo[0] == -1 and len(paths[0][0]) == 0
    assert st[1] == 0 and len(paths[1][0]) >= 1


def check_cigar(q, text, runs, dist, exact):
    """Walks the CIGAR over the read and the path text: every '=' base equal, every 'X' base
    different, both sequences consumed; its cost is the optimal end-to-end distance of the two,
    at most the traced distance (equal with the exact start state)."""
    i = j = cost = 0
    for x in runs:
        n, op = int(x) >> 4, int(x) & 15
        assert n > 0
        if op == 7:
            assert q[i:i + n] == text[j:j + n]
            i, j = i + n, j + n
        elif op == 8:
            assert all(q[i + t] != text[j + t] for t in range(n))
            i, j, cost = i + n, j + n, cost + n
        elif op == 1:
            i, cost = i + n, cost + n
        elif op == 2:
            j, cost = j + n, cost + n
        else:
            raise AssertionError("op %d" % op)
    assert i == len(q) and j == len(text)
    assert cost == edit_distance(q, text)
    assert cost == dist if exact else cost <= dist
    return cost


@pytest.mark.parametrize("exact", [True, False])
def test_cigars_on_bubble_graph(G, exact):
    w = G.load_workload("config2", n=200)
    g = w["graph"]
    g.index()
    flags = G.GWF_F_EXACT_START if exact else 0
    reads = _reads(w, 200)
    d0, _ = g.ed_batch(reads, w["v0"], flags=flags)
    d, st, eo, pn, pv, pa, cn, cg = g.ed_path(reads, w["v0"], flags=flags, max_ops=512, as_arrays=True)
    assert np.array_equal(d, d0) and (st == 0).all() and (cn > 0).all()
    seqs, arcs = g.seqs(), g.arcs()
    for i in range(0, 200, 2):
        text = path_text(g, seqs, arcs, pv[i, :pn[i]], pa[i, :pn[i]], eo[i])
        check_cigar(reads[i], text, cg[i, :cn[i]], d[i], exact)
    _, _, _, _, cigars = g.ed_path(reads[:3], w["v0"][:3], flags=flags, max_ops=512)
    assert all(c and c[-1] in "=XID" for c in cigars)


def test_cigars_on_random_graphs(G, O):
    checked = 0
    for t, (seqs_in, arcs_in, v0, v1, q) in enumerate(cases(818, 150, v1_prob=0.3)):
        exact = bool(t & 1)
        og = O.OracleGraph(seqs_in, arcs_in)
        od, ost = og.ed(q, v0, v1, exact_start=exact)
        if ost.flags & O.F_NONTERM:
            continue
        g = G.Graph.from_arrays(seqs_in, arcs_in)
        g.index()
        d, st, eo, pn, pv, pa, cn, cg = g.ed_path([q], [v0], v1=v1, flags=G.GWF_F_EXACT_START if exact else 0,
                                                   max_ops=256, as_arrays=True)
        assert st[0] == 0 and d[0] == od
        if d[0] >= 0:
            assert cn[0] > 0
            text = path_text(g, g.seqs(), g.arcs(), pv[0, :pn[0]], pa[0, :pn[0]], eo[0])
            check_cigar(q, text, cg[0, :cn[0]], d[0], exact and v1 < 0)
        else:
            assert cn[0] == -1
        checked += 1
        g.close()
    assert checked > 100


def test_cigars_on_long_reads(G):
    w = G.load_workload("config5", n=12)
    g = w["graph"]
    g.index()
    reads = _reads(w, 12)
    d, st, eo, pn, pv, pa, cn, cg = g.ed_path(reads, w["v0"], flags=G.GWF_F_EXACT_START, max_ops=8192,
                                               as_arrays=True)
    assert (st == 0).all() and (cn > 0).all()
    seqs, arcs = g.seqs(), g.arcs()
    for i in range(12):
        if len(reads[i]) > 6000:
            continue  # the test's numpy DP is quadratic
        text = path_text(g, seqs, arcs, pv[i, :pn[i]], pa[i, :pn[i]], eo[i])
        check_cigar(reads[i], text, cg[i, :cn[i]], d[i], True)
    # a row narrower than the CIGAR: the count is still the full count
    _, _, _, _, _, _, cn2, cg2 = g.ed_path(reads[:2], w["v0"][:2], flags=G.GWF_F_EXACT_START, max_ops=4,
                                           as_arrays=True)
    assert np.array_equal(cn2, cn[:2]) and np.array_equal(cg2[:, :4], cg[:2, :4])
