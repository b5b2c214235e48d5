"""Streamed uploads (gwf_ed_batch_concat, persistent form with one warp per read): the read bytes
go to the device in 4 MiB chunks on a copy stream while the kernel already aligns the reads whose
chunks have arrived, each warp packing its own read. The distances must equal those of a resident
batch, whose bytes were all on the device before its kernel started, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _resident(G, g, cat, offs, lens, v0, **kw):
    b = G.ResidentBatch(g, cat, offs, lens, v0, mode=G.MODE_PERSISTENT, **kw)
    b.run(warps_per_read=1)
    d, st = b.results()
    b.close()
    return d, st


@pytest.mark.parametrize("name,n", [("config2", 20000), ("config3", 20000)])
def test_streamed_equals_resident(G, O, name, n):
    """Batches large enough for one warp per read, from pageable and from pinned host memory,
    spanning 5-10 chunks; reads cross chunk boundaries."""
    w = G.load_workload(name, n=n)
    g = w["graph"]
    g.index()
    d0, s0 = _resident(G, g, w["cat"], w["offs"], w["lens"], w["v0"])
    assert (s0 == 0).all()
    d1, s1 = g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"], mode=G.MODE_PERSISTENT)
    assert np.array_equal(s1, s0) and np.array_equal(d1, d0)
    wp = G.load_workload(name, n=n, pinned=True)
    d2, s2 = g.ed_batch((wp["cat"], wp["offs"], wp["lens"]), wp["v0"], mode=G.MODE_PERSISTENT)
    assert np.array_equal(s2, s0) and np.array_equal(d2, d0)
    sel = np.linspace(0, n - 1, 300).astype(np.int64)
    od, _, _ = O.OracleGraph.from_graph(g).ed_batch(w["cat"], w["offs"][sel], w["lens"][sel], w["v0"][sel],
                                                    stats=False)
    assert np.array_equal(d1[sel], od)


def test_streamed_byte_compares_and_options(G, O):
    """Reads with N and lower-case bases (the byte-compare path reads the streamed bytes
    directly), the exact start state, lag pruning, and reads that overflow their arena and are
    re-run after the streamed launch."""
    w = G.load_workload("config2", n=12000)
    g = w["graph"]
    g.index()
    rng = np.random.default_rng(17)
    reads = [bytearray(w["cat"][o:o + l]) for o, l in zip(w["offs"], w["lens"])]
    for i in rng.choice(len(reads), 400, replace=False):
        for j in rng.choice(len(reads[i]), 3, replace=False):
            reads[i][j] = ord(rng.choice([b"N", b"a", b"c"]))
    for i in rng.choice(len(reads), 5, replace=False):
        reads[i] = bytearray(rng.choice(list(b"ACGT"), size=800).astype(np.uint8))
    cat, offs, lens = G.pack_reads([bytes(r) for r in reads])
    v0 = w["v0"]
    for flags, lag in ((0, 0), (G.GWF_F_EXACT_START, 0), (G.GWF_F_MAX_LAG, 7)):
        d0, s0 = _resident(G, g, cat, offs, lens, v0, flags=flags) if lag == 0 else (None, None)
        d1, s1 = g.ed_batch((cat, offs, lens), v0, mode=G.MODE_PERSISTENT, flags=flags, max_lag=lag)
        assert (s1 == 0).all()
        if lag == 0:
            assert np.array_equal(d1, d0)
        else:
            sel = np.arange(0, len(lens), 97)
            og = O.OracleGraph.from_graph(g)
            od = [og.ed(bytes(cat[offs[i]:offs[i] + lens[i]]), int(v0[i]), max_lag=lag)[0] for i in sel]
            assert list(d1[sel]) == od
