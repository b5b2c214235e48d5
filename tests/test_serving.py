"""Serving loop (gwf_srv_*): requests of mixed sizes, submitted while others are on the GPU, get
exactly the distances and statuses they get when aligned alone through gwf_ed_batch (tolerance 0:
int32 distances)."""
import random
import time

import numpy as np
import pytest

from randgraph import rand_graph, walk_read

pytestmark = pytest.mark.gpu


def _subset(w, idx):
    offs = w["offs"][idx]
    lens = w["lens"][idx]
    return (w["cat"], np.ascontiguousarray(offs), np.ascontiguousarray(lens)), np.ascontiguousarray(w["v0"][idx])


def _requests(w, rng, max_reads=48):
    reqs, i, n = [], 0, len(w["lens"])
    while i < n:
        m = int(rng.integers(1, max_reads))
        reqs.append(np.arange(i, min(n, i + m)))
        i += m
    return reqs


def _serve_and_compare(G, g, w, reqs, v1s, **srv_kw):
    rng = np.random.default_rng(7)
    srv = G.Server(g, **srv_kw)
    try:
        ids = []
        for r, v1 in zip(reqs, v1s):
            reads, v0 = _subset(w, r)
            ids.append(srv.submit(reads, v0, v1))
            time.sleep(float(rng.uniform(0, 0.003)))
        served = [srv.wait(rid, k, timeout_s=300) for rid, k in ids]
        for rid, k in ids:
            t_sub, t_adm, t_done = srv.times(rid)
            assert t_sub <= t_adm <= t_done
        stats = srv.stats()
    finally:
        srv.close()
    for r, v1, (d, st) in zip(reqs, v1s, served):
        reads, v0 = _subset(w, r)
        solo, st2 = g.ed_batch(reads, v0, v1=v1)
        assert np.array_equal(st, st2)
        assert np.array_equal(d, solo)
    return served, stats


def test_mixed_requests_equal_solo_results(G):
    w = G.load_workload("config3", n=400)
    g = w["graph"]
    g.index()
    reqs = _requests(w, np.random.default_rng(5))
    served, stats = _serve_and_compare(G, g, w, reqs, [-1] * len(reqs))
    assert all((st == 0).all() for _, st in served)


@pytest.mark.parametrize("nw", [2, 4, 8])
def test_groups_of_warps_equal_solo_results(G, nw):
    """warps_per_read > 1: each read is aligned by a group of warps of the resident kernel; the
    results are those of the batch call, also with lag pruning and v1 targets."""
    w = G.load_workload("config5", n=60)
    g = w["graph"]
    g.index()
    reqs = _requests(w, np.random.default_rng(nw), max_reads=12)
    served, stats = _serve_and_compare(G, g, w, reqs, [-1] * len(reqs), arena_budget_bytes=8 << 30,
                                       warps_per_read=nw)
    assert all((st == 0).all() for _, st in served)
    w3 = G.load_workload("config3", n=120)
    g3 = w3["graph"]
    g3.index()
    reqs3 = _requests(w3, np.random.default_rng(nw + 1), max_reads=20)
    v1s = [-1 if i % 2 else 7 for i in range(len(reqs3))]
    _serve_and_compare(G, g3, w3, reqs3, v1s, warps_per_read=nw)
    with pytest.raises(G.GwfError):
        G.Server(g3, warps_per_read=3)
    assert stats["launches"] >= 1 and stats["arena_used"] == 0


def test_lag_pruning_in_serving_equals_batch(G):
    """GWF_F_MAX_LAG through the serving options: each read gets the pruned distance that
    gwf_ed_batch gives with the same lag (and the lag is applied: some reads differ from the
    exact distance)."""
    w = G.load_workload("config2", n=300)
    g = w["graph"]
    g.index()
    lag = 2
    srv = G.Server(g, flags=G.GWF_F_MAX_LAG, max_lag=lag)
    try:
        ids = []
        for r in _requests(w, np.random.default_rng(9)):
            reads, v0 = _subset(w, r)
            ids.append((r, srv.submit(reads, v0)))
        served = [(r, srv.wait(rid, k, timeout_s=300)) for r, (rid, k) in ids]
    finally:
        srv.close()
    d_all = np.empty(300, dtype=np.int32)
    for r, (d, st) in served:
        assert (st == 0).all()
        d_all[r] = d
    reads = (w["cat"], w["offs"], w["lens"])
    pruned, _ = g.ed_batch(reads, w["v0"], flags=G.GWF_F_MAX_LAG, max_lag=lag)
    exact, _ = g.ed_batch(reads, w["v0"])
    assert np.array_equal(d_all, pruned)
    assert (pruned != exact).any()


def test_small_arena_budget_and_target_vertex(G):
    """An 8 MiB arena budget (a few dozen small arenas at once, one of the largest class): admission
    waits for memory. Requests with a target vertex (v1 >= 0) are mixed with v1 = -1 ones, on a
    random graph with N bases (byte-compare path)."""
    rng = random.Random(17)
    seqs, arcs = rand_graph(rng, 40, 40, False, "ACGTN")
    g = G.Graph.from_arrays(seqs, arcs)
    g.index()
    reads, v0s = [], []
    for _ in range(160):
        v0 = rng.randrange(len(seqs))
        reads.append(walk_read(rng, seqs, arcs, v0, rng.randint(1, 120), rng.choice([0.0, 0.05, 0.2])))
        v0s.append(v0)
    cat, offs, lens = G.pack_reads(reads)
    w = {"cat": cat, "offs": offs, "lens": lens, "v0": np.array(v0s, dtype=np.int32)}
    reqs = _requests(w, np.random.default_rng(9), max_reads=12)
    v1s = [-1 if i % 3 else rng.randrange(len(seqs)) for i in range(len(reqs))]
    _serve_and_compare(G, g, w, reqs, v1s, arena_budget_bytes=8 << 20)


def test_arena_overflow_is_retried(G):
    """Reads unrelated to the graph overflow the first arena class; the server re-queues them in
    larger arenas and ends with the batch path's distances and statuses."""
    w = G.load_workload("config1", n=16)
    g = w["graph"]
    g.index()
    rng = np.random.default_rng(3)
    junk = [bytes(rng.choice(list(b"ACGT"), size=700).astype(np.uint8)) for _ in range(3)]
    reads = [bytes(w["cat"][o:o + l]) for o, l in zip(w["offs"][:5], w["lens"][:5])] + junk
    v0 = np.concatenate([w["v0"][:5], np.zeros(3, np.int32)]).astype(np.int32)
    srv = G.Server(g)
    try:
        rid, k = srv.submit(reads, v0)
        d, st = srv.wait(rid, k, timeout_s=300)
        stats = srv.stats()
    finally:
        srv.close()
    solo, st2 = g.ed_batch(reads, v0)
    assert np.array_equal(st, st2) and np.array_equal(d, solo)
    assert stats["retries"] > 0


def test_kernel_closes_when_idle_and_relaunches(G):
    """After the queue runs dry the resident kernel ends as a whole; a later request starts a new
    launch with every warp, so it runs as fast as the first."""
    w = G.load_workload("config3", n=600)
    g = w["graph"]
    g.index()
    reads = (w["cat"], w["offs"], w["lens"])
    srv = G.Server(g)
    try:
        t = []
        for rep in range(2):
            t0 = time.perf_counter()
            rid, k = srv.submit(reads, w["v0"])
            d, st = srv.wait(rid, k, timeout_s=300)
            t.append(time.perf_counter() - t0)
            assert (st == 0).all()
            for _ in range(400):  # the kernel closes ~5 ms after the last read
                if srv.stats()["kernel_running"] == 0:
                    break
                time.sleep(0.005)
            assert srv.stats()["kernel_running"] == 0
        assert srv.stats()["launches"] == 2
        assert t[1] < 3 * t[0] + 0.5
    finally:
        srv.close()
    solo, _ = g.ed_batch(reads, w["v0"])
    assert np.array_equal(d, solo)


def test_poll_and_unknown_request(G):
    w = G.load_workload("config1", n=8)
    g = w["graph"]
    g.index()
    srv = G.Server(g)
    try:
        rid, k = srv.submit((w["cat"], w["offs"], w["lens"]), w["v0"])
        res = None
        for _ in range(2000):
            res = srv.poll(rid, k)
            if res is not None:
                break
            time.sleep(0.005)
        assert res is not None and (res[1] == 0).all()
        with pytest.raises(G.GwfError):
            srv.wait(10_000, 1, timeout_s=0.1)
    finally:
        srv.close()


def test_failures_come_back_as_statuses(G):
    """Host-side fault cases: an arena budget too small for a long read completes that read
    with GWF_E_CAPACITY and still serves the short ones; a budget the device cannot hold makes
    creation fail with an error, not a fault."""
    w = G.load_workload("config3", n=200)
    g = w["graph"]
    g.index()
    long_i = int(np.argmax(w["lens"]))
    short = [i for i in range(len(w["lens"])) if w["lens"][i] < 1000][:6]
    idx = np.array(short + [long_i])
    reads, v0 = _subset(w, idx)
    srv = G.Server(g, arena_budget_bytes=2 << 20)  # holds a few arenas of short reads only
    try:
        rid, k = srv.submit(reads, v0)
        d, st = srv.wait(rid, k, timeout_s=120)
    finally:
        srv.close()
    assert st[-1] == G.GWF_E_CAPACITY and d[-1] == -1
    solo, st2 = g.ed_batch((reads[0], reads[1][:-1], reads[2][:-1]), v0[:-1])
    assert (st[:-1] == 0).all() and np.array_equal(d[:-1], solo)
    with pytest.raises(G.GwfError):
        G.Server(g, arena_budget_bytes=1 << 50)
