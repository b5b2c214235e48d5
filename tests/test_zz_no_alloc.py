"""gwf_ed_batch_noalloc, the batch entry point that allocates nothing.

It serves callers that must not call cudaMalloc while they align: for example, a framework
whose caching allocator owns the device heap, or a latency-bound serving loop that cannot
afford cudaMalloc's implicit device synchronisation. The caller passes its own device buffers
(allocated here with torch, standing in for such a framework), and the call's scratch lives in a
fixed array inside the library. Its distances must equal the allocating batch entry point's, bit
for bit, on two calls in a row (the second reuses the scratch left by the first).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_inputs(torch, w):
    dev = torch.device("cuda", 0)
    n = len(w["lens"])
    tot = int(w["offs"][-1] + w["lens"][-1])
    seqs = torch.zeros(tot + 16, dtype=torch.uint8, device=dev)  # 16 readable bytes past the end
    seqs[:tot] = torch.from_numpy(np.ascontiguousarray(w["cat"][:tot])).to(dev)
    offs = torch.from_numpy(np.ascontiguousarray(w["offs"])).to(dev)
    ql = torch.from_numpy(np.ascontiguousarray(w["lens"])).to(dev)
    v0 = torch.from_numpy(np.ascontiguousarray(w["v0"])).to(dev)
    dist = torch.empty(n, dtype=torch.int32, device=dev)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    return seqs, offs, ql, v0, dist, status


def test_noalloc_equals_allocating_batch_on_two_calls(G):
    import torch

    w = G.load_workload("config2", n=3000)
    g = w["graph"]
    g.index()
    expect, st = g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"])
    assert (st == 0).all()
    seqs, offs, ql, v0, dist, status = _device_inputs(torch, w)
    n, max_ql = len(w["lens"]), int(w["lens"].max())
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        dist.fill_(-7)
        status.fill_(-7)
        rc = G.lib().gwf_ed_batch_noalloc(g.ptr, n, max_ql, seqs.data_ptr(), offs.data_ptr(), ql.data_ptr(),
                                          v0.data_ptr(), -1, dist.data_ptr(), status.data_ptr(), 0, stream)
        assert rc == 0, G.last_error()
        torch.cuda.synchronize()
        assert (status.cpu().numpy() == 0).all()
        assert np.array_equal(dist.cpu().numpy(), expect)


def _noalloc(G, torch, g, w, flags=0):
    seqs, offs, ql, v0, dist, status = _device_inputs(torch, w)
    dist.fill_(-7)
    status.fill_(-7)
    rc = G.lib().gwf_ed_batch_noalloc(g.ptr, len(w["lens"]), int(w["lens"].max()), seqs.data_ptr(),
                                      offs.data_ptr(), ql.data_ptr(), v0.data_ptr(), -1, dist.data_ptr(),
                                      status.data_ptr(), flags, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, G.last_error()
    torch.cuda.synchronize()
    return dist.cpu().numpy(), status.cpu().numpy()


@pytest.mark.parametrize("n", [1, 5, 9])
def test_noalloc_small_batches(G, n):
    """Batches smaller than one CTA's eight warps (a single read, as a serving loop sends) are
    aligned like any other."""
    import torch

    w = G.load_workload("config2", n=16)
    w = {k: (v[:n] if k in ("offs", "lens", "v0") else v) for k, v in w.items()}
    g = w["graph"]
    g.index()
    for flags in (0, G.GWF_F_EXACT_START):
        expect, st = g.ed_batch((w["cat"], w["offs"], w["lens"]), w["v0"], flags=flags)
        d, s = _noalloc(G, torch, g, w, flags)
        assert (s == 0).all() and (st == 0).all()
        assert np.array_equal(d, expect)


def test_noalloc_arena_overflow_is_per_read(G):
    """Reads unrelated to the graph outgrow the fixed arena: they come back as GWF_E_CAPACITY
    with distance -1 (this entry point has no larger arena to retry in), and every other read of
    the same call is exact."""
    import torch

    w = G.load_workload("config1", n=40)
    g = w["graph"]
    g.index()
    rng = np.random.default_rng(12)
    reads = [bytes(w["cat"][o:o + l]) for o, l in zip(w["offs"], w["lens"])]
    junk_at = [3, 17, 31]
    for i in junk_at:
        # a random read's wavefront reaches ~2,000 diagonals, past the 1,792 of the fixed arena
        reads[i] = bytes(rng.choice(list(b"ACGT"), size=2040).astype(np.uint8))
    cat, offs, lens = G.pack_reads(reads)
    w2 = {"cat": cat, "offs": offs, "lens": lens, "v0": w["v0"].copy()}
    expect, st = g.ed_batch((cat, offs, lens), w2["v0"])  # the allocating call retries in larger arenas
    assert (st == 0).all()
    d, s = _noalloc(G, torch, g, w2)
    ok = np.ones(len(lens), dtype=bool)
    ok[junk_at] = False
    assert (s[~ok] == G.GWF_E_CAPACITY).all() and (d[~ok] == -1).all()
    assert (s[ok] == 0).all() and np.array_equal(d[ok], expect[ok])


def test_noalloc_rejects_unsupported_flags(G):
    w = G.load_workload("config1", n=4)
    g = w["graph"]
    g.index()
    rc = G.lib().gwf_ed_batch_noalloc(g.ptr, 4, 100, 8, 8, 8, 8, -1, 8, 8, G.GWF_F_MAX_LAG, None)
    assert rc == G.GWF_E_BAD_INPUT and "GWF_F_EXACT_START" in G.last_error()


def test_noalloc_rejects_sizes_beyond_its_limits(G):
    w = G.load_workload("config1", n=4)
    g = w["graph"]
    g.index()
    L = G.lib()
    # rejected before any device pointer is used
    assert L.gwf_ed_batch_noalloc(g.ptr, 262145, 100, 8, 8, 8, 8, -1, 8, 8, 0, None) == G.GWF_E_CAPACITY
    assert "262144" in G.last_error()
    assert L.gwf_ed_batch_noalloc(g.ptr, 4, 2049, 8, 8, 8, 8, -1, 8, 8, 0, None) == G.GWF_E_CAPACITY
    assert "2048" in G.last_error()
