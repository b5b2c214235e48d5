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
