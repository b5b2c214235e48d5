"""Multi-rank logic of bench.py on CPU: two gloo ranks, each with its own seeded shard of the
workload (reads are independent, so there is no collective on the data path), timings reduced
as the max over ranks, and the reference arm doing no work on ranks other than 0. The oracle
stands in for the kernel, which needs a GPU."""
import os
import socket
import sys
import time
from datetime import timedelta

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        G = bench.pkg()
        w = G.load_workload("config1", n=40, seed=bench.shard_seed("config1", rank))
        O = bench.oracle_mod()
        og = O.OracleGraph.from_graph(w["graph"])
        dist.barrier()
        t0 = time.perf_counter()
        d, _, _ = og.ed_batch(w["cat"], w["offs"], w["lens"], w["v0"], stats=False, threads=1)
        el = time.perf_counter() - t0
        m = bench.reduce_max(el, dist, "cpu")
        digest = int(np.frombuffer(w["cat"].tobytes(), dtype=np.uint8).astype(np.int64).sum())
        seen = [None] * world
        dist.all_gather_object(seen, (el, digest, int(d.sum())))

        class A:
            workload, steps, warmup, ref_step_seconds = "config1", 1, 1, 0.1
        t0 = time.perf_counter()
        ref = bench.run_reference(A, rank, world) if rank != 0 else None
        q.put((rank, m, seen, ref, time.perf_counter() - t0))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, m, seen, ref, t_ref = q.get(timeout=240)
        out[rank] = (m, seen, ref, t_ref)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m0, seen0, _, _ = out[0]
    m1, seen1, ref1, t_ref1 = out[1]
    assert seen0 == seen1
    assert m0 == m1 == max(e for e, _, _ in seen0)
    assert seen0[0][1] != seen0[1][1]  # each rank aligns its own reads
    assert ref1 is None and t_ref1 < 1.0  # the reference arm runs on rank 0 only


def test_rank0_shard_is_the_published_workload(G):
    import importlib
    sys.path.insert(0, ROOT)
    bench = importlib.import_module("bench")
    a = G.load_workload("config1", n=30, seed=bench.shard_seed("config1", 0))
    b = G.load_workload("config1", n=30)
    assert np.array_equal(a["cat"], b["cat"]) and np.array_equal(a["v0"], b["v0"])
    assert bench.reduce_max(1.5) == 1.5


def _split_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        G = bench.pkg()
        rng = np.random.default_rng(7)  # the same batch on every rank
        reads = [bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(50, 400))).astype(np.uint8)) for _ in range(101)]
        v0 = rng.integers(0, 9, 101).astype(np.int32)
        seen = []

        def fake(cat, offs, lens, vv):  # stands in for the GPU: a function of the read's bytes
            seen.append(len(lens))
            d = np.array([int(cat[o:o + l].astype(np.int64).sum()) % 1000 + int(x) for o, l, x in zip(offs, lens, vv)],
                         dtype=np.int32)
            return d, np.full(len(lens), rank, dtype=np.int32)

        d, st = G.align_sharded(None, reads, v0, align_fn=fake)
        q.put((rank, d.tolist(), st.tolist(), seen))
    finally:
        dist.destroy_process_group()


def test_split_batch_over_two_gloo_ranks(G):
    """align_sharded: one batch split by cost over two ranks, each rank aligns only its range,
    and the all-gather gives both ranks the full results in input order."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, d, st, seen = q.get(timeout=240)
        out[rank] = (d, st, seen)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rng = np.random.default_rng(7)
    reads = [bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(50, 400))).astype(np.uint8)) for _ in range(101)]
    v0 = rng.integers(0, 9, 101).astype(np.int32)
    want = [sum(r) % 1000 + int(x) for r, x in zip(reads, v0)]
    parts = G.partition_reads([len(r) for r in reads], 2)
    assert out[0][0] == out[1][0] == want
    assert out[0][1] == out[1][1] == [0] * parts[0][1] + [1] * (101 - parts[0][1])
    assert out[0][2] == [parts[0][1] - parts[0][0]] and out[1][2] == [parts[1][1] - parts[1][0]]


def test_partition_is_contiguous_and_balanced(G):
    rng = np.random.default_rng(3)
    lens = rng.integers(500, 10000, 5000)
    for world in (1, 2, 4, 8):
        parts = G.partition_reads(lens, world)
        assert parts[0][0] == 0 and parts[-1][1] == len(lens)
        assert all(parts[k][1] == parts[k + 1][0] for k in range(world - 1))
        loads = [float((lens[a:b].astype(float) ** 2).sum()) for a, b in parts]
        assert max(loads) <= 1.02 * sum(loads) / world
