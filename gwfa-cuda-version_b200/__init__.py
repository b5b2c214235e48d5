"""Python mirror of the GWFA B200 C ABI (include/gwfa.h), for tests, benchmarks and scripting.

The compute path is libgwfa_b200.so (hand-written sm_100a CUDA behind a C ABI). This module only
marshals arguments with ctypes; it has no fallback: when the library or a B200 is missing, calls
raise GwfError.

Mirrors the reference interface: gwf_ed_index / gwf_cleanup (main.cu:246-277), gwf_ed
(gwfa.h:95, host-callable here), the GFA loader + gwf_gfa2gwf (main.cu:294-359), plus batch,
resident-batch and serving entry points that replace the stream loop of main.cu:620-735.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgwfa_b200.so")

GWF_OK = 0
GWF_NO_ALIGNMENT = -1
GWF_E_BAD_INPUT = -2
GWF_E_UNSUPPORTED = -3
GWF_E_CAPACITY = -4
GWF_E_CUDA = -5
GWF_E_NOT_INDEXED = -6
GWF_E_BAD_GRAPH = -7
GWF_E_TIMEOUT = -8
GWF_E_NOMEM = -9
GWF_E_BUSY = -10

GWF_F_EXACT_START = 1
GWF_F_MAX_LAG = 2
GWF_F_BOTH_STRANDS = 4
MODE_AUTO, MODE_PLAIN, MODE_PERSISTENT = 0, 1, 2


class GwfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gwfa error {code}: {msg}")
        self.code = code


class GwfArc(ctypes.Structure):
    _fields_ = [("a", ctypes.c_uint64), ("o", ctypes.c_int32)]


class GwfGraph(ctypes.Structure):
    _fields_ = [
        ("n_vtx", ctypes.c_uint32), ("n_arc", ctypes.c_uint32),
        ("len", ctypes.POINTER(ctypes.c_uint32)), ("src", ctypes.POINTER(ctypes.c_uint32)),
        ("seq", ctypes.POINTER(ctypes.c_char_p)), ("arc", ctypes.POINTER(GwfArc)),
        ("aux", ctypes.POINTER(ctypes.c_uint64)),
    ]


class BatchOpts(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int32), ("flags", ctypes.c_int32), ("device", ctypes.c_int32),
                ("warps_per_read", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32),
                ("use_graph", ctypes.c_int32), ("reserved", ctypes.c_int32 * 10)]


class SrvOpts(ctypes.Structure):
    _fields_ = [("arena_budget_bytes", ctypes.c_int64), ("max_inflight_reads", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("device", ctypes.c_int32), ("max_lag", ctypes.c_int32),
                ("warps_per_read", ctypes.c_int32), ("reserved", ctypes.c_int32 * 5)]


class GwfReads(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("n_bases", ctypes.c_int64), ("seqs", ctypes.c_void_p),
                ("offs", ctypes.POINTER(ctypes.c_int64)), ("lens", ctypes.POINTER(ctypes.c_int32))]


_lib = None
P = ctypes.c_void_p
I32, I64, U32, U64, DBL = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double
PG = ctypes.POINTER(GwfGraph)

# name -> (restype, argtypes): every entry point of include/gwfa.h and include/gwfa_synth.h
SIGNATURES = {
    "gwf_ed_index": (None, [PG]),
    "gwf_cleanup": (None, [PG]),
    "gwf_ed": (I32, [P, PG, I32, ctypes.c_char_p, I32, I32, U32, I32]),
    "gwf_ed_batch": (ctypes.c_int, [PG, I32, P, P, P, I32, U32, P, P, P]),
    "gwf_ed_batch_concat": (ctypes.c_int, [PG, I32, P, P, P, P, I32, U32, P, P, P]),
    "gwf_ed_batch_strand": (ctypes.c_int, [PG, I32, P, P, P, P, I32, U32, P, P, P, P]),
    "gwf_ed_batch_path": (ctypes.c_int, [PG, I32, P, P, P, P, I32, I32, I32, P, P, P, P, P, P]),
    "gwf_reads_load": (ctypes.POINTER(GwfReads), [ctypes.c_char_p]),
    "gwf_reads_free": (None, [ctypes.POINTER(GwfReads)]),
    "gwf_ed_batch_align": (ctypes.c_int, [PG, I32, P, P, P, P, I32, I32, I32, I32, P, P, P, P, P, P, P, P]),
    "gwf_batch_create": (P, [PG, I32, P, P, P, P, I32, P]),
    "gwf_batch_run": (ctypes.c_int, [P, P, P]),
    "gwf_batch_results": (ctypes.c_int, [P, P, P]),
    "gwf_batch_launches": (I32, [P]),
    "gwf_batch_steps": (ctypes.c_int, [P, P]),
    "gwf_batch_destroy": (None, [P]),
    "gwf_ed_batch_noalloc": (ctypes.c_int, [PG, I32, I32, P, P, P, P, I32, P, P, I32, P]),
    "gwf_tune": (ctypes.c_int, [PG, I32, P, P, P, P, I32, I32, ctypes.c_char_p]),
    "gwf_tune_load": (ctypes.c_int, [ctypes.c_char_p, I32]),
    "gwf_tune_get": (ctypes.c_int, [I32, I32, P, P, P]),
    "gwf_tune_get_shape": (ctypes.c_int, [I32, I32, P, P, P, P]),
    "gwf_tune_clear": (None, [I32]),
    "gwf_pinned_alloc": (P, [I64]),
    "gwf_pinned_free": (None, [P]),
    "gwf_srv_create": (P, [PG, P]),
    "gwf_srv_submit": (I64, [P, I32, P, P, P, P, I32]),
    "gwf_srv_poll": (ctypes.c_int, [P, I64, P, P]),
    "gwf_srv_wait": (ctypes.c_int, [P, I64, P, P, DBL]),
    "gwf_srv_times": (ctypes.c_int, [P, I64, P, P, P]),
    "gwf_srv_strand": (ctypes.c_int, [P, I64, P]),
    "gwf_srv_stats": (ctypes.c_int, [P, P, I32]),
    "gwf_srv_destroy": (None, [P]),
    "gwf_gfa_load": (PG, [ctypes.c_char_p, ctypes.c_char_p]),
    "gwf_gfa_load_mem": (PG, [ctypes.c_char_p, I64, ctypes.c_char_p]),
    "gwf_graph_free": (None, [PG]),
    "gwf_graph_dump": (I64, [PG, ctypes.c_char_p, I64]),
    "gwf_last_error": (ctypes.c_char_p, []),
    "gwf_version": (ctypes.c_char_p, []),
    "gwf_synth_graph_new": (P, [I64, I32, DBL, I32, I32, I32, I32, U64]),
    "gwf_synth_graph_free": (None, [P]),
    "gwf_synth_graph_gfa": (I64, [P, ctypes.c_char_p, I64]),
    "gwf_synth_graph_nseg": (I32, [P]),
    "gwf_synth_reads_new": (P, [P, I32, I32, DBL, DBL, I32, I32, DBL, DBL, U64]),
    "gwf_synth_reads_bytes": (I64, [P]),
    "gwf_synth_reads_copy": (None, [P, P, P, P, P, P]),
    "gwf_synth_reads_free": (None, [P]),
}


def lib():
    """Loads libgwfa_b200.so (building it first when only sources are present)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from importlib import util
            spec = util.spec_from_file_location("_gwfa_build", os.path.join(HERE, "build.py"))
            mod = util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build()
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    m = lib().gwf_last_error()
    return m.decode() if m else ""


def _ptr(a):
    return a.ctypes.data if a is not None else None


def load_reads(path):
    """gwf_reads_load: a FASTA/FASTQ file (plain or gzip) as (cat, offs, lens) numpy copies, the
    layout ed_batch takes."""
    r = lib().gwf_reads_load(path.encode())
    if not r:
        raise GwfError(GWF_E_BAD_INPUT, last_error())
    try:
        n, nb = r.contents.n, r.contents.n_bases
        cat = np.frombuffer(ctypes.string_at(r.contents.seqs, nb + 16), dtype=np.uint8).copy()
        offs = np.ctypeslib.as_array(r.contents.offs, shape=(max(n, 1),))[:n].copy()
        lens = np.ctypeslib.as_array(r.contents.lens, shape=(max(n, 1),))[:n].copy()
    finally:
        lib().gwf_reads_free(r)
    return cat, offs, lens


def pack_reads(reads):
    """list of bytes/str -> (concatenated uint8 array, int64 offsets, int32 lengths)."""
    bs = [r.encode() if isinstance(r, str) else bytes(r) for r in reads]
    lens = np.array([len(b) for b in bs], dtype=np.int32)
    offs = np.zeros(len(bs), dtype=np.int64)
    if len(bs) > 1:
        offs[1:] = np.cumsum(lens[:-1], dtype=np.int64)
    cat = np.frombuffer(b"".join(bs) + b"\0", dtype=np.uint8).copy()
    return cat, offs, lens


class Graph:
    """A gwf_graph_t owned by the library (loaded from GFA) or built from arrays."""

    def __init__(self, ptr, owned=True, keep=None):
        if not ptr:
            raise GwfError(GWF_E_BAD_INPUT, last_error())
        self.ptr = ptr
        self.owned = owned
        self._keep = keep
        self.indexed = False

    @classmethod
    def from_gfa(cls, path, start_seg=None):
        p = lib().gwf_gfa_load(path.encode(), start_seg.encode() if start_seg else None)
        return cls(p)

    @classmethod
    def from_gfa_text(cls, text, start_seg=None):
        b = text.encode() if isinstance(text, str) else bytes(text)
        p = lib().gwf_gfa_load_mem(b, len(b), start_seg.encode() if start_seg else None)
        return cls(p)

    @classmethod
    def from_arrays(cls, seqs, arcs):
        """seqs: list of bytes per vertex; arcs: list of (v, w, overlap). Not owned by the library."""
        n = len(seqs)
        g = GwfGraph()
        lens = (ctypes.c_uint32 * max(n, 1))(*[len(s) for s in seqs])
        src = (ctypes.c_uint32 * max(n, 1))(*[2 * i for i in range(n)])
        bufs = [ctypes.create_string_buffer(bytes(s)) for s in seqs]
        seqp = (ctypes.c_char_p * max(n, 1))(*[ctypes.cast(b, ctypes.c_char_p) for b in bufs])
        arcv = (GwfArc * max(len(arcs), 1))(*[GwfArc((v << 32) | w, o) for v, w, o in arcs])
        g.n_vtx, g.n_arc = n, len(arcs)
        g.len = ctypes.cast(lens, ctypes.POINTER(ctypes.c_uint32))
        g.src = ctypes.cast(src, ctypes.POINTER(ctypes.c_uint32))
        g.seq = ctypes.cast(seqp, ctypes.POINTER(ctypes.c_char_p))
        g.arc = ctypes.cast(arcv, ctypes.POINTER(GwfArc))
        g.aux = None
        return cls(ctypes.pointer(g), owned=False, keep=(g, lens, src, bufs, seqp, arcv))

    @property
    def g(self):
        return self.ptr.contents

    @property
    def n_vtx(self):
        return self.g.n_vtx

    def lens(self):
        return np.array([self.g.len[i] for i in range(self.n_vtx)], dtype=np.uint32)

    def srcs(self):
        return np.array([self.g.src[i] for i in range(self.n_vtx)], dtype=np.uint32)

    def seqs(self):
        return [ctypes.string_at(self.g.seq[i], self.g.len[i]) for i in range(self.n_vtx)]

    def arcs(self):
        return [(self.g.arc[i].a >> 32, self.g.arc[i].a & 0xffffffff, self.g.arc[i].o) for i in range(self.g.n_arc)]

    def aux(self):
        if not self.g.aux:
            return None
        return np.array([self.g.aux[i] for i in range(self.n_vtx)], dtype=np.uint64)

    def dump(self):
        n = lib().gwf_graph_dump(self.ptr, None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        lib().gwf_graph_dump(self.ptr, buf, n + 1)
        return buf.raw[:n]

    def vertex_of_segment(self):
        """GFA segment id (0-based) -> gwf vertex (forward strand)."""
        out = {}
        for i, s in enumerate(self.srcs()):
            if s & 1 == 0:
                out[int(s) >> 1] = i
        return out

    def index(self):
        """gwf_ed_index: host CSR + device upload. Raises when the device part fails."""
        lib().gwf_ed_index(self.ptr)
        err = last_error()
        self.indexed = True
        return err

    def cleanup(self):
        lib().gwf_cleanup(self.ptr)
        self.indexed = False

    def close(self):
        if self.ptr:
            if self.owned:
                lib().gwf_graph_free(self.ptr)
            else:
                lib().gwf_cleanup(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- alignment
    def ed(self, q, v0=0, v1=-1, max_lag=0, traceback=0):
        """gwf_ed: distance, -1 when no alignment; raises GwfError for error codes."""
        b = q.encode() if isinstance(q, str) else bytes(q)
        r = lib().gwf_ed(None, self.ptr, len(b), b, v0, v1, max_lag, traceback)
        if r < -1:
            raise GwfError(r, last_error())
        return r

    def ed_batch(self, reads, v0, v1=-1, mode=MODE_AUTO, flags=0, concat=True, max_lag=0, use_graph=0,
                 warps_per_read=0):
        """Batch alignment. reads: list of bytes, or (cat, offs, lens). Returns (dist, status).
        warps_per_read: 1, 2, 4 or 8 warps align each read of the persistent form (0 = per
        length bucket: tuned for MODE_AUTO, else the library's default)."""
        if isinstance(reads, tuple):
            cat, offs, lens = reads
        else:
            cat, offs, lens = pack_reads(reads)
        n = len(lens)
        v0 = np.ascontiguousarray(np.broadcast_to(np.asarray(v0, dtype=np.int32), (n,)))
        dist = np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        opt = BatchOpts(mode=mode, flags=flags, use_graph=use_graph, warps_per_read=warps_per_read)
        if concat:
            rc = lib().gwf_ed_batch_concat(self.ptr, n, _ptr(cat), _ptr(offs), _ptr(lens), _ptr(v0), v1,
                                           max_lag, _ptr(dist), _ptr(st), ctypes.byref(opt))
        else:
            ptrs = (ctypes.c_char_p * max(n, 1))(*[ctypes.c_char_p(cat[o:o + l].tobytes()) for o, l in zip(offs, lens)])
            rc = lib().gwf_ed_batch(self.ptr, n, ptrs, _ptr(lens), _ptr(v0), v1, max_lag, _ptr(dist),
                                    _ptr(st), ctypes.byref(opt))
        if rc != 0:
            raise GwfError(rc, last_error())
        return dist, st

    def ed_strand(self, reads, v0, v1=-1, mode=MODE_AUTO, flags=0, max_lag=0, use_graph=0, warps_per_read=0):
        """Both-strand alignment (gwf_ed_batch_strand): each read and its reverse complement from
        v0. Returns (dist, status, strand), strand 0 = as given, 1 = reverse complement, -1 =
        none."""
        cat, offs, lens = reads if isinstance(reads, tuple) else pack_reads(reads)
        n = len(lens)
        v0 = np.ascontiguousarray(np.broadcast_to(np.asarray(v0, dtype=np.int32), (n,)))
        dist, st, strand = (np.zeros(n, dtype=np.int32) for _ in range(3))
        opt = BatchOpts(mode=mode, flags=flags, use_graph=use_graph, warps_per_read=warps_per_read)
        rc = lib().gwf_ed_batch_strand(self.ptr, n, _ptr(cat), _ptr(offs), _ptr(lens), _ptr(v0), v1, max_lag,
                                       _ptr(dist), _ptr(st), _ptr(strand), ctypes.byref(opt))
        if rc != 0:
            raise GwfError(rc, last_error())
        return dist, st, strand

    def ed_path(self, reads, v0, v1=-1, flags=0, max_nv=4096, as_arrays=False, max_ops=0):
        """Alignment with traceback (gwf_ed_batch_path; gwf_ed_batch_align when max_ops > 0).
        Returns (dist, status, end_off, paths), paths[i] = (vertices, arcs): the first
        min(path_n, max_nv) path vertices from v0 and the index in the indexed graph's arcs of the
        arc into each (-1 for the first). With max_ops > 0 a fifth item, cigars[i]: the read's
        CIGAR against its path text as a string ("12=1X3=2I..."), or None. as_arrays=True returns
        (dist, status, end_off, path_n, path_v, path_arc[, cigar_n, cigar]) as the library wrote
        them."""
        cat, offs, lens = reads if isinstance(reads, tuple) else pack_reads(reads)
        n = len(lens)
        v0 = np.ascontiguousarray(np.broadcast_to(np.asarray(v0, dtype=np.int32), (n,)))
        dist = np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        end_off = np.zeros(n, dtype=np.int32)
        path_n = np.zeros(n, dtype=np.int32)
        pv = np.zeros((max(n, 1), max(max_nv, 1)), dtype=np.int32)
        pa = np.zeros((max(n, 1), max(max_nv, 1)), dtype=np.int32)
        if max_ops > 0:
            cn = np.zeros(n, dtype=np.int32)
            cg = np.zeros((max(n, 1), max_ops), dtype=np.uint32)
            rc = lib().gwf_ed_batch_align(self.ptr, n, _ptr(cat), _ptr(offs), _ptr(lens), _ptr(v0), v1, flags, max_nv,
                                          max_ops, _ptr(dist), _ptr(st), _ptr(end_off), _ptr(path_n), _ptr(pv),
                                          _ptr(pa), _ptr(cn), _ptr(cg))
        else:
            rc = lib().gwf_ed_batch_path(self.ptr, n, _ptr(cat), _ptr(offs), _ptr(lens), _ptr(v0), v1, flags, max_nv,
                                         _ptr(dist), _ptr(st), _ptr(end_off), _ptr(path_n), _ptr(pv), _ptr(pa))
        if rc != 0:
            raise GwfError(rc, last_error())
        if as_arrays:
            out = (dist, st, end_off, path_n, pv[:n], pa[:n])
            return out + ((cn, cg[:n]) if max_ops > 0 else ())
        paths = [(pv[i, :min(path_n[i], max_nv)].copy(), pa[i, :min(path_n[i], max_nv)].copy()) for i in range(n)]
        if max_ops <= 0:
            return dist, st, end_off, paths
        cigars = [cigar_string(cg[i, :cn[i]]) if 0 <= cn[i] <= max_ops else None for i in range(n)]
        return dist, st, end_off, paths, cigars

# ---- one batch over several GPUs (one process per GPU, torch.distributed)
def partition_reads(lens, world, cost=None):
    """Cost-balanced split of a batch into `world` contiguous ranges of reads: the boundaries cut
    the running sum of the per-read cost (default ql^2, the work of a read grows with its length
    times its score) into equal parts. Contiguous ranges keep each rank's upload to its own
    bytes; inside a range the persistent queue orders the reads longest first. Returns
    [(start, end)] per rank."""
    lens = np.asarray(lens)
    n = len(lens)
    c = (lens.astype(np.float64) ** 2) if cost is None else np.asarray(cost, dtype=np.float64)
    cum = np.cumsum(c)
    total = float(cum[-1]) if n else 0.0
    cuts = [0] + [int(np.searchsorted(cum, total * k / world, side="left")) + 1 for k in range(1, world)] + [n]
    cuts = np.minimum(np.maximum.accumulate(np.array(cuts)), n)
    return [(int(cuts[k]), int(cuts[k + 1])) for k in range(world)]


def align_sharded(graph, reads, v0, v1=-1, mode=MODE_AUTO, flags=0, group=None, align_fn=None):
    """Aligns a batch that every rank holds, split across the ranks of torch.distributed's default
    group (or `group`) by partition_reads: each rank aligns its range on its own GPU, then the
    int32 distances and statuses are all-gathered (NCCL over NVLink with CUDA tensors, gloo on
    CPU), so every rank returns the full (dist, status). The graph is replicated: every rank has
    indexed its own copy. Without an initialised process group this is graph.ed_batch.
    align_fn(cat, offs, lens, v0) -> (dist, status) stands in for graph.ed_batch (tests)."""
    cat, offs, lens = reads if isinstance(reads, tuple) else pack_reads(reads)
    n = len(lens)
    v0 = np.ascontiguousarray(np.broadcast_to(np.asarray(v0, dtype=np.int32), (n,)))
    run = align_fn or (lambda c, o, l, v: graph.ed_batch((c, o, l), v, v1=v1, mode=mode, flags=flags))
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return run(cat, offs, lens, v0)
    import torch
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    parts = partition_reads(lens, world)
    a, b = parts[rank]
    d, st = run(cat, np.ascontiguousarray(offs[a:b]), np.ascontiguousarray(lens[a:b]), np.ascontiguousarray(v0[a:b]))
    width = max(1, max(e - s for s, e in parts))
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    buf = torch.full((2, width), -1, dtype=torch.int32)
    buf[0, :b - a] = torch.from_numpy(np.asarray(d, dtype=np.int32))
    buf[1, :b - a] = torch.from_numpy(np.asarray(st, dtype=np.int32))
    buf = buf.to(device)
    out = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    dist_all = np.empty(n, dtype=np.int32)
    st_all = np.empty(n, dtype=np.int32)
    for r, (s0, e0) in enumerate(parts):
        x = out[r].cpu().numpy()
        dist_all[s0:e0] = x[0, :e0 - s0]
        st_all[s0:e0] = x[1, :e0 - s0]
    return dist_all, st_all


CIGAR_OPS = {0: "M", 1: "I", 2: "D", 7: "=", 8: "X"}


def cigar_string(runs):
    """BAM-coded runs (len << 4 | op) as a CIGAR string."""
    return "".join("%d%s" % (int(x) >> 4, CIGAR_OPS[int(x) & 15]) for x in runs)


TUNE_BUCKET_MAX = (1500, 3000, 6000, 12000, None)  # upper ql bound (exclusive) per bucket


def tune(graph, reads, v0, v1=-1, max_reads_per_bucket=0, json_path=None):
    """gwf_tune: times the launch shapes per read-length bucket on these reads and keeps the
    fastest for GWF_MODE_AUTO. reads: list of bytes or (cat, offs, lens). Returns tune_table()."""
    cat, offs, lens = reads if isinstance(reads, tuple) else pack_reads(reads)
    n = len(lens)
    v0 = np.ascontiguousarray(np.broadcast_to(np.asarray(v0, dtype=np.int32), (n,)))
    rc = lib().gwf_tune(graph.ptr, n, _ptr(cat), _ptr(offs), _ptr(lens), _ptr(v0), v1, max_reads_per_bucket,
                        json_path.encode() if json_path else None)
    if rc != 0:
        raise GwfError(rc, last_error())
    return tune_table()


def tune_load(json_path, device=-1):
    rc = lib().gwf_tune_load(json_path.encode(), device)
    if rc != 0:
        raise GwfError(rc, last_error())
    return tune_table(device)


def tune_table(device=-1, with_warps=False):
    """{bucket: (form, ctas_per_sm, reads_per_s)} for the buckets with an entry; with_warps=True
    adds the bucket's warps per read: (form, ctas_per_sm, warps_per_read, reads_per_s)."""
    out = {}
    for b in range(len(TUNE_BUCKET_MAX)):
        f, c, nw, r = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_float()
        if lib().gwf_tune_get_shape(device, b, ctypes.byref(f), ctypes.byref(c), ctypes.byref(nw),
                                    ctypes.byref(r)) == 1:
            out[b] = (f.value, c.value, nw.value, r.value) if with_warps else (f.value, c.value, r.value)
    return out


def tune_clear(device=-1):
    lib().gwf_tune_clear(device)


class ResidentBatch:
    """gwf_batch_*: reads uploaded once, run many times (device-timed)."""

    def __init__(self, graph, cat, offs, lens, v0, v1=-1, mode=MODE_AUTO, flags=0):
        self.graph = graph
        self.n = len(lens)
        self.opt = BatchOpts(mode=mode, flags=flags)
        v0 = np.ascontiguousarray(np.broadcast_to(np.asarray(v0, dtype=np.int32), (self.n,)))
        self.ptr = lib().gwf_batch_create(graph.ptr, self.n, _ptr(cat), _ptr(offs), _ptr(lens), _ptr(v0),
                                          v1, ctypes.byref(self.opt))
        if not self.ptr:
            raise GwfError(GWF_E_CUDA, last_error())

    def run(self, mode=None, flags=None, ctas_per_sm=0, use_graph=0, warps_per_read=0):
        opt = BatchOpts(mode=self.opt.mode if mode is None else mode,
                        flags=self.opt.flags if flags is None else flags, ctas_per_sm=ctas_per_sm,
                        use_graph=use_graph, warps_per_read=warps_per_read)
        ms = ctypes.c_float(0)
        rc = lib().gwf_batch_run(self.ptr, ctypes.byref(opt), ctypes.byref(ms))
        if rc != 0:
            raise GwfError(rc, last_error())
        return ms.value

    def results(self):
        dist = np.zeros(self.n, dtype=np.int32)
        st = np.zeros(self.n, dtype=np.int32)
        rc = lib().gwf_batch_results(self.ptr, _ptr(dist), _ptr(st))
        if rc != 0:
            raise GwfError(rc, last_error())
        return dist, st

    def steps(self):
        s = np.zeros(self.n, dtype=np.int32)
        rc = lib().gwf_batch_steps(self.ptr, _ptr(s))
        if rc != 0:
            raise GwfError(rc, last_error())
        return s

    def launches(self):
        return lib().gwf_batch_launches(self.ptr)

    def close(self):
        if self.ptr:
            lib().gwf_batch_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """gwf_srv_*: continuous batching on a resident graph."""

    def __init__(self, graph, arena_budget_bytes=0, max_inflight_reads=0, flags=0, max_lag=0, warps_per_read=0):
        self.graph = graph
        opt = SrvOpts(arena_budget_bytes=arena_budget_bytes, max_inflight_reads=max_inflight_reads, flags=flags,
                      max_lag=max_lag, warps_per_read=warps_per_read)
        self.ptr = lib().gwf_srv_create(graph.ptr, ctypes.byref(opt))
        if not self.ptr:
            raise GwfError(GWF_E_CUDA, last_error())

    def submit(self, reads, v0, v1=-1):
        cat, offs, lens = reads if isinstance(reads, tuple) else pack_reads(reads)
        n = len(lens)
        v0 = np.ascontiguousarray(np.broadcast_to(np.asarray(v0, dtype=np.int32), (n,)))
        rid = lib().gwf_srv_submit(self.ptr, n, _ptr(cat), _ptr(offs), _ptr(lens), _ptr(v0), v1)
        if rid < 0:
            raise GwfError(rid, last_error())
        return rid, n

    def wait(self, rid, n, timeout_s=60.0):
        dist = np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        rc = lib().gwf_srv_wait(self.ptr, rid, _ptr(dist), _ptr(st), timeout_s)
        if rc != 1:
            raise GwfError(rc, last_error())
        return dist, st

    def poll(self, rid, n):
        dist = np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        rc = lib().gwf_srv_poll(self.ptr, rid, _ptr(dist), _ptr(st))
        if rc < 0:
            raise GwfError(rc, last_error())
        return (dist, st) if rc == 1 else None

    def strand(self, rid, n):
        """Strand per read of a finished request of a both-strand server (GWF_F_BOTH_STRANDS)."""
        out = np.zeros(n, dtype=np.int32)
        rc = lib().gwf_srv_strand(self.ptr, rid, _ptr(out))
        if rc != 0:
            raise GwfError(rc, last_error())
        return out

    def times(self, rid):
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        rc = lib().gwf_srv_times(self.ptr, rid, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        if rc != 0:
            raise GwfError(rc, last_error())
        return a.value, b.value, c.value

    STATS = ("launches", "retries", "arena_used", "published", "completed", "in_flight", "pending_requests",
             "kernel_running")

    def stats(self):
        """The server's counters (gwf_srv_stats) as a dict."""
        out = np.zeros(len(self.STATS), dtype=np.int64)
        rc = lib().gwf_srv_stats(self.ptr, _ptr(out), len(out))
        if rc < 0:
            raise GwfError(rc, last_error())
        return dict(zip(self.STATS, (int(x) for x in out)))

    def close(self):
        if self.ptr:
            lib().gwf_srv_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- synthetic inputs (include/gwfa_synth.h)
class SynthGraph:
    """Seeded variation graph; .gfa is the GFA text, segments s1..sN."""

    def __init__(self, backbone_len, site_every=500, p_snp=0.7, indel_max=10, sv_every=0, sv_min=1000,
                 sv_max=5000, seed=1):
        self.ptr = lib().gwf_synth_graph_new(backbone_len, site_every, p_snp, indel_max, sv_every, sv_min, sv_max, seed)
        if not self.ptr:
            raise GwfError(GWF_E_BAD_INPUT, "bad synthetic graph parameters")
        n = lib().gwf_synth_graph_gfa(self.ptr, None, 0)
        buf = ctypes.create_string_buffer(n)
        lib().gwf_synth_graph_gfa(self.ptr, buf, n)
        self.gfa = buf.raw[:n]

    def reads(self, n, len_kind=0, len_a=1000, len_b=0.0, len_min=1, len_max=1 << 30, err_min=0.01,
              err_max=0.01, seed=1, pinned=False):
        """Returns dict(cat, offs, lens, origin_seg, err)."""
        r = lib().gwf_synth_reads_new(self.ptr, n, len_kind, float(len_a), float(len_b), len_min, len_max,
                                      float(err_min), float(err_max), seed)
        tot = lib().gwf_synth_reads_bytes(r)
        if pinned:
            raw = lib().gwf_pinned_alloc(tot + 16)
            cat = np.ctypeslib.as_array((ctypes.c_uint8 * (tot + 16)).from_address(raw))
        else:
            raw = None
            cat = np.zeros(tot + 16, dtype=np.uint8)
        offs = np.zeros(n, dtype=np.int64)
        lens = np.zeros(n, dtype=np.int32)
        org = np.zeros(n, dtype=np.int32)
        err = np.zeros(n, dtype=np.float32)
        lib().gwf_synth_reads_copy(r, _ptr(cat), _ptr(offs), _ptr(lens), _ptr(org), _ptr(err))
        lib().gwf_synth_reads_free(r)
        return {"cat": cat, "offs": offs, "lens": lens, "origin_seg": org, "err": err, "pinned_ptr": raw}

    def close(self):
        if self.ptr:
            lib().gwf_synth_graph_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def workload_spec(kind, n=None, seed=None):
    """Parameters of the five seeded benchmark workloads, as plain data (no library call):
    {"graph": gwf_synth_graph_new arguments, "parts": [gwf_synth_reads_new arguments after the
    graph, one tuple per read set]}.

    config1: 100 kbp graph, 1,000 x 1 kbp reads at 1%
    config2: same graph, 100,000 x 1 kbp reads (50,000 at 5%, 50,000 at 10%)
    config3: same graph, 200,000 reads, lognormal length (median 2 kbp, sigma 0.6) in
             [500, 10000], error U[1%, 10%]
    config4: 5 Mbp graph (site every 50 bp, SV every 50 kbp), 20,000 x 10 kbp reads at 5%
    config5: config-4 graph, reads of U[500, 20000] bp at U[1%, 10%] (serving requests)
    """
    if kind in ("config1", "config2", "config3"):
        graph = (100_000, 500, 0.7, 10, 0, 0, 0, 1)
    elif kind in ("config4", "config5"):
        graph = (5_000_000, 50, 0.7, 20, 50_000, 1000, 5000, 4)
    else:
        raise ValueError(kind)
    if kind == "config1":
        parts = [(n or 1000, 0, 1000, 0, 1000, 1000, 0.01, 0.01, seed if seed is not None else 11)]
    elif kind == "config2":
        h = (n or 100_000) // 2
        parts = [(h, 0, 1000, 0, 1000, 1000, 0.05, 0.05, 21 if seed is None else seed),
                 ((n or 100_000) - h, 0, 1000, 0, 1000, 1000, 0.10, 0.10, 22 if seed is None else seed + 1)]
    elif kind == "config3":
        parts = [(n or 200_000, 1, 2000, 0.6, 500, 10000, 0.01, 0.10, 3 if seed is None else seed)]
    elif kind == "config4":
        parts = [(n or 20_000, 0, 10000, 0, 10000, 10000, 0.05, 0.05, 41 if seed is None else seed)]
    else:
        parts = [(n or 1000, 2, 500, 20000, 500, 20000, 0.01, 0.10, 5 if seed is None else seed)]
    return {"graph": graph, "parts": parts}


def concat_parts(parts, alloc=None):
    """Read sets (dicts of cat, offs, lens, origin_seg, err) -> one concatenated set; alloc(nbytes)
    returns the uint8 array that receives the bytes (pinned memory), default numpy."""
    if len(parts) == 1:
        p = parts[0]
        return p["cat"], p["offs"], p["lens"], p["origin_seg"], p["err"]
    base = 0
    cats, offss = [], []
    for p in parts:
        tot = int(p["offs"][-1] + p["lens"][-1]) if len(p["lens"]) else 0
        cats.append(p["cat"][:tot])
        offss.append(p["offs"] + base)
        base += tot
    cat = np.concatenate(cats + [np.zeros(16, np.uint8)])
    if alloc is not None:
        pc = alloc(len(cat))
        pc[:] = cat
        cat = pc
    return (cat, np.concatenate(offss), np.concatenate([p["lens"] for p in parts]),
            np.concatenate([p["origin_seg"] for p in parts]), np.concatenate([p["err"] for p in parts]))


def _pinned_array(nbytes):
    raw = lib().gwf_pinned_alloc(nbytes)
    return np.ctypeslib.as_array((ctypes.c_uint8 * nbytes).from_address(raw))


def load_workload(kind, n=None, seed=None, pinned=False):
    """Synthetic workloads of the five benchmark configurations (seeded; workload_spec).
    Returns dict(graph=Graph, synth=SynthGraph, cat, offs, lens, v0, err)."""
    spec = workload_spec(kind, n, seed)
    sg = SynthGraph(*spec["graph"][:7], seed=spec["graph"][7])
    g = Graph.from_gfa_text(sg.gfa)
    seg2v = g.vertex_of_segment()
    parts = [sg.reads(*pa[:8], seed=pa[8], pinned=pinned) for pa in spec["parts"]]
    cat, offs, lens, org, err = concat_parts(parts, _pinned_array if pinned else None)
    v0 = np.array([seg2v[int(o)] for o in org], dtype=np.int32)
    return {"graph": g, "synth": sg, "cat": cat, "offs": offs, "lens": lens, "v0": v0, "err": err}
