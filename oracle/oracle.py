"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of oracle/liboracle.so, the CPU restatement of the
reference GWFA routine (gwf-ed.cu) and an independent dynamic program (see gwf_oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, always as
the checker or the timed CPU baseline, never as the product path.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

F_TMP_DROP = 0x001
F_SWAP_DROP = 0x002
F_UNSAFE_MASK = 0x7F0
F_NONTERM = 0x400
O_EXACT_START = 0x1
O_ENTRY_KEY = 0x2


class Stats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int32), ("flags", ctypes.c_int32), ("W", ctypes.c_int64),
                ("E", ctypes.c_int64), ("n_keys", ctypes.c_int64), ("max_na", ctypes.c_int32),
                ("max_nB", ctypes.c_int32), ("max_nA", ctypes.c_int32), ("max_ntmp", ctypes.c_int32),
                ("max_nintv", ctypes.c_int32), ("pad", ctypes.c_int32)]


class _Arc(ctypes.Structure):
    _fields_ = [("a", ctypes.c_uint64), ("o", ctypes.c_int32)]


class _Graph(ctypes.Structure):
    _fields_ = [("n_vtx", ctypes.c_uint32), ("n_arc", ctypes.c_uint32),
                ("len", ctypes.POINTER(ctypes.c_uint32)), ("src", ctypes.POINTER(ctypes.c_uint32)),
                ("seq", ctypes.POINTER(ctypes.c_char_p)), ("arc", ctypes.POINTER(_Arc)),
                ("aux", ctypes.POINTER(ctypes.c_uint64))]


_lib = None


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "gwf_oracle.c")
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
            subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        L.gwfo_index.argtypes = [P]
        L.gwfo_index_free.argtypes = [P]
        L.gwfo_ed.argtypes = [P, ctypes.c_int32, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32,
                              ctypes.c_int32, P]
        L.gwfo_ed.restype = ctypes.c_int32
        L.gwfo_ed_lag.argtypes = [P, ctypes.c_int32, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32,
                                  ctypes.c_int32, ctypes.c_int32, P]
        L.gwfo_ed_lag.restype = ctypes.c_int32
        L.gwfo_ed_batch.argtypes = [P, ctypes.c_int32, P, P, P, P, ctypes.c_int32, ctypes.c_int32, P, P,
                                    ctypes.c_int32]
        L.gwfo_ed_batch.restype = ctypes.c_int32
        L.gwfo_dp.argtypes = [P, ctypes.c_int32, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32]
        L.gwfo_dp.restype = ctypes.c_int32
        _lib = L
    return _lib


class OracleGraph:
    """Oracle-owned copy of a graph: seqs (list of bytes per vertex), arcs [(v, w, overlap)]."""

    def __init__(self, seqs, arcs):
        n = len(seqs)
        self._lens = (ctypes.c_uint32 * max(n, 1))(*[len(s) for s in seqs])
        self._src = (ctypes.c_uint32 * max(n, 1))(*[2 * i for i in range(n)])
        self._bufs = [ctypes.create_string_buffer(bytes(s)) for s in seqs]
        self._seqp = (ctypes.c_char_p * max(n, 1))(*[ctypes.cast(b, ctypes.c_char_p) for b in self._bufs])
        self._arcs = (_Arc * max(len(arcs), 1))(*[_Arc((int(v) << 32) | int(w), int(o)) for v, w, o in arcs])
        g = _Graph()
        g.n_vtx, g.n_arc = n, len(arcs)
        g.len = ctypes.cast(self._lens, ctypes.POINTER(ctypes.c_uint32))
        g.src = ctypes.cast(self._src, ctypes.POINTER(ctypes.c_uint32))
        g.seq = ctypes.cast(self._seqp, ctypes.POINTER(ctypes.c_char_p))
        g.arc = ctypes.cast(self._arcs, ctypes.POINTER(_Arc))
        g.aux = None
        self._g = g
        self.ptr = ctypes.pointer(g)
        lib().gwfo_index(self.ptr)

    @classmethod
    def from_graph(cls, graph):
        """Copy of a product Graph (gwfa_b200.Graph): same vertices and arcs."""
        return cls(graph.seqs(), graph.arcs())

    def aux(self):
        return np.array([self._g.aux[i] for i in range(self._g.n_vtx)], dtype=np.uint64)

    def arcs_sorted(self):
        return [(self._g.arc[i].a >> 32, self._g.arc[i].a & 0xffffffff, self._g.arc[i].o) for i in range(self._g.n_arc)]

    def ed(self, q, v0, v1=-1, exact_start=False, max_lag=0, entry_key=False):
        """max_lag > 0: the product's lag pruning (GWF_F_MAX_LAG) after each step. entry_key: the
        product's arrival key (differs from the reference's only where the arcs into a vertex
        carry different overlaps)."""
        b = q.encode() if isinstance(q, str) else bytes(q)
        st = Stats()
        opts = (O_EXACT_START if exact_start else 0) | (O_ENTRY_KEY if entry_key else 0)
        d = lib().gwfo_ed_lag(self.ptr, len(b), b, v0, v1, opts, max_lag, ctypes.byref(st))
        return d, st

    def ed_batch(self, cat, offs, lens, v0, v1=-1, exact_start=False, threads=0, stats=True, entry_key=False):
        n = len(lens)
        cat = np.ascontiguousarray(cat, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.int64)
        lens = np.ascontiguousarray(lens, dtype=np.int32)
        v0 = np.ascontiguousarray(np.broadcast_to(np.asarray(v0, dtype=np.int32), (n,)))
        dist = np.zeros(n, dtype=np.int32)
        st = (Stats * max(n, 1))() if stats else None
        used = lib().gwfo_ed_batch(self.ptr, n, cat.ctypes.data, offs.ctypes.data, lens.ctypes.data,
                                   v0.ctypes.data, v1,
                                   (O_EXACT_START if exact_start else 0) | (O_ENTRY_KEY if entry_key else 0),
                                   dist.ctypes.data, st, threads)
        return dist, st, used

    def dp(self, q, v0, v1=-1):
        b = q.encode() if isinstance(q, str) else bytes(q)
        return lib().gwfo_dp(self.ptr, len(b), b, v0, v1)

    def __del__(self):
        try:
            lib().gwfo_index_free(self.ptr)
        except Exception:
            pass


def _synth_sigs(L):
    P, I32, I64, U64, DBL = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double
    for name, res, args in (("gwf_synth_graph_new", P, [I64, I32, DBL, I32, I32, I32, I32, U64]),
                            ("gwf_synth_graph_free", None, [P]),
                            ("gwf_synth_graph_gfa", I64, [P, ctypes.c_char_p, I64]),
                            ("gwf_synth_reads_new", P, [P, I32, I32, DBL, DBL, I32, I32, DBL, DBL, U64]),
                            ("gwf_synth_reads_bytes", I64, [P]),
                            ("gwf_synth_reads_copy", None, [P, P, P, P, P, P]),
                            ("gwf_synth_reads_free", None, [P])):
        f = getattr(L, name)
        f.restype, f.argtypes = res, args


def parse_gfa(text):
    """Segments and links of a GFA text whose links all join forward strands ("L a + b + nM" or
    "*"), as the seeded generator writes: (seqs in S-line order, arcs (v, w, overlap on w)).
    Vertex i is the i-th S line."""
    seqs, name2v, links = [], {}, []
    for line in text.split(b"\n"):
        f = line.rstrip(b"\r").split(b"\t")
        if f[0] == b"S":
            name2v[f[1]] = len(seqs)
            seqs.append(f[2])
        elif f[0] == b"L":
            if f[2] != b"+" or f[4] != b"+":
                raise ValueError("parse_gfa: reverse-strand link")
            ov = f[5] if len(f) > 5 else b"*"
            links.append((f[1], f[3], 0 if ov in (b"*", b"") else int(ov.rstrip(b"M"))))
    return seqs, [(name2v[a], name2v[b], o) for a, b, o in links]


def synth_workload(spec):
    """The seeded workload of a spec (the product package's workload_spec: graph arguments and
    read sets), made with the generator compiled into liboracle.so, as an OracleGraph plus the
    concatenated reads. Loads no product library: the CPU baseline's own input path. Vertices
    are numbered in S-line order; the distances equal those on the product's loader numbering."""
    L = lib()
    _synth_sigs(L)
    ga = spec["graph"]
    sg = L.gwf_synth_graph_new(*ga)
    try:
        n = L.gwf_synth_graph_gfa(sg, None, 0)
        buf = ctypes.create_string_buffer(n)
        L.gwf_synth_graph_gfa(sg, buf, n)
        seqs, arcs = parse_gfa(buf.raw[:n])
        parts = []
        for pa in spec["parts"]:
            r = L.gwf_synth_reads_new(sg, *pa)
            tot = L.gwf_synth_reads_bytes(r)
            m = pa[0]
            cat = np.zeros(tot + 16, dtype=np.uint8)
            offs, lens = np.zeros(m, dtype=np.int64), np.zeros(m, dtype=np.int32)
            org, err = np.zeros(m, dtype=np.int32), np.zeros(m, dtype=np.float32)
            L.gwf_synth_reads_copy(r, cat.ctypes.data, offs.ctypes.data, lens.ctypes.data, org.ctypes.data,
                                   err.ctypes.data)
            L.gwf_synth_reads_free(r)
            parts.append((cat[:tot], offs, lens, org))
    finally:
        L.gwf_synth_graph_free(sg)
    base, cats = 0, []
    offs_all, lens_all, org_all = [], [], []
    for cat, offs, lens, org in parts:
        cats.append(cat)
        offs_all.append(offs + base)
        base += len(cat)
        lens_all.append(lens)
        org_all.append(org)
    cat = np.concatenate(cats + [np.zeros(16, np.uint8)])
    return {"graph": OracleGraph(seqs, arcs), "cat": cat, "offs": np.concatenate(offs_all),
            "lens": np.concatenate(lens_all), "v0": np.concatenate(org_all).astype(np.int32)}


def stats_arrays(st, n):
    """Stats array -> dict of numpy arrays."""
    out = {}
    for name, _ in Stats._fields_:
        out[name] = np.array([getattr(st[i], name) for i in range(n)])
    return out
