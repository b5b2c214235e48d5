"""The C ABI: every symbol declared in include/*.h is exported; host-side logic that needs no
GPU (CSR index, argument validation, error codes)."""
import ctypes
import os
import re

import numpy as np

from conftest import ROOT


def declared_functions():
    names = []
    for h in ("gwfa.h", "gwfa_synth.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(gwf_\w+)\s*\(", src, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_every_declared_symbol(G):
    lib = G.lib()
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(G.SIGNATURES), set(names) ^ set(G.SIGNATURES)


def test_version_string(G):
    assert b"sm_100a" in G.lib().gwf_version()


def test_index_builds_reference_csr_without_gpu(G, O):
    """gwf_ed_index sorts arcs and fills aux like main.cu:246-270 even when the device upload
    is impossible (no GPU here); the oracle's own index agrees."""
    sg = G.SynthGraph(5_000, 60, 0.6, 8, 0, 0, 0, seed=3)
    g = G.Graph.from_gfa_text(sg.gfa)
    og = O.OracleGraph(g.seqs(), list(reversed(g.arcs())))
    g.index()
    assert g.aux() is not None
    assert np.array_equal(g.aux(), og.aux())
    assert g.arcs() == og.arcs_sorted()


def test_unindexed_graph_and_bad_arguments(G):
    g = G.Graph.from_gfa_text(b"S\ta\tACGT\n")
    L = G.lib()
    assert L.gwf_ed(None, g.ptr, 4, b"ACGT", 0, -1, 0, 1) == G.GWF_E_UNSUPPORTED  # traceback
    assert L.gwf_ed(None, g.ptr, 0, b"", 0, -1, 0, 0) == G.GWF_E_BAD_INPUT
    assert L.gwf_ed(None, g.ptr, 4, b"ACGT", 5, -1, 0, 0) == G.GWF_E_BAD_INPUT
    r = L.gwf_ed(None, g.ptr, 4, b"ACGT", 0, -1, 0, 0)
    assert r in (G.GWF_E_NOT_INDEXED, G.GWF_E_CUDA)
    assert G.last_error()


def test_synthetic_reads_are_deterministic(G):
    sg = G.SynthGraph(30_000, 500, 0.7, 10, seed=1)
    a = sg.reads(50, 0, 800, 0, 800, 800, 0.05, 0.05, seed=9)
    b = sg.reads(50, 0, 800, 0, 800, 800, 0.05, 0.05, seed=9)
    assert np.array_equal(a["cat"], b["cat"]) and np.array_equal(a["origin_seg"], b["origin_seg"])
    assert abs(int(a["lens"].mean()) - 800) < 20
    c = sg.reads(200, 1, 2000, 0.6, 500, 10000, 0.01, 0.10, seed=3)
    assert c["lens"].min() >= 450 and c["lens"].max() <= 10600
    assert 0.01 <= c["err"].min() and c["err"].max() <= 0.10


def test_path_entry_point_arguments(G):
    """gwf_ed_batch_path checks its arguments before it needs a device: negative counts, missing
    output rows, an unindexed graph."""
    g = G.Graph.from_gfa_text(b"S\ta\tACGT\n")
    L = G.lib()
    i32 = lambda n: np.zeros(n, dtype=np.int32)
    cat = np.frombuffer(b"ACGT" + b"\0" * 16, dtype=np.uint8)
    offs = np.zeros(1, dtype=np.int64)
    lens, v0 = np.array([4], dtype=np.int32), i32(1)
    d, st, eo, pn = i32(1), i32(1), i32(1), i32(1)
    P = lambda a: a.ctypes.data
    assert L.gwf_ed_batch_path(g.ptr, -1, P(cat), P(offs), P(lens), P(v0), -1, 0, 4, P(d), P(st), P(eo), P(pn),
                               P(i32(4)), P(i32(4))) == G.GWF_E_BAD_INPUT
    assert L.gwf_ed_batch_path(g.ptr, 1, P(cat), P(offs), P(lens), P(v0), -1, 0, 4, P(d), P(st), P(eo), P(pn),
                               None, None) == G.GWF_E_BAD_INPUT
    assert L.gwf_ed_batch_path(g.ptr, 1, P(cat), P(offs), P(lens), P(v0), -1, 0, 4, P(d), P(st), P(eo), P(pn),
                               P(i32(4)), P(i32(4))) in (G.GWF_E_NOT_INDEXED, G.GWF_E_CUDA)
