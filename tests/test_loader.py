"""GFA loader parity: the product loader's gwf_graph_print dump equals the reference
`gwf-test -p` output (tests/golden/*.ref_dump.txt, from the reference binary)."""
import os

import pytest

from conftest import GOLD


@pytest.mark.parametrize("name", ["graph_1000", "grafo_test"])
def test_dump_matches_reference(G, name):
    g = G.Graph.from_gfa(os.path.join(GOLD, name + ".gfa"))
    ref = open(os.path.join(GOLD, name + ".ref_dump.txt"), "rb").read()
    assert g.dump() == ref


def test_in_memory_load_equals_file_load(G):
    text = open(os.path.join(GOLD, "graph_1000.gfa"), "rb").read()
    a = G.Graph.from_gfa_text(text).dump()
    b = G.Graph.from_gfa(os.path.join(GOLD, "graph_1000.gfa")).dump()
    assert a == b


def test_synthetic_graph_is_topologically_ordered(G):
    sg = G.SynthGraph(20_000, 100, 0.7, 10, 5000, 1000, 2000, seed=7)
    g = G.Graph.from_gfa_text(sg.gfa)
    assert g.n_vtx == G.lib().gwf_synth_graph_nseg(sg.ptr)
    for v, w, o in g.arcs():
        assert v < w and o == 0
    assert sum(len(s) for s in g.seqs()) == int(g.lens().sum())


def test_start_segment_and_orientation(G):
    gfa = b"S\ta\tAAAC\nS\tb\tGGT\nS\tc\tTTA\nL\ta\t+\tb\t+\t0M\nL\tb\t+\tc\t-\t0M\n"
    g = G.Graph.from_gfa_text(gfa, start_seg="b")
    # b first, then c on its reverse strand (reverse complement, main.cu:320-326)
    assert g.seqs() == [b"GGT", b"TAA"]
    assert g.arcs() == [(0, 1, 0)]
    with pytest.raises(G.GwfError):
        G.Graph.from_gfa_text(gfa, start_seg="zz")
    # a strand suffix picks the start strand: "b+" is the default, "c+" walks c+ -> b- -> a-
    assert G.Graph.from_gfa_text(gfa, start_seg="b+").seqs() == g.seqs()
    gc = G.Graph.from_gfa_text(gfa, start_seg="c+")
    assert gc.seqs() == [b"TTA", b"ACC", b"GTTT"] and gc.arcs() == [(0, 1, 0), (1, 2, 0)]
    gb = G.Graph.from_gfa_text(gfa, start_seg="b-")
    assert gb.seqs() == [b"ACC", b"GTTT"] and gb.arcs() == [(0, 1, 0)]
    assert G.Graph.from_gfa_text(gfa, start_seg="c-").seqs() == [b"TAA"]
    with pytest.raises(G.GwfError):
        G.Graph.from_gfa_text(gfa, start_seg="zz-")


def test_overlap_cigar_and_missing_overlap(G):
    gfa = b"S\ta\tAAACG\nS\tb\tCGTTT\nS\tc\tGG\nL\ta\t+\tb\t+\t2M\nL\tb\t+\tc\t+\n"
    g = G.Graph.from_gfa_text(gfa)
    assert (0, 1, 2) in g.arcs() and (1, 2, 0) in g.arcs()


def test_fasta_as_graph(G):
    g = G.Graph.from_gfa_text(b">x desc\nACGT\nAC\n>y\nTT\n")
    assert g.n_vtx == 1 and g.seqs() == [b"ACGTAC"]
