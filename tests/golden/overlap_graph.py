"""Seeded GFA graphs whose links carry overlaps ("L a + b + nM"), with reads sampled along walks.

The reference enters the target of a link at the link's overlap on the target (gwf_gfa2gwf,
main.cu:333-334; gwf-ed.cu:1190-1199). The benchmark graphs have "0M" links only, so these
graphs cover the other case:
  uniform  every link into a segment has the same overlap (what GFA assemblies give: the
           overlap is a property of the junction), so the reference's arrival key names one
           graph position and its result does not depend on queue order;
  mixed    each link its own overlap, where the reference's result depends on its FIFO order.
Used by tests/golden/make_golden.py (reference goldens) and tests/test_gpu_parity.py.
"""
import random


def overlap_gfa(seed, n_seg=300, mode="uniform"):
    """(GFA text, segment sequences, links [(i, j, overlap)]) of a DAG in which segment i links to
    i + 1 and to up to two of i + 2 .. i + 4. Overlaps are below the length of both segments."""
    rng = random.Random(seed)
    seqs = ["".join(rng.choice("ACGT") for _ in range(rng.randint(8, 60))) for _ in range(n_seg)]
    links = set()
    for i in range(n_seg - 1):
        links.add((i, i + 1))
        for _ in range(rng.randint(0, 2)):
            j = rng.randint(i + 2, i + 4)
            if j < n_seg:
                links.add((i, j))
    links = sorted(links)
    srcmin = [10 ** 9] * n_seg
    for i, j in links:
        srcmin[j] = min(srcmin[j], len(seqs[i]))
    cap = [min(srcmin[j], len(seqs[j])) - 1 for j in range(n_seg)]
    ow = [rng.randint(0, max(0, min(c, 7))) for c in cap]
    out = []
    for i, j in links:
        o = ow[j] if mode == "uniform" else rng.randint(0, max(0, min(cap[j], 7)))
        out.append((i, j, o))
    text = "".join("S\ts%d\t%s\n" % (i + 1, s) for i, s in enumerate(seqs))
    text += "".join("L\ts%d\t+\ts%d\t+\t%dM\n" % (i + 1, j + 1, o) for i, j, o in out)
    return text.encode(), [s.encode() for s in seqs], out


def overlap_reads(seed, seqs, links, n=300):
    """n reads of 150-400 bases along random walks (the first segment from offset 0, each later
    one from its link's overlap), with errors at 0-10% (substitution:insertion:deletion 6:2:2).
    Returns (reads, start segment per read)."""
    rng = random.Random(seed)
    out = {}
    for i, j, o in links:
        out.setdefault(i, []).append((j, o))
    reads, starts = [], []
    for _ in range(n):
        v = rng.randrange(len(seqs) - 20)
        starts.append(v)
        length, err = rng.randint(150, 400), rng.uniform(0.0, 0.10)
        s, o = b"", 0
        while len(s) < length and v in out:
            s += seqs[v][o:]
            v, o = rng.choice(out[v])
        s = s[:length]
        r = bytearray()
        for c in s:
            x = rng.random()
            if x < err * 0.6:
                r.append(rng.choice(b"ACGT"))
            elif x < err * 0.8:
                r.append(rng.choice(b"ACGT"))
                r.append(c)
            elif x >= err:
                r.append(c)
        reads.append(bytes(r) or b"A")
    return reads, starts
