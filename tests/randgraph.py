"""Seeded small random graphs and reads for exhaustive parity cases (DAGs and cycles, short
vertices that trigger the reference start-state behaviour, non-ACGT and lower-case bytes)."""
import random


def rand_graph(rng, nv, maxlen, cyclic=False, alpha="ACGT", overlap="zero"):
    """overlap: "zero" (every arc enters its target at offset 0), "uniform" (all arcs into a
    vertex share one offset in [0, len - 1], as GFA links "nM" give), or "mixed" (each arc its
    own offset)."""
    seqs = ["".join(rng.choice(alpha) for _ in range(rng.randint(1, maxlen))).encode() for _ in range(nv)]
    ow = [rng.randrange(len(s)) if overlap == "uniform" else 0 for s in seqs]
    arcs = {}
    for v in range(nv):
        for _ in range(rng.randint(0, 3)):
            w = rng.randrange(nv) if cyclic else rng.randint(min(v + 1, nv - 1), nv - 1)
            if w == v and not cyclic:
                continue
            arcs[(v, w)] = rng.randrange(len(seqs[w])) if overlap == "mixed" else ow[w]
    return seqs, sorted((v, w, o) for (v, w), o in arcs.items())


def walk_text(rng, seqs, arcs, v0, length):
    """The text of a random walk from offset 0 of v0: each later vertex from its arc's offset."""
    out = {}
    for v, w, o in arcs:
        out.setdefault(v, []).append((w, o))
    s, v, o = b"", v0, 0
    while len(s) < length:
        s += seqs[v][o:]
        if v not in out:
            break
        v, o = rng.choice(out[v])
    return s[:length]


def walk_read(rng, seqs, arcs, v0, length, err):
    s = walk_text(rng, seqs, arcs, v0, length)
    r = bytearray()
    for c in s:
        x = rng.random()
        if x < err * 0.6:
            r.append(rng.choice(b"ACGT"))
        elif x < err * 0.8:
            r.append(rng.choice(b"ACGT"))
            r.append(c)
        elif x < err:
            pass
        else:
            r.append(c)
    return bytes(r) or b"A"


def cases(seed, n, v1_prob=0.0, overlap="zero"):
    """Yields (seqs, arcs, v0, v1, read) tuples."""
    rng = random.Random(seed)
    for _ in range(n):
        nv = rng.randint(1, 12)
        alpha = rng.choice(["ACGT", "ACGT", "ACGTN", "ACgt", "AC"])
        seqs, arcs = rand_graph(rng, nv, rng.choice([3, 8, 40]), rng.random() < 0.3, alpha, overlap)
        v0 = rng.randrange(nv)
        q = walk_read(rng, seqs, arcs, v0, rng.randint(1, 80), rng.choice([0.0, 0.05, 0.2, 0.6]))
        if rng.random() < 0.1:
            q = bytes(rng.choice(b"ACGTN") for _ in range(rng.randint(1, 40)))
        v1 = rng.randrange(nv) if rng.random() < v1_prob else -1
        yield seqs, arcs, v0, v1, q
