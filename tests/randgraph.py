"""Seeded small random graphs and reads for exhaustive parity cases (DAGs and cycles, short
vertices that trigger the reference start-state behaviour, non-ACGT and lower-case bytes)."""
import random


def rand_graph(rng, nv, maxlen, cyclic=False, alpha="ACGT"):
    seqs = ["".join(rng.choice(alpha) for _ in range(rng.randint(1, maxlen))).encode() for _ in range(nv)]
    arcs = set()
    for v in range(nv):
        for _ in range(rng.randint(0, 3)):
            w = rng.randrange(nv) if cyclic else rng.randint(min(v + 1, nv - 1), nv - 1)
            if w == v and not cyclic:
                continue
            arcs.add((v, w, 0))
    return seqs, sorted(arcs)


def walk_read(rng, seqs, arcs, v0, length, err):
    out = {}
    for v, w, _ in arcs:
        out.setdefault(v, []).append(w)
    s, v = b"", v0
    while len(s) < length:
        s += seqs[v]
        if v not in out:
            break
        v = rng.choice(out[v])
    s = s[:length]
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


def cases(seed, n, v1_prob=0.0):
    """Yields (seqs, arcs, v0, v1, read) tuples."""
    rng = random.Random(seed)
    for _ in range(n):
        nv = rng.randint(1, 12)
        alpha = rng.choice(["ACGT", "ACGT", "ACGTN", "ACgt", "AC"])
        seqs, arcs = rand_graph(rng, nv, rng.choice([3, 8, 40]), rng.random() < 0.3, alpha)
        v0 = rng.randrange(nv)
        q = walk_read(rng, seqs, arcs, v0, rng.randint(1, 80), rng.choice([0.0, 0.05, 0.2, 0.6]))
        if rng.random() < 0.1:
            q = bytes(rng.choice(b"ACGTN") for _ in range(rng.randint(1, 40)))
        v1 = rng.randrange(nv) if rng.random() < v1_prob else -1
        yield seqs, arcs, v0, v1, q
