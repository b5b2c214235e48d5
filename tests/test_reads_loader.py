"""gwf_reads_load: FASTA (multi-line, CRLF, empty records, text before the first header) and
FASTQ, plain and gzip, parsed on one thread and on several, equal a straightforward Python
parse; the CLI reads through it."""
import gzip
import os

import numpy as np
import pytest


def parse_py(data):
    lines = data.replace(b"\r\n", b"\n").split(b"\n")
    first = next((ln for ln in lines if ln), b"")
    out = []
    if first.startswith(b"@"):
        st = 0
        for ln in lines:
            if st == 0:
                st = 1 if ln.startswith(b"@") else 0
            elif st == 1:
                out.append(ln)
                st = 2
            elif st == 2:
                st = 3
            else:
                st = 0
        return out
    cur = None
    for ln in lines:
        if ln.startswith(b">"):
            if cur is not None:
                out.append(cur)
            cur = b""
        elif cur is not None:
            cur += ln
    if cur is not None:
        out.append(cur)
    return out


def random_fasta(rng, n, crlf=False):
    parts = [b"junk line before the first header\n"]
    for i in range(n):
        parts.append(b">r%d some description\n" % i)
        L = int(rng.integers(0, 300)) if i % 17 else 0
        seq = bytes(rng.choice(list(b"ACGTN"), size=L).astype(np.uint8))
        w = int(rng.integers(10, 90))
        for j in range(0, L, w):
            parts.append(seq[j:j + w] + (b"\r\n" if crlf else b"\n"))
    return b"".join(parts)


def random_fastq(rng, n):
    parts = []
    for i in range(n):
        L = int(rng.integers(1, 300))
        seq = bytes(rng.choice(list(b"ACGT"), size=L).astype(np.uint8))
        parts.append(b"@q%d\n%s\n+\n%s\n" % (i, seq, b"@" * L))
    return b"".join(parts)


def as_list(cat, offs, lens):
    return [cat[o:o + l].tobytes() for o, l in zip(offs, lens)]


@pytest.mark.parametrize("threads", ["1", "4"])
@pytest.mark.parametrize("kind", ["fasta", "fasta_crlf", "fastq"])
@pytest.mark.parametrize("gz", [False, True])
def test_reads_equal_python_parse(G, tmp_path, monkeypatch, threads, kind, gz):
    monkeypatch.setenv("GWF_READS_THREADS", threads)
    rng = np.random.default_rng(hash((threads, kind, gz)) & 0xffff)
    data = random_fastq(rng, 300) if kind == "fastq" else random_fasta(rng, 300, crlf=kind == "fasta_crlf")
    path = tmp_path / ("r.fa.gz" if gz else "r.fa")
    if gz:
        with gzip.open(path, "wb") as f:
            f.write(data)
    else:
        path.write_bytes(data)
    cat, offs, lens = G.load_reads(str(path))
    assert as_list(cat, offs, lens) == parse_py(data)
    assert (np.diff(offs) >= 0).all() and (cat[-16:] == 0).all()


def test_large_fasta_on_all_cores(G, tmp_path, monkeypatch):
    monkeypatch.delenv("GWF_READS_THREADS", raising=False)
    rng = np.random.default_rng(5)
    data = random_fasta(rng, 40000)  # ~6 MB: more than one 4 MiB chunk
    path = tmp_path / "big.fa"
    path.write_bytes(data)
    cat, offs, lens = G.load_reads(str(path))
    assert as_list(cat, offs, lens) == parse_py(data)


def test_missing_file_is_an_error(G, tmp_path):
    with pytest.raises(G.GwfError):
        G.load_reads(str(tmp_path / "nope.fa"))
