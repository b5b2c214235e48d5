"""Shared fixtures: the product package (loaded from its in-tree directory), the oracle, and
workload helpers. The `gpu` marker tags tests that need a B200."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
PKG_DIR = os.path.join(ROOT, "gwfa-cuda-version_b200")
GOLD = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU")


def load_pkg():
    if "gwfa_b200" in sys.modules:
        return sys.modules["gwfa_b200"]
    spec = importlib.util.spec_from_file_location("gwfa_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gwfa_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    d = os.path.join(ROOT, "oracle")
    if d not in sys.path:
        sys.path.insert(0, d)
    import oracle
    return oracle


@pytest.fixture(scope="session")
def G():
    return load_pkg()


@pytest.fixture(scope="session")
def O():
    return load_oracle()


def read_fasta(path):
    reads = []
    for line in open(path, "rb"):
        line = line.rstrip(b"\r\n")
        if line.startswith(b">"):
            reads.append(b"")
        elif reads:
            reads[-1] += line
    return reads


def read_golden(name):
    """tests/golden/ref_<name>.txt -> (indices, distances) or (None, distances)."""
    rows = [l.split() for l in open(os.path.join(GOLD, name)) if l.strip() and not l.startswith("#")]
    if len(rows[0]) == 1:
        return None, [int(r[0]) for r in rows]
    return [int(r[0]) for r in rows], [int(r[1]) for r in rows]
