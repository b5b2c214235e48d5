"""Build recipe of libgwfa_b200.so (in-tree, sm_100a only).

    python gwfa-cuda-version_b200/build.py            # build if sources changed
    python gwfa-cuda-version_b200/build.py --force    # rebuild
    python gwfa-cuda-version_b200/build.py --ptxas    # print registers / spills per kernel
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgwfa_b200.so")
CLI = os.path.join(HERE, "gwf-b200")
SOURCES = ["gwf_runtime.cu", "gwf_serve.cu", "gwf_tune.cu", "gwf_noalloc.cu", "gfa_loader.cpp", "reads_loader.cpp",
           "synth.cpp"]
# gwf_cli.cpp is the command-line driver (a separate executable, not part of the library)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files += [os.path.join(HERE, "..", "include", f) for f in os.listdir(os.path.join(HERE, "..", "include"))]
    return [f for f in files if os.path.isfile(f)]


def needs_build():
    if not os.path.exists(LIB) or not os.path.exists(CLI):
        return True
    t = min(os.path.getmtime(LIB), os.path.getmtime(CLI))
    return any(os.path.getmtime(f) > t for f in _deps())


def build(force=False, ptxas=False, verbose=False):
    if not force and not ptxas and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-shared",
           "-o", LIB]
    if ptxas:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES] + ["-lz", "-lpthread"]
    if verbose or ptxas:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if ptxas:
        print(res.stdout + res.stderr)
    # the gwf-test compatible command-line driver, linked against the library next to it
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-O2", "-std=c++17", "-o", CLI, os.path.join(CSRC, "gwf_cli.cpp"), "-L" + HERE, "-lgwfa_b200",
           "-Wl,-rpath,$ORIGIN", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("g++ failed:\n" + res.stdout + res.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, ptxas="--ptxas" in sys.argv, verbose=True)
    print(LIB)
