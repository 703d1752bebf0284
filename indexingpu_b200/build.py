"""Build libmt_b200.so (the CUDA library behind the C ABI in include/mt_masstree.h).

The library is compiled in-tree for sm_100a only, so that the built file
travels with the source tree.  `python -m indexingpu_b200.build` rebuilds it.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libmt_b200.so")
SOURCES = ["mt_capi.cu"]
HEADERS = ["mt_tile.cuh", "mt_pool.cuh", "mt_node.cuh", "mt_suffix.cuh", "mt_tree.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=True, extra_flags=()):
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "mt_masstree.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = ["nvcc", *NVCC_FLAGS, *extra_flags, *[os.path.join(CSRC, s) for s in SOURCES], "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
