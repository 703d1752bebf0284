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
SOURCES = ["mt_capi.cu", "mt_batches.cu", "mt_serve.cu", "mt_host.cu", "mt_bulk.cu", "mt_merge.cu",
           "mt_grouped.cu"]
HEADERS = ["mt_tile.cuh", "mt_pool.cuh", "mt_node.cuh", "mt_suffix.cuh", "mt_tree.cuh", "mt_internal.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
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
    # One object per translation unit, compiled in parallel, then linked; an
    # object newer than its source and every header, and built with the same
    # flags, is kept.
    headers = [d for d in deps if not d.endswith(".cu")]
    stamp = os.path.join(CSRC, ".objects_built_with")
    flags = " ".join([*NVCC_FLAGS, *extra_flags])
    same_flags = os.path.exists(stamp) and open(stamp).read() == flags
    objs, procs = [], []
    for src in SOURCES:
        obj = os.path.join(CSRC, src.replace(".cu", ".o"))
        objs.append(obj)
        if not force and same_flags and not _stale(obj, [os.path.join(CSRC, src), *headers]):
            continue
        cmd = ["nvcc", *NVCC_FLAGS, *extra_flags, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append(subprocess.Popen(cmd))
    for pr in procs:
        if pr.wait() != 0:
            raise subprocess.CalledProcessError(pr.returncode, "nvcc")
    with open(stamp, "w") as f:
        f.write(flags)
    link = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.check_call(link)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
