"""The universal-bench adapter (include/universal_bench/gpu_masstree_adapter.hpp) compiles
against libmt_b200.so and parses the reference adapter's arguments; on a GPU
the check program runs every adapter call against a host model, and the
allocator line of print_stats parses the way the reference's evaluate.py
reads it (the token holding '%', stripped of '()%')."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "adapter_check.cpp")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(tmp_path):
    exe = str(tmp_path / "adapter_check")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", SRC, "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(CUDA, "include"), "-L", os.path.join(ROOT, "indexingpu_b200"), "-lmt_b200", "-L",
           os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{os.path.join(ROOT, 'indexingpu_b200')}",
           f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}", "-o", exe]
    subprocess.check_call(cmd)
    return exe


def _space_values(stdout):
    """evaluate.py's parse of allocator lines."""
    out = []
    for line in stdout.split("\n"):
        if "simple_slab" in line:
            for token in line.split(" "):
                if "%" in token:
                    out.append(float(re.sub(r"[()%]", "", token)))
                    break
    return out


def test_adapter_arguments(tmp_path):
    """Argument checks run without a GPU (device checks are skipped there)."""
    out = subprocess.run([_build(tmp_path)], capture_output=True, text=True, timeout=120,
                         env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert out.returncode == 0, out.stdout + out.stderr
    assert "    tile_size=32" in out.stdout and "    merge_level=2" in out.stdout
    assert "    lookup_concurrent=1" in out.stdout and "    write_tile_size=16" in out.stdout
    assert "0 mismatches" in out.stdout


@pytest.mark.gpu
def test_adapter_runs_every_call(tmp_path):
    out = subprocess.run([_build(tmp_path)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "adapter: 0 mismatches" in out.stdout
    space = _space_values(out.stdout)
    assert len(space) == 2
    assert 0.0 < space[0] < 100.0  # the populated tree
    assert space[1] < space[0]      # a re-initialized tree holds only its root
