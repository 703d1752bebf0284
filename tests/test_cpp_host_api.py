"""The C++ host mirror (include/mt/gpu_masstree.hpp) compiles and links against
libmt_b200.so; on a GPU the small program also runs and checks itself."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "host_api_check.cpp")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(tmp_path):
    exe = str(tmp_path / "host_api_check")
    cmd = ["g++", "-std=c++17", "-O1", SRC, "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           "-L", os.path.join(ROOT, "indexingpu_b200"), "-lmt_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{os.path.join(ROOT, 'indexingpu_b200')}", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}",
           "-o", exe]
    subprocess.check_call(cmd)
    return exe


def test_cpp_host_mirror_builds(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_cpp_host_mirror_runs(tmp_path):
    out = subprocess.run([_build(tmp_path)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "0 mismatches" in out.stdout
