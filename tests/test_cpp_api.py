"""The C++ front-end (tamm_b200/include/tamm_b200/tamm.hpp): compiles against the C ABI
on the CPU, and its TAMM-style test program (tests/cpp/test_api.cpp) passes on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_api.cpp")
LIBDIR = os.path.join(ROOT, "tamm_b200")


def _build(tmp_path):
    exe = os.path.join(str(tmp_path), "test_api")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", SRC, f"-I{ROOT}/include", f"-I{ROOT}/tamm_b200/include",
           f"-L{LIBDIR}", "-ltamm_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_front_end_compiles(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_cpp_front_end_runs(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASSED" in r.stdout
