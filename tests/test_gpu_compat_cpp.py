"""The reference's C++ call surface (include/b200sssp/compat.hpp) compiled into
a standalone C++ program (tests/cpp/compat_test.cpp) and run on the GPU."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_cpp_compat_program(b2, cuda, tmp_path):
    libdir = os.path.join(ROOT, "rips2026-amd_b200")
    exe = str(tmp_path / "compat_test")
    cmd = ["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "compat_test.cpp"),
           "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           "-L", libdir, "-lb200sssp", "-L", "/usr/local/cuda/lib64", "-lcudart",
           f"-Wl,-rpath,{libdir}", "-Wl,-rpath,/usr/local/cuda/lib64", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASSED" in r.stdout
