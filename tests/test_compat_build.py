"""CPU: the reference's C++ call surface (include/b200sssp/compat.hpp) and the
C header compile and link into the standalone C++ test program against the
built library; running it needs a GPU (tests/test_gpu_compat_cpp.py)."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(os.path.join(CUDA, "include")),
                    reason="needs g++ and the CUDA headers")
def test_cpp_compat_program_builds(b2, tmp_path):
    libdir = os.path.join(ROOT, "rips2026-amd_b200")
    exe = str(tmp_path / "compat_test")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", os.path.join(ROOT, "tests", "cpp", "compat_test.cpp"),
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           "-L", libdir, "-lb200sssp", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{libdir}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert os.path.getsize(exe) > 0


def test_c_header_compiles_as_c(tmp_path):
    """include/b200sssp.h is plain C (C11, no CUDA headers needed)."""
    src = tmp_path / "h.c"
    src.write_text('#include "b200sssp.h"\nint main(void) { return B2_ABI_VERSION == 1 ? 0 : 1; }\n')
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                        "-o", str(tmp_path / "h")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
