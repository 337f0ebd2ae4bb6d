"""Build libb200sssp.so in-tree with nvcc for sm_100a.

Usage: python rips2026-amd_b200/build.py [--force] [--jobs N]

Every .cu / .cpp under csrc/ is compiled to an object under _build/ and
linked into rips2026-amd_b200/libb200sssp.so (static CUDA runtime, so the
library does not depend on which libcudart the host process loaded first).
Objects are rebuilt when the source or any header under csrc/ or include/ is
newer.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libb200sssp.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "--extended-lambda", "-I", INCLUDE, "-I", CSRC]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def cuda_home() -> str:
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc())))


def _headers_mtime() -> float:
    t = 0.0
    for d in (CSRC, INCLUDE):
        for dp, _, files in os.walk(d):
            for f in files:
                if f.endswith((".h", ".hpp", ".cuh")):
                    t = max(t, os.path.getmtime(os.path.join(dp, f)))
    return t


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def compile_one(src: str, force: bool, hdr_t: float) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_t)):
        return obj
    if src.endswith(".cu"):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj]
    else:
        cmd = ["g++", *CXX_FLAGS, "-I", os.path.join(cuda_home(), "include"), "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr_t = _headers_mtime()
    srcs = sources()
    with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force, hdr_t), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB + ".tmp", *objs,
               "-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
        if verbose:
            print(f"linked {LIB}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    try:
        print(build(force=a.force, jobs=a.jobs, verbose=True))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
