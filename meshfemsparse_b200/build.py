"""Build the in-tree shared library ``libmfs_b200.so`` (sm_100a CUDA + C++ host code).

Usage: ``python -m meshfemsparse_b200.build`` (or ``build_library()`` from Python).
Objects go to ``meshfemsparse_b200/_build/``; the library is written next to this
file so it travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libmfs_b200.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I", str(INCLUDE), "-I", str(CSRC)]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-march=x86-64-v2", "-I", str(INCLUDE), "-I", str(CSRC)]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(CSRC.glob("*.cu")), sorted(CSRC.glob("*.cpp"))


def _stale(obj: Path, deps) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compile every source under csrc/ for sm_100a and link the shared library."""
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    cu, cpp = _sources()
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    jobs, objs = [], []
    for src in cu:
        obj = BUILD / (src.stem + ".cu.o")
        objs.append(obj)
        if force or _stale(obj, [src, *headers]):
            jobs.append([nvcc, *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)])
    for src in cpp:
        obj = BUILD / (src.stem + ".cpp.o")
        objs.append(obj)
        if force or _stale(obj, [src, *headers]):
            jobs.append(["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for out in ex.map(_compile, jobs):
                if verbose and out.strip():
                    print(out)
    if force or jobs or not LIB.exists() or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        _compile([nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"])
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    print(LIB)
