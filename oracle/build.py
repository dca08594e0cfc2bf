"""Build recipe for the CPU oracle (test infrastructure, never the product).

Compiles ``oracle/mfs_oracle.c`` with gcc into ``oracle/_build/libmfs_oracle.so``.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "mfs_oracle.c"
OUT = HERE / "_build" / "libmfs_oracle.so"


def build_oracle(force: bool = False) -> Path:
    OUT.parent.mkdir(exist_ok=True)
    if not force and OUT.exists() and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    cmd = ["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", str(SRC), "-o", str(OUT), "-ldl", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return OUT


if __name__ == "__main__":
    print(build_oracle(force=True))
