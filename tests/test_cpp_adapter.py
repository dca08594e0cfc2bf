"""The header-only C++ host interface (include/mfs_b200_factorizer.hpp) compiles
with g++, links the C-ABI library and agrees with the Python binding on an
analysis-only handle (no GPU)."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from meshfemsparse_b200 import B200Factorizer, _lib

from helpers import path_hessian

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_cpp_adapter_matches_python(tmp_path):
    exe = tmp_path / "adapter_check"
    lib_dir = _lib.LIB_PATH.parent
    cmd = ["g++", "-std=c++17", "-O1", "-I", str(ROOT / "include"), str(ROOT / "tests/cpp/adapter_check.cpp"),
           "-L", str(lib_dir), "-lmfs_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()
    head = out[0].split()
    n, nr, nnz, flops = int(head[1]), int(head[3]), int(head[5]), float(head[7])
    H = path_hessian(20)
    f = B200Factorizer(device=-1)
    f.factorizeSymbolic(H, [0, 1, 2])
    assert (n, nr) == (60, 57)
    assert nnz == f.getFactorNNZ() and flops == pytest.approx(f.getFlopEstimate())
    assert int(head[9]) == 1
    iperm = np.array([int(v) for v in out[1].split()[1:]])
    assert np.array_equal(iperm, f.getInversePermutation())
    # solve without a factor -> runtime_error; numeric on an analysis-only handle and a
    # non-upper pattern -> invalid_argument
    assert out[2] == "caught 7"
    # pins (one partial block: scalar analysis), row maps and the forest against the Python binding
    f.factorizeSymbolic(H, [0, 1, 2, 7])
    assert out[3] == "fixed 1 4 posdef 0"
    x = np.arange(60) + 0.5
    for permute in (0, 1):
        xr = np.array([float(v) for v in out[4 + 2 * permute].split()[1:]])
        assert np.array_equal(xr, f.removeFixedEntries(x, permute=bool(permute)))
        full = np.array([float(v) for v in out[5 + 2 * permute].split()[1:]])
        assert np.array_equal(full, f.extractFullSolution(xr, permute=bool(permute)))
    nd = f.ndOrdering()
    assert out[8].split() == ["nd", "1", str(nd.CParent.size), str(nd.CMember.size), str(nd.blockSize)]
