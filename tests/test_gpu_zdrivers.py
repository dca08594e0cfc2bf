"""Drivers and host interfaces on the GPU: recorded-sequence replay, the C++ host
interface, and the solve_system CLI. Collected after the kernel-level GPU tests."""
import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from meshfemsparse_b200 import _lib
from meshfemsparse_b200.recorder import MatrixRecorder, replay
from meshfemsparse_b200.solve_system import write_triplet_binary

ROOT = Path(__file__).resolve().parents[1]


def spd_triplets(n, seed):
    rng = np.random.default_rng(seed)
    M = rng.normal(size=(n, n)) * 0.2
    K = M @ M.T + n * np.eye(n)
    K[np.abs(K) < 0.5] = 0.0
    K = 0.5 * (K + K.T) + np.eye(n)
    I, J = np.nonzero(K)
    return K, I, J, K[I, J]


@pytest.mark.gpu
def test_replay_recorded_newton_steps_on_gpu(tmp_path):
    """A recorded sequence (one pattern, three value sets) replayed through the GPU factorizer."""
    from meshfemsparse_b200 import B200Factorizer, SystemAssembler, fem
    from oracle import pyoracle
    nodes, tets = fem.tet_cube(3, jitter=0.1, seed=2)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    pins = fem.bottom_pins(nodes)
    rec = MatrixRecorder()
    rec.recordMatrices(str(tmp_path))
    rec.countSparsityUpdateCall()
    rec.recordSymbolic(H, pins)
    for scale in (1.0, 2.0, 0.5):
        Ke = fem.linear_elastic_hessians(nodes, tets, scale, 0.3)
        H.Ax = pyoracle.assemble(H.numBlocks, H.Ap, H.Ai, tets, Ke)
        rec.recordNumeric(H)
    out = replay(tmp_path, B200Factorizer())
    assert [o["kind"] for o in out] == ["symbolic", "numeric", "numeric", "numeric"]
    assert max(o["residual"] for o in out[1:]) <= 1e-10


@pytest.mark.gpu
@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_cpp_adapter_factor_and_solve_on_gpu(tmp_path):
    exe = tmp_path / "adapter_solve"
    lib_dir = _lib.LIB_PATH.parent
    cmd = ["g++", "-std=c++17", "-O1", "-I", str(ROOT / "include"), str(ROOT / "tests/cpp/adapter_solve.cpp"),
           "-L", str(lib_dir), "-lmfs_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=300).stdout.splitlines()
    res = {ln.split()[0]: float(ln.split()[2]) for ln in out}
    assert res["fp64"] <= 1e-12 and res["fp32+refine"] <= 1e-10


@pytest.mark.gpu
def test_cli_on_gpu(tmp_path):
    K, I, J, V = spd_triplets(40, 2)
    write_triplet_binary(tmp_path / "m.bin", I, J, V)
    b = np.linspace(-1, 1, 40)
    np.savetxt(tmp_path / "rhs.txt", b)
    out = subprocess.run([sys.executable, "-m", "meshfemsparse_b200.solve_system", str(tmp_path / "m.bin"),
                          str(tmp_path / "rhs.txt")], capture_output=True, text=True, cwd=ROOT, check=True)
    u = np.array([float(v) for v in out.stdout.split()])
    assert np.linalg.norm(K @ u - b) <= 1e-12 * np.linalg.norm(b)


@pytest.mark.gpu
@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("rank", [0, 2])
def test_bordered_solve_through_gpu_factorizer(single, rank):
    """BorderedSparseHessian (BorderedSparseHessian.hh:56-75): the sparse block factored
    and solved on the GPU (one multi-RHS solve for the border columns), against the
    dense solve of the whole system; FP32 + refinement as well as FP64."""
    from meshfemsparse_b200 import B200Factorizer
    from meshfemsparse_b200.bordered import BorderedSparseFactorization, BorderedSparseHessian
    from helpers import random_stencil_hessian
    rng = np.random.default_rng(7 + rank)
    Hs = random_stencil_hessian(5)
    ns, nd = Hs.n, 3
    H = BorderedSparseHessian(Hs, rng.normal(size=(ns, nd)) * 0.3, np.diag(rng.uniform(1, 2, nd)) * 50.0)
    if rank:
        H.addLowRank(rng.normal(size=(ns + nd, rank)), 0.5)
    M = np.zeros((ns + nd, ns + nd))
    M[:ns, :ns] = H.H_ss.to_scipy_full().toarray()
    M[:ns, ns:] = H.H_sd
    M[ns:, :ns] = H.H_sd.T
    M[ns:, ns:] = H.H_dd
    V = np.vstack([H.V_s, H.V_d])
    M = M + V @ V.T
    pins = np.array([0, 1, 2])
    F = BorderedSparseFactorization(H, B200Factorizer(single, refine=single), pins)
    x = rng.normal(size=ns + nd)
    b = M @ x
    keep = np.ones(ns + nd, dtype=bool)
    keep[pins] = False
    xr = np.zeros_like(x)
    xr[keep] = np.linalg.solve(M[np.ix_(keep, keep)], b[keep])
    got = F.solve(b)
    assert np.linalg.norm(got - xr) <= 1e-9 * np.linalg.norm(xr)
    assert np.all(got[pins] == 0.0)


@pytest.mark.gpu
def test_bordered_equality_constraints_through_gpu_factorizer():
    """Equality constraints through Lagrange multipliers over the GPU factorization,
    against the dense KKT solve."""
    from meshfemsparse_b200 import B200Factorizer
    from meshfemsparse_b200.bordered import BorderedSparseFactorization, BorderedSparseHessian
    from helpers import random_stencil_hessian
    rng = np.random.default_rng(11)
    Hs = random_stencil_hessian(8)
    ns, nd, m = Hs.n, 2, 3
    H = BorderedSparseHessian(Hs, rng.normal(size=(ns, nd)) * 0.3, np.diag(rng.uniform(1, 2, nd)) * 50.0)
    H.addLowRank(rng.normal(size=(ns + nd, 1)), 0.5)
    C = rng.normal(size=(m, ns + nd))
    H.setConstraints(C)
    F = BorderedSparseFactorization(H, B200Factorizer(), [])
    b = rng.normal(size=ns + nd)
    r = rng.normal(size=m)
    x, lam = F.solve(b, r, return_multipliers=True)
    M = np.zeros((ns + nd, ns + nd))
    M[:ns, :ns] = H.H_ss.to_scipy_full().toarray()
    M[:ns, ns:] = H.H_sd
    M[ns:, :ns] = H.H_sd.T
    M[ns:, ns:] = H.H_dd
    V = np.vstack([H.V_s, H.V_d])
    M = M + V @ V.T
    K = np.block([[M, C.T], [C, np.zeros((m, m))]])
    ref = np.linalg.solve(K, np.concatenate([b, r]))
    assert np.linalg.norm(x - ref[:ns + nd]) <= 1e-9 * np.linalg.norm(ref[:ns + nd])
    assert np.linalg.norm(lam - ref[ns + nd:]) <= 1e-8 * np.linalg.norm(ref[ns + nd:])
