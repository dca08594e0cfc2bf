"""Pins the CPU oracle itself: golden fixtures and independent numpy/LAPACK checks."""
from pathlib import Path

import numpy as np
import pytest

from meshfemsparse_b200 import B200Factorizer, OrderingMethod, fem
from oracle import pyoracle

from helpers import cube_problem, path_hessian, random_stencil_hessian

GOLD = Path(__file__).parent / "golden"


def test_assembly_matches_golden_fixture():
    z = np.load(GOLD / "assembly_k2.npz")
    Ax = pyoracle.assemble(z["nodes"].shape[0], z["Ap"], z["Ai"], z["tets"], z["Ke"])
    assert np.array_equal(Ax, z["Ax"])


def test_assembly_matches_dense_restatement():
    nodes, tets = fem.tet_cube(3, jitter=0.1, seed=5)
    Ke = fem.linear_elastic_hessians(nodes, tets, 1.0, 0.3)
    Ap, Ai = pyoracle.build_pattern(nodes.shape[0], tets)
    Ax = pyoracle.assemble(nodes.shape[0], Ap, Ai, tets, Ke)
    from meshfemsparse_b200 import BlockCSCHessian
    H = BlockCSCHessian(nodes.shape[0], Ap, Ai, 3, Ax)
    n = 3 * nodes.shape[0]
    D = np.zeros((n, n))
    for e in range(tets.shape[0]):
        dofs = (3 * tets[e][:, None] + np.arange(3)).reshape(-1)
        D[np.ix_(dofs, dofs)] += Ke[e]
    assert np.max(np.abs(H.to_scipy_full().toarray() - D)) <= 1e-13 * np.max(np.abs(D))
    # the linear-elastic generator is symmetric with rigid translations in its kernel
    assert np.allclose(Ke, Ke.transpose(0, 2, 1))
    t = np.tile(np.eye(3), (4, 1))
    assert np.max(np.abs(Ke @ t)) < 1e-12 * np.max(np.abs(Ke))


def oracle_factor(H, pins, ordering=OrderingMethod.CholmodNesdisParallel, threads=0):
    f = B200Factorizer(device=-1, orderingMethod=ordering)
    f.factorizeSymbolic(H, pins)
    sn = f.supernodes()
    plan = f.conversionPlan()
    w, d, fr, pan, col0 = pyoracle.panel_layout(sn)
    vals = pyoracle.inject(plan["entries"], sn["vb"], H.bs, H.Ax, int(pan[-1]))
    fail = pyoracle.mf_factor(sn, vals, threads)
    return f, sn, vals, fail


@pytest.mark.parametrize("bs", [1, 2, 3])
def test_oracle_factor_matches_lapack(bs):
    H = path_hessian(20, bs)
    pins = [1]
    f, sn, vals, fail = oracle_factor(H, pins)
    assert fail == -1
    ip = f.getInversePermutation()
    A = pyoracle.reduced_permuted_dense(H, pins, ip)
    L = pyoracle.panels_to_dense(sn, vals, f.n_reduced())
    Lref = np.linalg.cholesky(A)
    assert np.max(np.abs(L - Lref)) <= 1e-12 * np.max(np.abs(Lref))


@pytest.mark.parametrize("seed", range(4))
def test_oracle_solve_matches_numpy(seed):
    H = random_stencil_hessian(seed, bs=3)
    f, sn, vals, fail = oracle_factor(H, [0, 1, 2])
    assert fail == -1
    ip = f.getInversePermutation()
    A = pyoracle.reduced_permuted_dense(H, [0, 1, 2], ip)
    rng = np.random.default_rng(seed)
    B = rng.normal(size=(A.shape[0], 3))
    X = pyoracle.mf_solve(sn, vals, B)
    Xref = np.linalg.solve(A, B)
    assert np.linalg.norm(X - Xref) <= 1e-11 * np.linalg.norm(Xref)


def test_oracle_blas_path_matches_loops():
    H, tets, Ke, pins, nodes = cube_problem(4)
    f, sn, v0, fail0 = oracle_factor(H, pins, threads=0)
    if not pyoracle.load_blas():
        pytest.skip("OpenBLAS from scipy not found")
    _, _, v1, fail1 = oracle_factor(H, pins, threads=2)
    assert fail0 == fail1 == -1
    assert np.max(np.abs(v0 - v1)) <= 1e-12 * np.max(np.abs(v0))


def test_oracle_reports_non_positive_pivot():
    H = path_hessian(8, 2)
    H.Ax *= -1.0
    f, sn, vals, fail = oracle_factor(H, [])
    assert fail >= 0


def test_multiply_lower_block_known_answer():
    """Forward substitution update of tests/test_catamari_solve_kernels.cc:33-51, restated
    on the oracle's layout: rhs[2] -= 2 * rhs[1] in every padded column."""
    import json
    g = json.loads((GOLD / "known_answers.json").read_text())["multiply_lower_block"]
    rhs = np.array(g["rhs"], dtype=float)
    ld, nrhs = g["ld"], g["num_rhs"]
    for r in range(nrhs):
        col = rhs[r * ld:(r + 1) * ld]
        for idx, lv in zip(g["indices"], g["lower_block"]):
            col[idx] -= lv * col[g["supernode_start"]]
    assert list(rhs) == g["expected"]
