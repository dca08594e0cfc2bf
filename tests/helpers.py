"""Shared test-matrix generators mirroring the reference's unit tests."""
from __future__ import annotations

import numpy as np

from meshfemsparse_b200 import BlockCSCHessian, ScalarCSC, SystemAssembler, fem


def path_hessian(nb: int = 20, bs: int = 3) -> BlockCSCHessian:
    """Path matrix of tests/test_catamari_factorizer.cc:100-110: blocks (i, i+1),
    diagonal 10.1, off-diagonal -0.1 (1 + (i + j) % 5)."""
    H = SystemAssembler(nb, bs).blockSparsityPattern([[i, i + 1] for i in range(nb - 1)])
    H.setZero()
    S = H.toScalar(sparsityOnly=True)
    for i, j in S.entries():
        H.addNZScalar(i, j, 10.1 if i == j else -0.1 * (1 + (i + j) % 5))
    return H


def plain_scalar_path(n: int = 20) -> ScalarCSC:
    """tests/test_catamari_factorizer.cc:151-162: 4.1 diagonal, -0.7 super-diagonal."""
    Ap = [0]
    Ai, Ax = [], []
    for j in range(n):
        if j > 0:
            Ai.append(j - 1); Ax.append(-0.7)
        Ai.append(j); Ax.append(4.1)
        Ap.append(len(Ai))
    return ScalarCSC(n, np.array(Ap, dtype=np.int64), np.array(Ai, dtype=np.int64), np.array(Ax))


def grid_forest(side: int = 13, bs: int = 3) -> BlockCSCHessian:
    """Two disconnected side x side grids (tests/test_catamari_factorizer.cc:345-362)."""
    comp = side * side
    n = 2 * comp
    edges = []
    for i in range(n):
        if i % side + 1 < side:
            edges.append([i, i + 1])
        if i % comp + side < comp:
            edges.append([i, i + side])
    H = SystemAssembler(n, bs).blockSparsityPattern(edges)
    H.setZero()
    for i, j in H.toScalar(sparsityOnly=True).entries():
        H.addNZScalar(i, j, 10.0 if i == j else -0.1)
    return H


def random_stencil_hessian(seed: int, bs: int = 3, spd: bool = True) -> BlockCSCHessian:
    """Random 4-variable stencils as in tests/test_block_csc_hessian.cc:10-50, with
    diagonally dominant values so the matrix is SPD."""
    rng = np.random.default_rng(seed)
    nb = 4 + 3 * int(rng.integers(0, 20))
    elems = []
    for e in range(nb):
        others = rng.choice(np.setdiff1d(np.arange(nb), [e]), size=3, replace=False)
        elems.append([e, *others])
    H = SystemAssembler(nb, bs).blockSparsityPattern(elems)
    H.setZero()
    H.Ax[:] = rng.uniform(-1, 1, size=H.Ax.size)
    if spd:
        # symmetric diagonal dominance on the scalar matrix
        S = H.toScalar()
        rowsum = np.zeros(S.n)
        cols = np.repeat(np.arange(S.n), np.diff(S.Ap))
        off = S.Ai != cols
        np.add.at(rowsum, S.Ai[off], np.abs(S.Ax[off]))
        np.add.at(rowsum, cols[off], np.abs(S.Ax[off]))
        for i in range(S.n):
            loc = H.locForScalar(i, i)
            H.Ax[loc] = rowsum[i] + 1.0 + rng.uniform(0, 1)
    return H


def cube_problem(k: int, jitter: float = 0.1, seed: int = 1, E=1.0, nu=0.3):
    """Linear-elastic tet cube: (H with values, conn, Ke, pins, nodes)."""
    nodes, tets = fem.tet_cube(k, jitter=jitter, seed=seed)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    Ke = fem.linear_elastic_hessians(nodes, tets, E=E, nu=nu)
    from oracle import pyoracle
    H.Ax = pyoracle.assemble(H.numBlocks, H.Ap, H.Ai, tets, Ke)
    pins = fem.bottom_pins(nodes)
    return H, tets, Ke, pins, nodes
