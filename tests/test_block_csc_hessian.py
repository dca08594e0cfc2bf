"""Layout identities of the block-CSC container (mirror of tests/test_block_csc_hessian.cc:52-214)."""
import numpy as np
import pytest

from meshfemsparse_b200 import BlockCSCHessian, SystemAssembler

from helpers import random_stencil_hessian


@pytest.mark.parametrize("bs", [1, 2, 3])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_layout_identities(bs, seed):
    H = random_stencil_hessian(seed, bs=bs, spd=False)
    rng = np.random.default_rng(seed + 10)
    # scalarOffsetForColumn / locForBlock follow the contiguous-block rule
    for bj in range(H.numBlocks):
        assert H.scalarOffsetForColumn(bj) == bs * bs * H.Ap[bj]
        for k in range(H.Ap[bj], H.Ap[bj + 1]):
            assert H.locForBlock(int(H.Ai[k]), bj) == bs * bs * k
    S = H.toScalar()
    # every scalar upper entry maps to its block slot
    offs = H.dataOffsetsForScalarCSCDataOffsets()
    assert offs.size == S.nz
    assert np.array_equal(S.Ax, H.Ax[offs])
    for idx, (i, j) in enumerate(S.entries()):
        assert H.locForScalar(i, j) == offs[idx]
    # trace
    dense = S.to_dense()
    assert abs(H.trace() - np.trace(dense)) <= 1e-10 * max(1.0, abs(np.trace(dense)))
    # addNZScalar + toScalar exact
    G = H.copy()
    G.setZero()
    for (i, j), v in zip(S.entries(), S.Ax):
        G.addNZScalar(i, j, v)
    assert np.array_equal(G.toScalar().Ax, S.Ax)
    # apply and quadratic form
    x = rng.normal(size=H.n)
    assert np.linalg.norm(H.apply(x) - dense @ x) <= 1e-8 * np.linalg.norm(dense @ x)
    assert abs(H.evalQuadraticForm(x) - x @ dense @ x) <= 1e-8 * max(1.0, abs(x @ dense @ x))
    # addDiag
    G = H.copy()
    G.addDiag(2.5)
    assert np.allclose(np.diag(G.toScalar().to_dense()), np.diag(dense) + 2.5, rtol=0, atol=1e-12)
    # setIdentity keeps the pattern
    G = H.copy().setIdentity()
    assert np.array_equal(G.toScalar().to_dense(), np.eye(H.n))
    # fromScalar round trip exact
    R = BlockCSCHessian.fromScalar(S, bs)
    assert np.array_equal(R.Ap, H.Ap) and np.array_equal(R.Ai, H.Ai)
    assert np.array_equal(R.toScalar().Ax, S.Ax)


def test_binary_round_trip(tmp_path):
    H = random_stencil_hessian(5, bs=3, spd=True)
    p = tmp_path / "h.bin"
    H.dumpBinary(str(p))
    R = BlockCSCHessian.readBinary(str(p))
    assert R.bs == 3 and np.array_equal(R.Ap, H.Ap) and np.array_equal(R.Ai, H.Ai)
    assert np.array_equal(R.toScalar().Ax, H.toScalar().Ax)


def test_pattern_for_star():
    H = SystemAssembler(12, 2).blockSparsityPattern([[0, e + 1] for e in range(11)])
    assert list(H.Ap[:4]) == [0, 1, 3, 5]
    assert list(H.Ai[1:3]) == [0, 1]
