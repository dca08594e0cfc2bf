"""Contact-like pattern sequences: the sparsity cache driving the symbolic analysis in
recorded-sequence replay (the reference's benchmark_sparsity_lru.cc loop), block
pattern enlargement, and the nested-dissection reuse when an edge joins two
previously separate bodies. CPU parts use an analysis-only handle or a recording
stand-in factorizer; the GPU test replays the same sequence through the GPU path."""
import numpy as np
import pytest

from meshfemsparse_b200 import B200Factorizer, SystemAssembler, fem
from meshfemsparse_b200.hessian import BlockCSCHessian
from meshfemsparse_b200.recorder import MatrixRecorder, replay
from oracle import pyoracle


def union_pattern(H: BlockCSCHessian, pairs) -> BlockCSCHessian:
    """H's block pattern plus the upper blocks of the node pairs."""
    cols = np.repeat(np.arange(H.numBlocks, dtype=np.int64), np.diff(H.Ap))
    rows = H.Ai
    if len(pairs):
        p = np.sort(np.asarray(pairs, dtype=np.int64), axis=1)
        rows = np.concatenate([rows, p[:, 0]])
        cols = np.concatenate([cols, p[:, 1]])
    key = np.unique(cols * H.numBlocks + rows)
    c, r = key // H.numBlocks, key % H.numBlocks
    Ap = np.zeros(H.numBlocks + 1, dtype=np.int64)
    np.add.at(Ap, c + 1, 1)
    return BlockCSCHessian(H.numBlocks, np.cumsum(Ap), r, H.bs)


def add_springs(H: BlockCSCHessian, pairs, k: float) -> None:
    """Penalty springs k (x_u - x_v)^2 / 2 per component between node pairs."""
    I = k * np.eye(3)
    for u, v in pairs:
        u, v = int(min(u, v)), int(max(u, v))
        for a, b, m in ((u, u, I), (v, v, I), (u, v, -I)):
            loc = H.locForBlock(a, b)
            H.Ax[loc:loc + 9] += m.reshape(-1, order="F")


def contact_sequence(k=4, seed=3):
    """A jittered cube with contact springs between top-face node pairs that come
    and go: the static pattern, then pair sets C1, C1, (none), C1, C2."""
    nodes, tets = fem.tet_cube(k, jitter=0.1, seed=seed)
    nn = nodes.shape[0]
    Hs = SystemAssembler(nn).blockSparsityPattern(tets)
    Ke = fem.linear_elastic_hessians(nodes, tets, 1.0, 0.3)
    Hs.Ax = pyoracle.assemble(Hs.numBlocks, Hs.Ap, Hs.Ai, tets, Ke)
    top = np.nonzero(np.isclose(nodes[:, 2], nodes[:, 2].max(), atol=0.2))[0]
    bottom = np.nonzero(np.isclose(nodes[:, 2], nodes[:, 2].min(), atol=0.2))[0]
    c1 = [(int(top[i]), int(bottom[i])) for i in range(0, 6, 2)]
    c2 = [(int(top[i]), int(bottom[-1 - i])) for i in range(1, 5, 2)]
    steps = [[], c1, c1, [], c1, c2]
    pins = fem.bottom_pins(nodes)
    return Hs, steps, pins


def record(tmp_path, Hs, steps, pins):
    rec = MatrixRecorder()
    rec.recordMatrices(str(tmp_path))
    mats = []
    for pairs in steps:
        H = union_pattern(Hs, pairs)
        rec.countSparsityUpdateCall()
        rec.recordSymbolic(H, pins)
        H.setZero().addWithSubSparsity(Hs)
        add_springs(H, pairs, 0.5)
        rec.recordNumeric(H)
        mats.append(H)
    return mats


class PatternRecorder:
    """Stand-in factorizer: keeps the analysed pattern and checks that every numeric
    matrix comes in exactly that pattern."""

    def __init__(self):
        self.symbolic = 0
        self.pattern = None
        self.numeric = []

    def factorizeSymbolic(self, H, pins):
        self.symbolic += 1
        self.pattern = (H.Ap.copy(), H.Ai.copy())

    def factorizeNumeric(self, H):
        assert np.array_equal(H.Ap, self.pattern[0]) and np.array_equal(H.Ai, self.pattern[1])
        self.numeric.append(H.copy())


def test_add_with_sub_sparsity_matches_dense():
    Hs, steps, pins = contact_sequence()
    H = union_pattern(Hs, steps[1])
    H.setZero().addWithSubSparsity(Hs, 2.0)
    assert np.allclose(H.to_scipy_full().toarray(), 2.0 * Hs.to_scipy_full().toarray())
    H.addWithSubSparsity(Hs, -1.0)
    assert np.allclose(H.to_scipy_full().toarray(), Hs.to_scipy_full().toarray())
    with pytest.raises(ValueError):
        Hs.copy().addWithSubSparsity(H)      # H has blocks outside Hs's pattern
    # a sparsity-only operand adds nothing
    assert np.allclose(H.copy().addWithSubSparsity(BlockCSCHessian(H.numBlocks, H.Ap, H.Ai)).to_scipy_full().toarray(),
                       H.to_scipy_full().toarray())


def test_replay_with_sparsity_cache_skips_covered_patterns(tmp_path):
    Hs, steps, pins = contact_sequence()
    mats = record(tmp_path, Hs, steps, pins)
    f = PatternRecorder()
    out = replay(tmp_path, f, solve=False, sparsity_cache=0.5)
    sym = [o for o in out if o["kind"] == "symbolic"]
    # static; C1 new; C1 again; none (C1 ages, kept); C1 again; C2 new
    assert [o["symbolic_factorization"] for o in sym] == [True, True, False, False, False, True]
    assert f.symbolic == 3
    # every numeric matrix keeps its values when enlarged into the cached pattern
    assert len(f.numeric) == len(mats)
    for got, want in zip(f.numeric, mats):
        assert np.allclose(got.to_scipy_full().toarray(), want.to_scipy_full().toarray())
    # without the cache every pattern is analysed
    f2 = PatternRecorder()
    replay(tmp_path, f2, solve=False)
    assert f2.symbolic == len(steps)


def test_nd_reuse_edge_joining_two_bodies_redissects_everything():
    """Two separate cubes (a forest of two separator trees), then one contact edge
    between them: no lowest common ancestor exists, so the whole graph is dissected
    afresh (persistent_separator_tree.hh:97-99) and the ordering stays a permutation."""
    nodes, tets = fem.tet_cube(5, seed=4)
    nn = nodes.shape[0]
    both = np.vstack([tets, tets + nn])
    edges = np.vstack([both[:, [a, b]] for a in range(4) for b in range(a + 1, 4)])
    H = SystemAssembler(2 * nn).blockSparsityPattern(edges)
    f = B200Factorizer(device=-1, nd_reuse_period=8)
    f.factorizeSymbolic(H, [])
    H2 = SystemAssembler(2 * nn).blockSparsityPattern(np.vstack([edges, [[0, nn + 1]]]))
    f.factorizeSymbolic(H2, [])
    st = f.stats()
    assert st["nd_rebuilt_vertices"] == 2 * nn
    perm = f.getInversePermutation()
    assert np.array_equal(np.sort(perm), np.arange(perm.size))
    fresh = B200Factorizer(device=-1)
    fresh.factorizeSymbolic(H2, [])
    assert f.getFactorNNZ() == fresh.getFactorNNZ()


@pytest.mark.gpu
def test_contact_sequence_replay_with_sparsity_cache_on_gpu(tmp_path):
    Hs, steps, pins = contact_sequence()
    record(tmp_path, Hs, steps, pins)
    out = replay(tmp_path, B200Factorizer(), sparsity_cache=0.5)
    num = [o for o in out if o["kind"] == "numeric"]
    assert len(num) == len(steps)
    assert max(o["residual"] for o in num) <= 1e-10
