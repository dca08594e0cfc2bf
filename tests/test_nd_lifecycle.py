"""The nested-dissection metadata lifecycle of the reference's test_nd_ordering.cc:20-70
(checkNDLifecycle) on analysis-only handles: a 24 x 24 triangle grid with 2 x 2 blocks,
the separator forest published after the symbolic analysis at the block size it ran at,
whole-block pins shrinking it, a partial pin falling back to the scalar analysis, no
forest for a non-ND ordering, and none after clearFactors. Host only."""
import numpy as np

from meshfemsparse_b200 import B200Factorizer, OrderingMethod, SystemAssembler


def grid_triangles(side=24):
    e = []
    for y in range(side - 1):
        for x in range(side - 1):
            a = y * side + x
            e.append((a, a + 1, a + side))
            e.append((a + 1, a + side + 1, a + side))
    return np.array(e, dtype=np.int64)


def test_nd_metadata_lifecycle():
    side = 24
    A = SystemAssembler(side * side, bs=2).blockSparsityPattern(grid_triangles(side))
    A.setZero()
    for i in range(A.n):
        A.addNZScalar(i, i, 2.0)
    f = B200Factorizer(device=-1)
    assert f.ndOrdering() is None
    f.factorizeSymbolic(A, [])
    snap = f.ndOrdering()
    assert snap is not None and snap.blockSize == 2
    assert snap.CMember.size == side * side and snap.CParent.size > 1
    # every component's parent follows it; every vertex belongs to one component
    assert np.all((snap.CParent == -1) | (snap.CParent > np.arange(snap.CParent.size)))
    assert snap.CMember.min() >= 0 and snap.CMember.max() < snap.CParent.size
    # the published indices describe the reduced ordering graph
    f.factorizeSymbolic(A, [0, 1])
    nd = f.ndOrdering()
    assert nd.CMember.size == side * side - 1 and nd.blockSize == 2
    assert f.hasFixedVars()
    # a partial pin falls back to the scalar analysis
    f.factorizeSymbolic(A, [0])
    nd = f.ndOrdering()
    assert nd.CMember.size == 2 * side * side - 1 and nd.blockSize == 1
    # a non-ND ordering publishes no forest
    g = B200Factorizer(device=-1, orderingMethod=OrderingMethod.AMD)
    g.factorizeSymbolic(A, [])
    assert g.ndOrdering() is None
    f.factorizeSymbolic(A, [])
    f.clearFactors()
    assert f.ndOrdering() is None
